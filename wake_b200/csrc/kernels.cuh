// Launch interface between the host engine and the per-lattice kernel
// translation units (kernels_q9.cu, kernels_q19.cu, kernels_q27.cu).
#pragma once

#include <cuda_runtime.h>

#include "rowpipe.cuh"
#include "rows.cuh"
#include "staged.cuh"
#include "stream_collide.cuh"

namespace wk {

struct Launch {
    int tpb;       // threads per block (one thread per node along x)
    int xchunks;   // blocks per row
    int rows;      // ny * nz
    cudaStream_t stream;
    int ny, nz;
    int tpb_fast;  // threads per block of k_step_fast (<= 256; one warp per segment)
};

struct FlagCfg {
    int zh_rule;         // 0 none, 1: 2D reference rule (columns x=0 / x=nx-1, rows 1..ny-2), 2: typed faces
    int inflow, outflow;
    int mem_enabled;
    float center[3];
    float r_max, r_max_sq;
};

// Per-lattice entry points (defined once per Q in kernels_impl.cuh).
#define WK_DECLARE_LAUNCHERS(Q)                                                                                   \
    cudaError_t launch_step_q##Q(int coll, int store, bool les, const StepArgs& a, const Launch& L, bool fast);  \
    cudaError_t launch_batch_q##Q(int coll, int store, bool les, const BatchArgs& b, int tpb,                   \
                                  cudaStream_t stream, bool fast, bool idx32);                                  \
    cudaError_t launch_tiles_q##Q(int coll, int store, bool les, const StepArgs& a, const TileArgs& t,          \
                                  cudaStream_t stream);                                                          \
    cudaError_t launch_materialise_q##Q(int store, const void* fin, const uint8_t* flags, const Geo& geo,        \
                                        const Links& links, const Physics& phys, const Out& out,                 \
                                        const Launch& L, int direct, const Thermal& th);                         \
    cudaError_t launch_initial_q##Q(int coll, int store, bool les, const float* f0, void* a, void* b,            \
                                    const uint8_t* flags, const Geo& geo, const Physics& phys, const Launch& L); \
    cudaError_t launch_flags_q##Q(const uint8_t* types, uint8_t* flags, const Geo& geo, const FlagCfg& cfg,      \
                                  const Launch& L);                                                              \
    cudaError_t launch_seg_class_q##Q(const uint8_t* flags, uint8_t* cls, const Geo& geo, long long nsegs,       \
                                      cudaStream_t stream);                                                      \
    cudaError_t launch_rows_q##Q(int store, bool les, const StepArgs& a, int rows, int tpb, cudaStream_t stream); \
    cudaError_t launch_rows_pipe_q##Q(int store, bool les, int cap, const StepArgs& a, const PipeArgs& p,         \
                                      cudaStream_t stream);

WK_DECLARE_LAUNCHERS(9)
// Initial collide of a D2Q9 flow with its coupled D2Q5 temperature (kernels_q9.cu).
cudaError_t launch_initial_thermal_q9(int coll, int store, bool les, const float* f0, const float* t0, void* a, void* b,
                                      float* ta, float* tb, const uint8_t* flags, const Geo& geo, const Physics& phys,
                                      const Thermal& th, const Launch& L);
WK_DECLARE_LAUNCHERS(19)
WK_DECLARE_LAUNCHERS(27)

// Marks FL_BFL on link nodes (clearing FL_FAST) and records each node's first link.
cudaError_t launch_link_marks(const int* link_node, int n_links, uint8_t* flags, int* node_start,
                              cudaStream_t stream);

}  // namespace wk
