// Host state of one resident lattice (wake_grid) shared by the single-lattice
// engine (engine.cu) and the batch of many lattices (batch.cu).
#pragma once

#include <algorithm>
#include <string>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "wake_gpu.h"

namespace wk {

// ---------------------------------------------------------------- host lattice tables
struct HostLat {
    int Q = 0, D = 0;
    int cx[27], cy[27], cz[27], opp[27];
    float w[27];
    explicit HostLat(int q) : Q(q) {
        auto fill = [&](auto lat) {
            using L = decltype(lat);
            D = L::D;
            for (int k = 0; k < Q; ++k) {
                cx[k] = L::cx(k);
                cy[k] = L::cy(k);
                cz[k] = L::cz(k);
                opp[k] = L::opp(k);
                w[k] = L::w(k);
            }
        };
        if (q == 9) fill(Lat<9>{});
        else if (q == 19) fill(Lat<19>{});
        else fill(Lat<27>{});
    }
};

// Bounding box (inclusive) and shape of a device rasteriser call (k_rasterise in engine.cu).
struct RasterBox {
    int x0, x1, y0, y1, z0, z1;
};
struct RasterShape {
    int kind;     // 0 circle, 1 sphere, 2 rotated ellipse
    float c[3];   // centre
    float p[4];   // circle / sphere: r^2; ellipse: cos, sin, 1/a^2, 1/b^2
};

cudaError_t launch_step_any(int Q, int coll, int store, bool les, const StepArgs& a, const Launch& L, bool fast);
cudaError_t launch_batch_any(int Q, int coll, int store, bool les, const BatchArgs& b, int tpb, cudaStream_t stream,
                             bool fast, bool idx32);
cudaError_t launch_tiles_any(int Q, int coll, int store, bool les, const StepArgs& a, const TileArgs& t,
                             cudaStream_t stream);
cudaError_t launch_rows_any(int Q, int store, bool les, const StepArgs& a, int rows, int tpb, cudaStream_t stream);
cudaError_t launch_rows_pipe_any(int Q, int store, bool les, int cap, const StepArgs& a, const PipeArgs& p,
                                 cudaStream_t stream);

}  // namespace wk

using wk::DevMem;
using wk::HostLat;
using wk::Physics;
using wk::Geo;
using wk::Links;
using wk::Launch;
using wk::StepArgs;

struct wake_grid {
    int Q = 0, D = 0, nx = 0, ny = 0, nz = 0, storage = 0;
    long long N = 0, pitch = 0;
    std::size_t elem = 4;
    HostLat lat{9};

    DevMem A, B;       // state buffers
    int cur = 0;       // 0: A holds the current state, 1: B
    // State machine. m_f (FP32) holds the reference-visible f^k whenever mf_valid.
    // `pending`: A/B do not hold Collide(f^k) for the current collision parameters
    // (fresh initial state, or tau / model / body force changed since the last
    // collide); the next step re-collides f^k from m_f first, exactly like the
    // reference, whose step k+1 starts by colliding f^k with that step's parameters.
    bool pending = true;
    bool mf_valid = false;
    float collided_g[3] = {0.f, 0.f, 0.f};  // body force the state buffers were collided with
    float last_step_g[3] = {0.f, 0.f, 0.f};  // body force of the last executed step
    DevMem d_types, d_flags, d_status, d_nodestart;
    // Cell types live in two copies: `types` on the host (single-cell edits, face setters,
    // reads) and d_types on the device (flag builds, link candidates, the shape rasterisers).
    // The flags say which copy holds edits the other lacks; copies move only when needed.
    std::vector<uint8_t> types;
    bool types_host_newer = true;
    bool types_dev_newer = false;
    bool geom_dirty = true;

    int collision = WAKE_MRT, les = 0;
    Physics phys{};
    int inflow = 0, outflow = 0, lid = 0, periodic_y = 0, periodic_z = 0;
    float uin[3] = {0.f, 0.f, 0.f}, rho_out = 1.0f, uw[3] = {0.f, 0.f, 0.f};

    std::vector<int> link_node, link_q;
    std::vector<float> link_delta, link_uw;  // uw: 3 per link
    DevMem d_link_node, d_link_q, d_link_delta, d_link_mom;
    int dev_links = 0;         // links currently on the device (the flags refer to these)
    bool links_dirty = false;  // host links differ from the device copy

    int mem_on = 0, hist_cap = 0;
    float center[3] = {0.f, 0.f, 0.f}, rmax = 0.f;
    DevMem d_counters, d_hist;         // counters: [0] unused, [1] history entries written
    DevMem d_warp_base, d_contrib;     // momentum-exchange slots (see MemCfg)
    int warps_per_row = 1, n_mem_nodes = 0;

    // pure-gather spans (0, row, x0, x1) handled by k_step_fast, and general segments
    // (SEG nodes of a row, numbered row * nseg + s) handled by k_step
    DevMem d_fast_rows, d_gen_rows;
    int n_fast = 0, n_gen = 0;
    std::vector<uint4> h_fast_rows;     // spans
    std::vector<unsigned> h_gen_rows;   // general segments
    long long fast_nodes() const {      // nodes in the pure-gather spans
        long long n = 0;
        for (const uint4& sp : h_fast_rows) n += sp.w - sp.z;
        return n;
    }
    // Identity of the current flags / row lists: a fresh process-wide number at every
    // rebuild (next_geom_version), so a batch never takes a new grid that happens to
    // reuse a destroyed grid's address for the old one.
    unsigned long long geom_version = 0;

    int tpb = 0, xchunks = 1, rows = 1, tpb_fast = 64;
    // step kernels: 0 automatic, 1 direct (k_step_fast for the pure-gather rows beside
    // k_step for the rest), 2 persistent tiles (k_step_tiles: pure-gather tiles staged in
    // shared memory plus the general rows, when the row shape allows it)
    int kernel_variant = 0;
    bool use_tiles() const { return kernel_variant == 2 && wk::tile_row_ok(nx, static_cast<int>(elem)); }
    // Whole-row TRT kernel (k_step_rows, variant 3): one block per row over the rows whose
    // every node is a pure gather (d_row_kind, ROW_* bytes); the pure-gather runs of the other
    // rows (d_mixed) go to k_step_fast beside the general segments. Not automatic: on the D3Q19
    // sphere channel the span kernel moves FP32 rows 3 % faster per node.
    DevMem d_row_kind;
    int n_row_fast = 0;           // rows marked ROW_FAST
    long long row_fast_nodes = 0;  // nodes in them
    bool use_rows() const {
        return kernel_variant == 3 && collision == WAKE_TRT && nx % 2 == 0 &&
               static_cast<long long>(Q) * pitch < (1ll << 32) && !th.on && n_row_fast > 0;
    }
    int tpb_rows() const { return nx <= 64 ? 32 : 64; }
    // Pipelined whole-row kernel (k_step_rows_pipe, variant 4, and the automatic choice for
    // 16-bit storage): the ROW_FAST rows as (row | descriptor << 28), staged through shared
    // memory by bulk copies. FP32 takes the span kernel automatically (measured faster there:
    // three CTAs per SM fill the shared memory).
    DevMem d_row_list;
    int pipe_cap() const { return nx <= 256 ? 256 : 512; }
    bool use_pipe() const {
        const bool chosen = kernel_variant == 4 || (kernel_variant == 0 && storage != 0);
        return chosen && collision == WAKE_TRT && nx % 2 == 0 && nx <= 512 &&
               (static_cast<long long>(nx) * static_cast<long long>(elem)) % 16 == 0 &&
               static_cast<long long>(Q) * pitch < (1ll << 32) && !th.on && n_row_fast > 0 && rows < (1 << 28);
    }
    // pure-gather tiles (0, (z << 16) | y0, rows, 0) and the segments of the other rows
    // (0, segment, general-segment entry, 0)
    DevMem d_tiles, d_gen4, d_mixed;
    int n_tiles = 0, n_tile_gen = 0, n_mixed = 0;
    std::vector<uint4> h_tiles, h_gen4, h_mixed;  // h_mixed: the spans of rows outside the tiles
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t side = nullptr;  // forked stream of the general-row launch
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    long long k = 0;

    DevMem m_f, m_rho, m_ux, m_uy, m_uz, m_speed, m_diag;
    DevMem m_an;  // field analytics: vorticity (2D) or omega x/y/z + Q (3D), and the |max| word

    // coupled D2Q5 temperature (D2Q9 lattices): post-collision populations in TA / TB
    // (same parity as A / B), FP32 start-up populations in m_t
    wk::Thermal th{};
    DevMem TA, TB, m_t;
    bool mt_valid = false;
    float* tbuf(int which) const { return static_cast<float*>(which == 0 ? TA.p : TB.p); }

    // CUDA graph of `graph_steps` fused steps starting from buffer parity graph_cur
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0, graph_cur = -1;
    float graph_g[3] = {0.f, 0.f, 0.f};
    bool graph_ok = false;

    // Optional CUDA-event timing of every pure-gather (bulk) launch; plain launches only.
    bool time_bulk = false;
    std::vector<cudaEvent_t> t_ev;  // pairs (start, end), reused
    std::size_t t_used = 0;         // events recorded since the last read

    explicit wake_grid(int q) : lat(q) {}
    ~wake_grid() {
        // every queued use of the blocks ends here, so they go back to the cache
        // (no device-wide cudaFree while other lattices run)
        bool idle = true;
        if (stream) idle = cudaStreamSynchronize(stream) == cudaSuccess;
        if (side) idle = idle && cudaStreamSynchronize(side) == cudaSuccess;
        if (idle) {
            DevMem* all[] = {&A, &B, &d_types, &d_flags, &d_status, &d_nodestart, &d_link_node, &d_link_q,
                             &d_link_delta, &d_link_mom, &d_counters, &d_hist, &d_warp_base, &d_contrib,
                             &d_fast_rows, &d_gen_rows, &d_tiles, &d_gen4, &d_mixed, &d_row_kind, &d_row_list, &m_f, &m_rho, &m_ux, &m_uy, &m_uz,
                             &m_speed, &m_diag, &TA, &TB, &m_t, &m_an};
            for (DevMem* m : all) m->release();
        }
        for (cudaEvent_t e : t_ev) cudaEventDestroy(e);
        if (graph) cudaGraphExecDestroy(graph);
        if (own_stream && stream) cudaStreamDestroy(stream);
        if (side) cudaStreamDestroy(side);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
    }

    void* buf(int which) { return which == 0 ? A.p : B.p; }

    Geo geo() const {
        Geo g{};
        g.nx = nx;
        g.ny = ny;
        g.nz = nz;
        g.periodic_y = (D == 3) ? periodic_y : 0;
        g.periodic_z = (D == 3) ? periodic_z : 0;
        g.pitch = pitch;
        for (int a = 0; a < 3; ++a) g.uin[a] = uin[a];
        g.rho_out = rho_out;
        for (int q = 0; q < Q; ++q) {
            // 2 w_q rho_0 / cs^2 (c_q . u_w) in the reference's float order (d2q9_streaming.ispc:49-53)
            const float ci_uw = float(lat.cx[q]) * uw[0] + float(lat.cy[q]) * uw[1] + float(lat.cz[q]) * uw[2];
            g.mom[q] = lid ? 2.0f * lat.w[q] * 1.0f * 3.0f * ci_uw : 0.0f;
        }
        return g;
    }
    Links links() const {
        Links l{};
        l.node_start = d_nodestart.as<int>();
        l.node = d_link_node.as<int>();
        l.q = d_link_q.as<int>();
        l.delta = d_link_delta.as<float>();
        l.mom = d_link_mom.as<float>();
        l.count = dev_links;
        return l;
    }
    Launch launch() const { return Launch{tpb, xchunks, rows, stream, ny, nz, tpb_fast}; }
    int blocks() const { return rows * xchunks; }

    void invalidate_graph() { graph_ok = false; }

    void choose_block(int want) {
        const int full = ((nx + 31) / 32) * 32;
        if (want > 0) tpb = want;
        else if (full <= 512) tpb = full;
        else {
            int best = 256;
            long long best_waste = -1;
            for (int t : {256, 384, 512}) {
                const long long chunks = (nx + t - 1) / t;
                const long long waste = chunks * t - nx;
                if (best_waste < 0 || waste < best_waste) {
                    best = t;
                    best_waste = waste;
                }
            }
            tpb = best;
        }
        xchunks = (nx + tpb - 1) / tpb;
        rows = ny * nz;
        // k_step_fast is limited to WK_FAST_MAX_THREADS threads. Least idle lanes over the row,
        // ties to the smaller block: 64-thread blocks measured fastest on 256-node rows (more
        // independent blocks in flight per SM, shorter tail per row).
        const int cap = std::min(want > 0 ? want : WK_FAST_MAX_THREADS, WK_FAST_MAX_THREADS);
        int best = -1, best_waste = 1 << 30;
        for (int t = 64; t <= cap; t += 32) {
            const int waste = ((nx + t - 1) / t) * t - nx;
            if (waste < best_waste) {
                best = t;
                best_waste = waste;
            }
        }
        tpb_fast = best > 0 ? best : 64;
    }
};

namespace wk {

// Validity check that records the error (WAKE_ERR_INVALID) for a null handle.
bool grid_valid(wake_grid* g);
// Bring a lattice to the point where its state buffers hold Collide(f^k) for the
// current geometry and parameters (rebuilds flags, re-collides when pending).
int grid_prepare(wake_grid* g);
unsigned long long next_geom_version();
// Step arguments of one lattice (rows and buffers left for the caller).
StepArgs grid_step_args(const wake_grid* g);
// Bookkeeping after n steps run outside wake_grid_step (by a batch).
void grid_advanced(wake_grid* g, int n);
// Error status word of the lattice: WAKE_OK or WAKE_ERR_NUMERIC (synchronizes its stream).
int grid_check_status(wake_grid* g);

}  // namespace wk
