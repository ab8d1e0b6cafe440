// Kernel instantiations and launch tables for one lattice. Included by
// kernels_q{9,19,27}.cu with WK_Q defined, so the three lattices compile in
// parallel translation units.
#pragma once

#include "kernels.cuh"

#ifndef WK_Q
#error "define WK_Q before including kernels_impl.cuh"
#endif

#define WK_CAT2(a, b) a##b
#define WK_CAT(a, b) WK_CAT2(a, b)

namespace wk {

// Per-node flag byte from the cell types (see FL_* in lattice.cuh).
template <int Q>
__global__ void k_flags(const uint8_t* __restrict__ types, uint8_t* __restrict__ flags, const Geo geo,
                        const FlagCfg cfg, int xchunks) {
    using L = Lat<Q>;
    const int row = blockIdx.x / xchunks;
    const int x = (blockIdx.x - row * xchunks) * blockDim.x + threadIdx.x;
    if (x >= geo.nx) return;
    const int nx = geo.nx, ny = geo.ny, nz = geo.nz;
    const int y = row % ny, z = row / ny;
    const long long i = static_cast<long long>(row) * nx + x;
    const uint8_t t = types[i] & FL_TYPE;
    uint8_t fl = t;
    if (t != CT_SOLID) {
        bool zh = false;
        if (cfg.zh_rule == 1) {
            const bool interior_row = (y >= 1) && (y <= ny - 2);
            if (cfg.inflow && x == 0 && interior_row) { fl |= FL_ZH_IN; zh = true; }
            if (cfg.outflow && x == nx - 1 && interior_row) { fl |= FL_ZH_OUT; zh = true; }
        } else if (cfg.zh_rule == 2) {
            if (cfg.inflow && x == 0 && t == CT_INFLOW) { fl |= FL_ZH_IN; zh = true; }
            if (cfg.outflow && x == nx - 1 && t == CT_OUTFLOW) { fl |= FL_ZH_OUT; zh = true; }
        }
        bool fast = true;  // Zou-He nodes gather purely too; the formula is applied after the gather
        (void)zh;
        bool mem = false;
#pragma unroll
        for (int q = 1; q < Q; ++q) {
            // pull source x - c_q
            const int sx = L::cx(q) ? wrap<Q>(x - L::cx(q), nx) : x;
            int sy = y - L::cy(q), sz = z - L::cz(q);
            if (L::cy(q) && geo.periodic_y) sy = wrap<Q>(sy, ny);
            if (L::cz(q) && geo.periodic_z) sz = wrap<Q>(sz, nz);
            if (sy < 0 || sy >= ny || sz < 0 || sz >= nz) {
                fast = false;
            } else {
                const uint8_t ts = types[(static_cast<long long>(sz) * ny + sy) * nx + sx] & FL_TYPE;
                if (ts == CT_SOLID || ts == CT_MOVING_WALL) fast = false;
            }
            // momentum-exchange link to x + c_q (forces_momentum_exchange.ispc:38-52)
            if (cfg.mem_enabled && t == CT_FLUID) {
                const int xn = L::cx(q) ? wrap<Q>(x + L::cx(q), nx) : x;
                const int yn = y + L::cy(q), zn = z + L::cz(q);
                if (yn >= 0 && yn < ny && zn >= 0 && zn < nz) {
                    const uint8_t tn = types[(static_cast<long long>(zn) * ny + yn) * nx + xn] & FL_TYPE;
                    if (tn == CT_SOLID || tn == CT_MOVING_WALL) {
                        const float rx = __fsub_rn(__fadd_rn(float(x), 0.5f * float(L::cx(q))), cfg.center[0]);
                        const float ry = __fsub_rn(__fadd_rn(float(y), 0.5f * float(L::cy(q))), cfg.center[1]);
                        const float rz = __fsub_rn(__fadd_rn(float(z), 0.5f * float(L::cz(q))), cfg.center[2]);
                        float r2 = __fadd_rn(__fmul_rn(rx, rx), __fmul_rn(ry, ry));
                        if (L::D == 3) r2 = __fadd_rn(r2, __fmul_rn(rz, rz));
                        if (cfg.r_max <= 0.0f || r2 <= cfg.r_max_sq) mem = true;
                    }
                }
            }
        }
        if (fast) fl |= FL_FAST;
        if (mem) fl |= FL_MEM;
    }
    flags[i] = fl;
}

// Segment classes for the two step kernels (one warp per segment of SEG nodes):
// bit 0 = every node is a pure gather (k_step_fast), bit 1 = the segment holds
// a momentum-exchange node, bit 2 = every node is solid (no launch needed).
template <int Q>
__global__ void k_seg_class(const uint8_t* __restrict__ flags, uint8_t* __restrict__ cls, const Geo geo,
                            long long nsegs) {
    const long long e = blockIdx.x * static_cast<long long>(blockDim.x >> 5) + (threadIdx.x >> 5);
    if (e >= nsegs) return;
    const Seg sg = seg_decode(static_cast<unsigned>(e), geo);
    const int lane = threadIdx.x & 31;
    int fast = 1, mem = 0, solid = 1;
    for (int x = sg.x0 + lane; x < sg.x1; x += 32) {
        const uint8_t fl = flags[sg.row0 + x];
        fast &= (fl & FL_FAST) ? 1 : 0;
        mem |= (fl & FL_MEM) ? 1 : 0;
        solid &= (fl & FL_TYPE) == CT_SOLID ? 1 : 0;
    }
    fast = __all_sync(0xffffffffu, fast);
    mem = __any_sync(0xffffffffu, mem);
    solid = __all_sync(0xffffffffu, solid);
    if (lane == 0) cls[e] = static_cast<uint8_t>((fast ? 1 : 0) | (mem ? 2 : 0) | (solid ? 4 : 0));
}

// Pull-free read of f^0 (state buffer holding pre-collision populations).
template <int Q, int S>
__global__ void __launch_bounds__(512) k_direct(const void* fin_v, const uint8_t* flags, Geo geo, Physics phys,
                                                Out out, int xchunks, Thermal th) {
    using L = Lat<Q>;
    using C = Codec<S>;
    const typename C::T* fin = static_cast<const typename C::T*>(fin_v);
    const int row = blockIdx.x / xchunks;
    const int x = (blockIdx.x - row * xchunks) * blockDim.x + threadIdx.x;
    if (x >= geo.nx) return;
    const long long i = static_cast<long long>(row) * geo.nx + x;
    float f[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) f[q] = C::load_plain(fin + q * geo.pitch + i, L::w(q));
    if (out.f) {
#pragma unroll
        for (int q = 0; q < Q; ++q) out.f[q * geo.pitch + i] = f[q];
    }
    if (out.rho) {
        float g[3] = {phys.g[0], phys.g[1], phys.g[2]};
        if (th.on) {  // local buoyancy of the state's temperature (sum of the current temperature buffer)
            float t5[5];
#pragma unroll
            for (int q = 0; q < 5; ++q) t5[q] = th.tin[q * geo.pitch + i];
            g[1] = buoyant_gy(th, phys.g[1], sum_t5(t5));
        }
        float rho, u[3];
        node_moments<Q>(f, g, rho, u);
        out.rho[i] = rho;
        out.ux[i] = u[0];
        out.uy[i] = u[1];
        if (out.uz) out.uz[i] = u[2];
        out.speed[i] = sqrtf(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    }
    (void)flags;
}

namespace {
constexpr int kQ = WK_Q;

template <int C, int S, bool LES>
void step_one(const StepArgs& a, const Launch& L, bool fast) {
    if (fast) {
        if (a.nspans <= 0) return;
        // one block per span; 32-bit element indexing whenever every index of the state buffer fits
        const bool idx32 = static_cast<long long>(kQ) * a.geo.pitch < (1ll << 32);
        if (idx32) k_step_fast<kQ, C, S, LES, true><<<a.nspans, L.tpb_fast, 0, L.stream>>>(a);
        else k_step_fast<kQ, C, S, LES, false><<<a.nspans, L.tpb_fast, 0, L.stream>>>(a);
    } else {
        if (a.nrows <= 0) return;
        k_step<kQ, C, S, LES><<<a.nrows, SEG, 0, L.stream>>>(a);
    }
}
template <int C, int S, bool LES>
void initial_one(const float* f0, void* A, void* B, const uint8_t* flags, const Geo& g, const Physics& p,
                 const Launch& L) {
    k_initial<kQ, C, S, LES><<<L.rows * L.xchunks, L.tpb, 0, L.stream>>>(f0, A, B, flags, g, p, L.xchunks);
}
template <int C, int S, bool LES>
void batch_one(const BatchArgs& b, int tpb, cudaStream_t st, bool fast, bool idx32) {
    if (fast) {
        if (b.nspans <= 0) return;
        if (idx32) k_step_fast_batch<kQ, C, S, LES, true><<<b.nspans, tpb, 0, st>>>(b);
        else k_step_fast_batch<kQ, C, S, LES, false><<<b.nspans, tpb, 0, st>>>(b);
    } else {
        if (b.nrows <= 0) return;
        k_step_batch<kQ, C, S, LES><<<b.nrows, SEG, 0, st>>>(b);
    }
}
// Persistent tile kernel: TILE_CTAS_PER_SM CTAs per SM (capped by the work), dynamic shared
// memory opted in once per kernel instantiation.
template <auto Kernel>
cudaError_t tiles_launch(unsigned smem, int work, cudaStream_t st, const StepArgs& a, const TileArgs& t) {
    static bool ready = false;
    if (!ready) {
        const cudaError_t e =
            cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        ready = true;
    }
    int sms = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = std::max(1, std::min(work, TILE_CTAS_PER_SM * sms));
    Kernel<<<blocks, TILE_THREADS, smem, st>>>(a, t);
    return cudaGetLastError();
}

template <int C, int S, bool LES>
cudaError_t tiles_one(const StepArgs& a, const TileArgs& t, cudaStream_t st) {
    constexpr unsigned smem = tile_smem_bytes<kQ, S>();
    const int work = std::max(std::max(t.ntiles, t.ngen), t.nspans);
    if (work <= 0) return cudaSuccess;
    if (t.dom) return tiles_launch<k_step_tiles<kQ, C, S, LES, true>>(smem, work, st, a, t);
    return tiles_launch<k_step_tiles<kQ, C, S, LES, false>>(smem, work, st, a, t);
}
using TilesFn = cudaError_t (*)(const StepArgs&, const TileArgs&, cudaStream_t);
using StepFn = void (*)(const StepArgs&, const Launch&, bool);
using BatchFn = void (*)(const BatchArgs&, int, cudaStream_t, bool, bool);
using InitFn = void (*)(const float*, void*, void*, const uint8_t*, const Geo&, const Physics&, const Launch&);

#define WK_ROW(C, S) {step_one<C, S, false>, step_one<C, S, true>}
#define WK_IROW(C, S) {initial_one<C, S, false>, initial_one<C, S, true>}
const StepFn kStep[3][4][2] = {{WK_ROW(0, 0), WK_ROW(0, 1), WK_ROW(0, 2), WK_ROW(0, 3)},
                               {WK_ROW(1, 0), WK_ROW(1, 1), WK_ROW(1, 2), WK_ROW(1, 3)},
                               {WK_ROW(2, 0), WK_ROW(2, 1), WK_ROW(2, 2), WK_ROW(2, 3)}};
const InitFn kInit[3][4][2] = {{WK_IROW(0, 0), WK_IROW(0, 1), WK_IROW(0, 2), WK_IROW(0, 3)},
                               {WK_IROW(1, 0), WK_IROW(1, 1), WK_IROW(1, 2), WK_IROW(1, 3)},
                               {WK_IROW(2, 0), WK_IROW(2, 1), WK_IROW(2, 2), WK_IROW(2, 3)}};
#define WK_BROW(C, S) {batch_one<C, S, false>, batch_one<C, S, true>}
const BatchFn kBatch[3][4][2] = {{WK_BROW(0, 0), WK_BROW(0, 1), WK_BROW(0, 2), WK_BROW(0, 3)},
                                 {WK_BROW(1, 0), WK_BROW(1, 1), WK_BROW(1, 2), WK_BROW(1, 3)},
                                 {WK_BROW(2, 0), WK_BROW(2, 1), WK_BROW(2, 2), WK_BROW(2, 3)}};
#define WK_SROW(C, S) {tiles_one<C, S, false>, tiles_one<C, S, true>}
const TilesFn kTiles[3][4][2] = {{WK_SROW(0, 0), WK_SROW(0, 1), WK_SROW(0, 2), WK_SROW(0, 3)},
                                 {WK_SROW(1, 0), WK_SROW(1, 1), WK_SROW(1, 2), WK_SROW(1, 3)},
                                 {WK_SROW(2, 0), WK_SROW(2, 1), WK_SROW(2, 2), WK_SROW(2, 3)}};
#undef WK_ROW
#undef WK_IROW
#undef WK_BROW
#undef WK_SROW

bool valid(int coll, int store) { return coll >= 0 && coll < 3 && store >= 0 && store < 4; }
}  // namespace

cudaError_t WK_CAT(launch_step_q, WK_Q)(int coll, int store, bool les, const StepArgs& a, const Launch& L,
                                       bool fast) {
    if (!valid(coll, store)) return cudaErrorInvalidValue;
    kStep[coll][store][les ? 1 : 0](a, L, fast);
    return cudaGetLastError();
}

cudaError_t WK_CAT(launch_batch_q, WK_Q)(int coll, int store, bool les, const BatchArgs& b, int tpb,
                                        cudaStream_t stream, bool fast, bool idx32) {
    if (!valid(coll, store)) return cudaErrorInvalidValue;
    kBatch[coll][store][les ? 1 : 0](b, tpb, stream, fast, idx32);
    return cudaGetLastError();
}

cudaError_t WK_CAT(launch_tiles_q, WK_Q)(int coll, int store, bool les, const StepArgs& a, const TileArgs& t,
                                        cudaStream_t stream) {
    if (!valid(coll, store)) return cudaErrorInvalidValue;
    return kTiles[coll][store][les ? 1 : 0](a, t, stream);
}

cudaError_t WK_CAT(launch_initial_q, WK_Q)(int coll, int store, bool les, const float* f0, void* a, void* b,
                                          const uint8_t* flags, const Geo& geo, const Physics& phys,
                                          const Launch& L) {
    if (!valid(coll, store)) return cudaErrorInvalidValue;
    kInit[coll][store][les ? 1 : 0](f0, a, b, flags, geo, phys, L);
    return cudaGetLastError();
}

cudaError_t WK_CAT(launch_materialise_q, WK_Q)(int store, const void* fin, const uint8_t* flags, const Geo& geo,
                                              const Links& links, const Physics& phys, const Out& out,
                                              const Launch& L, int direct, const Thermal& th) {
    const int blocks = L.rows * L.xchunks;
#define WK_MAT(S)                                                                               \
    if (direct) k_direct<kQ, S><<<blocks, L.tpb, 0, L.stream>>>(fin, flags, geo, phys, out, L.xchunks, th); \
    else k_materialise<kQ, S><<<blocks, L.tpb, 0, L.stream>>>(fin, flags, geo, links, phys, out, L.xchunks, th)
    switch (store) {
        case 0: WK_MAT(0); break;
        case 1: WK_MAT(1); break;
        case 2: WK_MAT(2); break;
        case 3: WK_MAT(3); break;
        default: return cudaErrorInvalidValue;
    }
#undef WK_MAT
    return cudaGetLastError();
}

#if WK_Q == 9
cudaError_t launch_initial_thermal_q9(int coll, int store, bool les, const float* f0, const float* t0, void* a, void* b,
                                      float* ta, float* tb, const uint8_t* flags, const Geo& geo, const Physics& phys,
                                      const Thermal& th, const Launch& L) {
    if (!valid(coll, store)) return cudaErrorInvalidValue;
    const int blocks = L.rows * L.xchunks;
#define WK_TI(C, S, LES) \
    k_initial_thermal<C, S, LES><<<blocks, L.tpb, 0, L.stream>>>(f0, t0, a, b, ta, tb, flags, geo, phys, th, L.xchunks)
    switch (coll * 8 + store * 2 + (les ? 1 : 0)) {
        case 0: WK_TI(0, 0, false); break;
        case 1: WK_TI(0, 0, true); break;
        case 2: WK_TI(0, 1, false); break;
        case 3: WK_TI(0, 1, true); break;
        case 4: WK_TI(0, 2, false); break;
        case 5: WK_TI(0, 2, true); break;
        case 6: WK_TI(0, 3, false); break;
        case 7: WK_TI(0, 3, true); break;
        case 8: WK_TI(1, 0, false); break;
        case 9: WK_TI(1, 0, true); break;
        case 10: WK_TI(1, 1, false); break;
        case 11: WK_TI(1, 1, true); break;
        case 12: WK_TI(1, 2, false); break;
        case 13: WK_TI(1, 2, true); break;
        case 14: WK_TI(1, 3, false); break;
        case 15: WK_TI(1, 3, true); break;
        case 16: WK_TI(2, 0, false); break;
        case 17: WK_TI(2, 0, true); break;
        case 18: WK_TI(2, 1, false); break;
        case 19: WK_TI(2, 1, true); break;
        case 20: WK_TI(2, 2, false); break;
        case 21: WK_TI(2, 2, true); break;
        case 22: WK_TI(2, 3, false); break;
        case 23: WK_TI(2, 3, true); break;
        default: return cudaErrorInvalidValue;
    }
#undef WK_TI
    return cudaGetLastError();
}
#endif

cudaError_t WK_CAT(launch_flags_q, WK_Q)(const uint8_t* types, uint8_t* flags, const Geo& geo, const FlagCfg& cfg,
                                        const Launch& L) {
    k_flags<kQ><<<L.rows * L.xchunks, L.tpb, 0, L.stream>>>(types, flags, geo, cfg, L.xchunks);
    return cudaGetLastError();
}

// Whole-row TRT kernel (rows.cuh): one block per row of the lattice.
cudaError_t WK_CAT(launch_rows_q, WK_Q)(int store, bool les, const StepArgs& a, int rows, int tpb,
                                       cudaStream_t stream) {
    if (rows <= 0) return cudaSuccess;
    switch (store * 2 + (les ? 1 : 0)) {
        case 0: k_step_rows<kQ, 0, false><<<rows, tpb, 0, stream>>>(a); break;
        case 1: k_step_rows<kQ, 0, true><<<rows, tpb, 0, stream>>>(a); break;
        case 2: k_step_rows<kQ, 1, false><<<rows, tpb, 0, stream>>>(a); break;
        case 3: k_step_rows<kQ, 1, true><<<rows, tpb, 0, stream>>>(a); break;
        case 4: k_step_rows<kQ, 2, false><<<rows, tpb, 0, stream>>>(a); break;
        case 5: k_step_rows<kQ, 2, true><<<rows, tpb, 0, stream>>>(a); break;
        case 6: k_step_rows<kQ, 3, false><<<rows, tpb, 0, stream>>>(a); break;
        case 7: k_step_rows<kQ, 3, true><<<rows, tpb, 0, stream>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

namespace {  // internal linkage: every lattice's translation unit has its own pipe_one (kQ differs)
// Pipelined whole-row TRT kernel (rowpipe.cuh): as many CTAs as fit on the device (capped by
// the rows), dynamic shared memory opted in once per instantiation.
template <int S, bool LES, int CAP>
cudaError_t pipe_one(const StepArgs& a, const PipeArgs& p, cudaStream_t stream) {
    constexpr unsigned smem = pipe_smem_bytes<kQ, S, CAP>();
    static int slots = 0;  // resident CTAs on the device
    if (slots == 0) {
        cudaError_t e = cudaFuncSetAttribute(k_step_rows_pipe<kQ, S, LES, CAP>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        // the stages are the kernel's working set: all of the SM's unified memory as shared memory
        e = cudaFuncSetAttribute(k_step_rows_pipe<kQ, S, LES, CAP>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
        if (e != cudaSuccess) return e;
        int per_sm = 0, sms = 0, dev = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_rows_pipe<kQ, S, LES, CAP>,
                                                          pipe_threads<CAP>(), smem);
        if (e != cudaSuccess) return e;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        slots = std::max(1, per_sm * sms);
    }
    const int blocks = std::min(p.nrows, slots);
    if (blocks <= 0) return cudaSuccess;
    k_step_rows_pipe<kQ, S, LES, CAP><<<blocks, pipe_threads<CAP>(), smem, stream>>>(a, p);
    return cudaGetLastError();
}
}  // namespace

cudaError_t WK_CAT(launch_rows_pipe_q, WK_Q)(int store, bool les, int cap, const StepArgs& a, const PipeArgs& p,
                                            cudaStream_t stream) {
    const int sel = (cap > 256 ? 8 : 0) + store * 2 + (les ? 1 : 0);
    switch (sel) {
        case 0: return pipe_one<0, false, 256>(a, p, stream);
        case 1: return pipe_one<0, true, 256>(a, p, stream);
        case 2: return pipe_one<1, false, 256>(a, p, stream);
        case 3: return pipe_one<1, true, 256>(a, p, stream);
        case 4: return pipe_one<2, false, 256>(a, p, stream);
        case 5: return pipe_one<2, true, 256>(a, p, stream);
        case 6: return pipe_one<3, false, 256>(a, p, stream);
        case 7: return pipe_one<3, true, 256>(a, p, stream);
        case 8: return pipe_one<0, false, 512>(a, p, stream);
        case 9: return pipe_one<0, true, 512>(a, p, stream);
        case 10: return pipe_one<1, false, 512>(a, p, stream);
        case 11: return pipe_one<1, true, 512>(a, p, stream);
        case 12: return pipe_one<2, false, 512>(a, p, stream);
        case 13: return pipe_one<2, true, 512>(a, p, stream);
        case 14: return pipe_one<3, false, 512>(a, p, stream);
        case 15: return pipe_one<3, true, 512>(a, p, stream);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t WK_CAT(launch_seg_class_q, WK_Q)(const uint8_t* flags, uint8_t* cls, const Geo& geo, long long nsegs,
                                            cudaStream_t stream) {
    if (nsegs <= 0) return cudaSuccess;
    const long long blocks = (nsegs + 7) / 8;
    k_seg_class<kQ><<<static_cast<unsigned>(blocks), 256, 0, stream>>>(flags, cls, geo, nsegs);
    return cudaGetLastError();
}

}  // namespace wk
