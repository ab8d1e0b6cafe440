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

// Row classes for the two step kernels: bit 0 = every node of the row is a pure
// gather (k_step_fast), bit 1 = the row holds a momentum-exchange node.
template <int Q>
__global__ void k_row_class(const uint8_t* __restrict__ flags, uint8_t* __restrict__ cls, const Geo geo) {
    const long long row0 = static_cast<long long>(blockIdx.x) * geo.nx;
    int all_fast = 1, any_mem = 0;
    for (int x = threadIdx.x; x < geo.nx; x += blockDim.x) {
        const uint8_t fl = flags[row0 + x];
        all_fast &= (fl & FL_FAST) ? 1 : 0;
        any_mem |= (fl & FL_MEM) ? 1 : 0;
    }
    all_fast = __syncthreads_and(all_fast);
    any_mem = __syncthreads_or(any_mem);
    if (threadIdx.x == 0) cls[blockIdx.x] = static_cast<uint8_t>((all_fast ? 1 : 0) | (any_mem ? 2 : 0));
}

// Pull-free read of f^0 (state buffer holding pre-collision populations).
template <int Q, int S>
__global__ void __launch_bounds__(512) k_direct(const void* fin_v, const uint8_t* flags, Geo geo, Physics phys,
                                                Out out, int xchunks) {
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
        float rho, u[3];
        node_moments<Q>(f, phys.g, rho, u);
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
    if (a.nrows <= 0) return;
    if (fast) {
        // 32-bit element indexing whenever every index of the state buffer fits
        const bool idx32 = static_cast<long long>(kQ) * a.geo.pitch < (1ll << 32);
        if (idx32) k_step_fast<kQ, C, S, LES, true><<<a.nrows, L.tpb_fast, 0, L.stream>>>(a);
        else k_step_fast<kQ, C, S, LES, false><<<a.nrows, L.tpb_fast, 0, L.stream>>>(a);
    } else {
        k_step<kQ, C, S, LES><<<a.nrows, L.tpb, 0, L.stream>>>(a);
    }
}
template <int C, int S, bool LES>
void initial_one(const float* f0, void* A, void* B, const uint8_t* flags, const Geo& g, const Physics& p,
                 const Launch& L) {
    k_initial<kQ, C, S, LES><<<L.rows * L.xchunks, L.tpb, 0, L.stream>>>(f0, A, B, flags, g, p, L.xchunks);
}
template <int C, int S, bool LES>
void batch_one(const BatchArgs& b, int tpb, cudaStream_t st, bool fast, bool idx32) {
    if (b.nrows <= 0) return;
    if (fast) {
        if (idx32) k_step_fast_batch<kQ, C, S, LES, true><<<b.nrows, tpb, 0, st>>>(b);
        else k_step_fast_batch<kQ, C, S, LES, false><<<b.nrows, tpb, 0, st>>>(b);
    } else {
        k_step_batch<kQ, C, S, LES><<<b.nrows, tpb, 0, st>>>(b);
    }
}
using StepFn = void (*)(const StepArgs&, const Launch&, bool);
using BatchFn = void (*)(const BatchArgs&, int, cudaStream_t, bool, bool);
using InitFn = void (*)(const float*, void*, void*, const uint8_t*, const Geo&, const Physics&, const Launch&);

#define WK_ROW(C, S) {step_one<C, S, false>, step_one<C, S, true>}
#define WK_IROW(C, S) {initial_one<C, S, false>, initial_one<C, S, true>}
const StepFn kStep[3][3][2] = {{WK_ROW(0, 0), WK_ROW(0, 1), WK_ROW(0, 2)},
                               {WK_ROW(1, 0), WK_ROW(1, 1), WK_ROW(1, 2)},
                               {WK_ROW(2, 0), WK_ROW(2, 1), WK_ROW(2, 2)}};
const InitFn kInit[3][3][2] = {{WK_IROW(0, 0), WK_IROW(0, 1), WK_IROW(0, 2)},
                               {WK_IROW(1, 0), WK_IROW(1, 1), WK_IROW(1, 2)},
                               {WK_IROW(2, 0), WK_IROW(2, 1), WK_IROW(2, 2)}};
#define WK_BROW(C, S) {batch_one<C, S, false>, batch_one<C, S, true>}
const BatchFn kBatch[3][3][2] = {{WK_BROW(0, 0), WK_BROW(0, 1), WK_BROW(0, 2)},
                                 {WK_BROW(1, 0), WK_BROW(1, 1), WK_BROW(1, 2)},
                                 {WK_BROW(2, 0), WK_BROW(2, 1), WK_BROW(2, 2)}};
#undef WK_ROW
#undef WK_IROW
#undef WK_BROW

bool valid(int coll, int store) { return coll >= 0 && coll < 3 && store >= 0 && store < 3; }
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

cudaError_t WK_CAT(launch_initial_q, WK_Q)(int coll, int store, bool les, const float* f0, void* a, void* b,
                                          const uint8_t* flags, const Geo& geo, const Physics& phys,
                                          const Launch& L) {
    if (!valid(coll, store)) return cudaErrorInvalidValue;
    kInit[coll][store][les ? 1 : 0](f0, a, b, flags, geo, phys, L);
    return cudaGetLastError();
}

cudaError_t WK_CAT(launch_materialise_q, WK_Q)(int store, const void* fin, const uint8_t* flags, const Geo& geo,
                                              const Links& links, const Physics& phys, const Out& out,
                                              const Launch& L, int direct) {
    const int blocks = L.rows * L.xchunks;
    if (direct) {
        switch (store) {
            case 0: k_direct<kQ, 0><<<blocks, L.tpb, 0, L.stream>>>(fin, flags, geo, phys, out, L.xchunks); break;
            case 1: k_direct<kQ, 1><<<blocks, L.tpb, 0, L.stream>>>(fin, flags, geo, phys, out, L.xchunks); break;
            case 2: k_direct<kQ, 2><<<blocks, L.tpb, 0, L.stream>>>(fin, flags, geo, phys, out, L.xchunks); break;
            default: return cudaErrorInvalidValue;
        }
    } else {
        switch (store) {
            case 0: k_materialise<kQ, 0><<<blocks, L.tpb, 0, L.stream>>>(fin, flags, geo, links, phys, out, L.xchunks); break;
            case 1: k_materialise<kQ, 1><<<blocks, L.tpb, 0, L.stream>>>(fin, flags, geo, links, phys, out, L.xchunks); break;
            case 2: k_materialise<kQ, 2><<<blocks, L.tpb, 0, L.stream>>>(fin, flags, geo, links, phys, out, L.xchunks); break;
            default: return cudaErrorInvalidValue;
        }
    }
    return cudaGetLastError();
}

cudaError_t WK_CAT(launch_flags_q, WK_Q)(const uint8_t* types, uint8_t* flags, const Geo& geo, const FlagCfg& cfg,
                                        const Launch& L) {
    k_flags<kQ><<<L.rows * L.xchunks, L.tpb, 0, L.stream>>>(types, flags, geo, cfg, L.xchunks);
    return cudaGetLastError();
}

cudaError_t WK_CAT(launch_row_class_q, WK_Q)(const uint8_t* flags, uint8_t* cls, const Geo& geo, const Launch& L) {
    k_row_class<kQ><<<L.rows, 256, 0, L.stream>>>(flags, cls, geo);
    return cudaGetLastError();
}

}  // namespace wk
