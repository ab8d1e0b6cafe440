// Whole-row step kernel for the TRT lattices: one block per lattice row, two
// adjacent nodes per thread.
//
// The pure-gather spans of k_step_fast carry their row in a table, so every
// load address is built per thread from the row it reads. Here the block index
// is the row itself (z * ny + y): the row, its source rows and, for every
// direction q, the element offset of the source row in plane q are the same for
// all threads of the launch's block, and a load is that offset plus one of four
// per-thread x positions computed once per 64-node chunk:
//
//   cx =  0: nodes x, x+1 read the 32-bit (16-bit storage) or 64-bit (FP32)
//            word at x of the source row
//   cx = +1: node x reads x-1 (wrapped to nx-1 at x = 0), node x+1 reads x
//   cx = -1: node x reads x+1, node x+1 reads x+2 (wrapped to 0 at x = nx-2)
//
// and every direction's two results leave with one 32-bit (16-bit storage) or
// 64-bit (FP32) streaming store. A row descriptor byte replaces the per-node
// flag reads: ROW_FAST marks a row whose every node is a pure gather (no solid,
// wall, curved link or momentum-exchange link in reach), with ROW_ZH_IN /
// ROW_ZH_OUT when its first / last node is a Zou-He inlet / outlet. Other rows
// exit at once; their pure-gather runs go to k_step_fast and the rest to k_step.
//
// Requirements (host-checked): TRT, nx even (rows start on a word boundary),
// Q * pitch < 2^32 (32-bit element offsets), no coupled temperature. The per-node
// arithmetic is trt_pairs2's, so results equal the span kernel's bit for bit.
#pragma once

#include "stream_collide.cuh"

namespace wk {

enum : uint8_t { ROW_FAST = 1u, ROW_ZH_IN = 2u, ROW_ZH_OUT = 4u };

// Two adjacent populations of one plane (x even): a 64-bit word (FP32) or a 32-bit word of
// two 16-bit values, as floats (node x in .x).
template <int S>
__device__ __forceinline__ float2 load_adjacent(const typename Codec<S>::T* p) {
    if constexpr (S == STORE_F32) {
        return __ldg(reinterpret_cast<const float2*>(p));
    } else if constexpr (S == STORE_F16C) {
        return f16c_decode_word(__ldg(reinterpret_cast<const unsigned*>(p)));
    } else {
        const unsigned w = __ldg(reinterpret_cast<const unsigned*>(p));
        return make_float2(raw_lo<S>(w), raw_hi<S>(w));
    }
}

template <int S>
__device__ __forceinline__ void store_adjacent(typename Codec<S>::T* p, float2 v) {
    if constexpr (S == STORE_F32) __stcs(reinterpret_cast<float2*>(p), v);
    else store_pair<S>(p, v);
}

template <int Q, int S, bool LES>
__global__ void __launch_bounds__(WK_FAST_MAX_THREADS, Q == 9 ? WK_FAST_TRT9_MIN_BLOCKS : WK_FAST_TRT_MIN_BLOCKS)
    k_step_rows(const StepArgs a) {
    using L = Lat<Q>;
    using T = typename Codec<S>::T;
    constexpr bool HS = S != STORE_F32;
    const unsigned row = blockIdx.x;
    const unsigned kind = a.row_kind[row];
    if (!(kind & ROW_FAST)) return;
    const int nx = a.geo.nx, ny = a.geo.ny, nz = a.geo.nz;
    const int y = static_cast<int>(row % static_cast<unsigned>(ny));
    const int z = static_cast<int>(row / static_cast<unsigned>(ny));
    // source rows of the shifts c = -1, 0, +1; in a pure-gather row every source is in
    // range after the periodic wraps, so the wraps apply unconditionally
    const int ys[3] = {y + 1 == ny ? 0 : y + 1, y, y == 0 ? ny - 1 : y - 1};
    const int zs[3] = {z + 1 == nz ? 0 : z + 1, z, z == 0 ? nz - 1 : z - 1};
    const unsigned P = static_cast<unsigned>(a.geo.pitch);
    const unsigned row0 = row * static_cast<unsigned>(nx);
    const T* fin = static_cast<const T*>(a.fin);
    T* fout = static_cast<T*>(a.fout);
    const int lane = threadIdx.x & 31;
    for (int x0 = (threadIdx.x >> 5) * 64; x0 < nx; x0 += (blockDim.x >> 5) * 64) {
        const int xa = x0 + 2 * lane;  // nodes xa, xa + 1 (nx even: both in the row)
        if (xa >= nx) break;
        const int xm = xa == 0 ? nx - 1 : xa - 1;
        const int xp = xa + 2 == nx ? 0 : xa + 2;
        float2 f[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const T* src = fin + (q * P + static_cast<unsigned>((zs[L::cz(q) + 1] * ny + ys[L::cy(q) + 1]) * nx));
            if (L::cx(q) == 0) f[q] = load_adjacent<S>(src + xa);
            else if (L::cx(q) > 0) f[q] = make_float2(load_raw<S>(src + xm), load_raw<S>(src + xa));
            else f[q] = make_float2(load_raw<S>(src + (xa + 1)), load_raw<S>(src + xp));
        }
        if ((kind & ROW_ZH_IN) && xa == 0) zou_he_half<Q, HS>(f, 0, FL_ZH_IN, a.geo);
        if ((kind & ROW_ZH_OUT) && xa + 2 == nx) zou_he_half<Q, HS>(f, 1, FL_ZH_OUT, a.geo);
        float2 rho, u[3];
        trt_pairs2<Q, LES, HS>(f, a.phys, rho, u);
        if (!(rho.x > 0.0f) || !(fabsf(u[0].x) < 1e30f) || !(rho.y > 0.0f) || !(fabsf(u[0].y) < 1e30f))
            atomicOr(a.status, ERR_NONFINITE);
#pragma unroll
        for (int q = 0; q < Q; ++q) store_adjacent<S>(fout + (q * P + row0) + xa, f[q]);
    }
}

}  // namespace wk
