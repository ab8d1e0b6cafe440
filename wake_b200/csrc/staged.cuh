// Persistent step kernel with the pure-gather rows staged in shared memory.
//
// Work of one step: the segments of the rows that are not entirely pure-gather
// (walls, solids, curved links, momentum exchange; per-node path of step_chunk,
// straight from global memory) and the pure-gather tiles. A tile is up to TILE_NODES nodes: `count` consecutive rows
// y0 .. y0+count-1 of one z plane, i.e. one contiguous range of node indices.
// For direction q the tile's pull sources are the rows y0-cy .. y0-cy+count-1 of
// plane z-cz: again one contiguous range of plane q (two when the range wraps
// around a periodic y). One cp.async.bulk per direction (per range) brings them
// into a shared-memory stage whose layout is the tile's own node order, so node
// n of the tile reads direction q at stage offset q*tile + n - cx (wrapped to
// the row's other end at x = 0 / nx-1: the x-periodic pull stays inside the
// copied row). No halo copies.
//
// Each CTA (TILE_CTAS_PER_SM per SM) walks its share of the tiles with TILE_STAGES stages in
// flight, so HBM latency is covered by bytes in flight in shared memory rather
// than by resident warps. The arithmetic is the two-node packed FP32 TRT of
// trt_pairs2 (thread t carries tile nodes t and t + TILE_THREADS); other
// collision models run one node at a time.
//
// Requirements (host-checked): nx * sizeof(T) a multiple of 16 and nx <= TILE_NODES.
#pragma once

#include <type_traits>

#include "stream_collide.cuh"

namespace wk {

enum : unsigned { ERR_STAGE_TIMEOUT = 4u };

constexpr int TILE_NODES = 512;  // nodes per tile (= 2 x TILE_THREADS)
constexpr int TILE_THREADS = 256;
constexpr int TILE_STAGES = 2;
constexpr int TILE_CTAS_PER_SM = 2;  // two CTAs interleave their load / compute phases

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Bounded wait for the phase with the given parity: false after ~2^22 polls
// (each poll may suspend the thread for a while), so a lost copy ends the
// kernel with an error instead of a hang.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
    for (int i = 0; i < (1 << 22); ++i) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void bulk_g2s(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Work lists of one launch. tiles: (member, (z << 16) | y0, count, 0);
// gen: (member, segment, entry, 0) for the general segments, entry = the
// segment's index in its member's general-segment list (momentum-exchange
// slots); spans: the pure-gather runs of the rows that hold general segments.
struct TileArgs {
    const uint4* tiles;
    int ntiles;
    const uint4* gen;
    int ngen;
    const BatchDom* dom;  // batch: member table; single lattice: null (the StepArgs parameter)
    int parity;
    const uint4* spans;   // pure-gather spans (member, row, x0, x1) of the rows outside the tiles
    int nspans;
};

template <bool BATCH>
__device__ __forceinline__ StepArgs tile_member(const StepArgs& a, const TileArgs& t, unsigned m) {
    if constexpr (BATCH) {
        const BatchDom* d = t.dom + m;
        StepArgs r = d->a;
        const int c = d->cur0 ^ t.parity;
        r.fin = d->buf[c];
        r.fout = d->buf[c ^ 1];
        r.th.tin = d->tbuf[c];
        r.th.tout = d->tbuf[c ^ 1];
        return r;
    } else {
        (void)t;
        (void)m;
        return a;
    }
}

// Issue the copies of one tile (warp 0): lane 0 posts the byte count, lane q
// issues direction q's one or two copies.
template <int Q, class T>
__device__ __forceinline__ void tile_issue(const StepArgs& a, uint4 tl, unsigned stage, unsigned bar) {
    using L = Lat<Q>;
    const int nx = a.geo.nx, ny = a.geo.ny, nz = a.geo.nz;
    const int y0 = static_cast<int>(tl.y & 0xffffu), z = static_cast<int>(tl.y >> 16), cnt = static_cast<int>(tl.z);
    const unsigned tile_b = static_cast<unsigned>(cnt * nx) * sizeof(T);
    const int lane = threadIdx.x & 31;
    if (lane == 0) mbar_expect_tx(bar, Q * tile_b);
    __syncwarp();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        if (lane != q) continue;
        int sz = z - L::cz(q);
        sz += (sz < 0) ? nz : 0;
        sz -= (sz >= nz) ? nz : 0;
        int sy = y0 - L::cy(q);  // first source row; the range may wrap around a periodic y
        sy += (sy < 0) ? ny : 0;
        sy -= (sy >= ny) ? ny : 0;
        const int first = min(cnt, ny - sy);  // rows before the wrap
        const T* plane = static_cast<const T*>(a.fin) + static_cast<long long>(q) * a.geo.pitch;
        const unsigned dst = stage + static_cast<unsigned>(q) * (TILE_NODES * sizeof(T));
        const unsigned b1 = static_cast<unsigned>(first * nx) * sizeof(T);
        bulk_g2s(dst, plane + (static_cast<long long>(sz) * ny + sy) * nx, b1, bar);
        if (first < cnt) bulk_g2s(dst + b1, plane + static_cast<long long>(sz) * ny * nx, tile_b - b1, bar);
    }
}

template <class T>
__device__ __forceinline__ float from_stage(T v) {
    if constexpr (std::is_same<T, float>::value) return v;
    else if constexpr (std::is_same<T, __half>::value) return __half2float(v);
    else if constexpr (std::is_same<T, f16c_t>::value) return f16c_decode(v.bits);
    else return __bfloat162float(v);
}

// One node of a tile for the scalar collision models (BGK, MRT).
template <int Q, int COLL, int S, bool LES>
__device__ __forceinline__ void tile_node_scalar(const StepArgs& a, const typename Codec<S>::T* st, long long base,
                                                 int n, int nx) {
    using L = Lat<Q>;
    using C = Codec<S>;
    using T = typename C::T;
    const int x = n % nx;
    const int im = (x == nx - 1) ? n - nx + 1 : n + 1;  // cx = -1 reads x + 1
    const int ip = (x == 0) ? n + nx - 1 : n - 1;       // cx = +1 reads x - 1
    const uint8_t fl = a.flags[base + n];
    float f[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int i = L::cx(q) > 0 ? ip : (L::cx(q) < 0 ? im : n);
        const float v = from_stage<T>(st[q * TILE_NODES + i]);
        f[q] = S == STORE_F32 ? v : fmaf(L::w(q), v, L::w(q));
    }
    if (fl & FL_ZH_IN) zou_he_inlet<Q>(f, a.geo.uin);
    if (fl & FL_ZH_OUT) zou_he_outlet<Q>(f, a.geo.rho_out);
    float rho, u[3];
    node_moments<Q>(f, a.phys.g, rho, u);
    collide<Q, COLL, LES>(f, rho, u, a.phys);
    if (!(rho > 0.0f) || !(fabsf(u[0]) < 1e30f)) atomicOr(a.status, ERR_NONFINITE);
    T* out = static_cast<T*>(a.fout);
#pragma unroll
    for (int q = 0; q < Q; ++q) C::store_stream(out + (q * a.geo.pitch + base + n), f[q], L::w(q));
}

// Nodes n and n + TILE_THREADS of a tile, TRT in packed FP32 (h-space for shifted storage).
template <int Q, int S, bool LES>
__device__ __forceinline__ void tile_pair_trt(const StepArgs& a, const typename Codec<S>::T* st, long long base,
                                              int na, int count_nodes, int nx) {
    using L = Lat<Q>;
    using T = typename Codec<S>::T;
    constexpr bool HS = S != STORE_F32;
    const bool vb = na + TILE_THREADS < count_nodes;
    const int nb = vb ? na + TILE_THREADS : na;  // a partial tile computes node a twice, stores it once
    const int xa = na % nx, xb = nb % nx;
    const int ima = (xa == nx - 1) ? na - nx + 1 : na + 1, ipa = (xa == 0) ? na + nx - 1 : na - 1;
    const int imb = (xb == nx - 1) ? nb - nx + 1 : nb + 1, ipb = (xb == 0) ? nb + nx - 1 : nb - 1;
    const uint8_t fa = a.flags[base + na], fb = a.flags[base + nb];
    float2 f[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int ia = L::cx(q) > 0 ? ipa : (L::cx(q) < 0 ? ima : na);
        const int ib = L::cx(q) > 0 ? ipb : (L::cx(q) < 0 ? imb : nb);
        f[q] = make_float2(from_stage<T>(st[q * TILE_NODES + ia]), from_stage<T>(st[q * TILE_NODES + ib]));
    }
    if ((fa | fb) & (FL_ZH_IN | FL_ZH_OUT)) {
        if (fa & (FL_ZH_IN | FL_ZH_OUT)) zou_he_half<Q, HS>(f, 0, fa, a.geo);
        if (fb & (FL_ZH_IN | FL_ZH_OUT)) zou_he_half<Q, HS>(f, 1, fb, a.geo);
    }
    float2 rho, u[3];
    trt_pairs2<Q, LES, HS>(f, a.phys, rho, u);
    const bool bad =
        !(rho.x > 0.0f) || !(fabsf(u[0].x) < 1e30f) || (vb && (!(rho.y > 0.0f) || !(fabsf(u[0].y) < 1e30f)));
    if (bad) atomicOr(a.status, ERR_NONFINITE);
    T* out = static_cast<T*>(a.fout) + (base + na);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        store_raw<S>(out + q * a.geo.pitch, f[q].x);
        if (vb) store_raw<S>(out + (q * a.geo.pitch + TILE_THREADS), f[q].y);
    }
}

template <int Q, int COLL, int S, bool LES, bool BATCH>
__global__ void __launch_bounds__(TILE_THREADS, TILE_CTAS_PER_SM) k_step_tiles(const StepArgs a0, const TileArgs t) {
    using T = typename Codec<S>::T;
    constexpr unsigned STAGE_B = Q * TILE_NODES * sizeof(T);
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem);
    unsigned char* stages = smem + 128;
    const unsigned stages_s = smem_addr(stages);
    const int first = blockIdx.x, stride = gridDim.x;
    const int mine = first < t.ntiles ? (t.ntiles - first + stride - 1) / stride : 0;
    const bool issuer = threadIdx.x < 32;
    if (threadIdx.x == 0) {
        for (int s = 0; s < TILE_STAGES; ++s) mbar_init(smem_addr(&bars[s]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // the first tiles' copies go out before the general rows, so they land meanwhile
    if (issuer) {
        for (int k = 0; k < TILE_STAGES && k < mine; ++k) {
            const uint4 tl = t.tiles[first + k * stride];
            tile_issue<Q, T>(tile_member<BATCH>(a0, t, tl.x), tl, stages_s + k * STAGE_B, smem_addr(&bars[k]));
        }
    }
    // rows outside the tiles, from global memory: general segments one warp per
    // 32-node chunk, pure-gather spans one CTA per span (the direct kernels' paths)
    {
        const int warps = blockDim.x >> 5;
        constexpr int CPS = SEG / 32;  // warp chunks per segment
        for (int g = first * warps + static_cast<int>(threadIdx.x >> 5); g < CPS * t.ngen; g += stride * warps) {
            const uint4 r = t.gen[g / CPS];
            step_chunk<Q, COLL, S, LES>(tile_member<BATCH>(a0, t, r.x), r.y, static_cast<int>(r.z), g % CPS);
        }
        for (int sp = first; sp < t.nspans; sp += stride) {
            const uint4 r = t.spans[sp];
            const StepArgs a = tile_member<BATCH>(a0, t, r.x);
            step_span_fast<Q, COLL, S, LES, false>(a, span_decode(r, a.geo));
        }
    }
    for (int it = 0; it < mine; ++it) {
        const int s = it % TILE_STAGES;
        const uint4 tl = t.tiles[first + it * stride];
        const StepArgs a = tile_member<BATCH>(a0, t, tl.x);
        const bool ok = mbar_wait(smem_addr(&bars[s]), static_cast<unsigned>((it / TILE_STAGES) & 1));
        if (!__syncthreads_and(ok)) {
            if (threadIdx.x == 0) atomicOr(a.status, ERR_STAGE_TIMEOUT);
            // give copies still in flight a bounded chance to land before the CTA exits
            for (int k = 0; k < TILE_STAGES; ++k) (void)mbar_wait(smem_addr(&bars[k]), 0u);
            return;
        }
        const T* st = reinterpret_cast<const T*>(stages + s * STAGE_B);
        const int nx = a.geo.nx;
        const int y0 = static_cast<int>(tl.y & 0xffffu), z = static_cast<int>(tl.y >> 16);
        const int count_nodes = static_cast<int>(tl.z) * nx;
        const long long base = (static_cast<long long>(z) * a.geo.ny + y0) * nx;
        if constexpr (COLL == COLL_TRT) {
            if (static_cast<int>(threadIdx.x) < count_nodes)
                tile_pair_trt<Q, S, LES>(a, st, base, threadIdx.x, count_nodes, nx);
        } else {
            for (int n = threadIdx.x; n < count_nodes; n += TILE_THREADS)
                tile_node_scalar<Q, COLL, S, LES>(a, st, base, n, nx);
        }
        __syncthreads();  // every read of stage s is done
        if (issuer && it + TILE_STAGES < mine) {
            fence_proxy_async_smem();
            const uint4 tn = t.tiles[first + (it + TILE_STAGES) * stride];
            tile_issue<Q, T>(tile_member<BATCH>(a0, t, tn.x), tn, stages_s + s * STAGE_B, smem_addr(&bars[s]));
        }
    }
}

template <int Q, int S>
constexpr unsigned tile_smem_bytes() {
    return 128 + TILE_STAGES * Q * TILE_NODES * sizeof(typename Codec<S>::T);
}

// A lattice whose rows allow the tile kernel: whole 16-byte chunks per row, a row fits a tile.
inline bool tile_row_ok(int nx, int elem_bytes) {
    return nx <= TILE_NODES && nx * elem_bytes >= 16 && (nx * elem_bytes) % 16 == 0;
}

}  // namespace wk
