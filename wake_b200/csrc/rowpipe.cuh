// Pipelined whole-row step kernel for the TRT lattices: the TMA engine's bulk
// copies move every pure-gather row through shared memory, in both directions.
//
// Work unit: one row (z, y) whose every node is a pure gather (ROW_FAST, rows.cuh).
// Its Q pull sources are whole rows: direction q reads row (y - cy, z - cz) of
// plane q (after the periodic wraps), and the x shift of the pull, including the
// x-periodic wrap, stays inside that row. So one cp.async.bulk per direction
// brings the sources of the whole row into shared memory, laid out as Q rows of
// CAP elements, and threads read them at compile-time offsets (q * CAP plus one of
// four per-thread x positions, as in k_step_rows). After the collision the
// results go back into the same stage, in place once every thread has read its
// inputs, and one bulk copy per direction writes the row of plane q. No thread
// builds a global address.
//
// Each CTA walks its share of the rows with NS stages and two roles. One producer
// warp issues every bulk copy, lane q taking direction q: it loads rows NS ahead, and
// once the compute threads mark a row's results in place (mbarrier `written`) it
// stores that row and, when the stores have read the stage, loads the row NS further
// on into it. CAP / 2 compute threads (one adjacent node pair each) wait for a stage's
// inputs (mbarrier `full`), compute, and meet at one named barrier per row before
// writing the results in place, so no CTA-wide barrier stalls the copies. Several
// CTAs per SM interleave their phases.
//
// Every wait is bounded: a stage that does not arrive within ~2^22 polls sets
// ERR_STAGE_TIMEOUT in the lattice's status word; the compute threads skip the
// row's arithmetic and leave together at the row's named barrier (it ANDs their
// wait results; nothing is written back), the producer gives up on its next
// bounded wait, drains its stores and gives loads in flight a bounded chance to land.
//
// Requirements (host-checked): TRT; nx even, nx <= CAP, nx * sizeof(T) a multiple
// of 16 bytes (bulk copies move whole 16-byte units from 16-byte-aligned
// addresses; the plane pitch is a multiple of 64 elements); Q * pitch < 2^32; no
// coupled temperature. The per-node arithmetic is trt_pairs2's, so results equal
// the span and row kernels' bit for bit.
#pragma once

#include "rows.cuh"
#include "staged.cuh"

namespace wk {

__device__ __forceinline__ void bulk_s2g(void* dst, unsigned src, unsigned bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Wait until every bulk group of this thread has finished reading shared memory.
__device__ __forceinline__ void bulk_wait_read_0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// Wait until every bulk group of this thread has completed.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Resident CTAs per SM the 256-wide 16-bit kernels are compiled for (register budget:
// 65536 / (WK_PIPE_MIN_BLOCKS * 160) per thread). FP32 stages are twice the bytes: three
// CTAs fill the shared memory, so that form keeps 127 registers.
#ifndef WK_PIPE_MIN_BLOCKS
#define WK_PIPE_MIN_BLOCKS 4
#endif

// Stages per CTA: FP32 rows take twice the bytes, so fewer of them.
template <int S, int CAP>
constexpr int pipe_stages() {
    return S == STORE_F32 ? (CAP > 256 ? 2 : 3) : 4;
}
template <int Q, int S, int CAP>
constexpr unsigned pipe_stage_bytes() {
    return static_cast<unsigned>(Q * CAP * sizeof(typename Codec<S>::T));
}
template <int Q, int S, int CAP>
constexpr unsigned pipe_smem_bytes() {
    return 128u + static_cast<unsigned>(pipe_stages<S, CAP>()) * pipe_stage_bytes<Q, S, CAP>();
}

// Rows of one launch: ROW_FAST rows as (row index | row descriptor << 28).
struct PipeArgs {
    const unsigned* rows;
    int nrows;
};

// (cy + 1) | (cz + 1) << 2 of directions base .. base + 15 in 4-bit fields, built at compile time.
template <int Q>
constexpr unsigned long long yz_codes(int base) {
    unsigned long long c = 0;
    for (int k = base; k < Q && k < base + 16; ++k)
        c |= static_cast<unsigned long long>((Lat<Q>::cy(k) + 1) | ((Lat<Q>::cz(k) + 1) << 2)) << (4 * (k - base));
    return c;
}

// y and z shifts of direction q, q known only at run time (a producer lane's direction).
template <int Q>
__device__ __forceinline__ void pull_shift(int q, int& cy, int& cz) {
    constexpr unsigned long long lo = yz_codes<Q>(0), hi = yz_codes<Q>(16);
    const unsigned long long w = q < 16 ? (lo >> (4 * q)) : (hi >> (4 * (q - 16)));
    cy = static_cast<int>(w & 3ull) - 1;
    cz = static_cast<int>((w >> 2) & 3ull) - 1;
}

// Producer lane q (< Q) copies direction q's source row of `row` into its slot of the stage
// (shared address `stage`); lane 0 posts the byte count first. All lanes issue at once.
template <int Q, int CAP, class T>
__device__ __forceinline__ void pipe_load(const StepArgs& a, unsigned row, unsigned stage, unsigned bar) {
    const int nx = a.geo.nx, ny = a.geo.ny, nz = a.geo.nz;
    const int y = static_cast<int>(row % static_cast<unsigned>(ny));
    const int z = static_cast<int>(row / static_cast<unsigned>(ny));
    const unsigned bytes = static_cast<unsigned>(nx) * sizeof(T);
    const int lane = threadIdx.x & 31;
    if (lane == 0) mbar_expect_tx(bar, Q * bytes);
    __syncwarp();
    if (lane < Q) {
        int cy, cz;
        pull_shift<Q>(lane, cy, cz);
        int sy = y - cy, sz = z - cz;
        sy += (sy < 0) ? ny : 0;
        sy -= (sy >= ny) ? ny : 0;
        sz += (sz < 0) ? nz : 0;
        sz -= (sz >= nz) ? nz : 0;
        const T* src = static_cast<const T*>(a.fin) + (static_cast<unsigned>(lane) * static_cast<unsigned>(a.geo.pitch) +
                                                       static_cast<unsigned>((sz * ny + sy) * nx));
        bulk_g2s(stage + static_cast<unsigned>(lane * CAP * sizeof(T)), src, bytes, bar);
    }
}

// Producer lane q writes direction q's row of results from the stage to plane q and commits it
// as one bulk group of its own.
template <int Q, int CAP, class T>
__device__ __forceinline__ void pipe_store(const StepArgs& a, unsigned row, unsigned stage) {
    const unsigned nx = static_cast<unsigned>(a.geo.nx);
    const unsigned bytes = nx * sizeof(T);
    const int lane = threadIdx.x & 31;
    if (lane < Q) {
        T* dst = static_cast<T*>(a.fout) + (static_cast<unsigned>(lane) * static_cast<unsigned>(a.geo.pitch) + row * nx);
        bulk_s2g(dst, stage + static_cast<unsigned>(lane * CAP * sizeof(T)), bytes);
        bulk_commit();
    }
}

template <int S>
__device__ __forceinline__ float2 smem_adjacent(const typename Codec<S>::T* p) {
    if constexpr (S == STORE_F32) {
        return *reinterpret_cast<const float2*>(p);
    } else if constexpr (S == STORE_F16C) {
        return f16c_decode_word(*reinterpret_cast<const unsigned*>(p));
    } else {
        const unsigned w = *reinterpret_cast<const unsigned*>(p);
        return make_float2(raw_lo<S>(w), raw_hi<S>(w));
    }
}
// 32-bit word of a 16-bit stage row at an even element index
template <class T>
__device__ __forceinline__ unsigned smem_word(const T* p) {
    return *reinterpret_cast<const unsigned*>(p);
}
template <int S>
__device__ __forceinline__ float smem_one(const typename Codec<S>::T* p) {
    if constexpr (S == STORE_F32) return *p;
    else if constexpr (S == STORE_F16) return __half2float(*p);
    else if constexpr (S == STORE_F16C) return f16c_decode(p->bits);
    else return __bfloat162float(*p);
}
template <int S>
__device__ __forceinline__ void smem_store_adjacent(typename Codec<S>::T* p, float2 v) {
    if constexpr (S == STORE_F32) {
        *reinterpret_cast<float2*>(p) = v;
    } else if constexpr (S == STORE_F16) {
        const __half2 h = __floats2half2_rn(v.x, v.y);
        *reinterpret_cast<__half2*>(p) = h;
    } else if constexpr (S == STORE_F16C) {
        *reinterpret_cast<unsigned*>(p) = f16c_encode2(v);
    } else {
        const __nv_bfloat162 h = __floats2bfloat162_rn(v.x, v.y);
        *reinterpret_cast<__nv_bfloat162*>(p) = h;
    }
}

__device__ __forceinline__ void mbar_arrive(unsigned bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Named barrier over the compute threads (id 1) that also ANDs a predicate across them, so
// that a timed-out wait ends the loop for every compute thread together.
__device__ __forceinline__ bool compute_bar_and(bool v, int nthreads) {
    int r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.s32 p, %1, 0;\n\t"
        "bar.red.and.pred q, 1, %2, p;\n\t"
        "selp.s32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"(v ? 1 : 0), "r"(nthreads)
        : "memory");
    return r != 0;
}

// CAP / 2 compute threads (one adjacent node pair each) and one producer warp.
template <int CAP>
constexpr int pipe_threads() {
    return CAP / 2 + 32;
}

template <int Q, int S, bool LES, int CAP>
__global__ void __launch_bounds__(CAP / 2 + 32, CAP > 256 ? 1 : (S == STORE_F32 ? 3 : WK_PIPE_MIN_BLOCKS))
    k_step_rows_pipe(const StepArgs a, const PipeArgs p) {
    using L = Lat<Q>;
    using T = typename Codec<S>::T;
    constexpr bool HS = S != STORE_F32;
    constexpr int NS = pipe_stages<S, CAP>();
    constexpr int NC = CAP / 2;  // compute threads
    constexpr unsigned STAGE_B = pipe_stage_bytes<Q, S, CAP>();
    extern __shared__ __align__(128) unsigned char smem[];
    // barriers: full[s] (the stage's inputs landed), written[s] (its results are in place)
    unsigned long long* full = reinterpret_cast<unsigned long long*>(smem);
    unsigned long long* written = full + NS;
    unsigned char* stages = smem + 128;
    const unsigned stages_s = smem_addr(stages);
    const int first = blockIdx.x, stride = gridDim.x;
    const int mine = first < p.nrows ? (p.nrows - first + stride - 1) / stride : 0;
    if (threadIdx.x == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(smem_addr(&full[s]), 1);
            mbar_init(smem_addr(&written[s]), NC);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x >= NC) {
        // ---- producer warp: loads NS rows ahead, stores each row once its results are in place
        int issued = 0;  // rows whose loads have been issued (row r goes to stage r % NS)
        for (; issued < NS && issued < mine; ++issued)
            pipe_load<Q, CAP, T>(a, p.rows[first + issued * stride] & 0x0fffffffu, stages_s + issued * STAGE_B,
                                 smem_addr(&full[issued]));
        for (int it = 0; it < mine; ++it) {
            const int s = it % NS;
            const bool ok = mbar_wait(smem_addr(&written[s]), static_cast<unsigned>((it / NS) & 1));
            if (!__all_sync(0xffffffffu, ok)) {
                if ((threadIdx.x & 31) == 0) atomicOr(a.status, ERR_STAGE_TIMEOUT);
                // the compute threads stopped: let the loads still in flight (rows it .. issued-1)
                // land before the CTA's shared memory goes away (bounded waits)
                for (int r = it; r < issued; ++r)
                    (void)mbar_wait(smem_addr(&full[r % NS]), static_cast<unsigned>((r / NS) & 1));
                break;
            }
            pipe_store<Q, CAP, T>(a, p.rows[first + it * stride] & 0x0fffffffu, stages_s + s * STAGE_B);
            if (issued < mine) {
                bulk_wait_read_0();  // this stage's stores have read it
                __syncwarp();
                pipe_load<Q, CAP, T>(a, p.rows[first + issued * stride] & 0x0fffffffu, stages_s + s * STAGE_B,
                                     smem_addr(&full[s]));
                ++issued;
            }
        }
        bulk_wait_all();  // the stores read shared memory until they complete
        return;
    }
    // ---- compute threads
    const int nx = a.geo.nx;
    const int xa = 2 * static_cast<int>(threadIdx.x);  // this thread's nodes xa, xa + 1
    const bool live = xa < nx;
    const int xm = xa == 0 ? nx - 1 : xa - 1;          // cx = +1 source of node xa
    const int xp = xa + 2 == nx ? 0 : xa + 2;          // cx = -1 source of node xa + 1
    for (int it = 0; it < mine; ++it) {
        const int s = it % NS;
        const unsigned kind = p.rows[first + it * stride] >> 28;
        const bool ok = mbar_wait(smem_addr(&full[s]), static_cast<unsigned>((it / NS) & 1));
        T* st = reinterpret_cast<T*>(stages + s * STAGE_B);
        float2 f[Q];
        if (live && ok) {
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const T* r = st + q * CAP;
                if (L::cx(q) == 0) {
                    f[q] = smem_adjacent<S>(r + xa);
                } else if constexpr (S == STORE_F16C) {
                    // the shifted pair from two aligned words: the high half of one, the low half
                    // of the next (xm - 1, xa, xp even)
                    f[q] = L::cx(q) > 0 ? f16c_decode_hl(smem_word(r + (xm - 1)), smem_word(r + xa))
                                        : f16c_decode_hl(smem_word(r + xa), smem_word(r + xp));
                } else if (L::cx(q) > 0) {
                    f[q] = make_float2(smem_one<S>(r + xm), smem_one<S>(r + xa));
                } else {
                    f[q] = make_float2(smem_one<S>(r + xa + 1), smem_one<S>(r + xp));
                }
            }
            if ((kind & ROW_ZH_IN) && xa == 0) zou_he_half<Q, HS>(f, 0, FL_ZH_IN, a.geo);
            if ((kind & ROW_ZH_OUT) && xa + 2 == nx) zou_he_half<Q, HS>(f, 1, FL_ZH_OUT, a.geo);
            float2 rho, u[3];
            trt_pairs2<Q, LES, HS>(f, a.phys, rho, u);
            if (!(rho.x > 0.0f) || !(fabsf(u[0].x) < 1e30f) || !(rho.y > 0.0f) || !(fabsf(u[0].y) < 1e30f))
                atomicOr(a.status, ERR_NONFINITE);
        }
        // one barrier per row: every input of the stage has been read (the results go back in
        // place), and a wait that ran out anywhere ends the loop for every compute thread
        if (!compute_bar_and(ok, NC)) {
            if (threadIdx.x == 0) atomicOr(a.status, ERR_STAGE_TIMEOUT);
            break;
        }
        if (live) {
#pragma unroll
            for (int q = 0; q < Q; ++q) smem_store_adjacent<S>(st + q * CAP + xa, f[q]);
        }
        fence_proxy_async_smem();  // the results are visible to the bulk copies
        mbar_arrive(smem_addr(&written[s]));
    }
}

}  // namespace wk
