// Lattice tables, storage codecs and node-local collision physics for the
// B200 lattice update. Everything here is per-node arithmetic in FP32
// registers; the kernels that move populations through HBM live in
// stream_collide.cuh.
//
// Lattice velocity orderings follow the reference's ISPC headers so that the
// population planes of a buffer line up with the reference's SoA layout
// [q][node]: include/wake/ispc/lbm_d2q9.isph:8-17, lbm_d3q19.isph:8-28,
// lbm_d3q27.isph:8-42.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cstdint>
#include <utility>

namespace wk {

// ---------------------------------------------------------------- cell types
// CellType codes (include/wake/core/types.hpp:69-77, include/wake/ispc/lbm_common.isph:12-18).
enum : uint8_t {
    CT_FLUID = 0,
    CT_SOLID = 1,
    CT_INFLOW = 2,
    CT_OUTFLOW = 3,
    CT_PERIODIC = 4,
    CT_SYMMETRY = 5,
    CT_MOVING_WALL = 6
};

// Per-node flag byte built on the device from the cell types.
//   bits 0-2  cell type
//   bit 3     FAST: not solid, every pull source in range and plain fluid,
//             no Zou-He, no curved link -> pure gather
//   bit 4     node owns curved-boundary (BFL) links
//   bit 5     Zou-He velocity inlet applies here
//   bit 6     Zou-He pressure outlet applies here
//   bit 7     node contributes a momentum-exchange link inside r_max
constexpr uint8_t FL_TYPE = 0x07, FL_FAST = 0x08, FL_BFL = 0x10, FL_ZH_IN = 0x20, FL_ZH_OUT = 0x40,
                  FL_MEM = 0x80;

// ---------------------------------------------------------------- tables
template <int Q>
struct Lat;

template <>
struct Lat<9> {
    static constexpr int D = 2;
    __host__ __device__ static constexpr int cx(int q) {
        constexpr int t[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
        return t[q];
    }
    __host__ __device__ static constexpr int cy(int q) {
        constexpr int t[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
        return t[q];
    }
    __host__ __device__ static constexpr int cz(int) { return 0; }
    __host__ __device__ static constexpr int opp(int q) {
        constexpr int t[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
        return t[q];
    }
    __host__ __device__ static constexpr float w(int q) {
        return q == 0 ? 4.0f / 9.0f : (q < 5 ? 1.0f / 9.0f : 1.0f / 36.0f);
    }
};

template <>
struct Lat<19> {
    static constexpr int D = 3;
    __host__ __device__ static constexpr int cx(int q) {
        constexpr int t[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
        return t[q];
    }
    __host__ __device__ static constexpr int cy(int q) {
        constexpr int t[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
        return t[q];
    }
    __host__ __device__ static constexpr int cz(int q) {
        constexpr int t[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
        return t[q];
    }
    __host__ __device__ static constexpr int opp(int q) {
        constexpr int t[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
        return t[q];
    }
    __host__ __device__ static constexpr float w(int q) {
        return q == 0 ? 1.0f / 3.0f : (q < 7 ? 1.0f / 18.0f : 1.0f / 36.0f);
    }
};

template <>
struct Lat<27> {
    static constexpr int D = 3;
    __host__ __device__ static constexpr int cx(int q) {
        constexpr int t[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};
        return t[q];
    }
    __host__ __device__ static constexpr int cy(int q) {
        constexpr int t[27] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1};
        return t[q];
    }
    __host__ __device__ static constexpr int cz(int q) {
        constexpr int t[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1};
        return t[q];
    }
    __host__ __device__ static constexpr int opp(int q) {
        // true opposites (c_opp = -c). The reference's table (lbm_d3q27.isph:35-40) pairs the
        // corners 19..26 with their x/y mirror images instead; see ref_opp_d3q27.
        constexpr int t[27] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15,
                               26, 25, 24, 23, 22, 21, 20, 19};
        return t[q];
    }
    __host__ __device__ static constexpr float w(int q) {
        return q == 0 ? 8.0f / 27.0f : (q < 7 ? 2.0f / 27.0f : (q < 19 ? 1.0f / 54.0f : 1.0f / 216.0f));
    }
};

// ---------------------------------------------------------------- storage codecs
// STORE_F32: plain populations. STORE_F16 / STORE_BF16 / STORE_F16C: the shifted,
// weight-normalised deviation h = f / w_q - 1, so f = w_q + w_q * h. All
// arithmetic stays in FP32; only the HBM representation narrows.
enum { STORE_F32 = 0, STORE_F16 = 1, STORE_BF16 = 2, STORE_F16C = 3 };

// FP16C: the 16-bit float format of Lehmann et al., "On the accuracy and performance of the
// lattice Boltzmann method with 64-bit, 32-bit, and customized 16-bit number formats",
// Phys. Rev. E 106, 015308 (2022): 1 sign, 4 exponent and 11 mantissa bits. Here the exponent
// field E = 1..15 encodes the binades 2^-14 .. 2^0, so a value is (-1)^s 2^(E-15) (1 + m/2^11),
// E = 0 holds subnormals (-1)^s 2^-14 m/2^11 (steps of 2^-25), the largest magnitude is
// 2 - 2^-11, and there is no infinity or NaN. Against IEEE half it trades the binades above 2,
// which no stable flow's h reaches (|h| < 2 is 0 < f < 3 w), for one more significant bit.
struct f16c_t {
    unsigned short bits;
};

// The 15 magnitude bits placed at float32 bits 12..26 read as a float32 whose exponent field is
// E: that float is 2^(E-127) (1 + m/2^11) (or, for E = 0, the float32 subnormal m 2^-137), and
// the exact scaling by 2^112 makes it the FP16C value. An arithmetic right shift by 4 of a
// register whose top half is the value puts the magnitude there and copies the sign into bits
// 27..31; one mask keeps bit 31. Needs subnormal float32 arithmetic (no flush to zero), which
// is this library's build.
__device__ __forceinline__ unsigned f16c_bits_hi(unsigned w) {  // value in bits 16..31 of w
    return static_cast<unsigned>(static_cast<int>(w) >> 4) & 0x87fff000u;
}
__device__ __forceinline__ unsigned f16c_bits_lo(unsigned w) {  // value in bits 0..15 of w
    return static_cast<unsigned>(static_cast<int>(w << 16) >> 4) & 0x87ffffffu;
}
__device__ __forceinline__ float f16c_decode(unsigned b) { return __uint_as_float(f16c_bits_lo(b)) * 0x1p112f; }
// .x from the high half of a, .y from the low half of b (one packed multiply)
__device__ __forceinline__ float2 f16c_decode_hl(unsigned a, unsigned b) {
    return __fmul2_rn(make_float2(__uint_as_float(f16c_bits_hi(a)), __uint_as_float(f16c_bits_lo(b))),
                      make_float2(0x1p112f, 0x1p112f));
}
// the two values of one 32-bit word: .x the low half, .y the high half
__device__ __forceinline__ float2 f16c_decode_word(unsigned w) {
    return __fmul2_rn(make_float2(__uint_as_float(f16c_bits_lo(w)), __uint_as_float(f16c_bits_hi(w))),
                      make_float2(0x1p112f, 0x1p112f));
}
// Nearest FP16C value, ties away from zero, magnitudes above the largest saturating to it. The
// float32 bits of h 2^-112 (exact, or a float32 subnormal below 2^-14, finer than the format's
// steps) plus half a unit of bit 12 round the magnitude (a mantissa carry moves into the
// exponent field); a signed minimum then saturates positive values and an unsigned one the
// magnitude of negative values (a NaN becomes the largest magnitude of one sign). The result
// keeps the sign in bit 31 and the 15 field bits in 12..26.
__device__ __forceinline__ unsigned f16c_rounded(float x_scaled) {
    const int t = min(static_cast<int>(__float_as_uint(x_scaled) + 0x800u), 0x07ffffff);
    return min(static_cast<unsigned>(t), 0x87ffffffu);
}
__device__ __forceinline__ unsigned f16c_encode(float h) {
    const unsigned r = f16c_rounded(__fmul_rn(h, 0x1p-112f));
    return ((r >> 12) & 0x7fffu) | ((r >> 16) & 0x8000u);
}
// two values to one 32-bit word (.x in the low half): one packed scaling, one byte permute
__device__ __forceinline__ unsigned f16c_encode2(float2 v) {
    const float2 x = __fmul2_rn(v, make_float2(0x1p-112f, 0x1p-112f));
    const unsigned a = f16c_rounded(x.x), b = f16c_rounded(x.y);
    const unsigned lo = ((a >> 12) & 0x7fffu) | ((a >> 16) & 0x8000u);
    const unsigned hi = ((b << 4) & 0x7fff0000u) | (b & 0x80000000u);  // only bytes 2, 3 are taken
    return __byte_perm(lo, hi, 0x7610);
}

template <int S>
struct Codec;

template <>
struct Codec<STORE_F32> {
    using T = float;
    __device__ static __forceinline__ float load(const T* p, float) { return __ldg(p); }
    __device__ static __forceinline__ float load_plain(const T* p, float) { return *p; }
    __device__ static __forceinline__ void store(T* p, float v, float) { *p = v; }
    // evict-first store for the step output: it is read again only in the next step
    __device__ static __forceinline__ void store_stream(T* p, float v, float) { __stcs(p, v); }
    __host__ __device__ static float decode(T v, float) { return v; }
};

template <>
struct Codec<STORE_F16> {
    using T = __half;
    __device__ static __forceinline__ float load(const T* p, float w) {
        return fmaf(w, __half2float(__ldg(p)), w);
    }
    __device__ static __forceinline__ float load_plain(const T* p, float w) { return fmaf(w, __half2float(*p), w); }
    __device__ static __forceinline__ void store(T* p, float v, float w) {
        *p = __float2half_rn(fmaf(v, 1.0f / w, -1.0f));
    }
    __device__ static __forceinline__ void store_stream(T* p, float v, float w) {
        __stcs(reinterpret_cast<unsigned short*>(p), __half_as_ushort(__float2half_rn(fmaf(v, 1.0f / w, -1.0f))));
    }
};

template <>
struct Codec<STORE_F16C> {
    using T = f16c_t;
    __device__ static __forceinline__ float load(const T* p, float w) {
        return fmaf(w, f16c_decode(__ldg(reinterpret_cast<const unsigned short*>(p))), w);
    }
    __device__ static __forceinline__ float load_plain(const T* p, float w) { return fmaf(w, f16c_decode(p->bits), w); }
    __device__ static __forceinline__ void store(T* p, float v, float w) {
        p->bits = static_cast<unsigned short>(f16c_encode(fmaf(v, 1.0f / w, -1.0f)));
    }
    __device__ static __forceinline__ void store_stream(T* p, float v, float w) {
        __stcs(reinterpret_cast<unsigned short*>(p),
               static_cast<unsigned short>(f16c_encode(fmaf(v, 1.0f / w, -1.0f))));
    }
};

template <>
struct Codec<STORE_BF16> {
    using T = __nv_bfloat16;
    __device__ static __forceinline__ float load(const T* p, float w) {
        return fmaf(w, __bfloat162float(__ldg(p)), w);
    }
    __device__ static __forceinline__ float load_plain(const T* p, float w) {
        return fmaf(w, __bfloat162float(*p), w);
    }
    __device__ static __forceinline__ void store(T* p, float v, float w) {
        *p = __float2bfloat16_rn(fmaf(v, 1.0f / w, -1.0f));
    }
    __device__ static __forceinline__ void store_stream(T* p, float v, float w) {
        __stcs(reinterpret_cast<unsigned short*>(p),
               __bfloat16_as_ushort(__float2bfloat16_rn(fmaf(v, 1.0f / w, -1.0f))));
    }
};

// ---------------------------------------------------------------- node physics
enum { COLL_BGK = 0, COLL_TRT = 1, COLL_MRT = 2 };

struct Physics {
    float tau;          // BGK tau / TRT tau_s / MRT tau_shear (before LES)
    float lambda_trt;   // TRT magic parameter (reference uses 1/4, lattice_grid_2d.cpp:221)
    float tau_bulk;     // MRT bulk relaxation (reference: 1.63 in 2D, 1.19 in 3D)
    float cs_smag;      // Smagorinsky constant
    float g[3];         // body force
    float s3, s4;       // D3Q27 MRT third- and higher-order rates
    int mrt_exact;      // D3Q19 MRT: 0 reference 7-digit inverse, 1 exact inverse
};

template <int Q>
__device__ __forceinline__ float feq(int q, float rho, float ux, float uy, float uz, float u2) {
    using L = Lat<Q>;
    const float cu = float(L::cx(q)) * ux + float(L::cy(q)) * uy + float(L::cz(q)) * uz;
    return L::w(q) * rho * (1.0f + 3.0f * cu + 4.5f * cu * cu - 1.5f * u2);
}

// Density, Guo-shifted velocity (d2q9_collision_bgk.ispc:37-51).
template <int Q>
__device__ __forceinline__ void node_moments(const float* f, const float g[3], float& rho, float u[3]) {
    using L = Lat<Q>;
    float r = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        r += f[q];
        if (L::cx(q)) jx += L::cx(q) > 0 ? f[q] : -f[q];
        if (L::cy(q)) jy += L::cy(q) > 0 ? f[q] : -f[q];
        if (L::cz(q)) jz += L::cz(q) > 0 ? f[q] : -f[q];
    }
    rho = r;
    const float inv = 1.0f / r;
    u[0] = (jx + 0.5f * r * g[0]) * inv;
    u[1] = (jy + 0.5f * r * g[1]) * inv;
    u[2] = (jz + 0.5f * r * g[2]) * inv;
}

// Smagorinsky tau from the local non-equilibrium stress (d2q9_les.ispc:19-55,
// d3q19_les.ispc:21-64), applied per node.
__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// tau_eff = (tau0 + sqrt(tau0^2 + 18 sqrt(2) Cs^2 sqrt(2 Pi:Pi) / rho)) / 2
// (d3q19_les.ispc:49-55 form). The approximate square root and division (a few
// ulp) cost a fraction of the exact sequences and perturb tau by ~1e-7. Every
// rounding is explicit, so the bits do not depend on which products of the
// loop-invariant tau0 / Cs the compiler hoists out of a kernel's node loop: a
// lattice gets the same tau_eff from every kernel that inlines this.
__device__ __forceinline__ float smagorinsky_tau_eff(float tau0, float cs, float rho, float sum) {
    const float qs = sqrt_approx(__fmul_rn(2.0f, sum));
    const float pref = __fmul_rn(__fmul_rn(18.0f * 1.4142135623730951f, cs), cs);
    const float t2 = __fmul_rn(tau0, tau0);
    return __fmul_rn(0.5f, __fadd_rn(tau0, sqrt_approx(__fmaf_rn(__fdividef(pref, rho), qs, t2))));
}

// TRT antisymmetric rate for a per-node tau (Lambda = (tau_s - 1/2)(tau_a - 1/2)),
// rounding explicit for the same reason.
__device__ __forceinline__ float trt_tau_a(float lambda, float tau) {
    return __fadd_rn(0.5f, __fdividef(lambda, fmaxf(1e-4f, __fsub_rn(tau, 0.5f))));
}

// Because c_opp = -c, the second-order tensor only sees the even part of each
// (q, opp) pair: Pi = sum over pairs c c^T (f_q + f_opp - 2 w rho (1 + 4.5 (c.u)^2 - 1.5 u^2)).
// The same even parts feed the TRT update, so the compiler shares them.
template <int Q>
__device__ __forceinline__ float smagorinsky_tau(const float* f, float rho, const float u[3], float tau0, float cs) {
    using L = Lat<Q>;
    const float u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    float pxx = 0.f, pyy = 0.f, pzz = 0.f, pxy = 0.f, pyz = 0.f, pxz = 0.f;
#pragma unroll
    for (int q = 1; q < Q; ++q) {
        const int o = L::opp(q);
        if (o < q) continue;
        const float cu = float(L::cx(q)) * u[0] + float(L::cy(q)) * u[1] + float(L::cz(q)) * u[2];
        const float base = L::w(q) * rho * (1.0f + 4.5f * cu * cu - 1.5f * u2);
        const float fn = (f[q] + f[o]) - 2.0f * base;
        const int x = L::cx(q), y = L::cy(q), z = L::cz(q);
        if (x) pxx += fn;
        if (y) pyy += fn;
        if (z) pzz += fn;
        if (x && y) pxy += (x * y > 0) ? fn : -fn;
        if (y && z) pyz += (y * z > 0) ? fn : -fn;
        if (x && z) pxz += (x * z > 0) ? fn : -fn;
    }
    const float sum = pxx * pxx + pyy * pyy + pzz * pzz + 2.0f * (pxy * pxy + pyz * pyz + pxz * pxz);
    return smagorinsky_tau_eff(tau0, cs, rho, sum);
}

template <int Q>
__device__ __forceinline__ void collide_bgk(float* f, float rho, const float u[3], const float g[3], float tau) {
    using L = Lat<Q>;
    const float om = 1.0f / tau, pre = 1.0f - 0.5f * om;
    const float u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const float ug = u[0] * g[0] + u[1] * g[1] + u[2] * g[2];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const float cu = float(L::cx(q)) * u[0] + float(L::cy(q)) * u[1] + float(L::cz(q)) * u[2];
        const float cg = float(L::cx(q)) * g[0] + float(L::cy(q)) * g[1] + float(L::cz(q)) * g[2];
        const float fi = pre * L::w(q) * rho * (3.0f * (cg - ug) + 9.0f * cu * cg);
        f[q] = f[q] - om * (f[q] - feq<Q>(q, rho, u[0], u[1], u[2], u2)) + fi;
    }
}

template <int Q>
__device__ __forceinline__ void collide_trt_t(float* f, float rho, const float u[3], const float g[3], float os,
                                              float oa, bool forced) {
    using L = Lat<Q>;
    const float ps = 1.0f - 0.5f * os, pa = 1.0f - 0.5f * oa;
    const float u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const float ug = forced ? u[0] * g[0] + u[1] * g[1] + u[2] * g[2] : 0.0f;
    // rest population: symmetric only
    {
        const float fe = feq<Q>(0, rho, u[0], u[1], u[2], u2);
        f[0] = f[0] - os * (f[0] - fe);
        if (forced) f[0] += ps * L::w(0) * rho * (-3.0f * ug);
    }
#pragma unroll
    for (int q = 1; q < Q; ++q) {
        const int o = L::opp(q);
        if (o < q) continue;  // handle each (q, opp) pair once
        const float cu = float(L::cx(q)) * u[0] + float(L::cy(q)) * u[1] + float(L::cz(q)) * u[2];
        const float base = L::w(q) * rho * (1.0f + 4.5f * cu * cu - 1.5f * u2);  // even part of feq
        const float odd = L::w(q) * rho * 3.0f * cu;                             // odd part of feq
        const float fs = 0.5f * (f[q] + f[o]), fa = 0.5f * (f[q] - f[o]);
        float ds = os * (fs - base);
        float da = oa * (fa - odd);
        if (forced) {
            const float cg = float(L::cx(q)) * g[0] + float(L::cy(q)) * g[1] + float(L::cz(q)) * g[2];
            ds -= ps * L::w(q) * rho * (-3.0f * ug + 9.0f * cu * cg);
            da -= pa * L::w(q) * rho * (3.0f * cg);
        }
        f[q] = f[q] - ds - da;
        f[o] = f[o] - ds + da;
    }
}

// Index of the direction that starts pair p (the member whose opposite is larger).
template <int Q>
__host__ __device__ constexpr int pair_q(int p) {
    int seen = 0;
    for (int q = 1; q < Q; ++q) {
        if (Lat<Q>::opp(q) < q) continue;
        if (seen == p) return q;
        ++seen;
    }
    return 0;
}

// Moments, Smagorinsky tau (LES) and TRT relaxation in one pass over the pair
// sums s = f_q + f_opp and differences d = f_q - f_opp, which all three share:
// rho = f_0 + sum s, j = sum c d, Pi = sum c c^T (s - 2 even(feq)), and the TRT
// update relaxes s/2 to the even and d/2 to the odd part of feq. Writes the
// post-collision populations back into f and the (Guo-shifted) moments.
template <int Q, bool LES>
__device__ __forceinline__ void trt_pairs(float* f, const Physics& P, float& rho, float u[3]) {
    using L = Lat<Q>;
    constexpr int NP = (Q - 1) / 2;
    float s[NP], d[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        const int q = pair_q<Q>(p), o = L::opp(q);
        s[p] = f[q] + f[o];
        d[p] = f[q] - f[o];
    }
    float r = f[0], jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        const int q = pair_q<Q>(p);
        r += s[p];
        if (L::cx(q)) jx += L::cx(q) > 0 ? d[p] : -d[p];
        if (L::cy(q)) jy += L::cy(q) > 0 ? d[p] : -d[p];
        if (L::cz(q)) jz += L::cz(q) > 0 ? d[p] : -d[p];
    }
    rho = r;
    const float inv = 1.0f / r;
    const float* g = P.g;
    u[0] = (jx + 0.5f * r * g[0]) * inv;
    u[1] = (jy + 0.5f * r * g[1]) * inv;
    u[2] = (jz + 0.5f * r * g[2]) * inv;
    const float u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const float a0 = 1.0f - 1.5f * u2;
    float os, oa;
    if (LES) {
        float pxx = 0.f, pyy = 0.f, pzz = 0.f, pxy = 0.f, pyz = 0.f, pxz = 0.f;
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const int q = pair_q<Q>(p);
            const int x = L::cx(q), y = L::cy(q), z = L::cz(q);
            const float cu = float(x) * u[0] + float(y) * u[1] + float(z) * u[2];
            const float fn = s[p] - 2.0f * (L::w(q) * r * (a0 + 4.5f * cu * cu));
            if (x) pxx += fn;
            if (y) pyy += fn;
            if (z) pzz += fn;
            if (x && y) pxy += (x * y > 0) ? fn : -fn;
            if (y && z) pyz += (y * z > 0) ? fn : -fn;
            if (x && z) pxz += (x * z > 0) ? fn : -fn;
        }
        const float sum = pxx * pxx + pyy * pyy + pzz * pzz + 2.0f * (pxy * pxy + pyz * pyz + pxz * pxz);
        const float tau = smagorinsky_tau_eff(P.tau, P.cs_smag, r, sum);
        os = __fdividef(1.0f, tau);
        oa = __fdividef(1.0f, trt_tau_a(P.lambda_trt, tau));
    } else {
        const float tau_a = 0.5f + P.lambda_trt / fmaxf(1e-4f, P.tau - 0.5f);
        os = 1.0f / P.tau;
        oa = 1.0f / tau_a;
    }
    const bool forced = (g[0] != 0.0f) || (g[1] != 0.0f) || (g[2] != 0.0f);
    const float ps = 1.0f - 0.5f * os, pa = 1.0f - 0.5f * oa;
    const float ug = u[0] * g[0] + u[1] * g[1] + u[2] * g[2];
    f[0] = f[0] - os * (f[0] - L::w(0) * r * a0);
    if (forced) f[0] += ps * L::w(0) * r * (-3.0f * ug);
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        const int q = pair_q<Q>(p), o = L::opp(q);
        const float cu = float(L::cx(q)) * u[0] + float(L::cy(q)) * u[1] + float(L::cz(q)) * u[2];
        const float wr = L::w(q) * r;
        float ds = os * (0.5f * s[p] - wr * (a0 + 4.5f * cu * cu));
        float da = oa * (0.5f * d[p] - 3.0f * wr * cu);
        if (forced) {
            const float cg = float(L::cx(q)) * g[0] + float(L::cy(q)) * g[1] + float(L::cz(q)) * g[2];
            ds -= ps * wr * (-3.0f * ug + 9.0f * cu * cg);
            da -= pa * wr * (3.0f * cg);
        }
        // f_q = (s + d)/2 - ds - da, f_opp = (s - d)/2 - ds + da
        const float hs = 0.5f * s[p] - ds, hd = 0.5f * d[p] - da;
        f[q] = hs + hd;
        f[o] = hs - hd;
    }
}

// Body-force terms only when a force is set: the unforced form saves the
// per-pair force arithmetic in the common case (uniform branch).
template <int Q>
__device__ __forceinline__ void collide_trt_omega(float* f, float rho, const float u[3], const float g[3], float os,
                                                  float oa) {
    if (g[0] != 0.0f || g[1] != 0.0f || g[2] != 0.0f) collide_trt_t<Q>(f, rho, u, g, os, oa, true);
    else collide_trt_t<Q>(f, rho, u, g, os, oa, false);
}

template <int Q>
__device__ __forceinline__ void collide_trt(float* f, float rho, const float u[3], const float g[3], float tau_s,
                                            float tau_a) {
    collide_trt_omega<Q>(f, rho, u, g, 1.0f / tau_s, 1.0f / tau_a);
}

// The reference's D3Q27 "opposite" table (include/wake/ispc/lbm_d3q27.isph:35-40):
// equal to the true opposite except that corner q pairs with its (x, y) mirror.
__host__ __device__ constexpr int ref_opp_d3q27(int q) {
    constexpr int t[27] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15,
                           22, 21, 20, 19, 26, 25, 24, 23};
    return t[q];
}

// TRT exactly as d3q27_collision_mrt.ispc:60-88 computes it, with the
// reference's pairing table: symmetric / antisymmetric parts of f and feq taken
// against ref_opp_d3q27(q). Used only by the drop-in d3q27_collide entry point.
__device__ __forceinline__ void collide_trt_d3q27_reference(float* f, float rho, const float u[3], const float g[3],
                                                            float tau_s, float tau_a) {
    using L = Lat<27>;
    const float os = 1.0f / tau_s, oa = 1.0f / tau_a;
    const float ps = 1.0f - 0.5f * os, pa = 1.0f - 0.5f * oa;
    const float u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const float ug = u[0] * g[0] + u[1] * g[1] + u[2] * g[2];
    float fe[27], in[27];
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        fe[q] = feq<27>(q, rho, u[0], u[1], u[2], u2);
        in[q] = f[q];
    }
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const int o = ref_opp_d3q27(q);
        const float fs = 0.5f * (in[q] + in[o]), fa = 0.5f * (in[q] - in[o]);
        const float es = 0.5f * (fe[q] + fe[o]), ea = 0.5f * (fe[q] - fe[o]);
        const float cu = float(L::cx(q)) * u[0] + float(L::cy(q)) * u[1] + float(L::cz(q)) * u[2];
        const float cg = float(L::cx(q)) * g[0] + float(L::cy(q)) * g[1] + float(L::cz(q)) * g[2];
        const float Fa = pa * L::w(q) * rho * (3.0f * cg);
        const float Fs = ps * L::w(q) * rho * (-3.0f * ug + 9.0f * cu * cg);
        f[q] = in[q] - os * (fs - es) - oa * (fa - ea) + Fs + Fa;
    }
}

// D2Q9 Lallemand-Luo MRT with moment-space Guo forcing (d2q9_collision_mrt.ispc:43-136).
__device__ __forceinline__ void collide_mrt_d2q9(float* f, float rho, const float u[3], const float g[3],
                                                 float tau_shear, float tau_bulk) {
    const float s_e = 1.0f / tau_bulk, s_eps = 1.4f, s_q = 1.6f, s_p = 1.0f / tau_shear;
    const float fc = f[1] + f[2] + f[3] + f[4], fd = f[5] + f[6] + f[7] + f[8];
    const float ex = f[1] - f[3], dx = f[5] - f[6] - f[7] + f[8];
    const float ey = f[2] - f[4], dy = f[5] + f[6] - f[7] - f[8];
    float m1 = -4.0f * f[0] - fc + 2.0f * fd;
    float m2 = 4.0f * f[0] - 2.0f * fc + fd;
    float m3 = ex + dx;
    float m4 = -2.0f * ex + dx;
    float m5 = ey + dy;
    float m6 = -2.0f * ey + dy;
    float m7 = f[1] - f[2] + f[3] - f[4];
    float m8 = f[5] - f[6] + f[7] - f[8];
    const float m0 = rho;
    const float ux = u[0], uy = u[1], ux2 = ux * ux, uy2 = uy * uy, u2 = ux2 + uy2;
    const float pre = 1.0f - 0.5f * s_p;
    const float F3 = rho * g[0], F5 = rho * g[1];
    const float uF = ux * F3 + uy * F5;
    m1 = m1 - s_e * (m1 - rho * (-2.0f + 3.0f * u2)) + pre * (6.0f * uF);
    m2 = m2 - s_eps * (m2 - rho * (1.0f - 3.0f * u2)) + pre * (-6.0f * uF);
    m3 = m3 + F3;
    m4 = m4 - s_q * (m4 + rho * ux) + pre * (-F3);
    m5 = m5 + F5;
    m6 = m6 - s_q * (m6 + rho * uy) + pre * (-F5);
    m7 = m7 - s_p * (m7 - rho * (ux2 - uy2)) + pre * (2.0f * (ux * F3 - uy * F5));
    m8 = m8 - s_p * (m8 - rho * ux * uy) + pre * (ux * F5 + uy * F3);
    const float a0 = m0 * (1.0f / 9.0f);
    const float ac = a0 - m1 * (1.0f / 36.0f) - m2 * (1.0f / 18.0f);
    const float ad = a0 + m1 * (1.0f / 18.0f) + m2 * (1.0f / 36.0f);
    const float jx = m3 * (1.0f / 6.0f), qx = m4 * (1.0f / 6.0f), qx2 = m4 * (1.0f / 12.0f);
    const float jy = m5 * (1.0f / 6.0f), qy = m6 * (1.0f / 6.0f), qy2 = m6 * (1.0f / 12.0f);
    f[0] = a0 - m1 * (1.0f / 9.0f) + m2 * (1.0f / 9.0f);
    f[1] = ac + jx - qx + 0.25f * m7;
    f[2] = ac + jy - qy - 0.25f * m7;
    f[3] = ac - jx + qx + 0.25f * m7;
    f[4] = ac - jy + qy - 0.25f * m7;
    f[5] = ad + jx + qx2 + jy + qy2 + 0.25f * m8;
    f[6] = ad - jx - qx2 + jy + qy2 - 0.25f * m8;
    f[7] = ad - jx - qx2 - jy - qy2 + 0.25f * m8;
    f[8] = ad + jx + qx2 - jy - qy2 - 0.25f * m8;
}

// D3Q19 d'Humieres basis as polynomials of c (d3q19_collision_mrt.ispc:60-103).
__host__ __device__ constexpr double d3q19_basis(int k, int q) {
    const double x = Lat<19>::cx(q), y = Lat<19>::cy(q), z = Lat<19>::cz(q);
    const double c2 = x * x + y * y + z * z;
    switch (k) {
        case 0: return 1.0;
        case 1: return 19.0 * c2 - 30.0;
        case 2: return (21.0 * c2 * c2 - 53.0 * c2 + 24.0) * 0.5;
        case 3: return x;
        case 4: return (5.0 * c2 - 9.0) * x;
        case 5: return y;
        case 6: return (5.0 * c2 - 9.0) * y;
        case 7: return z;
        case 8: return (5.0 * c2 - 9.0) * z;
        case 9: return 3.0 * x * x - c2;
        case 10: return (3.0 * c2 - 5.0) * (3.0 * x * x - c2);
        case 11: return y * y - z * z;
        case 12: return (3.0 * c2 - 5.0) * (y * y - z * z);
        case 13: return x * y;
        case 14: return y * z;
        case 15: return x * z;
        case 16: return (y * y - z * z) * x;
        case 17: return (z * z - x * x) * y;
        default: return (y * y - x * x) * z;
    }
}
__host__ __device__ constexpr double d3q19_norm(int k) {
    double n = 0.0;
    for (int q = 0; q < 19; ++q) n += d3q19_basis(k, q) * d3q19_basis(k, q);
    return n;
}
__host__ __device__ constexpr double round7(double v) {
    const double t = v * 1e7;
    const long long r = static_cast<long long>(t + (t >= 0.0 ? 0.5 : -0.5));
    return static_cast<double>(r) / 1e7;
}
// Inverse M^T diag(1/|M_k|^2); ROUNDED reproduces the reference's 7-decimal table
// (d3q19_collision_mrt.ispc:4-24), whose column sums are off by ~1e-7.
template <bool ROUNDED, int q, int k>
struct D3Q19Minv {
    static constexpr float v = static_cast<float>(ROUNDED ? round7(d3q19_basis(k, q) / d3q19_norm(k))
                                                          : d3q19_basis(k, q) / d3q19_norm(k));
};
template <int k, int q>
struct D3Q19M {
    static constexpr float v = static_cast<float>(d3q19_basis(k, q));
};

template <int k, int... q>
__device__ __forceinline__ float d3q19_row(const float* f, std::integer_sequence<int, q...>) {
    float a = 0.f;
    ((a = (D3Q19M<k, q>::v == 0.f) ? a : fmaf(D3Q19M<k, q>::v, f[q], a)), ...);
    return a;
}
template <int... k>
__device__ __forceinline__ void d3q19_forward(const float* f, float* m, std::integer_sequence<int, k...>) {
    ((m[k] = d3q19_row<k>(f, std::make_integer_sequence<int, 19>{})), ...);
}
template <bool R, int q, int... k>
__device__ __forceinline__ float d3q19_inv_row(const float* m, std::integer_sequence<int, k...>) {
    float a = 0.f;
    ((a = (D3Q19Minv<R, q, k>::v == 0.f) ? a : fmaf(D3Q19Minv<R, q, k>::v, m[k], a)), ...);
    return a;
}
template <bool R, int... q>
__device__ __forceinline__ void d3q19_inverse(float* f, const float* m, std::integer_sequence<int, q...>) {
    ((f[q] = d3q19_inv_row<R, q>(m, std::make_integer_sequence<int, 19>{})), ...);
}

__device__ __forceinline__ void collide_mrt_d3q19(float* f, float rho, const float u[3], const float g[3],
                                                  float tau_shear, float tau_bulk, int exact) {
    // rates d3q19_collision_mrt.ispc:41-48; equilibria :119-138; forcing on j and q :141-148
    const float sn = 1.0f / tau_shear;
    float m[19];
    d3q19_forward(f, m, std::make_integer_sequence<int, 19>{});
    m[0] = rho;
    const float ux = u[0], uy = u[1], uz = u[2];
    const float ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz, u2 = ux2 + uy2 + uz2;
    const float meq9 = rho * (2.0f * ux2 - uy2 - uz2), meq11 = rho * (uy2 - uz2);
    m[1] = m[1] - (1.0f / tau_bulk) * (m[1] - rho * (-11.0f + 19.0f * u2));
    m[2] = m[2] - 1.4f * (m[2] - rho * (3.0f - 5.5f * u2));
    m[3] = m[3] + rho * g[0];
    m[4] = m[4] - 1.2f * (m[4] + (2.0f / 3.0f) * rho * ux) - (2.0f / 3.0f) * rho * g[0];
    m[5] = m[5] + rho * g[1];
    m[6] = m[6] - 1.2f * (m[6] + (2.0f / 3.0f) * rho * uy) - (2.0f / 3.0f) * rho * g[1];
    m[7] = m[7] + rho * g[2];
    m[8] = m[8] - 1.2f * (m[8] + (2.0f / 3.0f) * rho * uz) - (2.0f / 3.0f) * rho * g[2];
    m[9] = m[9] - sn * (m[9] - meq9);
    m[10] = m[10] - 1.4f * (m[10] + 0.5f * meq9);
    m[11] = m[11] - sn * (m[11] - meq11);
    m[12] = m[12] - 1.4f * (m[12] + 0.5f * meq11);
    m[13] = m[13] - sn * (m[13] - rho * ux * uy);
    m[14] = m[14] - sn * (m[14] - rho * uy * uz);
    m[15] = m[15] - sn * (m[15] - rho * ux * uz);
    m[16] = m[16] - 1.98f * m[16];
    m[17] = m[17] - 1.98f * m[17];
    m[18] = m[18] - 1.98f * m[18];
    if (exact) d3q19_inverse<false>(f, m, std::make_integer_sequence<int, 19>{});
    else d3q19_inverse<true>(f, m, std::make_integer_sequence<int, 19>{});
}

// Runtime-indexed table lookups for the rare paths (a curved link carries its
// direction in memory): unrolled selects over compile-time constants.
template <int Q>
__device__ __forceinline__ void rt_dir(int q, int& cx, int& cy, int& cz, int& opp, float& w) {
    using L = Lat<Q>;
    cx = cy = cz = opp = 0;
    w = 0.f;
#pragma unroll
    for (int k = 0; k < Q; ++k)
        if (k == q) {
            cx = L::cx(k);
            cy = L::cy(k);
            cz = L::cz(k);
            opp = L::opp(k);
            w = L::w(k);
        }
}
__device__ __forceinline__ float rt_w19(int q) {
    float w = 0.f;
#pragma unroll
    for (int k = 0; k < 19; ++k)
        if (k == q) w = Lat<19>::w(k);
    return w;
}

// ---------------------------------------------------------------- D3Q27 raw-moment MRT
// Raw moments m_abc = sum_q cx^a cy^b cz^c f_q (a,b,c in {0,1,2}) factorise as a
// tensor product of the 1D map (v-, v0, v+) -> (v-+v0+v+, v+-v-, v++v-), so the
// 27x27 transform is three sweeps of nine 3-point transforms. The relaxation
// (no reference implementation): conserved moments unchanged, deviatoric
// second order at 1/tau, trace at 1/tau_bulk, third order at s3, higher at s4;
// Guo forcing enters as (I - S/2) M F.
__host__ __device__ constexpr int d3q27_slot(int q) {  // q -> (cx+1) + 3 (cy+1) + 9 (cz+1)
    return (Lat<27>::cx(q) + 1) + 3 * (Lat<27>::cy(q) + 1) + 9 * (Lat<27>::cz(q) + 1);
}

__device__ __forceinline__ void raw_forward(float v[27]) {
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        const int st = axis == 0 ? 1 : (axis == 1 ? 3 : 9);
#pragma unroll
        for (int l = 0; l < 9; ++l) {
            // base index of line l along this axis
            const int o1 = axis == 0 ? 3 : 1, o2 = axis == 2 ? 3 : 9;
            const int base = (l % 3) * o1 + (l / 3) * o2;
            const float a = v[base], b = v[base + st], c = v[base + 2 * st];
            v[base] = a + b + c;
            v[base + st] = c - a;
            v[base + 2 * st] = c + a;
        }
    }
}

__device__ __forceinline__ void raw_inverse(float v[27]) {
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        const int st = axis == 0 ? 1 : (axis == 1 ? 3 : 9);
#pragma unroll
        for (int l = 0; l < 9; ++l) {
            const int o1 = axis == 0 ? 3 : 1, o2 = axis == 2 ? 3 : 9;
            const int base = (l % 3) * o1 + (l / 3) * o2;
            const float k0 = v[base], k1 = v[base + st], k2 = v[base + 2 * st];
            v[base] = 0.5f * (k2 - k1);
            v[base + st] = k0 - k2;
            v[base + 2 * st] = 0.5f * (k1 + k2);
        }
    }
}

// Moment index m = a + 3 b + 9 c after raw_forward (a,b,c the powers).
__device__ __forceinline__ void raw_relax(float m[27], float s_nu, float s_b, float s3, float s4) {
#pragma unroll
    for (int k = 0; k < 27; ++k) {
        const int a = k % 3, b = (k / 3) % 3, c = k / 9, o = a + b + c;
        if (o <= 1) m[k] = 0.f;
        else if (o == 2) {
            if (a == 2 || b == 2 || c == 2) continue;
            m[k] *= s_nu;
        } else if (o == 3) m[k] *= s3;
        else m[k] *= s4;
    }
    const float A = m[2] + m[6] + m[18], B = m[2] - m[6], C = m[2] - m[18];
    const float A2 = s_b * A, B2 = s_nu * B, C2 = s_nu * C;
    m[2] = (A2 + B2 + C2) * (1.0f / 3.0f);
    m[6] = (A2 - 2.0f * B2 + C2) * (1.0f / 3.0f);
    m[18] = (A2 + B2 - 2.0f * C2) * (1.0f / 3.0f);
}

__device__ __forceinline__ void collide_mrt_d3q27(float* f, float rho, const float u[3], const float g[3],
                                                  float tau, float tau_bulk, float s3, float s4) {
    const float u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const float s_nu = 1.0f / tau, s_b = 1.0f / tau_bulk;
    float d[27];
#pragma unroll
    for (int q = 0; q < 27; ++q) d[d3q27_slot(q)] = f[q] - feq<27>(q, rho, u[0], u[1], u[2], u2);
    raw_forward(d);
    raw_relax(d, s_nu, s_b, s3, s4);
    const bool forced = (g[0] != 0.f) || (g[1] != 0.f) || (g[2] != 0.f);
    if (forced) {
        const float ug = u[0] * g[0] + u[1] * g[1] + u[2] * g[2];
        float F[27];
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            using L = Lat<27>;
            const float cu = float(L::cx(q)) * u[0] + float(L::cy(q)) * u[1] + float(L::cz(q)) * u[2];
            const float cg = float(L::cx(q)) * g[0] + float(L::cy(q)) * g[1] + float(L::cz(q)) * g[2];
            F[d3q27_slot(q)] = L::w(q) * rho * (3.0f * (cg - ug) + 9.0f * cu * cg);
        }
        raw_forward(F);
        // (I - S/2): conserved rows keep F, others scale by 1 - s/2
        float h[27];
#pragma unroll
        for (int k = 0; k < 27; ++k) h[k] = F[k];
        raw_relax(h, s_nu, s_b, s3, s4);  // h = S F
#pragma unroll
        for (int k = 0; k < 27; ++k) d[k] = d[k] - (F[k] - 0.5f * h[k]);
    }
    raw_inverse(d);
#pragma unroll
    for (int q = 0; q < 27; ++q) f[q] -= d[d3q27_slot(q)];
}

// ---------------------------------------------------------------- dispatch
template <int Q, int COLL, bool LES>
__device__ __forceinline__ void collide(float* f, float rho, const float u[3], const Physics& P) {
    float tau = P.tau;
    if (LES) tau = smagorinsky_tau<Q>(f, rho, u, P.tau, P.cs_smag);
    if (COLL == COLL_BGK) {
        collide_bgk<Q>(f, rho, u, P.g, tau);
    } else if (COLL == COLL_TRT) {
        // tau_a from the magic parameter (lattice_grid_2d.cpp:219-222)
        if (LES) {
            // per-node rates: approximate divisions (see smagorinsky_tau)
            collide_trt_omega<Q>(f, rho, u, P.g, __fdividef(1.0f, tau), __fdividef(1.0f, trt_tau_a(P.lambda_trt, tau)));
        } else {
            const float tau_a = 0.5f + P.lambda_trt / fmaxf(1e-4f, tau - 0.5f);
            collide_trt<Q>(f, rho, u, P.g, tau, tau_a);
        }
    } else {
        if constexpr (Q == 9) collide_mrt_d2q9(f, rho, u, P.g, tau, P.tau_bulk);
        else if constexpr (Q == 19) collide_mrt_d3q19(f, rho, u, P.g, tau, P.tau_bulk, P.mrt_exact);
        else collide_mrt_d3q27(f, rho, u, P.g, tau, P.tau_bulk, P.s3, P.s4);
    }
}

// ---------------------------------------------------------------- Zou-He
// 2D: d2q9_boundaries.ispc:43-121. 3D: Hecht & Harting (2010) on-site velocity
// inlet / pressure outlet for D3Q19 (no reference implementation).
template <int Q>
__device__ __forceinline__ void zou_he_inlet(float* f, const float uin[3]) {
    if constexpr (Q == 9) {
        const float rho = (f[0] + f[2] + f[4] + 2.0f * (f[3] + f[6] + f[7])) / (1.0f - uin[0]);
        f[1] = f[3] + (2.0f / 3.0f) * rho * uin[0];
        f[5] = f[7] - 0.5f * (f[2] - f[4]) + (1.0f / 6.0f) * rho * uin[0] + 0.5f * rho * uin[1];
        f[8] = f[6] + 0.5f * (f[2] - f[4]) + (1.0f / 6.0f) * rho * uin[0] - 0.5f * rho * uin[1];
    } else if constexpr (Q == 19) {
        const float s0 = f[0] + f[3] + f[4] + f[5] + f[6] + f[15] + f[16] + f[17] + f[18];
        const float sm = f[2] + f[8] + f[10] + f[12] + f[14];
        const float rho = (s0 + 2.0f * sm) / (1.0f - uin[0]);
        const float Ny = 0.5f * (f[3] + f[15] + f[17] - f[4] - f[16] - f[18]) - rho * uin[1] / 3.0f;
        const float Nz = 0.5f * (f[5] + f[15] + f[16] - f[6] - f[17] - f[18]) - rho * uin[2] / 3.0f;
        f[1] = f[2] + rho * uin[0] / 3.0f;
        f[7] = f[10] + rho * (uin[0] + uin[1]) / 6.0f - Ny;
        f[9] = f[8] + rho * (uin[0] - uin[1]) / 6.0f + Ny;
        f[11] = f[14] + rho * (uin[0] + uin[2]) / 6.0f - Nz;
        f[13] = f[12] + rho * (uin[0] - uin[2]) / 6.0f + Nz;
    }
}

template <int Q>
__device__ __forceinline__ void zou_he_outlet(float* f, float rho_out) {
    if constexpr (Q == 9) {
        const float ux = -1.0f + (f[0] + f[2] + f[4] + 2.0f * (f[1] + f[5] + f[8])) / rho_out;
        f[3] = f[1] - (2.0f / 3.0f) * rho_out * ux;
        f[6] = f[8] - 0.5f * (f[2] - f[4]) - (1.0f / 6.0f) * rho_out * ux;
        f[7] = f[5] + 0.5f * (f[2] - f[4]) - (1.0f / 6.0f) * rho_out * ux;
    } else if constexpr (Q == 19) {
        const float s0 = f[0] + f[3] + f[4] + f[5] + f[6] + f[15] + f[16] + f[17] + f[18];
        const float sp = f[1] + f[7] + f[9] + f[11] + f[13];
        const float ux = -1.0f + (s0 + 2.0f * sp) / rho_out;
        const float Ny = 0.5f * (f[3] + f[15] + f[17] - f[4] - f[16] - f[18]);
        const float Nz = 0.5f * (f[5] + f[15] + f[16] - f[6] - f[17] - f[18]);
        f[2] = f[1] - rho_out * ux / 3.0f;
        f[10] = f[7] - rho_out * ux / 6.0f + Ny;
        f[8] = f[9] - rho_out * ux / 6.0f - Ny;
        f[14] = f[11] - rho_out * ux / 6.0f + Nz;
        f[12] = f[13] - rho_out * ux / 6.0f - Nz;
    }
}

}  // namespace wk
