// TRT (+ Smagorinsky) for two nodes at once in packed FP32.
//
// sm_100 executes add / mul / fma on a pair of FP32 values as one instruction
// (PTX add/mul/fma .f32x2, CUDA __fadd2_rn / __fmul2_rn / __ffma2_rn), so a
// thread that carries two nodes in the two halves of float2 registers issues
// half the arithmetic of the one-node form. The algebra is the pair form of
// trt_pairs (lattice.cuh): pair sums s = f_q + f_opp and differences
// d = f_q - f_opp, rho = f_0 + sum s, j = sum c d, LES stress from
// s - s_eq, and the update
//     f_q'   = f_q   - omega_s/2 (s - s_eq) - omega_a/2 (d - d_eq)
//     f_opp' = f_opp - omega_s/2 (s - s_eq) + omega_a/2 (d - d_eq)
// with s_eq = 2 w rho (1 - 1.5 u^2 + 4.5 (c.u)^2) and d_eq = 6 w rho (c.u).
//
// HS = true works on shifted populations h = f / w - 1 (the FP16 / BF16
// storage format) directly: with S = h_q + h_opp, D = h_q - h_opp,
//     rho = 1 + w_0 h_0 + sum w S,   j = sum c w D,
//     S_eq = 2 rho (1 - 1.5 u^2 + 4.5 (c.u)^2) - 2,   D_eq = 6 rho (c.u),
// and the same update in h, so stored values are used without decoding.
// Every rounding is explicit (packed ops are never contracted by the compiler).
#pragma once

#include "lattice.cuh"

namespace wk {

__device__ __forceinline__ float2 bc2(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// acc + c v (f-space) or acc + c w v (h-space) for a lattice component c in {-1, 0, 1};
// the branches fold away once the pair loop is unrolled
__device__ __forceinline__ float2 acc_c(float2 acc, int c, float2 v) {
    return c > 0 ? add2(acc, v) : (c < 0 ? sub2(acc, v) : acc);
}
__device__ __forceinline__ float2 acc_cw(float2 acc, int c, float w, float2 v) {
    return c > 0 ? fma2(bc2(w), v, acc) : (c < 0 ? fma2(bc2(-w), v, acc) : acc);
}
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

template <int Q, bool LES, bool HS>
__device__ __forceinline__ void trt_pairs2(float2* f, const Physics& P, float2& rho, float2 u[3]) {
    using L = Lat<Q>;
    constexpr int NP = (Q - 1) / 2;
    float2 s[NP], d[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        const int q = pair_q<Q>(p), o = L::opp(q);
        s[p] = add2(f[q], f[o]);
        d[p] = sub2(f[q], f[o]);
    }
    float2 r, jx = bc2(0.f), jy = bc2(0.f), jz = bc2(0.f);
    if constexpr (HS) {
        r = fma2(bc2(L::w(0)), f[0], bc2(1.0f));
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const int q = pair_q<Q>(p);
            r = fma2(bc2(L::w(q)), s[p], r);
            jx = acc_cw(jx, L::cx(q), L::w(q), d[p]);
            jy = acc_cw(jy, L::cy(q), L::w(q), d[p]);
            jz = acc_cw(jz, L::cz(q), L::w(q), d[p]);
        }
    } else {
        r = f[0];
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const int q = pair_q<Q>(p);
            r = add2(r, s[p]);
            jx = acc_c(jx, L::cx(q), d[p]);
            jy = acc_c(jy, L::cy(q), d[p]);
            jz = acc_c(jz, L::cz(q), d[p]);
        }
    }
    rho = r;
    const float2 inv = make_float2(__fdividef(1.0f, r.x), __fdividef(1.0f, r.y));
    const float* g = P.g;
    const bool forced = (g[0] != 0.0f) || (g[1] != 0.0f) || (g[2] != 0.0f);
    const float2 hr = mul2(bc2(0.5f), r);
    u[0] = mul2(forced ? fma2(hr, bc2(g[0]), jx) : jx, inv);
    u[1] = mul2(forced ? fma2(hr, bc2(g[1]), jy) : jy, inv);
    u[2] = mul2(forced ? fma2(hr, bc2(g[2]), jz) : jz, inv);
    const float2 u2 = fma2(u[2], u[2], fma2(u[1], u[1], mul2(u[0], u[0])));
    const float2 a0 = fma2(bc2(-1.5f), u2, bc2(1.0f));
    // per pair: c.u and the non-equilibrium parts nS = s - s_eq, nD = d - d_eq, with the even
    // equilibrium written s_eq = (9 w rho (c.u)) (c.u) + 2 w rho a0 (h-space: w = 1 and - 2)
    float2 nS[NP], nD[NP];
    const float2 rm6 = mul2(bc2(-6.0f), r);
    const float2 e0h = fma2(add2(r, r), a0, bc2(-2.0f)), r9 = mul2(bc2(9.0f), r);  // h-space
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        const int q = pair_q<Q>(p);
        // c.u from the nonzero components (no multiplications by +-1)
        const int cx = L::cx(q), cy = L::cy(q), cz = L::cz(q);
        float2 cu = cx ? (cx > 0 ? u[0] : neg2(u[0])) : bc2(0.f);
        if (cy) cu = cx ? acc_c(cu, cy, u[1]) : (cy > 0 ? u[1] : neg2(u[1]));
        if (cz) cu = (cx || cy) ? acc_c(cu, cz, u[2]) : (cz > 0 ? u[2] : neg2(u[2]));
        if constexpr (HS) {
            nS[p] = sub2(s[p], fma2(mul2(r9, cu), cu, e0h));
            nD[p] = fma2(rm6, cu, d[p]);
        } else {
            // the weight-class products (2 w rho a0, 9 w rho, -6 w rho) are shared by the pairs of a class
            const float w = L::w(q);
            const float2 e0w = mul2(mul2(bc2(2.0f * w), r), a0);
            nS[p] = sub2(s[p], fma2(mul2(mul2(bc2(9.0f * w), r), cu), cu, e0w));
            nD[p] = fma2(mul2(bc2(-6.0f * w), r), cu, d[p]);
        }
    }
    float2 hs, ha;  // omega_s / 2, omega_a / 2 per node
    if constexpr (LES) {
        float2 pxx = bc2(0.f), pyy = bc2(0.f), pzz = bc2(0.f), pxy = bc2(0.f), pyz = bc2(0.f), pxz = bc2(0.f);
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const int q = pair_q<Q>(p);
            const int x = L::cx(q), y = L::cy(q), z = L::cz(q);
            // f-space stress contribution s - s_eq (h-space: w (S - S_eq))
            const float wq = HS ? L::w(q) : 1.0f;
            if (x) pxx = fma2(bc2(wq), nS[p], pxx);
            if (y) pyy = fma2(bc2(wq), nS[p], pyy);
            if (z) pzz = fma2(bc2(wq), nS[p], pzz);
            if (x && y) pxy = fma2(bc2(x * y > 0 ? wq : -wq), nS[p], pxy);
            if (y && z) pyz = fma2(bc2(y * z > 0 ? wq : -wq), nS[p], pyz);
            if (x && z) pxz = fma2(bc2(x * z > 0 ? wq : -wq), nS[p], pxz);
        }
        const float2 off = fma2(pxz, pxz, fma2(pyz, pyz, mul2(pxy, pxy)));
        const float2 sum = fma2(bc2(2.0f), off, fma2(pzz, pzz, fma2(pyy, pyy, mul2(pxx, pxx))));
        const float tx = smagorinsky_tau_eff(P.tau, P.cs_smag, r.x, sum.x);
        const float ty = smagorinsky_tau_eff(P.tau, P.cs_smag, r.y, sum.y);
        hs = make_float2(__fdividef(0.5f, tx), __fdividef(0.5f, ty));
        ha = make_float2(__fdividef(0.5f, trt_tau_a(P.lambda_trt, tx)), __fdividef(0.5f, trt_tau_a(P.lambda_trt, ty)));
    } else {
        const float tau_a = 0.5f + P.lambda_trt / fmaxf(1e-4f, P.tau - 0.5f);
        hs = bc2(0.5f / P.tau);
        ha = bc2(0.5f / tau_a);
    }
    // rest population: relaxes to w_0 rho a0 (h-space: rho a0 - 1)
    const float2 e0 = HS ? fma2(r, a0, bc2(-1.0f)) : mul2(mul2(bc2(L::w(0)), r), a0);
    f[0] = fma2(mul2(bc2(-2.0f), hs), sub2(f[0], e0), f[0]);
    float2 ug;
    float2 ps, pa;
    if (forced) {
        ug = fma2(u[2], bc2(g[2]), fma2(u[1], bc2(g[1]), mul2(u[0], bc2(g[0]))));
        ps = fma2(bc2(-1.0f), hs, bc2(1.0f));  // 1 - omega_s / 2
        pa = fma2(bc2(-1.0f), ha, bc2(1.0f));
        // Guo term of the rest population: (1 - omega_s/2) w_0 rho (-3 u.g), h-space without w_0
        const float2 fr = HS ? r : mul2(bc2(L::w(0)), r);
        f[0] = fma2(mul2(ps, fr), mul2(bc2(-3.0f), ug), f[0]);
    }
    if (!forced) {
        // f_q' = f_q - hs nS - ha nD, f_opp' = f_opp - hs nS + ha nD, two fused steps each
        const float2 nhs = neg2(hs), nha = neg2(ha);
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const int q = pair_q<Q>(p), o = L::opp(q);
            f[q] = fma2(nhs, nS[p], fma2(nha, nD[p], f[q]));
            f[o] = fma2(nhs, nS[p], fma2(ha, nD[p], f[o]));
        }
        return;
    }
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        const int q = pair_q<Q>(p), o = L::opp(q);
        float2 A = mul2(hs, nS[p]), B = mul2(ha, nD[p]);
        {
            // Guo forcing of the pair (collide_trt_t in lattice.cuh): even part
            // (1 - omega_s/2) w rho (-3 u.g + 9 (c.u)(c.g)), odd part (1 - omega_a/2) w rho 3 (c.g)
            const float cg = float(L::cx(q)) * g[0] + float(L::cy(q)) * g[1] + float(L::cz(q)) * g[2];
            float2 cu = fma2(bc2(float(L::cz(q))), u[2], fma2(bc2(float(L::cy(q))), u[1], mul2(bc2(float(L::cx(q))), u[0])));
            const float2 fr = HS ? r : mul2(bc2(L::w(q)), r);
            const float2 ev = mul2(mul2(ps, fr), fma2(bc2(9.0f * cg), cu, mul2(bc2(-3.0f), ug)));
            const float2 od = mul2(mul2(pa, fr), bc2(3.0f * cg));
            A = sub2(A, ev);
            B = sub2(B, od);
        }
        const float2 fq = sub2(sub2(f[q], A), B);
        const float2 fo = add2(sub2(f[o], A), B);
        f[q] = fq;
        f[o] = fo;
    }
}

}  // namespace wk
