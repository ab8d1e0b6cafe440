// Field analytics on the device: 2D vorticity, 3D vorticity vector and
// Q-criterion from the macroscopic velocity (src/ispc/analytics_kernels.ispc:4-110),
// and the largest |value| of a field (src/analytics/field_analytics.cpp:56-62).
//
// The stencil is the reference's: central differences with periodic wrap on
// every axis. Every product and sum is rounded explicitly (__fmul_rn/__fadd_rn)
// in the reference's evaluation order, so no multiply-add is contracted and the
// results equal a plain IEEE float32 evaluation of the same expressions.
//
// Blocks are 32 x 8 tiles of an x-y plane, so the x and y neighbours of a tile are
// mostly read by the same block (L1). In 3D each thread marches along z through a
// chunk of ANALYTICS_ZC planes and keeps the z-1 / z / z+1 values of its column in
// registers, so DRAM sees each velocity component about once. Algorithmic traffic
// is 8 B in + 4 B out per node in 2D and 12 B in + 16 B out per node in 3D.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace wk {

__device__ __forceinline__ float half_diff(float a, float b) { return __fmul_rn(0.5f, __fsub_rn(a, b)); }

// z planes per chunk: 8 measured 12% faster than 32 on 256^3 fields (more blocks in flight).
#ifndef WK_ANALYTICS_ZC
#define WK_ANALYTICS_ZC 8
#endif
constexpr int ANALYTICS_TX = 32, ANALYTICS_TY = 8, ANALYTICS_ZC = WK_ANALYTICS_ZC;

// Grid of both stencils: x tiles in blockIdx.x, y tiles strided over blockIdx.y (any ny),
// z chunks of ANALYTICS_ZC planes in blockIdx.z (3D; 1 in 2D). Block 32 x 8.
static __global__ void __launch_bounds__(ANALYTICS_TX * ANALYTICS_TY)
    k_vorticity_2d(const float* __restrict__ ux, const float* __restrict__ uy, float* __restrict__ vort, int nx,
                   int ny) {
    const int x = blockIdx.x * ANALYTICS_TX + threadIdx.x;
    if (x >= nx) return;
    const int xm = x == 0 ? nx - 1 : x - 1, xp = x + 1 == nx ? 0 : x + 1;
    for (long long yt = blockIdx.y; yt * ANALYTICS_TY < ny; yt += gridDim.y) {
        const long long yl = yt * ANALYTICS_TY + threadIdx.y;
        if (yl >= ny) break;
        const int y = static_cast<int>(yl);
        const int ym = y == 0 ? ny - 1 : y - 1, yp = y + 1 == ny ? 0 : y + 1;
        const long long row = static_cast<long long>(y) * nx;
        const float duy_dx = half_diff(uy[row + xp], uy[row + xm]);
        const float dux_dy =
            half_diff(ux[static_cast<long long>(yp) * nx + x], ux[static_cast<long long>(ym) * nx + x]);
        vort[row + x] = __fsub_rn(duy_dx, dux_dy);
    }
}

__device__ __forceinline__ float sq(float a) { return __fmul_rn(a, a); }

static __global__ void __launch_bounds__(ANALYTICS_TX * ANALYTICS_TY)
    k_vorticity_q_3d(const float* __restrict__ ux, const float* __restrict__ uy, const float* __restrict__ uz,
                     float* __restrict__ ox, float* __restrict__ oy, float* __restrict__ oz, float* __restrict__ qc,
                     int nx, int ny, int nz) {
    const int x = blockIdx.x * ANALYTICS_TX + threadIdx.x;
    if (x >= nx) return;
    const int xm = x == 0 ? nx - 1 : x - 1, xp = x + 1 == nx ? 0 : x + 1;
    const long long plane = static_cast<long long>(nx) * ny;
    const int z0 = static_cast<int>(blockIdx.z) * ANALYTICS_ZC;
    const int z1 = z0 + ANALYTICS_ZC < nz ? z0 + ANALYTICS_ZC : nz;
    for (long long yt = blockIdx.y; yt * ANALYTICS_TY < ny; yt += gridDim.y) {
        const long long yl = yt * ANALYTICS_TY + threadIdx.y;
        if (yl >= ny) break;
        const int y = static_cast<int>(yl);
        const int ym = y == 0 ? ny - 1 : y - 1, yp = y + 1 == ny ? 0 : y + 1;
        const long long oc = static_cast<long long>(y) * nx + x;
        const long long oym = static_cast<long long>(ym) * nx + x, oyp = static_cast<long long>(yp) * nx + x;
        const long long ocm = static_cast<long long>(y) * nx + xm, ocp = static_cast<long long>(y) * nx + xp;
        // the column's values at z - 1 (lo), z (mid) and z + 1 (hi); each plane loads the next one
        const long long pz0 = static_cast<long long>(z0) * plane;
        const long long pzm = static_cast<long long>(z0 == 0 ? nz - 1 : z0 - 1) * plane;
        float lo_x = ux[pzm + oc], lo_y = uy[pzm + oc], lo_z = uz[pzm + oc];
        float mid_x = ux[pz0 + oc], mid_y = uy[pz0 + oc], mid_z = uz[pz0 + oc];
        const long long pz1 = static_cast<long long>(z0 + 1 == nz ? 0 : z0 + 1) * plane;
        float hi_x = ux[pz1 + oc], hi_y = uy[pz1 + oc], hi_z = uz[pz1 + oc];
        for (int z = z0; z < z1; ++z) {
            const long long pz = static_cast<long long>(z) * plane;
            // the column's value one plane further, loaded while this plane is computed
            float nx_x = 0.f, nx_y = 0.f, nx_z = 0.f;
            if (z + 1 < z1) {
                const int z2 = z + 2 >= nz ? z + 2 - nz : z + 2;
                const long long pz2 = static_cast<long long>(z2) * plane;
                nx_x = ux[pz2 + oc], nx_y = uy[pz2 + oc], nx_z = uz[pz2 + oc];
            }

            const float dux_dx = half_diff(ux[pz + ocp], ux[pz + ocm]);
            const float dux_dy = half_diff(ux[pz + oyp], ux[pz + oym]);
            const float dux_dz = half_diff(hi_x, lo_x);
            const float duy_dx = half_diff(uy[pz + ocp], uy[pz + ocm]);
            const float duy_dy = half_diff(uy[pz + oyp], uy[pz + oym]);
            const float duy_dz = half_diff(hi_y, lo_y);
            const float duz_dx = half_diff(uz[pz + ocp], uz[pz + ocm]);
            const float duz_dy = half_diff(uz[pz + oyp], uz[pz + oym]);
            const float duz_dz = half_diff(hi_z, lo_z);

            ox[pz + oc] = __fsub_rn(duz_dy, duy_dz);
            oy[pz + oc] = __fsub_rn(dux_dz, duz_dx);
            oz[pz + oc] = __fsub_rn(duy_dx, dux_dy);

            // strain rate S and rotation Omega (symmetric / antisymmetric halves of grad u)
            const float s_xy = __fmul_rn(0.5f, __fadd_rn(dux_dy, duy_dx));
            const float s_yz = __fmul_rn(0.5f, __fadd_rn(duy_dz, duz_dy));
            const float s_xz = __fmul_rn(0.5f, __fadd_rn(dux_dz, duz_dx));
            const float norm_s = __fadd_rn(__fadd_rn(__fadd_rn(sq(dux_dx), sq(duy_dy)), sq(duz_dz)),
                                           __fmul_rn(2.0f, __fadd_rn(__fadd_rn(sq(s_xy), sq(s_yz)), sq(s_xz))));
            const float o_xy = half_diff(dux_dy, duy_dx);
            const float o_yz = half_diff(duy_dz, duz_dy);
            const float o_xz = half_diff(dux_dz, duz_dx);
            const float norm_o = __fmul_rn(2.0f, __fadd_rn(__fadd_rn(sq(o_xy), sq(o_yz)), sq(o_xz)));
            qc[pz + oc] = __fmul_rn(0.5f, __fsub_rn(norm_o, norm_s));

            lo_x = mid_x, lo_y = mid_y, lo_z = mid_z;
            mid_x = hi_x, mid_y = hi_y, mid_z = hi_z;
            hi_x = nx_x, hi_y = nx_y, hi_z = nx_z;
        }
    }
}

// Largest |v| over n values, NaN skipped (std::max(m, |v|) from m = 0 keeps m
// when v is NaN). The maximum of non-negative floats is order-independent, so
// the atomic on their bit patterns gives one answer whatever the schedule.
static __global__ void k_absmax(const float* __restrict__ v, long long n, unsigned* __restrict__ out) {
    float m = 0.0f;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const float a = fabsf(v[i]);
        if (a > m) m = a;  // false for NaN
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

inline dim3 analytics_grid_3d(int nx, int ny, int nz) {
    const long long ytiles = (static_cast<long long>(ny) + ANALYTICS_TY - 1) / ANALYTICS_TY;
    return dim3(static_cast<unsigned>((nx + ANALYTICS_TX - 1) / ANALYTICS_TX),
                static_cast<unsigned>(ytiles < 65535 ? ytiles : 65535),
                static_cast<unsigned>((nz + ANALYTICS_ZC - 1) / ANALYTICS_ZC));
}
inline dim3 analytics_block() { return dim3(ANALYTICS_TX, ANALYTICS_TY); }

}  // namespace wk
