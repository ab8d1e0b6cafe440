// Field analytics on the device: 2D vorticity, 3D vorticity vector and
// Q-criterion from the macroscopic velocity (src/ispc/analytics_kernels.ispc:4-110),
// and the largest |value| of a field (src/analytics/field_analytics.cpp:56-62).
//
// The stencil is the reference's: central differences with periodic wrap on
// every axis. Every product and sum is rounded explicitly (__fmul_rn/__fadd_rn)
// in the reference's evaluation order, so no multiply-add is contracted and the
// results equal a plain IEEE float32 evaluation of the same expressions.
//
// One thread per node; a block covers a run of one x-row, consecutive blocks
// the neighbouring rows, so the y and z neighbours of a block are read from L1/L2
// and DRAM sees each velocity component about once: algorithmic traffic is
// 8 B in + 4 B out per node in 2D and 12 B in + 16 B out per node in 3D.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace wk {

__device__ __forceinline__ float half_diff(float a, float b) { return __fmul_rn(0.5f, __fsub_rn(a, b)); }

// Grids of both stencils: x-blocks in blockIdx.x, rows (y + ny*z) spread over
// blockIdx.y and blockIdx.z (analytics_grid_3d).
static __global__ void k_vorticity_2d(const float* __restrict__ ux, const float* __restrict__ uy, float* __restrict__ vort,
                                      int nx, int ny) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const long long r = static_cast<long long>(blockIdx.y) + static_cast<long long>(blockIdx.z) * gridDim.y;
    if (x >= nx || r >= ny) return;
    const int y = static_cast<int>(r);
    const int ym = y == 0 ? ny - 1 : y - 1, yp = y + 1 == ny ? 0 : y + 1;
    const int xm = x == 0 ? nx - 1 : x - 1, xp = x + 1 == nx ? 0 : x + 1;
    const long long row = static_cast<long long>(y) * nx;
    const float duy_dx = half_diff(uy[row + xp], uy[row + xm]);
    const float dux_dy = half_diff(ux[static_cast<long long>(yp) * nx + x], ux[static_cast<long long>(ym) * nx + x]);
    vort[row + x] = __fsub_rn(duy_dx, dux_dy);
}

__device__ __forceinline__ float sq(float a) { return __fmul_rn(a, a); }

static __global__ void k_vorticity_q_3d(const float* __restrict__ ux, const float* __restrict__ uy,
                                        const float* __restrict__ uz, float* __restrict__ ox, float* __restrict__ oy,
                                        float* __restrict__ oz, float* __restrict__ qc, int nx, int ny, int nz) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const long long r = static_cast<long long>(blockIdx.y) + static_cast<long long>(blockIdx.z) * gridDim.y;
    if (x >= nx || r >= static_cast<long long>(ny) * nz) return;
    const int y = static_cast<int>(r % ny), z = static_cast<int>(r / ny);
    const int ym = y == 0 ? ny - 1 : y - 1, yp = y + 1 == ny ? 0 : y + 1;
    const int zm = z == 0 ? nz - 1 : z - 1, zp = z + 1 == nz ? 0 : z + 1;
    const int xm = x == 0 ? nx - 1 : x - 1, xp = x + 1 == nx ? 0 : x + 1;
    const long long c = r * nx;
    const long long cyp = (static_cast<long long>(z) * ny + yp) * nx, cym = (static_cast<long long>(z) * ny + ym) * nx;
    const long long czp = (static_cast<long long>(zp) * ny + y) * nx, czm = (static_cast<long long>(zm) * ny + y) * nx;

    const float dux_dx = half_diff(ux[c + xp], ux[c + xm]);
    const float dux_dy = half_diff(ux[cyp + x], ux[cym + x]);
    const float dux_dz = half_diff(ux[czp + x], ux[czm + x]);
    const float duy_dx = half_diff(uy[c + xp], uy[c + xm]);
    const float duy_dy = half_diff(uy[cyp + x], uy[cym + x]);
    const float duy_dz = half_diff(uy[czp + x], uy[czm + x]);
    const float duz_dx = half_diff(uz[c + xp], uz[c + xm]);
    const float duz_dy = half_diff(uz[cyp + x], uz[cym + x]);
    const float duz_dz = half_diff(uz[czp + x], uz[czm + x]);

    ox[c + x] = __fsub_rn(duz_dy, duy_dz);
    oy[c + x] = __fsub_rn(dux_dz, duz_dx);
    oz[c + x] = __fsub_rn(duy_dx, dux_dy);

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
    qc[c + x] = __fmul_rn(0.5f, __fsub_rn(norm_o, norm_s));
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

inline dim3 analytics_grid_3d(int nx, int ny, int nz, int tpb) {
    const long long rows = static_cast<long long>(ny) * nz;
    const unsigned gy = static_cast<unsigned>(rows < 65535 ? rows : 65535);
    const unsigned gz = static_cast<unsigned>((rows + gy - 1) / gy);
    return dim3(static_cast<unsigned>((nx + tpb - 1) / tpb), gy, gz);
}

}  // namespace wk
