// Drop-in entry points with the reference's ISPC export signatures
// (src/ispc/*.ispc; declared in include/wake_gpu.h with file:line citations).
//
// Each call is synchronous, like the ISPC functions it replaces. Pointers to
// device or managed memory are used in place; pointers to host memory are
// staged through a per-thread device arena (copied in before the kernel and
// the outputs copied back after it). Work runs on the legacy default stream,
// which orders it after work the caller queued on that stream.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "lattice.cuh"
#include "analytics.cuh"
#include "stream_collide.cuh"
#include "wake_gpu.h"

namespace wk {
namespace {

// ---------------------------------------------------------------- staging
// Where a caller's pointer lives, seen from the current device.
enum class PtrKind { Host, Here, OtherDevice };

PtrKind pointer_kind(const void* p) {
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return PtrKind::Host;
    }
    if (attr.type == cudaMemoryTypeManaged) return PtrKind::Here;
    if (attr.type != cudaMemoryTypeDevice) return PtrKind::Host;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        (void)cudaGetLastError();
        return PtrKind::OtherDevice;
    }
    // device memory of another GPU: its kernels here would read peer memory (or fault
    // without peer access), so callers get WAKE_ERR_INVALID instead
    return attr.device == dev ? PtrKind::Here : PtrKind::OtherDevice;
}

struct Arena {
    DevMem mem;
};
thread_local Arena t_arena;

struct Item {
    void* user;
    std::size_t bytes;
    std::size_t offset;
    bool in, out, staged;
    void* dev;
};

class Stager {
   public:
    template <class T>
    T* in(const T* p, std::size_t n) { return static_cast<T*>(add(const_cast<T*>(p), n * sizeof(T), true, false)); }
    template <class T>
    T* inout(T* p, std::size_t n) { return static_cast<T*>(add(p, n * sizeof(T), true, true)); }
    // Outputs are copied in as well: like the reference, kernels leave some
    // entries (e.g. moments at solid nodes) untouched, and those keep the caller's values.
    template <class T>
    T* out(T* p, std::size_t n) { return static_cast<T*>(add(p, n * sizeof(T), true, true)); }
    // An output the kernel writes in full: nothing to copy in.
    template <class T>
    T* full_out(T* p, std::size_t n) { return static_cast<T*>(add(p, n * sizeof(T), false, true)); }

    // Allocate the arena and copy staged inputs. Returns 0 or an error code.
    int begin() {
        if (bad_) return set_error(WAKE_ERR_INVALID, "null pointer argument");
        if (foreign_)
            return set_error(WAKE_ERR_INVALID, "pointer to another GPU's memory: make that GPU current, or pass "
                                               "memory of the current GPU");
        if (total_ > 0) {
            const cudaError_t e = t_arena.mem.ensure(total_);
            if (e != cudaSuccess) return set_error(WAKE_ERR_NOMEM, std::string("staging: ") + cudaGetErrorString(e));
        }
        for (Item& it : items_) {
            if (!it.staged) continue;
            it.dev = static_cast<char*>(t_arena.mem.p) + it.offset;
            if (it.in) WK_CUDA(cudaMemcpyAsync(it.dev, it.user, it.bytes, cudaMemcpyHostToDevice, 0));
        }
        return WAKE_OK;
    }
    // Copy staged outputs back and wait for the device.
    int end() {
        WK_CUDA(cudaGetLastError());
        for (Item& it : items_)
            if (it.staged && it.out) WK_CUDA(cudaMemcpyAsync(it.user, it.dev, it.bytes, cudaMemcpyDeviceToHost, 0));
        WK_CUDA(cudaStreamSynchronize(0));
        return WAKE_OK;
    }
    template <class T>
    T* ptr(int k) const { return static_cast<T*>(items_[k].dev); }

   private:
    void* add(void* p, std::size_t bytes, bool in, bool out) {
        Item it{p, bytes, 0, in, out, false, p};
        if (!p && bytes > 0) bad_ = true;
        if (p) {
            const PtrKind k = pointer_kind(p);
            if (k == PtrKind::OtherDevice) foreign_ = true;
            if (k == PtrKind::Host) {
                it.staged = true;
                it.offset = total_;
                total_ += (bytes + 255) / 256 * 256;
            }
        }
        items_.push_back(it);
        return p;  // replaced by dev(k) after begin()
    }
    std::vector<Item> items_;
    std::size_t total_ = 0;
    bool bad_ = false;
    bool foreign_ = false;
};

inline int blocks_for(long long n, int t = 256) { return static_cast<int>((n + t - 1) / t); }

// ---------------------------------------------------------------- kernels
// Collision kernels (d2q9_collision_{bgk,trt,mrt}.ispc, d3q19_collision_*.ispc,
// d3q27_collision_mrt.ispc): solid copy-through, pre-collision moments written.
template <int Q, int COLL>
__global__ void k_collide(const float* __restrict__ fin, float* __restrict__ fout, const uint8_t* __restrict__ ct,
                          float* rho, float* ux, float* uy, float* uz, float p0, float p1, float gx, float gy,
                          float gz, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const long long n = count;
    float f[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) f[q] = fin[q * n + i];
    if (ct[i] == CT_SOLID) {
#pragma unroll
        for (int q = 0; q < Q; ++q) fout[q * n + i] = f[q];
        return;
    }
    const float g[3] = {gx, gy, gz};
    float r, u[3];
    node_moments<Q>(f, g, r, u);
    rho[i] = r;
    ux[i] = u[0];
    uy[i] = u[1];
    if (uz) uz[i] = u[2];
    if (COLL == COLL_BGK) collide_bgk<Q>(f, r, u, g, p0);
    else if (COLL == COLL_TRT && Q == 27) collide_trt_d3q27_reference(f, r, u, g, p0, p1);
    else if (COLL == COLL_TRT) collide_trt<Q>(f, r, u, g, p0, p1);
    else if constexpr (Q == 9) collide_mrt_d2q9(f, r, u, g, p0, p1);
    else collide_mrt_d3q19(f, r, u, g, p0, p1, 0);
#pragma unroll
    for (int q = 0; q < Q; ++q) fout[q * n + i] = f[q];
}

// Fully periodic pull (d2q9_streaming.ispc:4-29, d3q19_streaming.ispc:4-35, d3q27_streaming.ispc:4-35).
template <int Q>
__global__ void k_stream_periodic(const float* __restrict__ src, float* __restrict__ dst, int nx, int ny, int nz) {
    using L = Lat<Q>;
    const long long n = static_cast<long long>(nx) * ny * nz;
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const int x = static_cast<int>(i % nx), y = static_cast<int>((i / nx) % ny), z = static_cast<int>(i / (static_cast<long long>(nx) * ny));
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int sx = wrap<Q>(x - L::cx(q), nx), sy = wrap<Q>(y - L::cy(q), ny), sz = wrap<Q>(z - L::cz(q), nz);
        dst[q * n + i] = src[q * n + (static_cast<long long>(sz) * ny + sy) * nx + sx];
    }
}

// Pull with half-way bounce-back (d2q9_streaming.ispc:33-95, d3q19_streaming.ispc:39-104).
template <int Q>
__global__ void k_stream_bounded(const float* __restrict__ src, float* __restrict__ dst, const uint8_t* __restrict__ ct,
                                 int nx, int ny, int nz, float uwx, float uwy, float uwz) {
    using L = Lat<Q>;
    const long long n = static_cast<long long>(nx) * ny * nz;
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const int x = static_cast<int>(i % nx), y = static_cast<int>((i / nx) % ny), z = static_cast<int>(i / (static_cast<long long>(nx) * ny));
    const bool solid = ct[i] == CT_SOLID;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        if (solid) {
            dst[q * n + i] = src[q * n + i];
            continue;
        }
        const int o = L::opp(q);
        const int sx = wrap<Q>(x - L::cx(q), nx), sy = y - L::cy(q), sz = z - L::cz(q);
        if (sy >= 0 && sy < ny && sz >= 0 && sz < nz) {
            const long long s = (static_cast<long long>(sz) * ny + sy) * nx + sx;
            const uint8_t t = ct[s];
            if (t == CT_SOLID) {
                dst[q * n + i] = src[o * n + i];
            } else if (t == CT_MOVING_WALL) {
                const float ci_uw = float(L::cx(q)) * uwx + float(L::cy(q)) * uwy + float(L::cz(q)) * uwz;
                dst[q * n + i] = src[o * n + i] + 2.0f * L::w(q) * 1.0f * 3.0f * ci_uw;
            } else {
                dst[q * n + i] = src[q * n + s];
            }
        } else {
            dst[q * n + i] = src[o * n + i];
        }
    }
}

// In-place full-way swap on solid / moving-wall nodes (d2q9_boundaries.ispc:5-39).
__global__ void k_bounce_back_d2q9(float* f, const uint8_t* ct, float uwx, float uwy, int count) {
    using L = Lat<9>;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    if (!(ct[i] == CT_SOLID || ct[i] == CT_MOVING_WALL)) return;
    const long long n = count;
    float c[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) c[q] = f[q * n + i];
#pragma unroll
    for (int q = 1; q < 9; ++q) {
        const float ci_uw = float(L::cx(q)) * uwx + float(L::cy(q)) * uwy;
        f[q * n + i] = c[L::opp(q)] + 2.0f * L::w(q) * 1.0f * 3.0f * ci_uw;
    }
}

__global__ void k_zou_he_2d(float* f, float* rho, float* ux, float* uy, float a, float b, int nx, int ny, int inlet) {
    const int y = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (y > ny - 2) return;
    const long long n = static_cast<long long>(nx) * ny;
    const long long idx = static_cast<long long>(y) * nx + (inlet ? 0 : nx - 1);
    float c[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) c[q] = f[q * n + idx];
    if (inlet) {
        const float uin[3] = {a, b, 0.f};
        zou_he_inlet<9>(c, uin);
        f[1 * n + idx] = c[1];
        f[5 * n + idx] = c[5];
        f[8 * n + idx] = c[8];
        // d2q9_boundaries.ispc:60-78: rho_in from the knowns, prescribed velocity
        rho[idx] = (c[0] + c[2] + c[4] + 2.0f * (c[3] + c[6] + c[7])) / (1.0f - a);
        ux[idx] = a;
        uy[idx] = b;
    } else {
        zou_he_outlet<9>(c, a);
        f[3 * n + idx] = c[3];
        f[6 * n + idx] = c[6];
        f[7 * n + idx] = c[7];
        // d2q9_boundaries.ispc:108-120: prescribed rho, u_x from the knowns
        rho[idx] = a;
        ux[idx] = -1.0f + (c[0] + c[2] + c[4] + 2.0f * (c[1] + c[5] + c[8])) / a;
        uy[idx] = 0.0f;
    }
}

// d2q9_boundaries.ispc:125-146
__global__ void k_convective_outflow(float* f, const float* fprev, float u_conv, int nx, int ny) {
    const int y = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (y > ny - 2) return;
    const long long n = static_cast<long long>(nx) * ny;
    const float alpha = u_conv / (1.0f + u_conv), beta = 1.0f / (1.0f + u_conv);
    const long long io = static_cast<long long>(y) * nx + (nx - 1), ii = io - 1;
#pragma unroll
    for (int q = 0; q < 9; ++q) f[q * n + io] = beta * fprev[q * n + io] + alpha * f[q * n + ii];
}

template <int Q>
__global__ void k_smagorinsky(const float* f, const float* rho, const float* ux, const float* uy, const float* uz,
                              float* tau_eff, float tau0, float cs, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const long long n = count;
    float c[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) c[q] = f[q * n + i];
    const float u[3] = {ux[i], uy[i], uz ? uz[i] : 0.f};
    tau_eff[i] = smagorinsky_tau<Q>(c, rho[i], u, tau0, cs);
}

template <int Q>
__global__ void k_moments(const float* f, float* rho, float* ux, float* uy, float* uz, float gx, float gy, float gz,
                          int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const long long n = count;
    float c[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) c[q] = f[q * n + i];
    const float g[3] = {gx, gy, gz};
    float r, u[3];
    node_moments<Q>(c, g, r, u);
    rho[i] = r;
    ux[i] = u[0];
    uy[i] = u[1];
    if (uz) uz[i] = u[2];
}

__global__ void k_speed(const float* ux, const float* uy, const float* uz, float* speed, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float a = ux[i], b = uy[i], c = uz ? uz[i] : 0.f;
    speed[i] = sqrtf(a * a + b * b + c * c);
}

// Momentum exchange (forces_momentum_exchange.ispc:6-138), FP64 block partials.
template <int Q>
__global__ void k_mem_partials(const float* __restrict__ f, const uint8_t* __restrict__ ct, int nx, int ny, int nz,
                               float cx, float cy, float cz, float rmax, double* __restrict__ part) {
    using L = Lat<Q>;
    __shared__ double red[3][256];
    const long long n = static_cast<long long>(nx) * ny * nz;
    double acc[3] = {0.0, 0.0, 0.0};
    const float rmax_sq = rmax * rmax;
    for (long long i = blockIdx.x * 256ll + threadIdx.x; i < n; i += 256ll * gridDim.x) {
        if (ct[i] != CT_FLUID) continue;
        const int x = static_cast<int>(i % nx), y = static_cast<int>((i / nx) % ny),
                  z = static_cast<int>(i / (static_cast<long long>(nx) * ny));
#pragma unroll
        for (int q = 1; q < Q; ++q) {
            const int xn = wrap<Q>(x + L::cx(q), nx), yn = y + L::cy(q), zn = z + L::cz(q);
            if (yn < 0 || yn >= ny || zn < 0 || zn >= nz) continue;
            const uint8_t t = ct[(static_cast<long long>(zn) * ny + yn) * nx + xn];
            if (t != CT_SOLID && t != CT_MOVING_WALL) continue;
            const float rx = __fsub_rn(__fadd_rn(float(x), 0.5f * float(L::cx(q))), cx);
            const float ry = __fsub_rn(__fadd_rn(float(y), 0.5f * float(L::cy(q))), cy);
            const float rz = __fsub_rn(__fadd_rn(float(z), 0.5f * float(L::cz(q))), cz);
            float r2 = __fadd_rn(__fmul_rn(rx, rx), __fmul_rn(ry, ry));
            if (L::D == 3) r2 = __fadd_rn(r2, __fmul_rn(rz, rz));
            if (!(rmax <= 0.0f || r2 <= rmax_sq)) continue;
            const double fv = f[q * n + i];
            const double dfx = 2.0 * fv * L::cx(q), dfy = 2.0 * fv * L::cy(q);
            acc[0] += dfx;
            acc[1] += dfy;
            acc[2] += (L::D == 2) ? double(rx) * dfy - double(ry) * dfx : 2.0 * fv * L::cz(q);
        }
    }
    for (int c = 0; c < 3; ++c) red[c][threadIdx.x] = acc[c];
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int c = 0; c < 3; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 3; ++c) part[3 * blockIdx.x + c] = red[c][0];
}

__global__ void k_mem_final(const double* part, int nblocks, float* o0, float* o1, float* o2) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s[3] = {0.0, 0.0, 0.0};
    for (int b = 0; b < nblocks; ++b)
        for (int c = 0; c < 3; ++c) s[c] += part[3 * b + c];
    *o0 = static_cast<float>(s[0]);
    *o1 = static_cast<float>(s[1]);
    *o2 = static_cast<float>(s[2]);
}

// BFL (d3q19_curved.ispc:7-71), one thread per link.
__global__ void k_bfl(float* fdst, const float* fsrc, const int* idx, const int* qd, const float* delta,
                      const float* uwx, const float* uwy, const float* uwz, int nx, int ny, int nz, int nl) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nl) return;
    const long long n = static_cast<long long>(nx) * ny * nz;
    const int i = idx[k], q = qd[k];
    // the links may come straight from device memory: skip malformed ones instead of faulting
    if (i < 0 || i >= n || q < 1 || q >= 19) return;
    int cx, cy, cz, o;
    float w;
    rt_dir<19>(q, cx, cy, cz, o, w);
    const float d = delta[k];
    const float ci_uw = float(cx) * uwx[k] + float(cy) * uwy[k] + float(cz) * uwz[k];
    const float fi = fsrc[q * n + i], fo = fsrc[o * n + i];
    float val;
    if (d < 0.5f) {
        const int zf = i / (nx * ny), rem = i - zf * nx * ny, yf = rem / nx, xf = rem - yf * nx;
        const int xff = wrap<19>(xf - cx, nx), yff = yf - cy, zff = zf - cz;
        float fff = fi;
        if (yff >= 0 && yff < ny && zff >= 0 && zff < nz) fff = fsrc[q * n + (static_cast<long long>(zff) * ny + yff) * nx + xff];
        const float mom = 2.0f * w * 1.0f * 3.0f * ci_uw;
        val = 2.0f * d * fi + (1.0f - 2.0f * d) * fff - mom;
    } else {
        const float i2d = 1.0f / (2.0f * d);
        const float mom = (1.0f / d) * w * 1.0f * 3.0f * ci_uw;
        val = i2d * fi + (1.0f - i2d) * fo - mom;
    }
    fdst[o * n + i] = val;
}

// Thermal D2Q9 (thermal_kernels.ispc:4-81).
__global__ void k_thermal_collide(const float* gin, float* gout, const uint8_t* ct, const float* ux, const float* uy,
                                  float* temp, float tau_T, int count) {
    using L = Lat<9>;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const long long n = count;
    float g[9], T = 0.f;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        g[q] = gin[q * n + i];
        T += g[q];
    }
    if (ct[i] == CT_SOLID) {
#pragma unroll
        for (int q = 0; q < 9; ++q) gout[q * n + i] = g[q];
        return;
    }
    temp[i] = T;
    const float om = 1.0f / tau_T, vx = ux[i], vy = uy[i];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const float cu = float(L::cx(q)) * vx + float(L::cy(q)) * vy;
        const float geq = L::w(q) * T * (1.0f + 3.0f * cu);
        gout[q * n + i] = g[q] - om * (g[q] - geq);
    }
}

__global__ void k_buoyancy(const float* T, float* gy, float tref, float beta, float grav, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) gy[i] += beta * (T[i] - tref) * grav;
}

__global__ void k_isothermal_wall(float* g, int nx, int ny, int yw, float tw) {
    using L = Lat<9>;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= nx) return;
    const long long n = static_cast<long long>(nx) * ny, idx = static_cast<long long>(yw) * nx + x;
    float c[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) c[q] = g[q * n + idx];
    // sequential in q on the live values, like the reference loop (thermal_kernels.ispc:73-79)
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const int o = L::opp(q);
        const float v = -c[q] + 2.0f * L::w(q) * tw;
#pragma unroll
        for (int k = 0; k < 9; ++k)
            if (k == o) c[k] = v;
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) g[q * n + idx] = c[q];
}

// ---------------------------------------------------------------- call wrappers
template <int Q, int COLL>
void collide_call(const float* fin, float* fout, const uint8_t* ct, float* rho, float* ux, float* uy, float* uz,
                  float p0, float p1, float gx, float gy, float gz, int count) {
    if (count <= 0) return;
    const std::size_t n = static_cast<std::size_t>(count);
    Stager s;
    s.in(fin, Q * n);
    s.out(fout, Q * n);
    s.in(ct, n);
    s.out(rho, n);
    s.out(ux, n);
    s.out(uy, n);
    if (Q != 9) s.out(uz, n);
    if (s.begin()) return;
    k_collide<Q, COLL><<<blocks_for(count), 256>>>(s.ptr<float>(0), s.ptr<float>(1), s.ptr<uint8_t>(2), s.ptr<float>(3),
                                                    s.ptr<float>(4), s.ptr<float>(5), Q != 9 ? s.ptr<float>(6) : nullptr,
                                                    p0, p1, gx, gy, gz, count);
    s.end();
}

template <int Q>
void mem_call(const float* f, const uint8_t* ct, int nx, int ny, int nz, float cx, float cy, float cz, float rmax,
              float* o0, float* o1, float* o2) {
    const long long n = static_cast<long long>(nx) * ny * nz;
    if (n <= 0) return;
    Stager s;
    s.in(f, Q * static_cast<std::size_t>(n));
    s.in(ct, static_cast<std::size_t>(n));
    s.out(o0, 1);
    s.out(o1, 1);
    s.out(o2, 1);
    if (s.begin()) return;
    const int nb = static_cast<int>(std::min<long long>(1184, (n + 255) / 256));
    DevMem part;
    if (part.ensure(sizeof(double) * 3 * nb) != cudaSuccess) {
        set_error(WAKE_ERR_NOMEM, "momentum exchange: partials");
        return;
    }
    k_mem_partials<Q><<<nb, 256>>>(s.ptr<float>(0), s.ptr<uint8_t>(1), nx, ny, nz, cx, cy, cz, rmax, part.as<double>());
    k_mem_final<<<1, 32>>>(part.as<double>(), nb, s.ptr<float>(2), s.ptr<float>(3), s.ptr<float>(4));
    s.end();
}

}  // namespace
}  // namespace wk

using namespace wk;

extern "C" {

void d2q9_collide_bgk(const float f_in[], float f_out[], const uint8_t cell_type[], float rho[], float ux[],
                      float uy[], float tau, float gx, float gy, int count) {
    collide_call<9, COLL_BGK>(f_in, f_out, cell_type, rho, ux, uy, nullptr, tau, 0.f, gx, gy, 0.f, count);
}
void d2q9_collide_trt(const float f_in[], float f_out[], const uint8_t cell_type[], float rho[], float ux[],
                      float uy[], float tau_s, float tau_a, float gx, float gy, int count) {
    collide_call<9, COLL_TRT>(f_in, f_out, cell_type, rho, ux, uy, nullptr, tau_s, tau_a, gx, gy, 0.f, count);
}
void d2q9_collide_mrt(const float f_in[], float f_out[], const uint8_t cell_type[], float rho[], float ux[],
                      float uy[], float tau_shear, float tau_bulk, float gx, float gy, int count) {
    collide_call<9, COLL_MRT>(f_in, f_out, cell_type, rho, ux, uy, nullptr, tau_shear, tau_bulk, gx, gy, 0.f, count);
}
void d3q19_collide_bgk(const float f_in[], float f_out[], const uint8_t cell_type[], float rho[], float ux[],
                       float uy[], float uz[], float tau, float gx, float gy, float gz, int count) {
    collide_call<19, COLL_BGK>(f_in, f_out, cell_type, rho, ux, uy, uz, tau, 0.f, gx, gy, gz, count);
}
void d3q19_collide_trt(const float f_in[], float f_out[], const uint8_t cell_type[], float rho[], float ux[],
                       float uy[], float uz[], float tau_s, float tau_a, float gx, float gy, float gz, int count) {
    collide_call<19, COLL_TRT>(f_in, f_out, cell_type, rho, ux, uy, uz, tau_s, tau_a, gx, gy, gz, count);
}
void d3q19_collide_mrt(const float f_in[], float f_out[], const uint8_t cell_type[], float rho[], float ux[],
                       float uy[], float uz[], float tau_shear, float tau_bulk, float gx, float gy, float gz,
                       int count) {
    collide_call<19, COLL_MRT>(f_in, f_out, cell_type, rho, ux, uy, uz, tau_shear, tau_bulk, gx, gy, gz, count);
}
void d3q27_collide(const float f_in[], float f_out[], const uint8_t cell_type[], float rho[], float ux[], float uy[],
                   float uz[], float tau_s, float tau_a, float gx, float gy, float gz, int count) {
    collide_call<27, COLL_TRT>(f_in, f_out, cell_type, rho, ux, uy, uz, tau_s, tau_a, gx, gy, gz, count);
}

static void stream_periodic_call(int Q, const float* src, float* dst, int nx, int ny, int nz) {
    const long long n = static_cast<long long>(nx) * ny * nz;
    if (nx <= 0 || ny <= 0 || nz <= 0) return;
    Stager s;
    s.in(src, Q * static_cast<std::size_t>(n));
    s.out(dst, Q * static_cast<std::size_t>(n));
    if (s.begin()) return;
    const int nb = blocks_for(n);
    if (Q == 9) k_stream_periodic<9><<<nb, 256>>>(s.ptr<float>(0), s.ptr<float>(1), nx, ny, nz);
    else if (Q == 19) k_stream_periodic<19><<<nb, 256>>>(s.ptr<float>(0), s.ptr<float>(1), nx, ny, nz);
    else k_stream_periodic<27><<<nb, 256>>>(s.ptr<float>(0), s.ptr<float>(1), nx, ny, nz);
    s.end();
}
void d2q9_stream_periodic(const float f_src[], float f_dst[], int nx, int ny) {
    stream_periodic_call(9, f_src, f_dst, nx, ny, 1);
}
void d3q19_stream_periodic(const float f_src[], float f_dst[], int nx, int ny, int nz) {
    stream_periodic_call(19, f_src, f_dst, nx, ny, nz);
}
void d3q27_stream_periodic(const float f_src[], float f_dst[], int nx, int ny, int nz) {
    stream_periodic_call(27, f_src, f_dst, nx, ny, nz);
}

static void stream_bounded_call(int Q, const float* src, float* dst, const uint8_t* ct, int nx, int ny, int nz,
                                float uwx, float uwy, float uwz) {
    const long long n = static_cast<long long>(nx) * ny * nz;
    if (nx <= 0 || ny <= 0 || nz <= 0) return;
    Stager s;
    s.in(src, Q * static_cast<std::size_t>(n));
    s.out(dst, Q * static_cast<std::size_t>(n));
    s.in(ct, static_cast<std::size_t>(n));
    if (s.begin()) return;
    const int nb = blocks_for(n);
    if (Q == 9) k_stream_bounded<9><<<nb, 256>>>(s.ptr<float>(0), s.ptr<float>(1), s.ptr<uint8_t>(2), nx, ny, nz, uwx, uwy, 0.f);
    else k_stream_bounded<19><<<nb, 256>>>(s.ptr<float>(0), s.ptr<float>(1), s.ptr<uint8_t>(2), nx, ny, nz, uwx, uwy, uwz);
    s.end();
}
void d2q9_stream_with_boundaries(const float f_src[], float f_dst[], const uint8_t cell_type[], int nx, int ny,
                                 float uw_x, float uw_y) {
    stream_bounded_call(9, f_src, f_dst, cell_type, nx, ny, 1, uw_x, uw_y, 0.f);
}
void d3q19_stream_with_boundaries(const float f_src[], float f_dst[], const uint8_t cell_type[], int nx, int ny,
                                  int nz, float uw_x, float uw_y, float uw_z) {
    stream_bounded_call(19, f_src, f_dst, cell_type, nx, ny, nz, uw_x, uw_y, uw_z);
}

void d2q9_apply_bounce_back(float f[], const uint8_t cell_type[], float uw_x, float uw_y, int count) {
    if (count <= 0) return;
    Stager s;
    s.inout(f, 9 * static_cast<std::size_t>(count));
    s.in(cell_type, static_cast<std::size_t>(count));
    if (s.begin()) return;
    k_bounce_back_d2q9<<<blocks_for(count), 256>>>(s.ptr<float>(0), s.ptr<uint8_t>(1), uw_x, uw_y, count);
    s.end();
}

static void zou_he_call(float* f, float* rho, float* ux, float* uy, float a, float b, int nx, int ny, int inlet) {
    if (nx <= 0 || ny <= 2) return;
    const std::size_t n = static_cast<std::size_t>(nx) * ny;
    Stager s;
    s.inout(f, 9 * n);
    s.inout(rho, n);
    s.inout(ux, n);
    s.inout(uy, n);
    if (s.begin()) return;
    k_zou_he_2d<<<blocks_for(ny - 2, 128), 128>>>(s.ptr<float>(0), s.ptr<float>(1), s.ptr<float>(2), s.ptr<float>(3), a,
                                                  b, nx, ny, inlet);
    s.end();
}
void d2q9_apply_zou_he_inflow_west(float f[], float rho[], float ux[], float uy[], float u_in_x, float u_in_y, int nx,
                                   int ny) {
    zou_he_call(f, rho, ux, uy, u_in_x, u_in_y, nx, ny, 1);
}
void d2q9_apply_zou_he_outflow_east(float f[], float rho[], float ux[], float uy[], float rho_out, int nx, int ny) {
    zou_he_call(f, rho, ux, uy, rho_out, 0.f, nx, ny, 0);
}

void d2q9_apply_convective_outflow_east(float f[], const float f_prev[], float u_conv, int nx, int ny) {
    if (nx <= 1 || ny <= 2) return;
    const std::size_t n = static_cast<std::size_t>(nx) * ny;
    Stager s;
    s.inout(f, 9 * n);
    s.in(f_prev, 9 * n);
    if (s.begin()) return;
    k_convective_outflow<<<blocks_for(ny - 2, 128), 128>>>(s.ptr<float>(0), s.ptr<float>(1), u_conv, nx, ny);
    s.end();
}

void d2q9_compute_smagorinsky_tau(const float f[], const float rho[], const float ux[], const float uy[],
                                  float tau_eff[], float tau_0, float smagorinsky_constant, int count) {
    if (count <= 0) return;
    const std::size_t n = static_cast<std::size_t>(count);
    Stager s;
    s.in(f, 9 * n);
    s.in(rho, n);
    s.in(ux, n);
    s.in(uy, n);
    s.out(tau_eff, n);
    if (s.begin()) return;
    k_smagorinsky<9><<<blocks_for(count), 256>>>(s.ptr<float>(0), s.ptr<float>(1), s.ptr<float>(2), s.ptr<float>(3),
                                                  nullptr, s.ptr<float>(4), tau_0, smagorinsky_constant, count);
    s.end();
}
void d3q19_compute_smagorinsky_tau(const float f[], const float rho[], const float ux[], const float uy[],
                                   const float uz[], float tau_eff[], float tau_0, float smagorinsky_constant,
                                   int count) {
    if (count <= 0) return;
    const std::size_t n = static_cast<std::size_t>(count);
    Stager s;
    s.in(f, 19 * n);
    s.in(rho, n);
    s.in(ux, n);
    s.in(uy, n);
    s.in(uz, n);
    s.out(tau_eff, n);
    if (s.begin()) return;
    k_smagorinsky<19><<<blocks_for(count), 256>>>(s.ptr<float>(0), s.ptr<float>(1), s.ptr<float>(2), s.ptr<float>(3),
                                                   s.ptr<float>(4), s.ptr<float>(5), tau_0, smagorinsky_constant, count);
    s.end();
}

static void moments_call(int Q, const float* f, float* rho, float* ux, float* uy, float* uz, float gx, float gy,
                         float gz, int count) {
    if (count <= 0) return;
    const std::size_t n = static_cast<std::size_t>(count);
    Stager s;
    s.in(f, Q * n);
    s.out(rho, n);
    s.out(ux, n);
    s.out(uy, n);
    if (Q != 9) s.out(uz, n);
    if (s.begin()) return;
    float* d_uz = Q != 9 ? s.ptr<float>(4) : nullptr;
    const int nb = blocks_for(count);
    if (Q == 9) k_moments<9><<<nb, 256>>>(s.ptr<float>(0), s.ptr<float>(1), s.ptr<float>(2), s.ptr<float>(3), nullptr, gx, gy, gz, count);
    else if (Q == 19) k_moments<19><<<nb, 256>>>(s.ptr<float>(0), s.ptr<float>(1), s.ptr<float>(2), s.ptr<float>(3), d_uz, gx, gy, gz, count);
    else k_moments<27><<<nb, 256>>>(s.ptr<float>(0), s.ptr<float>(1), s.ptr<float>(2), s.ptr<float>(3), d_uz, gx, gy, gz, count);
    s.end();
}
void d2q9_compute_macroscopic_moments(const float f[], float rho[], float ux[], float uy[], int count) {
    moments_call(9, f, rho, ux, uy, nullptr, 0.f, 0.f, 0.f, count);
}
void d2q9_compute_macroscopic_moments_forced(const float f[], float rho[], float ux[], float uy[], float gx, float gy,
                                             int count) {
    moments_call(9, f, rho, ux, uy, nullptr, gx, gy, 0.f, count);
}
void d3q19_compute_macroscopic_moments(const float f[], float rho[], float ux[], float uy[], float uz[], int count) {
    moments_call(19, f, rho, ux, uy, uz, 0.f, 0.f, 0.f, count);
}
void d3q19_compute_macroscopic_moments_forced(const float f[], float rho[], float ux[], float uy[], float uz[],
                                              float gx, float gy, float gz, int count) {
    moments_call(19, f, rho, ux, uy, uz, gx, gy, gz, count);
}
void d3q27_compute_macroscopic_moments(const float f[], float rho[], float ux[], float uy[], float uz[], int count) {
    moments_call(27, f, rho, ux, uy, uz, 0.f, 0.f, 0.f, count);
}

static void speed_call(const float* ux, const float* uy, const float* uz, float* speed, int count) {
    if (count <= 0) return;
    const std::size_t n = static_cast<std::size_t>(count);
    Stager s;
    s.in(ux, n);
    s.in(uy, n);
    if (uz) s.in(uz, n);
    s.out(speed, n);
    if (s.begin()) return;
    k_speed<<<blocks_for(count), 256>>>(s.ptr<float>(0), s.ptr<float>(1), uz ? s.ptr<float>(2) : nullptr,
                                        s.ptr<float>(uz ? 3 : 2), count);
    s.end();
}
void d2q9_compute_velocity_magnitude(const float ux[], const float uy[], float speed[], int count) {
    speed_call(ux, uy, nullptr, speed, count);
}
void d3q19_compute_velocity_magnitude(const float ux[], const float uy[], const float uz[], float speed[], int count) {
    speed_call(ux, uy, uz, speed, count);
}

void d2q9_compute_momentum_exchange_forces(const float f_post_collision[], const uint8_t cell_type[], int nx, int ny,
                                           float center_x, float center_y, float max_radius, float* fx_out,
                                           float* fy_out, float* torque_z_out) {
    mem_call<9>(f_post_collision, cell_type, nx, ny, 1, center_x, center_y, 0.f, max_radius, fx_out, fy_out,
                torque_z_out);
}
void d3q19_compute_momentum_exchange_forces(const float f_post_collision[], const uint8_t cell_type[], int nx, int ny,
                                            int nz, float center_x, float center_y, float center_z, float max_radius,
                                            float* fx_out, float* fy_out, float* fz_out) {
    mem_call<19>(f_post_collision, cell_type, nx, ny, nz, center_x, center_y, center_z, max_radius, fx_out, fy_out,
                 fz_out);
}

}  // extern "C"

// ---------------------------------------------------------------- allocation-free momentum exchange
// Some callers cannot allocate device memory while they run: a serving loop that
// has committed all of HBM to resident lattices (an allocation would fail or
// force an eviction), or a latency-critical loop in which cudaMalloc / cudaFree
// would synchronise the device and stall the other streams. For them this
// variant of d3q19_compute_momentum_exchange_forces keeps its scratch (one
// FP64 partial sum per 256-node block) in a fixed array of this file instead of
// allocating it. The array is 16384 blocks x 3 doubles = 384 KiB, so lattices of
// up to 16384 x 256 = 4,194,304 nodes are accepted; every GPU that loads the
// library keeps the array until the process exits.
namespace {
constexpr int kNoAllocMaxBlocks = 16384;
constexpr long long kNoAllocMaxNodes = static_cast<long long>(kNoAllocMaxBlocks) * 256;
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_scratch_addr[kNoAllocMaxDevices] = {};
}  // namespace

static __device__ __align__(256) double g_noalloc_mem_partials[3 * kNoAllocMaxBlocks];

// Device memory of the current GPU, or managed memory.
static bool device_accessible(const void* p) { return wk::pointer_kind(p) == wk::PtrKind::Here; }

extern "C" int d3q19_compute_momentum_exchange_forces_noalloc(const float f_post_collision[],
                                                               const uint8_t cell_type[], int nx, int ny, int nz,
                                                               float center_x, float center_y, float center_z,
                                                               float max_radius, float* fx_out, float* fy_out,
                                                               float* fz_out) {
    if (nx <= 0 || ny <= 0 || nz <= 0)
        return set_error(WAKE_ERR_INVALID, "momentum exchange (no-alloc): lattice sizes must be positive");
    const long long n = static_cast<long long>(nx) * ny * nz;
    if (n > kNoAllocMaxNodes)
        return set_error(WAKE_ERR_INVALID, "momentum exchange (no-alloc): " + std::to_string(n) +
                                               " nodes exceed the fixed scratch limit of " +
                                               std::to_string(kNoAllocMaxNodes) + " nodes");
    const void* ptrs[5] = {f_post_collision, cell_type, fx_out, fy_out, fz_out};
    for (const void* p : ptrs)
        if (!p || !device_accessible(p))
            return set_error(WAKE_ERR_INVALID, "momentum exchange (no-alloc): every pointer must be memory of the "
                                               "current GPU or managed memory (host buffers would need allocated "
                                               "staging)");
    int dev = 0;
    WK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        return set_error(WAKE_ERR_INVALID, "momentum exchange (no-alloc): device ordinal out of range");
    double* part = nullptr;
    {
        // one-time set-up per device, with that device current: the array's device address
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc_scratch_addr[dev]) {
            void* addr = nullptr;
            WK_CUDA(cudaGetSymbolAddress(&addr, g_noalloc_mem_partials));
            g_noalloc_scratch_addr[dev] = addr;
        }
        part = static_cast<double*>(g_noalloc_scratch_addr[dev]);
    }
    // one block per 256 nodes, so each block writes its own partial before the
    // final kernel reads it: nothing from an earlier call is read back
    const int nb = static_cast<int>((n + 255) / 256);
    k_mem_partials<19><<<nb, 256>>>(f_post_collision, cell_type, nx, ny, nz, center_x, center_y, center_z, max_radius,
                                     part);
    WK_CUDA(cudaGetLastError());
    k_mem_final<<<1, 32>>>(part, nb, fx_out, fy_out, fz_out);
    WK_CUDA(cudaGetLastError());
    WK_CUDA(cudaStreamSynchronize(0));
    return WAKE_OK;
}

// ---------------------------------------------------------------- immersed boundary (2D)
// Roma-Peskin 4-point regularised delta, one dimension (src/ispc/ibm_kernels.ispc:3-8).
__device__ __forceinline__ float peskin_1d(float r) {
    const float a = fabsf(r);
    if (a >= 2.0f) return 0.0f;
    return 0.25f * (1.0f + cosf(0.5f * 3.14159265358979323846f * a));
}

__device__ __forceinline__ int wrap_x(int px, int nx) { return (px % nx + nx) % nx; }

// Velocity at each marker: the 5 x 5 lattice neighbourhood weighted by the delta kernel,
// periodic in x, rows outside [0, ny) skipped (ibm_kernels.ispc:12-52). Thread per marker.
__global__ void k_ibm_interpolate(const float* __restrict__ ux, const float* __restrict__ uy,
                                  const float* __restrict__ mx_, const float* __restrict__ my_,
                                  float* __restrict__ mux, float* __restrict__ muy, int nx, int ny, int n) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    const float mx = mx_[m], my = my_[m];
    const int fx = static_cast<int>(floorf(mx)), fy = static_cast<int>(floorf(my));
    float iu = 0.0f, iv = 0.0f;
    for (int iy = -2; iy <= 2; ++iy) {
        const int py = fy + iy;
        if (py < 0 || py >= ny) continue;
        const float wy = peskin_1d(static_cast<float>(py) - my);
        const long long row = static_cast<long long>(py) * nx;
        for (int ix = -2; ix <= 2; ++ix) {
            const int px = fx + ix;
            const float w = peskin_1d(static_cast<float>(px) - mx) * wy;
            const long long e = row + wrap_x(px, nx);
            iu += w * ux[e];
            iv += w * uy[e];
        }
    }
    mux[m] = iu;
    muy[m] = iv;
}

// Force spreading (ibm_kernels.ispc:56-99): marker force times its arc length onto the 5 x 5
// neighbourhood, x weight from the delta kernel, y weight 0.25 (1 + cos(pi |py - my| / 2))
// without the kernel's |r| < 2 cut-off, as the reference computes it. One thread per (marker,
// stencil point); overlapping markers add with atomics, so sums may differ from the reference's
// marker-order loop in the last bits.
__global__ void k_ibm_spread(const float* __restrict__ mx_, const float* __restrict__ my_,
                             const float* __restrict__ mfx, const float* __restrict__ mfy,
                             const float* __restrict__ mds, float* __restrict__ gx, float* __restrict__ gy, int nx,
                             int ny, int n) {
    const long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (t >= 25ll * n) return;
    const int m = static_cast<int>(t / 25), k = static_cast<int>(t % 25);
    const float mx = mx_[m], my = my_[m];
    const int py = static_cast<int>(floorf(my)) - 2 + k / 5;
    if (py < 0 || py >= ny) return;
    const int px = static_cast<int>(floorf(mx)) - 2 + k % 5;
    const float fx = mfx[m] * mds[m], fy = mfy[m] * mds[m];
    const float wy = 0.25f * (1.0f + cosf(0.5f * 3.14159265358979323846f * fabsf(static_cast<float>(py) - my)));
    const float w = peskin_1d(static_cast<float>(px) - mx) * wy;
    const long long e = static_cast<long long>(py) * nx + wrap_x(px, nx);
    atomicAdd(gx + e, w * fx);
    atomicAdd(gy + e, w * fy);
}

extern "C" {

void d3q19_apply_curved_bfl(float f_dst[], const float f_src[], const int fluid_indices[], const int q_dirs[],
                            const float delta_fractions[], const float uw_x[], const float uw_y[], const float uw_z[],
                            int nx, int ny, int nz, int num_boundary_links) {
    if (num_boundary_links <= 0) return;
    const std::size_t n = static_cast<std::size_t>(nx) * ny * nz, nl = static_cast<std::size_t>(num_boundary_links);
    Stager s;
    s.inout(f_dst, 19 * n);
    s.in(f_src, 19 * n);
    s.in(fluid_indices, nl);
    s.in(q_dirs, nl);
    s.in(delta_fractions, nl);
    s.in(uw_x, nl);
    s.in(uw_y, nl);
    s.in(uw_z, nl);
    if (s.begin()) return;
    k_bfl<<<blocks_for(num_boundary_links), 256>>>(s.ptr<float>(0), s.ptr<float>(1), s.ptr<int>(2), s.ptr<int>(3),
                                                   s.ptr<float>(4), s.ptr<float>(5), s.ptr<float>(6), s.ptr<float>(7),
                                                   nx, ny, nz, num_boundary_links);
    s.end();
}

void thermal_collide_d2q9(const float g_in[], float g_out[], const uint8_t cell_type[], const float ux[],
                          const float uy[], float temperature[], float tau_T, int count) {
    if (count <= 0) return;
    const std::size_t n = static_cast<std::size_t>(count);
    Stager s;
    s.in(g_in, 9 * n);
    s.out(g_out, 9 * n);
    s.in(cell_type, n);
    s.in(ux, n);
    s.in(uy, n);
    s.inout(temperature, n);
    if (s.begin()) return;
    k_thermal_collide<<<blocks_for(count), 256>>>(s.ptr<float>(0), s.ptr<float>(1), s.ptr<uint8_t>(2), s.ptr<float>(3),
                                                  s.ptr<float>(4), s.ptr<float>(5), tau_T, count);
    s.end();
}
void thermal_compute_buoyancy_force_2d(const float temperature[], float gy_body[], float t_ref, float beta,
                                       float g_gravity, int count) {
    if (count <= 0) return;
    const std::size_t n = static_cast<std::size_t>(count);
    Stager s;
    s.in(temperature, n);
    s.inout(gy_body, n);
    if (s.begin()) return;
    k_buoyancy<<<blocks_for(count), 256>>>(s.ptr<float>(0), s.ptr<float>(1), t_ref, beta, g_gravity, count);
    s.end();
}
void thermal_apply_isothermal_wall(float g[], int nx, int ny, int y_wall, float t_wall) {
    if (nx <= 0 || ny <= 0 || y_wall < 0 || y_wall >= ny) return;
    Stager s;
    s.inout(g, 9 * static_cast<std::size_t>(nx) * ny);
    if (s.begin()) return;
    k_isothermal_wall<<<blocks_for(nx, 128), 128>>>(s.ptr<float>(0), nx, ny, y_wall, t_wall);
    s.end();
}

// src/ispc/ibm_kernels.ispc:12-22
void ibm_interpolate_velocity_2d(const float ux[], const float uy[], const float marker_x[], const float marker_y[],
                                 float marker_ux[], float marker_uy[], int nx, int ny, int num_markers) {
    if (num_markers <= 0 || nx <= 0 || ny <= 0) return;
    const std::size_t n = static_cast<std::size_t>(nx) * ny, nm = static_cast<std::size_t>(num_markers);
    Stager s;
    s.in(ux, n);
    s.in(uy, n);
    s.in(marker_x, nm);
    s.in(marker_y, nm);
    s.full_out(marker_ux, nm);
    s.full_out(marker_uy, nm);
    if (s.begin()) return;
    k_ibm_interpolate<<<blocks_for(num_markers, 128), 128>>>(s.ptr<float>(0), s.ptr<float>(1), s.ptr<float>(2),
                                                             s.ptr<float>(3), s.ptr<float>(4), s.ptr<float>(5), nx,
                                                             ny, num_markers);
    s.end();
}

// src/ispc/ibm_kernels.ispc:56-67
void ibm_spread_force_2d(const float marker_x[], const float marker_y[], const float marker_fx[],
                         const float marker_fy[], const float marker_ds[], float euler_gx[], float euler_gy[], int nx,
                         int ny, int num_markers) {
    if (num_markers <= 0 || nx <= 0 || ny <= 0) return;
    const std::size_t n = static_cast<std::size_t>(nx) * ny, nm = static_cast<std::size_t>(num_markers);
    Stager s;
    s.in(marker_x, nm);
    s.in(marker_y, nm);
    s.in(marker_fx, nm);
    s.in(marker_fy, nm);
    s.in(marker_ds, nm);
    s.inout(euler_gx, n);
    s.inout(euler_gy, n);
    if (s.begin()) return;
    k_ibm_spread<<<blocks_for(25ll * num_markers, 256), 256>>>(s.ptr<float>(0), s.ptr<float>(1), s.ptr<float>(2),
                                                               s.ptr<float>(3), s.ptr<float>(4), s.ptr<float>(5),
                                                               s.ptr<float>(6), nx, ny, num_markers);
    s.end();
}

// src/ispc/analytics_kernels.ispc:4-29
void compute_vorticity_2d(const float ux[], const float uy[], float vorticity[], int nx, int ny) {
    if (nx <= 0 || ny <= 0) return;
    const std::size_t n = static_cast<std::size_t>(nx) * ny;
    Stager s;
    s.in(ux, n);
    s.in(uy, n);
    s.full_out(vorticity, n);
    if (s.begin()) return;
    k_vorticity_2d<<<analytics_grid_3d(nx, ny, 1), analytics_block()>>>(s.ptr<float>(0), s.ptr<float>(1),
                                                                         s.ptr<float>(2), nx, ny);
    s.end();
}

// src/ispc/analytics_kernels.ispc:31-110
void compute_vorticity_and_q_criterion_3d(const float ux[], const float uy[], const float uz[], float omega_x[],
                                          float omega_y[], float omega_z[], float q_criterion[], int nx, int ny,
                                          int nz) {
    if (nx <= 0 || ny <= 0 || nz <= 0) return;
    const std::size_t n = static_cast<std::size_t>(nx) * ny * nz;
    Stager s;
    s.in(ux, n);
    s.in(uy, n);
    s.in(uz, n);
    s.full_out(omega_x, n);
    s.full_out(omega_y, n);
    s.full_out(omega_z, n);
    s.full_out(q_criterion, n);
    if (s.begin()) return;
    k_vorticity_q_3d<<<analytics_grid_3d(nx, ny, nz), analytics_block()>>>(
        s.ptr<float>(0), s.ptr<float>(1), s.ptr<float>(2), s.ptr<float>(3), s.ptr<float>(4), s.ptr<float>(5),
        s.ptr<float>(6), nx, ny, nz);
    s.end();
}

}  // extern "C"
