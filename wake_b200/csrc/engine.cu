// Host engine of the fused lattice update: one resident lattice per
// wake_grid handle (C ABI in include/wake_gpu.h).
//
// Mirrors the reference's LatticeGrid2D / LatticeGrid3D (src/grid/lattice_grid_2d.cpp,
// src/grid/lattice_grid_3d.cpp): same geometry setters, same step semantics,
// same readable state (f_src, rho, u, speed) after every step. The difference
// is where the work happens: the state lives in HBM as two SoA population
// buffers and one step is one kernel launch (stream_collide.cuh).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "analytics.cuh"
#include "engine.cuh"

namespace wk {

namespace {
thread_local std::string t_err;
thread_local int t_code = 0;
}  // namespace

unsigned long long next_geom_version() {
    static std::atomic<unsigned long long> counter{0};
    return ++counter;
}

int set_error(int code, const std::string& msg) {
    t_err = msg;
    t_code = code;
    return code;
}
void clear_error() {
    t_err.clear();
    t_code = 0;
}

cudaError_t launch_step_any(int Q, int coll, int store, bool les, const StepArgs& a, const Launch& L, bool fast) {
    if (Q == 9) return launch_step_q9(coll, store, les, a, L, fast);
    if (Q == 19) return launch_step_q19(coll, store, les, a, L, fast);
    return launch_step_q27(coll, store, les, a, L, fast);
}
cudaError_t launch_batch_any(int Q, int coll, int store, bool les, const BatchArgs& b, int tpb, cudaStream_t stream,
                             bool fast, bool idx32) {
    if (Q == 9) return launch_batch_q9(coll, store, les, b, tpb, stream, fast, idx32);
    if (Q == 19) return launch_batch_q19(coll, store, les, b, tpb, stream, fast, idx32);
    return launch_batch_q27(coll, store, les, b, tpb, stream, fast, idx32);
}
cudaError_t launch_tiles_any(int Q, int coll, int store, bool les, const StepArgs& a, const TileArgs& t,
                             cudaStream_t stream) {
    if (Q == 9) return launch_tiles_q9(coll, store, les, a, t, stream);
    if (Q == 19) return launch_tiles_q19(coll, store, les, a, t, stream);
    return launch_tiles_q27(coll, store, les, a, t, stream);
}
cudaError_t launch_rows_any(int Q, int store, bool les, const StepArgs& a, int rows, int tpb, cudaStream_t stream) {
    if (Q == 9) return launch_rows_q9(store, les, a, rows, tpb, stream);
    if (Q == 19) return launch_rows_q19(store, les, a, rows, tpb, stream);
    return launch_rows_q27(store, les, a, rows, tpb, stream);
}
cudaError_t launch_rows_pipe_any(int Q, int store, bool les, int cap, const StepArgs& a, const PipeArgs& p,
                                 cudaStream_t stream) {
    if (Q == 9) return launch_rows_pipe_q9(store, les, cap, a, p, stream);
    if (Q == 19) return launch_rows_pipe_q19(store, les, cap, a, p, stream);
    return launch_rows_pipe_q27(store, les, cap, a, p, stream);
}
cudaError_t launch_initial_any(int Q, int coll, int store, bool les, const float* f0, void* a, void* b,
                               const uint8_t* flags, const Geo& geo, const Physics& phys, const Launch& L) {
    if (Q == 9) return launch_initial_q9(coll, store, les, f0, a, b, flags, geo, phys, L);
    if (Q == 19) return launch_initial_q19(coll, store, les, f0, a, b, flags, geo, phys, L);
    return launch_initial_q27(coll, store, les, f0, a, b, flags, geo, phys, L);
}
cudaError_t launch_materialise_any(int Q, int store, const void* fin, const uint8_t* flags, const Geo& geo,
                                   const Links& links, const Physics& phys, const Out& out, const Launch& L,
                                   int direct, const Thermal& th) {
    if (Q == 9) return launch_materialise_q9(store, fin, flags, geo, links, phys, out, L, direct, th);
    if (Q == 19) return launch_materialise_q19(store, fin, flags, geo, links, phys, out, L, direct, th);
    return launch_materialise_q27(store, fin, flags, geo, links, phys, out, L, direct, th);
}
cudaError_t launch_flags_any(int Q, const uint8_t* types, uint8_t* flags, const Geo& geo, const FlagCfg& cfg,
                             const Launch& L) {
    if (Q == 9) return launch_flags_q9(types, flags, geo, cfg, L);
    if (Q == 19) return launch_flags_q19(types, flags, geo, cfg, L);
    return launch_flags_q27(types, flags, geo, cfg, L);
}
cudaError_t launch_seg_class_any(int Q, const uint8_t* flags, uint8_t* cls, const Geo& geo, long long nsegs,
                                 cudaStream_t stream) {
    if (Q == 9) return launch_seg_class_q9(flags, cls, geo, nsegs, stream);
    if (Q == 19) return launch_seg_class_q19(flags, cls, geo, nsegs, stream);
    return launch_seg_class_q27(flags, cls, geo, nsegs, stream);
}

// ---------------------------------------------------------------- small kernels
__global__ void k_link_marks(const int* __restrict__ node, int n, uint8_t* __restrict__ flags,
                             int* __restrict__ node_start) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = node[k];
    if (k == 0 || node[k - 1] != i) {
        node_start[i] = k;
        flags[i] = static_cast<uint8_t>((flags[i] | FL_BFL) & ~FL_FAST);
    }
}

// Shape rasterisers on the device: one thread per cell of the shape's bounding box marks the
// cells whose centre (integer coordinates) lies inside. The float rules are the reference
// setters' (LatticeGrid2D::set_solid_circle, lattice_grid_2d.cpp:143-158;
// LatticeGrid3D::set_solid_sphere, lattice_grid_3d.cpp:160-182) and the ellipse rule of
// wake_grid_set_solid_ellipse, with every rounding explicit so that the compiler cannot
// contract them: kind 0 circle (dx^2 + dy^2 <= r^2, every z), 1 sphere
// (dx^2 + dy^2 + dz^2 <= r^2), 2 rotated ellipse (u^2 / a^2 + v^2 / b^2 <= 1, every z).
__global__ void k_rasterise(uint8_t* __restrict__ types, int nx, int ny, wk::RasterBox b, wk::RasterShape sh) {
    const int bx = b.x1 - b.x0 + 1, by = b.y1 - b.y0 + 1, bz = b.z1 - b.z0 + 1;
    const long long n = static_cast<long long>(bx) * by * bz;
    for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < n;
         t += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = b.x0 + static_cast<int>(t % bx);
        const int y = b.y0 + static_cast<int>((t / bx) % by);
        const int z = b.z0 + static_cast<int>(t / (static_cast<long long>(bx) * by));
        const float dx = __fsub_rn(static_cast<float>(x), sh.c[0]);
        const float dy = __fsub_rn(static_cast<float>(y), sh.c[1]);
        bool inside;
        if (sh.kind == 0) {
            inside = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)) <= sh.p[0];
        } else if (sh.kind == 1) {
            const float dz = __fsub_rn(static_cast<float>(z), sh.c[2]);
            inside = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)) <= sh.p[0];
        } else {
            const float u = __fadd_rn(__fmul_rn(dx, sh.p[0]), __fmul_rn(dy, sh.p[1]));
            const float v = __fadd_rn(__fmul_rn(-dx, sh.p[1]), __fmul_rn(dy, sh.p[0]));
            inside = __fadd_rn(__fmul_rn(__fmul_rn(u, u), sh.p[2]), __fmul_rn(__fmul_rn(v, v), sh.p[3])) <= 1.0f;
        }
        if (inside) types[(static_cast<long long>(z) * ny + y) * nx + x] = CT_SOLID;
    }
}

// Row descriptors of the whole-row kernel (rows.cuh), one warp per row: ROW_FAST when every
// node of the row is a pure gather and Zou-He appears only as the inlet at x = 0 and the
// outlet at x = nx - 1 (with ROW_ZH_IN / ROW_ZH_OUT for those), 0 otherwise.
__global__ void k_row_kind(const uint8_t* __restrict__ flags, uint8_t* __restrict__ kind, int nx, int rows) {
    const int row = blockIdx.x * (blockDim.x >> 5) + static_cast<int>(threadIdx.x >> 5);
    if (row >= rows) return;
    const int lane = threadIdx.x & 31;
    const uint8_t* f = flags + static_cast<long long>(row) * nx;
    int ok = 1, zin = 0, zout = 0;
    for (int x = lane; x < nx; x += 32) {
        const uint8_t fl = f[x];
        ok &= (fl & FL_FAST) ? 1 : 0;
        if (fl & FL_ZH_IN) {
            if (x == 0) zin = 1;
            else ok = 0;
        }
        if (fl & FL_ZH_OUT) {
            if (x == nx - 1) zout = 1;
            else ok = 0;
        }
    }
    ok = __all_sync(0xffffffffu, ok);
    zin = __any_sync(0xffffffffu, zin);
    zout = __any_sync(0xffffffffu, zout);
    if (lane == 0)
        kind[row] = ok ? static_cast<uint8_t>(wk::ROW_FAST | (zin ? wk::ROW_ZH_IN : 0) | (zout ? wk::ROW_ZH_OUT : 0))
                       : static_cast<uint8_t>(0);
}

// Deterministic per-block partial sums for the diagnostics:
// [0] mass over Fluid, [1] kinetic energy over Fluid, [2] max speed over Fluid,
// [3] mass over every non-solid cell.
__global__ void k_diag_partials(const float* __restrict__ rho, const float* __restrict__ speed,
                                const uint8_t* __restrict__ flags, long long n, double* __restrict__ part) {
    __shared__ double s[4][256];
    double m = 0.0, ke = 0.0, mx = 0.0, mall = 0.0;
    for (long long i = blockIdx.x * 256ll + threadIdx.x; i < n; i += 256ll * gridDim.x) {
        const uint8_t t = flags[i] & FL_TYPE;
        if (t == CT_FLUID) {
            const double r = rho[i], sp = speed[i];
            m += r;
            ke += 0.5 * r * sp * sp;
            mx = fmax(mx, sp);
        }
        if (t != CT_SOLID) mall += rho[i];
    }
    s[0][threadIdx.x] = m;
    s[1][threadIdx.x] = ke;
    s[2][threadIdx.x] = mx;
    s[3][threadIdx.x] = mall;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s[0][threadIdx.x] += s[0][threadIdx.x + o];
            s[1][threadIdx.x] += s[1][threadIdx.x + o];
            s[2][threadIdx.x] = fmax(s[2][threadIdx.x], s[2][threadIdx.x + o]);
            s[3][threadIdx.x] += s[3][threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 4; ++c) part[4 * blockIdx.x + c] = s[c][0];
}

// Sum the per-node momentum-exchange contributions of one step in slot order
// (one block: thread t takes slots t, t + 256, ... in order, then a fixed tree)
// and append the force to the history. Launched after the step kernel that
// wrote the slots, on the same stream.
__global__ void __launch_bounds__(256) k_mem_reduce(const double* __restrict__ contrib, int n, unsigned* hist_step,
                                                    double* hist, int hist_cap) {
    mem_reduce_block(contrib, n, hist_step, hist, hist_cap);
}

// ---------------------------------------------------------------- device initialisation
// Initial populations f = feq(rho, u) written straight into the FP32 scratch,
// in the reference's float order (lattice_grid_2d.cpp:90-119) with every
// rounding explicit, so they equal the host formula bit for bit. The velocity is
// uniform, uniform plus seeded noise, or read per node from device arrays.
struct InitSpec {
    int mode;                 // 0 uniform, 1 uniform + noise, 2 per-node fields
    float rho, u[3];
    float amp;                // noise: u_a += amp * (2 r - 1), r a 24-bit uniform
    unsigned long long seed;  // SplitMix64 stream; component a of node i takes output offset + 1 + a*N + i
    long long offset;
    const float *rho_p, *ux_p, *uy_p, *uz_p;
};

__device__ __forceinline__ float splitmix_uniform24(unsigned long long seed, unsigned long long i) {
    // SplitMix64 (Steele, Lea & Flood, OOPSLA 2014): output i of the stream of `seed`, top 24 bits
    unsigned long long z = seed + i * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return __fmul_rn(static_cast<float>(z >> 40), 5.9604644775390625e-8f);  // * 2^-24
}

template <int Q>
__global__ void k_init_eq(float* __restrict__ f, long long pitch, long long n, int dims, InitSpec s) {
    using L = Lat<Q>;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        float rho = s.rho, u[3] = {s.u[0], s.u[1], s.u[2]};
        if (s.mode == 2) {
            rho = s.rho_p[i];
            u[0] = s.ux_p[i];
            u[1] = s.uy_p[i];
            u[2] = (s.uz_p && dims == 3) ? s.uz_p[i] : 0.f;
        } else if (s.mode == 1) {
            for (int a = 0; a < dims; ++a) {
                const float r = splitmix_uniform24(s.seed, static_cast<unsigned long long>(s.offset + 1 + a * n + i));
                u[a] = __fadd_rn(u[a], __fmul_rn(s.amp, __fsub_rn(__fmul_rn(2.0f, r), 1.0f)));
            }
        }
        const float usq = __fadd_rn(__fadd_rn(__fmul_rn(u[0], u[0]), __fmul_rn(u[1], u[1])), __fmul_rn(u[2], u[2]));
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float cu = __fadd_rn(__fadd_rn(__fmul_rn(float(L::cx(q)), u[0]), __fmul_rn(float(L::cy(q)), u[1])),
                                       __fmul_rn(float(L::cz(q)), u[2]));
            float t = __fadd_rn(1.0f, __fmul_rn(3.0f, cu));
            t = __fadd_rn(t, __fmul_rn(__fmul_rn(4.5f, cu), cu));
            t = __fsub_rn(t, __fmul_rn(1.5f, usq));
            f[q * pitch + i] = __fmul_rn(__fmul_rn(L::w(q), rho), t);
        }
    }
}

cudaError_t launch_init_eq(int Q, float* f, long long pitch, long long n, int dims, const InitSpec& s,
                           cudaStream_t stream) {
    const int blocks = static_cast<int>(std::min<long long>((n + 255) / 256, 148ll * 16));
    if (Q == 9) k_init_eq<9><<<blocks, 256, 0, stream>>>(f, pitch, n, dims, s);
    else if (Q == 19) k_init_eq<19><<<blocks, 256, 0, stream>>>(f, pitch, n, dims, s);
    else k_init_eq<27><<<blocks, 256, 0, stream>>>(f, pitch, n, dims, s);
    return cudaGetLastError();
}

// Fluid nodes with a Solid neighbour (x periodic, y / z in range, no wrap): the
// candidates of the curved-link builder. Each found node appends (index, direction
// mask) through one atomic counter; the host sorts the short list by node, so the
// order of the result does not depend on the launch.
template <int Q>
__global__ void k_solid_neighbours(const uint8_t* __restrict__ types, int nx, int ny, int nz,
                                   unsigned* __restrict__ count, int2* __restrict__ list, unsigned cap) {
    using L = Lat<Q>;
    const long long n = static_cast<long long>(nx) * ny * nz;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        if ((types[i] & FL_TYPE) != CT_FLUID) continue;
        const int x = static_cast<int>(i % nx), y = static_cast<int>((i / nx) % ny), z = static_cast<int>(i / (static_cast<long long>(nx) * ny));
        int mask = 0;
#pragma unroll
        for (int q = 1; q < Q; ++q) {
            const int xn = (x + L::cx(q) + nx) % nx, yn = y + L::cy(q), zn = z + L::cz(q);
            if (yn < 0 || yn >= ny || zn < 0 || zn >= nz) continue;
            if ((types[(static_cast<long long>(zn) * ny + yn) * nx + xn] & FL_TYPE) == CT_SOLID) mask |= 1 << q;
        }
        if (mask) {
            const unsigned slot = atomicAdd(count, 1u);
            if (slot < cap) list[slot] = make_int2(static_cast<int>(i), mask);
        }
    }
}

// Temperature populations at rest: g_q = w_q T (D2Q5 weights), from a per-node temperature.
__global__ void k_t5_equilibrium(const float* __restrict__ T, float* __restrict__ t5, long long pitch, long long n) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const float v = T[i];
#pragma unroll
        for (int q = 0; q < 5; ++q) t5[q * pitch + i] = __fmul_rn(D2Q5::w(q), v);
    }
}

// T = sum of the temperature populations (in the order q = 0..4).
__global__ void k_t5_sum(const float* __restrict__ t5, long long pitch, long long n, float* __restrict__ T) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        float t[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) t[q] = t5[q * pitch + i];
        T[i] = sum_t5(t);
    }
}

cudaError_t launch_link_marks(const int* link_node, int n_links, uint8_t* flags, int* node_start,
                              cudaStream_t stream) {
    if (n_links <= 0) return cudaSuccess;
    k_link_marks<<<(n_links + 255) / 256, 256, 0, stream>>>(link_node, n_links, flags, node_start);
    return cudaGetLastError();
}

}  // namespace wk

using namespace wk;

// ==================================================================== grid
namespace {

bool valid_grid(wake_grid* g) {
    if (!g) {
        set_error(WAKE_ERR_INVALID, "null wake_grid handle");
        return false;
    }
    return true;
}

long long idx3(const wake_grid* g, int x, int y, int z) {
    return (static_cast<long long>(z) * g->ny + y) * g->nx + x;
}

int upload_links(wake_grid* g);

// Bring the host copy of the cell types up to date (after device-side edits).
int host_types(wake_grid* g) {
    if (!g->types_dev_newer) return WAKE_OK;
    WK_CUDA(cudaMemcpyAsync(g->types.data(), g->d_types.p, g->N, cudaMemcpyDeviceToHost, g->stream));
    WK_CUDA(cudaStreamSynchronize(g->stream));
    g->types_dev_newer = false;
    return WAKE_OK;
}

// Bring the device copy up to date (after host-side edits).
int dev_types(wake_grid* g) {
    if (!g->types_host_newer) return WAKE_OK;
    WK_CUDA(cudaMemcpyAsync(g->d_types.p, g->types.data(), g->N, cudaMemcpyHostToDevice, g->stream));
    WK_CUDA(cudaStreamSynchronize(g->stream));  // the host vector may change right after
    g->types_host_newer = false;
    return WAKE_OK;
}

// Mark the cells of a shape solid on the device (k_rasterise); the host copy follows on demand.
int rasterise(wake_grid* g, const wk::RasterBox& b, const wk::RasterShape& sh) {
    if (b.x1 < b.x0 || b.y1 < b.y0 || b.z1 < b.z0) return WAKE_OK;  // the box misses the lattice
    const int r = dev_types(g);
    if (r) return r;
    const long long n = static_cast<long long>(b.x1 - b.x0 + 1) * (b.y1 - b.y0 + 1) * (b.z1 - b.z0 + 1);
    const int blocks = static_cast<int>(std::min<long long>((n + 255) / 256, 148ll * 8));
    k_rasterise<<<blocks, 256, 0, g->stream>>>(g->d_types.as<uint8_t>(), g->nx, g->ny, b, sh);
    WK_CUDA(cudaGetLastError());
    g->types_dev_newer = true;
    g->geom_dirty = true;
    return WAKE_OK;
}

// Upload types and links, rebuild flags and momentum-exchange slots.
int rebuild_flags(wake_grid* g) {
    if (g->links_dirty) {
        const int r = upload_links(g);
        if (r) return r;
        g->links_dirty = false;
    }
    {
        const int r = dev_types(g);
        if (r) return r;
    }
    FlagCfg cfg{};
    cfg.zh_rule = (g->Q == 9) ? 1 : 2;
    cfg.inflow = g->inflow;
    cfg.outflow = g->outflow;
    cfg.mem_enabled = g->mem_on;
    for (int a = 0; a < 3; ++a) cfg.center[a] = g->center[a];
    cfg.r_max = g->rmax;
    cfg.r_max_sq = g->rmax * g->rmax;
    const Geo geo = g->geo();
    WK_CUDA(launch_flags_any(g->Q, g->d_types.as<uint8_t>(), g->d_flags.as<uint8_t>(), geo, cfg, g->launch()));
    const int nl = g->dev_links;
    if (nl > 0) {
        WK_CUDA(g->d_nodestart.ensure(sizeof(int) * g->N));
        WK_CUDA(cudaMemsetAsync(g->d_nodestart.p, 0xff, sizeof(int) * g->N, g->stream));
        WK_CUDA(launch_link_marks(g->d_link_node.as<int>(), nl, g->d_flags.as<uint8_t>(), g->d_nodestart.as<int>(),
                                  g->stream));
    }
    // split the rows into SEG-node segments for the two step kernels
    {
        const int nseg = (g->nx + SEG - 1) / SEG;
        const long long nsegs = static_cast<long long>(g->rows) * nseg;
        if (nsegs >= (1ll << 32)) return set_error(WAKE_ERR_INVALID, "lattice too large for 32-bit segment numbers");
        DevMem cls;
        WK_CUDA(cls.ensure(static_cast<std::size_t>(nsegs)));
        WK_CUDA(launch_seg_class_any(g->Q, g->d_flags.as<uint8_t>(), cls.as<uint8_t>(), geo, nsegs, g->stream));
        std::vector<uint8_t> h(static_cast<std::size_t>(nsegs));
        WK_CUDA(cudaMemcpyAsync(h.data(), cls.p, h.size(), cudaMemcpyDeviceToHost, g->stream));
        WK_CUDA(cudaStreamSynchronize(g->stream));
        cls.release();
        // general segments; pure-gather spans: whole rows, or the runs of pure-gather
        // segments of the rows that hold general segments
        if (g->th.on)  // the coupled temperature runs on the general per-node path only
            for (auto& c : h) c = static_cast<uint8_t>(c & ~1u);
        std::vector<unsigned> gen;
        std::vector<uint4> spans, mixed_spans;
        std::vector<uint8_t> row_fast(static_cast<std::size_t>(g->rows), 1);
        for (long long e = 0; e < nsegs; ++e) {
            if (h[e] & 1) continue;
            row_fast[static_cast<std::size_t>(e / nseg)] = 0;
            if (h[e] & 4) continue;  // every node solid: frozen in both buffers, nothing to launch
            gen.push_back(static_cast<unsigned>(e));
        }
        for (int r = 0; r < g->rows; ++r) {
            if (row_fast[r]) {
                spans.push_back(make_uint4(0u, static_cast<unsigned>(r), 0u, static_cast<unsigned>(g->nx)));
                continue;
            }
            for (int sg = 0; sg < nseg;) {
                if (!(h[static_cast<long long>(r) * nseg + sg] & 1)) {
                    ++sg;
                    continue;
                }
                int s1 = sg + 1;
                while (s1 < nseg && (h[static_cast<long long>(r) * nseg + s1] & 1)) ++s1;
                const uint4 sp = make_uint4(0u, static_cast<unsigned>(r), static_cast<unsigned>(sg * SEG),
                                            static_cast<unsigned>(std::min(g->nx, s1 * SEG)));
                spans.push_back(sp);
                mixed_spans.push_back(sp);
                sg = s1;
            }
        }
        g->n_fast = static_cast<int>(spans.size());
        g->n_gen = static_cast<int>(gen.size());
        WK_CUDA(g->d_fast_rows.ensure(sizeof(uint4) * std::max<std::size_t>(1, spans.size())));
        WK_CUDA(g->d_gen_rows.ensure(sizeof(unsigned) * std::max<std::size_t>(1, gen.size())));
        if (!spans.empty())
            WK_CUDA(cudaMemcpyAsync(g->d_fast_rows.p, spans.data(), sizeof(uint4) * spans.size(),
                                    cudaMemcpyHostToDevice, g->stream));
        if (!gen.empty())
            WK_CUDA(cudaMemcpyAsync(g->d_gen_rows.p, gen.data(), sizeof(unsigned) * gen.size(), cudaMemcpyHostToDevice,
                                    g->stream));
        // momentum-exchange slots: per general segment and 32-node chunk, the number of
        // FL_MEM nodes before it (node order), so slots are dense and ordered
        g->warps_per_row = SEG / 32;
        g->n_mem_nodes = 0;
        std::vector<int> warp_base;
        if (g->mem_on) {
            std::vector<uint8_t> fl(g->N);
            WK_CUDA(cudaMemcpyAsync(fl.data(), g->d_flags.p, g->N, cudaMemcpyDeviceToHost, g->stream));
            WK_CUDA(cudaStreamSynchronize(g->stream));
            warp_base.assign(std::max<std::size_t>(1, gen.size() * g->warps_per_row), 0);
            int count = 0;
            for (std::size_t k = 0; k < gen.size(); ++k) {
                const long long row = gen[k] / nseg, x0 = (gen[k] % nseg) * SEG;
                for (int c = 0; c < g->warps_per_row; ++c) {
                    warp_base[k * g->warps_per_row + c] = count;
                    const long long xa = x0 + 32 * c, xe = std::min<long long>(g->nx, xa + 32);
                    for (long long x = xa; x < xe; ++x) count += (fl[row * g->nx + x] & FL_MEM) ? 1 : 0;
                }
            }
            g->n_mem_nodes = count;
            WK_CUDA(g->d_warp_base.ensure(sizeof(int) * warp_base.size()));
            WK_CUDA(cudaMemcpyAsync(g->d_warp_base.p, warp_base.data(), sizeof(int) * warp_base.size(),
                                    cudaMemcpyHostToDevice, g->stream));
            WK_CUDA(g->d_contrib.ensure(sizeof(double) * 3 * std::max(1, count)));
        }
        // persistent-kernel work: tiles of consecutive all-pure-gather rows of one z plane
        // (at most TILE_NODES nodes), the general segments with their slot entry, and the
        // pure-gather runs of the other rows
        {
            const int per_tile = std::max(1, TILE_NODES / g->nx);
            std::vector<uint4> tiles, gen4;
            for (int r = 0; r < g->rows;) {
                if (!row_fast[r]) {
                    ++r;
                    continue;
                }
                const int z = r / g->ny, y0 = r % g->ny;
                int cnt = 1;
                while (cnt < per_tile && r + cnt < g->rows && row_fast[r + cnt] && (r + cnt) / g->ny == z) ++cnt;
                tiles.push_back(make_uint4(0u, (static_cast<unsigned>(z) << 16) | static_cast<unsigned>(y0),
                                           static_cast<unsigned>(cnt), 0u));
                r += cnt;
            }
            for (std::size_t k = 0; k < gen.size(); ++k)
                gen4.push_back(make_uint4(0u, gen[k], static_cast<unsigned>(k), 0u));
            WK_CUDA(g->d_tiles.ensure(sizeof(uint4) * std::max<std::size_t>(1, tiles.size())));
            WK_CUDA(g->d_gen4.ensure(sizeof(uint4) * std::max<std::size_t>(1, gen4.size())));
            WK_CUDA(g->d_mixed.ensure(sizeof(uint4) * std::max<std::size_t>(1, mixed_spans.size())));
            if (!tiles.empty())
                WK_CUDA(cudaMemcpyAsync(g->d_tiles.p, tiles.data(), sizeof(uint4) * tiles.size(), cudaMemcpyHostToDevice,
                                        g->stream));
            if (!gen4.empty())
                WK_CUDA(cudaMemcpyAsync(g->d_gen4.p, gen4.data(), sizeof(uint4) * gen4.size(), cudaMemcpyHostToDevice,
                                        g->stream));
            if (!mixed_spans.empty())
                WK_CUDA(cudaMemcpyAsync(g->d_mixed.p, mixed_spans.data(), sizeof(uint4) * mixed_spans.size(),
                                        cudaMemcpyHostToDevice, g->stream));
            WK_CUDA(cudaStreamSynchronize(g->stream));  // the host vectors go out of scope
            g->n_tiles = static_cast<int>(tiles.size());
            g->n_tile_gen = static_cast<int>(gen4.size());
            g->n_mixed = static_cast<int>(mixed_spans.size());
            g->h_tiles = std::move(tiles);
            g->h_gen4 = std::move(gen4);
            g->h_mixed = std::move(mixed_spans);
        }
        // whole-row kernel: one descriptor byte per row (rows.cuh), kept only where it agrees
        // with the segment classes (ROW_FAST exactly on the rows whose segments are all pure)
        {
            WK_CUDA(g->d_row_kind.ensure(static_cast<std::size_t>(g->rows)));
            const int rows_per_block = 8;
            k_row_kind<<<(g->rows + rows_per_block - 1) / rows_per_block, 32 * rows_per_block, 0, g->stream>>>(
                g->d_flags.as<uint8_t>(), g->d_row_kind.as<uint8_t>(), g->nx, g->rows);
            WK_CUDA(cudaGetLastError());
            std::vector<uint8_t> kinds(static_cast<std::size_t>(g->rows));
            WK_CUDA(cudaMemcpyAsync(kinds.data(), g->d_row_kind.p, kinds.size(), cudaMemcpyDeviceToHost, g->stream));
            WK_CUDA(cudaStreamSynchronize(g->stream));
            int n_rf = 0;
            bool agree = true;
            for (int r = 0; r < g->rows; ++r) {
                const bool k = (kinds[r] & wk::ROW_FAST) != 0;
                agree = agree && (k == (row_fast[r] != 0));
                n_rf += k ? 1 : 0;
            }
            g->n_row_fast = agree ? n_rf : 0;
            g->row_fast_nodes = static_cast<long long>(g->n_row_fast) * g->nx;
            std::vector<unsigned> list;
            if (g->n_row_fast > 0 && g->rows < (1 << 28)) {
                list.reserve(static_cast<std::size_t>(g->n_row_fast));
                for (int r = 0; r < g->rows; ++r)
                    if (kinds[r] & wk::ROW_FAST) list.push_back(static_cast<unsigned>(r) | (unsigned(kinds[r]) << 28));
                WK_CUDA(g->d_row_list.ensure(sizeof(unsigned) * list.size()));
                WK_CUDA(cudaMemcpyAsync(g->d_row_list.p, list.data(), sizeof(unsigned) * list.size(),
                                        cudaMemcpyHostToDevice, g->stream));
                WK_CUDA(cudaStreamSynchronize(g->stream));  // the host list goes out of scope
            }
        }
        g->h_fast_rows = std::move(spans);
        g->h_gen_rows = std::move(gen);
    }
    g->geom_version = next_geom_version();
    g->geom_dirty = false;
    g->invalidate_graph();
    return WAKE_OK;
}

// Upload the links (sorted by fluid node) and their moving-wall terms.
int upload_links(wake_grid* g) {
    const int n = static_cast<int>(g->link_node.size());
    g->dev_links = 0;
    if (n == 0) return WAKE_OK;
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return g->link_node[a] < g->link_node[b]; });
    std::vector<int> node(n), q(n);
    std::vector<float> delta(n), mom(n);
    for (int j = 0; j < n; ++j) {
        const int k = order[j];
        node[j] = g->link_node[k];
        q[j] = g->link_q[k];
        delta[j] = g->link_delta[k];
        const int qq = q[j];
        const float ci_uw = float(g->lat.cx[qq]) * g->link_uw[3 * k] + float(g->lat.cy[qq]) * g->link_uw[3 * k + 1] +
                            float(g->lat.cz[qq]) * g->link_uw[3 * k + 2];
        // d3q19_curved.ispc:57 (delta < 1/2) and :62 (delta >= 1/2)
        mom[j] = (delta[j] < 0.5f) ? 2.0f * g->lat.w[qq] * 1.0f * 3.0f * ci_uw
                                   : (1.0f / delta[j]) * g->lat.w[qq] * 1.0f * 3.0f * ci_uw;
    }
    WK_CUDA(g->d_link_node.ensure(sizeof(int) * n));
    WK_CUDA(g->d_link_q.ensure(sizeof(int) * n));
    WK_CUDA(g->d_link_delta.ensure(sizeof(float) * n));
    WK_CUDA(g->d_link_mom.ensure(sizeof(float) * n));
    WK_CUDA(cudaMemcpyAsync(g->d_link_node.p, node.data(), sizeof(int) * n, cudaMemcpyHostToDevice, g->stream));
    WK_CUDA(cudaMemcpyAsync(g->d_link_q.p, q.data(), sizeof(int) * n, cudaMemcpyHostToDevice, g->stream));
    WK_CUDA(cudaMemcpyAsync(g->d_link_delta.p, delta.data(), sizeof(float) * n, cudaMemcpyHostToDevice, g->stream));
    WK_CUDA(cudaMemcpyAsync(g->d_link_mom.p, mom.data(), sizeof(float) * n, cudaMemcpyHostToDevice, g->stream));
    WK_CUDA(cudaStreamSynchronize(g->stream));
    g->dev_links = n;
    return WAKE_OK;
}

Out scratch_out(wake_grid* g, bool want_f, bool want_macro) {
    Out o{};
    if (want_f) o.f = g->m_f.as<float>();
    if (want_macro) {
        o.rho = g->m_rho.as<float>();
        o.ux = g->m_ux.as<float>();
        o.uy = g->m_uy.as<float>();
        o.uz = g->m_uz.as<float>();
        o.speed = g->m_speed.as<float>();
    }
    return o;
}

int ensure_macro(wake_grid* g) {
    const std::size_t b = sizeof(float) * g->N;
    WK_CUDA(g->m_rho.ensure(b));
    WK_CUDA(g->m_ux.ensure(b));
    WK_CUDA(g->m_uy.ensure(b));
    WK_CUDA(g->m_uz.ensure(b));
    WK_CUDA(g->m_speed.ensure(b));
    return WAKE_OK;
}

// Temperature view of the current state for the readers: the current post-collision
// temperature buffer (its sum is the temperature of the reported step). Before the
// first step the fields are reported as initialised, without the buoyancy shift.
Thermal state_thermal(const wake_grid* g) {
    Thermal t = g->th;
    t.on = g->th.on && g->k > 0;
    t.tin = t.on ? g->tbuf(g->cur) : nullptr;
    t.tout = nullptr;
    return t;
}

// Physics for reporting the state after the last step: the moments carry the
// Guo shift of the body force that step used (lattice_grid_2d.cpp:257-259);
// before any step there is none (initialize() stores the fields as given).
Physics report_phys(const wake_grid* g) {
    Physics p = g->phys;
    for (int a = 0; a < 3; ++a) p.g[a] = g->k > 0 ? g->last_step_g[a] : 0.f;
    return p;
}

// Bring the reference-visible f^k (into m_f) and/or its moments (into the
// macro scratch) up to date. Uses the current device flags, i.e. the geometry
// the last step ran with, as the reference's f_src is untouched by setters.
int materialise(wake_grid* g, bool want_f, bool want_macro) {
    if (want_macro) {
        const int r = ensure_macro(g);
        if (r) return r;
    }
    const Physics rp = report_phys(g);
    if (g->mf_valid) {
        if (!want_macro) return WAKE_OK;
        const Out o = scratch_out(g, false, true);
        WK_CUDA(launch_materialise_any(g->Q, STORE_F32, g->m_f.p, g->d_flags.as<uint8_t>(), g->geo(), g->links(), rp, o,
                                       g->launch(), 1, state_thermal(g)));
        return WAKE_OK;
    }
    if (want_f) WK_CUDA(g->m_f.ensure(sizeof(float) * g->Q * g->pitch));
    const Out o = scratch_out(g, want_f, want_macro);
    // before the first step the other buffer holds f^0 itself (k_initial), read in place;
    // after it, f^k is re-gathered from g^{k-1}
    WK_CUDA(launch_materialise_any(g->Q, g->storage, g->buf(1 - g->cur), g->d_flags.as<uint8_t>(), g->geo(),
                                   g->links(), rp, o, g->launch(), g->k == 0 ? 1 : 0, state_thermal(g)));
    if (want_f) g->mf_valid = true;
    return WAKE_OK;
}

// Collide f^k (FP32 in m_f) with the current parameters: A <- Collide(f^k), B <- f^k.
int initial_from_scratch(wake_grid* g) {
    if (g->th.on) {
        // the temperature has no re-derivable pre-collision state, so it collides from its start only
        if (g->k != 0 || !g->mt_valid)
            return set_error(WAKE_ERR_INVALID, "a coupled temperature collides from its initial state only: "
                                               "model, tau and body force are fixed once a thermal grid has stepped");
        WK_CUDA(launch_initial_thermal_q9(g->collision, g->storage, g->les != 0, g->m_f.as<float>(), g->m_t.as<float>(),
                                          g->A.p, g->B.p, g->tbuf(0), g->tbuf(1), g->d_flags.as<uint8_t>(), g->geo(),
                                          g->phys, g->th, g->launch()));
    } else {
        WK_CUDA(launch_initial_any(g->Q, g->collision, g->storage, g->les != 0, g->m_f.as<float>(), g->A.p, g->B.p,
                                   g->d_flags.as<uint8_t>(), g->geo(), g->phys, g->launch()));
    }
    g->cur = 0;
    g->pending = false;
    for (int a = 0; a < 3; ++a) g->collided_g[a] = g->phys.g[a];
    g->invalidate_graph();
    return WAKE_OK;
}

// Called at the start of a step (phys holds that step's parameters). If the
// geometry or any collision parameter changed, f^k is re-derived with the old
// flags, the flags rebuilt and f^k re-collided with the new parameters.
int apply_geometry(wake_grid* g) {
    if (!g->geom_dirty) return WAKE_OK;
    if (!g->mf_valid) {
        const int r = materialise(g, true, false);  // f^k under the old flags
        if (r) return r;
    }
    const int r = rebuild_flags(g);
    if (r) return r;
    g->pending = true;
    return WAKE_OK;
}

int prepare(wake_grid* g) {
    const int r = apply_geometry(g);
    if (r) return r;
    if (!g->pending) return WAKE_OK;
    if (!g->mf_valid) {
        const int r2 = materialise(g, true, false);
        if (r2) return r2;
    }
    return initial_from_scratch(g);
}

// The FP32 scratch now holds f^0: the next step collides it (fresh run, step 0).
void f0_written(wake_grid* g) {
    g->mf_valid = true;
    g->pending = true;
    g->k = 0;
    g->invalidate_graph();
}

int upload_f0(wake_grid* g, const float* f, cudaMemcpyKind kind) {
    WK_CUDA(g->m_f.ensure(sizeof(float) * g->Q * g->pitch));
    WK_CUDA(cudaMemcpy2DAsync(g->m_f.p, sizeof(float) * g->pitch, f, sizeof(float) * g->N, sizeof(float) * g->N,
                              g->Q, kind, g->stream));
    WK_CUDA(cudaStreamSynchronize(g->stream));
    f0_written(g);
    return WAKE_OK;
}

int init_on_device(wake_grid* g, const InitSpec& s) {
    WK_CUDA(g->m_f.ensure(sizeof(float) * g->Q * g->pitch));
    WK_CUDA(launch_init_eq(g->Q, g->m_f.as<float>(), g->pitch, g->N, g->D, s, g->stream));
    f0_written(g);
    return WAKE_OK;
}

int do_steps(wake_grid* g, int n) {
    for (int s = 0; s < n; ++s) {
        StepArgs a = wk::grid_step_args(g);
        a.fin = g->buf(g->cur);
        a.fout = g->buf(1 - g->cur);
        a.th.tin = g->tbuf(g->cur);
        a.th.tout = g->tbuf(1 - g->cur);
        if (g->use_tiles()) {
            // one persistent launch for the general rows and the staged pure-gather tiles,
            // then the momentum-exchange sum of the slots it wrote
            const TileArgs t{g->d_tiles.as<uint4>(), g->n_tiles, g->d_gen4.as<uint4>(), g->n_tile_gen, nullptr, 0,
                             g->d_mixed.as<uint4>(), g->n_mixed};
            const bool timed = g->time_bulk;
            if (timed) {
                while (g->t_ev.size() < g->t_used + 2) {
                    cudaEvent_t e = nullptr;
                    WK_CUDA(cudaEventCreate(&e));
                    g->t_ev.push_back(e);
                }
                WK_CUDA(cudaEventRecord(g->t_ev[g->t_used], g->stream));
            }
            WK_CUDA(launch_tiles_any(g->Q, g->collision, g->storage, g->les != 0, a, t, g->stream));
            if (timed) {
                WK_CUDA(cudaEventRecord(g->t_ev[g->t_used + 1], g->stream));
                g->t_used += 2;
            }
            if (g->mem_on) {
                k_mem_reduce<<<1, 256, 0, g->stream>>>(a.mem.contrib, a.mem.n_nodes, a.mem.hist_step, a.mem.hist,
                                                       a.mem.hist_cap);
                WK_CUDA(cudaGetLastError());
            }
            g->cur ^= 1;
            g->mf_valid = false;
            for (int c = 0; c < 3; ++c) g->last_step_g[c] = g->phys.g[c];
            ++g->k;
            continue;
        }
        // The pure-gather rows and the rows with boundaries / momentum exchange write
        // disjoint nodes of the output, so the small general launch runs on a forked
        // stream beside the bulk launch (a fork/join that CUDA graph capture keeps).
        StepArgs gen = a;
        gen.rows = g->d_gen_rows.as<unsigned>();
        gen.nrows = g->n_gen;
        // with the whole-row kernel, the pure-gather runs of the other rows go beside the general segments
        const bool pipe_k = g->use_pipe();
        const bool rows_k = pipe_k || g->use_rows();
        StepArgs part = a;
        part.spans = g->d_mixed.as<uint4>();
        part.nspans = rows_k ? g->n_mixed : 0;
        a.spans = g->d_fast_rows.as<uint4>();
        a.nspans = rows_k ? 0 : g->n_fast;
        a.row_kind = g->d_row_kind.as<uint8_t>();
        const bool bulk = rows_k || g->n_fast > 0;
        const bool fork = bulk && (g->n_gen > 0 || part.nspans > 0);
        Launch side = g->launch();
        if (fork) {
            side.stream = g->side;
            WK_CUDA(cudaEventRecord(g->ev_fork, g->stream));
            WK_CUDA(cudaStreamWaitEvent(g->side, g->ev_fork, 0));
        }
        WK_CUDA(launch_step_any(g->Q, g->collision, g->storage, g->les != 0, gen, side, false));
        if (part.nspans > 0) WK_CUDA(launch_step_any(g->Q, g->collision, g->storage, g->les != 0, part, side, true));
        if (g->mem_on) {
            // the step's force from the slots the general launch just wrote (zero if none)
            k_mem_reduce<<<1, 256, 0, side.stream>>>(a.mem.contrib, a.mem.n_nodes, a.mem.hist_step, a.mem.hist,
                                                     a.mem.hist_cap);
            WK_CUDA(cudaGetLastError());
        }
        const bool timed = g->time_bulk && (rows_k || a.nspans > 0);
        if (timed) {
            while (g->t_ev.size() < g->t_used + 2) {
                cudaEvent_t e = nullptr;
                WK_CUDA(cudaEventCreate(&e));
                g->t_ev.push_back(e);
            }
            WK_CUDA(cudaEventRecord(g->t_ev[g->t_used], g->stream));
        }
        if (pipe_k) {
            const wk::PipeArgs pa{g->d_row_list.as<unsigned>(), g->n_row_fast};
            WK_CUDA(launch_rows_pipe_any(g->Q, g->storage, g->les != 0, g->pipe_cap(), a, pa, g->stream));
        } else if (rows_k) {
            WK_CUDA(launch_rows_any(g->Q, g->storage, g->les != 0, a, g->rows, g->tpb_rows(), g->stream));
        } else {
            WK_CUDA(launch_step_any(g->Q, g->collision, g->storage, g->les != 0, a, g->launch(), true));
        }
        if (timed) {
            WK_CUDA(cudaEventRecord(g->t_ev[g->t_used + 1], g->stream));
            g->t_used += 2;
        }
        if (fork) {
            WK_CUDA(cudaEventRecord(g->ev_join, g->side));
            WK_CUDA(cudaStreamWaitEvent(g->stream, g->ev_join, 0));
        }
        g->cur ^= 1;
        g->mf_valid = false;
        for (int c = 0; c < 3; ++c) g->last_step_g[c] = g->phys.g[c];
        ++g->k;
    }
    return WAKE_OK;
}

}  // namespace

namespace wk {

bool grid_valid(wake_grid* g) { return valid_grid(g); }
int grid_prepare(wake_grid* g) { return prepare(g); }

StepArgs grid_step_args(const wake_grid* g) {
    StepArgs a{};
    a.flags = g->d_flags.as<uint8_t>();
    a.status = g->d_status.as<unsigned>();
    a.geo = g->geo();
    a.links = g->links();
    a.mem.enabled = g->mem_on;
    if (g->mem_on) {
        for (int c = 0; c < 3; ++c) a.mem.center[c] = g->center[c];
        a.mem.r_max = g->rmax;
        a.mem.r_max_sq = g->rmax * g->rmax;
        a.mem.warp_base = g->d_warp_base.as<int>();
        a.mem.warps_per_row = g->warps_per_row;
        a.mem.contrib = g->d_contrib.as<double>();
        a.mem.n_nodes = g->n_mem_nodes;
        a.mem.hist_step = g->d_counters.as<unsigned>() + 1;
        a.mem.hist = g->d_hist.as<double>();
        a.mem.hist_cap = g->hist_cap;
    }
    a.phys = g->phys;
    a.th = g->th;
    return a;
}

void grid_advanced(wake_grid* g, int n) {
    if (n <= 0) return;
    g->cur ^= (n & 1);
    g->k += n;
    g->mf_valid = false;
    for (int c = 0; c < 3; ++c) g->last_step_g[c] = g->phys.g[c];
}

int grid_check_status(wake_grid* g) { return wake_grid_synchronize(g); }

}  // namespace wk

// ==================================================================== C ABI
extern "C" {

const char* wake_gpu_last_error(void) { return t_err.c_str(); }
int wake_gpu_last_error_code(void) { return t_code; }
void wake_gpu_clear_error(void) { clear_error(); }
const char* wake_gpu_version(void) { return "wake_b200 0.1.0 (sm_100a)"; }

wake_grid* wake_grid_create(int q, int nx, int ny, int nz, float tau, int storage) {
    if (!(q == 9 || q == 19 || q == 27) || nx < 1 || ny < 1 || nz < 1 || (q == 9 && nz != 1) ||
        storage < 0 || storage > 3 || !(tau > 0.5f)) {
        set_error(WAKE_ERR_INVALID, "wake_grid_create: invalid lattice, size, tau or storage");
        return nullptr;
    }
    const long long N = static_cast<long long>(nx) * ny * nz;
    if (N >= (1ll << 31) || ny > 65535 || nz > 65535) {
        set_error(WAKE_ERR_INVALID, "wake_grid_create: more than 2^31 - 1 nodes, or ny / nz above 65535");
        return nullptr;
    }
    auto* g = new wake_grid(q);
    g->Q = q;
    g->D = g->lat.D;
    g->nx = nx;
    g->ny = ny;
    g->nz = nz;
    g->N = N;
    g->pitch = (N + 63) / 64 * 64;
    g->storage = storage;
    g->elem = storage == WAKE_STORE_F32 ? 4 : 2;
    g->phys.tau = tau;
    g->phys.lambda_trt = 0.25f;
    g->phys.tau_bulk = (q == 9) ? 1.63f : (q == 19 ? 1.19f : 1.0f);
    g->phys.cs_smag = 0.14f;
    g->phys.s3 = 1.0f;
    g->phys.s4 = 1.0f;
    g->phys.mrt_exact = 0;
    g->types.assign(N, WAKE_CELL_FLUID);
    g->choose_block(0);
    cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) g->own_stream = true;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->ev_join, cudaEventDisableTiming);
    const std::size_t sb = g->elem * static_cast<std::size_t>(q) * g->pitch;
    if (e == cudaSuccess) e = g->A.ensure(sb);
    if (e == cudaSuccess) e = g->B.ensure(sb);
    if (e == cudaSuccess) e = g->d_types.ensure(N);
    if (e == cudaSuccess) e = g->d_flags.ensure(N);
    if (e == cudaSuccess) e = g->d_status.ensure(sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemsetAsync(g->d_status.p, 0, sizeof(unsigned), g->stream);
    if (e != cudaSuccess) {
        set_error(e == cudaErrorMemoryAllocation ? WAKE_ERR_NOMEM : WAKE_ERR_CUDA,
                  std::string("wake_grid_create: ") + cudaGetErrorString(e));
        delete g;
        return nullptr;
    }
    if (wake_grid_initialize(g, 1.0f, 0.f, 0.f, 0.f) != WAKE_OK) {
        delete g;
        return nullptr;
    }
    return g;
}

void wake_grid_destroy(wake_grid* g) {
    if (!g) return;
    if (g->stream) cudaStreamSynchronize(g->stream);
    delete g;
}

int wake_grid_set_stream(wake_grid* g, void* stream) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    WK_CUDA(cudaStreamSynchronize(g->stream));
    if (g->own_stream) cudaStreamDestroy(g->stream);
    g->own_stream = false;
    if (stream) {
        g->stream = static_cast<cudaStream_t>(stream);
    } else {
        WK_CUDA(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
        g->own_stream = true;
    }
    g->invalidate_graph();
    return WAKE_OK;
}

int wake_grid_set_model(wake_grid* g, int collision, int les, float cs_smag, float lambda_trt, float tau_bulk,
                        int mrt_exact, float s3, float s4) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    if (collision < 0 || collision > 2 || !(tau_bulk > 0.5f) || !(lambda_trt > 0.f))
        return set_error(WAKE_ERR_INVALID, "wake_grid_set_model: invalid collision, tau_bulk or lambda");
    g->collision = collision;
    g->les = les ? 1 : 0;
    g->phys.cs_smag = cs_smag;
    g->phys.lambda_trt = lambda_trt;
    g->phys.tau_bulk = tau_bulk;
    g->phys.mrt_exact = mrt_exact ? 1 : 0;
    g->phys.s3 = s3;
    g->phys.s4 = s4;
    g->pending = true;  // the next step collides f^k with the new model
    g->invalidate_graph();
    return WAKE_OK;
}

int wake_grid_set_relaxation_time(wake_grid* g, float tau) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    if (!(tau > 0.5f)) return set_error(WAKE_ERR_INVALID, "tau must exceed 1/2");
    g->phys.tau = tau;
    g->pending = true;
    g->invalidate_graph();
    return WAKE_OK;
}

int wake_grid_set_cell_type(wake_grid* g, int x, int y, int z, int type) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    // out-of-range coordinates are ignored, as in LatticeGrid2D::set_cell_type (lattice_grid_2d.cpp:122-126)
    if (x < 0 || x >= g->nx || y < 0 || y >= g->ny || z < 0 || z >= g->nz) return WAKE_OK;
    const int r = host_types(g);
    if (r) return r;
    g->types[idx3(g, x, y, z)] = static_cast<uint8_t>(type & FL_TYPE);
    g->types_host_newer = true;
    g->geom_dirty = true;
    return WAKE_OK;
}

int wake_grid_set_cell_types(wake_grid* g, const uint8_t* types) {
    if (!valid_grid(g) || !types) return set_error(WAKE_ERR_INVALID, "null argument");
    for (long long i = 0; i < g->N; ++i) g->types[i] = types[i] & FL_TYPE;
    g->types_dev_newer = false;  // every cell overwritten
    g->types_host_newer = true;
    g->geom_dirty = true;
    return WAKE_OK;
}

int wake_grid_get_cell_types(wake_grid* g, uint8_t* types) {
    if (!valid_grid(g) || !types) return set_error(WAKE_ERR_INVALID, "null argument");
    const int r = host_types(g);
    if (r) return r;
    std::memcpy(types, g->types.data(), g->N);
    return WAKE_OK;
}

int wake_grid_set_solid_box(wake_grid* g, int x0, int y0, int z0, int x1, int y1, int z1) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    const int r = host_types(g);
    if (r) return r;
    for (int z = std::max(0, z0); z <= std::min(g->nz - 1, z1); ++z)
        for (int y = std::max(0, y0); y <= std::min(g->ny - 1, y1); ++y)
            for (int x = std::max(0, x0); x <= std::min(g->nx - 1, x1); ++x) g->types[idx3(g, x, y, z)] = WAKE_CELL_SOLID;
    g->types_host_newer = true;
    g->geom_dirty = true;
    return WAKE_OK;
}

// LatticeGrid2D::set_solid_circle (lattice_grid_2d.cpp:143-158): bounding box
// truncated with int casts, cell centres at integer coordinates, r^2 test in float.
int wake_grid_set_solid_circle(wake_grid* g, float cx, float cy, float radius) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    const float r_sq = radius * radius;
    wk::RasterBox b{};
    b.x0 = std::max(0, static_cast<int>(cx - radius - 1));
    b.x1 = std::min(g->nx - 1, static_cast<int>(cx + radius + 1));
    b.y0 = std::max(0, static_cast<int>(cy - radius - 1));
    b.y1 = std::min(g->ny - 1, static_cast<int>(cy + radius + 1));
    b.z0 = 0;
    b.z1 = g->nz - 1;
    wk::RasterShape sh{};
    sh.kind = 0;
    sh.c[0] = cx;
    sh.c[1] = cy;
    sh.p[0] = r_sq;
    return rasterise(g, b, sh);
}

// LatticeGrid3D::set_solid_sphere (lattice_grid_3d.cpp:160-182).
int wake_grid_set_solid_sphere(wake_grid* g, float cx, float cy, float cz, float radius) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    const float r_sq = radius * radius;
    wk::RasterBox b{};
    b.x0 = std::max(0, static_cast<int>(cx - radius - 1));
    b.x1 = std::min(g->nx - 1, static_cast<int>(cx + radius + 1));
    b.y0 = std::max(0, static_cast<int>(cy - radius - 1));
    b.y1 = std::min(g->ny - 1, static_cast<int>(cy + radius + 1));
    b.z0 = std::max(0, static_cast<int>(cz - radius - 1));
    b.z1 = std::min(g->nz - 1, static_cast<int>(cz + radius + 1));
    wk::RasterShape sh{};
    sh.kind = 1;
    sh.c[0] = cx;
    sh.c[1] = cy;
    sh.c[2] = cz;
    sh.p[0] = r_sq;
    return rasterise(g, b, sh);
}

// Rotated ellipse (no reference counterpart; same cell-centre rule and float
// arithmetic as GeometryPrimitives::voxelize_ellipsoid, src/geometry/primitives.cpp:73-99):
// node (x, y) is solid when u^2/a^2 + v^2/b^2 <= 1 with (u, v) the offset from
// (cx, cy) rotated by -angle (radians), u = dx cos + dy sin, v = -dx sin + dy cos.
// Extruded along z in 3D.
int wake_grid_set_solid_ellipse(wake_grid* g, float cx, float cy, float a, float b, float angle) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    if (!(a > 0.f) || !(b > 0.f)) return set_error(WAKE_ERR_INVALID, "wake_grid_set_solid_ellipse: semi-axes must be positive");
    const float r = std::max(a, b);
    wk::RasterBox bx{};
    bx.x0 = std::max(0, static_cast<int>(cx - r - 1));
    bx.x1 = std::min(g->nx - 1, static_cast<int>(cx + r + 1));
    bx.y0 = std::max(0, static_cast<int>(cy - r - 1));
    bx.y1 = std::min(g->ny - 1, static_cast<int>(cy + r + 1));
    bx.z0 = 0;
    bx.z1 = g->nz - 1;
    wk::RasterShape sh{};
    sh.kind = 2;
    sh.c[0] = cx;
    sh.c[1] = cy;
    sh.p[0] = std::cos(angle);
    sh.p[1] = std::sin(angle);
    sh.p[2] = 1.0f / (a * a);
    sh.p[3] = 1.0f / (b * b);
    return rasterise(g, bx, sh);
}

int wake_grid_enable_thermal(wake_grid* g, float tau_t, float t_ref, float beta_g, float t_south, float t_north) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    if (g->Q != 9) return set_error(WAKE_ERR_INVALID, "wake_grid_enable_thermal: D2Q9 lattices only");
    if (!(tau_t > 0.5f)) return set_error(WAKE_ERR_INVALID, "wake_grid_enable_thermal: tau_t must exceed 1/2");
    if (g->k != 0) return set_error(WAKE_ERR_INVALID, "wake_grid_enable_thermal: only before the first step");
    const std::size_t b = sizeof(float) * 5 * g->pitch;
    WK_CUDA(g->TA.ensure(b));
    WK_CUDA(g->TB.ensure(b));
    g->th.on = 1;
    g->th.omega_t = 1.0f / tau_t;
    g->th.t_ref = t_ref;
    g->th.beta_g = beta_g;
    g->th.t_south = t_south;
    g->th.t_north = t_north;
    g->geom_dirty = true;  // every segment moves to the general path
    g->pending = true;
    g->invalidate_graph();
    if (!g->mt_valid) {  // start from the reference temperature everywhere
        std::vector<float> T(static_cast<std::size_t>(g->N), t_ref);
        return wake_grid_initialize_temperature(g, T.data());
    }
    return WAKE_OK;
}

int wake_grid_initialize_temperature(wake_grid* g, const float* T) {
    if (!valid_grid(g) || !T) return set_error(WAKE_ERR_INVALID, "null temperature");
    if (!g->th.on) return set_error(WAKE_ERR_INVALID, "wake_grid_initialize_temperature: enable the temperature first");
    if (g->k != 0 && !g->mf_valid)
        return set_error(WAKE_ERR_INVALID, "wake_grid_initialize_temperature: initialise the flow again first");
    WK_CUDA(g->m_t.ensure(sizeof(float) * 5 * g->pitch));
    DevMem tmp;
    WK_CUDA(tmp.ensure(sizeof(float) * g->N));
    WK_CUDA(cudaMemcpyAsync(tmp.p, T, sizeof(float) * g->N, cudaMemcpyDefault, g->stream));
    const int blocks = static_cast<int>(std::min<long long>((g->N + 255) / 256, 148ll * 16));
    k_t5_equilibrium<<<blocks, 256, 0, g->stream>>>(tmp.as<float>(), g->m_t.as<float>(), g->pitch, g->N);
    WK_CUDA(cudaGetLastError());
    WK_CUDA(cudaStreamSynchronize(g->stream));
    tmp.release();
    g->mt_valid = true;
    g->pending = true;
    g->k = 0;  // a coupled run restarts from the flow state in the FP32 scratch
    g->invalidate_graph();
    return WAKE_OK;
}

int wake_grid_get_temperature(wake_grid* g, float* T) {
    if (!valid_grid(g) || !T) return set_error(WAKE_ERR_INVALID, "null output");
    if (!g->th.on) return set_error(WAKE_ERR_INVALID, "wake_grid_get_temperature: no coupled temperature");
    DevMem tmp;
    WK_CUDA(tmp.ensure(sizeof(float) * g->N));
    const int blocks = static_cast<int>(std::min<long long>((g->N + 255) / 256, 148ll * 16));
    if (g->pending || g->k == 0) {
        // not stepped yet: the initial temperature populations
        if (!g->mt_valid) return set_error(WAKE_ERR_INVALID, "wake_grid_get_temperature: no temperature state");
        k_t5_sum<<<blocks, 256, 0, g->stream>>>(g->m_t.as<float>(), g->pitch, g->N, tmp.as<float>());
    } else {
        // BGK conserves sum g, so the current post-collision buffer sums to the step's temperature
        k_t5_sum<<<blocks, 256, 0, g->stream>>>(g->tbuf(g->cur), g->pitch, g->N, tmp.as<float>());
    }
    WK_CUDA(cudaGetLastError());
    WK_CUDA(cudaMemcpyAsync(T, tmp.p, sizeof(float) * g->N, cudaMemcpyDefault, g->stream));
    WK_CUDA(cudaStreamSynchronize(g->stream));
    tmp.release();
    return WAKE_OK;
}

int wake_grid_set_inflow_west(wake_grid* g, float ux, float uy, float uz) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    g->inflow = 1;
    g->uin[0] = ux;
    g->uin[1] = uy;
    g->uin[2] = uz;
    {
        const int r = host_types(g);
        if (r) return r;
    }
    for (int z = 0; z < g->nz; ++z)
        for (int y = 0; y < g->ny; ++y) g->types[idx3(g, 0, y, z)] = WAKE_CELL_INFLOW;
    g->types_host_newer = true;
    g->geom_dirty = true;
    return WAKE_OK;
}

int wake_grid_set_outflow_east(wake_grid* g, float rho_out) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    if (!(rho_out > 0.f)) return set_error(WAKE_ERR_INVALID, "rho_out must be positive");
    g->outflow = 1;
    g->rho_out = rho_out;
    {
        const int r = host_types(g);
        if (r) return r;
    }
    for (int z = 0; z < g->nz; ++z)
        for (int y = 0; y < g->ny; ++y) g->types[idx3(g, g->nx - 1, y, z)] = WAKE_CELL_OUTFLOW;
    g->types_host_newer = true;
    g->geom_dirty = true;
    return WAKE_OK;
}

// 2D: LatticeGrid2D::set_moving_wall_north (lattice_grid_2d.cpp:178-184);
// 3D: LatticeGrid3D::set_moving_wall_top (lattice_grid_3d.cpp:205-215).
int wake_grid_set_moving_wall(wake_grid* g, float uw_x, float uw_y, float uw_z) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    g->lid = 1;
    g->uw[0] = uw_x;
    g->uw[1] = uw_y;
    g->uw[2] = uw_z;
    {
        const int r = host_types(g);
        if (r) return r;
    }
    for (int z = 0; z < g->nz; ++z)
        for (int x = 0; x < g->nx; ++x) g->types[idx3(g, x, g->ny - 1, z)] = WAKE_CELL_MOVING_WALL;
    g->types_host_newer = true;
    g->geom_dirty = true;
    return WAKE_OK;
}

int wake_grid_set_periodic(wake_grid* g, int periodic_y, int periodic_z) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    if (g->D != 3 && (periodic_y || periodic_z)) return set_error(WAKE_ERR_INVALID, "periodic y/z needs a 3D lattice");
    g->periodic_y = periodic_y ? 1 : 0;
    g->periodic_z = periodic_z ? 1 : 0;
    g->geom_dirty = true;
    return WAKE_OK;
}

int wake_grid_set_curved_links(wake_grid* g, int n, const int* fluid_indices, const int* q_dirs, const float* delta,
                               const float* uw_x, const float* uw_y, const float* uw_z) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    if (g->Q != 19 && n > 0) return set_error(WAKE_ERR_INVALID, "curved links are D3Q19 only");
    if (n < 0 || (n > 0 && (!fluid_indices || !q_dirs || !delta)))
        return set_error(WAKE_ERR_INVALID, "wake_grid_set_curved_links: bad arguments");
    for (int k = 0; k < n; ++k)
        if (fluid_indices[k] < 0 || fluid_indices[k] >= g->N || q_dirs[k] < 1 || q_dirs[k] >= g->Q ||
            !(delta[k] > 0.f))
            return set_error(WAKE_ERR_INVALID, "wake_grid_set_curved_links: link out of range");
    g->link_node.assign(fluid_indices, fluid_indices + n);
    g->link_q.assign(q_dirs, q_dirs + n);
    g->link_delta.assign(delta, delta + n);
    g->link_uw.assign(3 * static_cast<std::size_t>(n), 0.f);
    for (int k = 0; k < n; ++k) {
        if (uw_x) g->link_uw[3 * k] = uw_x[k];
        if (uw_y) g->link_uw[3 * k + 1] = uw_y[k];
        if (uw_z) g->link_uw[3 * k + 2] = uw_z[k];
    }
    g->links_dirty = true;
    g->geom_dirty = true;
    return WAKE_OK;
}

// LatticeGrid3D::build_curved_sphere_links (lattice_grid_3d.cpp:217-290): for
// every Fluid node and direction whose neighbour (x periodic, y/z in range) is
// Solid, intersect the link with the sphere; delta defaults to 1/2 and is
// clamped to [0.01, 0.99].
int wake_grid_build_curved_sphere_links(wake_grid* g, float cx, float cy, float cz, float radius) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    if (g->Q != 19) return set_error(WAKE_ERR_INVALID, "curved links are D3Q19 only");
    // candidates on the device: the full-lattice neighbour scan is the costly part of
    // the reference's host loop; only the few boundary nodes come back
    const unsigned cap = static_cast<unsigned>(std::min<long long>(g->N, std::max<long long>(4096, g->N / 16)));
    DevMem d_list, d_count;
    WK_CUDA(d_list.ensure(sizeof(int2) * cap));
    WK_CUDA(d_count.ensure(sizeof(unsigned)));
    {
        const int r = dev_types(g);
        if (r) return r;
    }
    WK_CUDA(cudaMemsetAsync(d_count.p, 0, sizeof(unsigned), g->stream));
    const int blocks = static_cast<int>(std::min<long long>((g->N + 255) / 256, 148ll * 16));
    k_solid_neighbours<19><<<blocks, 256, 0, g->stream>>>(g->d_types.as<uint8_t>(), g->nx, g->ny, g->nz,
                                                            d_count.as<unsigned>(), d_list.as<int2>(), cap);
    WK_CUDA(cudaGetLastError());
    unsigned found = 0;
    WK_CUDA(cudaMemcpyAsync(&found, d_count.p, sizeof(unsigned), cudaMemcpyDeviceToHost, g->stream));
    WK_CUDA(cudaStreamSynchronize(g->stream));
    std::vector<int2> cand;
    if (found <= cap) {
        cand.resize(found);
        if (found)
            WK_CUDA(cudaMemcpyAsync(cand.data(), d_list.p, sizeof(int2) * found, cudaMemcpyDeviceToHost, g->stream));
        WK_CUDA(cudaStreamSynchronize(g->stream));
        std::sort(cand.begin(), cand.end(), [](const int2& a, const int2& b) { return a.x < b.x; });
    } else {
        // more boundary nodes than the list holds (solid-heavy lattice): scan on the host
        const int r = host_types(g);
        if (r) return r;
        for (long long i = 0; i < g->N; ++i) {
            if (g->types[i] != WAKE_CELL_FLUID) continue;
            const int x = static_cast<int>(i % g->nx), y = static_cast<int>((i / g->nx) % g->ny),
                      z = static_cast<int>(i / (static_cast<long long>(g->nx) * g->ny));
            int mask = 0;
            for (int q = 1; q < 19; ++q) {
                const int xn = (x + g->lat.cx[q] + g->nx) % g->nx, yn = y + g->lat.cy[q], zn = z + g->lat.cz[q];
                if (yn < 0 || yn >= g->ny || zn < 0 || zn >= g->nz) continue;
                if (g->types[idx3(g, xn, yn, zn)] == WAKE_CELL_SOLID) mask |= 1 << q;
            }
            if (mask) cand.push_back(make_int2(static_cast<int>(i), mask));
        }
    }
    // delta from the analytic sphere, in the reference's float arithmetic (lattice_grid_3d.cpp:237-256)
    std::vector<int> idx, qd;
    std::vector<float> delta;
    for (const int2& c : cand) {
        const long long i = c.x;
        const int x = static_cast<int>(i % g->nx), y = static_cast<int>((i / g->nx) % g->ny),
                  z = static_cast<int>(i / (static_cast<long long>(g->nx) * g->ny));
        for (int q = 1; q < 19; ++q) {
            if (!(c.y & (1 << q))) continue;
            const float px = static_cast<float>(x) - cx, py = static_cast<float>(y) - cy, pz = static_cast<float>(z) - cz;
            const float dx = float(g->lat.cx[q]), dy = float(g->lat.cy[q]), dz = float(g->lat.cz[q]);
            const float a = dx * dx + dy * dy + dz * dz;
            const float b = 2.0f * (px * dx + py * dy + pz * dz);
            const float cc = (px * px + py * py + pz * pz) - radius * radius;
            const float disc = b * b - 4.0f * a * cc;
            float d = 0.5f;
            if (disc >= 0.0f) {
                const float t1 = (-b - std::sqrt(disc)) / (2.0f * a);
                const float t2 = (-b + std::sqrt(disc)) / (2.0f * a);
                if (t1 >= 0.0f && t1 <= 1.0f) d = t1;
                else if (t2 >= 0.0f && t2 <= 1.0f) d = t2;
            }
            d = std::clamp(d, 0.01f, 0.99f);
            idx.push_back(static_cast<int>(i));
            qd.push_back(q);
            delta.push_back(d);
        }
    }
    d_list.release();
    d_count.release();
    return wake_grid_set_curved_links(g, static_cast<int>(idx.size()), idx.data(), qd.data(), delta.data(), nullptr,
                                      nullptr, nullptr);
}

int wake_grid_num_curved_links(wake_grid* g) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    return static_cast<int>(g->link_node.size());
}

int wake_grid_get_curved_links(wake_grid* g, int* fluid_indices, int* q_dirs, float* delta) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    const std::size_t n = g->link_node.size();
    if (fluid_indices) std::copy(g->link_node.begin(), g->link_node.end(), fluid_indices);
    if (q_dirs) std::copy(g->link_q.begin(), g->link_q.end(), q_dirs);
    if (delta) std::copy(g->link_delta.begin(), g->link_delta.end(), delta);
    return static_cast<int>(n);
}

int wake_grid_initialize(wake_grid* g, float rho, float ux, float uy, float uz) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    InitSpec s{};
    s.mode = 0;
    s.rho = rho;
    s.u[0] = ux;
    s.u[1] = uy;
    s.u[2] = (g->D == 3) ? uz : 0.f;
    return init_on_device(g, s);
}

int wake_grid_initialize_noise(wake_grid* g, float rho, float ux, float uy, float uz, float amplitude,
                               unsigned long long seed, long long offset) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    if (offset < 0) return set_error(WAKE_ERR_INVALID, "wake_grid_initialize_noise: negative stream offset");
    InitSpec s{};
    s.mode = 1;
    s.rho = rho;
    s.u[0] = ux;
    s.u[1] = uy;
    s.u[2] = (g->D == 3) ? uz : 0.f;
    s.amp = amplitude;
    s.seed = seed;
    s.offset = offset;
    return init_on_device(g, s);
}

int wake_grid_initialize_fields(wake_grid* g, const float* rho, const float* ux, const float* uy, const float* uz) {
    if (!valid_grid(g) || !rho || !ux || !uy) return set_error(WAKE_ERR_INVALID, "null field");
    int r = ensure_macro(g);
    if (r) return r;
    const std::size_t b = sizeof(float) * g->N;
    WK_CUDA(cudaMemcpyAsync(g->m_rho.p, rho, b, cudaMemcpyDefault, g->stream));
    WK_CUDA(cudaMemcpyAsync(g->m_ux.p, ux, b, cudaMemcpyDefault, g->stream));
    WK_CUDA(cudaMemcpyAsync(g->m_uy.p, uy, b, cudaMemcpyDefault, g->stream));
    const bool has_z = uz && g->D == 3;
    if (has_z) WK_CUDA(cudaMemcpyAsync(g->m_uz.p, uz, b, cudaMemcpyDefault, g->stream));
    InitSpec s{};
    s.mode = 2;
    s.rho_p = g->m_rho.as<float>();
    s.ux_p = g->m_ux.as<float>();
    s.uy_p = g->m_uy.as<float>();
    s.uz_p = has_z ? g->m_uz.as<float>() : nullptr;
    r = init_on_device(g, s);
    if (r) return r;
    WK_CUDA(cudaStreamSynchronize(g->stream));  // the caller may free its arrays on return
    return WAKE_OK;
}

int wake_grid_set_populations(wake_grid* g, const float* f) {
    if (!valid_grid(g) || !f) return set_error(WAKE_ERR_INVALID, "null populations");
    return upload_f0(g, f, cudaMemcpyHostToDevice);
}

int wake_grid_set_populations_device(wake_grid* g, const float* f_dev) {
    if (!valid_grid(g) || !f_dev) return set_error(WAKE_ERR_INVALID, "null populations");
    return upload_f0(g, f_dev, cudaMemcpyDeviceToDevice);
}

int wake_grid_enable_forces(wake_grid* g, float cx, float cy, float cz, float r_max, int history_capacity) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    if (history_capacity < 1) return set_error(WAKE_ERR_INVALID, "history capacity must be positive");
    g->mem_on = 1;
    g->center[0] = cx;
    g->center[1] = cy;
    g->center[2] = (g->D == 3) ? cz : 0.f;
    g->rmax = r_max;
    g->hist_cap = history_capacity;
    WK_CUDA(g->d_hist.ensure(sizeof(double) * 3 * history_capacity));
    WK_CUDA(g->d_counters.ensure(sizeof(unsigned) * 2));
    WK_CUDA(cudaMemsetAsync(g->d_counters.p, 0, sizeof(unsigned) * 2, g->stream));
    WK_CUDA(cudaMemsetAsync(g->d_hist.p, 0, sizeof(double) * 3 * history_capacity, g->stream));
    // the flags carry the momentum-exchange bit; a pending geometry change
    // is applied (with its state resync) by the next step instead
    if (!g->geom_dirty) {
        const int r = rebuild_flags(g);
        if (r) return r;
    }
    WK_CUDA(cudaStreamSynchronize(g->stream));
    return WAKE_OK;
}

int wake_grid_disable_forces(wake_grid* g) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    g->mem_on = 0;
    if (!g->geom_dirty) {
        const int r = rebuild_flags(g);
        if (r) return r;
    }
    WK_CUDA(cudaStreamSynchronize(g->stream));
    return WAKE_OK;
}

long long wake_grid_force_count(wake_grid* g) {
    if (!valid_grid(g) || !g->mem_on) return 0;
    unsigned c[2] = {0, 0};
    if (cudaMemcpyAsync(c, g->d_counters.p, sizeof(c), cudaMemcpyDeviceToHost, g->stream) != cudaSuccess ||
        cudaStreamSynchronize(g->stream) != cudaSuccess)
        return set_error(WAKE_ERR_CUDA, "wake_grid_force_count: copy failed");
    return c[1];
}

int wake_grid_get_force_history(wake_grid* g, double* out, int max) {
    if (!valid_grid(g) || !out || max < 0) return set_error(WAKE_ERR_INVALID, "bad arguments");
    if (!g->mem_on) return 0;
    const long long count = wake_grid_force_count(g);
    if (count < 0) return static_cast<int>(count);
    // the oldest step still in the ring, then at most `max` steps in order: one or two
    // contiguous runs of the ring, copied straight into the caller's buffer
    const long long cap = g->hist_cap;
    const long long first = std::max(0ll, count - cap);
    const long long n = std::min(count, first + static_cast<long long>(max)) - first;
    if (n <= 0) return 0;
    const long long s0 = first % cap, run1 = std::min(n, cap - s0);
    const double* ring = g->d_hist.as<double>();
    WK_CUDA(cudaMemcpyAsync(out, ring + 3 * s0, sizeof(double) * 3 * run1, cudaMemcpyDefault, g->stream));
    if (n > run1)
        WK_CUDA(cudaMemcpyAsync(out + 3 * run1, ring, sizeof(double) * 3 * (n - run1), cudaMemcpyDefault, g->stream));
    WK_CUDA(cudaStreamSynchronize(g->stream));
    return static_cast<int>(n);
}

// Set the body force of the next steps; the buffers hold Collide(f^k) for the body force they
// were collided with and the reference collides f^k with this step's force, so a change
// re-collides (prepare).
static int set_step_force(wake_grid* g, float gx, float gy, float gz) {
    const float gnew[3] = {gx, gy, (g->D == 3) ? gz : 0.f};
    for (int a = 0; a < 3; ++a) g->phys.g[a] = gnew[a];
    if (gnew[0] != g->collided_g[0] || gnew[1] != g->collided_g[1] || gnew[2] != g->collided_g[2]) g->pending = true;
    return prepare(g);
}

// (Re)capture the graph of graph_steps steps from the current buffer parity unless the
// instantiated one already starts there. Captures only: nothing runs on the device.
static int capture_graph(wake_grid* g) {
    if (g->graph_ok && g->graph_cur == g->cur) return WAKE_OK;
    if (g->graph) {
        cudaGraphExecDestroy(g->graph);
        g->graph = nullptr;
    }
    g->graph_ok = false;
    const int cur0 = g->cur;
    const long long k0 = g->k;
    cudaGraph_t graph = nullptr;
    WK_CUDA(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
    const int r = do_steps(g, g->graph_steps);
    cudaError_t e = cudaStreamEndCapture(g->stream, &graph);
    g->cur = cur0;
    g->k = k0;
    if (r) {
        if (graph) cudaGraphDestroy(graph);
        return r;
    }
    if (e != cudaSuccess) return set_error(WAKE_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&g->graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return set_error(WAKE_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    // move the graph's work descriptors to the device now rather than at its first launch
    e = cudaGraphUpload(g->graph, g->stream);
    if (e != cudaSuccess) return set_error(WAKE_ERR_CUDA, std::string("graph upload: ") + cudaGetErrorString(e));
    g->graph_cur = cur0;
    g->graph_ok = true;
    return WAKE_OK;
}

int wake_grid_step(wake_grid* g, int n, float gx, float gy, float gz) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    if (n < 0) return set_error(WAKE_ERR_INVALID, "negative step count");
    if (n == 0) return WAKE_OK;
    int r = set_step_force(g, gx, gy, gz);
    if (r) return r;
    int done = 0;
    if (g->graph_steps > 0 && n >= g->graph_steps && !g->time_bulk) {
        const int gs = g->graph_steps;
        r = capture_graph(g);
        if (r) return r;
        while (n - done >= gs && g->cur == g->graph_cur) {
            WK_CUDA(cudaGraphLaunch(g->graph, g->stream));
            g->k += gs;
            g->mf_valid = false;
            for (int c = 0; c < 3; ++c) g->last_step_g[c] = g->phys.g[c];
            done += gs;
        }
    }
    return do_steps(g, n - done);
}

int wake_grid_prepare_steps(wake_grid* g, float gx, float gy, float gz) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    int r = set_step_force(g, gx, gy, gz);
    if (r) return r;
    if (g->graph_steps > 0 && !g->time_bulk) r = capture_graph(g);
    if (r) return r;
    WK_CUDA(cudaStreamSynchronize(g->stream));
    return WAKE_OK;
}

int wake_grid_use_graph(wake_grid* g, int steps_per_graph) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    if (steps_per_graph < 0) return set_error(WAKE_ERR_INVALID, "negative graph size");
    // an even count returns to the same buffer parity, so one graph serves every replay
    g->graph_steps = steps_per_graph > 0 && steps_per_graph % 2 ? steps_per_graph + 1 : steps_per_graph;
    g->invalidate_graph();
    return WAKE_OK;
}

long long wake_grid_step_count(wake_grid* g) { return g ? g->k : -1; }

int wake_grid_synchronize(wake_grid* g) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    WK_CUDA(cudaStreamSynchronize(g->stream));
    unsigned st = 0;
    WK_CUDA(cudaMemcpy(&st, g->d_status.p, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (st & ERR_STAGE_TIMEOUT) return set_error(WAKE_ERR_CUDA, "a staged tile copy did not complete (bounded wait expired)");
    if (st & ERR_NONFINITE) return set_error(WAKE_ERR_NUMERIC, "non-finite or non-positive density on the device");
    return WAKE_OK;
}

int wake_grid_get_populations(wake_grid* g, float* f) {
    if (!valid_grid(g) || !f) return set_error(WAKE_ERR_INVALID, "null output");
    const int r = materialise(g, true, false);
    if (r) return r;
    WK_CUDA(cudaMemcpy2DAsync(f, sizeof(float) * g->N, g->m_f.p, sizeof(float) * g->pitch, sizeof(float) * g->N, g->Q,
                              cudaMemcpyDefault, g->stream));
    WK_CUDA(cudaStreamSynchronize(g->stream));
    return WAKE_OK;
}

int wake_grid_get_macroscopic(wake_grid* g, float* rho, float* ux, float* uy, float* uz, float* speed) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    const int r = materialise(g, false, true);
    if (r) return r;
    const std::size_t b = sizeof(float) * g->N;
    if (rho) WK_CUDA(cudaMemcpyAsync(rho, g->m_rho.p, b, cudaMemcpyDefault, g->stream));
    if (ux) WK_CUDA(cudaMemcpyAsync(ux, g->m_ux.p, b, cudaMemcpyDefault, g->stream));
    if (uy) WK_CUDA(cudaMemcpyAsync(uy, g->m_uy.p, b, cudaMemcpyDefault, g->stream));
    if (uz) WK_CUDA(cudaMemcpyAsync(uz, g->m_uz.p, b, cudaMemcpyDefault, g->stream));
    if (speed) WK_CUDA(cudaMemcpyAsync(speed, g->m_speed.p, b, cudaMemcpyDefault, g->stream));
    WK_CUDA(cudaStreamSynchronize(g->stream));
    return WAKE_OK;
}

static int diag_all(wake_grid* g, double out[4]) {
    int r = apply_geometry(g);  // the sums run over the current cell types
    if (r) return r;
    r = materialise(g, false, true);
    if (r) return r;
    const int nb = 592;  // 4 x 148 SMs
    WK_CUDA(g->m_diag.ensure(sizeof(double) * 4 * nb));
    k_diag_partials<<<nb, 256, 0, g->stream>>>(g->m_rho.as<float>(), g->m_speed.as<float>(), g->d_flags.as<uint8_t>(),
                                                g->N, g->m_diag.as<double>());
    WK_CUDA(cudaGetLastError());
    std::vector<double> h(4 * nb);
    WK_CUDA(cudaMemcpyAsync(h.data(), g->m_diag.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, g->stream));
    WK_CUDA(cudaStreamSynchronize(g->stream));
    out[0] = out[1] = out[2] = out[3] = 0.0;
    for (int b = 0; b < nb; ++b) {
        out[0] += h[4 * b];
        out[1] += h[4 * b + 1];
        out[2] = std::max(out[2], h[4 * b + 2]);
        out[3] += h[4 * b + 3];
    }
    return WAKE_OK;
}

int wake_grid_diagnostics(wake_grid* g, double* total_mass, double* kinetic_energy, double* max_speed) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    double d[4];
    const int r = diag_all(g, d);
    if (r) return r;
    if (total_mass) *total_mass = d[0];
    if (kinetic_energy) *kinetic_energy = d[1];
    if (max_speed) *max_speed = d[2];
    return WAKE_OK;
}

// ---------------------------------------------------------------- field analytics
// FieldAnalytics::compute_vorticity / compute_3d_features / compute_max_vorticity_2d
// (src/analytics/field_analytics.cpp:18-63) on the device, from the moments of
// the current state. Outputs may be host or device memory (one float per node).
static bool on_device(const void* p) {
    cudaPointerAttributes a{};
    const cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int wake_grid_compute_vorticity(wake_grid* g, float* vorticity) {
    if (!valid_grid(g) || !vorticity) return set_error(WAKE_ERR_INVALID, "null vorticity output");
    if (g->D != 2) return set_error(WAKE_ERR_INVALID, "wake_grid_compute_vorticity: D2Q9 lattices only");
    int r = apply_geometry(g);
    if (r) return r;
    r = materialise(g, false, true);
    if (r) return r;
    const std::size_t b = sizeof(float) * g->N;
    float* out = vorticity;
    if (!on_device(vorticity)) {
        WK_CUDA(g->m_an.ensure(b));
        out = g->m_an.as<float>();
    }
    k_vorticity_2d<<<analytics_grid_3d(g->nx, g->ny, 1), analytics_block(), 0, g->stream>>>(
        g->m_ux.as<float>(), g->m_uy.as<float>(), out, g->nx, g->ny);
    WK_CUDA(cudaGetLastError());
    if (out != vorticity) WK_CUDA(cudaMemcpyAsync(vorticity, out, b, cudaMemcpyDeviceToHost, g->stream));
    WK_CUDA(cudaStreamSynchronize(g->stream));
    return WAKE_OK;
}

int wake_grid_compute_3d_features(wake_grid* g, float* omega_x, float* omega_y, float* omega_z, float* q_criterion) {
    if (!valid_grid(g) || !omega_x || !omega_y || !omega_z || !q_criterion)
        return set_error(WAKE_ERR_INVALID, "null vorticity or Q-criterion output");
    if (g->D != 3) return set_error(WAKE_ERR_INVALID, "wake_grid_compute_3d_features: 3D lattices only");
    int r = apply_geometry(g);
    if (r) return r;
    r = materialise(g, false, true);
    if (r) return r;
    const std::size_t b = sizeof(float) * g->N;
    float* user[4] = {omega_x, omega_y, omega_z, q_criterion};
    float* out[4];
    bool staged = false;
    for (int i = 0; i < 4; ++i) staged = staged || !on_device(user[i]);
    if (staged) WK_CUDA(g->m_an.ensure(4 * b));
    for (int i = 0; i < 4; ++i) out[i] = on_device(user[i]) ? user[i] : g->m_an.as<float>() + i * g->N;
    k_vorticity_q_3d<<<analytics_grid_3d(g->nx, g->ny, g->nz), analytics_block(), 0, g->stream>>>(
        g->m_ux.as<float>(), g->m_uy.as<float>(), g->m_uz.as<float>(), out[0], out[1], out[2], out[3], g->nx, g->ny,
        g->nz);
    WK_CUDA(cudaGetLastError());
    for (int i = 0; i < 4; ++i)
        if (out[i] != user[i]) WK_CUDA(cudaMemcpyAsync(user[i], out[i], b, cudaMemcpyDeviceToHost, g->stream));
    WK_CUDA(cudaStreamSynchronize(g->stream));
    return WAKE_OK;
}

// Largest |v| of device values on `stream` (k_absmax), synchronous.
static int abs_max_device(const float* values, long long count, float* out, cudaStream_t stream, DevMem& word) {
    WK_CUDA(word.ensure(sizeof(unsigned)));
    WK_CUDA(cudaMemsetAsync(word.p, 0, sizeof(unsigned), stream));
    if (count > 0) {
        const long long want = (count + 255) / 256;
        const int blocks = static_cast<int>(want < 148 * 8 ? want : 148 * 8);
        k_absmax<<<blocks, 256, 0, stream>>>(values, count, word.as<unsigned>());
        WK_CUDA(cudaGetLastError());
    }
    unsigned bits = 0;
    WK_CUDA(cudaMemcpyAsync(&bits, word.p, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
    WK_CUDA(cudaStreamSynchronize(stream));
    std::memcpy(out, &bits, sizeof(float));
    return WAKE_OK;
}

int wake_grid_max_vorticity(wake_grid* g, float* max_vorticity) {
    if (!valid_grid(g) || !max_vorticity) return set_error(WAKE_ERR_INVALID, "null output");
    if (g->D != 2) return set_error(WAKE_ERR_INVALID, "wake_grid_max_vorticity: D2Q9 lattices only");
    const std::size_t b = sizeof(float) * g->N;
    WK_CUDA(g->m_an.ensure(b));
    float* v = g->m_an.as<float>();
    const int r = wake_grid_compute_vorticity(g, v);
    if (r) return r;
    DevMem word;
    return abs_max_device(v, static_cast<long long>(g->N), max_vorticity, g->stream, word);
}

int wake_field_abs_max(const float* values, long long count, float* out) {
    if (!out || count < 0 || (!values && count > 0))
        return set_error(WAKE_ERR_INVALID, "wake_field_abs_max: bad argument");
    if (count == 0) {
        *out = 0.0f;
        return WAKE_OK;
    }
    DevMem staged, word;
    const float* v = values;
    if (!on_device(values)) {
        WK_CUDA(staged.ensure(sizeof(float) * static_cast<std::size_t>(count)));
        WK_CUDA(cudaMemcpy(staged.p, values, sizeof(float) * static_cast<std::size_t>(count), cudaMemcpyHostToDevice));
        v = staged.as<float>();
    }
    return abs_max_device(v, count, out, nullptr, word);
}

int wake_grid_total_mass(wake_grid* g, double* mass) {
    if (!valid_grid(g) || !mass) return set_error(WAKE_ERR_INVALID, "null output");
    double d[4];
    const int r = diag_all(g, d);
    if (r) return r;
    *mass = d[3];
    return WAKE_OK;
}

int wake_grid_info(wake_grid* g, int* q, int* nx, int* ny, int* nz, int* storage, long long* pitch) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    if (q) *q = g->Q;
    if (nx) *nx = g->nx;
    if (ny) *ny = g->ny;
    if (nz) *nz = g->nz;
    if (storage) *storage = g->storage;
    if (pitch) *pitch = g->pitch;
    return WAKE_OK;
}

long long wake_grid_device_bytes(wake_grid* g) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    const DevMem* all[] = {&g->A, &g->B, &g->d_types, &g->d_flags, &g->d_status, &g->d_nodestart, &g->d_link_node,
                           &g->d_link_q, &g->d_link_delta, &g->d_link_mom, &g->d_counters, &g->d_hist,
                           &g->d_warp_base, &g->d_contrib, &g->d_fast_rows, &g->d_gen_rows, &g->m_f, &g->m_rho,
                           &g->m_ux, &g->m_uy, &g->m_uz, &g->m_speed, &g->m_diag, &g->TA, &g->TB, &g->m_t,
                           &g->d_tiles, &g->d_gen4, &g->d_mixed, &g->m_an};
    long long sum = 0;
    for (const DevMem* m : all) sum += static_cast<long long>(m->bytes);
    return sum;
}

long long wake_grid_estimate_bytes(int q, int nx, int ny, int nz, int storage, int with_fields) {
    const bool thermal = (with_fields & 2) != 0;
    with_fields &= 1;
    if (!(q == 9 || q == 19 || q == 27) || nx < 1 || ny < 1 || nz < 1 || storage < 0 || storage > 3)
        return set_error(WAKE_ERR_INVALID, "wake_grid_estimate_bytes: invalid lattice, size or storage");
    const long long N = static_cast<long long>(nx) * ny * nz, pitch = (N + 63) / 64 * 64;
    const long long elem = storage == WAKE_STORE_F32 ? 4 : 2;
    long long b = 2 * q * pitch * elem;  // state buffers
    b += q * pitch * 4;                  // FP32 populations for (re)initialisation
    b += 2 * N + 4 * N;                  // cell types, flags, per-node first curved link
    b += 8ll * ny * nz;                  // row lists
    if (with_fields) b += 5 * 4 * N;     // rho, ux, uy, uz, speed
    if (thermal) b += 3 * 5 * 4 * pitch;  // coupled temperature: two state buffers and the start-up populations
    return b + (1ll << 20);              // history ring, slots and small tables
}

int wake_grid_release_scratch(wake_grid* g) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    const int r = prepare(g);  // a pending re-collide consumes the FP32 populations first
    if (r) return r;
    // every queued use of the scratch has finished, so its blocks go back to the process cache:
    // no cudaFree, which would wait for the whole device (other lattices' steps included)
    WK_CUDA(cudaStreamSynchronize(g->stream));
    if (g->side) WK_CUDA(cudaStreamSynchronize(g->side));
    g->m_f.release();
    g->mf_valid = false;
    if (g->k > 0 || !g->pending) {  // the initial temperature populations were collided already
        g->m_t.release();
        g->mt_valid = false;
    }
    g->m_an.release();
    g->m_rho.release();
    g->m_ux.release();
    g->m_uy.release();
    g->m_uz.release();
    g->m_speed.release();
    g->m_diag.release();
    return WAKE_OK;
}

void* wake_grid_state_buffer(wake_grid* g, int which) {
    if (!g) return nullptr;
    return g->buf(which == 0 ? g->cur : 1 - g->cur);
}

int wake_grid_set_block(wake_grid* g, int threads_per_block) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    if (threads_per_block < 32 || threads_per_block > 512 || threads_per_block % 32)
        return set_error(WAKE_ERR_INVALID, "threads per block must be a multiple of 32 in [32, 512]");
    g->choose_block(threads_per_block);
    g->geom_dirty = true;  // momentum-exchange block slots depend on the launch shape
    return WAKE_OK;
}

int wake_grid_get_block(wake_grid* g) { return g ? g->tpb : WAKE_ERR_INVALID; }

int wake_grid_set_kernel(wake_grid* g, int variant) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    if (variant < 0 || variant > 4) return set_error(WAKE_ERR_INVALID, "wake_grid_set_kernel: variant 0 to 4");
    g->kernel_variant = variant;
    g->invalidate_graph();
    return WAKE_OK;
}

int wake_grid_get_kernel(wake_grid* g) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    const int r = prepare(g);
    if (r) return r;
    return g->use_tiles() ? 2 : (g->use_pipe() ? 4 : (g->use_rows() ? 3 : 1));
}

int wake_grid_launches_per_step(wake_grid* g) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    const int r = prepare(g);
    if (r) return r;
    if (g->use_tiles()) return 1 + (g->mem_on ? 1 : 0);
    if (g->use_pipe() || g->use_rows()) return 1 + (g->n_mixed > 0 ? 1 : 0) + (g->n_gen > 0 ? 1 : 0) + (g->mem_on ? 1 : 0);
    return (g->n_fast > 0 ? 1 : 0) + (g->n_gen > 0 ? 1 : 0) + (g->mem_on ? 1 : 0);
}

int wake_grid_time_bulk_launches(wake_grid* g, int on) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    WK_CUDA(cudaStreamSynchronize(g->stream));
    g->time_bulk = on != 0;
    g->t_used = 0;
    return WAKE_OK;
}

int wake_grid_bulk_launch_times(wake_grid* g, double* total_ms, long long* launches, long long* nodes_per_launch) {
    if (!valid_grid(g)) return WAKE_ERR_INVALID;
    WK_CUDA(cudaStreamSynchronize(g->stream));
    double sum = 0.0;
    for (std::size_t i = 0; i + 1 < g->t_used; i += 2) {
        float ms = 0.f;
        WK_CUDA(cudaEventElapsedTime(&ms, g->t_ev[i], g->t_ev[i + 1]));
        sum += ms;
    }
    if (total_ms) *total_ms = sum;
    if (launches) *launches = static_cast<long long>(g->t_used / 2);
    // the persistent launch also updates the general rows
    if (nodes_per_launch) *nodes_per_launch = g->use_tiles() ? g->N : (g->use_pipe() || g->use_rows() ? g->row_fast_nodes : g->fast_nodes());
    g->t_used = 0;
    return WAKE_OK;
}

}  // extern "C"
