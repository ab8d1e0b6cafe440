// Fused pull-stream + boundary + moments + momentum-exchange + collide kernels.
//
// State between steps is the POST-collision population buffer g^k (A/B
// ping-pong, SoA planes [q][node], plane pitch a multiple of 64 elements).
// The reference keeps the post-stream, pre-collision f^k instead
// (src/grid/lattice_grid_2d.cpp:195-265): f^{k+1} = ZouHe(BFL(Stream(Collide(f^k)))).
// With g^k = Collide(f^k), one fused launch computes, per node,
//
//   f^{k+1}(x) = ZouHe(BFL(Pull(g^k)))(x)      -- reference steps 3-5
//   rho, u, momentum exchange from f^{k+1}(x)   -- reference step 6 + scenario MEM
//   g^{k+1}(x) = Collide(f^{k+1}(x))            -- next step's collide
//
// so every quantity the reference exposes after k steps is available from
// g^{k-1} (re-gathered by the materialise kernel), and one step moves
// 2*Q*sizeof(pop) + 1 flag byte per node through HBM.
#pragma once

#include "common.cuh"
#include "lattice.cuh"
#include "pairs2.cuh"

namespace wk {

// Device-side error word bits (read by the host after a launch sequence).
enum : unsigned { ERR_NONFINITE = 1u, ERR_BAD_CONFIG = 2u };

struct Geo {
    int nx, ny, nz;
    int periodic_y, periodic_z;   // 3D: wrap y / z instead of half-way bounce-back walls
    long long pitch;              // elements per population plane
    float uin[3];                 // Zou-He inlet velocity
    float rho_out;                // Zou-He outlet density
    float mom[27];                // moving-wall term 2 w_q 3 (c_q . u_w) (d2q9_streaming.ispc:49-53)
};

struct Links {                    // curved-boundary (BFL) links sorted by fluid node
    const int* node_start;        // [N] first link of the node, read only where FL_BFL is set
    const int* node;              // [n] fluid node index
    const int* q;                 // [n] direction pointing into the solid
    const float* delta;           // [n] wall distance fraction
    const float* mom;             // [n] moving-wall term of the branch taken (d3q19_curved.ispc:57,62)
    int count;
};

struct MemCfg {                   // momentum-exchange monitor
    int enabled;
    float center[3];
    float r_max, r_max_sq;
    // Every node carrying FL_MEM owns one fixed slot of `contrib`, numbered in node
    // order: slot = warp_base[entry * warps_per_row + chunk] + (rank of the node
    // among the FL_MEM nodes of its 32-node chunk of a general segment). k_mem_reduce
    // sums the slots in slot order, so the force is reproducible bit for bit and
    // needs no barrier.
    const int* warp_base;         // [general segments][warps_per_row]
    int warps_per_row;            // 32-node chunks per segment (SEG / 32)
    double* contrib;              // [n_nodes][3]
    int n_nodes;
    unsigned* hist_step;          // number of entries written so far
    double* hist;                 // [hist_cap][3]: (Fx, Fy, Tz) in 2D, (Fx, Fy, Fz) in 3D
    int hist_cap;
};

struct Out {                      // optional outputs of the materialise kernel
    float* f;                     // FP32 f^k planes (pitch as the state buffers)
    float* rho;
    float* ux;
    float* uy;
    float* uz;
    float* speed;
};

template <int Q>
__device__ __forceinline__ int wrap(int v, int n) {
    v += (v < 0) ? n : 0;
    v -= (v >= n) ? n : 0;
    return v;
}

// Pure gather of a node whose pull sources are all in range (after the periodic
// wraps) and plain fluid: the three x positions and the row bases of the
// (dy, dz) shifts are built once, then each load is a warp-uniform plane
// pointer plus a 32-bit in-plane offset.
template <int Q, int S>
__device__ __forceinline__ void gather_pure(const typename Codec<S>::T* __restrict__ fin, const Geo& G, int x, int y,
                                            int z, float f[Q]) {
    using L = Lat<Q>;
    using C = Codec<S>;
    const long long P = G.pitch;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const int xs[3] = {x == nx - 1 ? 0 : x + 1, x, x == 0 ? nx - 1 : x - 1};  // source x for cx = -1, 0, +1
    int ys[3] = {y + 1, y, y - 1}, zs[3] = {z + 1, z, z - 1};                // source rows for c = -1, 0, +1
    if (G.periodic_y) {
        ys[0] = ys[0] == ny ? 0 : ys[0];
        ys[2] = ys[2] < 0 ? ny - 1 : ys[2];
    }
    if (G.periodic_z) {
        zs[0] = zs[0] == nz ? 0 : zs[0];
        zs[2] = zs[2] < 0 ? nz - 1 : zs[2];
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const unsigned off =
            static_cast<unsigned>((zs[L::cz(q) + 1] * ny + ys[L::cy(q) + 1]) * nx + xs[L::cx(q) + 1]);
        f[q] = C::load(fin + q * P + off, L::w(q));
    }
}

// Pull f^{k+1}(x) out of g^k. `bb` gets bit q when the pull of q bounced off a
// solid or moving-wall node (in range), which marks the momentum-exchange link
// (x, opp(q)).
template <int Q, int S>
__device__ __forceinline__ void gather(const typename Codec<S>::T* __restrict__ fin, const Geo& G,
                                       const uint8_t* __restrict__ flags, const Links& B, int x, int y, int z,
                                       long long i, uint8_t fl, float f[Q], unsigned& bb) {
    using L = Lat<Q>;
    using C = Codec<S>;
    const long long P = G.pitch;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    bb = 0u;
    if (fl & FL_FAST) {
        gather_pure<Q, S>(fin, G, x, y, z, f);
        if (fl & FL_ZH_IN) zou_he_inlet<Q>(f, G.uin);
        if (fl & FL_ZH_OUT) zou_he_outlet<Q>(f, G.rho_out);
        return;
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int o = L::opp(q);
        const int sx = L::cx(q) ? wrap<Q>(x - L::cx(q), nx) : x;
        int sy = y - L::cy(q), sz = z - L::cz(q);
        if (L::cy(q) && G.periodic_y) sy = wrap<Q>(sy, ny);
        if (L::cz(q) && G.periodic_z) sz = wrap<Q>(sz, nz);
        const bool inr = (sy >= 0) && (sy < ny) && (sz >= 0) && (sz < nz);
        if (!inr) {
            f[q] = C::load(fin + o * P + i, L::w(o));  // domain wall: half-way bounce-back
            continue;
        }
        const long long s = (static_cast<long long>(sz) * ny + sy) * nx + sx;
        const uint8_t t = flags[s] & FL_TYPE;
        if (t == CT_SOLID) {
            f[q] = C::load(fin + o * P + i, L::w(o));
            bb |= 1u << q;
        } else if (t == CT_MOVING_WALL) {
            f[q] = C::load(fin + o * P + i, L::w(o)) + G.mom[q];
            bb |= 1u << q;
        } else {
            f[q] = C::load(fin + q * P + s, L::w(q));
        }
    }
    if constexpr (Q == 19) {
        if (fl & FL_BFL) {
            // Bouzidi linear interpolation from post-collision values (d3q19_curved.ispc:36-68).
            for (int k = B.node_start[i]; k < B.count && B.node[k] == i; ++k) {
                const int q = B.q[k];
                int qcx, qcy, qcz, o;
                float wq;
                rt_dir<19>(q, qcx, qcy, qcz, o, wq);
                const float delta = B.delta[k];
                const float fi = C::load(fin + q * P + i, wq);
                float val;
                if (delta < 0.5f) {
                    const int xff = wrap<Q>(x - qcx, nx);
                    const int yff = y - qcy, zff = z - qcz;
                    float fff = fi;
                    if (yff >= 0 && yff < ny && zff >= 0 && zff < nz) {
                        const long long s = (static_cast<long long>(zff) * ny + yff) * nx + xff;
                        fff = C::load(fin + q * P + s, wq);
                    }
                    val = 2.0f * delta * fi + (1.0f - 2.0f * delta) * fff - B.mom[k];
                } else {
                    const float fo = C::load(fin + o * P + i, rt_w19(o));
                    const float i2d = 1.0f / (2.0f * delta);
                    val = i2d * fi + (1.0f - i2d) * fo - B.mom[k];
                }
#pragma unroll
                for (int qq = 0; qq < Q; ++qq)
                    if (qq == o) f[qq] = val;
            }
        }
    }
    if (fl & FL_ZH_IN) zou_he_inlet<Q>(f, G.uin);
    if (fl & FL_ZH_OUT) zou_he_outlet<Q>(f, G.rho_out);
}

// Momentum-exchange contributions of one fluid node (forces_momentum_exchange.ispc:33-63):
// links (x, q) with a Solid / MovingWall node at x + c_q (x periodic, y/z in range)
// within r_max of the centre; F += 2 f_q c_q, torque from r x F in 2D.
template <int Q>
__device__ __forceinline__ void mem_node(const float* f, unsigned bb, int x, int y, int z, const Geo& G,
                                         const MemCfg& M, double acc[3]) {
    using L = Lat<Q>;
#pragma unroll
    for (int q = 1; q < Q; ++q) {
        if (!(bb & (1u << L::opp(q)))) continue;
        const int yn = y + L::cy(q), zn = z + L::cz(q);
        if (yn < 0 || yn >= G.ny || zn < 0 || zn >= G.nz) continue;
        // same float roundings as the reference's filter: no contraction
        const float rx = __fsub_rn(__fadd_rn(float(x), 0.5f * float(L::cx(q))), M.center[0]);
        const float ry = __fsub_rn(__fadd_rn(float(y), 0.5f * float(L::cy(q))), M.center[1]);
        const float rz = __fsub_rn(__fadd_rn(float(z), 0.5f * float(L::cz(q))), M.center[2]);
        float r2 = __fadd_rn(__fmul_rn(rx, rx), __fmul_rn(ry, ry));
        if (L::D == 3) r2 = __fadd_rn(r2, __fmul_rn(rz, rz));
        if (!(M.r_max <= 0.0f || r2 <= M.r_max_sq)) continue;
        const double fv = f[q];
        const double dfx = 2.0 * fv * L::cx(q), dfy = 2.0 * fv * L::cy(q);
        acc[0] += dfx;
        acc[1] += dfy;
        if (L::D == 2) acc[2] += double(rx) * dfy - double(ry) * dfx;
        else acc[2] += 2.0 * fv * L::cz(q);
    }
}

// D2Q5 temperature coupled to a D2Q9 flow (no reference counterpart; the
// reference's thermal solver uses a D2Q9 temperature and one domain-averaged
// force, src/thermal/thermal_solver.cpp:83-123, src/scenarios/thermal_convection.cpp:70).
// Per node: T = sum g, the flow collides with the body force g + (0, beta_g (T - T_ref)),
// the temperature relaxes to w_q T (1 + 3 c_q.u) with omega_t (first-order equilibrium
// as thermal_kernels.ispc:32). Streaming: anti-bounce-back g_q = -g*_opp + 2 w_q T_wall
// through the y walls (Dirichlet), bounce-back at solid nodes (adiabatic).
struct Thermal {
    int on;
    float omega_t, t_ref, beta_g, t_south, t_north;
    const float* tin;  // post-collision temperature populations of the last step [5][pitch]
    float* tout;
};

struct D2Q5 {  // rest, +x, +y, -x, -y; c_s^2 = 1/3
    __host__ __device__ static constexpr int cx(int q) { return q == 1 ? 1 : (q == 3 ? -1 : 0); }
    __host__ __device__ static constexpr int cy(int q) { return q == 2 ? 1 : (q == 4 ? -1 : 0); }
    __host__ __device__ static constexpr int opp(int q) { return q == 0 ? 0 : (q + 1) % 4 + 1; }
    __host__ __device__ static constexpr float w(int q) { return q == 0 ? 1.0f / 3.0f : 1.0f / 6.0f; }
};

// Pull the temperature populations of node (x, y) (2D, i its index).
__device__ __forceinline__ void gather_t5(const Thermal& th, const uint8_t* __restrict__ flags, const Geo& G,
                                          long long P, int x, int y, long long i, float t[5]) {
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        const int o = D2Q5::opp(q);
        const int sx = D2Q5::cx(q) ? wrap<9>(x - D2Q5::cx(q), G.nx) : x, sy = y - D2Q5::cy(q);
        if (sy < 0 || sy >= G.ny) {
            const float tw = sy < 0 ? th.t_south : th.t_north;
            t[q] = __fadd_rn(-th.tin[o * P + i], __fmul_rn(2.0f * D2Q5::w(q), tw));
        } else {
            const long long s = static_cast<long long>(sy) * G.nx + sx;
            t[q] = ((flags[s] & FL_TYPE) == CT_SOLID) ? th.tin[o * P + i] : th.tin[q * P + s];
        }
    }
}

__device__ __forceinline__ float sum_t5(const float t[5]) {
    float T = t[0];
#pragma unroll
    for (int q = 1; q < 5; ++q) T = __fadd_rn(T, t[q]);
    return T;
}

// Body force of a node with temperature T: g + (0, beta_g (T - T_ref), 0), explicit roundings.
__device__ __forceinline__ float buoyant_gy(const Thermal& th, float gy, float T) {
    return __fadd_rn(gy, __fmul_rn(th.beta_g, __fsub_rn(T, th.t_ref)));
}

// BGK relaxation of the temperature populations toward w_q T (1 + 3 c_q.u).
__device__ __forceinline__ void collide_t5(float t[5], float T, const float u[3], float om) {
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        const float cu = __fadd_rn(__fmul_rn(float(D2Q5::cx(q)), u[0]), __fmul_rn(float(D2Q5::cy(q)), u[1]));
        const float geq = __fmul_rn(__fmul_rn(D2Q5::w(q), T), __fadd_rn(1.0f, __fmul_rn(3.0f, cu)));
        t[q] = __fsub_rn(t[q], __fmul_rn(om, __fsub_rn(t[q], geq)));
    }
}

struct StepArgs {
    const void* fin;
    void* fout;
    const uint8_t* flags;
    unsigned* status;
    Geo geo;
    Links links;
    MemCfg mem;
    Physics phys;
    const unsigned* rows;  // general segments of this launch (seg_decode); one block per segment
    int nrows;
    const uint4* spans;    // pure-gather spans (member, row, x0, x1); one block per span
    int nspans;
    Thermal th;            // D2Q9 lattices only; th.on = 0 otherwise
    const uint8_t* row_kind;  // per-row descriptor bytes of k_step_rows (rows.cuh); one block per row
};

// Work unit of the step kernels: a segment of up to SEG consecutive nodes of one
// row, numbered row * nseg + s with nseg = ceil(nx / SEG) and row = z * ny + y.
// Rows are split so that only the segments next to a wall, obstacle or curved
// link take the general per-node path. The general kernels run one warp per
// 32-node chunk of a segment.
#ifndef WK_SEG
#define WK_SEG 64
#endif
constexpr int SEG = WK_SEG;
static_assert(SEG == 32 || SEG == 64, "segments of one or two warp chunks");

struct Seg {
    int y, z, x0, x1;
    long long row0;  // index of node (0, y, z)
};

__device__ __forceinline__ Seg seg_decode(unsigned e, const Geo& g) {
    const unsigned nseg = static_cast<unsigned>((g.nx + SEG - 1) / SEG);
    const unsigned row = e / nseg;
    Seg s;
    s.x0 = static_cast<int>(e - row * nseg) * SEG;
    s.x1 = min(g.nx, s.x0 + SEG);
    s.y = static_cast<int>(row % static_cast<unsigned>(g.ny));
    s.z = static_cast<int>(row / static_cast<unsigned>(g.ny));
    s.row0 = static_cast<long long>(row) * g.nx;
    return s;
}

// A span: nodes x0 .. x1-1 of one row, all pure gathers (a whole row, or a run of
// pure-gather segments of a row that also holds general segments).
__device__ __forceinline__ Seg span_decode(uint4 sp, const Geo& g) {
    Seg s;
    s.y = static_cast<int>(sp.y % static_cast<unsigned>(g.ny));
    s.z = static_cast<int>(sp.y / static_cast<unsigned>(g.ny));
    s.x0 = static_cast<int>(sp.z);
    s.x1 = static_cast<int>(sp.w);
    s.row0 = static_cast<long long>(sp.y) * g.nx;
    return s;
}

// One fused time step of one 32-node chunk (0 or 1) of segment e, by one warp:
// g^{k+1} = Collide(ZouHe(BFL(Pull(g^k)))). Solid nodes are not touched: both
// buffers hold their frozen populations. `entry` is the segment's index in its
// lattice's general-segment list; momentum-exchange slots are numbered per
// (entry, chunk).
template <int Q, int COLL, int S, bool LES>
__device__ __forceinline__ void step_chunk(const StepArgs& a, unsigned e, int entry, int chunk) {
    using L = Lat<Q>;
    using C = Codec<S>;
    using T = typename C::T;
    const Seg sg = seg_decode(e, a.geo);
    const int y = sg.y, z = sg.z;
    const long long row0 = sg.row0;
    const int lane = threadIdx.x & 31;
    const int xb = sg.x0 + 32 * chunk;
    if (xb >= sg.x1) return;
    {
        const int x = xb + lane;
        const bool live_node = x < sg.x1;
        const long long i = row0 + (live_node ? x : xb);
        const uint8_t fl = a.flags[i];
        int slot = -1;
        if (a.mem.enabled) {
            // slot = chunk base + rank among this chunk's momentum-exchange nodes
            const bool m = live_node && (fl & FL_MEM) != 0;
            const unsigned bal = __ballot_sync(0xffffffffu, m);
            if (m) slot = a.mem.warp_base[entry * a.mem.warps_per_row + chunk] + __popc(bal & ((1u << lane) - 1u));
        }
        if (!live_node) return;
        if ((fl & FL_TYPE) == CT_SOLID) return;
        float f[Q];
        unsigned bb;
        gather<Q, S>(static_cast<const T*>(a.fin), a.geo, a.flags, a.links, x, y, z, i, fl, f, bb);
        Physics ph = a.phys;  // a coupled temperature adds the node's buoyancy to the body force
        float t5[5], Tn = 0.f;
        if constexpr (Q == 9) {
            if (a.th.on) {
                gather_t5(a.th, a.flags, a.geo, a.geo.pitch, x, y, i, t5);
                Tn = sum_t5(t5);
                ph.g[1] = buoyant_gy(a.th, a.phys.g[1], Tn);
            }
        }
        float rho, u[3];
        node_moments<Q>(f, ph.g, rho, u);
        if (slot >= 0) {
            double acc[3] = {0.0, 0.0, 0.0};
            mem_node<Q>(f, bb, x, y, z, a.geo, a.mem, acc);
            double* c = a.mem.contrib + 3 * static_cast<long long>(slot);
            c[0] = acc[0];
            c[1] = acc[1];
            c[2] = acc[2];
        }
        if (!(rho > 0.0f) || !(fabsf(u[0]) < 1e30f)) atomicOr(a.status, ERR_NONFINITE);
        collide<Q, COLL, LES>(f, rho, u, ph);
        T* out = static_cast<T*>(a.fout);
#pragma unroll
        for (int q = 0; q < Q; ++q) C::store_stream(out + q * a.geo.pitch + i, f[q], L::w(q));
        if constexpr (Q == 9) {
            if (a.th.on) {
                collide_t5(t5, Tn, u, a.th.omega_t);
#pragma unroll
                for (int q = 0; q < 5; ++q) __stcs(a.th.tout + q * a.geo.pitch + i, t5[q]);
            }
        }
    }
}

// Value stored for population q: FP32 holds f, FP16 / BF16 / FP16C hold h = f / w - 1.
// load_h / store_h move the stored value itself (no decode) for the h-space math.
template <int S>
__device__ __forceinline__ float load_raw(const typename Codec<S>::T* p) {
    if constexpr (S == STORE_F32) return __ldg(p);
    else if constexpr (S == STORE_F16) return __half2float(__ldg(p));
    else if constexpr (S == STORE_F16C) return f16c_decode(__ldg(reinterpret_cast<const unsigned short*>(p)));
    else return __bfloat162float(__ldg(p));
}
template <int S>
__device__ __forceinline__ void store_raw(typename Codec<S>::T* p, float v) {
    if constexpr (S == STORE_F32) __stcs(p, v);
    else if constexpr (S == STORE_F16) __stcs(reinterpret_cast<unsigned short*>(p), __half_as_ushort(__float2half_rn(v)));
    else if constexpr (S == STORE_F16C) __stcs(reinterpret_cast<unsigned short*>(p), static_cast<unsigned short>(f16c_encode(v)));
    else __stcs(reinterpret_cast<unsigned short*>(p), __bfloat16_as_ushort(__float2bfloat16_rn(v)));
}

// The two 16-bit values of a 32-bit word (little endian: node x in the low half) as floats,
// and two floats stored as one rounded 16-bit pair (streaming store).
template <int S>
__device__ __forceinline__ float raw_lo(unsigned w) {
    if constexpr (S == STORE_F16) return __half2float(__ushort_as_half(static_cast<unsigned short>(w & 0xffffu)));
    else if constexpr (S == STORE_F16C) return f16c_decode(w & 0xffffu);
    else return __bfloat162float(__ushort_as_bfloat16(static_cast<unsigned short>(w & 0xffffu)));
}
template <int S>
__device__ __forceinline__ float raw_hi(unsigned w) {
    if constexpr (S == STORE_F16) return __half2float(__ushort_as_half(static_cast<unsigned short>(w >> 16)));
    else if constexpr (S == STORE_F16C) return f16c_decode(w >> 16);
    else return __bfloat162float(__ushort_as_bfloat16(static_cast<unsigned short>(w >> 16)));
}
template <int S>
__device__ __forceinline__ void store_pair(typename Codec<S>::T* p, float2 v) {
    unsigned w;
    if constexpr (S == STORE_F16) {
        const __half2 h = __floats2half2_rn(v.x, v.y);  // .x in the low half
        w = *reinterpret_cast<const unsigned*>(&h);
    } else if constexpr (S == STORE_F16C) {
        w = f16c_encode2(v);
    } else {
        const __nv_bfloat162 h = __floats2bfloat162_rn(v.x, v.y);
        w = *reinterpret_cast<const unsigned*>(&h);
    }
    __stcs(reinterpret_cast<unsigned*>(p), w);
}

// Zou-He on one of the two nodes of a packed pair (lane 0 = .x, 1 = .y); the
// formulas work on f, so shifted values are decoded and encoded around them.
template <int Q, bool HS>
__device__ __forceinline__ void zou_he_half(float2* f, int lane, uint8_t fl, const Geo& G) {
    using L = Lat<Q>;
    float t[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const float v = lane ? f[q].y : f[q].x;
        t[q] = HS ? fmaf(L::w(q), v, L::w(q)) : v;
    }
    if (fl & FL_ZH_IN) zou_he_inlet<Q>(t, G.uin);
    if (fl & FL_ZH_OUT) zou_he_outlet<Q>(t, G.rho_out);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const float v = HS ? fmaf(t[q], 1.0f / L::w(q), -1.0f) : t[q];
        if (lane) f[q].y = v;
        else f[q].x = v;
    }
}

// 16-bit storage with adjacent node pairs: a thread steps nodes x and x + 1 (x even),
// which sit in one 32-bit word of every plane. Directions without an x component
// load both nodes with one 32-bit load; every direction stores both with one packed
// conversion and one 32-bit store. Needs nx even (every row, hence every pair, starts
// on a 4-byte boundary; the plane pitch is a multiple of 64) and an even span start.
// The arithmetic is the same per node as in step_span_fast2, so results are identical.
template <int Q, int S, bool LES>
__device__ __forceinline__ void step_span_adjacent(const StepArgs& a, const Seg& sg) {
    using L = Lat<Q>;
    using C = Codec<S>;
    using T = typename C::T;
    const int nx = a.geo.nx, ny = a.geo.ny, nz = a.geo.nz;
    const int y = sg.y, z = sg.z;
    const unsigned row0 = static_cast<unsigned>(sg.row0);
    const int yl = (y + 1 == ny) ? (a.geo.periodic_y ? 0 : y + 1) : y + 1;
    const int yh = (y == 0) ? (a.geo.periodic_y ? ny - 1 : -1) : y - 1;
    const int zl = (z + 1 == nz) ? (a.geo.periodic_z ? 0 : z + 1) : z + 1;
    const int zh = (z == 0) ? (a.geo.periodic_z ? nz - 1 : -1) : z - 1;
    const int ysrc[3] = {yl, y, yh}, zsrc[3] = {zl, z, zh};
    const T* fin = static_cast<const T*>(a.fin);
    T* out = static_cast<T*>(a.fout);
    const unsigned P = static_cast<unsigned>(a.geo.pitch);
    const int lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    for (int base = sg.x0 + (threadIdx.x >> 5) * 64; base < sg.x1; base += nwarps * 64) {
        const int xa = base + 2 * lane;  // even
        if (xa >= sg.x1) continue;
        const bool vb = xa + 1 < sg.x1;  // node b = xa + 1 < nx always (nx even); unused when outside the span
        const uint8_t fa = a.flags[row0 + xa], fb = vb ? a.flags[row0 + xa + 1] : fa;
        float2 f[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const unsigned rowsrc = static_cast<unsigned>((zsrc[L::cz(q) + 1] * ny + ysrc[L::cy(q) + 1]) * nx);
            const T* pl = fin + (q * P + rowsrc);
            if (L::cx(q) == 0) {
                const unsigned w = __ldg(reinterpret_cast<const unsigned*>(pl + xa));
                f[q] = make_float2(raw_lo<S>(w), raw_hi<S>(w));
            } else {
                // source x - c_x of each node, wrapped in x
                int sa = xa - L::cx(q), sb = xa + 1 - L::cx(q);
                sa = sa < 0 ? sa + nx : (sa >= nx ? sa - nx : sa);
                sb = sb < 0 ? sb + nx : (sb >= nx ? sb - nx : sb);
                f[q] = make_float2(load_raw<S>(pl + sa), load_raw<S>(pl + sb));
            }
        }
        if (!vb) {  // node b lies outside the span: step a copy of node a, store nothing
#pragma unroll
            for (int q = 0; q < Q; ++q) f[q].y = f[q].x;
        }
        if ((fa | fb) & (FL_ZH_IN | FL_ZH_OUT)) {
            if (fa & (FL_ZH_IN | FL_ZH_OUT)) zou_he_half<Q, true>(f, 0, fa, a.geo);
            if (vb && (fb & (FL_ZH_IN | FL_ZH_OUT))) zou_he_half<Q, true>(f, 1, fb, a.geo);
        }
        float2 rho, u[3];
        trt_pairs2<Q, LES, true>(f, a.phys, rho, u);
        const bool bad = !(rho.x > 0.0f) || !(fabsf(u[0].x) < 1e30f) || (vb && (!(rho.y > 0.0f) || !(fabsf(u[0].y) < 1e30f)));
        if (bad) atomicOr(a.status, ERR_NONFINITE);
        T* oa = out + (row0 + xa);
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            if (vb) store_pair<S>(oa + q * P, f[q]);
            else store_raw<S>(oa + q * P, f[q].x);
        }
    }
}

// TRT pure-gather span, one block: each warp takes 64-node chunks, two nodes per
// thread (base + lane and base + lane + 32) in packed FP32 (trt_pairs2); shifted
// storage is updated in h directly.
template <int Q, int S, bool LES, bool IDX32>
__device__ __forceinline__ void step_span_fast2(const StepArgs& a, const Seg& sg) {
    using L = Lat<Q>;
    using C = Codec<S>;
    using T = typename C::T;
    constexpr bool HS = S != STORE_F32;
    if constexpr (HS && IDX32) {
        if ((a.geo.nx & 1) == 0 && (sg.x0 & 1) == 0) {  // uniform over the block
            step_span_adjacent<Q, S, LES>(a, sg);
            return;
        }
    }
    const int nx = a.geo.nx, ny = a.geo.ny, nz = a.geo.nz;
    const int y = sg.y, z = sg.z;
    const long long row0 = sg.row0;
    const int yl = (y + 1 == ny) ? (a.geo.periodic_y ? 0 : y + 1) : y + 1;
    const int yh = (y == 0) ? (a.geo.periodic_y ? ny - 1 : -1) : y - 1;
    const int zl = (z + 1 == nz) ? (a.geo.periodic_z ? 0 : z + 1) : z + 1;
    const int zh = (z == 0) ? (a.geo.periodic_z ? nz - 1 : -1) : z - 1;
    const int ysrc[3] = {yl, y, yh}, zsrc[3] = {zl, z, zh};
    const T* fin = static_cast<const T*>(a.fin);
    T* out = static_cast<T*>(a.fout);
    const int lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    for (int base = sg.x0 + (threadIdx.x >> 5) * 64; base < sg.x1; base += nwarps * 64) {
        const int xa = base + lane;
        if (xa >= sg.x1) continue;
        const bool vb = xa + 32 < sg.x1;
        const int xb = vb ? xa + 32 : xa;  // a short chunk computes node a twice and stores it once
        const uint8_t fa = a.flags[row0 + xa], fb = a.flags[row0 + xb];
        float2 f[Q];
        const int xsa[3] = {xa + 1 == nx ? 0 : xa + 1, xa, xa == 0 ? nx - 1 : xa - 1};
        const int xsb[3] = {xb + 1 == nx ? 0 : xb + 1, xb, xb == 0 ? nx - 1 : xb - 1};
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            if constexpr (IDX32) {
                const unsigned P = static_cast<unsigned>(a.geo.pitch);
                const unsigned rowsrc = static_cast<unsigned>((zsrc[L::cz(q) + 1] * ny + ysrc[L::cy(q) + 1]) * nx);
                const T* pl = fin + (q * P + rowsrc);
                f[q] = make_float2(load_raw<S>(pl + xsa[L::cx(q) + 1]), load_raw<S>(pl + xsb[L::cx(q) + 1]));
            } else {
                const long long rowsrc = (static_cast<long long>(zsrc[L::cz(q) + 1]) * ny + ysrc[L::cy(q) + 1]) * nx;
                const T* pl = fin + (q * a.geo.pitch + rowsrc);
                f[q] = make_float2(load_raw<S>(pl + xsa[L::cx(q) + 1]), load_raw<S>(pl + xsb[L::cx(q) + 1]));
            }
        }
        if ((fa | fb) & (FL_ZH_IN | FL_ZH_OUT)) {
            if (fa & (FL_ZH_IN | FL_ZH_OUT)) zou_he_half<Q, HS>(f, 0, fa, a.geo);
            if (fb & (FL_ZH_IN | FL_ZH_OUT)) zou_he_half<Q, HS>(f, 1, fb, a.geo);
        }
        float2 rho, u[3];
        trt_pairs2<Q, LES, HS>(f, a.phys, rho, u);
        const bool bad = !(rho.x > 0.0f) || !(fabsf(u[0].x) < 1e30f) || (vb && (!(rho.y > 0.0f) || !(fabsf(u[0].y) < 1e30f)));
        if (bad) atomicOr(a.status, ERR_NONFINITE);
        T* oa = out + (row0 + xa);
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            if constexpr (IDX32) {
                const unsigned P = static_cast<unsigned>(a.geo.pitch);
                store_raw<S>(oa + q * P, f[q].x);
                if (vb) store_raw<S>(oa + (q * P + 32u), f[q].y);
            } else {
                store_raw<S>(oa + q * a.geo.pitch, f[q].x);
                if (vb) store_raw<S>(oa + (q * a.geo.pitch + 32), f[q].y);
            }
        }
    }
}

// The same step for a row whose every node is a pure gather (no solid, no
// bounce-back, no curved link; Zou-He allowed) -- the bulk of a domain. Without
// the rare paths the kernel fits 64 registers.
template <int Q, int COLL, int S, bool LES, bool IDX32>
__device__ __forceinline__ void step_span_fast(const StepArgs& a, const Seg& sg) {
    if constexpr (COLL == COLL_TRT) {
        step_span_fast2<Q, S, LES, IDX32>(a, sg);
        return;
    }
    using L = Lat<Q>;
    using C = Codec<S>;
    using T = typename C::T;
    const int nx = a.geo.nx, ny = a.geo.ny, nz = a.geo.nz;
    const int y = sg.y, z = sg.z;
    const long long row0 = sg.row0;
    // Source-row offsets of the (cy, cz) shifts relative to this row, y / z wraps
    // applied: uniform across the warp, so with the plane offsets they form
    // warp-uniform address terms and each load is a per-thread base plus a uniform offset.
    const int yl = (y + 1 == ny) ? (a.geo.periodic_y ? 0 : y + 1) : y + 1;  // source row for cy = -1
    const int yh = (y == 0) ? (a.geo.periodic_y ? ny - 1 : -1) : y - 1;     // source row for cy = +1
    const int zl = (z + 1 == nz) ? (a.geo.periodic_z ? 0 : z + 1) : z + 1;
    const int zh = (z == 0) ? (a.geo.periodic_z ? nz - 1 : -1) : z - 1;
    const int ysrc[3] = {yl, y, yh}, zsrc[3] = {zl, z, zh};
    const T* fin = static_cast<const T*>(a.fin);
    T* out = static_cast<T*>(a.fout);
    for (int x = sg.x0 + threadIdx.x; x < sg.x1; x += blockDim.x) {
        const uint8_t fl = a.flags[row0 + x];
        // source x for cx = -1, 0, +1 (periodic in x)
        const int xs[3] = {x + 1 == nx ? 0 : x + 1, x, x == 0 ? nx - 1 : x - 1};
        float f[Q];
        if constexpr (IDX32) {
            // element index in 32-bit unsigned arithmetic (Q * pitch < 2^32): the
            // plane + source-row part is uniform, each access adds x and scales once
            const unsigned P = static_cast<unsigned>(a.geo.pitch);
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const unsigned rowsrc = static_cast<unsigned>((zsrc[L::cz(q) + 1] * ny + ysrc[L::cy(q) + 1]) * nx);
                f[q] = C::load(fin + (q * P + rowsrc + static_cast<unsigned>(xs[L::cx(q) + 1])), L::w(q));
            }
        } else {
            const long long P = a.geo.pitch;
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const long long rowsrc = (static_cast<long long>(zsrc[L::cz(q) + 1]) * ny + ysrc[L::cy(q) + 1]) * nx;
                f[q] = C::load(fin + (q * P + rowsrc + xs[L::cx(q) + 1]), L::w(q));
            }
        }
        if (fl & FL_ZH_IN) zou_he_inlet<Q>(f, a.geo.uin);
        if (fl & FL_ZH_OUT) zou_he_outlet<Q>(f, a.geo.rho_out);
        float rho, u[3];
        if constexpr (COLL == COLL_TRT) {
            trt_pairs<Q, LES>(f, a.phys, rho, u);
        } else {
            node_moments<Q>(f, a.phys.g, rho, u);
            collide<Q, COLL, LES>(f, rho, u, a.phys);
        }
        if (!(rho > 0.0f) || !(fabsf(u[0]) < 1e30f)) atomicOr(a.status, ERR_NONFINITE);
        if constexpr (IDX32) {
            const unsigned P = static_cast<unsigned>(a.geo.pitch), i = static_cast<unsigned>(row0 + x);
#pragma unroll
            for (int q = 0; q < Q; ++q) C::store_stream(out + (q * P + i), f[q], L::w(q));
        } else {
            const long long P = a.geo.pitch, i = row0 + x;
#pragma unroll
            for (int q = 0; q < Q; ++q) C::store_stream(out + (q * P + i), f[q], L::w(q));
        }
    }
}

// Single lattice. General segments: one SEG-thread block per segment (a warp per
// 32-node chunk). Pure-gather spans: one block per span.
template <int Q, int COLL, int S, bool LES>
__global__ void __launch_bounds__(64) k_step(const StepArgs a) {
    step_chunk<Q, COLL, S, LES>(a, a.rows[blockIdx.x], blockIdx.x, threadIdx.x >> 5);
}

// TRT segments carry two nodes per thread (twice the registers, half the threads per node).
// Register budget: WK_FAST_MAX_THREADS / WK_FAST_*_MIN_BLOCKS (common.cuh).
template <int Q, int COLL, int S, bool LES, bool IDX32>
__global__ void __launch_bounds__(WK_FAST_MAX_THREADS, COLL == COLL_TRT ? (Q == 9 ? WK_FAST_TRT9_MIN_BLOCKS
                                                                                   : WK_FAST_TRT_MIN_BLOCKS)
                                                                        : WK_FAST_OTHER_MIN_BLOCKS)
    k_step_fast(const StepArgs a) {
    step_span_fast<Q, COLL, S, LES, IDX32>(a, span_decode(a.spans[blockIdx.x], a.geo));
}

// ------------------------------------------------------------------ many lattices
// A batch advances many independent lattices (same Q, collision model and
// storage; any sizes, parameters and geometry) with one launch per row kind.
// Each member's step arguments live in device memory; its buffers swap with the
// batch's step parity, so the table stays valid while the members step together.
struct BatchDom {
    StepArgs a;        // fin / fout (th.tin / th.tout) unused: taken from buf[] (tbuf[]) by parity
    void* buf[2];      // the member's two state buffers
    float* tbuf[2];    // its two temperature buffers (thermal members)
    int cur0;          // index of the buffer holding the state at batch parity 0
    int gen_first;     // first entry of this member in the general-row list
};

struct BatchArgs {
    const BatchDom* dom;
    const uint2* rows;   // general segments (member, segment), one block per entry
    int nrows;
    int parity;          // batch step parity of this launch
    const uint4* spans;  // pure-gather spans (member, row, x0, x1), one block per entry
    int nspans;
};

__device__ __forceinline__ StepArgs batch_member(const BatchArgs& b, unsigned m) {
    const BatchDom* d = b.dom + m;
    StepArgs a = d->a;
    const int c = d->cur0 ^ b.parity;
    a.fin = d->buf[c];
    a.fout = d->buf[c ^ 1];
    a.th.tin = d->tbuf[c];
    a.th.tout = d->tbuf[c ^ 1];
    return a;
}

template <int Q, int COLL, int S, bool LES>
__global__ void __launch_bounds__(64) k_step_batch(const BatchArgs b) {
    const uint2 r = b.rows[blockIdx.x];
    const StepArgs a = batch_member(b, r.x);
    step_chunk<Q, COLL, S, LES>(a, r.y, static_cast<int>(blockIdx.x) - b.dom[r.x].gen_first, threadIdx.x >> 5);
}

template <int Q, int COLL, int S, bool LES, bool IDX32>
__global__ void __launch_bounds__(WK_FAST_MAX_THREADS, COLL == COLL_TRT ? (Q == 9 ? WK_FAST_TRT9_MIN_BLOCKS
                                                                                   : WK_FAST_TRT_MIN_BLOCKS)
                                                                        : WK_FAST_OTHER_MIN_BLOCKS)
    k_step_fast_batch(const BatchArgs b) {
    const uint4 sp = b.spans[blockIdx.x];
    const StepArgs a = batch_member(b, sp.x);
    step_span_fast<Q, COLL, S, LES, IDX32>(a, span_decode(sp, a.geo));
}

// Sum one step's momentum-exchange slots in slot order with one 256-thread block
// (thread t takes slots t, t + 256, ... in order, then a fixed tree) and append
// the force to the history ring. Same sum for any launch, so forces are
// reproducible bit for bit.
__device__ __forceinline__ void mem_reduce_block(const double* __restrict__ contrib, int n, unsigned* hist_step,
                                                 double* hist, int hist_cap) {
    __shared__ double red[3][256];
    double s[3] = {0.0, 0.0, 0.0};
    for (int j = threadIdx.x; j < n; j += 256)
        for (int c = 0; c < 3; ++c) s[c] += contrib[3 * static_cast<long long>(j) + c];
    for (int c = 0; c < 3; ++c) red[c][threadIdx.x] = s[c];
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int c = 0; c < 3; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const unsigned step = *hist_step;
        double* h = hist + 3 * static_cast<long long>(step % static_cast<unsigned>(hist_cap));
        h[0] = red[0][0];
        h[1] = red[1][0];
        h[2] = red[2][0];
        *hist_step = step + 1u;
    }
}

// Re-gather f^k from g^{k-1} and write FP32 populations and/or macroscopic fields
// (the reference's f_src and its rho/u/speed arrays after step k,
// lattice_grid_2d.cpp:257-262). Solid nodes report their frozen populations.
template <int Q, int S>
__global__ void __launch_bounds__(512) k_materialise(const void* fin_v, const uint8_t* flags, Geo geo, Links links,
                                                     Physics phys, Out out, int xchunks, Thermal th) {
    using L = Lat<Q>;
    using C = Codec<S>;
    using T = typename C::T;
    const T* fin = static_cast<const T*>(fin_v);
    const int row = blockIdx.x / xchunks;
    const int x = (blockIdx.x - row * xchunks) * blockDim.x + threadIdx.x;
    if (x >= geo.nx) return;
    const int y = row % geo.ny, z = row / geo.ny;
    const long long i = static_cast<long long>(row) * geo.nx + x;
    const uint8_t fl = flags[i];
    float f[Q];
    if ((fl & FL_TYPE) == CT_SOLID) {
#pragma unroll
        for (int q = 0; q < Q; ++q) f[q] = C::load(fin + q * geo.pitch + i, L::w(q));
    } else {
        unsigned bb;
        gather<Q, S>(fin, geo, flags, links, x, y, z, i, fl, f, bb);
    }
    if (out.f) {
#pragma unroll
        for (int q = 0; q < Q; ++q) out.f[q * geo.pitch + i] = f[q];
    }
    if (out.rho) {
        float g[3] = {phys.g[0], phys.g[1], phys.g[2]};
        if (th.on) {  // the step's local buoyancy: T^k is the sum of the current post-collision temperature
            float t5[5];
#pragma unroll
            for (int q = 0; q < 5; ++q) t5[q] = th.tin[q * geo.pitch + i];
            g[1] = buoyant_gy(th, phys.g[1], sum_t5(t5));
        }
        float rho, u[3];
        node_moments<Q>(f, g, rho, u);
        out.rho[i] = rho;
        out.ux[i] = u[0];
        out.uy[i] = u[1];
        if (out.uz) out.uz[i] = u[2];
        out.speed[i] = sqrtf(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    }
}

// Initial collide of a coupled flow + temperature state (f^0 and T populations
// g^0 in FP32 scratch): A <- Collide(f^0) with the local buoyancy, TA <- Collide_T(g^0);
// B <- f^0, TB <- g^0. Solid nodes copy through.
template <int COLL, int S, bool LES>
__global__ void __launch_bounds__(512) k_initial_thermal(const float* f0, const float* t0, void* a_v, void* b_v,
                                                         float* ta, float* tb, const uint8_t* flags, Geo geo,
                                                         Physics phys, Thermal th, int xchunks) {
    using L = Lat<9>;
    using C = Codec<S>;
    using T = typename C::T;
    const int row = blockIdx.x / xchunks;
    const int x = (blockIdx.x - row * xchunks) * blockDim.x + threadIdx.x;
    if (x >= geo.nx) return;
    const long long i = static_cast<long long>(row) * geo.nx + x;
    const long long P = geo.pitch;
    float f[9], t5[5];
#pragma unroll
    for (int q = 0; q < 9; ++q) f[q] = f0[q * P + i];
#pragma unroll
    for (int q = 0; q < 5; ++q) t5[q] = t0[q * P + i];
    T* A = static_cast<T*>(a_v);
    T* Bf = static_cast<T*>(b_v);
#pragma unroll
    for (int q = 0; q < 9; ++q) C::store(Bf + q * P + i, f[q], L::w(q));
#pragma unroll
    for (int q = 0; q < 5; ++q) tb[q * P + i] = t5[q];
    if ((flags[i] & FL_TYPE) != CT_SOLID) {
        const float Tn = sum_t5(t5);
        Physics ph = phys;
        ph.g[1] = buoyant_gy(th, phys.g[1], Tn);
        float rho, u[3];
        node_moments<9>(f, ph.g, rho, u);
        collide<9, COLL, LES>(f, rho, u, ph);
        collide_t5(t5, Tn, u, th.omega_t);
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) C::store(A + q * P + i, f[q], L::w(q));
#pragma unroll
    for (int q = 0; q < 5; ++q) ta[q * P + i] = t5[q];
}

// Initial collide from FP32 populations f^0: buffer A <- g^0 = Collide(f^0)
// (solid nodes copy through, d2q9_collision_bgk.ispc:22-28), buffer B <- f^0.
// B's fluid entries are overwritten by the first step; until then B is the
// reference's f_src, and its solid entries stay the frozen populations.
template <int Q, int COLL, int S, bool LES>
__global__ void __launch_bounds__(512) k_initial(const float* f0, void* a_v, void* b_v, const uint8_t* flags,
                                                 Geo geo, Physics phys, int xchunks) {
    using L = Lat<Q>;
    using C = Codec<S>;
    using T = typename C::T;
    const int row = blockIdx.x / xchunks;
    const int x = (blockIdx.x - row * xchunks) * blockDim.x + threadIdx.x;
    if (x >= geo.nx) return;
    const long long i = static_cast<long long>(row) * geo.nx + x;
    float f[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) f[q] = f0[q * geo.pitch + i];
    T* A = static_cast<T*>(a_v);
    T* Bf = static_cast<T*>(b_v);
#pragma unroll
    for (int q = 0; q < Q; ++q) C::store(Bf + q * geo.pitch + i, f[q], L::w(q));
    if ((flags[i] & FL_TYPE) != CT_SOLID) {
        float rho, u[3];
        node_moments<Q>(f, phys.g, rho, u);
        collide<Q, COLL, LES>(f, rho, u, phys);
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) C::store(A + q * geo.pitch + i, f[q], L::w(q));
}

}  // namespace wk
