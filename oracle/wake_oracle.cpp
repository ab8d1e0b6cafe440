// wake lattice-update ORACLE — CPU restatement used only as a test checker.
//
// This file is test infrastructure. Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg load it; the product (wake_b200/) never does.
//
// It restates, in plain C++ templated on the arithmetic type (float for
// parity with the reference's FP32 kernels, double for the FP64 error
// reference), the algorithms of the reference's lattice update:
//
//   lattice tables ........ include/wake/ispc/lbm_d2q9.isph:8-24, lbm_d3q19.isph:8-41, lbm_d3q27.isph:8-55
//   BGK + Guo forcing ..... src/ispc/d2q9_collision_bgk.ispc:5-86, d3q19_collision_bgk.ispc:4-75
//   TRT + split Guo ....... src/ispc/d2q9_collision_trt.ispc:7-92, d3q19_collision_trt.ispc:5-93,
//                           d3q27_collision_mrt.ispc:5-91 (a TRT despite the file name)
//   MRT ................... src/ispc/d2q9_collision_mrt.ispc:6-137 (Lallemand-Luo),
//                           src/ispc/d3q19_collision_mrt.ispc:26-176 (d'Humieres; 7-digit inverse :4-24)
//   pull streaming ........ src/ispc/d2q9_streaming.ispc:4-95, d3q19_streaming.ispc:4-104, d3q27_streaming.ispc:4-35
//   Zou-He 2D ............. src/ispc/d2q9_boundaries.ispc:43-121
//   BFL curved links ...... src/ispc/d3q19_curved.ispc:7-71; link build src/grid/lattice_grid_3d.cpp:217-290
//   Smagorinsky tau ....... src/ispc/d2q9_les.ispc:6-57, d3q19_les.ispc:7-66
//   moments / speed ....... src/ispc/d2q9_moments.ispc:4-79, d3q19_moments.ispc:4-82, d3q27_moments.ispc:4-32
//   momentum exchange ..... src/ispc/forces_momentum_exchange.ispc:6-138
//   thermal D2Q9 .......... src/ispc/thermal_kernels.ispc:4-81
//   step order ............ src/grid/lattice_grid_2d.cpp:195-265, src/grid/lattice_grid_3d.cpp:301-380
//   Strouhal FFT .......... src/forces/strouhal_analyzer.cpp:8-89
//
// and the pieces the reference does not have (no reference source; checked
// only against analytic properties and this oracle):
//   * Smagorinsky tau applied per node (the reference computes it and drops it,
//     lattice_grid_2d.cpp:205, lattice_grid_3d.cpp:312),
//   * D3Q19 Zou-He velocity inlet / pressure outlet (Hecht & Harting 2010,
//     J. Stat. Mech. P01018),
//   * y/z periodic wrap together with solids in 3D,
//   * D3Q27 raw-moment MRT on the tensor-product monomial basis
//     (d'Humieres et al. 2002; Geier et al. 2015 factorisation),
//   * exact (unrounded) D3Q19 MRT inverse M^T diag(1/|M_k|^2),
//   * D2Q5 temperature coupled to the D2Q9 flow with a local Boussinesq force
//     (the reference couples a D2Q9 temperature through one domain-averaged
//     force, src/scenarios/thermal_convection.cpp:70): per node
//       T = sum g,  a_y = beta_g (T - T_ref) added to the body force of the
//       flow collision, g_q* = g_q - (g_q - w_q T (1 + 3 c_q.u)) / tau_T with u
//       the flow's forced velocity (first-order equilibrium as thermal_kernels.ispc:32),
//     streaming with anti-bounce-back g_q = -g*_opp + 2 w_q T_wall through the
//     y walls (Dirichlet; Ginzburg 2005) and bounce-back at solid nodes (adiabatic).
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

namespace {

// Runs fn(begin, end) over [0, n) split into contiguous ranges on host threads
// (WAKE_ORACLE_THREADS, default: every hardware thread). Used only for loops
// whose iterations write disjoint outputs and read nothing another iteration
// writes, so the result does not depend on the thread count.
template <class Fn>
void parallel_ranges(std::size_t n, Fn&& fn) {
    unsigned t = std::thread::hardware_concurrency();
    if (const char* e = std::getenv("WAKE_ORACLE_THREADS")) t = static_cast<unsigned>(std::max(1, std::atoi(e)));
    t = std::max(1u, std::min<unsigned>(t, 64u));
    if (t == 1 || n < 4096) {
        fn(std::size_t(0), n);
        return;
    }
    const std::size_t chunk = (n + t - 1) / t;
    std::vector<std::thread> pool;
    for (unsigned k = 0; k < t; ++k) {
        const std::size_t b = k * chunk, e = std::min(n, b + chunk);
        if (b >= e) break;
        pool.emplace_back([&fn, b, e] { fn(b, e); });
    }
    for (auto& th : pool) th.join();
}

enum Cell : uint8_t { FLUID = 0, SOLID = 1, INFLOW = 2, OUTFLOW = 3, MOVING_WALL = 6 };

// ----------------------------------------------------------------------------- lattice tables
struct D2Q9T {
    static constexpr int Q = 9, D = 2;
    static constexpr int cx[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
    static constexpr int cy[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
    static constexpr int cz[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    static constexpr int opp[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
    static constexpr double wn[9] = {4, 1, 1, 1, 1, 0.25, 0.25, 0.25, 0.25};  // w = wn / 9
    static constexpr double wd = 9.0;
};
struct D3Q19T {
    static constexpr int Q = 19, D = 3;
    static constexpr int cx[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    static constexpr int cy[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
    static constexpr int cz[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
    static constexpr int opp[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
    static constexpr double wn[19] = {12, 2, 2, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1};  // w = wn / 36
    static constexpr double wd = 36.0;
};
struct D3Q27T {
    static constexpr int Q = 27, D = 3;
    static constexpr int cx[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};
    static constexpr int cy[27] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1};
    static constexpr int cz[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1};
    // true opposites; the reference's table (lbm_d3q27.isph:35-40) mis-pairs the corners
    static constexpr int opp[27] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15,
                                    26, 25, 24, 23, 22, 21, 20, 19};
    static constexpr double wn[27] = {64, 16, 16, 16, 16, 16, 16, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4,
                                      1, 1, 1, 1, 1, 1, 1, 1};  // w = wn / 216
    static constexpr double wd = 216.0;
};

template <class L, class R>
inline R wq(int q) {
    return static_cast<R>(L::wn[q]) / static_cast<R>(L::wd);
}

template <class L, class R>
inline R feq(int q, R rho, R ux, R uy, R uz) {
    const R cu = R(L::cx[q]) * ux + R(L::cy[q]) * uy + R(L::cz[q]) * uz;
    const R u2 = ux * ux + uy * uy + uz * uz;
    return wq<L, R>(q) * rho * (R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * u2);
}

// Pre-collision moments with the Guo half-force velocity shift (d2q9_collision_bgk.ispc:37-51).
template <class L, class R>
inline void moments(const R* f, R g[3], R& rho, R u[3]) {
    R r = 0, j[3] = {0, 0, 0};
    for (int q = 0; q < L::Q; ++q) {
        r += f[q];
        j[0] += f[q] * R(L::cx[q]);
        j[1] += f[q] * R(L::cy[q]);
        j[2] += f[q] * R(L::cz[q]);
    }
    rho = r;
    const R inv = R(1) / r;
    for (int a = 0; a < 3; ++a) u[a] = (j[a] + R(0.5) * r * g[a]) * inv;
}

// ----------------------------------------------------------------------------- Smagorinsky
// d2q9_les.ispc:6-57 / d3q19_les.ispc:7-66: Pi^neq from f - feq(rho,u), Q = sqrt(2 Pi:Pi),
// tau_eff = (tau0 + sqrt(tau0^2 + 18 sqrt(2) Cs^2 Q / rho)) / 2.
template <class L, class R>
inline R smagorinsky_tau(const R* f, R rho, const R u[3], R tau0, R cs) {
    R pi[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int q = 0; q < L::Q; ++q) {
        const R fn = f[q] - feq<L, R>(q, rho, u[0], u[1], u[2]);
        const R c[3] = {R(L::cx[q]), R(L::cy[q]), R(L::cz[q])};
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) pi[a][b] += c[a] * c[b] * fn;
    }
    R sum = 0;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) sum += pi[a][b] * pi[a][b];
    const R qs = std::sqrt(R(2) * sum);
    const R pref = R(18) * R(1.4142135623730951) * cs * cs;
    return R(0.5) * (tau0 + std::sqrt(tau0 * tau0 + (pref / rho) * qs));
}

// ----------------------------------------------------------------------------- collisions
template <class L, class R>
inline void collide_bgk(const R* f, R* out, R rho, const R u[3], const R g[3], R tau) {
    const R om = R(1) / tau, pre = R(1) - R(0.5) * om;
    const R ug = u[0] * g[0] + u[1] * g[1] + u[2] * g[2];
    for (int q = 0; q < L::Q; ++q) {
        const R cu = R(L::cx[q]) * u[0] + R(L::cy[q]) * u[1] + R(L::cz[q]) * u[2];
        const R cg = R(L::cx[q]) * g[0] + R(L::cy[q]) * g[1] + R(L::cz[q]) * g[2];
        const R fi = pre * wq<L, R>(q) * rho * (R(3) * (cg - ug) + R(9) * cu * cg);
        out[q] = f[q] - om * (f[q] - feq<L, R>(q, rho, u[0], u[1], u[2])) + fi;
    }
}

template <class L, class R>
inline void collide_trt(const R* f, R* out, R rho, const R u[3], const R g[3], R tau_s, R tau_a) {
    const R os = R(1) / tau_s, oa = R(1) / tau_a;
    const R ps = R(1) - R(0.5) * os, pa = R(1) - R(0.5) * oa;
    const R ug = u[0] * g[0] + u[1] * g[1] + u[2] * g[2];
    R fe[L::Q];
    for (int q = 0; q < L::Q; ++q) fe[q] = feq<L, R>(q, rho, u[0], u[1], u[2]);
    for (int q = 0; q < L::Q; ++q) {
        const int o = L::opp[q];
        const R fs = R(0.5) * (f[q] + f[o]), fa = R(0.5) * (f[q] - f[o]);
        const R es = R(0.5) * (fe[q] + fe[o]), ea = R(0.5) * (fe[q] - fe[o]);
        const R cu = R(L::cx[q]) * u[0] + R(L::cy[q]) * u[1] + R(L::cz[q]) * u[2];
        const R cg = R(L::cx[q]) * g[0] + R(L::cy[q]) * g[1] + R(L::cz[q]) * g[2];
        const R Fa = pa * wq<L, R>(q) * rho * (R(3) * cg);
        const R Fs = ps * wq<L, R>(q) * rho * (-R(3) * ug + R(9) * cu * cg);
        out[q] = f[q] - os * (fs - es) - oa * (fa - ea) + Fs + Fa;
    }
}

// D2Q9 Lallemand-Luo basis (d2q9_collision_mrt.ispc:44-52) as polynomials of c.
inline double d2q9_basis(int k, int q) {
    const double x = D2Q9T::cx[q], y = D2Q9T::cy[q], c2 = x * x + y * y;
    switch (k) {
        case 0: return 1;
        case 1: return 3 * c2 - 4;
        case 2: return 4.5 * c2 * c2 - 10.5 * c2 + 4;
        case 3: return x;
        case 4: return (3 * c2 - 5) * x;
        case 5: return y;
        case 6: return (3 * c2 - 5) * y;
        case 7: return x * x - y * y;
        default: return x * y;
    }
}

template <class R>
inline void collide_mrt_d2q9(const R* f, R* out, R rho, const R u[3], const R g[3], R tau_shear, R tau_bulk) {
    // rates d2q9_collision_mrt.ispc:19-25; forcing :82-91; relaxation :94-102
    const R s[9] = {0, R(1) / tau_bulk, R(1.4), 0, R(1.6), 0, R(1.6), R(1) / tau_shear, R(1) / tau_shear};
    R m[9];
    for (int k = 0; k < 9; ++k) {
        R a = 0;
        for (int q = 0; q < 9; ++q) a += R(d2q9_basis(k, q)) * f[q];
        m[k] = a;
    }
    const R ux = u[0], uy = u[1], ux2 = ux * ux, uy2 = uy * uy, u2 = ux2 + uy2;
    const R meq[9] = {rho, rho * (R(-2) + R(3) * u2), rho * (R(1) - R(3) * u2), rho * ux, -rho * ux,
                      rho * uy, -rho * uy, rho * (ux2 - uy2), rho * ux * uy};
    const R pre = R(1) - R(0.5) * s[8];
    const R F3 = rho * g[0], F5 = rho * g[1];
    const R F[9] = {0, R(6) * (ux * F3 + uy * F5), R(-6) * (ux * F3 + uy * F5), F3, -F3, F5, -F5,
                    R(2) * (ux * F3 - uy * F5), ux * F5 + uy * F3};
    for (int k = 0; k < 9; ++k) {
        const R fk = (k == 3 || k == 5) ? F[k] : (k == 0 ? R(0) : pre * F[k]);
        m[k] = m[k] - s[k] * (m[k] - meq[k]) + fk;
    }
    static const double norm[9] = {9, 36, 36, 6, 12, 6, 12, 4, 4};
    for (int q = 0; q < 9; ++q) {
        R a = 0;
        for (int k = 0; k < 9; ++k) a += R(d2q9_basis(k, q) / norm[k]) * m[k];
        out[q] = a;
    }
}

// D3Q19 d'Humieres basis (d3q19_collision_mrt.ispc:60-103) as polynomials of c.
inline double d3q19_basis(int k, int q) {
    const double x = D3Q19T::cx[q], y = D3Q19T::cy[q], z = D3Q19T::cz[q], c2 = x * x + y * y + z * z;
    switch (k) {
        case 0: return 1;
        case 1: return 19 * c2 - 30;
        case 2: return (21 * c2 * c2 - 53 * c2 + 24) / 2;
        case 3: return x;
        case 4: return (5 * c2 - 9) * x;
        case 5: return y;
        case 6: return (5 * c2 - 9) * y;
        case 7: return z;
        case 8: return (5 * c2 - 9) * z;
        case 9: return 3 * x * x - c2;
        case 10: return (3 * c2 - 5) * (3 * x * x - c2);
        case 11: return y * y - z * z;
        case 12: return (3 * c2 - 5) * (y * y - z * z);
        case 13: return x * y;
        case 14: return y * z;
        case 15: return x * z;
        case 16: return (y * y - z * z) * x;
        case 17: return (z * z - x * x) * y;
        default: return (y * y - x * x) * z;
    }
}

// Inverse M^T diag(1/|M_k|^2); `rounded` reproduces the reference's 7-decimal table
// (d3q19_collision_mrt.ispc:4-24), whose column sums differ from the exact ones by ~1e-7.
struct D3Q19Inverse {
    double exact[19][19];
    double rounded[19][19];
    D3Q19Inverse() {
        for (int k = 0; k < 19; ++k) {
            double n = 0;
            for (int q = 0; q < 19; ++q) n += d3q19_basis(k, q) * d3q19_basis(k, q);
            for (int q = 0; q < 19; ++q) {
                exact[q][k] = d3q19_basis(k, q) / n;
                rounded[q][k] = std::nearbyint(exact[q][k] * 1e7) / 1e7;
            }
        }
    }
};
const D3Q19Inverse& d3q19_inverse() {
    static const D3Q19Inverse inv;
    return inv;
}

template <class R>
inline void collide_mrt_d3q19(const R* f, R* out, R rho, const R u[3], const R g[3], R tau_shear, R tau_bulk,
                              bool exact) {
    // rates d3q19_collision_mrt.ispc:41-48; equilibria :119-138; forcing on j and q :141-148
    const R sn = R(1) / tau_shear;
    const R s[19] = {0, R(1) / tau_bulk, R(1.4), 0, R(1.2), 0, R(1.2), 0, R(1.2), sn, R(1.4), sn, R(1.4),
                     sn, sn, sn, R(1.98), R(1.98), R(1.98)};
    R m[19];
    for (int k = 0; k < 19; ++k) {
        R a = 0;
        for (int q = 0; q < 19; ++q) a += R(d3q19_basis(k, q)) * f[q];
        m[k] = a;
    }
    const R ux = u[0], uy = u[1], uz = u[2];
    const R ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz, u2 = ux2 + uy2 + uz2;
    R meq[19];
    meq[0] = rho;
    meq[1] = rho * (R(-11) + R(19) * u2);
    meq[2] = rho * (R(3) - R(5.5) * u2);
    meq[3] = rho * ux;
    meq[4] = R(-2) / R(3) * rho * ux;
    meq[5] = rho * uy;
    meq[6] = R(-2) / R(3) * rho * uy;
    meq[7] = rho * uz;
    meq[8] = R(-2) / R(3) * rho * uz;
    meq[9] = rho * (R(2) * ux2 - uy2 - uz2);
    meq[10] = R(-0.5) * meq[9];
    meq[11] = rho * (uy2 - uz2);
    meq[12] = R(-0.5) * meq[11];
    meq[13] = rho * ux * uy;
    meq[14] = rho * uy * uz;
    meq[15] = rho * ux * uz;
    meq[16] = meq[17] = meq[18] = 0;
    R F[19] = {0};
    F[3] = rho * g[0];
    F[4] = R(-2) / R(3) * rho * g[0];
    F[5] = rho * g[1];
    F[6] = R(-2) / R(3) * rho * g[1];
    F[7] = rho * g[2];
    F[8] = R(-2) / R(3) * rho * g[2];
    for (int k = 0; k < 19; ++k) m[k] = m[k] - s[k] * (m[k] - meq[k]) + F[k];
    const D3Q19Inverse& inv = d3q19_inverse();
    for (int q = 0; q < 19; ++q) {
        R a = 0;
        for (int k = 0; k < 19; ++k) a += R(exact ? inv.exact[q][k] : inv.rounded[q][k]) * m[k];
        out[q] = a;
    }
}

// D3Q27 raw-moment MRT (no reference implementation). Basis: monomials
// c_x^a c_y^b c_z^c, a,b,c in {0,1,2}; the inverse is built numerically here
// (Gauss-Jordan), independently of the factorised transform used on the GPU.
// Conserved moments relax at 0, the deviatoric second-order block at 1/tau,
// the trace at 1/tau_bulk, third order at s3, fourth order and above at s4.
// Guo forcing enters as M^-1 (I - S/2) M F_i.
struct D3Q27Basis {
    double M[27][27];
    double Minv[27][27];
    int order[27];
    int a[27], b[27], c[27];
    D3Q27Basis() {
        int k = 0;
        for (int az = 0; az < 3; ++az)
            for (int ay = 0; ay < 3; ++ay)
                for (int ax = 0; ax < 3; ++ax, ++k) {
                    a[k] = ax; b[k] = ay; c[k] = az;
                    order[k] = ax + ay + az;
                    for (int q = 0; q < 27; ++q)
                        M[k][q] = std::pow(double(D3Q27T::cx[q]), ax) * std::pow(double(D3Q27T::cy[q]), ay) *
                                  std::pow(double(D3Q27T::cz[q]), az);
                }
        double A[27][54];
        for (int i = 0; i < 27; ++i)
            for (int j = 0; j < 54; ++j) A[i][j] = j < 27 ? M[i][j] : (j - 27 == i ? 1.0 : 0.0);
        for (int col = 0; col < 27; ++col) {
            int piv = col;
            for (int r = col + 1; r < 27; ++r)
                if (std::fabs(A[r][col]) > std::fabs(A[piv][col])) piv = r;
            for (int j = 0; j < 54; ++j) std::swap(A[col][j], A[piv][j]);
            const double d = A[col][col];
            for (int j = 0; j < 54; ++j) A[col][j] /= d;
            for (int r = 0; r < 27; ++r)
                if (r != col) {
                    const double fct = A[r][col];
                    for (int j = 0; j < 54; ++j) A[r][j] -= fct * A[col][j];
                }
        }
        for (int i = 0; i < 27; ++i)
            for (int j = 0; j < 27; ++j) Minv[i][j] = A[i][j + 27];
    }
    int idx(int ax, int ay, int az) const { return ax + 3 * ay + 9 * az; }
};
const D3Q27Basis& d3q27_basis() {
    static const D3Q27Basis b;
    return b;
}

template <class R>
inline void d3q27_relax_moments(R* md, R s_nu, R s_b, R s3, R s4, bool half) {
    // md: moment vector; applies S (or I - S/2 when half) in place.
    const D3Q27Basis& B = d3q27_basis();
    auto rate = [&](R s) { return half ? (R(1) - R(0.5) * s) : s; };
    const int i200 = B.idx(2, 0, 0), i020 = B.idx(0, 2, 0), i002 = B.idx(0, 0, 2);
    const R A = md[i200] + md[i020] + md[i002];
    const R Bd = md[i200] - md[i020];
    const R Cd = md[i200] - md[i002];
    const R A2 = rate(s_b) * A, B2 = rate(s_nu) * Bd, C2 = rate(s_nu) * Cd;
    for (int k = 0; k < 27; ++k) {
        const int o = B.order[k];
        if (o <= 1) md[k] = half ? md[k] : R(0);
        else if (o == 2) {
            if (k == i200 || k == i020 || k == i002) continue;
            md[k] *= rate(s_nu);
        } else if (o == 3) md[k] *= rate(s3);
        else md[k] *= rate(s4);
    }
    md[i200] = (A2 + B2 + C2) / R(3);
    md[i020] = (A2 - R(2) * B2 + C2) / R(3);
    md[i002] = (A2 + B2 - R(2) * C2) / R(3);
}

template <class R>
inline void collide_mrt_d3q27(const R* f, R* out, R rho, const R u[3], const R g[3], R tau, R tau_bulk, R s3,
                              R s4) {
    const D3Q27Basis& B = d3q27_basis();
    R d[27], md[27], Fi[27], mF[27];
    const R ug = u[0] * g[0] + u[1] * g[1] + u[2] * g[2];
    for (int q = 0; q < 27; ++q) {
        d[q] = f[q] - feq<D3Q27T, R>(q, rho, u[0], u[1], u[2]);
        const R cu = R(D3Q27T::cx[q]) * u[0] + R(D3Q27T::cy[q]) * u[1] + R(D3Q27T::cz[q]) * u[2];
        const R cg = R(D3Q27T::cx[q]) * g[0] + R(D3Q27T::cy[q]) * g[1] + R(D3Q27T::cz[q]) * g[2];
        Fi[q] = wq<D3Q27T, R>(q) * rho * (R(3) * (cg - ug) + R(9) * cu * cg);
    }
    for (int k = 0; k < 27; ++k) {
        R a = 0, b = 0;
        for (int q = 0; q < 27; ++q) {
            a += R(B.M[k][q]) * d[q];
            b += R(B.M[k][q]) * Fi[q];
        }
        md[k] = a;
        mF[k] = b;
    }
    d3q27_relax_moments<R>(md, R(1) / tau, R(1) / tau_bulk, s3, s4, false);
    d3q27_relax_moments<R>(mF, R(1) / tau, R(1) / tau_bulk, s3, s4, true);
    for (int q = 0; q < 27; ++q) {
        R a = 0;
        for (int k = 0; k < 27; ++k) a += R(B.Minv[q][k]) * (mF[k] - md[k]);
        out[q] = f[q] + a;
    }
}

// ----------------------------------------------------------------------------- Zou-He
// 2D velocity inlet / pressure outlet, d2q9_boundaries.ispc:43-121 (node-local).
template <class R>
inline void zou_he_in_d2q9(R* f, R uxin, R uyin) {
    const R rho = (f[0] + f[2] + f[4] + R(2) * (f[3] + f[6] + f[7])) / (R(1) - uxin);
    f[1] = f[3] + (R(2) / R(3)) * rho * uxin;
    f[5] = f[7] - R(0.5) * (f[2] - f[4]) + (R(1) / R(6)) * rho * uxin + R(0.5) * rho * uyin;
    f[8] = f[6] + R(0.5) * (f[2] - f[4]) + (R(1) / R(6)) * rho * uxin - R(0.5) * rho * uyin;
}
template <class R>
inline void zou_he_out_d2q9(R* f, R rho) {
    const R ux = R(-1) + (f[0] + f[2] + f[4] + R(2) * (f[1] + f[5] + f[8])) / rho;
    const R uy = 0;
    f[3] = f[1] - (R(2) / R(3)) * rho * ux;
    f[6] = f[8] - R(0.5) * (f[2] - f[4]) - (R(1) / R(6)) * rho * ux + R(0.5) * rho * uy;
    f[7] = f[5] + R(0.5) * (f[2] - f[4]) - (R(1) / R(6)) * rho * ux - R(0.5) * rho * uy;
}
// D3Q19 (Hecht & Harting 2010). Unknowns at the west face: c_x=+1 (1,7,9,11,13).
template <class R>
inline void zou_he_in_d3q19(R* f, const R u[3]) {
    const R s0 = f[0] + f[3] + f[4] + f[5] + f[6] + f[15] + f[16] + f[17] + f[18];
    const R sm = f[2] + f[8] + f[10] + f[12] + f[14];
    const R rho = (s0 + R(2) * sm) / (R(1) - u[0]);
    const R Ny = R(0.5) * (f[3] + f[15] + f[17] - f[4] - f[16] - f[18]) - rho * u[1] / R(3);
    const R Nz = R(0.5) * (f[5] + f[15] + f[16] - f[6] - f[17] - f[18]) - rho * u[2] / R(3);
    f[1] = f[2] + rho * u[0] / R(3);
    f[7] = f[10] + rho * (u[0] + u[1]) / R(6) - Ny;
    f[9] = f[8] + rho * (u[0] - u[1]) / R(6) + Ny;
    f[11] = f[14] + rho * (u[0] + u[2]) / R(6) - Nz;
    f[13] = f[12] + rho * (u[0] - u[2]) / R(6) + Nz;
}
// East face pressure outlet, u_y = u_z = 0. Unknowns c_x=-1 (2,8,10,12,14).
template <class R>
inline void zou_he_out_d3q19(R* f, R rho) {
    const R s0 = f[0] + f[3] + f[4] + f[5] + f[6] + f[15] + f[16] + f[17] + f[18];
    const R sp = f[1] + f[7] + f[9] + f[11] + f[13];
    const R ux = R(-1) + (s0 + R(2) * sp) / rho;
    const R Ny = R(0.5) * (f[3] + f[15] + f[17] - f[4] - f[16] - f[18]);
    const R Nz = R(0.5) * (f[5] + f[15] + f[16] - f[6] - f[17] - f[18]);
    f[2] = f[1] - rho * ux / R(3);
    f[10] = f[7] - rho * ux / R(6) + Ny;
    f[8] = f[9] - rho * ux / R(6) - Ny;
    f[14] = f[11] - rho * ux / R(6) + Nz;
    f[12] = f[13] - rho * ux / R(6) - Nz;
}

// D2Q5 temperature lattice: rest, +x, +y, -x, -y (the first five D2Q9 directions), c_s^2 = 1/3.
struct D2Q5T {
    static constexpr int Q = 5;
    static constexpr int cx[5] = {0, 1, 0, -1, 0};
    static constexpr int cy[5] = {0, 0, 1, 0, -1};
    static constexpr int opp[5] = {0, 3, 4, 1, 2};
    static constexpr double wn[5] = {2, 1, 1, 1, 1};  // w = wn / 6
    static constexpr double wd = 6.0;
};

// ----------------------------------------------------------------------------- grid oracle
struct Params {
    int collision;      // 0 BGK, 1 TRT, 2 MRT
    int les;            // 1: Smagorinsky tau applied per node
    int mrt_exact;      // D3Q19 MRT: 0 reference-rounded inverse, 1 exact
    int periodic_y;     // 3D only: wrap y (else half-way bounce-back walls)
    int periodic_z;     // 3D only: wrap z
    int inflow;         // Zou-He velocity inlet on the west face
    int outflow;        // Zou-He pressure outlet on the east face
    int mem;            // accumulate momentum-exchange forces every step
    double tau, tau_bulk, lambda_trt, cs_smag;
    double g[3];
    double u_in[3];
    double rho_out;
    double u_wall[3];
    double center[3];
    double r_max;
    double s3, s4;      // D3Q27 MRT higher-order rates
    int thermal;        // D2Q9 only: D2Q5 temperature with local Boussinesq force
    double tau_t, t_ref, beta_g, t_south, t_north;
};

template <class L, class R>
struct Grid {
    int nx, ny, nz;
    std::size_t n;
    std::vector<R> fsrc, fdst;
    std::vector<R> rho, ux, uy, uz, speed;
    std::vector<uint8_t> type;
    std::vector<int> link_idx, link_q;
    std::vector<R> link_delta, link_uw;
    std::vector<R> tsrc, tdst;  // D2Q5 temperature populations [5][n] (thermal only)
    Params p{};

    Grid(int nx_, int ny_, int nz_) : nx(nx_), ny(ny_), nz(nz_), n(std::size_t(nx_) * ny_ * nz_) {
        tsrc.assign(5 * n, R(0));
        tdst.assign(5 * n, R(0));
        fsrc.assign(L::Q * n, R(0));
        fdst.assign(L::Q * n, R(0));
        rho.assign(n, R(1));
        ux.assign(n, R(0));
        uy.assign(n, R(0));
        uz.assign(n, R(0));
        speed.assign(n, R(0));
        type.assign(n, FLUID);
    }
    std::size_t at(int x, int y, int z) const { return (std::size_t(z) * ny + y) * nx + x; }

    // pull source coordinates; false if the source is off the domain in a wall direction
    bool source(int x, int y, int z, int q, std::size_t& s) const {
        int sx = x - L::cx[q], sy = y - L::cy[q], sz = z - L::cz[q];
        sx = (sx + nx) % nx;  // x is always periodic (d2q9_streaming.ispc:65, d3q19_streaming.ispc:78)
        if (L::D == 3 && p.periodic_y) sy = (sy + ny) % ny;
        if (L::D == 3 && p.periodic_z) sz = (sz + nz) % nz;
        if (sy < 0 || sy >= ny || sz < 0 || sz >= nz) return false;
        s = at(sx, sy, sz);
        return true;
    }

    R node_tau(const R* f, R r, const R u[3]) const {
        if (!p.les) return R(p.tau);
        return smagorinsky_tau<L, R>(f, r, u, R(p.tau), R(p.cs_smag));
    }

    void collide_node(const R* f, R* out, R& r, R u[3], R extra_gy = R(0)) const {
        R g[3] = {R(p.g[0]), R(p.g[1]) + extra_gy, R(p.g[2])};
        moments<L, R>(f, g, r, u);
        const R tau = node_tau(f, r, u);
        if (p.collision == 0) {
            collide_bgk<L, R>(f, out, r, u, g, tau);
        } else if (p.collision == 1) {
            // tau_a from the magic parameter, lattice_grid_2d.cpp:219-222
            const R diff = std::max(R(1e-4), tau - R(0.5));
            const R tau_a = R(0.5) + R(p.lambda_trt) / diff;
            collide_trt<L, R>(f, out, r, u, g, tau, tau_a);
        } else {
            if constexpr (L::Q == 9) collide_mrt_d2q9<R>(f, out, r, u, g, tau, R(p.tau_bulk));
            else if constexpr (L::Q == 19) collide_mrt_d3q19<R>(f, out, r, u, g, tau, R(p.tau_bulk), p.mrt_exact != 0);
            else collide_mrt_d3q27<R>(f, out, r, u, g, tau, R(p.tau_bulk), R(p.s3), R(p.s4));
        }
    }

    void step() {
        const int Q = L::Q;
        // 1-2. collide f_src -> f_dst; solid nodes copy through (d2q9_collision_bgk.ispc:22-28)
        parallel_ranges(n, [&](std::size_t i0, std::size_t i1) {
        for (std::size_t i = i0; i < i1; ++i) {
            R f[L::Q], o[L::Q], r, u[3];
            for (int q = 0; q < Q; ++q) f[q] = fsrc[q * n + i];
            if (type[i] == SOLID) {
                for (int q = 0; q < Q; ++q) fdst[q * n + i] = f[q];
                continue;
            }
            if (thermal_on()) {
                // local Boussinesq force from this node's temperature, then the temperature collide
                R t5[5], T = R(0);
                for (int q = 0; q < 5; ++q) {
                    t5[q] = tsrc[q * n + i];
                    T += t5[q];
                }
                collide_node(f, o, r, u, R(p.beta_g) * (T - R(p.t_ref)));
                const R om = R(1) / R(p.tau_t);
                for (int q = 0; q < 5; ++q) {
                    const R cu = R(D2Q5T::cx[q]) * u[0] + R(D2Q5T::cy[q]) * u[1];
                    const R geq = wq<D2Q5T, R>(q) * T * (R(1) + R(3) * cu);
                    tdst[q * n + i] = t5[q] - om * (t5[q] - geq);
                }
            } else {
                collide_node(f, o, r, u);
            }
            for (int q = 0; q < Q; ++q) fdst[q * n + i] = o[q];
        }
        });
        if (thermal_on())
            for (std::size_t i = 0; i < n; ++i)
                if (type[i] == SOLID)
                    for (int q = 0; q < 5; ++q) tdst[q * n + i] = tsrc[q * n + i];
        // 3. pull stream f_dst -> f_src with half-way bounce-back (d2q9_streaming.ispc:33-95,
        //    d3q19_streaming.ispc:39-104)
        R mom[L::Q];
        for (int q = 0; q < Q; ++q) {
            const R cuw = R(L::cx[q]) * R(p.u_wall[0]) + R(L::cy[q]) * R(p.u_wall[1]) + R(L::cz[q]) * R(p.u_wall[2]);
            mom[q] = R(2) * wq<L, R>(q) * R(3) * cuw;
        }
        parallel_ranges(std::size_t(nz) * ny, [&](std::size_t r0, std::size_t r1) {
        for (std::size_t row = r0; row < r1; ++row) {
            const int z = static_cast<int>(row / ny), y = static_cast<int>(row % ny);
                for (int x = 0; x < nx; ++x) {
                    const std::size_t i = at(x, y, z);
                    for (int q = 0; q < Q; ++q) {
                        if (type[i] == SOLID) {
                            fsrc[q * n + i] = fdst[q * n + i];
                            continue;
                        }
                        std::size_t s;
                        const int o = L::opp[q];
                        if (!source(x, y, z, q, s)) fsrc[q * n + i] = fdst[o * n + i];
                        else if (type[s] == SOLID) fsrc[q * n + i] = fdst[o * n + i];
                        else if (type[s] == MOVING_WALL) fsrc[q * n + i] = fdst[o * n + i] + mom[q];
                        else fsrc[q * n + i] = fdst[q * n + s];
                    }
                }
        }
        });
        // 3b. temperature: pull, anti-bounce-back through the y walls, bounce-back at solids
        if (thermal_on()) {
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    const std::size_t i = at(x, y, 0);
                    for (int q = 0; q < 5; ++q) {
                        if (type[i] == SOLID) {
                            tsrc[q * n + i] = tdst[q * n + i];
                            continue;
                        }
                        const int o = D2Q5T::opp[q];
                        const int sx = (x - D2Q5T::cx[q] + nx) % nx, sy = y - D2Q5T::cy[q];
                        if (sy < 0 || sy >= ny) {
                            const R tw = R(sy < 0 ? p.t_south : p.t_north);
                            tsrc[q * n + i] = -tdst[o * n + i] + R(2) * wq<D2Q5T, R>(q) * tw;
                        } else if (type[at(sx, sy, 0)] == SOLID) {
                            tsrc[q * n + i] = tdst[o * n + i];
                        } else {
                            tsrc[q * n + i] = tdst[q * n + at(sx, sy, 0)];
                        }
                    }
                }
        }
        // 4. BFL curved links, reading post-collision values (d3q19_curved.ispc:7-71)
        if constexpr (L::Q == 19) {
            for (std::size_t k = 0; k < link_idx.size(); ++k) {
                const int idx = link_idx[k], q = link_q[k], o = L::opp[q];
                const R delta = link_delta[k];
                const R cuw = R(L::cx[q]) * link_uw[3 * k] + R(L::cy[q]) * link_uw[3 * k + 1] +
                              R(L::cz[q]) * link_uw[3 * k + 2];
                const R fi = fdst[q * n + idx], fo = fdst[o * n + idx];
                R val;
                if (delta < R(0.5)) {
                    const int zf = idx / (nx * ny), rem = idx - zf * nx * ny, yf = rem / nx, xf = rem - yf * nx;
                    const int xff = (xf - L::cx[q] + nx) % nx, yff = yf - L::cy[q], zff = zf - L::cz[q];
                    R fff = fi;
                    if (yff >= 0 && yff < ny && zff >= 0 && zff < nz) fff = fdst[q * n + at(xff, yff, zff)];
                    const R m = R(2) * wq<L, R>(q) * R(3) * cuw;
                    val = R(2) * delta * fi + (R(1) - R(2) * delta) * fff - m;
                } else {
                    const R i2d = R(1) / (R(2) * delta);
                    const R m = (R(1) / delta) * wq<L, R>(q) * R(3) * cuw;
                    val = i2d * fi + (R(1) - i2d) * fo - m;
                }
                fsrc[o * n + idx] = val;
            }
        }
        // 5. Zou-He (2D: column x=0 / x=nx-1, rows 1..ny-2, any cell type, d2q9_boundaries.ispc:56,98;
        //    3D: Inflow/Outflow-typed nodes of the west/east faces)
        if (p.inflow || p.outflow) {
            for (int z = 0; z < nz; ++z)
                for (int y = 0; y < ny; ++y)
                    for (int side = 0; side < 2; ++side) {
                        if ((side == 0 && !p.inflow) || (side == 1 && !p.outflow)) continue;
                        const int x = side == 0 ? 0 : nx - 1;
                        const std::size_t i = at(x, y, z);
                        if constexpr (L::D == 2) {
                            if (y < 1 || y > ny - 2) continue;
                        } else {
                            if (type[i] != (side == 0 ? INFLOW : OUTFLOW)) continue;
                        }
                        R f[L::Q];
                        for (int q = 0; q < Q; ++q) f[q] = fsrc[q * n + i];
                        if constexpr (L::Q == 9) {
                            if (side == 0) zou_he_in_d2q9<R>(f, R(p.u_in[0]), R(p.u_in[1]));
                            else zou_he_out_d2q9<R>(f, R(p.rho_out));
                        } else if constexpr (L::Q == 19) {
                            const R u[3] = {R(p.u_in[0]), R(p.u_in[1]), R(p.u_in[2])};
                            if (side == 0) zou_he_in_d3q19<R>(f, u);
                            else zou_he_out_d3q19<R>(f, R(p.rho_out));
                        }
                        for (int q = 0; q < Q; ++q) fsrc[q * n + i] = f[q];
                    }
        }
        // 6. forced moments + speed over all nodes (lattice_grid_2d.cpp:257-262)
        refresh_macro();
    }

    bool thermal_on() const { return L::Q == 9 && p.thermal != 0; }

    R temperature(std::size_t i) const {
        R T = R(0);
        for (int q = 0; q < 5; ++q) T += tsrc[q * n + i];
        return T;
    }

    void refresh_macro() {
        parallel_ranges(n, [&](std::size_t i0, std::size_t i1) {
        for (std::size_t i = i0; i < i1; ++i) {
            R g[3] = {R(p.g[0]), R(p.g[1]), R(p.g[2])};
            if (thermal_on()) g[1] += R(p.beta_g) * (temperature(i) - R(p.t_ref));
            R f[L::Q], r, u[3];
            for (int q = 0; q < L::Q; ++q) f[q] = fsrc[q * n + i];
            moments<L, R>(f, g, r, u);
            rho[i] = r;
            ux[i] = u[0];
            uy[i] = u[1];
            uz[i] = u[2];
            speed[i] = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        }
        });
    }

    // Momentum exchange on f_src (forces_momentum_exchange.ispc:6-138): fluid nodes only,
    // links to Solid or MovingWall neighbours at x + c_q (x periodic, y/z in range), within r_max.
    void forces(double out[3]) const {
        double F[3] = {0, 0, 0}, tz = 0;
        const R rmax = R(p.r_max), rmax2 = rmax * rmax;
        for (int q = 1; q < L::Q; ++q)
            for (int z = 0; z < nz; ++z)
                for (int y = 0; y < ny; ++y)
                    for (int x = 0; x < nx; ++x) {
                        const std::size_t i = at(x, y, z);
                        if (type[i] != FLUID) continue;
                        const int xn = (x + L::cx[q] + nx) % nx, yn = y + L::cy[q], zn = z + L::cz[q];
                        if (yn < 0 || yn >= ny || zn < 0 || zn >= nz) continue;
                        const uint8_t t = type[at(xn, yn, zn)];
                        if (t != SOLID && t != MOVING_WALL) continue;
                        const R rx = (R(x) + R(0.5) * R(L::cx[q])) - R(p.center[0]);
                        const R ry = (R(y) + R(0.5) * R(L::cy[q])) - R(p.center[1]);
                        const R rz = (R(z) + R(0.5) * R(L::cz[q])) - R(p.center[2]);
                        const R r2 = L::D == 2 ? rx * rx + ry * ry : rx * rx + ry * ry + rz * rz;
                        if (!(rmax <= R(0) || r2 <= rmax2)) continue;
                        const double fv = fsrc[q * n + i];
                        const double dfx = 2.0 * fv * L::cx[q], dfy = 2.0 * fv * L::cy[q];
                        F[0] += dfx;
                        F[1] += dfy;
                        F[2] += 2.0 * fv * L::cz[q];
                        tz += double(rx) * dfy - double(ry) * dfx;
                    }
        out[0] = F[0];
        out[1] = F[1];
        out[2] = L::D == 2 ? tz : F[2];
    }
};

struct AnyGrid {
    int q, prec;
    void* g;
};

template <class Fn>
auto dispatch(AnyGrid* h, Fn&& fn) {
    if (h->q == 9) {
        if (h->prec == 32) return fn(static_cast<Grid<D2Q9T, float>*>(h->g));
        return fn(static_cast<Grid<D2Q9T, double>*>(h->g));
    }
    if (h->q == 19) {
        if (h->prec == 32) return fn(static_cast<Grid<D3Q19T, float>*>(h->g));
        return fn(static_cast<Grid<D3Q19T, double>*>(h->g));
    }
    if (h->prec == 32) return fn(static_cast<Grid<D3Q27T, float>*>(h->g));
    return fn(static_cast<Grid<D3Q27T, double>*>(h->g));
}

// ----------------------------------------------------------------------------- Strouhal
// Hann window, mean removal, zero pad to 2^k capped at 4096, radix-2 FFT, peak bin >= 1
// (strouhal_analyzer.cpp:39-84). All in double.
double strouhal_frequency(const double* s, int n, double dt) {
    if (n < 16 || dt <= 0) return 0;
    double mean = 0;
    for (int i = 0; i < n; ++i) mean += s[i];
    mean /= n;
    std::size_t N = 1;
    while (N < std::size_t(n)) N <<= 1;
    if (N > 4096) N = 4096;
    const std::size_t len = std::min<std::size_t>(N, n);
    std::vector<std::complex<double>> a(N, 0.0);
    const double two_pi = 6.283185307179586;
    for (std::size_t i = 0; i < len; ++i) {
        const double w = 0.5 * (1 - std::cos(two_pi * double(i) / double(len - 1)));
        a[i] = (s[i] - mean) * w;
    }
    for (std::size_t i = 1, j = 0; i < N; ++i) {
        std::size_t bit = N >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (std::size_t L2 = 2; L2 <= N; L2 <<= 1) {
        for (std::size_t i = 0; i < N; i += L2)
            for (std::size_t j = 0; j < L2 / 2; ++j) {
                const double ang = -two_pi * double(j) / double(L2);
                const std::complex<double> w(std::cos(ang), std::sin(ang));
                const std::complex<double> u = a[i + j], v = a[i + j + L2 / 2] * w;
                a[i + j] = u + v;
                a[i + j + L2 / 2] = u - v;
            }
    }
    std::size_t peak = 1;
    double best = 0;
    for (std::size_t i = 1; i < N / 2; ++i) {
        const double pw = std::norm(a[i]);
        if (pw > best) {
            best = pw;
            peak = i;
        }
    }
    return double(peak) / (double(N) * dt);
}

}  // namespace

// ============================================================================= C interface
extern "C" {

void* og_create(int q, int nx, int ny, int nz, int prec) {
    auto* h = new AnyGrid{q, prec, nullptr};
    if (q == 9) {
        if (prec == 32) h->g = new Grid<D2Q9T, float>(nx, ny, 1);
        else h->g = new Grid<D2Q9T, double>(nx, ny, 1);
    } else if (q == 19) {
        if (prec == 32) h->g = new Grid<D3Q19T, float>(nx, ny, nz);
        else h->g = new Grid<D3Q19T, double>(nx, ny, nz);
    } else {
        if (prec == 32) h->g = new Grid<D3Q27T, float>(nx, ny, nz);
        else h->g = new Grid<D3Q27T, double>(nx, ny, nz);
    }
    return h;
}

void og_destroy(void* hp) {
    auto* h = static_cast<AnyGrid*>(hp);
    dispatch(h, [](auto* g) { delete g; return 0; });
    delete h;
}

void og_set_params(void* hp, const Params* p) {
    dispatch(static_cast<AnyGrid*>(hp), [&](auto* g) { g->p = *p; return 0; });
}

void og_set_cell_types(void* hp, const uint8_t* t) {
    dispatch(static_cast<AnyGrid*>(hp), [&](auto* g) { std::memcpy(g->type.data(), t, g->n); return 0; });
}

// Initial populations f_src (Q x N, double) and the macroscopic arrays the
// reference's initialize_custom leaves behind (rho/u as given).
void og_set_state(void* hp, const double* f, const double* rho, const double* ux, const double* uy,
                  const double* uz) {
    dispatch(static_cast<AnyGrid*>(hp), [&](auto* g) {
        using R = typename std::remove_reference_t<decltype(g->fsrc)>::value_type;
        for (std::size_t k = 0; k < g->fsrc.size(); ++k) g->fsrc[k] = g->fdst[k] = R(f[k]);
        for (std::size_t i = 0; i < g->n; ++i) {
            g->rho[i] = R(rho[i]);
            g->ux[i] = R(ux[i]);
            g->uy[i] = R(uy[i]);
            g->uz[i] = uz ? R(uz[i]) : R(0);
            g->speed[i] = std::sqrt(g->ux[i] * g->ux[i] + g->uy[i] * g->uy[i] + g->uz[i] * g->uz[i]);
        }
        return 0;
    });
}

void og_set_links(void* hp, int nl, const int* idx, const int* q, const double* delta, const double* uw) {
    dispatch(static_cast<AnyGrid*>(hp), [&](auto* g) {
        using R = typename std::remove_reference_t<decltype(g->fsrc)>::value_type;
        g->link_idx.assign(idx, idx + nl);
        g->link_q.assign(q, q + nl);
        g->link_delta.resize(nl);
        g->link_uw.assign(3 * std::size_t(nl), R(0));
        for (int k = 0; k < nl; ++k) {
            g->link_delta[k] = R(delta[k]);
            if (uw)
                for (int a = 0; a < 3; ++a) g->link_uw[3 * k + a] = R(uw[3 * k + a]);
        }
        return 0;
    });
}

// Advance nsteps; if hist is non-null and p.mem is set, write forces [nsteps][3] after each step.
// Temperature populations [5][n] (pre-collision, the state of the next step).
void og_set_thermal_state(void* hp, const double* t5) {
    dispatch(static_cast<AnyGrid*>(hp), [&](auto* g) {
        using R = typename std::remove_reference_t<decltype(g->tsrc)>::value_type;
        for (std::size_t k = 0; k < 5 * g->n; ++k) g->tsrc[k] = g->tdst[k] = R(t5[k]);
        g->refresh_macro();
        return 0;
    });
}

void og_get_temperature(void* hp, double* T) {
    dispatch(static_cast<AnyGrid*>(hp), [&](auto* g) {
        for (std::size_t i = 0; i < g->n; ++i) T[i] = g->temperature(i);
        return 0;
    });
}

void og_step(void* hp, int nsteps, double* hist) {
    dispatch(static_cast<AnyGrid*>(hp), [&](auto* g) {
        for (int s = 0; s < nsteps; ++s) {
            g->step();
            if (hist && g->p.mem) g->forces(hist + 3 * s);
        }
        return 0;
    });
}

void og_get_f(void* hp, double* out) {
    dispatch(static_cast<AnyGrid*>(hp), [&](auto* g) {
        for (std::size_t k = 0; k < g->fsrc.size(); ++k) out[k] = double(g->fsrc[k]);
        return 0;
    });
}

void og_get_macro(void* hp, double* rho, double* ux, double* uy, double* uz, double* speed) {
    dispatch(static_cast<AnyGrid*>(hp), [&](auto* g) {
        for (std::size_t i = 0; i < g->n; ++i) {
            rho[i] = g->rho[i];
            ux[i] = g->ux[i];
            uy[i] = g->uy[i];
            if (uz) uz[i] = g->uz[i];
            speed[i] = g->speed[i];
        }
        return 0;
    });
}

void og_forces(void* hp, double* out3) {
    dispatch(static_cast<AnyGrid*>(hp), [&](auto* g) { g->forces(out3); return 0; });
}

// Equilibrium populations for given fields (host initialisation, lattice_grid_2d.cpp:90-120).
void og_equilibrium(int q, int prec, long long n, const double* rho, const double* ux, const double* uy,
                    const double* uz, double* f) {
    auto run = [&](auto lat, auto real) {
        using L = decltype(lat);
        using R = decltype(real);
        for (long long i = 0; i < n; ++i)
            for (int k = 0; k < L::Q; ++k)
                f[k * n + i] = double(feq<L, R>(k, R(rho[i]), R(ux[i]), R(uy[i]), uz ? R(uz[i]) : R(0)));
    };
    if (q == 9) prec == 32 ? run(D2Q9T{}, 0.f) : run(D2Q9T{}, 0.0);
    else if (q == 19) prec == 32 ? run(D3Q19T{}, 0.f) : run(D3Q19T{}, 0.0);
    else prec == 32 ? run(D3Q27T{}, 0.f) : run(D3Q27T{}, 0.0);
}

// Single-node collision (any lattice / model) for per-call parity tests:
// f [n][Q] node-major in, out [n][Q], moments rho/u [n] written.
void og_collide_nodes(void* hp, long long n, const double* f, const uint8_t* type, double* out, double* rho,
                      double* ux, double* uy, double* uz) {
    dispatch(static_cast<AnyGrid*>(hp), [&](auto* g) {
        using R = typename std::remove_reference_t<decltype(g->fsrc)>::value_type;
        const int QQ = static_cast<int>(g->fsrc.size() / g->n);
        for (long long i = 0; i < n; ++i) {
            R fi[27], o[27], r, u[3];
            for (int q = 0; q < QQ; ++q) fi[q] = R(f[i * QQ + q]);
            if (type && type[i] == SOLID) {
                for (int q = 0; q < QQ; ++q) out[i * QQ + q] = double(fi[q]);
                continue;
            }
            g->collide_node(fi, o, r, u);
            for (int q = 0; q < QQ; ++q) out[i * QQ + q] = double(o[q]);
            rho[i] = r;
            ux[i] = u[0];
            uy[i] = u[1];
            if (uz) uz[i] = u[2];
        }
        return 0;
    });
}

double og_d3q19_minv(int rounded, int q, int k) {
    return rounded ? d3q19_inverse().rounded[q][k] : d3q19_inverse().exact[q][k];
}

double og_strouhal_frequency(const double* s, int n, double dt) { return strouhal_frequency(s, n, dt); }

// Smagorinsky tau for one node (lattice q), used by per-call LES parity tests.
double og_smagorinsky_tau(int q, const double* f, double rho, double ux, double uy, double uz, double tau0,
                          double cs) {
    const double u[3] = {ux, uy, uz};
    if (q == 9) return smagorinsky_tau<D2Q9T, double>(f, rho, u, tau0, cs);
    if (q == 19) return smagorinsky_tau<D3Q19T, double>(f, rho, u, tau0, cs);
    return smagorinsky_tau<D3Q27T, double>(f, rho, u, tau0, cs);
}

}  // extern "C"
