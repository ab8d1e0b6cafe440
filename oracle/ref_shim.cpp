// extern "C" shim over the reference's own host classes (test infrastructure only).
//
// Compiled by oracle/build_ref.py together with the reference sources
// (src/grid/lattice_grid_{2d,3d}.cpp, src/forces/strouhal_analyzer.cpp,
// src/export/csv_telemetry.cpp, src/export/vtk_exporter.cpp) and the
// mechanically translated ISPC kernels. It lets the Python tests drive
// wake::LatticeGrid2D / wake::LatticeGrid3D exactly as the reference scenarios do
// (src/scenarios/karman_vortex.cpp:62-124, src/scenarios/sphere_3d_wake.cpp:64-105)
// and read back every buffer, including the private BFL link arrays, which
// pin this project's own link builder.
#include <cstdint>
#include <cstring>
#include <vector>

#define private public
#include "wake/grid/lattice_grid_2d.hpp"
#include "wake/grid/lattice_grid_3d.hpp"
#undef private
#include "wake/forces/strouhal_analyzer.hpp"
#include "wake/export/csv_telemetry.hpp"
#include "wake/export/vtk_exporter.hpp"

namespace ispc {
extern "C" {
void d2q9_compute_momentum_exchange_forces(const float f_post_collision[], const uint8_t cell_type[],
                                           int nx, int ny, float center_x, float center_y, float max_radius,
                                           float& fx_out, float& fy_out, float& torque_z_out);
void d3q19_compute_momentum_exchange_forces(const float f_post_collision[], const uint8_t cell_type[],
                                            int nx, int ny, int nz, float center_x, float center_y,
                                            float center_z, float max_radius, float& fx_out, float& fy_out,
                                            float& fz_out);
}
}

using wake::CellType;
using wake::CollisionType;
using wake::LatticeGrid2D;
using wake::LatticeGrid3D;

extern "C" {

// ---------------------------------------------------------------- 2D
void* ref2d_create(int nx, int ny, float tau) { return new LatticeGrid2D(nx, ny, tau); }
void ref2d_destroy(void* h) { delete static_cast<LatticeGrid2D*>(h); }

void ref2d_init_fields(void* h, const float* rho, const float* ux, const float* uy) {
    auto* g = static_cast<LatticeGrid2D*>(h);
    const int nx = g->nx();
    g->initialize_custom([&](int x, int y, float& r, float& u, float& v) {
        const std::size_t i = static_cast<std::size_t>(y) * nx + x;
        r = rho[i];
        u = ux[i];
        v = uy[i];
    });
}
void ref2d_set_cell_type(void* h, int x, int y, int t) {
    static_cast<LatticeGrid2D*>(h)->set_cell_type(x, y, static_cast<CellType>(t));
}
void ref2d_set_solid_circle(void* h, float cx, float cy, float r) {
    static_cast<LatticeGrid2D*>(h)->set_solid_circle(cx, cy, r);
}
void ref2d_set_inflow_west(void* h, float ux, float uy) { static_cast<LatticeGrid2D*>(h)->set_inflow_west(ux, uy); }
void ref2d_set_outflow_east(void* h, float rho) { static_cast<LatticeGrid2D*>(h)->set_outflow_east(rho); }
void ref2d_set_moving_wall_north(void* h, float uw) { static_cast<LatticeGrid2D*>(h)->set_moving_wall_north(uw); }

void ref2d_step(void* h, int collision, float gx, float gy, int use_les, float cs, int nsteps) {
    auto* g = static_cast<LatticeGrid2D*>(h);
    for (int s = 0; s < nsteps; ++s) g->step(static_cast<CollisionType>(collision), gx, gy, use_les != 0, cs);
}

// Steps like KarmanVortexScenario::step: grid step, then the MEM kernel on f_src.
void ref2d_step_forces(void* h, int collision, float gx, float gy, int use_les, float cs, int nsteps,
                       float cx, float cy, float r_max, float* hist /* [nsteps][3] */) {
    auto* g = static_cast<LatticeGrid2D*>(h);
    for (int s = 0; s < nsteps; ++s) {
        g->step(static_cast<CollisionType>(collision), gx, gy, use_les != 0, cs);
        float fx = 0.f, fy = 0.f, tz = 0.f;
        ispc::d2q9_compute_momentum_exchange_forces(g->f_src_data(), g->cell_type_data(), g->nx(), g->ny(), cx, cy,
                                                    r_max, fx, fy, tz);
        hist[3 * s + 0] = fx;
        hist[3 * s + 1] = fy;
        hist[3 * s + 2] = tz;
    }
}

void ref2d_get_f(void* h, float* out) {
    auto* g = static_cast<LatticeGrid2D*>(h);
    std::memcpy(out, g->f_src_data(), sizeof(float) * 9 * g->total_nodes());
}
void ref2d_get_macro(void* h, float* rho, float* ux, float* uy, float* speed) {
    auto* g = static_cast<LatticeGrid2D*>(h);
    const std::size_t n = g->total_nodes();
    std::memcpy(rho, g->rho_data(), sizeof(float) * n);
    std::memcpy(ux, g->ux_data(), sizeof(float) * n);
    std::memcpy(uy, g->uy_data(), sizeof(float) * n);
    std::memcpy(speed, g->speed_data(), sizeof(float) * n);
}
void ref2d_get_cell_types(void* h, uint8_t* out) {
    auto* g = static_cast<LatticeGrid2D*>(h);
    std::memcpy(out, g->cell_type_data(), g->total_nodes());
}
float ref2d_total_mass(void* h) { return static_cast<LatticeGrid2D*>(h)->compute_total_mass(); }
float ref2d_total_ke(void* h) { return static_cast<LatticeGrid2D*>(h)->compute_total_kinetic_energy(); }
float ref2d_max_speed(void* h) { return static_cast<LatticeGrid2D*>(h)->compute_max_speed(); }

// ---------------------------------------------------------------- 3D
void* ref3d_create(int nx, int ny, int nz, float tau) { return new LatticeGrid3D(nx, ny, nz, tau); }
void ref3d_destroy(void* h) { delete static_cast<LatticeGrid3D*>(h); }

void ref3d_init_fields(void* h, const float* rho, const float* ux, const float* uy, const float* uz) {
    auto* g = static_cast<LatticeGrid3D*>(h);
    const int nx = g->nx(), ny = g->ny();
    g->initialize_custom([&](int x, int y, int z, float& r, float& u, float& v, float& w) {
        const std::size_t i = (static_cast<std::size_t>(z) * ny + y) * nx + x;
        r = rho[i];
        u = ux[i];
        v = uy[i];
        w = uz[i];
    });
}
void ref3d_set_periodic(void* h, int p) { static_cast<LatticeGrid3D*>(h)->set_periodic(p != 0); }
void ref3d_set_cell_type(void* h, int x, int y, int z, int t) {
    static_cast<LatticeGrid3D*>(h)->set_cell_type(x, y, z, static_cast<CellType>(t));
}
void ref3d_set_solid_sphere(void* h, float cx, float cy, float cz, float r) {
    static_cast<LatticeGrid3D*>(h)->set_solid_sphere(cx, cy, cz, r);
}
void ref3d_build_curved_sphere_links(void* h, float cx, float cy, float cz, float r) {
    static_cast<LatticeGrid3D*>(h)->build_curved_sphere_links(cx, cy, cz, r);
}
void ref3d_set_moving_wall_top(void* h, float uwx, float uwz) {
    static_cast<LatticeGrid3D*>(h)->set_moving_wall_top(uwx, uwz);
}
void ref3d_step(void* h, int collision, float gx, float gy, float gz, int use_les, float cs, int nsteps) {
    auto* g = static_cast<LatticeGrid3D*>(h);
    for (int s = 0; s < nsteps; ++s) g->step(static_cast<CollisionType>(collision), gx, gy, gz, use_les != 0, cs);
}
// Steps like Sphere3DWakeScenario::step: grid step, then the MEM kernel on f_src.
void ref3d_step_forces(void* h, int collision, float gx, float gy, float gz, int use_les, float cs, int nsteps,
                       float cx, float cy, float cz, float r_max, float* hist /* [nsteps][3] */) {
    auto* g = static_cast<LatticeGrid3D*>(h);
    for (int s = 0; s < nsteps; ++s) {
        g->step(static_cast<CollisionType>(collision), gx, gy, gz, use_les != 0, cs);
        float fx = 0.f, fy = 0.f, fz = 0.f;
        ispc::d3q19_compute_momentum_exchange_forces(g->f_src_data(), g->cell_type_data(), g->nx(), g->ny(),
                                                     g->nz(), cx, cy, cz, r_max, fx, fy, fz);
        hist[3 * s + 0] = fx;
        hist[3 * s + 1] = fy;
        hist[3 * s + 2] = fz;
    }
}
void ref3d_get_f(void* h, float* out) {
    auto* g = static_cast<LatticeGrid3D*>(h);
    std::memcpy(out, g->f_src_data(), sizeof(float) * 19 * g->total_nodes());
}
void ref3d_get_macro(void* h, float* rho, float* ux, float* uy, float* uz, float* speed) {
    auto* g = static_cast<LatticeGrid3D*>(h);
    const std::size_t n = g->total_nodes();
    std::memcpy(rho, g->rho_data(), sizeof(float) * n);
    std::memcpy(ux, g->ux_data(), sizeof(float) * n);
    std::memcpy(uy, g->uy_data(), sizeof(float) * n);
    std::memcpy(uz, g->uz_data(), sizeof(float) * n);
    std::memcpy(speed, g->speed_data(), sizeof(float) * n);
}
void ref3d_get_cell_types(void* h, uint8_t* out) {
    auto* g = static_cast<LatticeGrid3D*>(h);
    std::memcpy(out, g->cell_type_data(), g->total_nodes());
}
int ref3d_num_links(void* h) { return static_cast<LatticeGrid3D*>(h)->num_bfl_links_; }
void ref3d_get_links(void* h, int* idx, int* q, float* delta) {
    auto* g = static_cast<LatticeGrid3D*>(h);
    for (int i = 0; i < g->num_bfl_links_; ++i) {
        idx[i] = g->bfl_fluid_indices_[i];
        q[i] = g->bfl_q_dirs_[i];
        delta[i] = g->bfl_delta_fractions_[i];
    }
}
int ref3d_is_periodic(void* h) { return static_cast<LatticeGrid3D*>(h)->is_periodic() ? 1 : 0; }
float ref3d_total_mass(void* h) { return static_cast<LatticeGrid3D*>(h)->compute_total_mass(); }
float ref3d_total_ke(void* h) { return static_cast<LatticeGrid3D*>(h)->compute_total_kinetic_energy(); }
float ref3d_max_speed(void* h) { return static_cast<LatticeGrid3D*>(h)->compute_max_speed(); }

// ---------------------------------------------------------------- Strouhal FFT
// ---------------------------------------------------------------- telemetry files
void* ref_telemetry_create() { return new wake::TelemetryExporter(); }
void ref_telemetry_destroy(void* t) { delete static_cast<wake::TelemetryExporter*>(t); }
void ref_telemetry_record_aero(void* t, unsigned long long step, float time, float fx, float fy, float fz,
                               float torque_z, float rho_inf, float u_inf, float area, float chord) {
    static_cast<wake::TelemetryExporter*>(t)->record_aero(
        {step, time, wake::compute_aerodynamic_coefficients(fx, fy, fz, torque_z, rho_inf, u_inf, area, chord)});
}
void ref_telemetry_record_performance(void* t, unsigned long long step, double ms, double mlups, float max_speed,
                                      float mass, float ke) {
    wake::PerformanceMetric p;
    p.step = step;
    p.step_time_ms = ms;
    p.mlups = mlups;
    p.max_speed = max_speed;
    p.total_mass = mass;
    p.kinetic_energy = ke;
    static_cast<wake::TelemetryExporter*>(t)->record_performance(p);
}
int ref_telemetry_write(void* t, int which, const char* path, const char* name, float st, float freq) {
    auto* e = static_cast<wake::TelemetryExporter*>(t);
    if (which == 0) return e->write_aero_csv(path) ? 0 : -1;
    if (which == 1) return e->write_performance_csv(path) ? 0 : -1;
    return e->write_summary_json(path, name, st, freq) ? 0 : -1;
}

// ---------------------------------------------------------------- VTK files
int ref_vtk_export_2d(void* h, const char* path, const float* vorticity) {
    return wake::VtkExporter::export_vti_2d(path, *static_cast<LatticeGrid2D*>(h), vorticity) ? 0 : -1;
}
// vorticity: n interleaved (x, y, z) triples, or NULL
int ref_vtk_export_3d(void* h, const char* path, const float* q_criterion, const float* vorticity) {
    auto* g = static_cast<LatticeGrid3D*>(h);
    std::vector<wake::Vec3> v;
    if (vorticity) {
        const std::size_t n = g->total_nodes();
        v.resize(n);
        for (std::size_t i = 0; i < n; ++i) v[i] = wake::Vec3(vorticity[3 * i], vorticity[3 * i + 1], vorticity[3 * i + 2]);
    }
    return wake::VtkExporter::export_vti_3d(path, *g, q_criterion, vorticity ? v.data() : nullptr) ? 0 : -1;
}
int ref_vtk_pvd(const char* path, const char* prefix, int start, int end, int interval, float dt) {
    return wake::VtkExporter::write_pvd_manifest(path, prefix, start, end, interval, dt) ? 0 : -1;
}

float ref_strouhal_frequency(const float* signal, int n, float dt) {
    wake::StrouhalAnalyzer a;
    std::vector<float> s(signal, signal + n);
    return a.analyze_frequency(s, dt);
}

}  // extern "C"
