// Telemetry files in the reference's formats: the aerodynamic CSV, the
// performance CSV and the summary JSON that wake::TelemetryExporter writes
// (src/export/csv_telemetry.cpp:21-125), byte for byte, so existing scripts
// (scripts/verify_strouhal.py) read them unchanged. Values are held as the
// reference holds them (float forces and coefficients, computed in float as
// compute_aerodynamic_coefficients does, include/wake/forces/momentum_exchange.hpp:20-37)
// and printed with the same stream formatting. The per-step force history of a
// grid (FP64, wake_grid_get_force_history) is turned into records by
// wake_telemetry_record_history.
#include <cmath>
#include <cstdint>
#include <fstream>
#include <iomanip>
#include <string>
#include <vector>

#include "wake_gpu.h"

struct wake_telemetry {
    struct Aero {
        uint64_t step;
        float time, fx, fy, fz, torque_z, cd, cl, cm;
    };
    struct Perf {
        uint64_t step;
        double step_time_ms, mlups;
        float max_speed, total_mass, kinetic_energy;
    };
    std::vector<Aero> aero;
    std::vector<Perf> perf;
};

namespace {

// compute_aerodynamic_coefficients in the reference's float arithmetic.
wake_telemetry::Aero coefficients(uint64_t step, float time, float fx, float fy, float fz, float tz, float rho_inf,
                                  float u_inf, float area, float chord) {
    wake_telemetry::Aero a{step, time, fx, fy, fz, tz, 0.f, 0.f, 0.f};
    const float dyn = 0.5f * rho_inf * u_inf * u_inf;
    if (dyn > 1e-8f && area > 1e-8f) {
        a.cd = fx / (dyn * area);
        a.cl = fy / (dyn * area);
        a.cm = tz / (dyn * area * chord);
    }
    return a;
}

}  // namespace

extern "C" {

wake_telemetry* wake_telemetry_create(void) { return new wake_telemetry(); }

void wake_telemetry_destroy(wake_telemetry* t) { delete t; }

void wake_telemetry_clear(wake_telemetry* t) {
    if (!t) return;
    t->aero.clear();
    t->perf.clear();
}

int wake_telemetry_record_aero(wake_telemetry* t, unsigned long long step, float time, float fx, float fy, float fz,
                               float torque_z, float rho_inf, float u_inf, float area, float chord) {
    if (!t) return WAKE_ERR_INVALID;
    t->aero.push_back(coefficients(step, time, fx, fy, fz, torque_z, rho_inf, u_inf, area, chord));
    return WAKE_OK;
}

int wake_telemetry_record_history(wake_telemetry* t, const double* hist, int n, long long first_step, int every,
                                  int is3d, float rho_inf, float u_inf, float area, float chord) {
    if (!t || (n > 0 && !hist) || every < 1 || first_step < 0) return WAKE_ERR_INVALID;
    for (int i = 0; i < n; ++i) {
        const long long step = first_step + i;
        if (step % every) continue;
        const float fx = static_cast<float>(hist[3 * i]), fy = static_cast<float>(hist[3 * i + 1]);
        const float c = static_cast<float>(hist[3 * i + 2]);
        t->aero.push_back(coefficients(static_cast<uint64_t>(step), static_cast<float>(step), fx, fy, is3d ? c : 0.f,
                                       is3d ? 0.f : c, rho_inf, u_inf, area, chord));
    }
    return WAKE_OK;
}

int wake_telemetry_record_performance(wake_telemetry* t, unsigned long long step, double step_time_ms, double mlups,
                                      float max_speed, float total_mass, float kinetic_energy) {
    if (!t) return WAKE_ERR_INVALID;
    t->perf.push_back({step, step_time_ms, mlups, max_speed, total_mass, kinetic_energy});
    return WAKE_OK;
}

int wake_telemetry_count(wake_telemetry* t, int which) {
    if (!t) return WAKE_ERR_INVALID;
    return static_cast<int>(which == 0 ? t->aero.size() : t->perf.size());
}

// Coefficients of record i: out[0..2] = cd, cl, cm.
int wake_telemetry_get_coefficients(wake_telemetry* t, int i, float* out) {
    if (!t || !out || i < 0 || i >= static_cast<int>(t->aero.size())) return WAKE_ERR_INVALID;
    out[0] = t->aero[i].cd;
    out[1] = t->aero[i].cl;
    out[2] = t->aero[i].cm;
    return WAKE_OK;
}

int wake_telemetry_write_aero_csv(wake_telemetry* t, const char* path) {
    if (!t || !path) return WAKE_ERR_INVALID;
    std::ofstream out(path);
    if (!out.is_open()) return WAKE_ERR_INVALID;
    out << "step,time,fx,fy,fz,cd,cl,cm\n";
    out << std::fixed << std::setprecision(6);
    for (const auto& s : t->aero)
        out << s.step << "," << s.time << "," << s.fx << "," << s.fy << "," << s.fz << "," << s.cd << "," << s.cl << ","
            << s.cm << "\n";
    return out.good() ? WAKE_OK : WAKE_ERR_INVALID;
}

int wake_telemetry_write_performance_csv(wake_telemetry* t, const char* path) {
    if (!t || !path) return WAKE_ERR_INVALID;
    std::ofstream out(path);
    if (!out.is_open()) return WAKE_ERR_INVALID;
    out << "step,step_time_ms,mlups,max_speed,total_mass,kinetic_energy\n";
    out << std::fixed << std::setprecision(6);
    for (const auto& p : t->perf)
        out << p.step << "," << p.step_time_ms << "," << p.mlups << "," << p.max_speed << "," << p.total_mass << ","
            << p.kinetic_energy << "\n";
    return out.good() ? WAKE_OK : WAKE_ERR_INVALID;
}

int wake_telemetry_write_summary_json(wake_telemetry* t, const char* path, const char* simulation_name,
                                      float strouhal_number, float shedding_frequency) {
    if (!t || !path || !simulation_name) return WAKE_ERR_INVALID;
    std::ofstream out(path);
    if (!out.is_open()) return WAKE_ERR_INVALID;
    // statistics in double over the float samples, as the reference aggregates them
    double mean_cd = 0.0, max_cd = -1e9, min_cd = 1e9, rms_cl = 0.0;
    if (!t->aero.empty()) {
        double sum_cd = 0.0, sum_cl_sq = 0.0;
        for (const auto& s : t->aero) {
            sum_cd += s.cd;
            sum_cl_sq += s.cl * s.cl;  // float product, as in the reference
            if (s.cd > max_cd) max_cd = s.cd;
            if (s.cd < min_cd) min_cd = s.cd;
        }
        mean_cd = sum_cd / t->aero.size();
        rms_cl = std::sqrt(sum_cl_sq / t->aero.size());
    } else {
        max_cd = 0.0;
        min_cd = 0.0;
    }
    double avg_mlups = 0.0;
    if (!t->perf.empty()) {
        double sum = 0.0;
        for (const auto& p : t->perf) sum += p.mlups;
        avg_mlups = sum / t->perf.size();
    }
    out << "{\n";
    out << "  \"simulation\": \"" << simulation_name << "\",\n";
    out << "  \"total_samples\": " << t->aero.size() << ",\n";
    out << "  \"performance\": {\n";
    out << "    \"average_mlups\": " << avg_mlups << "\n";
    out << "  },\n";
    out << "  \"aerodynamics\": {\n";
    out << "    \"mean_drag_coefficient\": " << mean_cd << ",\n";
    out << "    \"max_drag_coefficient\": " << max_cd << ",\n";
    out << "    \"min_drag_coefficient\": " << min_cd << ",\n";
    out << "    \"rms_lift_coefficient\": " << rms_cl << ",\n";
    out << "    \"shedding_frequency\": " << shedding_frequency << ",\n";
    out << "    \"strouhal_number\": " << strouhal_number << "\n";
    out << "  }\n";
    out << "}\n";
    return out.good() ? WAKE_OK : WAKE_ERR_INVALID;
}

}  // extern "C"
