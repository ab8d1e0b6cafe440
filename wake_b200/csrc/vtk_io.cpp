// VTK XML ImageData (.vti) and ParaView collection (.pvd) writers with the
// bytes of wake::VtkExporter (src/export/vtk_exporter.cpp:8-223), for
// post-processing pipelines written against the reference's files.
//
// The reference streams every value with std::ostream's default float format,
// which is printf's "%.6g" of the value widened to double; each row of nx
// values ends with "\n". Here the rows of one array are formatted on several
// host threads into separate buffers and written in row order, so the bytes do
// not depend on the thread count. Host code only.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <string>
#include <thread>
#include <vector>

#include "wake_gpu.h"

namespace wk {
int set_error(int code, const std::string& msg);
}

namespace {

void put_float(std::string& s, float v) {
    char b[48];
    const int n = std::snprintf(b, sizeof b, "%.*g", 6, static_cast<double>(v));
    s.append(b, static_cast<std::size_t>(n));
}

void put_int(std::string& s, long long v) {
    char b[32];
    const int n = std::snprintf(b, sizeof b, "%lld", v);
    s.append(b, static_cast<std::size_t>(n));
}

// Formats rows [0, nrows) of nx nodes each with `node(s, i)` appending node i's
// text; each row ends with "\n". Returns the concatenation in row order.
template <class NodeFn>
std::vector<std::string> format_rows(long long nrows, long long nx, int threads, NodeFn node) {
    const int T = static_cast<int>(std::max(1LL, std::min<long long>(threads, nrows)));
    std::vector<std::string> part(T);
    auto work = [&](int t) {
        const long long r0 = nrows * t / T, r1 = nrows * (t + 1) / T;
        std::string& s = part[t];
        s.reserve(static_cast<std::size_t>((r1 - r0) * nx * 14));
        for (long long r = r0; r < r1; ++r) {
            for (long long x = 0; x < nx; ++x) node(s, r * nx + x);
            s.push_back('\n');
        }
    };
    if (T == 1) {
        work(0);
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < T; ++t) pool.emplace_back(work, t);
        for (auto& th : pool) th.join();
    }
    return part;
}

int thread_count(int threads) {
    if (threads > 0) return threads;
    const unsigned h = std::thread::hardware_concurrency();
    return h ? static_cast<int>(h) : 1;
}

class Writer {
   public:
    explicit Writer(const char* path) : f_(path ? std::fopen(path, "wb") : nullptr) {}
    ~Writer() {
        if (f_) std::fclose(f_);
    }
    bool ok() const { return f_ != nullptr && good_; }
    void put(const std::string& s) {
        if (f_ && std::fwrite(s.data(), 1, s.size(), f_) != s.size()) good_ = false;
    }
    void put(const std::vector<std::string>& parts) {
        for (const auto& p : parts) put(p);
    }
    bool close() {
        if (!f_) return false;
        const bool r = std::fclose(f_) == 0 && good_;
        f_ = nullptr;
        return r;
    }

   private:
    std::FILE* f_;
    bool good_ = true;
};

std::string header(int nx, int ny, int nz) {
    std::string s = "<?xml version=\"1.0\"?>\n";
    s += "<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n";
    std::string ext = "0 ";
    put_int(ext, nx - 1);
    ext += " 0 ";
    put_int(ext, ny - 1);
    ext += " 0 ";
    put_int(ext, nz - 1);
    s += "  <ImageData WholeExtent=\"" + ext + "\" Origin=\"0 0 0\" Spacing=\"1 1 1\">\n";
    s += "    <Piece Extent=\"" + ext + "\">\n";
    s += "      <PointData Vectors=\"Velocity\" Scalars=\"Speed\">\n";
    return s;
}

std::string array_open(const char* type, const char* name, int comps) {
    std::string s = "        <DataArray type=\"";
    s += type;
    s += "\" Name=\"";
    s += name;
    s += "\" NumberOfComponents=\"";
    put_int(s, comps);
    s += "\" format=\"ascii\">\n";
    return s;
}

const char* kArrayClose = "        </DataArray>\n";
const char* kFooter = "      </PointData>\n    </Piece>\n  </ImageData>\n</VTKFile>\n";

void scalar_array(Writer& w, const char* name, const float* v, long long rows, long long nx, int T) {
    w.put(array_open("Float32", name, 1));
    w.put(format_rows(rows, nx, T, [v](std::string& s, long long i) {
        put_float(s, v[i]);
        s.push_back(' ');
    }));
    w.put(std::string(kArrayClose));
}

void cell_type_array(Writer& w, const uint8_t* t, long long rows, long long nx, int T) {
    w.put(array_open("UInt8", "CellType", 1));
    w.put(format_rows(rows, nx, T, [t](std::string& s, long long i) {
        put_int(s, static_cast<int>(t[i]));
        s.push_back(' ');
    }));
    w.put(std::string(kArrayClose));
}

}  // namespace

extern "C" {

// VtkExporter::export_vti_2d (src/export/vtk_exporter.cpp:8-89)
int wake_vtk_write_vti_2d(const char* path, int nx, int ny, const float* ux, const float* uy, const float* speed,
                          const float* rho, const float* vorticity, const uint8_t* cell_type, int threads) {
    if (nx < 1 || ny < 1 || !ux || !uy || !speed || !rho || !cell_type)
        return wk::set_error(WAKE_ERR_INVALID, "wake_vtk_write_vti_2d: bad size or null field");
    Writer w(path);
    if (!w.ok()) return wk::set_error(WAKE_ERR_INVALID, std::string("cannot open ") + (path ? path : "(null)"));
    const int T = thread_count(threads);
    w.put(header(nx, ny, 1));
    w.put(array_open("Float32", "Velocity", 3));
    w.put(format_rows(ny, nx, T, [ux, uy](std::string& s, long long i) {
        put_float(s, ux[i]);
        s.push_back(' ');
        put_float(s, uy[i]);
        s += " 0 ";
    }));
    w.put(std::string(kArrayClose));
    scalar_array(w, "Speed", speed, ny, nx, T);
    scalar_array(w, "Density", rho, ny, nx, T);
    if (vorticity) scalar_array(w, "Vorticity", vorticity, ny, nx, T);
    cell_type_array(w, cell_type, ny, nx, T);
    w.put(std::string(kFooter));
    if (!w.close()) return wk::set_error(WAKE_ERR_INVALID, std::string("write failed: ") + path);
    return WAKE_OK;
}

// VtkExporter::export_vti_3d (src/export/vtk_exporter.cpp:91-196)
int wake_vtk_write_vti_3d(const char* path, int nx, int ny, int nz, const float* ux, const float* uy,
                          const float* uz, const float* speed, const float* rho, const float* q_criterion,
                          const float* vorticity_x, const float* vorticity_y, const float* vorticity_z,
                          const uint8_t* cell_type, int threads) {
    if (nx < 1 || ny < 1 || nz < 1 || !ux || !uy || !uz || !speed || !rho || !cell_type)
        return wk::set_error(WAKE_ERR_INVALID, "wake_vtk_write_vti_3d: bad size or null field");
    const bool vort = vorticity_x && vorticity_y && vorticity_z;
    if (!vort && (vorticity_x || vorticity_y || vorticity_z))
        return wk::set_error(WAKE_ERR_INVALID, "wake_vtk_write_vti_3d: give all three vorticity components or none");
    Writer w(path);
    if (!w.ok()) return wk::set_error(WAKE_ERR_INVALID, std::string("cannot open ") + (path ? path : "(null)"));
    const int T = thread_count(threads);
    const long long rows = static_cast<long long>(ny) * nz;
    w.put(header(nx, ny, nz));
    w.put(array_open("Float32", "Velocity", 3));
    w.put(format_rows(rows, nx, T, [ux, uy, uz](std::string& s, long long i) {
        put_float(s, ux[i]);
        s.push_back(' ');
        put_float(s, uy[i]);
        s.push_back(' ');
        put_float(s, uz[i]);
        s.push_back(' ');
    }));
    w.put(std::string(kArrayClose));
    scalar_array(w, "Speed", speed, rows, nx, T);
    scalar_array(w, "Density", rho, rows, nx, T);
    if (q_criterion) scalar_array(w, "Q_Criterion", q_criterion, rows, nx, T);
    if (vort) {
        w.put(array_open("Float32", "Vorticity", 3));
        w.put(format_rows(rows, nx, T, [vorticity_x, vorticity_y, vorticity_z](std::string& s, long long i) {
            put_float(s, vorticity_x[i]);
            s.push_back(' ');
            put_float(s, vorticity_y[i]);
            s.push_back(' ');
            put_float(s, vorticity_z[i]);
            s.push_back(' ');
        }));
        w.put(std::string(kArrayClose));
    }
    cell_type_array(w, cell_type, rows, nx, T);
    w.put(std::string(kFooter));
    if (!w.close()) return wk::set_error(WAKE_ERR_INVALID, std::string("write failed: ") + path);
    return WAKE_OK;
}

// VtkExporter::write_pvd_manifest (src/export/vtk_exporter.cpp:198-221). File
// names are prefix_NNNNNN.vti: the step right-aligned in 6 characters padded
// with '0' (std::setw + std::setfill, which pads a negative step before its sign).
int wake_vtk_write_pvd(const char* manifest_path, const char* file_prefix, int start_step, int end_step,
                       int step_interval, float dt) {
    if (!file_prefix) return wk::set_error(WAKE_ERR_INVALID, "wake_vtk_write_pvd: null prefix");
    if (step_interval <= 0 && start_step <= end_step)
        return wk::set_error(WAKE_ERR_INVALID, "wake_vtk_write_pvd: the step interval must be positive");
    Writer w(manifest_path);
    if (!w.ok())
        return wk::set_error(WAKE_ERR_INVALID, std::string("cannot open ") + (manifest_path ? manifest_path : "(null)"));
    std::string s = "<?xml version=\"1.0\"?>\n";
    s += "<VTKFile type=\"Collection\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
    s += "  <Collection>\n";
    for (long long st = start_step; st <= end_step; st += step_interval) {
        std::string num;
        put_int(num, st);
        if (num.size() < 6) num.insert(0, 6 - num.size(), '0');
        const float t = static_cast<float>(static_cast<int>(st)) * dt;
        s += "    <DataSet timestep=\"";
        put_float(s, t);
        s += "\" group=\"\" part=\"0\" file=\"";
        s += file_prefix;
        s += "_" + num + ".vti\"/>\n";
    }
    s += "  </Collection>\n";
    s += "</VTKFile>\n";
    w.put(s);
    if (!w.close()) return wk::set_error(WAKE_ERR_INVALID, std::string("write failed: ") + manifest_path);
    return WAKE_OK;
}

// The grid's current state as the reference's exporter sees it after a step:
// moments, cell types and (analytics != 0) the device-computed vorticity and,
// in 3D, the Q-criterion.
int wake_grid_export_vti(wake_grid* g, const char* path, int analytics, int threads) {
    int q = 0, nx = 0, ny = 0, nz = 0, storage = 0;
    long long pitch = 0;
    int r = wake_grid_info(g, &q, &nx, &ny, &nz, &storage, &pitch);
    if (r) return r;
    const std::size_t n = static_cast<std::size_t>(nx) * ny * nz;
    std::vector<float> rho(n), ux(n), uy(n), uz(q == 9 ? 0 : n), speed(n);
    std::vector<uint8_t> types(n);
    r = wake_grid_get_macroscopic(g, rho.data(), ux.data(), uy.data(), q == 9 ? nullptr : uz.data(), speed.data());
    if (r) return r;
    r = wake_grid_get_cell_types(g, types.data());
    if (r) return r;
    if (q == 9) {
        std::vector<float> vort(analytics ? n : 0);
        if (analytics && (r = wake_grid_compute_vorticity(g, vort.data()))) return r;
        return wake_vtk_write_vti_2d(path, nx, ny, ux.data(), uy.data(), speed.data(), rho.data(),
                                     analytics ? vort.data() : nullptr, types.data(), threads);
    }
    std::vector<float> ox(analytics ? n : 0), oy(analytics ? n : 0), oz(analytics ? n : 0), qc(analytics ? n : 0);
    if (analytics && (r = wake_grid_compute_3d_features(g, ox.data(), oy.data(), oz.data(), qc.data()))) return r;
    return wake_vtk_write_vti_3d(path, nx, ny, nz, ux.data(), uy.data(), uz.data(), speed.data(), rho.data(),
                                 analytics ? qc.data() : nullptr, analytics ? ox.data() : nullptr,
                                 analytics ? oy.data() : nullptr, analytics ? oz.data() : nullptr, types.data(),
                                 threads);
}

}  // extern "C"
