// csv.cpp — snapshots in the reference's CSV v1 format.
//
// Reference: CSVWriter (src/writers/csv_writer.cpp:18-170) writes a 50-line
// "# Key: Value" header (provenance, unit system, simulation state, physics
// parameters, energies, column descriptions), one column-name line and one
// row per particle: id, pos, vel, acc, mass, dens, pres, ene, sml, sound,
// alpha, balsara, gradh, phi, neighbor — doubles through an iostream set to
// std::scientific with the writer's precision (16 by default), which prints
// exactly what printf's "%.*e" prints.  OutputManager::build_metadata
// (src/output_manager.cpp:254-299) fills the header; load_for_resume
// (src/output_manager.cpp:150-233) reads it back with CSVWriter::read_metadata
// / read_particles (src/writers/csv_writer.cpp:172-369).
//
// The text is produced on host threads: every double must be converted to
// decimal with the C library's correctly rounded conversion, byte for byte as
// the reference prints it.  Rows are formatted in parallel chunks and written
// in order.
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "sphgpu.h"

namespace {

// the 19 double columns after id, in the reference's order (neighbor last, int)
const int kCols[19] = {SPHGPU_F_POS_X, SPHGPU_F_POS_Y, SPHGPU_F_POS_Z, SPHGPU_F_VEL_X, SPHGPU_F_VEL_Y,
                       SPHGPU_F_VEL_Z, SPHGPU_F_ACC_X, SPHGPU_F_ACC_Y, SPHGPU_F_ACC_Z, SPHGPU_F_MASS,
                       SPHGPU_F_DENS,  SPHGPU_F_PRES,  SPHGPU_F_ENE,   SPHGPU_F_SML,   SPHGPU_F_SOUND,
                       SPHGPU_F_ALPHA, SPHGPU_F_BALSARA, SPHGPU_F_GRADH, SPHGPU_F_PHI};

// OutputMetadata::get_sph_type_name / get_kernel_type_name (src/output_metadata.cpp:50-65):
// types without a name there print "Unknown".
const char* sph_type_name(int t)
{
    switch(t) {
        case SPHGPU_SSPH: return "Standard SPH";
        case SPHGPU_DISPH: return "Density Independent SPH";
        case SPHGPU_GSPH: return "Godunov SPH";
        default: return "Unknown";
    }
}

const char* kernel_name(int k)
{
    switch(k) {
        case SPHGPU_CUBIC_SPLINE: return "Cubic Spline";
        case SPHGPU_WENDLAND: return "Wendland C4";
        default: return "Unknown";
    }
}

struct Out {
    std::string s;
    char buf[64];
    int prec;
    void d(double v)
    {
        const int k = std::snprintf(buf, sizeof(buf), "%.*e", prec, v);
        s.append(buf, (size_t)k);
    }
    void i(long long v)
    {
        const int k = std::snprintf(buf, sizeof(buf), "%lld", v);
        s.append(buf, (size_t)k);
    }
    void t(const char* x) { s.append(x); }
};

std::string timestamp_now()
{
    // OutputMetadata::generate_timestamp: ISO 8601, UTC
    std::time_t now = std::time(nullptr);
    std::tm tm{};
    gmtime_r(&now, &tm);
    char b[32];
    std::strftime(b, sizeof(b), "%Y-%m-%dT%H:%M:%SZ", &tm);
    return b;
}

void header(Out& o, int64_t n, const sphgpu_csv_meta& m)
{
    o.t("# SPH Simulation Output - CSV Format v1\n# Timestamp: ");
    o.t(m.timestamp && m.timestamp[0] ? m.timestamp : timestamp_now().c_str());
    o.t("\n# Simulation: SPH Simulation\n#\n");
    // code units (UnitSystem's default): every factor 1
    o.t("# === Unit System ===\n# Type: Code\n# Length: code_length (");
    o.d(1.0);
    o.t(" cm)\n# Mass: code_mass (");
    o.d(1.0);
    o.t(" g)\n# Time: code_time (");
    o.d(1.0);
    o.t(" s)\n# Velocity: code_velocity (");
    o.d(1.0);
    o.t(" cm/s)\n#\n");
    o.t("# === Simulation State ===\n# Step: ");
    o.i(m.step);
    o.t("\n# Time (code): ");
    o.d(m.time);
    o.t("\n# Time (physical): ");
    o.d(m.time);
    o.t(" code_time\n# Particle Count: ");
    o.i(n);
    o.t("\n#\n# === Physics Parameters ===\n# Gamma: ");
    o.d(m.gamma);
    o.t("\n# G: ");
    o.d(m.g_constant);
    o.t("\n# Neighbor Number: ");
    o.i(m.neighbor_number);
    o.t("\n# SPH Type: ");
    o.t(sph_type_name(m.sph_type));
    o.t("\n# Kernel: ");
    o.t(kernel_name(m.kernel));
    o.t(m.use_gravity ? "\n# Gravity: enabled" : "\n# Gravity: disabled");
    o.t(m.use_balsara ? "\n# Balsara Switch: enabled" : "\n# Balsara Switch: disabled");
    o.t(m.use_time_dependent_av ? "\n# Time-Dependent AV: enabled" : "\n# Time-Dependent AV: disabled");
    o.t("\n#\n# === Energy ===\n# Kinetic: ");
    o.d(m.kinetic);
    o.t(" [code units]\n# Thermal: ");
    o.d(m.thermal);
    o.t(" [code units]\n# Potential: ");
    o.d(m.potential);
    o.t(" [code units]\n# Total: ");
    o.d(m.kinetic + m.thermal + m.potential);
    o.t(" [code units]\n#\n");
    o.t("# === Columns ===\n"
        "# id: Particle ID\n"
        "# pos_x, pos_y, pos_z: Position [code units]\n"
        "# vel_x, vel_y, vel_z: Velocity [code units]\n"
        "# acc_x, acc_y, acc_z: Acceleration [code units]\n"
        "# mass: Particle mass [code units]\n"
        "# dens: Density [code units]\n"
        "# pres: Pressure [code units]\n"
        "# ene: Specific internal energy [code units]\n"
        "# sml: Smoothing length [code units]\n"
        "# sound: Sound speed [code units]\n"
        "# alpha: Artificial viscosity coefficient\n"
        "# balsara: Balsara factor\n"
        "# gradh: grad-h term factor\n"
        "# phi: Gravitational potential [code units]\n"
        "# neighbor: Number of neighbors\n"
        "#\n"
        "id,pos_x,pos_y,pos_z,vel_x,vel_y,vel_z,acc_x,acc_y,acc_z,"
        "mass,dens,pres,ene,sml,sound,alpha,balsara,gradh,phi,neighbor\n");
}

double field_or_zero(const double* const* f, int k, int64_t i) { return f[k] ? f[k][i] : 0.0; }

}  // namespace

extern "C" {

int sphgpu_csv_write_host(const char* path, int64_t n, const double* const* fields, const int64_t* ids,
                          const sphgpu_csv_meta* meta)
{
    if(!path || !fields || !meta || n < 0 || meta->precision < 1 || meta->precision > 30) return SPHGPU_ERR_ARG;
    std::FILE* fp = std::fopen(path, "wb");
    if(!fp) return SPHGPU_ERR_ARG;
    Out h{std::string(), {}, meta->precision};
    header(h, n, *meta);
    bool ok = std::fwrite(h.s.data(), 1, h.s.size(), fp) == h.s.size();
    // rows: formatted in parallel chunks, written in order
    const int64_t chunk = 1 << 16;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    for(int64_t base = 0; ok && base < n; base += chunk * (int64_t)hw) {
        std::vector<std::string> parts(hw);
        std::vector<std::thread> pool;
        for(unsigned t = 0; t < hw; ++t) {
            const int64_t a = base + (int64_t)t * chunk;
            if(a >= n) break;
            const int64_t b = std::min(n, a + chunk);
            pool.emplace_back([&, t, a, b]() {
                Out o{std::string(), {}, meta->precision};
                o.s.reserve((size_t)(b - a) * (size_t)(19 * (meta->precision + 8) + 24));
                for(int64_t i = a; i < b; ++i) {
                    o.i(ids ? ids[i] : i);
                    for(int c = 0; c < 19; ++c) {
                        o.s.push_back(',');
                        o.d(field_or_zero(fields, kCols[c], i));
                    }
                    o.s.push_back(',');
                    o.i((long long)field_or_zero(fields, SPHGPU_F_NEIGHBOR, i));
                    o.s.push_back('\n');
                }
                parts[t] = std::move(o.s);
            });
        }
        for(auto& th : pool) th.join();
        for(auto& p : parts) {
            if(!p.empty() && std::fwrite(p.data(), 1, p.size(), fp) != p.size()) ok = false;
        }
    }
    if(std::fclose(fp) != 0) ok = false;
    return ok ? SPHGPU_OK : SPHGPU_ERR_ARG;
}

int sphgpu_csv_read_host(const char* path, int64_t* n, int64_t cap, double* const* fields, int64_t* ids,
                         sphgpu_csv_meta* meta)
{
    if(!path || !n) return SPHGPU_ERR_ARG;
    std::ifstream in(path);
    if(!in) return SPHGPU_ERR_ARG;
    std::string line;
    // header: "# Key: Value" lines among the first 50 (CSVWriter::read_metadata)
    for(int k = 0; k < 50; ++k) {
        if(!std::getline(in, line)) return SPHGPU_ERR_ARG;
        if(!meta || line.size() < 2 || line[0] != '#') continue;
        const size_t colon = line.find(':');
        if(colon == std::string::npos || colon < 2) continue;
        std::string key = line.substr(2, colon - 2), val = colon + 2 <= line.size() ? line.substr(colon + 2) : "";
        auto num = [&](const std::string& v) { return std::strtod(v.c_str(), nullptr); };
        auto pre = [&](const std::string& v) { return v.substr(0, v.find(" [")); };
        if(key == "Step") meta->step = std::atoi(val.c_str());
        else if(key == "Time (code)") meta->time = num(val);
        else if(key == "Gamma") meta->gamma = num(val);
        else if(key == "G") meta->g_constant = num(val);
        else if(key == "Neighbor Number") meta->neighbor_number = std::atoi(val.c_str());
        else if(key == "Kinetic") meta->kinetic = num(pre(val));
        else if(key == "Thermal") meta->thermal = num(pre(val));
        else if(key == "Potential") meta->potential = num(pre(val));
    }
    if(!std::getline(in, line)) return SPHGPU_ERR_ARG;  // column names
    // rows (CSVWriter::read_particles): 21 comma-separated columns each
    int64_t count = 0;
    while(std::getline(in, line)) {
        if(line.empty()) continue;
        if(fields && count < cap) {
            const char* p = line.c_str();
            char* end = nullptr;
            const long long id = std::strtoll(p, &end, 10);
            if(end == p || *end != ',') return SPHGPU_ERR_ARG;
            if(ids) ids[count] = id;
            for(int c = 0; c < 19; ++c) {
                p = end + 1;
                const double v = std::strtod(p, &end);
                if(end == p || *end != ',') return SPHGPU_ERR_ARG;
                if(fields[kCols[c]]) fields[kCols[c]][count] = v;
            }
            p = end + 1;
            const long long nb = std::strtoll(p, &end, 10);
            if(end == p || (*end != '\0' && *end != '\r')) return SPHGPU_ERR_ARG;
            if(fields[SPHGPU_F_NEIGHBOR]) fields[SPHGPU_F_NEIGHBOR][count] = (double)nb;
        }
        ++count;
    }
    *n = count;
    if(fields && count > cap) return SPHGPU_ERR_ARG;
    return SPHGPU_OK;
}

}  // extern "C"
