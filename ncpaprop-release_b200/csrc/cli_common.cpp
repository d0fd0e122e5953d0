// Shared pieces of the Modess and ModBB front ends (see cli_common.hpp).
#include "cli_common.hpp"

#include <cmath>
#include <cstdio>
#include <memory>

namespace ncpa_cli {

namespace {
constexpr double kPi = 3.14159265358979323846;

struct File {
    std::FILE* f = nullptr;
    File(const std::string& path, const char* mode) : f(std::fopen(path.c_str(), mode)) {
        if (!f) throw RunError("file " + path + " could not be opened.");
    }
    ~File() {
        if (f) std::fclose(f);
    }
};
}  // namespace

void check(ncpa_ctx* ctx, ncpa_status s, const char* what) {
    if (s == NCPA_OK) return;
    std::string msg = std::string(what) + ": " + ncpa_status_str(s);
    if (ctx && *ncpa_last_error(ctx)) msg += std::string(" (") + ncpa_last_error(ctx) + ")";
    throw RunError(msg);
}

Gpu::Gpu() {
    ncpa_ctx_opts o{0};
    check(nullptr, ncpa_ctx_create(&ctx_, &o), "creating the GPU context");
}
Gpu::~Gpu() {
    if (ctx_) ncpa_ctx_destroy(ctx_);
}

ncpa_profile* load_profile(ncpa_ctx* ctx, const std::string& atmosfile, const std::string& headerfile,
                           const std::string& attn_file) {
    ncpa_profile* prof = nullptr;
    check(ctx, ncpa_profile_load(ctx, atmosfile.c_str(), headerfile.empty() ? nullptr : headerfile.c_str(), &prof),
          ("reading atmospheric profile " + atmosfile).c_str());
    if (!attn_file.empty()) {
        ncpa_status s = ncpa_profile_load_attn(prof, attn_file.c_str());
        if (s != NCPA_OK) {
            std::string msg = ncpa_last_error(ctx);
            ncpa_profile_destroy(prof);
            throw RunError("reading attenuation file " + attn_file + ": " + msg);
        }
    }
    return prof;
}

ncpa_profile* create_profile(ncpa_ctx* ctx, const ncpa_profile_desc* atm, const std::string& attn_file) {
    ncpa_profile* prof = nullptr;
    check(ctx, ncpa_profile_create(ctx, atm, &prof), "uploading the caller's atmospheric profile");
    if (!attn_file.empty()) {
        ncpa_status s = ncpa_profile_load_attn(prof, attn_file.c_str());
        if (s != NCPA_OK) {
            std::string msg = ncpa_last_error(ctx);
            ncpa_profile_destroy(prof);
            throw RunError("reading attenuation file " + attn_file + ": " + msg);
        }
    }
    return prof;
}

std::string tag_filename(const std::string& tag, const std::string& name) {
    return tag.empty() ? name : tag + "." + name;
}

Modes get_modes(ncpa_ctx* ctx, const ncpa_modes* m, int problem) {
    Modes r;
    check(ctx, ncpa_modes_count(m, problem, &r.M), "mode count");
    check(ctx, ncpa_modes_info(m, problem, &r.freq, &r.az, &r.dz, nullptr, nullptr, &r.rho_src, &r.rho_rcv),
          "mode info");
    r.kr.resize(r.M);
    r.ki.resize(r.M);
    r.vs.resize(r.M);
    r.vr.resize(r.M);
    r.vg.resize(r.M);
    check(ctx, ncpa_modes_get(m, problem, r.kr.data(), r.ki.data(), r.vs.data(), r.vr.data(), r.vg.data()),
          "fetching modes");
    return r;
}

// ModeSolver::getTLoss1D output (ModeSolver.cpp:364-369)
void write_tloss_1d(const std::string& path, int nr, double dr, const double* re, const double* im,
                    const double* inc) {
    File f(path, "w");
    for (int i = 0; i < nr; ++i)
        std::fprintf(f.f, "%f %20.12e %20.12e %20.12e\n", (i + 1) * dr / 1000.0, re[i], im[i], inc[i]);
}

// ModeSolver::getTLoss1DNx2 output (ModeSolver.cpp:410-489)
void write_tloss_nx2(const std::string& path, bool append, double az, int nr, double dr, const double* re,
                     const double* im, const double* inc) {
    File f(path, append ? "a" : "w");
    for (int i = 0; i < nr; ++i)
        std::fprintf(f.f, "%10.3f %8.3f %20.12e %20.12e %20.12e\n", (i + 1) * dr / 1000.0, az, re[i], im[i],
                     inc[i]);
    std::fprintf(f.f, "\n");
}

// ModeSolver::getTLoss2D output (ModeSolver.cpp:520-556); re/im [nr x nzo]
void write_tloss_2d(const std::string& path, int nr, double dr, int nzo, const double* z, const double* re,
                    const double* im) {
    File f(path, "w");
    for (int i = 0; i < nr; ++i) {
        const double r = (i + 1) * dr;
        for (int j = 0; j < nzo; ++j)
            std::fprintf(f.f, "%f %f %15.8e %15.8e\n", r / 1000.0, z[j] / 1000.0, re[(size_t)i * nzo + j],
                         im[(size_t)i * nzo + j]);
        std::fprintf(f.f, "\n");
    }
}

// ModeSolver::writePhaseSpeeds (ModeSolver.cpp:603-614)
void write_phase_speeds(const std::string& path, const Modes& m) {
    File f(path, "w");
    for (int j = 0; j < m.M; ++j) std::fprintf(f.f, "%d %f %15.8e\n", j, (2 * kPi * m.freq) / m.kr[j], m.ki[j]);
}

// ESSModeSolver::writePhaseAndGroupSpeeds (ESSModeSolver.cpp:726-752); the
// group speeds come from the eigenvector kernel's fused sum of v^2 / c_eff^2
void write_speeds(const std::string& path, const Modes& m) {
    File f(path, "w");
    for (int j = 0; j < m.M; ++j)
        std::fprintf(f.f, "%4d %9.3f %9.3f %15.8e\n", j + 1, (2 * kPi * m.freq) / m.kr[j], m.vg[j], m.ki[j]);
}

// ModeSolver::writeEigenFunctions (ModeSolver.cpp:618-641); v is [nz x M]
void write_mode_files(const std::string& tag, int nz, double dz, int M, const std::vector<double>& v) {
    const double dz_km = dz / 1000.0;
    for (int j = 0; j < M; ++j) {
        char name[40];
        std::snprintf(name, sizeof name, "mode_%d.nm", j);
        File f(tag_filename(tag, name), "w");
        double chk = 0.0;
        for (int n = 0; n < nz; ++n) {
            const double x = v[(size_t)n * M + j];
            std::fprintf(f.f, "%f %15.8e\n", n * dz_km, x);
            chk += x * x * dz;
        }
        if (std::fabs(1.0 - chk) > 0.1) std::printf("Check if eigenfunction %d is normalized!\n", j);
    }
    std::printf("           %d mode files created\n", M);
}

// ESSModeSolver::getModalStarter output (ESSModeSolver.cpp:714-719)
void write_starter(const std::string& path, int n, const double* z_km, const double* re, const double* im) {
    File f(path, "w");
    for (int j = 0; j < n; ++j) std::fprintf(f.f, "%10.3f   %16.12e   %16.12e\n", z_km[j], re[j], im[j]);
    std::fprintf(f.f, "\n");
}

// ModeSolver::writeDispersion (ModeSolver.cpp:569-589)
void append_dispersion_line(std::FILE* f, const Modes& m) {
    std::fprintf(f, "%.7e   %d    %.7e   %.7e", m.freq, m.M, m.rho_src, m.rho_rcv);
    for (int i = 0; i < m.M; ++i) {
        std::fprintf(f, "   %.12e   %.12e", m.kr[i], m.ki[i]);
        std::fprintf(f, "   %.12e   %.12e", m.vs[i], m.vr[i]);
    }
    std::fprintf(f, "\n");
}

// Atmosphere1D::print_atmosphere with the key list of ESSModeSolver.cpp:
// 468-484: scalars (Z0 when the profile has it, then the azimuth), the column
// descriptors, then one line per knot in %.6e
void write_atm_profile(const std::string& path, ncpa_profile* prof, double az) {
    int n = 0;
    double zlo, zhi;
    check(nullptr, ncpa_profile_info(prof, &n, &zlo, &zhi), "profile info");
    std::vector<double> z(n), u(n), v(n), t(n), p(n), rho(n), c0(n), ce(n);
    check(nullptr,
          ncpa_profile_knots(prof, az, z.data(), u.data(), v.data(), t.data(), p.data(), rho.data(), c0.data(),
                             ce.data()),
          "profile knots");
    double z0 = 0;
    int has_z0 = 0;
    check(nullptr, ncpa_profile_z0(prof, &z0, &has_z0), "profile Z0");
    File f(path, "w");
    if (has_z0) std::fprintf(f.f, "#%% 0, Z0, m, %g\n", z0);
    std::fprintf(f.f, "#%% 0, AZ, deg CW from N, %g\n", az);
    std::fprintf(f.f, "#%% 1, Z, m\n");
    const char* keys[] = {"U, m/s", "V, m/s", "T, K", "RHO, kg/m3", "P, Pa", "C0, m/s", "CEFF, m/s"};
    for (int k = 0; k < 7; ++k) std::fprintf(f.f, "#%% %d, %s\n", k + 2, keys[k]);
    for (int i = 0; i < n; ++i)
        std::fprintf(f.f, "%.6e %.6e %.6e %.6e %.6e %.6e %.6e %.6e\n", z[i], u[i], v[i], t[i], rho[i], p[i], c0[i],
                     ce[i]);
}

}  // namespace ncpa_cli
