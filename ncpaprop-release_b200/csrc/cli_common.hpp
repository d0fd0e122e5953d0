// Shared pieces of the Modess and ModBB front ends: the GPU context, profile
// loading, mode retrieval and the reference's text output formats
// (ModeSolver.cpp:292-641, ESSModeSolver.cpp:670-752,
// Atmosphere1D::print_atmosphere, Atmosphere1D.cpp:924-970).
#pragma once

#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "ncpa_gpu.h"

namespace ncpa_cli {

struct RunError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// throws RunError with the library's message when s != NCPA_OK
void check(ncpa_ctx* ctx, ncpa_status s, const char* what);

class Gpu {
public:
    Gpu();
    ~Gpu();
    Gpu(const Gpu&) = delete;
    Gpu& operator=(const Gpu&) = delete;
    ncpa_ctx* ctx() const { return ctx_; }

private:
    ncpa_ctx* ctx_ = nullptr;
};

// profile file (+ optional header file and attenuation table file)
// the caller's in-memory profile (plus an optional attenuation file)
ncpa_profile* create_profile(ncpa_ctx* ctx, const ncpa_profile_desc* atm, const std::string& attn_file);
ncpa_profile* load_profile(ncpa_ctx* ctx, const std::string& atmosfile, const std::string& headerfile,
                           const std::string& attn_file);

// "<tag>.<name>" when a file tag is set (ModeSolver::tag_filename)
std::string tag_filename(const std::string& tag, const std::string& name);

// the modes of one problem on the host
struct Modes {
    int M = 0;
    double freq = 0, az = 0, dz = 0, rho_src = 1, rho_rcv = 1;
    std::vector<double> kr, ki, vs, vr, vg;
};
Modes get_modes(ncpa_ctx* ctx, const ncpa_modes* m, int problem);

// writers (one call = one file, or one appended block)
void write_tloss_1d(const std::string& path, int nr, double dr, const double* re, const double* im,
                    const double* inc);
void write_tloss_nx2(const std::string& path, bool append, double az, int nr, double dr, const double* re,
                     const double* im, const double* inc);
void write_tloss_2d(const std::string& path, int nr, double dr, int nzo, const double* z, const double* re,
                    const double* im);
void write_phase_speeds(const std::string& path, const Modes& m);
void write_speeds(const std::string& path, const Modes& m);
void write_mode_files(const std::string& tag, int nz, double dz, int M, const std::vector<double>& v);
void write_starter(const std::string& path, int n, const double* z_km, const double* re, const double* im);
void append_dispersion_line(std::FILE* f, const Modes& m);
void write_atm_profile(const std::string& path, ncpa_profile* prof, double az);

}  // namespace ncpa_cli
