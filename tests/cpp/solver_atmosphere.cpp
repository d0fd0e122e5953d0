// Test driver for the solver classes' in-memory atmosphere
// (ncpa_gpu_solvers::ESSModeSolver(Params*, Atmosphere1D*), as the
// reference's ESSModeSolver(ParameterSet*, Atmosphere1D*)).
//
//   solver_atmosphere <profile> <out_dir>
//
// Reads the profile into an Atmosphere1D, adds a 30 m/s zonal jet at 50 km
// in memory, writes the changed profile to <out_dir>/changed.dat, then runs
// the ESS solve three times in <out_dir>: on the in-memory atmosphere
// (filetag "mem"), on the written file (filetag "file") and on the original
// file (filetag "orig").  The caller compares the output files.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "cli_ess.hpp"
#include "cli_params.hpp"
#include "solvers.hpp"

namespace {

ncpa_cli::Params params(const std::string& atmosfile, const std::string& tag) {
    ncpa_cli::Params p;
    ncpa_cli::configure_modess(p);
    std::vector<std::string> args = {"solver_atmosphere", "--singleprop", "--atmosfile", atmosfile, "--freq", "0.1",
                                     "--azimuth", "90", "--Nz_grid", "8000", "--write_2d_tloss", "--filetag", tag};
    std::vector<char*> argv;
    for (auto& a : args) argv.push_back(&a[0]);
    p.parse_command_line((int)argv.size(), argv.data());
    return p;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: solver_atmosphere <profile> <out_dir>\n");
        return 2;
    }
    const std::string prof = argv[1], dir = argv[2];
    try {
        ncpa_gpu_solvers::Atmosphere1D atm(prof);
        const std::vector<double>& z = atm.get("Z");
        std::vector<double>& u = atm.get("U");
        for (size_t i = 0; i < z.size(); ++i) u[i] += 30.0 * std::exp(-std::pow((z[i] - 50000.0) / 8000.0, 2));
        const std::string changed = dir + "/changed.dat";
        atm.write(changed);
        const ncpa_cli::Params pm = params("unused-by-the-in-memory-solve", dir + "/mem");
        ncpa_gpu_solvers::ESSModeSolver(&pm, &atm).solve();
        const ncpa_cli::Params pf = params(changed, dir + "/file");
        ncpa_gpu_solvers::ESSModeSolver(&pf).solve();
        const ncpa_cli::Params po = params(prof, dir + "/orig");
        ncpa_gpu_solvers::ESSModeSolver(&po).solve();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "solver_atmosphere: %s\n", e.what());
        return 1;
    }
    return 0;
}
