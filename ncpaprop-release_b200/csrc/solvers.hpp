// The reference's solver classes for this path, on the GPU library:
//   NCPA::ESSModeSolver (src/libmodes/ESSModeSolver.h:53-80, the
//     AtmosphericTransferFunctionSolver / ModeSolver interface: construct
//     from the parameter set, solve(), printParams())
//   NCPA::WModeSolver (src/libmodes/WModeSolver.h:45-61, the same interface
//     for the wide-angle high-Mach solve; ModBB --method wmod)
//   NCPA::ModalBroadbandPropagator (src/libbroadband/ModalBroadbandPropagator.h:
//     10-28, the BroadbandPropagator interface: construct from the parameter
//     set, calculate_waveform())
// Like the reference's ESSModeSolver(ParameterSet*, Atmosphere1D*)
// (ESSModeSolver.h:53-80), the mode solvers take the caller's atmosphere:
// an Atmosphere1D read from a profile file or built from arrays, and changed
// in memory as the caller needs (the reference's solvers add and remove
// derived properties on it; these leave it as it is).  Constructed from the
// parameter set alone, solve() reads the profile named by the atmosfile
// option itself.  Errors are thrown as in the reference (std::exception
// subclasses); the methods return 0.
#pragma once

#include <string>
#include <vector>

#include "atmosphere.hpp"
#include "cli_params.hpp"
#include "ncpa_gpu.h"

namespace ncpa_gpu_solvers {

// The caller's atmospheric profile (the role of NCPA::Atmosphere1D,
// src/atmosphere/Atmosphere1D.h): knot arrays in SI units.
class Atmosphere1D {
public:
    // read an NCPA profile file, with an optional separate header file
    // (Atmosphere1D(file, header), Atmosphere1D.cpp:44-60); units converted
    // to SI as ESSModeSolver::setParams does (ESSModeSolver.cpp:159-220)
    explicit Atmosphere1D(const std::string& file, const std::string& header = "");
    // from arrays: z [m], u, v [m/s], t [K], p [Pa], rho [kg/m3], same length
    Atmosphere1D(std::vector<double> z, std::vector<double> u, std::vector<double> v, std::vector<double> t,
                 std::vector<double> p, std::vector<double> rho);
    // a property's knot values, changeable in place: "Z" [m], "U", "V"
    // [m/s], "T" [K], "P" [Pa], "RHO" [kg/m3], "C0" [m/s] (only if present)
    std::vector<double>& get(const std::string& key);
    const std::vector<double>& get(const std::string& key) const;
    bool contains(const std::string& key) const;
    int nz() const { return (int)s_.z.size(); }
    // ground height Z0 [m] of the profile (the scalar of the file header)
    bool has_z0() const { return s_.has_z0; }
    double z0() const { return s_.z0; }
    void set_z0(double z0_m);
    // the knot description ncpa_profile_create takes (points into this object)
    ncpa_profile_desc desc() const;
    // an NCPA profile file of the current values (SI units, 17 digits)
    void write(const std::string& path) const;

private:
    ncpa::SiProfile s_;
};

class ESSModeSolver {
public:
    explicit ESSModeSolver(const ncpa_cli::Params* param) : param_(*param) {}
    ESSModeSolver(const ncpa_cli::Params* param, const Atmosphere1D* atm) : param_(*param), atm_(atm) {}
    int solve();
    void printParams() const;

private:
    ncpa_cli::Params param_;
    const Atmosphere1D* atm_ = nullptr;
};

class WModeSolver {
public:
    explicit WModeSolver(const ncpa_cli::Params* param) : param_(*param) {}
    WModeSolver(const ncpa_cli::Params* param, const Atmosphere1D* atm) : param_(*param), atm_(atm) {}
    int solve();

private:
    ncpa_cli::Params param_;
    const Atmosphere1D* atm_ = nullptr;
};

class ModalBroadbandPropagator {
public:
    explicit ModalBroadbandPropagator(const ncpa_cli::Params* param) : param_(*param) {}
    int calculate_waveform();

private:
    ncpa_cli::Params param_;
};

}  // namespace ncpa_gpu_solvers
