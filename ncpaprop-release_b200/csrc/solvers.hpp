// The reference's solver classes for this path, on the GPU library:
//   NCPA::ESSModeSolver (src/libmodes/ESSModeSolver.h:53-80, the
//     AtmosphericTransferFunctionSolver / ModeSolver interface: construct
//     from the parameter set, solve(), printParams())
//   NCPA::WModeSolver (src/libmodes/WModeSolver.h:45-61, the same interface
//     for the wide-angle high-Mach solve; ModBB --method wmod)
//   NCPA::ModalBroadbandPropagator (src/libbroadband/ModalBroadbandPropagator.h:
//     10-28, the BroadbandPropagator interface: construct from the parameter
//     set, calculate_waveform())
// The reference's ESSModeSolver also takes the Atmosphere1D its caller read;
// here the profile named by the atmosfile option is read and uploaded by
// solve() itself.  Errors are thrown as in the reference (std::exception
// subclasses); the methods return 0.
#pragma once

#include "cli_params.hpp"

namespace ncpa_gpu_solvers {

class ESSModeSolver {
public:
    explicit ESSModeSolver(const ncpa_cli::Params* param) : param_(*param) {}
    int solve();
    void printParams() const;

private:
    ncpa_cli::Params param_;
};

class WModeSolver {
public:
    explicit WModeSolver(const ncpa_cli::Params* param) : param_(*param) {}
    int solve();

private:
    ncpa_cli::Params param_;
};

class ModalBroadbandPropagator {
public:
    explicit ModalBroadbandPropagator(const ncpa_cli::Params* param) : param_(*param) {}
    int calculate_waveform();

private:
    ncpa_cli::Params param_;
};

}  // namespace ncpa_gpu_solvers
