// ESS solve loop shared by the Modess and ModBB front ends (cli_ess.cpp).
#pragma once

#include "cli_params.hpp"

namespace ncpa_cli {

// Runs ESSModeSolver::solve's work for the options in prm (Modess's option
// set, or ModBB's with its broadband / dummy entries); throws RunError.
void run_ess(const Params& prm);

}  // namespace ncpa_cli
