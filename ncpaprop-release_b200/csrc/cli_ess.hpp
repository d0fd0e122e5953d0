// ESS solve loop shared by the Modess and ModBB front ends (cli_ess.cpp).
#pragma once

#include "cli_params.hpp"

namespace ncpa_cli {

// Runs ESSModeSolver::solve's work for the options in prm (Modess's option
// set, or ModBB's with its broadband / dummy entries), or with wmod set
// WModeSolver::solve's (the wide-angle solve: no group speeds, no Lamb-wave
// condition outputs beyond the ESS ones); throws RunError.
void run_ess(const Params& prm, bool wmod);

}  // namespace ncpa_cli
