// ESS solve loop shared by the Modess and ModBB front ends (cli_ess.cpp).
#pragma once

#include "cli_params.hpp"
#include "ncpa_gpu.h"

namespace ncpa_cli {

// Runs ESSModeSolver::solve's work for the options in prm (Modess's option
// set, or ModBB's with its broadband / dummy entries), or with wmod set
// WModeSolver::solve's (the wide-angle solve: no group speeds, no Lamb-wave
// condition outputs beyond the ESS ones); throws RunError.  With atm given
// the profile comes from those knot arrays (the caller's atmosphere) instead
// of the atmosfile option.
void run_ess(const Params& prm, bool wmod, const ncpa_profile_desc* atm = nullptr);

// The option set of the Modess front end (src/modess/modess_parameters.cpp:
// 29-189): keys, defaults and tests.
void configure_modess(Params& ps);

}  // namespace ncpa_cli
