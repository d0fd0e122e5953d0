// ModBB --propagation (cli_bb.cpp).
#pragma once

#include "cli_params.hpp"

namespace ncpa_cli {

// Runs ModalBroadbandPropagator::calculate_waveform's work for the options in
// prm; throws RunError.  Returns 0.
int run_propagation(const Params& prm);

}  // namespace ncpa_cli
