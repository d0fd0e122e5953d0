// Modess: effective-sound-speed normal modes, single frequency, one azimuth
// (--singleprop) or N x 2-D (--multiprop).  Same options, defaults, checks and
// output files as the reference front end (src/modess/Modess_main.cpp,
// src/modess/modess_parameters.cpp:29-189); the solve runs on the GPU
// through the C ABI.
#include <ctime>
#include <iostream>
#include <sstream>

#include "cli_common.hpp"
#include "cli_ess.hpp"
#include "cli_params.hpp"
#include "solvers.hpp"

using ncpa_cli::Params;

namespace {

void usage(std::ostream& os) {
    os << "Modess -- effective sound speed normal modes (GPU)\n\n"
          "Options (command line \"--key value\" or a \"key: value\" line in the parameter file\n"
          "modess.param; command-line options override file options):\n"
          "  --atmosfile F            atmospheric profile (required)\n"
          "  --atmosheaderfile F      separate profile header\n"
          "  --freq f                 frequency [Hz] (required)\n"
          "  --singleprop --azimuth a   |  --multiprop --azimuth_start a --azimuth_end b --azimuth_step d\n"
          "  --maxheight_km [150] --zground_km [0] --Nz_grid [20000]\n"
          "  --sourceheight_km [0] --receiverheight_km [0] --maxrange_km [1000] --Nrng_steps [1000]\n"
          "  --ground_impedence_model [rigid] --Lamb_wave_BC --turnoff_WKB\n"
          "  --wvnum_filter --c_min c --c_max c   --use_attn_file F\n"
          "  --write_2d_tloss --write_lossless --write_phase_speeds --write_speeds --write_modes\n"
          "  --write_atm_profile --modal_starter_file F --dispersion_file F --append_dispersion_file\n"
          "  --filetag T --paramfile F --printparams\n\n"
          "Output files: tloss_1d.nm, tloss_1d.lossless.nm, tloss_2d.nm, tloss_2d.lossless.nm,\n"
          "Nby2D_tloss_1d.nm, Nby2D_tloss_1d.lossless.nm, phasespeeds.nm, speeds.nm, mode_<n>.nm,\n"
          "atm_profile.nm, and the modal starter / dispersion files named by their options.\n";
}

}  // namespace

int main(int argc, char** argv) {
    Params param;
    ncpa_cli::configure_modess(param);
    try {
        param.parse_command_line(argc, argv);
        if (param.found("help") || param.found("h")) {
            usage(std::cout);
            return 1;
        }
        param.parse_file(param.get_string("paramfile"));
        param.parse_command_line(argc, argv);
        if (param.found("printparams")) param.print(std::cout);
    } catch (const std::exception& e) {
        std::cout << "Parameter validation failed: " << std::endl << e.what() << std::endl;
    }
    std::ostringstream failures;
    if (!param.validate(failures)) {
        std::cout << "Parameter validation failed:" << std::endl << failures.str();
        return 0;
    }
    const std::time_t t1 = std::time(nullptr);
    try {
        ncpa_gpu_solvers::ESSModeSolver a(&param);  // as Modess_main.cpp:87-97
        a.solve();
        a.printParams();
    } catch (const std::exception& e) {
        std::cerr << "Modess: " << e.what() << std::endl;
        return 2;
    }
    std::cout << std::endl << " ... main() is done." << std::endl;
    std::cout << "Run duration: " << std::difftime(std::time(nullptr), t1) << " seconds." << std::endl;
    return 0;
}
