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

void configure(Params& ps) {
    ps.add_flag("help");
    ps.add_flag("h");
    ps.add_string("paramfile", "modess.param");
    ps.add_flag("printparams");
    ps.add_string_nodefault("atmosfile");
    ps.require("atmosfile");
    ps.add_float_nodefault("freq");
    ps.require("freq");
    ps.float_gt("freq", 0.0);
    ps.add_string("atmosheaderfile", "");
    ps.add_float("maxheight_km", 150.0);
    ps.float_ge("maxheight_km", 0.1);
    ps.add_float("zground_km", 0.0);
    ps.add_int("Nz_grid", 20000);
    ps.int_ge("Nz_grid", 10);
    ps.add_float("sourceheight_km", 0.0);
    ps.add_float("receiverheight_km", 0.0);
    ps.add_float("maxrange_km", 1000.0);
    ps.float_ge("maxrange_km", 0.01);
    ps.add_int("Nrng_steps", 1000);
    ps.int_gt("Nrng_steps", 0);
    ps.add_string("ground_impedence_model", "rigid");
    ps.string_set("ground_impedence_model", {"rigid"});
    ps.add_string("use_attn_file", "");
    ps.add_string("modal_starter_file", "");
    ps.add_string("dispersion_file", "");
    ps.add_flag("append_dispersion_file");
    ps.add_string("filetag", "");
    ps.add_flag("singleprop");
    ps.add_flag("multiprop");
    ps.radio("operation_mode", {"singleprop", "multiprop"});
    ps.add_float_nodefault("azimuth");
    ps.float_ge("azimuth", 0.0);
    ps.float_lt("azimuth", 360.0);
    ps.require_if("azimuth", "singleprop");
    for (const char* k : {"azimuth_start", "azimuth_end", "azimuth_step"}) {
        ps.add_float_nodefault(k);
        ps.float_ge(k, 0.0);
        ps.float_le(k, 360.0);
        ps.require_if(k, "multiprop");
    }
    for (const char* k : {"write_2d_tloss", "write_lossless", "write_phase_speeds", "write_speeds", "write_modes",
                          "write_atm_profile", "Lamb_wave_BC", "turnoff_WKB", "wvnum_filter"})
        ps.add_flag(k);
    for (const char* k : {"c_min", "c_max"}) {
        ps.add_float_nodefault(k);
        ps.float_gt(k, 0.0);
        ps.require_if(k, "wvnum_filter");
    }
    ps.add_flag("broadband");
    ps.add_float("f_min", 0.0);
    ps.add_float("f_max", 0.0);
    ps.add_float("f_step", 0.0);
}

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
    configure(param);
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
