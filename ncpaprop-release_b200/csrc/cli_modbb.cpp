// ModBB: broadband ESS normal modes.  --dispersion writes the dispersion file
// (one line per frequency) with the ESS solve on the GPU; --propagation reads
// a dispersion file and synthesises pulses at the receivers.  Options,
// defaults, checks and files follow the reference front end
// (src/modbb/ModBB_main.cpp, src/modbb/modbb_parameters.cpp:42-234,
// src/libbroadband/ModalBroadbandPropagator.cpp:25-231,
// src/libbroadband/BroadbandPropagator.cpp:244-414).
#include <cmath>
#include <cstdio>
#include <ctime>
#include <fstream>
#include <iostream>
#include <sstream>

#include "cli_common.hpp"
#include "cli_ess.hpp"
#include "cli_params.hpp"
#include "solvers.hpp"

using ncpa_cli::Params;
using ncpa_cli::RunError;

namespace {

void configure(Params& ps) {
    ps.add_flag("help");
    ps.add_flag("h");
    ps.add_string("paramfile", "modbb.param");
    ps.add_flag("printparams");
    ps.add_flag("dispersion");
    ps.add_flag("propagation");
    ps.radio("operation_mode", {"dispersion", "propagation"});
    ps.add_string("method", "modess");
    ps.string_set("method", {"modess", "wmod"});
    ps.require_if("method", "dispersion");
    ps.add_string("dispersion_file", "");
    ps.require_if("dispersion_file", "dispersion");
    ps.add_flag("append_dispersion_file", true);
    ps.add_float_nodefault("azimuth");
    ps.float_ge("azimuth", 0.0);
    ps.float_lt("azimuth", 360.0);
    ps.require_if("azimuth", "dispersion");
    for (const char* k : {"f_min", "f_max", "f_step"}) {
        ps.add_float_nodefault(k);
        ps.float_gt(k, 0.0);
        ps.require_if(k, "dispersion");
    }
    ps.add_string_nodefault("atmosfile");
    ps.require_if("atmosfile", "dispersion");
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
    ps.add_flag("Lamb_wave_BC");
    ps.add_flag("write_atm_profile");
    ps.add_string("use_attn_file", "");
    ps.add_flag("use_zero_attenuation");
    ps.add_flag("wvnum_filter");
    for (const char* k : {"c_min", "c_max"}) {
        ps.add_float_nodefault(k);
        ps.float_gt(k, 0.0);
        ps.require_if(k, "wvnum_filter");
    }
    ps.add_string("input_dispersion_file", "");
    ps.require_if("input_dispersion_file", "propagation");
    ps.add_string("dispersion_cache", "");  // binary copy of the parsed dispersion file (no reference counterpart)
    ps.add_string("output_waveform_file", "");
    ps.require_if("output_waveform_file", "propagation");
    ps.add_string("source", "impulse");
    ps.string_set("source", {"impulse", "pulse1", "pulse2", "waveform", "spectrum"});
    ps.add_string("source_file", "");
    ps.add_float("f_center", -1.0);
    ps.add_int("nfft", 0);
    ps.int_ge("nfft", 0);
    ps.add_float("max_celerity", 340.0);
    ps.int_gt("max_celerity", 0);
    ps.add_string("receiver", "single");
    ps.string_set("receiver", {"single", "multiple"});
    for (const char* k : {"range_km", "start_range_km", "end_range_km", "range_step_km"}) ps.add_float(k, 0.0);
    // entries ESSModeSolver::setParams reads (modbb_parameters.cpp:216-233)
    ps.add_flag("broadband", true);
    ps.add_string("modal_starter_file", "");
    for (const char* k : {"write_2d_tloss", "write_phase_speeds", "write_speeds", "write_modes", "write_lossless",
                          "multiprop", "turnoff_WKB"})
        ps.add_flag(k);
    ps.add_string("filetag", "");
}

void usage(std::ostream& os) {
    os << "ModBB -- broadband effective sound speed normal modes (GPU)\n\n"
          "Options (command line or \"key: value\" lines in modbb.param):\n"
          "  --dispersion --dispersion_file F --atmosfile F --azimuth a --f_min f --f_step d --f_max f\n"
          "      [--method modess] [--Nz_grid 20000] [--maxheight_km 150] [--zground_km 0]\n"
          "      [--sourceheight_km 0] [--receiverheight_km 0] [--Lamb_wave_BC] [--use_attn_file F]\n"
          "      [--wvnum_filter --c_min c --c_max c] [--write_atm_profile] [--append_dispersion_file]\n"
          "  --propagation --input_dispersion_file F --output_waveform_file F\n"
          "      [--source impulse|pulse1|pulse2|spectrum|waveform] [--source_file F] [--f_center f]\n"
          "      [--receiver single --range_km r | --receiver multiple --start_range_km a\n"
          "       --end_range_km b --range_step_km d] [--nfft n] [--max_celerity 340]\n"
          "      [--use_zero_attenuation] [--dispersion_cache F]\n\n"
          "Output files: the dispersion file; source_waveform_input.dat, source_spectrum_input.dat\n"
          "and the waveform file (r [km], t [s], 2 Re p) for --propagation.\n";
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
        if (param.get_bool("dispersion")) {
            const std::string disp = param.get_string("dispersion_file");
            if (!disp.empty()) std::ofstream(disp, std::ios_base::trunc).close();
            if (param.get_string("method") == "modess") {  // as ModBB_main.cpp:84-91
                ncpa_gpu_solvers::ESSModeSolver solver(&param);
                solver.solve();
            } else {
                ncpa_gpu_solvers::WModeSolver solver(&param);
                solver.solve();
            }
            std::cout << "Finished computing and saving dispersion data" << std::endl;
        } else if (param.get_bool("propagation")) {
            ncpa_gpu_solvers::ModalBroadbandPropagator prop(&param);  // as ModBB_main.cpp:108-110
            prop.calculate_waveform();
        }
    } catch (const std::exception& e) {
        std::cerr << "ModBB: " << e.what() << std::endl;
        return 2;
    }
    std::cout << "\nRun duration: " << std::difftime(std::time(nullptr), t1) << " seconds." << std::endl;
    std::cout << " ... main() broadband version is done." << std::endl;
    return 0;
}
