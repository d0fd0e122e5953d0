// The reference's solver classes over the GPU front-end code (solvers.hpp).
#include "solvers.hpp"

#include <cstdio>

#include "cli_bb.hpp"
#include "cli_ess.hpp"

namespace ncpa_gpu_solvers {

int ESSModeSolver::solve() {
    ncpa_cli::run_ess(param_, false);
    return 0;
}

int WModeSolver::solve() {
    ncpa_cli::run_ess(param_, true);
    return 0;
}

// the parameter summary of ESSModeSolver::printParams (ESSModeSolver.cpp:243-290)
void ESSModeSolver::printParams() const {
    const auto& p = param_;
    auto has = [&](const char* k) { return p.found(k) || !p.get_string(k).empty(); };
    std::printf(" Effective Sound Speed Normal Modes Solver Parameters:\n");
    if (p.get_bool("broadband")) {
        std::printf("                  f_min : %g\n", p.get_float("f_min"));
        std::printf("                 f_step : %g\n", p.get_float("f_step"));
        std::printf("                  f_max : %g\n", p.get_float("f_max"));
    } else {
        std::printf("                   freq : %g\n", p.get_float("freq"));
    }
    const bool multiprop = p.get_bool("multiprop");
    if (!multiprop) {
        std::printf("                azimuth : %g\n", p.get_float("azimuth"));
    } else {
        std::printf("     azimuth_start (deg): %g\n", p.get_float("azimuth_start"));
        std::printf("       azimuth_end (deg): %g\n", p.get_float("azimuth_end"));
        std::printf("      azimuth_step (deg): %g\n", p.get_float("azimuth_step"));
    }
    std::printf("                Nz_grid : %d\n", p.get_int("Nz_grid"));
    std::printf("      z_min (meters MSL): %g\n", p.get_float("zground_km") * 1000.0);
    std::printf("      maxheight_km (MSL): %g\n", p.get_float("maxheight_km"));
    std::printf("   sourceheight_km (AGL): %g\n", p.get_float("sourceheight_km"));
    std::printf(" receiverheight_km (AGL): %g\n", p.get_float("receiverheight_km"));
    std::printf("             Nrng_steps : %d\n", p.get_int("Nrng_steps"));
    std::printf("            maxrange_km : %g\n", p.get_float("maxrange_km"));
    std::printf("          gnd_imp_model : %s\n", p.get_string("ground_impedence_model").c_str());
    std::printf("Lamb wave boundary cond : %d\n", (int)p.get_bool("Lamb_wave_BC"));
    std::printf("  eigen-solve tolerance : %g (FP64 Sturm bisection, units of h^2 A)\n", 1.0e-15);
    std::printf("    write_lossless flag : %d\n", (int)p.get_bool("write_lossless"));
    std::printf("    write_2d_tloss flag : %d\n", (int)p.get_bool("write_2d_tloss"));
    std::printf("write_phase_speeds flag : %d\n", (int)p.get_bool("write_phase_speeds"));
    std::printf("      write_speeds flag : %d\n", (int)p.get_bool("write_speeds"));
    std::printf("       write_modes flag : %d\n", (int)p.get_bool("write_modes"));
    std::printf("         multiprop flag : %d\n", (int)multiprop);
    std::printf("       turnoff_WKB flag : %d\n", (int)p.get_bool("turnoff_WKB"));
    std::printf("    atmospheric profile : %s\n", p.get_string("atmosfile").c_str());
    if (has("dispersion_file") && !p.get_string("dispersion_file").empty()) {
        std::printf("        dispersion file : %s\n", p.get_string("dispersion_file").c_str());
        std::printf(" Dispersion file append : %d\n", (int)p.get_bool("append_dispersion_file"));
    }
    if (!p.get_string("use_attn_file").empty())
        std::printf("  User attenuation file : %s\n", p.get_string("use_attn_file").c_str());
    if (!p.get_string("modal_starter_file").empty())
        std::printf(" modal starter saved in : %s\n", p.get_string("modal_starter_file").c_str());
    std::printf("       wvnum_filter_flg : %d\n", (int)p.get_bool("wvnum_filter"));
    if (p.get_bool("wvnum_filter")) {
        std::printf("                  c_min : %g m/s\n", p.get_float("c_min"));
        std::printf("                  c_max : %g m/s\n", p.get_float("c_max"));
    }
}

int ModalBroadbandPropagator::calculate_waveform() { return ncpa_cli::run_propagation(param_); }

}  // namespace ncpa_gpu_solvers
