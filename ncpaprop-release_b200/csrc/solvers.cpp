// The reference's solver classes over the GPU front-end code (solvers.hpp).
#include "solvers.hpp"

#include <cstdio>
#include <stdexcept>

#include "cli_bb.hpp"
#include "cli_ess.hpp"

namespace ncpa_gpu_solvers {

Atmosphere1D::Atmosphere1D(const std::string& file, const std::string& header)
    : s_(ncpa::to_si_profile(ncpa::read_profile(file, header))) {}

Atmosphere1D::Atmosphere1D(std::vector<double> z, std::vector<double> u, std::vector<double> v,
                           std::vector<double> t, std::vector<double> p, std::vector<double> rho) {
    const size_t n = z.size();
    if (n < 3 || u.size() != n || v.size() != n || t.size() != n || p.size() != n || rho.size() != n)
        throw std::invalid_argument("Atmosphere1D: need at least 3 knots and arrays of equal length");
    s_.z = std::move(z);
    s_.u = std::move(u);
    s_.v = std::move(v);
    s_.t = std::move(t);
    s_.p = std::move(p);
    s_.rho = std::move(rho);
}

bool Atmosphere1D::contains(const std::string& key) const {
    return key == "Z" || key == "U" || key == "V" || key == "T" || key == "P" || key == "RHO" ||
           (key == "C0" && s_.has_c0);
}

const std::vector<double>& Atmosphere1D::get(const std::string& key) const {
    if (key == "Z") return s_.z;
    if (key == "U") return s_.u;
    if (key == "V") return s_.v;
    if (key == "T") return s_.t;
    if (key == "P") return s_.p;
    if (key == "RHO") return s_.rho;
    if (key == "C0" && s_.has_c0) return s_.c0;
    throw std::out_of_range("Atmosphere1D: no property " + key);
}

std::vector<double>& Atmosphere1D::get(const std::string& key) {
    return const_cast<std::vector<double>&>(static_cast<const Atmosphere1D*>(this)->get(key));
}

void Atmosphere1D::set_z0(double z0_m) {
    s_.z0 = z0_m;
    s_.has_z0 = true;
}

ncpa_profile_desc Atmosphere1D::desc() const {
    const size_t n = s_.z.size();
    for (const auto* a : {&s_.u, &s_.v, &s_.t, &s_.p, &s_.rho})
        if (a->size() != n) throw std::invalid_argument("Atmosphere1D: property arrays changed length");
    if (s_.has_c0 && s_.c0.size() != n) throw std::invalid_argument("Atmosphere1D: property arrays changed length");
    ncpa_profile_desc d{};
    d.n_knots = (int)n;
    d.z = s_.z.data();
    d.u = s_.u.data();
    d.v = s_.v.data();
    d.t = s_.t.data();
    d.p = s_.p.data();
    d.rho = s_.rho.data();
    d.c0 = s_.has_c0 ? s_.c0.data() : nullptr;
    d.attn = nullptr;
    d.z0_m = s_.z0;
    d.has_z0 = s_.has_z0;
    return d;
}

void Atmosphere1D::write(const std::string& path) const {
    ncpa::ParsedProfile pp;
    pp.z = s_.z;
    pp.z_units = "m";
    std::vector<std::string> keys = {"U", "V", "T", "P", "RHO"};
    const char* units[] = {"m/s", "m/s", "K", "Pa", "kg/m3"};
    for (size_t i = 0; i < keys.size(); ++i) {
        pp.vectors[keys[i]] = get(keys[i]);
        pp.vector_units[keys[i]] = units[i];
    }
    if (s_.has_c0) {
        keys.push_back("C0");
        pp.vectors["C0"] = s_.c0;
        pp.vector_units["C0"] = "m/s";
    }
    if (s_.has_z0) {
        pp.scalars["Z0"] = s_.z0;
        pp.scalar_units["Z0"] = "m";
    }
    ncpa::write_ncpa_profile(pp, keys, path);
}

int ESSModeSolver::solve() {
    if (atm_) {
        const ncpa_profile_desc d = atm_->desc();
        ncpa_cli::run_ess(param_, false, &d);
    } else {
        ncpa_cli::run_ess(param_, false);
    }
    return 0;
}

int WModeSolver::solve() {
    if (atm_) {
        const ncpa_profile_desc d = atm_->desc();
        ncpa_cli::run_ess(param_, true, &d);
    } else {
        ncpa_cli::run_ess(param_, true);
    }
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
