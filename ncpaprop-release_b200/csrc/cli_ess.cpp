// The ESS solve loop shared by Modess and ModBB --dispersion: the option
// handling of ESSModeSolver::setParams (ESSModeSolver.cpp:30-240) and the
// per-(frequency, azimuth) outputs of ESSModeSolver::solve
// (ESSModeSolver.cpp:291-510), with every problem of a frequency batch solved
// in one ncpa_ess_solve call on the GPU.  ModBB --method wmod runs the same
// loop with the wide-angle solve (WModeSolver::setParams / solve,
// WModeSolver.cpp:30-120, 257-486: the same options and outputs, without
// group speeds).
#include <cmath>
#include <cstdio>
#include <iostream>
#include <memory>

#include "cli_common.hpp"
#include "cli_ess.hpp"

namespace ncpa_cli {

namespace {
struct ModesHandle {
    ncpa_modes* m = nullptr;
    ~ModesHandle() {
        if (m) ncpa_modes_destroy(m);
    }
};
struct ProfileHandle {
    ncpa_profile* p = nullptr;
    ~ProfileHandle() {
        if (p) ncpa_profile_destroy(p);
    }
};
}  // namespace

void run_ess(const Params& prm, bool wmod, const ncpa_profile_desc* atm) {
    const std::string tag = prm.get_string("filetag");
    const std::string gnd = prm.get_string("ground_impedence_model");
    if (gnd != "rigid") throw RunError("This ground impedance model is not implemented yet: " + gnd);

    ncpa_ess_params ep;
    ncpa_ess_params_default(&ep);
    ep.method = wmod ? NCPA_METHOD_WMOD : NCPA_METHOD_ESS;
    ep.nz_grid = prm.get_int("Nz_grid");
    ep.maxheight_km = prm.get_float("maxheight_km");
    ep.zground_km = prm.get_float("zground_km");
    ep.sourceheight_km = prm.get_float("sourceheight_km");
    ep.receiverheight_km = prm.get_float("receiverheight_km");
    ep.lamb_wave_bc = prm.get_bool("Lamb_wave_BC");
    const bool write_2d = prm.get_bool("write_2d_tloss");
    const bool write_lossless = prm.get_bool("write_lossless");
    const bool write_phase = prm.get_bool("write_phase_speeds");
    const bool want_speeds = !wmod && prm.get_bool("write_speeds");
    const bool write_modes = prm.get_bool("write_modes");
    const bool write_atm = prm.get_bool("write_atm_profile");
    const bool multiprop = prm.get_bool("multiprop");
    const std::string disp_file = prm.get_string("dispersion_file");
    const bool append_disp = prm.get_bool("append_dispersion_file");
    const std::string starter_file = prm.get_string("modal_starter_file");
    ep.turnoff_wkb = prm.get_bool("turnoff_WKB");
    // ESSModeSolver.cpp:78-81 (WModeSolver.cpp:75-77): any of these outputs
    // turns the WKB estimate off
    if (write_phase || want_speeds || write_2d || write_modes || !disp_file.empty()) ep.turnoff_wkb = 1;
    ep.wvnum_filter = prm.get_bool("wvnum_filter");
    if (ep.wvnum_filter) {
        ep.c_min = prm.get_float("c_min");
        ep.c_max = prm.get_float("c_max");
    }
    const bool single = !multiprop;
    ep.want_group_speed = !wmod && single && (want_speeds || write_modes);
    ep.want_vectors = single && (write_modes || write_2d || !starter_file.empty());

    // azimuths (ESSModeSolver.cpp:83-95)
    std::vector<double> az;
    if (multiprop) {
        const double a0 = prm.get_float("azimuth_start"), a1 = prm.get_float("azimuth_end");
        const double step = prm.get_float("azimuth_step");
        if (!(step > 0.0)) throw RunError("azimuth_step must be greater than 0 for --multiprop");
        const int naz = (int)((a1 - a0) / step) + 1;
        if (naz < 1) throw RunError("azimuth_end must not be below azimuth_start");
        for (int i = 0; i < naz; ++i) az.push_back(a0 + i * step);
    } else {
        az.push_back(prm.get_float("azimuth"));
    }
    // frequencies (ESSModeSolver.cpp:98-120)
    std::vector<double> freqs;
    if (prm.get_bool("broadband")) {
        const double f_min = prm.get_float("f_min"), f_step = prm.get_float("f_step"),
                     f_max = prm.get_float("f_max");
        if (f_min >= f_max) throw RunError("f_min must be less than f_max!");
        if (!(f_step > 0.0)) throw RunError("f_step must be greater than 0");
        const int nf = (int)std::floor((f_max - f_min) / f_step) + 1;
        for (int i = 0; i < nf; ++i) freqs.push_back(f_min + (double)i * f_step);
    } else {
        freqs.push_back(prm.get_float("freq"));
    }

    const double maxrange = prm.get_float("maxrange_km") * 1000.0;
    const int nr = prm.get_int("Nrng_steps");
    const double dr = maxrange / nr;

    Gpu gpu;
    ncpa_ctx* ctx = gpu.ctx();
    ProfileHandle prof;
    prof.p = atm ? create_profile(ctx, atm, prm.get_string("use_attn_file"))
                 : load_profile(ctx, prm.get_string("atmosfile"), prm.get_string("atmosheaderfile"),
                                prm.get_string("use_attn_file"));

    // batches of frequencies: one frequency at a time when full eigenvectors
    // are kept, else up to 4096 problems per solve
    const int na = (int)az.size();
    const int per_batch = ep.want_vectors ? 1 : std::max(1, 4096 / na);
    const std::string f1d = tag_filename(tag, multiprop ? "Nby2D_tloss_1d.nm" : "tloss_1d.nm");
    const std::string f1d_ll = tag_filename(tag, multiprop ? "Nby2D_tloss_1d.lossless.nm" : "tloss_1d.lossless.nm");
    for (size_t f0 = 0; f0 < freqs.size(); f0 += per_batch) {
        const int nf = (int)std::min<size_t>(per_batch, freqs.size() - f0);
        ModesHandle mh;
        check(ctx, ncpa_ess_solve(ctx, prof.p, &ep, &freqs[f0], nf, az.data(), na, &mh.m),
              wmod ? "wide-angle mode solve" : "ESS mode solve");
        const int P = nf * na;
        ncpa_tl_params tp{nr, dr, 0};
        std::vector<double> re((size_t)P * nr), im((size_t)P * nr), inc((size_t)P * nr);
        std::vector<double> re_ll, im_ll, inc_ll;
        check(ctx, ncpa_tl_1d(ctx, mh.m, &tp, re.data(), im.data(), inc.data()), "1-D transmission loss");
        if (write_lossless) {
            tp.lossless = 1;
            re_ll.resize(re.size());
            im_ll.resize(re.size());
            inc_ll.resize(re.size());
            check(ctx, ncpa_tl_1d(ctx, mh.m, &tp, re_ll.data(), im_ll.data(), inc_ll.data()), "lossless 1-D TL");
            tp.lossless = 0;
        }
        for (int fi = 0; fi < nf; ++fi) {
            for (int it = 0; it < na; ++it) {
                const int p = fi * na + it;
                const Modes m = get_modes(ctx, mh.m, p);
                const size_t o = (size_t)p * nr;
                std::cout << "\nNow processing azimuth = " << az[it] << " (" << it + 1 << " of " << na << ")\n";
                std::printf("______________________________________________________________________\n\n");
                std::printf(" -> Normal mode solution at %5.3f Hz and %5.2f deg (%d modes)...\n", m.freq, m.az, m.M);
                if (multiprop) {
                    write_tloss_nx2(f1d, it != 0, m.az, nr, dr, &re[o], &im[o], &inc[o]);
                    if (write_lossless) write_tloss_nx2(f1d_ll, it != 0, m.az, nr, dr, &re_ll[o], &im_ll[o], &inc_ll[o]);
                    continue;
                }
                std::printf("Writing to file: 1D transmission loss\n");
                write_tloss_1d(f1d, nr, dr, &re[o], &im[o], &inc[o]);
                if (write_lossless) write_tloss_1d(f1d_ll, nr, dr, &re_ll[o], &im_ll[o], &inc_ll[o]);
                if (!starter_file.empty()) {
                    int ns = 0;
                    check(ctx, ncpa_modal_starter(ctx, mh.m, p, &ns, nullptr, nullptr, nullptr), "modal starter");
                    std::vector<double> z(ns), sr(ns), si(ns);
                    check(ctx, ncpa_modal_starter(ctx, mh.m, p, &ns, z.data(), sr.data(), si.data()),
                          "modal starter");
                    write_starter(tag_filename(tag, starter_file), ns, z.data(), sr.data(), si.data());
                }
                if (write_2d) {
                    int nzo = 0;
                    check(ctx, ncpa_tl_2d_heights(mh.m, p, &nzo), "2-D TL heights");
                    std::vector<double> z(nzo), r2((size_t)nr * nzo), i2((size_t)nr * nzo);
                    check(ctx, ncpa_tl_2d(ctx, mh.m, p, &tp, z.data(), r2.data(), i2.data()), "2-D TL");
                    write_tloss_2d(tag_filename(tag, "tloss_2d.nm"), nr, dr, nzo, z.data(), r2.data(), i2.data());
                    if (write_lossless) {
                        tp.lossless = 1;
                        check(ctx, ncpa_tl_2d(ctx, mh.m, p, &tp, z.data(), r2.data(), i2.data()), "2-D TL");
                        tp.lossless = 0;
                        write_tloss_2d(tag_filename(tag, "tloss_2d.lossless.nm"), nr, dr, nzo, z.data(), r2.data(),
                                       i2.data());
                    }
                }
                if (write_phase) write_phase_speeds(tag_filename(tag, "phasespeeds.nm"), m);
                if (write_modes) {
                    std::vector<double> v((size_t)m.M * ep.nz_grid);
                    if (m.M) check(ctx, ncpa_modes_get_vectors(mh.m, p, v.data()), "eigenvectors");
                    write_mode_files(tag, ep.nz_grid, m.dz, m.M, v);
                }
                if (!wmod && (write_modes || want_speeds)) write_speeds(tag_filename(tag, "speeds.nm"), m);
                if (!disp_file.empty()) {
                    std::printf("Writing to file %s: dispersion at freq = %8.3f Hz...\n", disp_file.c_str(), m.freq);
                    std::FILE* df = std::fopen(disp_file.c_str(), append_disp ? "a" : "w");
                    if (!df) throw RunError("file " + disp_file + " could not be opened.");
                    append_dispersion_line(df, m);
                    std::fclose(df);
                }
                if (write_atm && f0 + fi == 0) write_atm_profile(tag_filename(tag, "atm_profile.nm"), prof.p, m.az);
            }
        }
    }
}

void configure_modess(Params& ps) {
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

}  // namespace ncpa_cli
