// ModBB --propagation: dispersion file in, source spectrum, pulse synthesis on
// the GPU, waveform file out (ModalBroadbandPropagator.cpp:25-231,
// BroadbandPropagator.cpp:244-414).
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>

#include "cli_bb.hpp"
#include "cli_common.hpp"

namespace ncpa_cli {

namespace {

// number of '\n' characters (NCPA::count_rows_arbcol, util.cpp:269-285)
int count_newlines(const std::string& path) {
    std::FILE* f = std::fopen(path.c_str(), "r");
    if (!f) throw RunError("file << " + path + " could not be opened.");
    int n = 0, c;
    while ((c = std::getc(f)) != EOF)
        if (c == '\n') ++n;
    std::fclose(f);
    return n;
}

// ModalBroadbandPropagator::read_dispersion_file (ModalBroadbandPropagator.cpp:98-138)
// through the library reader, with its binary cache when cache is not empty
struct Dispersion {
    ncpa_dispersion* h = nullptr;
    ncpa_dispersion_desc d{};
    int rows = 0, from_cache = 0;
    Dispersion(const std::string& path, const std::string& cache) {
        std::FILE* fp = std::fopen(path.c_str(), "r");
        if (!fp) throw RunError("file << " + path + " could not be opened.");
        std::fclose(fp);
        std::printf("--> Opening dispersion file %s ...if the program chokes here the file may be corrupt.\n",
                    path.c_str());
        if (ncpa_dispersion_read(path.c_str(), cache.empty() ? nullptr : cache.c_str(), &h) != NCPA_OK)
            throw RunError(path + ": read_dispersion_data format error" +
                           (cache.empty() ? std::string() : " (or dispersion cache " + cache + " not writable)"));
        ncpa_dispersion_desc_get(h, &d, &rows, &from_cache);
        if (from_cache) std::printf("--> Parsed arrays taken from the dispersion cache %s\n", cache.c_str());
        std::printf("--> Found modes at %d positive frequencies in file %s\n", d.n_freq, path.c_str());
    }
    ~Dispersion() { ncpa_dispersion_destroy(h); }
    Dispersion(const Dispersion&) = delete;
    Dispersion& operator=(const Dispersion&) = delete;
};

// two-column (time, amplitude) or three-column (f, Re, Im) source files, read
// the way the reference's stream loops do (BroadbandPropagator.cpp:478-537):
// a last row not followed by whitespace is dropped
std::vector<std::vector<double>> read_columns(const std::string& path, int ncol) {
    std::ifstream in(path);
    if (!in) throw RunError("file " + path + " could not be opened.");
    std::vector<std::vector<double>> cols(ncol);
    std::vector<double> row(ncol);
    for (int c = 0; c < ncol; ++c) in >> row[c];
    while (!in.eof()) {
        for (int c = 0; c < ncol; ++c) cols[c].push_back(row[c]);
        for (int c = 0; c < ncol; ++c) in >> row[c];
        if (in.fail() && !in.eof()) throw RunError("file " + path + ": malformed row");
    }
    return cols;
}

}  // namespace

int run_propagation(const Params& prm) {
    const std::string src_type = prm.get_string("source");
    const std::string src_file = prm.get_string("source_file");
    const std::string out_file = prm.get_string("output_waveform_file");
    const double max_cel = prm.get_float("max_celerity");
    std::vector<double> ranges;
    if (prm.get_string("receiver") == "single") {
        ranges.push_back(prm.get_float("range_km") * 1000.0);
    } else {
        const double rmin = prm.get_float("start_range_km"), rmax = prm.get_float("end_range_km");
        const double rstep = prm.get_float("range_step_km");
        if (rmax <= rmin) throw RunError("end_range_km must be greater than start_range_km");
        if (!(rstep > 0.0)) throw RunError("range_step_km must be greater than 0");
        const int nr = (int)std::floor((rmax - rmin) / rstep) + 1;
        for (int i = 0; i < nr; ++i) ranges.push_back((rmin + (double)i * rstep) * 1000.0);
    }
    const std::string disp_path = prm.get_string("input_dispersion_file");
    const Dispersion disp(disp_path, prm.get_string("dispersion_cache"));
    const ncpa_dispersion_desc& dd = disp.d;
    const int rows = disp.rows;
    const double* freq = dd.f;
    const int nfreq = dd.n_freq;
    if (nfreq != rows + 1)
        std::printf("Warning: %d lines but %d frequencies in %s\n", rows, nfreq - 1, disp_path.c_str());
    if (nfreq < 3) throw RunError("the dispersion file needs at least two frequencies");
    const double f_step = freq[2] - freq[1];
    // NFFT rule (ModalBroadbandPropagator.cpp:66-84)
    int nfft = prm.get_int("nfft");
    if (nfft < 4 * nfreq) {
        nfft = 4 * nfreq;
        std::printf("Minimum NFFT is set to NFFT = %d\n", nfft);
    }
    if (src_type == "waveform") {
        const int lines = count_newlines(src_file);
        while (lines > nfft) {
            nfft *= 2;
            std::cout << "File " << src_file << " has " << lines << " lines, increasing NFFT to " << nfft << "\n";
        }
    }
    const double fmx = (double)nfft * f_step;

    ncpa_cli::Gpu gpu;
    ncpa_ctx* ctx = gpu.ctx();
    std::vector<double> s_re(nfreq, 0.0), s_im(nfreq, 0.0), pulse(nfft, 0.0);
    if (src_type == "impulse" || src_type == "pulse1" || src_type == "pulse2") {
        const int kind = src_type == "impulse" ? 0 : src_type == "pulse1" ? 1 : 2;
        ncpa_cli::check(ctx,
                        ncpa_source_spectrum_builtin(ctx, kind, freq, nfreq, prm.get_float("f_center"), nfft,
                                                     s_re.data(), s_im.data()),
                        "source spectrum");
    } else if (src_type == "spectrum") {
        std::cout << "Loading source spectrum from file " << src_file << std::endl;
        auto c = read_columns(src_file, 3);
        if ((int)c[0].size() > nfft) throw RunError("file " + src_file + " has more points than NFFT");
        if (c[0].empty() || std::fabs(c[0][0] - freq[0]) > 1.0e-8)
            throw RunError("The frequencies from the source spectrum file " + src_file +
                           " do not appear to match the ones from the provided dispersion file");
        for (int i = 0; i < nfreq && i < (int)c[0].size(); ++i) {
            s_re[i] = c[1][i];
            s_im[i] = c[2][i];
        }
    } else {  // waveform
        std::cout << "Loading time domain source pulse from file " << src_file << std::endl;
        auto c = read_columns(src_file, 2);
        if (c[0].size() < 2) throw RunError("file " + src_file + " needs at least two samples");
        const double dt = c[0][1] - c[0][0];
        for (size_t i = 0; i < c[1].size(); ++i) pulse[i] = c[1][i];
        ncpa_cli::check(ctx,
                        ncpa_source_spectrum_waveform(ctx, c[1].data(), (int)c[1].size(), dt, nfft, nfreq,
                                                      s_re.data(), s_im.data()),
                        "source spectrum of the waveform");
    }
    if (src_type != "waveform")  // f_step * FFT of the zero-padded spectrum, x2
        ncpa_cli::check(ctx, ncpa_source_waveform(ctx, freq, nfreq, s_re.data(), s_im.data(), nfft,
                                                  pulse.data()),
                        "source waveform");
    {
        std::FILE* f = std::fopen("source_waveform_input.dat", "w");
        if (!f) throw RunError("file source_waveform_input.dat could not be opened.");
        for (int i = 0; i < nfft / 2; ++i) std::fprintf(f, "%12.6f %15.6e\n", 1.0 * i / fmx, pulse[i]);
        std::fclose(f);
        std::cout << "--> Initial source waveform saved in file 'source_waveform_input.dat' " << std::endl
                  << " with format: | Time (s) | Amplitude |" << std::endl;
        f = std::fopen("source_spectrum_input.dat", "w");
        if (!f) throw RunError("file source_spectrum_input.dat could not be opened.");
        for (int i = 0; i < nfreq; ++i) std::fprintf(f, "%14.9f %15.6e %15.6e\n", freq[i], s_re[i], s_im[i]);
        std::fclose(f);
        std::cout << "--> The source spectrum is saved in file 'source_spectrum_input.dat' " << std::endl
                  << "with format: | Freq (Hz) | Re(S) | Imag(S) |" << std::endl;
    }

    ncpa_bb_params bp{};
    bp.n_ranges = (int)ranges.size();
    bp.ranges_m = ranges.data();
    bp.max_celerity = max_cel;
    bp.nfft = nfft;
    bp.src_re = s_re.data();
    bp.src_im = s_im.data();
    bp.zero_attn = prm.get_bool("use_zero_attenuation");
    std::vector<double> wave((size_t)ranges.size() * nfft);
    ncpa_cli::check(ctx, ncpa_bb_synthesize(ctx, &dd, &bp, wave.data()), "pulse synthesis");

    std::cout << "--> Propagating pulse from source-to-receivers on grid ..." << std::endl;
    std::printf("----------------------------------------------\n");
    std::printf("max_celerity     t0             R\n");
    std::printf("    m/s          sec            km\n");
    std::printf("----------------------------------------------\n");
    std::FILE* f = std::fopen(out_file.c_str(), "w");
    if (!f) throw RunError("file " + out_file + " could not be opened.");
    for (size_t n = 0; n < ranges.size(); ++n) {
        const double rr = ranges[n], t0 = rr / max_cel;
        std::printf("%8.3f     %9.3f      %9.3f\n", max_cel, t0, rr / 1000.0);
        const double* w = &wave[n * nfft];
        for (int i = 0; i < nfft; ++i) std::fprintf(f, "%10.3f %12.6f %15.6e\n", rr / 1000.0, 1.0 * i / fmx + t0, w[i]);
        std::fprintf(f, "\n");
    }
    std::fclose(f);
    std::printf("f_step = %f   1/f_step = %f\n", f_step, 1.0 / f_step);
    std::printf("Time array length = %d; delta_t = %g s\n", nfft, 1.0 / fmx);
    std::printf("Propagation results saved in file: %s\n", out_file.c_str());
    std::printf("with columns: R (km) | time (s) | pulse(R,t) |\n");
    return 0;
}

}  // namespace ncpa_cli
