/*
 * ncpa_gpu.h -- C ABI of the B200 effective-sound-speed normal-mode library
 * (Modess / ModBB hot path of ncpaprop).
 *
 * Plain C types only: status codes are returned (never thrown), the library
 * owns device memory, the caller owns every host buffer it passes.  One
 * context per host thread; a context owns one CUDA stream on one device.
 *
 * The reference exposes this path as C++ virtual classes (no C ABI); each
 * entry point below names the reference interface whose work it replaces.
 */
#ifndef NCPA_GPU_H
#define NCPA_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    NCPA_OK = 0,
    NCPA_EINVAL = 1,    /* bad argument (message via ncpa_last_error) */
    NCPA_ENOMEM = 2,    /* device or host allocation failed */
    NCPA_ECUDA = 3,     /* CUDA runtime error */
    NCPA_EPARSE = 4,    /* malformed profile / dispersion / source file */
    NCPA_ETOOMANY = 5,  /* more modes than ncpa_ess_params.max_modes */
    NCPA_EIO = 6,       /* file could not be opened */
    NCPA_ETIMEDOUT = 7, /* a bounded device wait gave up */
    NCPA_ENODEV = 8     /* no CUDA device or the kernels are missing */
} ncpa_status;

typedef struct ncpa_ctx ncpa_ctx;
typedef struct ncpa_profile ncpa_profile;
typedef struct ncpa_modes ncpa_modes;

typedef struct {
    int device; /* CUDA device ordinal */
} ncpa_ctx_opts;

/* Context: device, stream, last-error text. */
ncpa_status ncpa_ctx_create(ncpa_ctx **ctx, const ncpa_ctx_opts *opts);
ncpa_status ncpa_ctx_destroy(ncpa_ctx *ctx);
const char *ncpa_status_str(ncpa_status s);
const char *ncpa_last_error(const ncpa_ctx *ctx);
ncpa_status ncpa_ctx_synchronize(ncpa_ctx *ctx);

/* ------------------------------------------------------------------------
 * Atmospheric profile (replaces NCPA::Atmosphere1D(file, header),
 * src/atmosphere/Atmosphere1D.cpp:44-60, 85-285, plus the derived
 * properties ESSModeSolver::setParams adds, ESSModeSolver.cpp:159-228).
 * Knot arrays are SI: z [m], u v [m/s], t [K], p [Pa], rho [kg/m^3],
 * c0 [m/s] (optional), attn [Np/m] (optional user attenuation at the knots,
 * replaces --use_attn_file).  The profile is resident in HBM until destroyed.
 * ---------------------------------------------------------------------- */
typedef struct {
    int n_knots;
    const double *z, *u, *v, *t, *p, *rho;
    const double *c0;   /* NULL: computed from p and rho as the reference does */
    const double *attn; /* NULL: Sutherland-Bass at each solve frequency */
    double z0_m;        /* ground height scalar Z0 of the profile file */
    int has_z0;
} ncpa_profile_desc;

ncpa_status ncpa_profile_create(ncpa_ctx *ctx, const ncpa_profile_desc *desc, ncpa_profile **out);
/* Parse an NCPA profile file ("#% col, KEY, units[, value]" header, optional
 * separate header file) and upload it. */
ncpa_status ncpa_profile_load(ncpa_ctx *ctx, const char *path, const char *header_path,
                              ncpa_profile **out);
ncpa_status ncpa_profile_destroy(ncpa_profile *prof);
/* G2S-style profiles (the layout of the reference's samples/g2sprofile.sample,
 * which its Atmosphere1D reader cannot take as it is): an optional first line
 * "Profile at (lat, lon)", '#' comments, then rows of Z [km], T [K], U, V
 * [m/s], P [mbar], RHO [g/cm3].  ncpa_g2s_convert writes the equivalent NCPA
 * profile file ("#%" header + columns; host only, no device needed) and
 * returns the location (NaN without a location line; NULL to skip);
 * ncpa_profile_load_g2s reads it straight into a device profile. */
ncpa_status ncpa_g2s_convert(const char *g2s_path, const char *ncpa_path, double *lat, double *lon);
ncpa_status ncpa_profile_load_g2s(ncpa_ctx *ctx, const char *path, ncpa_profile **out);
/* User attenuation table (height km, Np/m), interpolated onto the profile
 * knots and used at every frequency instead of Sutherland-Bass (replaces
 * Atmosphere1D::read_attenuation_from_file, Atmosphere1D.cpp:307-424). */
ncpa_status ncpa_profile_set_attn(ncpa_profile *prof, const double *z_km, const double *attn, int n);
/* same, from a two-column text file "height_km  attenuation_Np/m" */
ncpa_status ncpa_profile_load_attn(ncpa_profile *prof, const char *path);
/* Knot columns in SI units (z [m], u, v [m/s], t [K], p [Pa], rho [kg/m^3]),
 * the static sound speed c0 and the effective sound speed for one azimuth at
 * the knots -- the columns of atm_profile.nm (ESSModeSolver.cpp:468-484,
 * Atmosphere1D::print_atmosphere, Atmosphere1D.cpp:924-970); any output
 * pointer may be NULL. */
ncpa_status ncpa_profile_knots(ncpa_profile *prof, double az_deg, double *z, double *u, double *v,
                               double *t, double *p, double *rho, double *c0, double *ceff);
/* ground height scalar Z0 [m] of the profile, if it has one */
ncpa_status ncpa_profile_z0(const ncpa_profile *prof, double *z0_m, int *has_z0);
/* Number of knots and the altitude range [m] of a loaded profile. */
ncpa_status ncpa_profile_info(const ncpa_profile *prof, int *n_knots, double *z_lo, double *z_hi);

/* ------------------------------------------------------------------------
 * Batched ESS eigen-solve over (frequency x azimuth) problems
 * (replaces ESSModeSolver::solve loop body: getModalTrace, getNumberOfModes,
 * EigenEngine::doESSCalculation, doSelect, doPerturb -- ESSModeSolver.cpp:
 * 320-383, 518-665; EigenEngine.cpp:10-172; ModeSolver.cpp:223-284).
 * Problem index p = f_index * n_az + az_index.
 * ---------------------------------------------------------------------- */
typedef struct {
    int nz_grid;              /* --Nz_grid            [20000] */
    double maxheight_km;      /* --maxheight_km       [150]   */
    double zground_km;        /* --zground_km         [0]     */
    double sourceheight_km;   /* --sourceheight_km    [0]     */
    double receiverheight_km; /* --receiverheight_km  [0]     */
    int lamb_wave_bc;         /* --Lamb_wave_BC               */
    int turnoff_wkb;          /* --turnoff_WKB (or implied by write flags) */
    int wvnum_filter;         /* --wvnum_filter with c_min, c_max [m/s] */
    double c_min, c_max;
    int want_group_speed;     /* compute group speeds (speeds.nm) */
    int want_vectors;         /* keep full eigenvectors (modes, 2-D TL, starter) */
    int max_modes;            /* per problem; 0 -> 4000 (reference MAX_MODES) */
    int keep_on_device;       /* leave mode arrays in HBM only (ncpa_modes_get
                                 then fetches them on demand) */
    int method;               /* NCPA_METHOD_ESS (Modess) or NCPA_METHOD_WMOD */
} ncpa_ess_params;

/* NCPA_METHOD_WMOD: the wide-angle modes of WModeSolver (ModBB --method wmod,
 * WModeSolver.cpp:257-629): the quadratic eigenproblem
 * (M k^2 + C k + D) v = 0 with M = (w/c0)^2 - 1, C = -2 omega w / c0^2 (w the
 * wind component along the azimuth), D the finite-difference operator with
 * (omega/c0)^2, solved in k by Sturm counts of T(k) = M k^2 + C k + D, plus
 * the reference's matrix spacing (maxheight - z_min) / Nz_grid.  Available
 * through ncpa_ess_solve and ncpa_ess_solve_jobs (so also in the serving
 * loop); plans take the ESS method only.  Group speeds are 0. */
enum { NCPA_METHOD_ESS = 0, NCPA_METHOD_WMOD = 1 };

void ncpa_ess_params_default(ncpa_ess_params *p);

ncpa_status ncpa_ess_solve(ncpa_ctx *ctx, const ncpa_profile *prof, const ncpa_ess_params *params,
                           const double *freqs, int n_freq, const double *az_deg, int n_az,
                           ncpa_modes **out);
/* Batched solve over independent jobs, each with its own profile, frequency
 * list, azimuth(s) and solver grid size, in one pass of the eigen-solve
 * kernels (the request batch of the serving loop, and sweeps whose grid
 * follows the wavelength; the reference solves one (profile, frequency,
 * azimuth) at a time in ESSModeSolver::solve, ESSModeSolver.cpp:320-383).
 * Each job's grid comes from its profile and nz_grid (0: params->nz_grid)
 * with the other params; problems are numbered job by job, frequency-major
 * then azimuth inside a job.  The result behaves like a one-azimuth solve of
 * sum(n_freq * n_az) problems; ncpa_modes_info reports each problem's own
 * grid spacing and densities. */
typedef struct {
    const ncpa_profile *profile;
    const double *freqs;
    int n_freq;
    double az_deg;            /* the job's azimuth when n_az == 0 */
    int nz_grid;              /* grid points of this job; 0 -> params->nz_grid */
    int n_az;                 /* > 0: the job sweeps az_list[0 .. n_az-1] */
    const double *az_list;
} ncpa_ess_job;
ncpa_status ncpa_ess_solve_jobs(ncpa_ctx *ctx, const ncpa_ess_job *jobs, int n_jobs,
                                const ncpa_ess_params *params, ncpa_modes **out);
ncpa_status ncpa_modes_destroy(ncpa_modes *modes);
ncpa_status ncpa_modes_problems(const ncpa_modes *modes, int *n_problems);
ncpa_status ncpa_modes_count(const ncpa_modes *modes, int problem, int *n_modes);
/* scalars of one problem: grid spacing dz [m], window, densities at the
 * source / receiver grid points, grid indices of source / receiver */
ncpa_status ncpa_modes_info(const ncpa_modes *modes, int problem, double *freq, double *az,
                            double *dz, double *k_min, double *k_max, double *rho_src,
                            double *rho_rcv);
/* modes of one problem in ascending Re k: k_pert = re_k + i im_k, mode values
 * at source and receiver (normalised so sum v^2 dz = 1), group speed [m/s]
 * (NULL to skip; zero unless want_group_speed). */
ncpa_status ncpa_modes_get(const ncpa_modes *modes, int problem, double *re_k, double *im_k,
                           double *v_src, double *v_rcv, double *v_group);
/* all problems at once, in CSR order: mode_off[n_problems + 1] offsets, the
 * arrays hold mode_off[n_problems] entries (NULL to skip; copied straight
 * from HBM) */
ncpa_status ncpa_modes_get_all(const ncpa_modes *modes, int *mode_off, double *re_k, double *im_k,
                               double *v_src, double *v_rcv, double *v_group);
/* full eigenvectors of one problem, layout [z_index * M + mode]
 * (needs want_vectors) */
ncpa_status ncpa_modes_get_vectors(const ncpa_modes *modes, int problem, double *v);

/* ------------------------------------------------------------------------
 * Transmission loss modal sums (ModeSolver::getTLoss1D / getTLoss1DNx2 /
 * getTLoss2D, ModeSolver.cpp:292-565).  Ranges are (i+1)*dr_m, i < n_ranges.
 * Outputs carry the reference's 1000 * 4 pi scaling (levels re 1 m).
 * ---------------------------------------------------------------------- */
typedef struct {
    int n_ranges;
    double dr_m;
    int lossless; /* use Re k only (tloss_*.lossless.nm) */
} ncpa_tl_params;

/* all problems at once: re/im/incoh are [n_problems x n_ranges]; pass all
 * three as NULL to keep the result in HBM (owned by the modes object) */
ncpa_status ncpa_tl_1d(ncpa_ctx *ctx, const ncpa_modes *modes, const ncpa_tl_params *tp,
                       double *re, double *im, double *incoh);
/* 1-D TL of problems first .. first + count - 1 only; re/im/incoh are
 * [count x n_ranges] host arrays (ModeSolver::getTLoss1D, ModeSolver.cpp:
 * 292-381, for a slice of a batch: each served request its own range grid) */
ncpa_status ncpa_tl_1d_range(ncpa_ctx *ctx, const ncpa_modes *modes, int first, int count,
                             const ncpa_tl_params *tp, double *re, double *im, double *incoh);
/* A modes object from host arrays (no counterpart in the reference): n
 * problems with CSR offsets mode_off[n + 1] (mode_off[0] = 0) into k = re_k +
 * i im_k and the mode values at the source and receiver.  The arrays are
 * uploaded and stay in HBM with the object; it serves ncpa_tl_1d /
 * ncpa_tl_1d_range / ncpa_modes_get / ncpa_modes_get_all (no grid, vectors
 * or group speeds: ncpa_modes_info reports zeros and unit densities). */
ncpa_status ncpa_modes_from_host(ncpa_ctx *ctx, int n_problems, const int *mode_off, const double *re_k,
                                 const double *im_k, const double *v_src, const double *v_rcv, ncpa_modes **out);
/* one problem on the reference's height sampling (every nz/500-th grid
 * point); heights [m] in z_out (n_heights entries), re/im [n_ranges x n_heights].
 * The sum runs in FP64 on the CUDA cores, or on the guarded tcgen05 sum
 * (NCPA_SUM_TC_GUARDED, within 0.05 dB wherever TL > -140 dB) in a context
 * created with NCPA_TL2D_SUM=3 in the environment. */
ncpa_status ncpa_tl_2d_heights(const ncpa_modes *modes, int problem, int *n_heights);
ncpa_status ncpa_tl_2d(ncpa_ctx *ctx, const ncpa_modes *modes, int problem, const ncpa_tl_params *tp,
                       double *z_out, double *re, double *im);

/* Modal sum at many receivers (ModeSolver::getTLoss2D's contraction,
 * ModeSolver.cpp:492-565, at arbitrary receiver heights): re/im are
 * [n_rcv x n_ranges], receiver j at grid point ceil(rcv_height_m[j] / dz),
 * ranges (i+1)*dr_m, with the 1000 * 4 pi scaling of the 1-D TL.  Needs
 * want_vectors.  NULL re and im keep the result in HBM.
 *   NCPA_SUM_FP64        FP64 sum on the CUDA cores (at most 1024 receivers)
 *   NCPA_SUM_TC_BF16X3   tcgen05 tensor cores: 3-term split-BF16 products with
 *                        FP32 accumulation; phases k r reduced mod 2 pi in
 *                        FP64 per 256-range tile (relative error ~1e-5 of
 *                        the modal terms' magnitude)
 *   NCPA_SUM_TC_TF32     tcgen05 tensor cores: TF32 products (operands
 *                        rounded to nearest) with FP32 accumulation, same
 *                        phase reduction (relative error ~1e-3)
 *   NCPA_SUM_TC_GUARDED  tcgen05 tensor cores, 6-term split-BF16 (operands
 *                        split into three bf16 parts, FP32-level products)
 *                        with an error guard: every point whose |P| is below
 *                        the bound that keeps its TL within 0.05 dB is
 *                        recomputed in FP64 on the CUDA cores, so TL agrees
 *                        with the FP64 sum within 0.05 dB everywhere.
 * BF16X3 and TF32 carry the stated relative errors only: in cancellation
 * nulls (|P| far below the modal terms' magnitude) their TL error grows
 * beyond 0.05 dB; use FP64 or GUARDED where every point must hold it. */
enum { NCPA_SUM_FP64 = 0, NCPA_SUM_TC_BF16X3 = 1, NCPA_SUM_TC_TF32 = 2, NCPA_SUM_TC_GUARDED = 3 };
ncpa_status ncpa_tl_multi(ncpa_ctx *ctx, const ncpa_modes *modes, int problem, int n_rcv,
                          const double *rcv_height_m, const ncpa_tl_params *tp, int method, double *re,
                          double *im);

/* Modal starter of one problem (ESSModeSolver::getModalStarter,
 * ESSModeSolver.cpp:670-723; needs want_vectors).  Call with NULL outputs to
 * get the number of heights in *n_out. */
ncpa_status ncpa_modal_starter(ncpa_ctx *ctx, const ncpa_modes *modes, int problem, int *n_out,
                               double *z_km, double *re, double *im);

/* ------------------------------------------------------------------------
 * ModBB pulse synthesis (ModalBroadbandPropagator::calculate_waveform and
 * BroadbandPropagator::fft_pulse_prop, ModalBroadbandPropagator.cpp:141-277,
 * BroadbandPropagator.cpp:573-662).
 * Dispersion arrays: n_freq entries of f (f[0] = 0, the DC slot),
 * mode_off[n_freq+1] CSR offsets into re_k/im_k/v_src/v_rcv.
 * ---------------------------------------------------------------------- */
typedef struct {
    int n_freq;
    const double *f;
    const int *mode_off;
    const double *re_k, *im_k, *v_src, *v_rcv;
    double rho_src, rho_rcv;
} ncpa_dispersion_desc;

typedef struct {
    int n_ranges;
    const double *ranges_m;
    double max_celerity;  /* t0 = r / max_celerity */
    int nfft;
    const double *src_re; /* source spectrum at the n_freq dispersion bins */
    const double *src_im;
    int zero_attn;        /* set Im k = 0 */
} ncpa_bb_params;

/* waveforms: [n_ranges x nfft], 2 Re p(t) at t = i/(nfft df) + t0; NULL
 * waveforms keeps the result in HBM */
/* Dispersion file of ModBB --dispersion on the host, read as
 * ModalBroadbandPropagator::read_dispersion_file does
 * (ModalBroadbandPropagator.cpp:98-138: "f M rho_src rho_rcv" then M
 * quadruples per line, at most 4000 modes, reading stops at the first
 * non-number, the DC slot f = 0 first).  With cache_path, a binary copy of
 * the parsed arrays stamped with the text file (size, modification time,
 * FNV-1a hash) is used when it matches, and written when it does not, so
 * repeated propagation runs skip the text parsing.  NCPA_EPARSE for a
 * malformed or missing text file; the arrays stay valid until destroy. */
typedef struct ncpa_dispersion ncpa_dispersion;
ncpa_status ncpa_dispersion_read(const char *text_path, const char *cache_path, ncpa_dispersion **out);
/* desc points into the set; text_rows = newline characters of the text
 * file; from_cache = 1 when the binary cache was used */
ncpa_status ncpa_dispersion_desc_get(const ncpa_dispersion *disp, ncpa_dispersion_desc *desc, int *text_rows,
                                     int *from_cache);
ncpa_status ncpa_dispersion_destroy(ncpa_dispersion *disp);

ncpa_status ncpa_bb_synthesize(ncpa_ctx *ctx, const ncpa_dispersion_desc *disp,
                               const ncpa_bb_params *bp, double *waveforms);
/* same, taking the dispersion of a device-resident batched solve (one
 * azimuth; frequencies must be uniformly spaced from df): no host round trip */
ncpa_status ncpa_bb_synthesize_modes(ncpa_ctx *ctx, const ncpa_modes *modes, int az_index,
                                     const ncpa_bb_params *bp, double *waveforms);
/* built-in source spectra at the n_freq dispersion bins f (f[0] = 0):
 * kind 0 impulse, 1 pulse1, 2 pulse2 (BroadbandPropagator::get_source_spectrum,
 * BroadbandPropagator.cpp:260-311, pulse_spec_fit :420-438, model_pulse_fft
 * :440-476); f_center < 0 selects f_max/5 */
ncpa_status ncpa_source_spectrum_builtin(ncpa_ctx *ctx, int kind, const double *f, int n_freq,
                                         double f_center, int nfft, double *s_re, double *s_im);
/* time series of a source spectrum: 2 Re( df sum_n S_n exp(-2 pi i k n / nfft) ),
 * k < nfft (the source_waveform_input.dat of BroadbandPropagator.cpp:360-404) */
ncpa_status ncpa_source_waveform(ncpa_ctx *ctx, const double *f, int n_freq, const double *s_re,
                                 const double *s_im, int nfft, double *out);
/* source spectrum of a sampled waveform: sum_n x_n exp(+2 pi i k n / nfft) dt
 * for k < n_freq (BroadbandPropagator.cpp:327-353) */
ncpa_status ncpa_source_spectrum_waveform(ncpa_ctx *ctx, const double *x, int n_samples, double dt,
                                          int nfft, int n_freq, double *s_re, double *s_im);

/* ------------------------------------------------------------------------
 * Serving loop (no counterpart in the reference, which runs one solve per
 * process): requests of different sizes (profile, frequency or band,
 * azimuth) arrive at any time; worker lanes, each with its own stream, take
 * every queued request that fits (problem count, HBM footprint) into one
 * batched solve (ncpa_ess_solve_jobs) plus 1-D TL, so requests that arrive
 * while others run are admitted as lanes and memory free up and their work
 * overlaps on the device.  Results stay with the server until released.
 * ---------------------------------------------------------------------- */
typedef struct ncpa_server ncpa_server;
typedef struct {
    int device;
    ncpa_ess_params params;  /* shared by every request (grid, heights, flags) */
    int n_ranges;            /* default 1-D TL range grid of a request: (i+1)*dr_m */
    double dr_m;
    int lanes;               /* batches in flight at once; 0 -> 2 */
    int max_batch_problems;  /* problems merged into one solve; 0 -> 1024 */
    double hbm_budget_bytes; /* admission limit on in-flight requests' estimated
                                device footprint plus the mode cache; 0 -> 8 GiB.
                                One request is always admitted when nothing else
                                runs. */
    double cache_bytes;      /* device-resident mode cache (0: none).  A request
                                whose profile (knot values), frequencies and
                                azimuth match a solved one skips the eigen-solve:
                                its modes stay in HBM, keyed by a hash of the
                                profile, the frequencies and the azimuth; least
                                recently used entries are evicted. */
} ncpa_server_opts;

typedef struct {
    ncpa_profile_desc profile; /* host knot arrays (SI); copied at submit */
    const double *freqs;
    int n_freq;
    double az_deg;
    int n_ranges;              /* this request's 1-D TL grid (i+1)*dr_m; 0 -> the server's */
    double dr_m;
    int n_wave_ranges;         /* > 0: pulse waveforms at wave_ranges_m (broadband
                                  requests; frequencies k df, k = 1..n_freq) */
    const double *wave_ranges_m;
    double max_celerity;       /* t0 = r / max_celerity; 0 -> 340 m/s */
    int nfft;                  /* 0 -> the NFFT rule: 4 (n_freq + 1) */
    int source;                /* built-in source spectrum: 0 impulse, 1 pulse1, 2 pulse2 */
} ncpa_request;

typedef struct {
    int status;                /* ncpa_status of this request */
    int n_freq;
    const int *mode_off;       /* [n_freq + 1] offsets into the mode arrays */
    const double *re_k, *im_k, *v_src, *v_rcv;
    const double *tl_re, *tl_im, *tl_incoh; /* [n_freq x n_ranges] */
    double latency_ms;         /* submit -> results ready */
    int batch_requests;        /* requests in the batch it was solved in */
    int n_ranges;              /* the TL grid's length */
    int n_wave_ranges, nfft;
    const double *waveforms;   /* [n_wave_ranges x nfft] (ncpa_bb_synthesize's
                                  layout), NULL without waveforms */
    int from_cache;            /* 1: modes from the cache, no eigen-solve */
} ncpa_result;

typedef struct {
    long long submitted, completed, batches;
    double mean_batch_requests;
    double p50_ms, p99_ms, max_ms; /* latency over completed requests */
    double peak_admitted_bytes;
    long long cache_hits, cache_entries;
    double cache_used_bytes;
} ncpa_server_stats;

void ncpa_server_opts_default(ncpa_server_opts *opts);
ncpa_status ncpa_server_create(const ncpa_server_opts *opts, ncpa_server **out);
ncpa_status ncpa_server_submit(ncpa_server *srv, const ncpa_request *req, unsigned long long *id);
/* waits up to timeout_ms (< 0: forever); NCPA_ETIMEDOUT if not ready yet.
 * The result's arrays stay valid until ncpa_server_release. */
ncpa_status ncpa_server_wait(ncpa_server *srv, unsigned long long id, int timeout_ms, ncpa_result *out);
ncpa_status ncpa_server_release(ncpa_server *srv, unsigned long long id);
ncpa_status ncpa_server_stats_get(ncpa_server *srv, ncpa_server_stats *out);
ncpa_status ncpa_server_destroy(ncpa_server *srv);

/* Number of this library's kernels launched on the context so far. */
long long ncpa_kernel_launches(const ncpa_ctx *ctx);
/* The context's CUDA stream (cudaStream_t) for event timing / interop. */
void *ncpa_ctx_stream(ncpa_ctx *ctx);

/* Captured solves ("plans"; no counterpart in the reference, whose
 * ESSModeSolver::solve, ESSModeSolver.cpp:291-510, re-runs setParams and the
 * SLEPc solve per problem).  A plan fixes the shape of a batched solve
 * without eigenvectors -- the jobs' profiles, frequencies, azimuths and grids,
 * the params and an optional 1-D TL range grid -- allocates every buffer once
 * and records the whole device sequence (knot splines, matrices, window,
 * Sturm scan, device-built work items, bisection, eigenvectors, 1-D TL) as ONE
 * CUDA graph.  ncpa_ess_plan_run replays it with one launch and waits once
 * for the totals.  The graph reads the profiles' device arrays, so
 * ncpa_profile_update followed by a run re-solves new atmospheric data of the
 * same shape.  With tune != 0 the plan times candidate launch shapes
 * (eigenvalues per bisection item; CTAs per SM of the bisection and of the
 * eigenvector kernel) by replaying captured graphs and keeps the fastest; the
 * choice is cached in the context per batch shape.  Another item size than
 * the default changes the bisection's bracketing, so eigenvalues may differ
 * from ncpa_ess_solve's in the last bits (well inside the 1e-9 relative
 * parity bound).  Plans need want_vectors = 0 and lamb_wave_bc = 0 (both
 * need host work inside the solve).  The profiles and the context must
 * outlive the plan. */
typedef struct ncpa_plan ncpa_plan;
ncpa_status ncpa_ess_plan_create(ncpa_ctx *ctx, const ncpa_ess_job *jobs, int n_jobs,
                                 const ncpa_ess_params *params, const ncpa_tl_params *tl, int tune,
                                 ncpa_plan **out);
ncpa_status ncpa_ess_plan_run(ncpa_plan *plan);
/* the result of the last run; owned by the plan (do not destroy it) */
ncpa_status ncpa_ess_plan_modes(ncpa_plan *plan, ncpa_modes **modes);
/* 1-D TL of the last run, [problem][range] on the plan's range grid */
ncpa_status ncpa_ess_plan_tl(ncpa_plan *plan, double *re, double *im, double *incoh);
/* launch shapes in use; ms = replay time of the chosen graph when tuned, else 0 */
ncpa_status ncpa_ess_plan_tuning(const ncpa_plan *plan, int *bis_item, int *bis_ctas_per_sm,
                                 int *ev_ctas_per_sm, double *ms);
ncpa_status ncpa_ess_plan_destroy(ncpa_plan *plan);
/* New knot values for a profile, in place: same knot count, altitudes and
 * ground height, and an attenuation column exactly when the profile has one
 * (desc->attn replaces it).  Plans that read the profile see the new data at
 * their next run. */
ncpa_status ncpa_profile_update(ncpa_profile *prof, const ncpa_profile_desc *desc);

/* Diagnostics (no counterpart in the reference): per-phase device times of
 * ncpa_ess_solve measured with CUDA events on the context stream.  Phases:
 * "knots+grid", "matrix", "window", "scan", "host-items", "bisect", "eigvec",
 * "fetch".  set_timing(ctx, 1) runs the bisection and eigenvector kernels
 * apart; set_timing(ctx, 2) keeps the fused launch that solves without
 * timing run, recorded as "bisect+eigvec" and "eigvec-rest" (the follow-up
 * launch that runs only items the fused launch left).  stats() returns
 * accumulated milliseconds and calls since the last reset; sturm_steps() the
 * number of Sturm recurrence steps (one shift over one grid point) run by the
 * bisection kernel since the last reset. */
ncpa_status ncpa_ctx_set_timing(ncpa_ctx *ctx, int on);
ncpa_status ncpa_ctx_phase_stats(const ncpa_ctx *ctx, const char *phase, double *total_ms, long long *calls);
ncpa_status ncpa_ctx_reset_stats(ncpa_ctx *ctx);
ncpa_status ncpa_ctx_sturm_steps(ncpa_ctx *ctx, long long *steps);
/* the same steps, and how many of them belong to chains that also carry
 * derivatives (the Laguerre / Newton chains of the isolated eigenvalues) */
ncpa_status ncpa_ctx_bisect_steps(ncpa_ctx *ctx, long long *steps, long long *deriv_steps);
/* Points the last NCPA_SUM_TC_GUARDED modal sum of this context recomputed
 * in FP64, and its receivers x ranges (waits for the context's stream). */
ncpa_status ncpa_ctx_sum_fixups(ncpa_ctx *ctx, long long *recomputed, long long *points);
/* Error model of the last NCPA_SUM_TC_GUARDED modal sum of this context:
 * eps bounds the tensor-core error of a point relative to S, the sum of the
 * magnitudes of its modal terms at the first range of its tile of
 * *tile_ranges ranges (|P_tc - P| <= eps S); points with |P_tc| < tau S were
 * recomputed in FP64 (tau = eps (1 + 1 / d), d = 1 - 10^(-0.05 / 20)).  eps
 * and tau are 0 before the first guarded sum; tile_ranges may be NULL. */
ncpa_status ncpa_ctx_sum_guard(ncpa_ctx *ctx, double *eps, double *tau, int *tile_ranges);
/* Schedule of the last tensor-core modal sum of this context: the depths of
 * its TMA ring and generated-operand ring.  The first tensor-core call of
 * each shape (format, receiver groups, mode chunks, range tiles) times every
 * schedule (variants of them, times_ms[v] in ms; the call waits for that)
 * and the context keeps the fastest; NCPA_MS_TUNE=0 at context creation
 * keeps the first (deepest rings).  Results do not depend on the schedule. */
ncpa_status ncpa_ctx_sum_schedule(ncpa_ctx *ctx, int *t_stages, int *g_stages, int *variants, double *times_ms);
/* Measured FP64 FMA throughput of this device [TFLOP/s, FMA = 2 flops]: a
 * dependent-FMA kernel on every SM for about 50 ms. */
ncpa_status ncpa_probe_fp64_peak(ncpa_ctx *ctx, double *tflops);

/* Allocation-free eigenvectors of one problem.  No counterpart in the
 * reference: this is for callers that cannot allocate device memory once
 * they run (an application that reserves all GPU memory at start-up, code
 * inside a memory budget it does not own, a runtime whose allocator must not
 * be re-entered).  It allocates nothing and needs no context: every pointer
 * is device memory owned by the caller, `stream` is a cudaStream_t (NULL for
 * the default stream) on the current device, and the call returns once the
 * results are in place.
 *   s[nz]      scaled diagonal of h^2 A (the matrix ncpa_ess_solve builds)
 *   w[nz]      attenuation weights 2 alpha omega / c_T on the same grid
 *   mu[n]      eigenvalues of h^2 A, ascending
 *   outputs    k_pert = re_k + i im_k and the normalised mode values at grid
 *              points isrc / ircv, n entries each
 * Scratch is one array inside the library of about 21 MiB per device, held
 * until the process exits; limits: nz <= 32768 (NCPA_EINVAL beyond),
 * n <= 4000 (NCPA_ETOOMANY beyond).  All calls share that array, so calls
 * that overlap on the GPU race.  The first call on a device looks the array
 * up; make it before any stream capture.  The looked-up address is kept until
 * the process exits, so do not call this again on a device after
 * cudaDeviceReset there.  Every call waits for its own work to finish before
 * returning.  NCPA_ETIMEDOUT: a bounded device wait gave up; NCPA_ECUDA: a
 * CUDA call failed or the kernel reported another device error. */
ncpa_status ncpa_eigvec_static(const double *s, const double *w, int nz, double dz, const double *mu,
                               int n, int isrc, int ircv, double omega, double *re_k, double *im_k,
                               double *v_src, double *v_rcv, void *stream);

#ifdef __cplusplus
}
#endif
#endif
