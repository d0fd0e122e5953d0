/*
 * CPU oracle for the effective-sound-speed normal-mode path (Modess / ModBB).
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm, used as the checker by tests/, by __graft_entry__.smoke() and as
 * the timed CPU baseline leg of bench.py.  The product (the CUDA library under
 * ncpaprop-release_b200/) never links, loads or calls anything in oracle/.
 *
 * Every function names the reference file:line it restates.  Parity is pinned
 * against the reference's shipped example outputs (tests/test_oracle_golden.py)
 * and cross-checked against LAPACK dstebz/dstein (tests/test_oracle_lapack.py).
 */
#ifndef NCPA_ORACLE_H
#define NCPA_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Steffen monotone cubic (gsl_interp_steffen, used by
 *      src/atmosphere/AtmosphericProperty1D.cpp:72-82) ---------------------- */
void orc_steffen_init(int n, const double *x, const double *y, double *coef /* 4*(n-1) */);
int orc_bsearch(int n, const double *x, double xq);
/* AtmosphericProperty1D::get (AtmosphericProperty1D.cpp:116-126): clamps to the
 * end values outside [x0, x_{n-1}] */
double orc_spline_get(int n, const double *x, const double *y, const double *coef, double xq);
/* AtmosphericProperty1D::get_first_derivative (:128-136): 0 outside the range */
double orc_spline_deriv(int n, const double *x, const double *coef, double xq);
void orc_spline_get_many(int n, const double *x, const double *y, const double *coef,
                         int m, const double *xq, double *out);

/* ---- src/atmosphere/AtmosphericModel.cpp:86-219 ---------------------------- */
double orc_attn_sutherland_bass(double z_km, double T, double P, double D, double freq);

/* ---- derived knot quantities (Atmosphere1D.cpp:484-610, 821-848) ----------- */
void orc_c0_from_p_rho(int n, const double *z, const double *p, const double *rho, double *c0);
void orc_c0_from_t(int n, const double *z, const double *t, double *c0);
void orc_wind_speed_dir(int n, const double *u, const double *v, double *ws, double *wd_deg);
void orc_wc_knots(int n, const double *ws, const double *wd_deg, double az_deg, double *wc);
void orc_ceff_knots(int n, const double *c0, const double *ws, const double *wd_deg,
                    double az_deg, double *ceff);

/* ---- one (frequency, azimuth) problem: ESSModeSolver::getModalTrace
 *      (src/libmodes/ESSModeSolver.cpp:518-645) plus the scaled matrix ------ */
typedef struct {
    int    nz;            /* Nz_grid */
    double z_min;         /* m, ground after Z0 adjustment */
    double dz_grid;       /* grid spacing used for Hgt[] (ESSModeSolver.cpp:151) */
    double dz;            /* spacing used for the matrix (ESSModeSolver.cpp:314) */
    double freq;
    double admittance;    /* 0 for rigid; Lamb: -rho'/(2 rho) */
    double src_h, rcv_h;  /* m */
    int    turnoff_wkb;
    int    wvnum_filter;
    double c_min, c_max;
} orc_grid_params;

typedef struct {
    double k_min, k_max;  /* final window (after WKB / wvnum_filter) */
    double ceffmin, ceffmax;
    int    used_wkb;
} orc_grid_result;

/* ceff grid sampling, diag (unscaled, reference's diag[] incl. BC) and the
 * scaled matrix S = h^2 A: s[i] = diag[i]*h^2 - 2, s[n-1] uses diag[n-2]
 * (the EigenEngine.cpp:57-71 last-row assembly).  Returns 0 on success. */
int orc_build_grid(const orc_grid_params *gp, int nk, const double *zk, const double *ceffk,
                   const double *ceff_coef, double *hgt, double *ceff, double *diag,
                   double *s, orc_grid_result *res);

/* ---- eigen-solve (replaces EigenEngine::doESSCalculation, EigenEngine.cpp:10-172) */
int  orc_sturm_count(int n, const double *s, double x);
void orc_bisect(int n, const double *s, double lo, double hi, int c_lo, int m,
                double tol, double *mu);
/* twisted-factorisation eigenvector at shift mu; returns per-mode reductions:
 * out[0] = v(isrc), out[1] = v(ircv)  (normalised so sum v^2 dz = 1)
 * out[2] = sum v^2 w dz  (w = attenuation weight; 0 if w == NULL)
 * out[3] = sum v^2 g dz  (g = 1/ceff^2; 0 if g == NULL)
 * out[4] = twist index r
 * vfull (optional, n doubles) receives the normalised eigenvector. */
void orc_eigvec(int n, const double *s, double mu, double dz, const double *w,
                const double *g, int isrc, int ircv, double *out, double *vfull);

/* whole batched solve of one problem: counts, bisection, eigenvectors,
 * perturbation (ModeSolver.cpp:263-284).  OpenMP over modes.
 * Outputs (arrays of length >= M): kr, ki (k_pert), vs, vr, vg (group speed or 0).
 * Returns M, or -1 if M > max_modes. */
int orc_solve_modes(int n, const double *s, double h2, double dz, double k_min, double k_max,
                    double omega, const double *w, const double *g, int isrc, int ircv,
                    double tol, int max_modes, double *kr, double *ki, double *vs, double *vr,
                    double *vg, double *vfull /* optional n*max_modes, [i*M + m] */);

/* ---- WMod (WModeSolver.cpp:257-629, EigenEngine.cpp:174-395) ---------------- */
/* h^2-scaled coefficients of T(k) = M k^2 + C k + D from c0 and the wind
 * component on the grid; row 0 carries the ground term */
void orc_wmod_coeffs(int n, const double *c0g, const double *wcg, double omega, double dz,
                     double admittance, double *a2, double *a1, double *a0);
int  orc_wmod_count(int n, const double *a2, const double *a1, const double *a0, double k);
/* modes in [k_min, k_max] (k relative tolerance tol); outputs as orc_solve_modes
 * without group speeds; vfull optional [i*M + m].  Returns M or -1. */
int  orc_wmod_solve(int n, const double *a2, const double *a1, const double *a0, double dz,
                    double k_min, double k_max, const double *w, int isrc, int ircv, double tol,
                    int max_modes, double *kr, double *ki, double *vs, double *vr, double *vfull);

/* ---- modal sums (ModeSolver.cpp:292-565) ------------------------------------ */
void orc_tl1d(int M, const double *kr, const double *ki, const double *vs, const double *vr,
              int nr, double dr, int lossless, double *re, double *im, double *incoh);
void orc_tl2d(int M, const double *kr, const double *ki, const double *vs_src,
              const double *vz /* nzo x M */, int nzo, int nr, double dr, int lossless,
              double *re, double *im /* nr x nzo */);

/* ---- ModBB synthesis (ModalBroadbandPropagator.cpp:245-277,
 *      BroadbandPropagator.cpp:573-662) --------------------------------------- */
void orc_bb_transfer(int nfreq, const int *mode_off, const double *re_k, const double *im_k,
                     const double *ms, const double *mr, double rho_s, double rho_r,
                     double range, double *h_re, double *h_im);
void orc_bb_pulse(int nfreq, const double *f_vec, const double *s_re, const double *s_im,
                  const double *h_re, const double *h_im, double t0, int nfft,
                  double *out /* nfft: 2*Re p */);
void orc_dft_source(int nsamp, const double *x, double dt, int nfft, int nfreq,
                    double *s_re, double *s_im);

int orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
