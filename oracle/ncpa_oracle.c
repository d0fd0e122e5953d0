/*
 * CPU oracle for the effective-sound-speed normal-mode path.  TEST
 * INFRASTRUCTURE ONLY: the checker used by tests/, __graft_entry__.smoke() and
 * the cpu_baseline leg of bench.py; never part of the shipped library.
 *
 * Restates, in plain C, the reference algorithm of
 *   src/libmodes/ESSModeSolver.cpp, src/libmodes/ModeSolver.cpp,
 *   src/libmodes/EigenEngine.cpp (matrix assembly; the SLEPc solve itself is
 *   replaced by Sturm bisection + twisted-factorisation eigenvectors),
 *   src/atmosphere/{Atmosphere1D,AtmosphericProperty1D,AtmosphericModel}.cpp,
 *   src/libbroadband/{ModalBroadband,Broadband}Propagator.cpp.
 * Third-party arithmetic restated from its published description:
 *   - GSL >= 2.0 gsl_interp_steffen (version unpinned by the reference build):
 *     M. Steffen, "A simple method for monotonic interpolation in one
 *     dimension", A&A 239, 443 (1990), eqs. 2-11, end slopes = one-sided
 *     secants (the paper's "simplest possibility", section 2.2).
 *   - FFTW3 (unpinned): replaced by a direct DFT with exact index reduction.
 *
 * Compiled with -ffp-contract=off; fused multiply-adds appear only where fma()
 * is written, so the arithmetic is the one the CUDA kernels perform.
 */
#include "ncpa_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.141592653589793 /* src/common/util.h:13-14 (also the value
                                    AtmosphericModel.cpp sees through
                                    ncpaprop_common.h -> util.h) */

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* Steffen monotone cubic                                                    */
/* ------------------------------------------------------------------------ */

static double sgn1(double v) { return v < 0.0 ? -1.0 : 1.0; } /* sign(0) = +1 */

void orc_steffen_init(int n, const double *x, const double *y, double *coef) {
    /* slopes y'_i (eq. 11 of Steffen 1990) */
    double *yp = (double *)malloc(sizeof(double) * (size_t)n);
    yp[0] = (y[1] - y[0]) / (x[1] - x[0]);
    for (int i = 1; i < n - 1; i++) {
        double hl = x[i] - x[i - 1], hr = x[i + 1] - x[i];
        double sl = (y[i] - y[i - 1]) / hl, sr = (y[i + 1] - y[i]) / hr;
        double pp = (sl * hr + sr * hl) / (hl + hr);
        double m = fabs(sl);
        if (fabs(sr) < m) m = fabs(sr);
        if (0.5 * fabs(pp) < m) m = 0.5 * fabs(pp);
        yp[i] = (sgn1(sl) + sgn1(sr)) * m;
    }
    yp[n - 1] = (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]);
    /* cubic on [x_i, x_{i+1}]: y = d + t(c + t(b + t a)), t = x - x_i (eqs. 2-5) */
    for (int i = 0; i < n - 1; i++) {
        double h = x[i + 1] - x[i];
        double s = (y[i + 1] - y[i]) / h;
        coef[4 * i + 0] = (yp[i] + yp[i + 1] - 2.0 * s) / h / h;
        coef[4 * i + 1] = (3.0 * s - 2.0 * yp[i] - yp[i + 1]) / h;
        coef[4 * i + 2] = yp[i];
        coef[4 * i + 3] = y[i];
    }
    free(yp);
}

/* largest i in [0, n-2] with x[i] <= xq (binary search over the knots) */
int orc_bsearch(int n, const double *x, double xq) {
    int lo = 0, hi = n - 1;
    while (hi > lo + 1) {
        int mid = (lo + hi) / 2;
        if (x[mid] > xq) hi = mid; else lo = mid;
    }
    return lo;
}

double orc_spline_get(int n, const double *x, const double *y, const double *coef, double xq) {
    if (xq > x[n - 1]) return y[n - 1];
    if (xq < x[0]) return y[0];
    int i = orc_bsearch(n, x, xq);
    const double *c = coef + 4 * i;
    double t = xq - x[i];
    return c[3] + t * (c[2] + t * (c[1] + t * c[0]));
}

double orc_spline_deriv(int n, const double *x, const double *coef, double xq) {
    if (xq > x[n - 1] || xq < x[0]) return 0.0;
    int i = orc_bsearch(n, x, xq);
    const double *c = coef + 4 * i;
    double t = xq - x[i];
    return c[2] + t * (2.0 * c[1] + t * 3.0 * c[0]);
}

void orc_spline_get_many(int n, const double *x, const double *y, const double *coef,
                         int m, const double *xq, double *out) {
    for (int k = 0; k < m; k++) out[k] = orc_spline_get(n, x, y, coef, xq[k]);
}

/* ------------------------------------------------------------------------ */
/* Sutherland-Bass absorption, AtmosphericModel.cpp:86-219 (z in km, T in K,  */
/* P in Pa, D in kg/m^3, result in Np/m)                                     */
/* ------------------------------------------------------------------------ */
double orc_attn_sutherland_bass(double z, double T_z, double P_z, double D_z, double freq) {
    const double mu_o = 18.192E-6, T_o = 293.15, P_o = 101325, S = 117.0;
    const double Cv_R[4] = {5.0 / 2.0, 5.0 / 2.0, 3.0, 3.0};
    const double Cp_R[4] = {7.0 / 2.0, 7.0 / 2.0, 4.0, 4.0};
    const double theta[4] = {2239.1, 3352.0, 915.0, 1037.0};
    const double PI = ORC_PI;

    double c_snd_z = sqrt(1.4 * P_z / D_z);
    double mu = mu_o * sqrt(T_z / T_o) * ((1.0 + S / T_o) / (1.0 + S / T_z));
    double nu = (8.0 * PI * freq * mu) / (3.0 * P_z);

    double X[7];
    /* gas-fraction fits, AtmosphericModel.cpp:114-162 */
    if (z > 90.0)
        X[0] = pow(10.0, 49.296 - (1.5524 * z) + (1.8714E-2 * pow(z, 2)) - (1.1069E-4 * pow(z, 3)) +
                             (3.199E-7 * pow(z, 4)) - (3.6211E-10 * pow(z, 5)));
    else
        X[0] = pow(10.0, -0.67887);
    if (z > 76.0)
        X[1] = pow(10.0, (1.3972E-1) - (5.6269E-3 * z) + (3.9407E-5 * pow(z, 2)) - (1.0737E-7 * pow(z, 3)));
    else
        X[1] = pow(10.0, -0.10744);
    X[2] = pow(10.0, -3.3979);
    if (z > 80.0)
        X[3] = pow(10.0, -4.234 - (3.0975E-2 * z));
    else
        X[3] = pow(10.0, -19.027 + (1.3093 * z) - (4.6496E-2 * pow(z, 2)) + (7.8543E-4 * pow(z, 3)) -
                             (6.5169E-6 * pow(z, 4)) + (2.1343E-8 * pow(z, 5)));
    if (z > 95.0)
        X[4] = pow(10.0, -3.2456 + (4.6642E-2 * z) - (2.6894E-4 * pow(z, 2)) + (5.264E-7 * pow(z, 3)));
    else
        X[4] = pow(10.0, -11.195 + (1.5408E-1 * z) - (1.4348E-3 * pow(z, 2)) + (1.0166E-5 * pow(z, 3)));
    X[5] = pow(10.0, -53.746 + (1.5439 * z) - (1.8824E-2 * pow(z, 2)) + (1.1587E-4 * pow(z, 3)) -
                         (3.5399E-7 * pow(z, 4)) + (4.2609E-10 * pow(z, 5)));
    /* the reference's z > 100 sub-branch sits inside z <= 30 and never runs */
    if (z > 30.0)
        X[6] = pow(10.0, -4.2563 + (7.6245E-2 * z) - (2.1824E-3 * pow(z, 2)) - (2.3010E-6 * pow(z, 3)) +
                             (2.4265E-7 * pow(z, 4)) - (1.2500E-09 * pow(z, 5)));
    else
        X[6] = pow(10.0, -1.7491 + (4.4986E-2 * z) - (6.8549E-2 * pow(z, 2)) + (5.4639E-3 * pow(z, 3)) -
                             (1.5539E-4 * pow(z, 4)) + (1.5063E-06 * pow(z, 5)));
    double X_ON = (X[0] + X[1]) / 0.9903;

    double Z_rot_0 = 54.1 * exp(-17.3 * (pow(T_z, -1.0 / 3.0)));
    double Z_rot_1 = 63.3 * exp(-16.7 * (pow(T_z, -1.0 / 3.0)));
    double Z_rot_ = 1.0 / ((X[1] / Z_rot_1) + (X[0] / Z_rot_0));

    double sigma = 5.0 / sqrt(21.0);
    double nn = (4.0 / 5.0) * sqrt(3.0 / 7.0) * Z_rot_;
    double chi = 3.0 * nn * nu / 4.0;
    double cchi = 2.36 * chi;

    double a_cl = (2 * PI * freq / c_snd_z) *
                  sqrt(0.5 * (sqrt(1 + pow(nu, 2)) - 1) * (1 + pow(cchi, 2)) /
                       ((1 + pow(nu, 2)) * (1 + pow(sigma * cchi, 2))));
    double a_rot = (2 * PI * freq / c_snd_z) * X_ON * ((pow(sigma, 2) - 1) * chi / (2 * sigma)) *
                   sqrt(0.5 * (sqrt(1 + pow(nu, 2)) + 1) / ((1 + pow(nu, 2)) * (1 + pow(cchi, 2))));
    double a_diff = 0.003 * a_cl;

    double Tr = pow(T_z / T_o, -1.0 / 3.0) - 1.0;
    double A1 = (X[0] + X[1]) * 24.0 * exp(-9.16 * Tr);
    double A2 = (X[4] + X[5]) * 2400.0;
    double B = 40400.0 * exp(10.0 * Tr);
    double C = 0.02 * exp(-11.2 * Tr);
    double Dd = 0.391 * exp(8.41 * Tr);
    double E = 9.0 * exp(-19.9 * Tr);
    double F = 60000.0;
    double G = 28000.0 * exp(-4.17 * Tr);
    double H = 22000.0 * exp(-7.68 * Tr);
    double I_ = 15100.0 * exp(-10.4 * Tr);
    double J = 11500.0 * exp(-9.17 * Tr);
    double K = (8.48E08) * exp(9.17 * Tr);
    double L = exp(-7.72 * Tr);
    double ZZ = H * X[2] + I_ * (X[0] + 0.5 * X[4]) + J * (X[1] + 0.5 * X[5]) + K * (X[6] + X[3]);
    double hu = 100.0 * (X[3] + X[6]);
    double f_vib[4];
    f_vib[0] = (P_z / P_o) * (mu_o / mu) * (A1 + A2 + B * hu * (C + hu) * (Dd + hu));
    f_vib[1] = (P_z / P_o) * (mu_o / mu) * (E + F * X[3] + G * X[6]);
    f_vib[2] = (P_z / P_o) * (mu_o / mu) * ZZ;
    f_vib[3] = (P_z / P_o) * (mu_o / mu) * (1.2E5) * L;

    double a_vib = 0.0;
    for (int m = 0; m < 4; m++) {
        double C_R = ((pow(theta[m] / T_z, 2)) * exp(-theta[m] / T_z)) / (pow(1 - exp(-theta[m] / T_z), 2));
        double A_max = (X[m] * (PI / 2) * C_R) / (Cp_R[m] * (Cv_R[m] + C_R));
        a_vib = a_vib + (A_max / c_snd_z) * ((2 * (pow(freq, 2)) / f_vib[m]) / (1 + pow(freq / f_vib[m], 2)));
    }
    return a_cl + a_rot + a_diff + a_vib;
}

/* ------------------------------------------------------------------------ */
/* derived knot quantities                                                   */
/* ------------------------------------------------------------------------ */

/* Atmosphere1D::calculate_sound_speed_from_pressure_and_density
 * (Atmosphere1D.cpp:821-848): splines of P and RHO evaluated at the knots */
void orc_c0_from_p_rho(int n, const double *z, const double *p, const double *rho, double *c0) {
    double *cp = (double *)malloc(sizeof(double) * 4 * (size_t)(n - 1));
    double *cr = (double *)malloc(sizeof(double) * 4 * (size_t)(n - 1));
    orc_steffen_init(n, z, p, cp);
    orc_steffen_init(n, z, rho, cr);
    for (int i = 0; i < n; i++) {
        double pv = orc_spline_get(n, z, p, cp, z[i]);
        double rv = orc_spline_get(n, z, rho, cr, z[i]);
        c0[i] = sqrt(1.4 * pv / rv); /* AtmosphericModel.cpp:28-31 */
    }
    free(cp);
    free(cr);
}

/* Atmosphere1D::calculate_sound_speed_from_temperature (Atmosphere1D.cpp:769-792) */
void orc_c0_from_t(int n, const double *z, const double *t, double *c0) {
    double *ct = (double *)malloc(sizeof(double) * 4 * (size_t)(n - 1));
    orc_steffen_init(n, z, t, ct);
    for (int i = 0; i < n; i++) c0[i] = sqrt(1.4 * 287.0 * orc_spline_get(n, z, t, ct, z[i]));
    free(ct);
}

/* Atmosphere1D.cpp:484-544: speed and direction (deg clockwise from N) */
void orc_wind_speed_dir(int n, const double *u, const double *v, double *ws, double *wd_deg) {
    for (int i = 0; i < n; i++) {
        ws[i] = sqrt(u[i] * u[i] + v[i] * v[i]);
        wd_deg[i] = (ORC_PI / 2.0 - atan2(v[i], u[i])) * 180.0 / ORC_PI;
    }
}

/* Atmosphere1D.cpp:546-610: wind component along the azimuth and c_eff */
void orc_ceff_knots(int n, const double *c0, const double *ws, const double *wd_deg,
                    double az_deg, double *ceff) {
    double az_rad = az_deg * ORC_PI / 180.0;
    for (int i = 0; i < n; i++) {
        double dir = wd_deg[i] * ORC_PI / 180.0;
        double wc = ws[i] * cos(dir - az_rad);
        ceff[i] = wc + c0[i];
    }
}

/* wind component along the azimuth at the knots, the wc term of
 * orc_ceff_knots (Atmosphere1D::calculate_wind_component) */
void orc_wc_knots(int n, const double *ws, const double *wd_deg, double az_deg, double *wc) {
    double az_rad = az_deg * ORC_PI / 180.0;
    for (int i = 0; i < n; i++) {
        double dir = wd_deg[i] * ORC_PI / 180.0;
        wc[i] = ws[i] * cos(dir - az_rad);
    }
}

/* ------------------------------------------------------------------------ */
/* getModalTrace (ESSModeSolver.cpp:518-621) and the scaled matrix            */
/* ------------------------------------------------------------------------ */
int orc_build_grid(const orc_grid_params *gp, int nk, const double *zk, const double *ceffk,
                   const double *ceff_coef, double *hgt, double *ceff, double *diag,
                   double *s, orc_grid_result *res) {
    const int nz = gp->nz;
    const double dz = gp->dz;
    const double omega = 2 * ORC_PI * gp->freq;
    for (int i = 0; i < nz; i++) {
        hgt[i] = gp->z_min + i * gp->dz_grid;
        ceff[i] = orc_spline_get(nk, zk, ceffk, ceff_coef, hgt[i]);
    }
    double ceff_grnd = orc_spline_get(nk, zk, ceffk, ceff_coef, gp->z_min);
    double ceffmin = ceff_grnd, ceffmax = ceff_grnd;
    for (int i = 0; i < nz; i++) {
        double t = omega / ceff[i];
        diag[i] = t * t;
        if (ceff[i] < ceffmin) ceffmin = ceff[i];
        if (ceff[i] > ceffmax) ceffmax = ceff[i];
    }
    double bnd_cnd = (1. / (dz * gp->admittance + 1)) / (dz * dz);
    diag[0] = bnd_cnd + diag[0];

    double k_max, k_min;
    int used_wkb = 0;
    if (fabs(gp->src_h) < 1.0e-3 && fabs(gp->rcv_h) < 1.0e-3 && !gp->turnoff_wkb) {
        used_wkb = 1;
        double k_max_full = omega / ceffmin;
        double k_gnd = omega / ceff_grnd;
        double dkk = (k_max_full * k_max_full - k_gnd * k_gnd) / 100.0;
        double kk = k_gnd * k_gnd;
        if (dkk > 1.0e-10) {
            for (kk = k_gnd * k_gnd; kk < k_max_full * k_max_full; kk = kk + dkk) {
                double integral = 0.0, term = 1.0;
                int i = 0;
                /* the reference walks up the grid until the integrand drops to
                 * dkk; the walk is bounded by the grid here */
                while (term > dkk && i < nz) {
                    double k_eff = omega / ceff[i];
                    term = fabs(kk - k_eff * k_eff);
                    integral = integral + dz * sqrt(term);
                    i++;
                }
                if (integral >= 10.0) break;
            }
        }
        k_max = sqrt(kk);
    } else {
        k_max = omega / ceffmin;
    }
    int top = nz - (nz / 10);
    int itop = top + 1 < nz ? top + 1 : nz - 1;
    k_min = omega / ceff[itop];
    if (used_wkb && k_max < k_min) k_max = omega / ceffmin;
    if (gp->wvnum_filter) { /* ESSModeSolver.cpp:366-369 */
        k_min = 2 * ORC_PI * gp->freq / gp->c_max;
        k_max = 2 * ORC_PI * gp->freq / gp->c_min;
    }
    /* scaled matrix: S = h^2 A, off-diagonal 1; last row repeats diag[n-2] */
    double h2 = dz * dz;
    for (int i = 0; i < nz - 1; i++) s[i] = diag[i] * h2 - 2.0;
    s[nz - 1] = diag[nz - 2] * h2 - 2.0;
    res->k_min = k_min;
    res->k_max = k_max;
    res->ceffmin = ceffmin;
    res->ceffmax = ceffmax;
    res->used_wkb = used_wkb;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Sturm counts, division-free                                                */
/* ------------------------------------------------------------------------ */

/* biased exponent field of |v| */
static inline int bexp(double v) {
    uint64_t b;
    memcpy(&b, &v, 8);
    return (int)((b >> 52) & 0x7ff);
}
/* overflow-only shift for recurrences whose squares are summed: keeps the
 * pair below 2^240 */
static inline int grow_shift(double a, double b) {
    int e = bexp(a), eb = bexp(b);
    if (eb > e) e = eb;
    e -= 1023;
    return e > 240 ? e : 0;
}
/* exponent shift that brings max(|a|,|b|) near 1, or 0 if not needed */
static inline int rescale_shift(double a, double b) {
    int e = bexp(a), eb = bexp(b);
    if (eb > e) e = eb;
    if (e == 0) return 0;
    e -= 1023;
    if (e > 480 || e < -480) return e;
    return 0;
}

/* number of eigenvalues of S (diag s, unit off-diagonal) below x: negative
 * pivots of the LDL^T factorisation of S - xI, read off as sign changes of
 * p_{-1}=1, p_0=s_0-x, p_i=(s_i-x)p_{i-1}-p_{i-2} (pivot_i = p_i/p_{i-1}).
 * Power-of-two rescaling every 16 steps is exact and leaves signs unchanged.
 * Replaces ModeSolver::sturmCount (ModeSolver.cpp:233-260) and the interval
 * inertia of the SLEPc spectrum slice (EigenEngine.cpp:109). */
int orc_sturm_count(int n, const double *s, double x) {
    double pm = 1.0, p = s[0] - x;
    int cnt = signbit(p) ? 1 : 0;
    for (int i = 1; i < n; i++) {
        double a = s[i] - x;
        double pn = fma(a, p, -pm);
        cnt += (signbit(pn) != 0) != (signbit(p) != 0);
        pm = p;
        p = pn;
        if ((i & 15) == 0) {
            int sh = rescale_shift(pm, p);
            if (sh) {
                pm = ldexp(pm, -sh);
                p = ldexp(p, -sh);
            }
        }
    }
    return cnt;
}

/* bisection for eigen-indices c_lo .. c_lo+m-1 on [lo, hi] */
void orc_bisect(int n, const double *s, double lo, double hi, int c_lo, int m, double tol, double *mu) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int e = 0; e < m; e++) {
        int j = c_lo + e;
        double a = lo, b = hi;
        while (b - a > tol) {
            double mid = 0.5 * (a + b);
            if (mid <= a || mid >= b) break;
            if (orc_sturm_count(n, s, mid) > j) b = mid; else a = mid;
        }
        mu[e] = 0.5 * (a + b);
    }
}

/* ------------------------------------------------------------------------ */
/* eigenvector by twisted factorisation                                      */
/* ------------------------------------------------------------------------ */
/* For S - mu I with unit off-diagonals the forward solution of rows 0..i-1 is
 * z_i = (-1)^i p_{i-1}, the backward solution of rows i+1..n-1 is
 * z_i = (-1)^(n-1-i) q_{i+1} with q_n = 1, q_{n-1} = s_{n-1}-mu,
 * q_i = (s_i-mu) q_{i+1} - q_{i+2}.  The twist r maximises |p_{r-1} q_{r+1}|
 * (equivalently minimises |gamma_r| = |det(S-mu)/(p_{r-1} q_{r+1})|), and
 *   z_i = (-1)^i p_{i-1} q_{r+1}  (i <= r),   z_i = (-1)^i p_{r-1} q_{i+1}  (i >= r)
 * solves (S - mu) z = gamma_r e_r: one inverse-iteration step from e_r.
 * Replaces the eigenvector half of EigenEngine.cpp:145-162; the reductions
 * replace ModeSolver::doPerturb (ModeSolver.cpp:263-284) and the group-speed
 * sum of ESSModeSolver::writePhaseAndGroupSpeeds (ESSModeSolver.cpp:738-744). */
/* order-preserving key of |v| * 2^e: (biased exponent + e) * 2^20 + top 20
 * mantissa bits; exact enough for an argmax and free of int64 overflow for
 * any exponent offset a grid can accumulate */
static inline int64_t mag_key(double v, int e) {
    uint64_t b;
    v = fabs(v);
    if (v == 0.0) return INT64_MIN / 2;
    memcpy(&b, &v, 8);
    int be = (int)((b >> 52) & 0x7ff);
    return (int64_t)(be + e) * 1048576 + (int64_t)((b >> 32) & 0xfffff);
}

void orc_eigvec(int n, const double *s, double mu, double dz, const double *w, const double *g,
                int isrc, int ircv, double *out, double *vfull) {
    double *q = (double *)malloc(sizeof(double) * (size_t)(n + 1));
    int *eq = (int *)malloc(sizeof(int) * (size_t)(n + 1));
    double *pv = vfull ? (double *)malloc(sizeof(double) * (size_t)n) : NULL;
    int *ep = vfull ? (int *)malloc(sizeof(int) * (size_t)n) : NULL;

    /* backward pass: q_{i} for i = n..0 */
    {
        double q2 = 0.0, q1 = 1.0; /* q_{i+2}, q_{i+1}; q_{n+1}=0, q_n=1 */
        int E = 0;
        q[n] = 1.0;
        eq[n] = 0;
        for (int i = n - 1; i >= 0; i--) {
            double a = s[i] - mu;
            double qi = fma(a, q1, -q2);
            q[i] = qi;
            eq[i] = E;
            q2 = q1;
            q1 = qi;
            if ((i & 15) == 0) {
                int sh = grow_shift(q1, q2);
                if (sh) {
                    q1 = ldexp(q1, -sh);
                    q2 = ldexp(q2, -sh);
                    E += sh;
                }
            }
        }
    }

    /* forward pass */
    double pm2 = 0.0, pm1 = 1.0; /* p_{i-2}, p_{i-1} */
    int Ep = 0;
    double An = 0, Aw = 0, Ag = 0;
    int64_t best = INT64_MIN;
    int r = 0;
    double Fn = 0, Fw = 0, Fg = 0, pr = 1.0, inv_qr = 1.0;
    int Epr = 0, Eqr = 0;
    double Tn = 0, Tw = 0, Tg = 0;
    double ps_src = 0, ps_rcv = 0, qr_src = 0, qr_rcv = 0;
    int Eps_src = 0, Eps_rcv = 0;
    for (int i = 0; i < n; i++) {
        double sq = pm1 * pm1;
        double wi = w ? w[i] : 0.0, gi = g ? g[i] : 0.0;
        An += sq;
        Aw += sq * wi;
        Ag += sq * gi;
        if (pv) {
            pv[i] = pm1;
            ep[i] = Ep;
        }
        double qn = q[i + 1];
        int64_t key = mag_key(pm1 * qn, Ep + eq[i + 1]);
        if (key > best) {
            best = key;
            r = i;
            Fn = An / sq;
            Fw = Aw / sq;
            Fg = Ag / sq;
            pr = pm1;
            Epr = Ep;
            inv_qr = 1.0 / qn;
            Eqr = eq[i + 1];
            Tn = Tw = Tg = 0.0;
        } else {
            double t = ldexp(qn * inv_qr, eq[i + 1] - Eqr);
            double t2 = t * t;
            Tn += t2;
            Tw += t2 * wi;
            Tg += t2 * gi;
        }
        if (i == isrc) {
            ps_src = pm1;
            Eps_src = Ep;
            qr_src = (r < i) ? ldexp(qn * inv_qr, eq[i + 1] - Eqr) : 1.0;
        }
        if (i == ircv) {
            ps_rcv = pm1;
            Eps_rcv = Ep;
            qr_rcv = (r < i) ? ldexp(qn * inv_qr, eq[i + 1] - Eqr) : 1.0;
        }
        double a = s[i] - mu;
        double p = fma(a, pm1, -pm2);
        pm2 = pm1;
        pm1 = p;
        if ((i & 15) == 15) {
            int sh = grow_shift(pm1, pm2);
            if (sh) {
                pm1 = ldexp(pm1, -sh);
                pm2 = ldexp(pm2, -sh);
                An = ldexp(An, -2 * sh);
                Aw = ldexp(Aw, -2 * sh);
                Ag = ldexp(Ag, -2 * sh);
                Ep += sh;
            }
        }
    }
    double nrm = Fn + Tn; /* sum z^2 / z_r^2 */
    double scale = 1.0 / sqrt(nrm * dz);
    double zs, zr;
    if (isrc <= r) zs = ldexp(ps_src / pr, Eps_src - Epr); else zs = qr_src;
    if (ircv <= r) zr = ldexp(ps_rcv / pr, Eps_rcv - Epr); else zr = qr_rcv;
    if ((isrc - r) & 1) zs = -zs;
    if ((ircv - r) & 1) zr = -zr;
    out[0] = zs * scale;
    out[1] = zr * scale;
    out[2] = (Fw + Tw) / nrm;
    out[3] = (Fg + Tg) / nrm;
    out[4] = (double)r;
    if (vfull) {
        double qref = 1.0 / inv_qr;
        for (int i = 0; i < n; i++) {
            double zi;
            if (i <= r) zi = ldexp(pv[i] / pr, ep[i] - Epr);
            else zi = ldexp(q[i + 1] / qref, eq[i + 1] - Eqr);
            if ((i - r) & 1) zi = -zi;
            vfull[i] = zi * scale;
        }
        free(pv);
        free(ep);
    }
    free(q);
    free(eq);
}

/* principal complex square root */
static double complex csqrt_p(double complex z) { return csqrt(z); }

int orc_solve_modes(int n, const double *s, double h2, double dz, double k_min, double k_max,
                    double omega, const double *w, const double *g, int isrc, int ircv,
                    double tol, int max_modes, double *kr, double *ki, double *vs, double *vr,
                    double *vg, double *vfull) {
    double lo = (k_min * k_min) * h2, hi = (k_max * k_max) * h2;
    int c_lo = orc_sturm_count(n, s, lo);
    int c_hi = orc_sturm_count(n, s, hi);
    int M = c_hi - c_lo;
    if (M < 0) M = 0;
    if (M > max_modes) return -1;
    double *mu = (double *)malloc(sizeof(double) * (size_t)(M > 0 ? M : 1));
    orc_bisect(n, s, lo, hi, c_lo, M, tol, mu);
#pragma omp parallel for schedule(dynamic, 1)
    for (int m = 0; m < M; m++) {
        double o[5];
        double *vcol = NULL;
        if (vfull) vcol = (double *)malloc(sizeof(double) * (size_t)n);
        orc_eigvec(n, s, mu[m], dz, w, g, isrc, ircv, o, vcol);
        double ks = sqrt(mu[m] / h2);
        double complex kp = csqrt_p(ks * ks + I * o[2]);
        kr[m] = creal(kp);
        ki[m] = cimag(kp);
        vs[m] = o[0];
        vr[m] = o[1];
        if (vg) {
            double vph = omega / kr[m];
            vg[m] = g ? 1.0 / (vph * o[3]) : 0.0;
        }
        if (vfull) {
            for (int i = 0; i < n; i++) vfull[(size_t)i * M + m] = vcol[i];
            free(vcol);
        }
    }
    free(mu);
    return M;
}

/* ------------------------------------------------------------------------ */
/* WMod: wide-angle modes (WModeSolver.cpp:257-629, EigenEngine.cpp:174-395)  */
/* ------------------------------------------------------------------------ */
/* The reference solves (M k^2 + C k + D) v = 0 (M = diag(md), C = diag(cd),
 * D tridiagonal with diagonal kd - 2/h^2 and off-diagonal 1/h^2) through the
 * linearised 2N pencil with SLEPc.  Here T(k) h^2 = diag(a2 k^2 + a1 k + a0)
 * with unit off-diagonal, a2 = md h^2, a1 = cd h^2, a0 = kd h^2 - 2, where
 *   kd = (omega/c0)^2 (+ the ground term (1/(dz adm + 1))/dz^2 in row 0),
 *   md = (wc/c0)^2 - 1,  cd = -2 omega wc / c0^2     (WModeSolver.cpp:544-565)
 * and no last-row repeat (EigenEngine.cpp:266-275).  For real k, dT/dk =
 * 2 M k + C is negative definite while |wc| is below c0 and k inside the
 * propagating window, so the number of negative eigenvalues of T(k) grows by
 * one at each real eigenvalue: Sturm counts in k locate them exactly. */
void orc_wmod_coeffs(int n, const double *c0g, const double *wcg, double omega, double dz, double admittance,
                     double *a2, double *a1, double *a0) {
    double h2 = dz * dz;
    double bnd = (1. / (dz * admittance + 1)) / (dz * dz);
    for (int i = 0; i < n; i++) {
        double t = omega / c0g[i];
        double kd = t * t;
        double u = wcg[i] / c0g[i];
        double md = u * u - 1;
        double cd = -2 * omega * (wcg[i] / (c0g[i] * c0g[i]));
        if (i == 0) kd = bnd + kd;
        a2[i] = md * h2;
        a1[i] = cd * h2;
        a0[i] = kd * h2 - 2.0;
    }
}

static inline double wmod_diag(const double *a2, const double *a1, const double *a0, int i, double k) {
    return fma(fma(a2[i], k, a1[i]), k, a0[i]);
}

/* number of negative eigenvalues of T(k) (sign changes of the division-free
 * recurrence, as orc_sturm_count) */
int orc_wmod_count(int n, const double *a2, const double *a1, const double *a0, double k) {
    double pm = 1.0, p = wmod_diag(a2, a1, a0, 0, k);
    int cnt = signbit(p) ? 1 : 0;
    for (int i = 1; i < n; i++) {
        double pn = fma(wmod_diag(a2, a1, a0, i, k), p, -pm);
        cnt += (signbit(pn) != 0) != (signbit(p) != 0);
        pm = p;
        p = pn;
        if ((i & 15) == 0) {
            int sh = rescale_shift(pm, p);
            if (sh) {
                pm = ldexp(pm, -sh);
                p = ldexp(p, -sh);
            }
        }
    }
    return cnt;
}

/* wide-angle modes of one problem in [k_min, k_max]: bisection in k to the
 * relative tolerance tol, eigenvector of T(k) by twisted factorisation, the
 * normalisation of SLEPc's unit-2-norm eigenvectors of the pencil [v; k v]
 * (sum v^2 dz = 1/(1+k^2), v = x/sqrt(dz), EigenEngine.cpp:368-379) and the
 * perturbative attenuation of ModeSolver::doPerturb (ModeSolver.cpp:263-284).
 * Returns M, or -1 above max_modes. */
int orc_wmod_solve(int n, const double *a2, const double *a1, const double *a0, double dz, double k_min,
                   double k_max, const double *w, int isrc, int ircv, double tol, int max_modes, double *kr,
                   double *ki, double *vs, double *vr, double *vfull) {
    int c_lo = orc_wmod_count(n, a2, a1, a0, k_min);
    int c_hi = orc_wmod_count(n, a2, a1, a0, k_max);
    int M = c_hi - c_lo;
    if (M < 0) M = 0;
    if (M > max_modes) return -1;
#pragma omp parallel for schedule(dynamic, 1)
    for (int e = 0; e < M; e++) {
        int j = c_lo + e;
        double a = k_min, b = k_max;
        while (b - a > tol * b) {
            double mid = 0.5 * (a + b);
            if (mid <= a || mid >= b) break;
            if (orc_wmod_count(n, a2, a1, a0, mid) > j) b = mid; else a = mid;
        }
        double k = 0.5 * (a + b);
        double *t = (double *)malloc(sizeof(double) * (size_t)n);
        double *vcol = vfull ? (double *)malloc(sizeof(double) * (size_t)n) : NULL;
        for (int i = 0; i < n; i++) t[i] = wmod_diag(a2, a1, a0, i, k);
        double o[5];
        orc_eigvec(n, t, 0.0, dz, w, NULL, isrc, ircv, o, vcol);
        double f = 1.0 / sqrt(1.0 + k * k);
        double complex kp = csqrt_p(k * k + I * (o[2] * f * f));
        kr[e] = creal(kp);
        ki[e] = cimag(kp);
        vs[e] = o[0] * f;
        vr[e] = o[1] * f;
        if (vfull) {
            for (int i = 0; i < n; i++) vfull[(size_t)i * M + e] = vcol[i] * f;
            free(vcol);
        }
        free(t);
    }
    return M;
}

/* ------------------------------------------------------------------------ */
/* modal sums                                                                 */
/* ------------------------------------------------------------------------ */
/* ModeSolver::getTLoss1D / getTLoss1DNx2 (ModeSolver.cpp:292-381, 387-489) */
void orc_tl1d(int M, const double *kr, const double *ki, const double *vs, const double *vr,
              int nr, double dr, int lossless, double *re, double *im, double *incoh) {
    const double PI = ORC_PI;
    double complex expov8pi = 4 * PI * I * cexp(-I * PI * 0.25) / sqrt(8.0 * PI);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nr; i++) {
        double r = (i + 1) * dr;
        double complex sc = 0;
        double si = 0;
        for (int m = 0; m < M; m++) {
            double complex k = lossless ? (double complex)kr[m] : kr[m] + I * ki[m];
            double vv = vs[m] * vr[m];
            sc += vv * cexp(I * k * r) / csqrt(k);
            if (lossless) si += (vv * vv) / kr[m];
            else si += (vv * vv) * exp(-2 * ki[m] * r) / cabs(k);
        }
        sc = 1000.0 * expov8pi * sc / sqrt(r);
        re[i] = creal(sc);
        im[i] = cimag(sc);
        incoh[i] = 1000.0 * 4 * PI * sqrt(si) * sqrt(1. / 8. / PI / r);
    }
}

/* ModeSolver::getTLoss2D (ModeSolver.cpp:492-565); vz rows are the sampled
 * heights, vs_src the mode values at the source height */
void orc_tl2d(int M, const double *kr, const double *ki, const double *vs_src, const double *vz,
              int nzo, int nr, double dr, int lossless, double *re, double *im) {
    const double PI = ORC_PI;
    double complex expov8pi = 4 * PI * I * cexp(-I * PI * 0.25) / sqrt(8.0 * PI);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nr; i++) {
        double r = (i + 1) * dr;
        double complex *b = (double complex *)malloc(sizeof(double complex) * (size_t)(M > 0 ? M : 1));
        for (int m = 0; m < M; m++) {
            double complex k = lossless ? (double complex)kr[m] : kr[m] + I * ki[m];
            b[m] = vs_src[m] * cexp(I * k * r) / csqrt(k);
        }
        for (int j = 0; j < nzo; j++) {
            double complex sum = 0;
            for (int m = 0; m < M; m++) sum += vz[(size_t)j * M + m] * b[m];
            sum = 1000.0 * expov8pi * sum / sqrt(r);
            re[(size_t)i * nzo + j] = creal(sum);
            im[(size_t)i * nzo + j] = cimag(sum);
        }
        free(b);
    }
}

/* ------------------------------------------------------------------------ */
/* ModBB synthesis                                                            */
/* ------------------------------------------------------------------------ */
/* BroadbandPropagator::half_hann (BroadbandPropagator.cpp:654-662).  With a
 * one-bin window (end == begin, 10 <= nfreq < 20) the reference divides 0 by
 * 0 and its waveforms come out NaN; here that bin keeps the limit value 1. */
static double half_hann(int begin, int end, int i) {
    if (i < begin) return 1.0;
    if (end == begin) return i == begin ? 1.0 : 0.0;
    if (begin <= i && i <= end) return 0.5 * (cos(ORC_PI * (i - begin) / (end - begin)) + 1.0);
    return 0.0;
}

/* ModalBroadbandPropagator::compute_modal_sum (ModalBroadbandPropagator.cpp:245-277) */
void orc_bb_transfer(int nfreq, const int *mode_off, const double *re_k, const double *im_k,
                     const double *ms, const double *mr, double rho_s, double rho_r,
                     double range, double *h_re, double *h_im) {
    const double PI = ORC_PI;
    double sqrt_rho_ratio = sqrt(rho_r / rho_s);
    double complex expov8pir = I * cexp(-I * PI * 0.25) / sqrt(8.0 * PI * range);
    for (int i = 0; i < nfreq; i++) {
        double complex cup = 0.0;
        for (int j = mode_off[i]; j < mode_off[i + 1]; j++) {
            double complex kh = re_k[j] + I * im_k[j];
            double complex pot = cexp(I * range * kh);
            pot = (ms[j] * mr[j]) * pot;
            pot = pot / csqrt(kh);
            cup = cup + pot;
        }
        double complex h = expov8pir * cup * sqrt_rho_ratio;
        h_re[i] = creal(h);
        h_im[i] = cimag(h);
    }
    int smooth = (int)floor(0.1 * nfreq);
    for (int i = nfreq - smooth; i < nfreq; i++) {
        double hh = half_hann(nfreq - smooth, nfreq - 1, i);
        h_re[i] *= hh;
        h_im[i] *= hh;
    }
}

/* BroadbandPropagator::fft_pulse_prop (BroadbandPropagator.cpp:573-651) with
 * the forward FFT written as a direct DFT over the nfreq non-zero bins, then
 * the factor 2 Re of ModalBroadbandPropagator.cpp:223-225 */
void orc_bb_pulse(int nfreq, const double *f_vec, const double *s_re, const double *s_im,
                  const double *h_re, const double *h_im, double t0, int nfft, double *out) {
    const double PI = ORC_PI;
    double df = f_vec[2] - f_vec[1]; /* f_step, ModalBroadbandPropagator.cpp:65 */
    double complex *arg = (double complex *)malloc(sizeof(double complex) * (size_t)nfreq);
    for (int i = 0; i < nfreq; i++) {
        double complex tph = cexp(-I * 2.0 * PI * f_vec[i] * t0);
        arg[i] = tph * (s_re[i] + I * s_im[i]) * (h_re[i] + I * h_im[i]);
    }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nfft; k++) {
        double complex acc = 0;
        for (int n = 0; n < nfreq; n++) {
            long long kn = ((long long)k * n) % nfft;
            double ang = -2.0 * PI * (double)kn / (double)nfft;
            acc += arg[n] * (cos(ang) + I * sin(ang));
        }
        out[k] = 2.0 * creal(df * acc);
    }
    free(arg);
}

/* source spectrum of a time-domain waveform: FFTW_BACKWARD of the zero-padded
 * series times dt, first nfreq bins (BroadbandPropagator.cpp:327-353) */
void orc_dft_source(int nsamp, const double *x, double dt, int nfft, int nfreq, double *s_re, double *s_im) {
    const double PI = ORC_PI;
    for (int k = 0; k < nfreq; k++) {
        double complex acc = 0;
        for (int n = 0; n < nsamp && n < nfft; n++) {
            long long kn = ((long long)k * n) % nfft;
            double ang = 2.0 * PI * (double)kn / (double)nfft;
            acc += x[n] * (cos(ang) + I * sin(ang));
        }
        s_re[k] = creal(acc) * dt;
        s_im[k] = cimag(acc) * dt;
    }
}
