// Wide-angle (WMod) normal modes: the quadratic eigenproblem
// (M k^2 + C k + D) v = 0 of WModeSolver::solve (WModeSolver.cpp:257-486),
// which the reference linearises to a 2N pencil and hands to SLEPc
// (EigenEngine::doWideAngleCalculation, EigenEngine.cpp:174-395).
//
// Here T(k) h^2 = diag(a2 k^2 + a1 k + a0) with unit off-diagonal:
//   a2 = ((wc/c0)^2 - 1) h^2,  a1 = -2 omega wc / c0^2 h^2,
//   a0 = (omega/c0)^2 h^2 - 2  (+ the ground term in row 0),
// (WModeSolver.cpp:544-565; no last-row repeat, EigenEngine.cpp:266-275).
// For real k inside the propagating window dT/dk = 2 M k + C is negative
// definite (subsonic winds), so the number of negative eigenvalues of T(k)
// grows by one at each real eigenvalue: the modes are found with Sturm counts
// in k (isolation scan, then per-lane bisection / safeguarded Newton on
// det T(k) with its k-derivative), and each eigenvector is the null vector of
// T(k) by twisted factorisation.  The coefficient rows are read from global
// memory: every lane of a warp reads the same row, so each load is one
// broadcast from L1 / L2.
#include "device_common.cuh"
#include "kernels.hpp"

namespace ncpa {

namespace {

constexpr int kWScanThreads = kScanPoints / 2;  // two shifts per thread
constexpr int kWWarps = 4;                      // warps per CTA of the bisection / eigenvector kernels
constexpr int kWMaxRounds = 400;                // bound on bisection / Newton rounds

__device__ __forceinline__ double wscan_x(double lo, double hi, int t) {
    if (t == 0) return lo;
    if (t == kScanPoints - 1) return hi;
    return lo + (hi - lo) * ((double)t / (double)(kScanPoints - 1));
}

__device__ __forceinline__ double wdiag(double a2, double a1, double a0, double k) {
    return fma(fma(a2, k, a1), k, a0);
}

}  // namespace

// wind component along each azimuth at the knots (the wc term of
// k_ceff_knots, same expression)
__global__ void k_wc_knots(int n, int n_az, const double* __restrict__ az, const double* __restrict__ ws,
                           const double* __restrict__ wd, double* __restrict__ wc) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int a = blockIdx.y;
    if (k >= n || a >= n_az) return;
    const double az_rad = az[a] * kPi / 180.0;
    const double dir = wd[k] * kPi / 180.0;
    wc[(size_t)a * n + k] = ws[k] * cos(dir - az_rad);
}

int launch_wc_knots(cudaStream_t st, int n, int n_az, const double* az, const double* ws, const double* wd,
                    double* wc) {
    dim3 grid((n + 255) / 256, n_az);
    k_wc_knots<<<grid, 256, 0, st>>>(n, n_az, az, ws, wd, wc);
    return 1;
}

// Coefficient rows of one group's problems (rows nz_pad apart, problem p =
// frequency-major over n_az azimuths) on the sampling grid z_min + i dz_grid
// (WModeSolver.cpp:196-208), with the matrix spacing dz; also (omega/c_eff)^2
// for the WKB search and the c_eff extrema / ground / top values of
// getModalTrace (WModeSolver.cpp:530-629).
__global__ void __launch_bounds__(256) k_wmod_build(int nk, const double* __restrict__ zk,
                                                    const double* __restrict__ c0k, const double* __restrict__ c0c,
                                                    const double* __restrict__ wck, const double* __restrict__ wcc,
                                                    const double* __restrict__ ceffk,
                                                    const double* __restrict__ ceffc, int n_az,
                                                    ProblemInfo* __restrict__ pinfo, int nz, int nz_pad,
                                                    double z_min, double dz_grid, double dz, double admittance,
                                                    double* __restrict__ a2, double* __restrict__ a1,
                                                    double* __restrict__ a0, double* __restrict__ kz2) {
    const int p = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int az = p % n_az;
    const double omega = pinfo[p].omega;
    double cmin = 1e300, cmax = -1e300;
    if (i < nz) {
        const double z = z_min + i * dz_grid;
        const double c0 = spline_get(nk, zk, c0k, c0c, z);
        const double wc = spline_get(nk, zk, wck + (size_t)az * nk, wcc + (size_t)az * 4 * (nk - 1), z);
        const double ce = spline_get(nk, zk, ceffk + (size_t)az * nk, ceffc + (size_t)az * 4 * (nk - 1), z);
        const double h2 = dz * dz;
        const double t = omega / c0;
        double kd = t * t;
        const double u = wc / c0;
        const double md = u * u - 1;
        const double cd = -2 * omega * (wc / (c0 * c0));
        if (i == 0) kd = (1. / (dz * admittance + 1)) / (dz * dz) + kd;
        const size_t o = (size_t)p * nz_pad + i;
        a2[o] = md * h2;
        a1[o] = cd * h2;
        a0[o] = kd * h2 - 2.0;
        if (kz2) {
            const double te = omega / ce;
            kz2[o] = te * te;
        }
        cmin = cmax = ce;
        if (i == 0) pinfo[p].ceff_grnd = ce;
        const int top = nz - (nz / 10);
        const int itop = top + 1 < nz ? top + 1 : nz - 1;
        if (i == itop) pinfo[p].ceff_top = ce;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        cmin = fmin(cmin, __shfl_xor_sync(0xffffffffu, cmin, o));
        cmax = fmax(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
    }
    __shared__ double smin[8], smax[8];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        smin[wid] = cmin;
        smax[wid] = cmax;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < 8; ++k) {
            cmin = fmin(cmin, smin[k]);
            cmax = fmax(cmax, smax[k]);
        }
        cmin = fmin(cmin, smin[0]);
        cmax = fmax(cmax, smax[0]);
        if (cmin < 1e300) {
            atomicMin(&pinfo[p].ceffmin_bits, (unsigned long long)__double_as_longlong(cmin));
            atomicMax(&pinfo[p].ceffmax_bits, (unsigned long long)__double_as_longlong(cmax));
        }
    }
}

int launch_wmod_build(cudaStream_t st, int nk, const double* zk, const double* c0k, const double* c0c,
                      const double* wck, const double* wcc, const double* ceffk, const double* ceffc, int n_az,
                      int P, ProblemInfo* pinfo, int nz, int nz_pad, double z_min, double dz_grid, double dz,
                      double admittance, double* a2, double* a1, double* a0, double* kz2) {
    dim3 grid((nz + 255) / 256, P);
    k_wmod_build<<<grid, 256, 0, st>>>(nk, zk, c0k, c0c, wck, wcc, ceffk, ceffc, n_az, pinfo, nz, nz_pad, z_min,
                                       dz_grid, dz, admittance, a2, a1, a0, kz2);
    return 1;
}

// one step of the division-free Sturm recurrence at k, sign change counted
__device__ __forceinline__ void wstep(double t, double& p0, double& p1, unsigned& prev, int& cnt) {
    const double q = fma(t, p1, -p0);
    const unsigned b = static_cast<unsigned>(__double2hiint(q)) >> 31;
    cnt += static_cast<int>(b ^ prev);
    prev = b;
    p0 = p1;
    p1 = q;
}

// isolation scan: kScanPoints counts per problem on an even grid of
// [k_min, k_max] (the layout k_make_items reads)
__global__ void __launch_bounds__(kWScanThreads) k_wscan(const ProblemInfo* __restrict__ pinfo,
                                                         const double* __restrict__ a2,
                                                         const double* __restrict__ a1,
                                                         const double* __restrict__ a0, int* __restrict__ counts) {
    const int p = blockIdx.x;
    const ProblemInfo pi = pinfo[p];
    const double* r2 = a2 + pi.s_off;
    const double* r1 = a1 + pi.s_off;
    const double* r0 = a0 + pi.s_off;
    const int t0 = threadIdx.x, t1 = threadIdx.x + kWScanThreads;
    const double x0 = wscan_x(pi.k_min, pi.k_max, t0), x1 = wscan_x(pi.k_min, pi.k_max, t1);
    double pa0 = 0.0, pa1 = 1.0, pb0 = 0.0, pb1 = 1.0;
    unsigned ba = 0u, bb = 0u;
    int ca = 0, cb = 0;
    for (int i = 0; i < pi.nz; ++i) {
        const double c2 = __ldg(r2 + i), c1 = __ldg(r1 + i), c0 = __ldg(r0 + i);
        wstep(wdiag(c2, c1, c0, x0), pa0, pa1, ba, ca);
        wstep(wdiag(c2, c1, c0, x1), pb0, pb1, bb, cb);
        if ((i & 31) == 31) {
            int sh = rescale_shift(pa0, pa1);
            if (sh) {
                const double sc = pow2(-sh);
                pa0 *= sc;
                pa1 *= sc;
            }
            sh = rescale_shift(pb0, pb1);
            if (sh) {
                const double sc = pow2(-sh);
                pb0 *= sc;
                pb1 *= sc;
            }
        }
    }
    counts[(size_t)p * kScanPoints + t0] = ca;
    counts[(size_t)p * kScanPoints + t1] = cb;
}

int launch_wscan(cudaStream_t st, int P, const ProblemInfo* pinfo, const double* a2, const double* a1,
                 const double* a0, int* counts) {
    if (P <= 0) return 0;
    k_wscan<<<P, kWScanThreads, 0, st>>>(pinfo, a2, a1, a0, counts);
    return 1;
}

// Per-lane bisection / safeguarded Newton in k.  A warp owns a work item of
// <= 32 consecutive eigen-indices of one problem, lane l eigen-index
// c_lo + j0 + l, bracket [a, b] from the isolation scan.  Each round every
// lane sweeps the grid once at its own point, carrying the Sturm count and
// the k-derivative of the recurrence: a lane whose bracket still holds more
// than one eigenvalue moves to the midpoint, an isolated one takes a Newton
// step on det T(k) (falling back to the midpoint outside the bracket).  A
// lane is final when the bracket or the correction is below tol relative to
// k, or when the quadratic-convergence model predicts the next correction
// below it (two in-bracket steps, fourfold shrink).
__global__ void __launch_bounds__(kWWarps * 32) k_wbisect(const ProblemInfo* __restrict__ pinfo,
                                                          const double* __restrict__ a2,
                                                          const double* __restrict__ a1,
                                                          const double* __restrict__ a0,
                                                          const int* __restrict__ counts,
                                                          const WorkItem* __restrict__ items,
                                                          const int* __restrict__ n_items_dev, double tol,
                                                          double* __restrict__ mu) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int n_items = *n_items_dev;
    const int warps_total = gridDim.x * kWWarps;
    for (int it = blockIdx.x * kWWarps + wid; it < n_items; it += warps_total) {
        const WorkItem w = items[it];
        const ProblemInfo pi = pinfo[w.problem];
        const int* cnt = counts + (size_t)w.problem * kScanPoints;
        const double* r2 = a2 + pi.s_off;
        const double* r1 = a1 + pi.s_off;
        const double* r0 = a0 + pi.s_off;
        const int J = pi.c_lo + w.j0 + lane;
        double a = pi.k_min, b = pi.k_min, x = pi.k_min, dprev = 0.0;
        int ca = 0, cb = 0, mode = 2;  // 0 bisect, 1 Newton, 2 final
        if (lane < w.m) {
            int t0 = 0;
            for (int t = 0; t < kScanPoints; ++t)
                if (cnt[t] <= J) t0 = t;
            int t1 = kScanPoints - 1;
            for (int t = kScanPoints - 1; t > t0; --t)
                if (cnt[t] > J) t1 = t;
            a = wscan_x(pi.k_min, pi.k_max, t0);
            b = wscan_x(pi.k_min, pi.k_max, t1);
            ca = cnt[t0];
            cb = cnt[t1];
            x = 0.5 * (a + b);
            mode = (ca == J && cb == J + 1) ? 1 : 0;
        }
        for (int round = 0; round < kWMaxRounds; ++round) {
            if (__ballot_sync(0xffffffffu, mode != 2) == 0u) break;
            // one sweep at x: count and det / d det
            double p0 = 0.0, p1 = 1.0, d0 = 0.0, d1 = 0.0;
            unsigned prev = 0u;
            int c = 0;
            for (int i = 0; i < pi.nz; ++i) {
                const double c2 = __ldg(r2 + i), c1 = __ldg(r1 + i), cc = __ldg(r0 + i);
                const double t = wdiag(c2, c1, cc, x);
                const double tp = fma(2.0 * c2, x, c1);
                const double e = fma(t, d1, fma(tp, p1, -d0));
                wstep(t, p0, p1, prev, c);
                d0 = d1;
                d1 = e;
                if ((i & 31) == 31) {
                    const int sh = rescale_shift(fmax(fabs(p0), fabs(d0)), fmax(fabs(p1), fabs(d1)));
                    if (sh) {
                        const double sc = pow2(-sh);
                        p0 *= sc;
                        p1 *= sc;
                        d0 *= sc;
                        d1 *= sc;
                    }
                }
            }
            if (mode == 0) {
                if (c <= J) {
                    a = x;
                    ca = c;
                } else {
                    b = x;
                    cb = c;
                }
                if (!(b - a > tol * b)) mode = 2;
                else if (ca == J && cb == J + 1) mode = 1;
                x = 0.5 * (a + b);
            } else if (mode == 1) {
                if (c <= J) {
                    a = x;
                    ca = c;
                } else {
                    b = x;
                    cb = c;
                }
                const double rN = p1 / d1;
                const double ad = fabs(rN);
                if (ad <= tol * x) {
                    x = fmin(fmax(x - rN, a), b);
                    mode = 2;
                } else {
                    const double xn = x - rN;
                    const bool ok = isfinite(xn) && xn > a && xn < b;
                    x = ok ? xn : 0.5 * (a + b);
                    if (!(b - a > tol * b)) {
                        mode = 2;
                    } else if (ok && dprev > 0.0 && ad <= 0.25 * dprev &&
                               ad * ad * ad <= tol * x * dprev * dprev) {
                        mode = 2;
                    }
                    dprev = ok ? ad : 0.0;
                }
            }
        }
        if (lane < w.m) mu[pi.off + w.j0 + lane] = x;
    }
}

int launch_wbisect(cudaStream_t st, int grid, const ProblemInfo* pinfo, const double* a2, const double* a1,
                   const double* a0, const int* counts, const WorkItem* items, const int* n_items_dev, double tol,
                   double* mu) {
    if (grid <= 0) return 0;
    k_wbisect<<<grid, kWWarps * 32, 0, st>>>(pinfo, a2, a1, a0, counts, items, n_items_dev, tol, mu);
    return 1;
}

// order-preserving key of |v| 2^e for the twist search (biased exponent plus
// e, then the top 20 mantissa bits)
__device__ __forceinline__ long long wmag_key(double v, int e) {
    v = fabs(v);
    if (v == 0.0) return -(1ll << 62);
    const long long bits = __double_as_longlong(v);
    const int be = (int)((bits >> 52) & 0x7ff);
    return (long long)(be + e) * 1048576ll + ((bits >> 32) & 0xfffff);
}

// Eigenvectors of T(k) at the converged k by twisted factorisation, one lane
// per eigenvalue, a warp per work item of <= 32 eigenvalues: pass 1 runs the
// backward recurrence q_i = t_i q_{i+1} - q_{i+2} (q_n = 1) and stores q (with
// its power-of-two exponent) in this warp's scratch slot, laid out [row][lane]
// so each store is 256 contiguous bytes; pass 2 runs the forward recurrence,
// picks the twist r maximising |p_{r-1} q_{r+1}| and accumulates
// sum z^2 and sum z^2 w below r (snapshot at each new maximum) and above r
// (from the stored q); an optional pass 3 writes the normalised vector.  The
// vector is scaled to sum v^2 dz = 1/(1+k^2), the normalisation of SLEPc's
// unit-2-norm eigenvectors of the linearised pencil [v; k v]
// (EigenEngine.cpp:368-379), and k_pert = sqrt(k^2 + i sum v^2 w dz)
// (ModeSolver::doPerturb, ModeSolver.cpp:263-284).
__global__ void __launch_bounds__(kWWarps * 32) k_weigvec(WmodEvArgs A) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int n_items = *A.n_items_dev;
    const int warps_total = gridDim.x * kWWarps;
    const size_t slot = (size_t)blockIdx.x * kWWarps + wid;
    double* qs = A.q_scr + slot * A.slot_stride;
    int* es = A.e_scr + slot * A.slot_stride;
    for (int it = blockIdx.x * kWWarps + wid; it < n_items; it += warps_total) {
        const WorkItem w = A.items[it];
        const ProblemInfo pi = A.pinfo[w.problem];
        const int n = pi.nz;
        const double* r2 = A.a2 + pi.s_off;
        const double* r1 = A.a1 + pi.s_off;
        const double* r0 = A.a0 + pi.s_off;
        const double* wp = A.w + pi.w_off;
        const bool active = lane < w.m;
        const double k = active ? A.mu[pi.off + w.j0 + lane] : pi.k_min;
        // ---- pass 1: backward, q_i stored at row i (i = 0 .. n) ----
        {
            double q2 = 0.0, q1 = 1.0;
            int E = 0;
            qs[(size_t)n * 32 + lane] = 1.0;
            es[(size_t)n * 32 + lane] = 0;
            for (int i = n - 1; i >= 0; --i) {
                const double qi = fma(wdiag(__ldg(r2 + i), __ldg(r1 + i), __ldg(r0 + i), k), q1, -q2);
                qs[(size_t)i * 32 + lane] = qi;
                es[(size_t)i * 32 + lane] = E;
                q2 = q1;
                q1 = qi;
                if ((i & 15) == 0) {
                    const int sh = grow_shift(q1, q2);
                    if (sh) {
                        const double sc = pow2(-sh);
                        q1 *= sc;
                        q2 *= sc;
                        E += sh;
                    }
                }
            }
        }
        __syncwarp();
        // ---- pass 2: forward, twist and sums ----
        double pm2 = 0.0, pm1 = 1.0;
        int Ep = 0;
        double An = 0.0, Aw = 0.0;
        long long best = -(1ll << 62) - 1;
        int r = 0, Epr = 0, Eqr = 0;
        double Fn = 0.0, Fw = 0.0, pr = 1.0, inv_qr = 1.0, Tn = 0.0, Tw = 0.0;
        double ps_src = 0.0, ps_rcv = 0.0, qr_src = 0.0, qr_rcv = 0.0;
        int Eps_src = 0, Eps_rcv = 0;
        for (int i = 0; i < n; ++i) {
            const double sq = pm1 * pm1;
            const double wi = __ldg(wp + i);
            An += sq;
            Aw += sq * wi;
            const double qn = qs[(size_t)(i + 1) * 32 + lane];
            const int eqn = es[(size_t)(i + 1) * 32 + lane];
            const long long key = wmag_key(pm1 * qn, Ep + eqn);
            if (key > best) {
                best = key;
                r = i;
                Fn = An / sq;
                Fw = Aw / sq;
                pr = pm1;
                Epr = Ep;
                inv_qr = 1.0 / qn;
                Eqr = eqn;
                Tn = Tw = 0.0;
            } else {
                const double t = scalbn(qn * inv_qr, eqn - Eqr);
                const double t2 = t * t;
                Tn += t2;
                Tw += t2 * wi;
            }
            if (i == pi.isrc) {
                ps_src = pm1;
                Eps_src = Ep;
                qr_src = (r < i) ? scalbn(qn * inv_qr, eqn - Eqr) : 1.0;
            }
            if (i == pi.ircv) {
                ps_rcv = pm1;
                Eps_rcv = Ep;
                qr_rcv = (r < i) ? scalbn(qn * inv_qr, eqn - Eqr) : 1.0;
            }
            const double p = fma(wdiag(__ldg(r2 + i), __ldg(r1 + i), __ldg(r0 + i), k), pm1, -pm2);
            pm2 = pm1;
            pm1 = p;
            if ((i & 15) == 15) {
                const int sh = grow_shift(pm1, pm2);
                if (sh) {
                    const double sc = pow2(-sh), sc2 = pow2(-2 * sh);
                    pm1 *= sc;
                    pm2 *= sc;
                    An *= sc2;
                    Aw *= sc2;
                    Ep += sh;
                }
            }
        }
        const double nrm = Fn + Tn;  // sum z^2 / z_r^2
        const double f = 1.0 / sqrt(1.0 + k * k);
        const double scale = f / sqrt(nrm * pi.dz);
        double zs = (pi.isrc <= r) ? scalbn(ps_src / pr, Eps_src - Epr) : qr_src;
        double zr = (pi.ircv <= r) ? scalbn(ps_rcv / pr, Eps_rcv - Epr) : qr_rcv;
        if ((pi.isrc - r) & 1) zs = -zs;
        if ((pi.ircv - r) & 1) zr = -zr;
        const double absorption = (Fw + Tw) / nrm * (f * f);
        const auto kp = csqrt_principal(k * k, absorption);
        if (active) {
            const int o = pi.off + w.j0 + lane;
            A.kr[o] = kp.real();
            A.ki[o] = kp.imag();
            A.vs[o] = zs * scale;
            A.vr[o] = zr * scale;
            if (A.vg) A.vg[o] = 0.0;
        }
        // ---- pass 3 (optional): the normalised vector ----
        if (A.vfull) {
            double* vout = A.vfull + A.vfull_off[w.problem];
            const int M = pi.M;
            double qa = 0.0, qb = 1.0;
            int Ea = 0;
            const double qref = 1.0 / inv_qr;
            for (int i = 0; i < n; ++i) {
                double zi;
                if (i <= r) {
                    zi = scalbn(qb / pr, Ea - Epr);
                } else {
                    zi = scalbn(qs[(size_t)(i + 1) * 32 + lane] / qref, es[(size_t)(i + 1) * 32 + lane] - Eqr);
                }
                if ((i - r) & 1) zi = -zi;
                if (active) vout[(size_t)i * M + w.j0 + lane] = zi * scale;
                const double p = fma(wdiag(__ldg(r2 + i), __ldg(r1 + i), __ldg(r0 + i), k), qb, -qa);
                qa = qb;
                qb = p;
                if ((i & 15) == 15) {
                    const int sh = grow_shift(qb, qa);
                    if (sh) {
                        const double sc = pow2(-sh);
                        qa *= sc;
                        qb *= sc;
                        Ea += sh;
                    }
                }
            }
        }
        __syncwarp();
    }
}

int launch_weigvec(cudaStream_t st, int grid, const WmodEvArgs& a) {
    if (grid <= 0) return 0;
    k_weigvec<<<grid, kWWarps * 32, 0, st>>>(a);
    return 1;
}

int wmod_warps_per_cta() { return kWWarps; }

}  // namespace ncpa
