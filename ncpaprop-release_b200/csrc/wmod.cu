// Wide-angle (WMod) normal modes: the quadratic eigenproblem
// (M k^2 + C k + D) v = 0 of WModeSolver::solve (WModeSolver.cpp:257-486),
// which the reference linearises to a 2N pencil and hands to SLEPc
// (EigenEngine::doWideAngleCalculation, EigenEngine.cpp:174-395).
//
// Here T(k) h^2 has unit off-diagonal and diagonal
//   t_i = (B_i - U_i kappa)^2 - kappa^2 - 2,  kappa = h k,
//   B_i = h omega / c0_i,  U_i = wc_i / c0_i,
// plus the ground term g0 in row 0: the polynomial a2 k^2 + a1 k + a0 of
// WModeSolver.cpp:544-565 (a2 = (U^2 - 1) h^2, a1 = -2 omega U / c0 h^2,
// a0 = (omega / c0)^2 h^2 - 2; no last-row repeat, EigenEngine.cpp:266-275)
// in factored form, two doubles per row.  For real k inside the propagating
// window dT/dk is negative definite (subsonic winds), so the number of
// negative eigenvalues of T grows by one at each real eigenvalue: the modes
// are found with Sturm counts in kappa (isolation scan, then per-lane
// bisection / safeguarded Newton on det T with its kappa-derivative) and each
// eigenvector is the null vector of T by twisted factorisation (k_eigvec with
// the WmodRows format, kernels.cu).  Every sweep streams the rows through
// shared memory by TMA bulk copies.
#include "device_common.cuh"
#include "kernels.hpp"

namespace ncpa {

namespace {

constexpr int kWScanThreads = kScanPoints / 2;  // two shifts per thread
constexpr int kWsRows = 512;                    // rows per scan ring chunk (8 KB)
constexpr int kWsBuf = 4;                       // scan ring slots
constexpr int kWbRows = 256;                    // rows per bisection ring chunk (4 KB)
constexpr int kWbBuf = 3;                       // bisection ring slots per warp
constexpr int kWbWarps = 4;                     // warps per bisection CTA
constexpr int kWMaxRounds = 400;                // bound on bisection / Newton rounds

__device__ __forceinline__ double wscan_x(double lo, double hi, int t) {
    if (t == 0) return lo;
    if (t == kScanPoints - 1) return hi;
    return lo + (hi - lo) * ((double)t / (double)(kScanPoints - 1));
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

// Rows (B_i, U_i) of one group's problems (nz_pad rows apart, problem p =
// frequency-major over n_az azimuths) on the sampling grid z_min + i dz_grid
// (WModeSolver.cpp:196-208), with the matrix spacing dz, and the ground term
// g0 = h^2 / (dz^2 (dz admittance + 1)); also (omega/c_eff)^2 for the WKB
// search and the c_eff extrema / ground / top values of getModalTrace
// (WModeSolver.cpp:530-629).  Padding rows are zero.
__global__ void __launch_bounds__(256) k_wmod_build(int nk, const double* __restrict__ zk,
                                                    const double* __restrict__ c0k, const double* __restrict__ c0c,
                                                    const double* __restrict__ wck, const double* __restrict__ wcc,
                                                    const double* __restrict__ ceffk,
                                                    const double* __restrict__ ceffc, int n_az,
                                                    ProblemInfo* __restrict__ pinfo, int nz, int nz_pad,
                                                    double z_min, double dz_grid, double dz, double admittance,
                                                    double2* __restrict__ rows, double* __restrict__ kz2) {
    const int p = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int az = p % n_az;
    const double omega = pinfo[p].omega;
    double cmin = 1e300, cmax = -1e300;
    if (i >= nz && i < nz_pad) rows[(size_t)p * nz_pad + i] = make_double2(0.0, 0.0);
    if (i < nz) {
        const double z = z_min + i * dz_grid;
        const double c0 = spline_get(nk, zk, c0k, c0c, z);
        const double wc = spline_get(nk, zk, wck + (size_t)az * nk, wcc + (size_t)az * 4 * (nk - 1), z);
        const double ce = spline_get(nk, zk, ceffk + (size_t)az * nk, ceffc + (size_t)az * 4 * (nk - 1), z);
        const size_t o = (size_t)p * nz_pad + i;
        rows[o] = make_double2(dz * (omega / c0), wc / c0);
        if (i == 0) pinfo[p].g0 = 1.0 / (dz * admittance + 1.0);
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
                      double admittance, double* rows, double* kz2) {
    dim3 grid((nz_pad + 255) / 256, P);
    k_wmod_build<<<grid, 256, 0, st>>>(nk, zk, c0k, c0c, wck, wcc, ceffk, ceffc, n_az, pinfo, nz, nz_pad, z_min,
                                       dz_grid, dz, admittance, reinterpret_cast<double2*>(rows), kz2);
    return 1;
}


// ---------------------------------------------------------------------------
// Sturm sweeps over the rows.  p_{-2} = -g0, p_{-1} = 1,
// p_i = t_i(kappa) p_{i-1} - p_{i-2}; a negative pivot is a sign change of
// consecutive p.  The kappa-derivative runs as e_i = t_i e_{i-1} +
// (U_i d_i + kappa) p_{i-1} - e_{i-2} with d_i = B_i - U_i kappa, which is
// -1/2 of d p_i / d kappa, so Newton's step is kappa + p / (2 e).
// ---------------------------------------------------------------------------
struct WChain {
    double p0, p1;
    unsigned prevbit;
    int cnt;
    __device__ __forceinline__ void reset(double g0) {
        p0 = -g0;
        p1 = 1.0;
        prevbit = 0u;
        cnt = 0;
    }
    __device__ __forceinline__ void fold(unsigned w) {
        const unsigned prev = (w >> 1) | (prevbit << 31);
        cnt += __popc(w ^ prev);
        prevbit = w & 1u;
    }
    __device__ __forceinline__ void step(double2 r, const WmodRows::Shift& s) {
        const double d = fma(-r.y, s.kap, r.x);
        const double q = fma(fma(d, d, s.c), p1, -p0);
        const unsigned b = static_cast<unsigned>(__double2hiint(q)) >> 31;
        cnt += static_cast<int>(b ^ prevbit);
        prevbit = b;
        p0 = p1;
        p1 = q;
    }
};

__device__ __forceinline__ void wchain_rescale(WChain& A) {
    const int sh = rescale_shift(A.p0, A.p1);
    if (sh) {
        const double sc = pow2(-sh);
        A.p0 *= sc;
        A.p1 *= sc;
    }
}

// 32 rows, two chains interleaved (counts only)
__device__ __forceinline__ void wword32_pair(WChain& A, WChain& B, const double2* __restrict__ r,
                                             const WmodRows::Shift& sa, const WmodRows::Shift& sb) {
    unsigned wa = 0u, wb = 0u;
    double pa0 = A.p0, pa1 = A.p1, pb0 = B.p0, pb1 = B.p1;
#pragma unroll
    for (int u = 0; u < 32; ++u) {
        const double2 rv = r[u];
        const double da = fma(-rv.y, sa.kap, rv.x);
        const double db = fma(-rv.y, sb.kap, rv.x);
        const double qa = fma(fma(da, da, sa.c), pa1, -pa0);
        const double qb = fma(fma(db, db, sb.c), pb1, -pb0);
        wa = __funnelshift_l(__double2hiint(qa), wa, 1);
        wb = __funnelshift_l(__double2hiint(qb), wb, 1);
        pa0 = pa1;
        pa1 = qa;
        pb0 = pb1;
        pb1 = qb;
    }
    A.p0 = pa0;
    A.p1 = pa1;
    B.p0 = pb0;
    B.p1 = pb1;
    A.fold(wa);
    B.fold(wb);
    wchain_rescale(A);
    wchain_rescale(B);
}

// 32 rows, one chain (counts only)
__device__ __forceinline__ void wword32(WChain& A, const double2* __restrict__ r, const WmodRows::Shift& sa) {
    unsigned wa = 0u;
    double pa0 = A.p0, pa1 = A.p1;
#pragma unroll
    for (int u = 0; u < 32; ++u) {
        const double2 rv = r[u];
        const double da = fma(-rv.y, sa.kap, rv.x);
        const double qa = fma(fma(da, da, sa.c), pa1, -pa0);
        wa = __funnelshift_l(__double2hiint(qa), wa, 1);
        pa0 = pa1;
        pa1 = qa;
    }
    A.p0 = pa0;
    A.p1 = pa1;
    A.fold(wa);
    wchain_rescale(A);
}

// 32 rows, one chain with its derivative chain (e0, e1)
__device__ __forceinline__ void wword32_deriv(WChain& A, double& e0, double& e1, const double2* __restrict__ r,
                                              const WmodRows::Shift& sa) {
    unsigned wa = 0u;
    double pa0 = A.p0, pa1 = A.p1;
#pragma unroll
    for (int u = 0; u < 32; ++u) {
        const double2 rv = r[u];
        const double da = fma(-rv.y, sa.kap, rv.x);
        const double ta = fma(da, da, sa.c);
        const double tp = fma(rv.y, da, sa.kap);
        const double qa = fma(ta, pa1, -pa0);
        const double ea = fma(ta, e1, fma(tp, pa1, -e0));
        wa = __funnelshift_l(__double2hiint(qa), wa, 1);
        pa0 = pa1;
        pa1 = qa;
        e0 = e1;
        e1 = ea;
    }
    A.p0 = pa0;
    A.p1 = pa1;
    A.fold(wa);
    const int sh = rescale_shift(fmax(fabs(A.p0), fabs(e0)), fmax(fabs(A.p1), fabs(e1)));
    if (sh) {
        const double sc = pow2(-sh);
        A.p0 *= sc;
        A.p1 *= sc;
        e0 *= sc;
        e1 *= sc;
    }
}

__device__ __forceinline__ void wstep_deriv(WChain& A, double& e0, double& e1, double2 rv, const WmodRows::Shift& s) {
    const double d = fma(-rv.y, s.kap, rv.x);
    const double t = fma(d, d, s.c);
    const double tp = fma(rv.y, d, s.kap);
    const double q = fma(t, A.p1, -A.p0);
    const double e = fma(t, e1, fma(tp, A.p1, -e0));
    const unsigned b = static_cast<unsigned>(__double2hiint(q)) >> 31;
    A.cnt += static_cast<int>(b ^ A.prevbit);
    A.prevbit = b;
    A.p0 = A.p1;
    A.p1 = q;
    e0 = e1;
    e1 = e;
}

// ---------------------------------------------------------------------------
// Isolation scan: kScanPoints counts per problem on an even grid of
// [kappa_min, kappa_max] (the layout k_make_items reads); the CTA streams the
// rows through a kWsBuf-deep TMA ring, each thread runs two shifts.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kWScanThreads) k_wscan(const ProblemInfo* __restrict__ pinfo,
                                                         const double* __restrict__ rows, int* __restrict__ counts,
                                                         unsigned* err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    double2* buf = reinterpret_cast<double2*>(smem_raw);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + (size_t)kWsBuf * kWsRows * 16);
    if (threadIdx.x == 0) {
        for (int k = 0; k < kWsBuf; ++k) mbar_init(&bars[k], 1);
        fence_mbar_init();
    }
    __syncthreads();
    const int p = blockIdx.x;
    const ProblemInfo pi = pinfo[p];
    const double2* src = reinterpret_cast<const double2*>(rows) + pi.s_off;
    const double lo = pi.k_min * pi.dz, hi = pi.k_max * pi.dz;
    const int t0 = threadIdx.x, t1 = threadIdx.x + kWScanThreads;
    const WmodRows::Shift sa = WmodRows::shift(wscan_x(lo, hi, t0)), sb = WmodRows::shift(wscan_x(lo, hi, t1));
    const int nz = pi.nz;
    const int nch = (nz + kWsRows - 1) / kWsRows;
    if (threadIdx.x == 0)
        for (int c = 0; c < nch && c < kWsBuf; ++c) {
            mbar_expect_tx(&bars[c], kWsRows * 16);
            tma_load_1d(buf + (size_t)c * kWsRows, src + (size_t)c * kWsRows, kWsRows * 16, &bars[c]);
        }
    WChain A, B;
    A.reset(pi.g0);
    B.reset(pi.g0);
    for (int c = 0; c < nch; ++c) {
        const int slot = c % kWsBuf;
        mbar_wait_bounded(&bars[slot], (c / kWsBuf) & 1u, err);
        const double2* b = buf + (size_t)slot * kWsRows;
        const int valid = min(kWsRows, nz - c * kWsRows);
        const int nw = valid >> 5;
        for (int w = 0; w < nw; ++w) wword32_pair(A, B, b + 32 * w, sa, sb);
        for (int i = nw * 32; i < valid; ++i) {
            A.step(b[i], sa);
            B.step(b[i], sb);
        }
        __syncthreads();
        if (threadIdx.x == 0 && c + kWsBuf < nch) {
            fence_proxy_async();
            mbar_expect_tx(&bars[slot], kWsRows * 16);
            tma_load_1d(buf + (size_t)slot * kWsRows, src + (size_t)(c + kWsBuf) * kWsRows, kWsRows * 16,
                        &bars[slot]);
        }
    }
    counts[(size_t)p * kScanPoints + t0] = A.cnt;
    counts[(size_t)p * kScanPoints + t1] = B.cnt;
}

int launch_wscan(cudaStream_t st, int P, const ProblemInfo* pinfo, const double* rows, int* counts, unsigned* err) {
    if (P <= 0) return 0;
    const size_t sm = (size_t)kWsBuf * kWsRows * 16 + kWsBuf * 8;
    k_wscan<<<P, kWScanThreads, sm, st>>>(pinfo, rows, counts, err);
    return 1;
}

// ---------------------------------------------------------------------------
// Per-lane bisection / safeguarded Newton in kappa.  A warp owns a work item
// of <= 32 consecutive eigen-indices of one problem, lane l eigen-index
// c_lo + j0 + l, bracket [a, b] from the isolation scan, and streams the
// problem's rows through its own TMA ring (kWbBuf chunks of kWbRows rows), so
// warps never wait on each other.  Each round every lane sweeps the rows once
// at its own point: a lane whose bracket still holds more than one eigenvalue
// moves to the midpoint, an isolated one takes a Newton step on det T
// (falling back to the midpoint outside the bracket); the derivative chain
// runs only in rounds with a Newton lane.  A lane is final when the bracket
// or the correction is below tol relative to kappa, or when the
// quadratic-convergence model predicts the next correction below it (two
// in-bracket steps, fourfold shrink).
// ---------------------------------------------------------------------------
struct WbRing {
    double2* buf;    // [kWbBuf][kWbRows]
    uint64_t* bars;  // [kWbBuf]
    unsigned loads;  // identical in all lanes
};

__device__ __forceinline__ void wbr_issue(WbRing& r, unsigned k, const double2* src) {
    const int slot = k % kWbBuf;
    mbar_expect_tx(&r.bars[slot], kWbRows * 16);
    tma_load_1d(r.buf + (size_t)slot * kWbRows, src, kWbRows * 16, &r.bars[slot]);
}

// one sweep of the warp's rows at this lane's shift; ratio = p / e (when
// deriv) for the Newton step kappa + ratio / 2
__device__ void wb_sweep(const double2* __restrict__ src, int nz, double g0, const WmodRows::Shift& sh, bool deriv,
                         WbRing& r, unsigned* err, int& cnt, double& ratio) {
    const int lane = threadIdx.x & 31;
    const int nch = (nz + kWbRows - 1) / kWbRows;
    const unsigned base = r.loads;
    if (lane == 0)
        for (int c = 0; c < nch && c < kWbBuf; ++c) wbr_issue(r, base + c, src + (size_t)c * kWbRows);
    __syncwarp();
    WChain A;
    A.reset(g0);
    double e0 = 0.0, e1 = 0.0;
    for (int c = 0; c < nch; ++c) {
        const unsigned k = base + c;
        const int slot = k % kWbBuf;
        mbar_wait_bounded(&r.bars[slot], (k / kWbBuf) & 1u, err);
        const double2* b = r.buf + (size_t)slot * kWbRows;
        const int valid = min(kWbRows, nz - c * kWbRows);
        const int nw = valid >> 5;
        if (deriv) {
            for (int w = 0; w < nw; ++w) wword32_deriv(A, e0, e1, b + 32 * w, sh);
            for (int i = nw * 32; i < valid; ++i) wstep_deriv(A, e0, e1, b[i], sh);
        } else {
            for (int w = 0; w < nw; ++w) wword32(A, b + 32 * w, sh);
            for (int i = nw * 32; i < valid; ++i) A.step(b[i], sh);
        }
        __syncwarp();
        if (lane == 0 && c + kWbBuf < nch) {
            fence_proxy_async();
            wbr_issue(r, base + c + kWbBuf, src + (size_t)(c + kWbBuf) * kWbRows);
        }
    }
    r.loads = base + nch;
    cnt = A.cnt;
    ratio = deriv ? A.p1 / e1 : 0.0;
}

__global__ void __launch_bounds__(kWbWarps * 32) k_wbisect(const ProblemInfo* __restrict__ pinfo,
                                                           const double* __restrict__ rows,
                                                           const int* __restrict__ counts,
                                                           const WorkItem* __restrict__ items,
                                                           const int* __restrict__ n_items_dev, double tol,
                                                           double* __restrict__ mu, unsigned* err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WbRing r;
    r.buf = reinterpret_cast<double2*>(smem_raw) + (size_t)wid * kWbBuf * kWbRows;
    r.bars = reinterpret_cast<uint64_t*>(smem_raw + (size_t)kWbWarps * kWbBuf * kWbRows * 16) + wid * kWbBuf;
    r.loads = 0;
    if (lane == 0) {
        for (int k = 0; k < kWbBuf; ++k) mbar_init(&r.bars[k], 1);
        fence_mbar_init();
    }
    __syncwarp();
    const int n_items = *n_items_dev;
    const int warps_total = gridDim.x * kWbWarps;
    for (int it = blockIdx.x * kWbWarps + wid; it < n_items; it += warps_total) {
        const WorkItem w = items[it];
        const ProblemInfo pi = pinfo[w.problem];
        const int* cnt = counts + (size_t)w.problem * kScanPoints;
        const double2* src = reinterpret_cast<const double2*>(rows) + pi.s_off;
        const double lo = pi.k_min * pi.dz, hi = pi.k_max * pi.dz;
        const int J = pi.c_lo + w.j0 + lane;
        double a = lo, b = lo, x = lo, dprev = 0.0;
        int ca = 0, cb = 0, mode = 2;  // 0 bisect, 1 Newton, 2 final
        if (lane < w.m) {
            int t0 = 0;
            for (int t = 0; t < kScanPoints; ++t)
                if (cnt[t] <= J) t0 = t;
            int t1 = kScanPoints - 1;
            for (int t = kScanPoints - 1; t > t0; --t)
                if (cnt[t] > J) t1 = t;
            if (cnt[t1] <= J) atomicOr(err, kErrBracket);
            a = wscan_x(lo, hi, t0);
            b = wscan_x(lo, hi, t1);
            ca = cnt[t0];
            cb = cnt[t1];
            x = 0.5 * (a + b);
            mode = (ca == J && cb == J + 1) ? 1 : 0;
        }
        for (int round = 0; round < kWMaxRounds; ++round) {
            if (__ballot_sync(0xffffffffu, mode != 2) == 0u) break;
            const bool deriv = __any_sync(0xffffffffu, mode == 1);
            int c;
            double ratio;
            wb_sweep(src, pi.nz, pi.g0, WmodRows::shift(x), deriv, r, err, c, ratio);
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
                const double step = 0.5 * ratio;  // kappa_new = x + step
                const double ad = fabs(step);
                if (ad <= tol * x) {
                    x = fmin(fmax(x + step, a), b);
                    mode = 2;
                } else {
                    const double xn = x + step;
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
            // a ring wait gave up: abandon the item (warp-uniform decision)
            if (__any_sync(0xffffffffu, (*((volatile unsigned*)err) & kErrTimeout) != 0u)) break;
        }
        if (lane < w.m) mu[pi.off + w.j0 + lane] = x;
    }
}

static size_t wbisect_smem() { return (size_t)kWbWarps * (kWbBuf * kWbRows * 16 + kWbBuf * 8); }

int launch_wbisect(cudaStream_t st, int grid, const ProblemInfo* pinfo, const double* rows, const int* counts,
                   const WorkItem* items, const int* n_items_dev, double tol, double* mu, unsigned* err) {
    if (grid <= 0) return 0;
    const size_t sm = wbisect_smem();
    cudaFuncSetAttribute(k_wbisect, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_wbisect<<<grid, kWbWarps * 32, sm, st>>>(pinfo, rows, counts, items, n_items_dev, tol, mu, err);
    return 1;
}

int wbisect_ctas_per_sm() {
    int n = 1;
    const size_t sm = wbisect_smem();
    cudaFuncSetAttribute(k_wbisect, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_wbisect, kWbWarps * 32, sm) != cudaSuccess) n = 1;
    return n < 1 ? 1 : n;
}

}  // namespace ncpa
