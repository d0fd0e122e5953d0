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
// are found with Sturm counts in kappa (the isolation scan here, then the
// multisection / safeguarded Newton of k_bisect on det T with its
// kappa-derivative) and each eigenvector is the null vector of T by twisted
// factorisation (k_bisect and k_eigvec with the WmodRows format,
// kernels.cu).  Every sweep streams the rows through shared memory by TMA
// bulk copies.
#include "device_common.cuh"
#include "kernels.hpp"

namespace ncpa {

namespace {

constexpr int kWScanThreads = kScanDefault / 2;  // two shifts per thread
constexpr int kWsRows = 512;                    // rows per scan ring chunk (8 KB)
constexpr int kWsBuf = 4;                       // scan ring slots

__device__ __forceinline__ double wscan_x(double lo, double hi, int t) {
    if (t == 0) return lo;
    if (t == kScanDefault - 1) return hi;
    return lo + (hi - lo) * ((double)t / (double)(kScanDefault - 1));
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
// (WModeSolver.cpp:530-629).  Padding rows are zero.  One thread per
// (azimuth, grid point) and kWbFreqs frequencies: the profile is sampled once.
constexpr int kWbFreqs = 16;

__global__ void __launch_bounds__(256) k_wmod_build(int nk, const double* __restrict__ zk,
                                                    const double* __restrict__ c0k, const double* __restrict__ c0c,
                                                    const double* __restrict__ wck, const double* __restrict__ wcc,
                                                    const double* __restrict__ ceffk,
                                                    const double* __restrict__ ceffc, int n_az, int n_f,
                                                    ProblemInfo* __restrict__ pinfo, int nz, int nz_pad,
                                                    double z_min, double dz_grid, double dz, double admittance,
                                                    double2* __restrict__ rows, double* __restrict__ kz2) {
    const int az = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int f0 = blockIdx.z * kWbFreqs, f1 = min(n_f, f0 + kWbFreqs);
    double cmin = 1e300, cmax = -1e300;
    const int top = nz - (nz / 10);
    const int itop = top + 1 < nz ? top + 1 : nz - 1;
    if (i >= nz && i < nz_pad)
        for (int f = f0; f < f1; ++f) rows[(size_t)(f * n_az + az) * nz_pad + i] = make_double2(0.0, 0.0);
    if (i < nz) {
        const double z = z_min + i * dz_grid;
        const double c0 = spline_get(nk, zk, c0k, c0c, z);
        const double wc = spline_get(nk, zk, wck + (size_t)az * nk, wcc + (size_t)az * 4 * (nk - 1), z);
        const double ce = spline_get(nk, zk, ceffk + (size_t)az * nk, ceffc + (size_t)az * 4 * (nk - 1), z);
        cmin = cmax = ce;
        for (int f = f0; f < f1; ++f) {
            const int p = f * n_az + az;
            const double omega = pinfo[p].omega;
            const size_t o = (size_t)p * nz_pad + i;
            rows[o] = make_double2(dz * (omega / c0), wc / c0);
            if (i == 0) pinfo[p].g0 = 1.0 / (dz * admittance + 1.0);
            if (kz2) {
                const double te = omega / ce;
                kz2[o] = te * te;
            }
            if (i == 0) pinfo[p].ceff_grnd = ce;
            if (i == itop) pinfo[p].ceff_top = ce;
        }
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
            for (int f = f0; f < f1; ++f) {
                const int p = f * n_az + az;
                atomicMin(&pinfo[p].ceffmin_bits, (unsigned long long)__double_as_longlong(cmin));
                atomicMax(&pinfo[p].ceffmax_bits, (unsigned long long)__double_as_longlong(cmax));
            }
        }
    }
}

int launch_wmod_build(cudaStream_t st, int nk, const double* zk, const double* c0k, const double* c0c,
                      const double* wck, const double* wcc, const double* ceffk, const double* ceffc, int n_az,
                      int P, ProblemInfo* pinfo, int nz, int nz_pad, double z_min, double dz_grid, double dz,
                      double admittance, double* rows, double* kz2) {
    if (n_az < 1 || P % n_az != 0) return -1;
    const int n_f = P / n_az;
    dim3 grid((nz_pad + 255) / 256, n_az, (n_f + kWbFreqs - 1) / kWbFreqs);
    k_wmod_build<<<grid, 256, 0, st>>>(nk, zk, c0k, c0c, wck, wcc, ceffk, ceffc, n_az, n_f, pinfo, nz, nz_pad, z_min,
                                       dz_grid, dz, admittance, reinterpret_cast<double2*>(rows), kz2);
    return 1;
}

// ---------------------------------------------------------------------------
// Isolation scan: kScanDefault counts per problem on an even grid of
// [kappa_min, kappa_max] (the layout k_make_items reads); the CTA streams the
// rows through a kWsBuf-deep TMA ring, each thread runs two shifts
// (WmodRows::pair: p_{-2} = -g0, p_{-1} = 1, p_i = t_i p_{i-1} - p_{i-2}).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kWScanThreads) k_wscan(const ProblemInfo* __restrict__ pinfo,
                                                         const double* __restrict__ rows, int* __restrict__ counts,
                                                         unsigned* err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    double* buf = reinterpret_cast<double*>(smem_raw);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + (size_t)kWsBuf * kWsRows * 16);
    if (threadIdx.x == 0) {
        for (int k = 0; k < kWsBuf; ++k) mbar_init(&bars[k], 1);
        fence_mbar_init();
    }
    __syncthreads();
    const int p = blockIdx.x;
    const ProblemInfo pi = pinfo[p];
    const double* src = rows + 2 * pi.s_off;
    const double lo = WmodRows::scan_lo(pi), hi = WmodRows::scan_hi(pi);
    const int t0 = threadIdx.x, t1 = threadIdx.x + kWScanThreads;
    const double xa = wscan_x(lo, hi, t0), xb = wscan_x(lo, hi, t1);
    const int nz = pi.nz;
    const int nch = (nz + kWsRows - 1) / kWsRows;
    if (threadIdx.x == 0)
        for (int c = 0; c < nch && c < kWsBuf; ++c) {
            mbar_expect_tx(&bars[c], kWsRows * 16);
            tma_load_1d(buf + (size_t)c * 2 * kWsRows, src + (size_t)c * 2 * kWsRows, kWsRows * 16, &bars[c]);
        }
    SturmState A, B;
    A.reset();
    B.reset();
    A.p0 = B.p0 = WmodRows::p_init(pi);
    for (int c = 0; c < nch; ++c) {
        const int slot = c % kWsBuf;
        mbar_wait_bounded(&bars[slot], (c / kWsBuf) & 1u, err);
        const double* b = buf + (size_t)slot * 2 * kWsRows;
        const int valid = min(kWsRows, nz - c * kWsRows);
        const int nw = valid >> 5;
        for (int w = 0; w < nw; ++w) WmodRows::pair(A, B, b + 64 * w, xa, xb);
        for (int i = nw * 32; i < valid; ++i) {
            WmodRows::step(A, b, i, xa);
            WmodRows::step(B, b, i, xb);
        }
        __syncthreads();
        if (threadIdx.x == 0 && c + kWsBuf < nch) {
            fence_proxy_async();
            mbar_expect_tx(&bars[slot], kWsRows * 16);
            tma_load_1d(buf + (size_t)slot * 2 * kWsRows, src + (size_t)(c + kWsBuf) * 2 * kWsRows, kWsRows * 16,
                        &bars[slot]);
        }
    }
    counts[(size_t)p * kScanMax + t0] = A.cnt;
    counts[(size_t)p * kScanMax + t1] = B.cnt;
}

int launch_wscan(cudaStream_t st, int P, const ProblemInfo* pinfo, const double* rows, int* counts, unsigned* err) {
    if (P <= 0) return 0;
    const size_t sm = (size_t)kWsBuf * kWsRows * 16 + kWsBuf * 8;
    k_wscan<<<P, kWScanThreads, sm, st>>>(pinfo, rows, counts, err);
    return 1;
}

}  // namespace ncpa
