// Device helpers shared by the sm_100a kernels of the ESS normal-mode path.
//
// Arithmetic conventions: the library is compiled with --fmad=false, so a
// fused multiply-add appears only where fma() is written.  Any CPU code that
// performs the same operations in the same order without contraction
// (-ffp-contract=off) reproduces the profile sampling, matrix build and Sturm
// counts bit-for-bit.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include <cuda/std/complex>

#include "kernels.hpp"

namespace ncpa {

constexpr double kPi = 3.141592653589793;  // value of PI in src/common/util.h:13-14


// ---------------------------------------------------------------------------
// Steffen monotone cubic on non-uniform knots (gsl_interp_steffen as used by
// src/atmosphere/AtmosphericProperty1D.cpp:72-136).  coef[4i..4i+3] = a,b,c,d
// with y = d + t (c + t (b + t a)), t = x - x_i.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int knot_search(int n, const double* __restrict__ x, double xq) {
    int lo = 0, hi = n - 1;
    while (hi > lo + 1) {
        int mid = (lo + hi) >> 1;
        if (x[mid] > xq) hi = mid; else lo = mid;
    }
    return lo;
}

__device__ __forceinline__ double spline_get(int n, const double* __restrict__ x,
                                             const double* __restrict__ y,
                                             const double* __restrict__ coef, double xq) {
    if (xq > x[n - 1]) return y[n - 1];
    if (xq < x[0]) return y[0];
    int i = knot_search(n, x, xq);
    const double* c = coef + 4 * i;
    double t = xq - x[i];
    return c[3] + t * (c[2] + t * (c[1] + t * c[0]));
}

__device__ __forceinline__ double spline_deriv(int n, const double* __restrict__ x,
                                               const double* __restrict__ coef, double xq) {
    if (xq > x[n - 1] || xq < x[0]) return 0.0;
    int i = knot_search(n, x, xq);
    const double* c = coef + 4 * i;
    double t = xq - x[i];
    return c[2] + t * (2.0 * c[1] + t * 3.0 * c[0]);
}

// ---------------------------------------------------------------------------
// power-of-two rescaling (exact)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int biased_exp(double v) {
    return (__double2hiint(v) >> 20) & 0x7ff;
}
// shift e such that max(|a|,|b|) * 2^-e is near 1, or 0 when inside 2^+-480
__device__ __forceinline__ int rescale_shift(double a, double b) {
    int e = max(biased_exp(a), biased_exp(b));
    if (e == 0) return 0;
    e -= 1023;
    return (e > 480 || e < -480) ? e : 0;
}
// overflow-only variant for recurrences whose squares are accumulated: keeps
// |a|,|b| below 2^240 so that sums of squares stay finite
__device__ __forceinline__ int grow_shift(double a, double b) {
    int e = max(biased_exp(a), biased_exp(b)) - 1023;
    return e > 240 ? e : 0;
}
// 2^k as a double; 0 below the normal range, +inf above it
__device__ __forceinline__ double pow2(int k) {
    if (k < -1022) return 0.0;
    if (k > 1023) return __longlong_as_double(0x7ff0000000000000ll);
    return __hiloint2double((k + 1023) << 20, 0);
}

// ---------------------------------------------------------------------------
// TMA bulk copies (cp.async.bulk, non-tensor) into shared memory with an
// mbarrier transaction count, and bounded waits.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// global -> shared bulk copy; dst, src 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait: gives up after one second of wall time (or at once when
// another wait of this launch already gave up), records kErrTimeout and
// returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, unsigned* err) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > 1000000000ull || (*((volatile unsigned*)err) & kErrTimeout)) break;
    }
    atomicOr(err, kErrTimeout);
    return false;
}

// Bounded wait for copies this block issued itself, used on the way out after
// another wait gave up: one second of wall time whatever the error word says.
__device__ __forceinline__ bool mbar_wait_drain(uint64_t* bar, uint32_t parity) {
    const uint64_t t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > 1000000000ull) return false;
    return true;
}

// ---------------------------------------------------------------------------
// Division-free Sturm sweep.  Matrix S = h^2 A: diagonal s_i, unit
// off-diagonal.  p_{-2}=0, p_{-1}=1, p_i = (s_i - x) p_{i-1} - p_{i-2};
// negative LDL^T pivot i <=> sign(p_i) != sign(p_{i-1}).  The sign bits of
// 32 consecutive p_i are packed with a funnel shift and the changes counted
// with one popc per word.
// ---------------------------------------------------------------------------
struct SturmState {
    double p0, p1;      // p_{i-2}, p_{i-1}
    unsigned prevbit;   // sign bit of p_{i-1}
    int cnt;
    __device__ __forceinline__ void reset() {
        p0 = 0.0;
        p1 = 1.0;
        prevbit = 0u;
        cnt = 0;
    }
    // 32 steps from s[0..31] (16-byte aligned shared memory)
    __device__ __forceinline__ void word32(const double* __restrict__ s, double x) {
        unsigned w = 0u;
#pragma unroll
        for (int u = 0; u < 32; u += 2) {
            double2 sv = *reinterpret_cast<const double2*>(s + u);
            double a0 = sv.x - x;
            double q0 = fma(a0, p1, -p0);
            double a1 = sv.y - x;
            double q1 = fma(a1, q0, -p1);
            w = __funnelshift_l(__double2hiint(q0), w, 1);
            w = __funnelshift_l(__double2hiint(q1), w, 1);
            p0 = q0;
            p1 = q1;
        }
        unsigned prev = (w >> 1) | (prevbit << 31);
        cnt += __popc(w ^ prev);
        prevbit = w & 1u;
        int sh = rescale_shift(p0, p1);
        if (sh) {
            double sc = pow2(-sh);
            p0 *= sc;
            p1 *= sc;
        }
    }
    // 32 steps carrying the x-derivative of the recurrence as well:
    // d_i = (s_i - x) d_{i-1} - (p_{i-1} + d_{i-2}); rescaled with p.  The sum
    // p_{i-1} + d_{i-2} is ready a step early, so the derivative chain costs
    // one dependent FMA per step, like p.
    __device__ __forceinline__ void word32_deriv(const double* __restrict__ s, double x, double& d0, double& d1) {
        unsigned w = 0u;
#pragma unroll
        for (int u = 0; u < 32; u += 2) {
            double2 sv = *reinterpret_cast<const double2*>(s + u);
            double a0 = sv.x - x;
            double q0 = fma(a0, p1, -p0);
            double e0 = fma(a0, d1, -(p1 + d0));
            double a1 = sv.y - x;
            double q1 = fma(a1, q0, -p1);
            double e1 = fma(a1, e0, -(q0 + d1));
            w = __funnelshift_l(__double2hiint(q0), w, 1);
            w = __funnelshift_l(__double2hiint(q1), w, 1);
            p0 = q0;
            p1 = q1;
            d0 = e0;
            d1 = e1;
        }
        unsigned prev = (w >> 1) | (prevbit << 31);
        cnt += __popc(w ^ prev);
        prevbit = w & 1u;
        int sh = rescale_shift(fmax(fabs(p0), fabs(d0)), fmax(fabs(p1), fabs(d1)));
        if (sh) {
            double sc = pow2(-sh);
            p0 *= sc;
            p1 *= sc;
            d0 *= sc;
            d1 *= sc;
        }
    }
    // 32 steps carrying the first and second x-derivatives:
    // e_i = (s_i - x) e_{i-1} - (2 d_{i-1} + e_{i-2}), rescaled with p
    __device__ __forceinline__ void word32_deriv2(const double* __restrict__ s, double x, double& d0, double& d1,
                                                  double& e0, double& e1) {
        unsigned w = 0u;
#pragma unroll
        for (int u = 0; u < 32; u += 2) {
            double2 sv = *reinterpret_cast<const double2*>(s + u);
            double a0 = sv.x - x;
            double q0 = fma(a0, p1, -p0);
            double f0 = fma(a0, d1, -(p1 + d0));
            double g0 = fma(a0, e1, -fma(2.0, d1, e0));
            double a1 = sv.y - x;
            double q1 = fma(a1, q0, -p1);
            double f1 = fma(a1, f0, -(q0 + d1));
            double g1 = fma(a1, g0, -fma(2.0, f0, e1));
            w = __funnelshift_l(__double2hiint(q0), w, 1);
            w = __funnelshift_l(__double2hiint(q1), w, 1);
            p0 = q0;
            p1 = q1;
            d0 = f0;
            d1 = f1;
            e0 = g0;
            e1 = g1;
        }
        unsigned prev = (w >> 1) | (prevbit << 31);
        cnt += __popc(w ^ prev);
        prevbit = w & 1u;
        int sh = rescale_shift(fmax(fmax(fabs(p0), fabs(d0)), fabs(e0)), fmax(fmax(fabs(p1), fabs(d1)), fabs(e1)));
        if (sh) {
            double sc = pow2(-sh);
            p0 *= sc;
            p1 *= sc;
            d0 *= sc;
            d1 *= sc;
            e0 *= sc;
            e1 *= sc;
        }
    }
    __device__ __forceinline__ void step_deriv2(double si, double x, double& d0, double& d1, double& e0,
                                                double& e1) {
        double a = si - x;
        double q = fma(a, p1, -p0);
        double f = fma(a, d1, -(p1 + d0));
        double g = fma(a, e1, -fma(2.0, d1, e0));
        unsigned b = static_cast<unsigned>(__double2hiint(q)) >> 31;
        cnt += static_cast<int>(b ^ prevbit);
        prevbit = b;
        p0 = p1;
        p1 = q;
        d0 = d1;
        d1 = f;
        e0 = e1;
        e1 = g;
    }
    __device__ __forceinline__ void step_deriv(double si, double x, double& d0, double& d1) {
        double a = si - x;
        double q = fma(a, p1, -p0);
        double e = fma(a, d1, -(p1 + d0));
        unsigned b = static_cast<unsigned>(__double2hiint(q)) >> 31;
        cnt += static_cast<int>(b ^ prevbit);
        prevbit = b;
        p0 = p1;
        p1 = q;
        d0 = d1;
        d1 = e;
    }
    // single guarded step (ragged tail)
    __device__ __forceinline__ void step(double si, double x) {
        double a = si - x;
        double q = fma(a, p1, -p0);
        unsigned b = static_cast<unsigned>(__double2hiint(q)) >> 31;
        cnt += static_cast<int>(b ^ prevbit);
        prevbit = b;
        p0 = p1;
        p1 = q;
    }
};

// Sign bits w of 32 steps (first step in bit 31) folded into a chain's count,
// then the exact power-of-two rescale of its last two values.
__device__ __forceinline__ void sturm_fold(SturmState& S, unsigned w) {
    const unsigned prev = (w >> 1) | (S.prevbit << 31);
    S.cnt += __popc(w ^ prev);
    S.prevbit = w & 1u;
    const int sh = rescale_shift(S.p0, S.p1);
    if (sh) {
        const double sc = pow2(-sh);
        S.p0 *= sc;
        S.p1 *= sc;
    }
}

// sign bits of 32 steps folded into a chain's count, then the joint exact
// power-of-two rescale of the chain and its derivative chain (d0, d1)
__device__ __forceinline__ void sturm_fold_deriv(SturmState& S, unsigned w, double& d0, double& d1) {
    const unsigned prev = (w >> 1) | (S.prevbit << 31);
    S.cnt += __popc(w ^ prev);
    S.prevbit = w & 1u;
    const int sh = rescale_shift(fmax(fabs(S.p0), fabs(d0)), fmax(fabs(S.p1), fabs(d1)));
    if (sh) {
        const double sc = pow2(-sh);
        S.p0 *= sc;
        S.p1 *= sc;
        d0 *= sc;
        d1 *= sc;
    }
}

// the same with the second-derivative chain (e0, e1) rescaled alongside
__device__ __forceinline__ void sturm_fold_deriv2(SturmState& S, unsigned w, double& d0, double& d1, double& e0,
                                                  double& e1) {
    const unsigned prev = (w >> 1) | (S.prevbit << 31);
    S.cnt += __popc(w ^ prev);
    S.prevbit = w & 1u;
    const int sh = rescale_shift(fmax(fmax(fabs(S.p0), fabs(d0)), fabs(e0)), fmax(fmax(fabs(S.p1), fabs(d1)), fabs(e1)));
    if (sh) {
        const double sc = pow2(-sh);
        S.p0 *= sc;
        S.p1 *= sc;
        d0 *= sc;
        d1 *= sc;
        e0 *= sc;
        e1 *= sc;
    }
}

// 32 steps of two independent chains (shifts xa, xb) interleaved step by
// step, so the warp always has two dependent FMA chains in flight; the
// arithmetic of each chain is exactly that of SturmState::word32
__device__ __forceinline__ void sturm_word32_pair(SturmState& A, SturmState& B, const double* __restrict__ s,
                                                  double xa, double xb) {
    unsigned wa = 0u, wb = 0u;
    double pa0 = A.p0, pa1 = A.p1, pb0 = B.p0, pb1 = B.p1;
#pragma unroll
    for (int u = 0; u < 32; u += 2) {
        const double2 sv = *reinterpret_cast<const double2*>(s + u);
        const double qa0 = fma(sv.x - xa, pa1, -pa0);
        const double qb0 = fma(sv.x - xb, pb1, -pb0);
        const double qa1 = fma(sv.y - xa, qa0, -pa1);
        const double qb1 = fma(sv.y - xb, qb0, -pb1);
        wa = __funnelshift_l(__double2hiint(qa0), wa, 1);
        wb = __funnelshift_l(__double2hiint(qb0), wb, 1);
        wa = __funnelshift_l(__double2hiint(qa1), wa, 1);
        wb = __funnelshift_l(__double2hiint(qb1), wb, 1);
        pa0 = qa0;
        pa1 = qa1;
        pb0 = qb0;
        pb1 = qb1;
    }
    A.p0 = pa0;
    A.p1 = pa1;
    B.p0 = pb0;
    B.p1 = pb1;
    sturm_fold(A, wa);
    sturm_fold(B, wb);
}

// same with chain A also carrying its x-derivative (SturmState::word32_deriv)
__device__ __forceinline__ void sturm_word32_deriv_pair(SturmState& A, double& d0, double& d1, SturmState& B,
                                                        const double* __restrict__ s, double xa, double xb) {
    unsigned wa = 0u, wb = 0u;
    double pa0 = A.p0, pa1 = A.p1, pb0 = B.p0, pb1 = B.p1;
#pragma unroll
    for (int u = 0; u < 32; u += 2) {
        const double2 sv = *reinterpret_cast<const double2*>(s + u);
        const double a0 = sv.x - xa, a1 = sv.y - xa;
        const double qa0 = fma(a0, pa1, -pa0);
        const double qb0 = fma(sv.x - xb, pb1, -pb0);
        const double e0 = fma(a0, d1, -(pa1 + d0));
        const double qa1 = fma(a1, qa0, -pa1);
        const double qb1 = fma(sv.y - xb, qb0, -pb1);
        const double e1 = fma(a1, e0, -(qa0 + d1));
        wa = __funnelshift_l(__double2hiint(qa0), wa, 1);
        wb = __funnelshift_l(__double2hiint(qb0), wb, 1);
        wa = __funnelshift_l(__double2hiint(qa1), wa, 1);
        wb = __funnelshift_l(__double2hiint(qb1), wb, 1);
        pa0 = qa0;
        pa1 = qa1;
        pb0 = qb0;
        pb1 = qb1;
        d0 = e0;
        d1 = e1;
    }
    A.p0 = pa0;
    A.p1 = pa1;
    B.p0 = pb0;
    B.p1 = pb1;
    {  // chain A: counts, then the joint rescale of p and its derivative
        const unsigned prev = (wa >> 1) | (A.prevbit << 31);
        A.cnt += __popc(wa ^ prev);
        A.prevbit = wa & 1u;
        const int sh = rescale_shift(fmax(fabs(A.p0), fabs(d0)), fmax(fabs(A.p1), fabs(d1)));
        if (sh) {
            const double sc = pow2(-sh);
            A.p0 *= sc;
            A.p1 *= sc;
            d0 *= sc;
            d1 *= sc;
        }
    }
    sturm_fold(B, wb);
}

// chain A with first and second derivatives, chain B counts only
__device__ __forceinline__ void sturm_word32_deriv2_pair(SturmState& A, double& d0, double& d1, double& e0,
                                                         double& e1, SturmState& B, const double* __restrict__ s,
                                                         double xa, double xb) {
    unsigned wa = 0u, wb = 0u;
    double pa0 = A.p0, pa1 = A.p1, pb0 = B.p0, pb1 = B.p1;
#pragma unroll
    for (int u = 0; u < 32; u += 2) {
        const double2 sv = *reinterpret_cast<const double2*>(s + u);
        const double a0 = sv.x - xa, a1 = sv.y - xa;
        const double qa0 = fma(a0, pa1, -pa0);
        const double qb0 = fma(sv.x - xb, pb1, -pb0);
        const double f0 = fma(a0, d1, -(pa1 + d0));
        const double g0 = fma(a0, e1, -fma(2.0, d1, e0));
        const double qa1 = fma(a1, qa0, -pa1);
        const double qb1 = fma(sv.y - xb, qb0, -pb1);
        const double f1 = fma(a1, f0, -(qa0 + d1));
        const double g1 = fma(a1, g0, -fma(2.0, f0, e1));
        wa = __funnelshift_l(__double2hiint(qa0), wa, 1);
        wb = __funnelshift_l(__double2hiint(qb0), wb, 1);
        wa = __funnelshift_l(__double2hiint(qa1), wa, 1);
        wb = __funnelshift_l(__double2hiint(qb1), wb, 1);
        pa0 = qa0;
        pa1 = qa1;
        pb0 = qb0;
        pb1 = qb1;
        d0 = f0;
        d1 = f1;
        e0 = g0;
        e1 = g1;
    }
    A.p0 = pa0;
    A.p1 = pa1;
    B.p0 = pb0;
    B.p1 = pb1;
    sturm_fold_deriv2(A, wa, d0, d1, e0, e1);
    sturm_fold(B, wb);
}

// One Laguerre step for the degree-n polynomial det(T - x), all of whose
// roots are real, from g = det'/det and h = g^2 - det''/det (Laguerre's method;
// e.g. Li & Zeng, SIAM J. Sci. Comput. 15 (1994), for symmetric tridiagonal
// matrices): x_new = x - n / (g +- sqrt((n - 1)(n h - g^2))).  The two signs
// step to the nearest root above and below x; up selects the root above.
// Returns the correction subtracted from x (not finite when g and h are not).
__device__ __forceinline__ double laguerre_step(double g, double h, double n, bool up) {
    const double disc = fmax((n - 1.0) * fma(n, h, -g * g), 0.0);
    const double sq = sqrt(disc);
    const double dp = n / (g + sq), dm = n / (g - sq);
    // x - dp and x - dm: the one above x has the negative correction
    return up ? (dp < 0.0 ? dp : dm) : (dp > 0.0 ? dp : dm);
}

// ---------------------------------------------------------------------------
// Row formats of the scaled tridiagonal matrices (unit off-diagonal) that the
// eigenvector kernel streams, and the diagonal entry t_i at a shift.
//  EssRows   S = h^2 A, one double per row: t_i(x) = s_i - x (x = h^2 k^2).
//  WmodRows  the wide-angle T(k) h^2, two doubles per row (B_i = h omega /
//            c0_i, U_i = wc_i / c0_i): t_i(kappa) = (B_i - U_i kappa)^2 -
//            kappa^2 - 2 with kappa = h k, the same polynomial as
//            h^2 ((wc^2/c0^2 - 1) k^2 - 2 omega wc / c0^2 k + omega^2 / c0^2) - 2
//            (WModeSolver.cpp:544-565) in factored form.  Row 0 adds the
//            ground term g0 (independent of kappa), carried into forward
//            recurrences as the starting value p_{-2} = -g0.
// ---------------------------------------------------------------------------
struct EssRows {
    static constexpr int kW = 1;  // doubles per row
    static constexpr bool kTwist = true;  // bisection sweeps as twisted counts (measured faster)
    // det(S - x) has only real roots (S symmetric): Laguerre steps, which
    // need the second derivative chain as well
    static constexpr bool kLaguerre = true;
    struct Shift {
        double x;
    };
    __device__ static __forceinline__ Shift shift(double mu) { return Shift{mu}; }
    __device__ static __forceinline__ double t(const double* __restrict__ b, int i, const Shift& s) {
        return b[i] - s.x;
    }
    __device__ static __forceinline__ double p_init(const ProblemInfo&) { return 0.0; }
    __device__ static __forceinline__ double idle_shift(const ProblemInfo& pi) { return pi.lo; }
    // the bisection interval and the scale of its tolerance
    __device__ static __forceinline__ double scan_lo(const ProblemInfo& pi) { return pi.lo; }
    __device__ static __forceinline__ double scan_hi(const ProblemInfo& pi) { return pi.hi; }
    __device__ static __forceinline__ double tol_scale(const ProblemInfo&) { return 1.0; }
    // Sturm sweeps over 32 staged rows at b (see SturmState)
    __device__ static __forceinline__ void pair(SturmState& A, SturmState& B, const double* __restrict__ b,
                                                double xa, double xb) {
        sturm_word32_pair(A, B, b, xa, xb);
    }
    __device__ static __forceinline__ void deriv_pair(SturmState& A, double& d0, double& d1, SturmState& B,
                                                      const double* __restrict__ b, double xa, double xb) {
        sturm_word32_deriv_pair(A, d0, d1, B, b, xa, xb);
    }
    __device__ static __forceinline__ void word_deriv(SturmState& A, const double* __restrict__ b, double x,
                                                      double& d0, double& d1) {
        A.word32_deriv(b, x, d0, d1);
    }
    __device__ static __forceinline__ void step(SturmState& A, const double* __restrict__ b, int i, double x) {
        A.step(b[i], x);
    }
    __device__ static __forceinline__ void step_deriv(SturmState& A, const double* __restrict__ b, int i, double x,
                                                      double& d0, double& d1) {
        A.step_deriv(b[i], x, d0, d1);
    }
    __device__ static __forceinline__ void deriv2_pair(SturmState& A, double& d0, double& d1, double& e0,
                                                       double& e1, SturmState& B, const double* __restrict__ b,
                                                       double xa, double xb) {
        sturm_word32_deriv2_pair(A, d0, d1, e0, e1, B, b, xa, xb);
    }
    __device__ static __forceinline__ void word_deriv2(SturmState& A, const double* __restrict__ b, double x,
                                                       double& d0, double& d1, double& e0, double& e1) {
        A.word32_deriv2(b, x, d0, d1, e0, e1);
    }
    __device__ static __forceinline__ void step_deriv2(SturmState& A, const double* __restrict__ b, int i,
                                                       double x, double& d0, double& d1, double& e0, double& e1) {
        A.step_deriv2(b[i], x, d0, d1, e0, e1);
    }
    // Newton correction (subtracted from x) from the last p and its derivative chain
    __device__ static __forceinline__ double newton(double p, double d) { return p / d; }
};

struct WmodRows {
    static constexpr int kW = 2;
    static constexpr bool kTwist = false;  // twisted sweeps measured 6 % slower here (register spills)
    // det T(kappa) also has non-real roots: Newton steps
    static constexpr bool kLaguerre = false;
    struct Shift {
        double kap, c;  // kappa and -(kappa^2 + 2)
    };
    __device__ static __forceinline__ Shift shift(double kap) { return Shift{kap, fma(-kap, kap, -2.0)}; }
    __device__ static __forceinline__ double t(const double* __restrict__ b, int i, const Shift& s) {
        const double2 r = *reinterpret_cast<const double2*>(b + 2 * i);
        const double d = fma(-r.y, s.kap, r.x);
        return fma(d, d, s.c);
    }
    __device__ static __forceinline__ double p_init(const ProblemInfo& pi) { return -pi.g0; }
    __device__ static __forceinline__ double idle_shift(const ProblemInfo& pi) { return pi.k_min * pi.dz; }
    __device__ static __forceinline__ double scan_lo(const ProblemInfo& pi) { return pi.k_min * pi.dz; }
    __device__ static __forceinline__ double scan_hi(const ProblemInfo& pi) { return pi.k_max * pi.dz; }
    __device__ static __forceinline__ double tol_scale(const ProblemInfo& pi) { return pi.k_max * pi.dz; }
    // Sturm sweeps over 32 staged rows at b.  The derivative chain carries
    // e_i = t_i e_{i-1} + (U_i d_i + kappa) p_{i-1} - e_{i-2}, d_i = B_i - U_i
    // kappa, which is -1/2 of d p_i / d kappa.
    __device__ static __forceinline__ void pair(SturmState& A, SturmState& B, const double* __restrict__ b,
                                                double xa, double xb) {
        const double ca = fma(-xa, xa, -2.0), cb = fma(-xb, xb, -2.0);
        unsigned wa = 0u, wb = 0u;
        double pa0 = A.p0, pa1 = A.p1, pb0 = B.p0, pb1 = B.p1;
#pragma unroll
        for (int u = 0; u < 32; ++u) {
            const double2 rv = *reinterpret_cast<const double2*>(b + 2 * u);
            const double da = fma(-rv.y, xa, rv.x);
            const double db = fma(-rv.y, xb, rv.x);
            const double qa = fma(fma(da, da, ca), pa1, -pa0);
            const double qb = fma(fma(db, db, cb), pb1, -pb0);
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
        sturm_fold(A, wa);
        sturm_fold(B, wb);
    }
    __device__ static __forceinline__ void deriv_pair(SturmState& A, double& d0, double& d1, SturmState& B,
                                                      const double* __restrict__ b, double xa, double xb) {
        const double ca = fma(-xa, xa, -2.0), cb = fma(-xb, xb, -2.0);
        unsigned wa = 0u, wb = 0u;
        double pa0 = A.p0, pa1 = A.p1, pb0 = B.p0, pb1 = B.p1;
#pragma unroll
        for (int u = 0; u < 32; ++u) {
            const double2 rv = *reinterpret_cast<const double2*>(b + 2 * u);
            const double da = fma(-rv.y, xa, rv.x);
            const double db = fma(-rv.y, xb, rv.x);
            const double ta = fma(da, da, ca);
            const double tp = fma(rv.y, da, xa);
            const double qa = fma(ta, pa1, -pa0);
            const double qb = fma(fma(db, db, cb), pb1, -pb0);
            const double ea = fma(ta, d1, fma(tp, pa1, -d0));
            wa = __funnelshift_l(__double2hiint(qa), wa, 1);
            wb = __funnelshift_l(__double2hiint(qb), wb, 1);
            pa0 = pa1;
            pa1 = qa;
            pb0 = pb1;
            pb1 = qb;
            d0 = d1;
            d1 = ea;
        }
        A.p0 = pa0;
        A.p1 = pa1;
        B.p0 = pb0;
        B.p1 = pb1;
        sturm_fold_deriv(A, wa, d0, d1);
        sturm_fold(B, wb);
    }
    __device__ static __forceinline__ void word_deriv(SturmState& A, const double* __restrict__ b, double x,
                                                      double& d0, double& d1) {
        const double c = fma(-x, x, -2.0);
        unsigned wa = 0u;
        double pa0 = A.p0, pa1 = A.p1;
#pragma unroll
        for (int u = 0; u < 32; ++u) {
            const double2 rv = *reinterpret_cast<const double2*>(b + 2 * u);
            const double da = fma(-rv.y, x, rv.x);
            const double ta = fma(da, da, c);
            const double tp = fma(rv.y, da, x);
            const double qa = fma(ta, pa1, -pa0);
            const double ea = fma(ta, d1, fma(tp, pa1, -d0));
            wa = __funnelshift_l(__double2hiint(qa), wa, 1);
            pa0 = pa1;
            pa1 = qa;
            d0 = d1;
            d1 = ea;
        }
        A.p0 = pa0;
        A.p1 = pa1;
        sturm_fold_deriv(A, wa, d0, d1);
    }
    __device__ static __forceinline__ void step(SturmState& A, const double* __restrict__ b, int i, double x) {
        const double2 rv = *reinterpret_cast<const double2*>(b + 2 * i);
        const double d = fma(-rv.y, x, rv.x);
        const double q = fma(fma(d, d, fma(-x, x, -2.0)), A.p1, -A.p0);
        const unsigned bit = static_cast<unsigned>(__double2hiint(q)) >> 31;
        A.cnt += static_cast<int>(bit ^ A.prevbit);
        A.prevbit = bit;
        A.p0 = A.p1;
        A.p1 = q;
    }
    __device__ static __forceinline__ void step_deriv(SturmState& A, const double* __restrict__ b, int i, double x,
                                                      double& d0, double& d1) {
        const double2 rv = *reinterpret_cast<const double2*>(b + 2 * i);
        const double d = fma(-rv.y, x, rv.x);
        const double t = fma(d, d, fma(-x, x, -2.0));
        const double tp = fma(rv.y, d, x);
        const double q = fma(t, A.p1, -A.p0);
        const double e = fma(t, d1, fma(tp, A.p1, -d0));
        const unsigned bit = static_cast<unsigned>(__double2hiint(q)) >> 31;
        A.cnt += static_cast<int>(bit ^ A.prevbit);
        A.prevbit = bit;
        A.p0 = A.p1;
        A.p1 = q;
        d0 = d1;
        d1 = e;
    }
    // d p / d kappa = -2 e: the correction subtracted from kappa is -p / (2 e)
    __device__ static __forceinline__ double newton(double p, double e) { return -0.5 * (p / e); }
};

// principal square root of x + i y
__device__ __forceinline__ cuda::std::complex<double> csqrt_principal(double x, double y) {
    double m = hypot(x, y);
    double t = sqrt(0.5 * (m + fabs(x)));
    if (x >= 0.0) return cuda::std::complex<double>(t, y / (2.0 * t));
    return cuda::std::complex<double>(fabs(y) / (2.0 * t), copysign(t, y));
}

}  // namespace ncpa
