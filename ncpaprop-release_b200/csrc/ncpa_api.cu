// C ABI of the B200 ESS normal-mode library (include/ncpa_gpu.h): context,
// resident profiles, the batched (frequency x azimuth) eigen-solve, modal
// sums and ModBB synthesis.  Host orchestration only; all arithmetic on the
// path runs in the kernels of kernels.cu.
#include "ncpa_gpu.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "atmosphere.hpp"
#include "kernels.hpp"

using ncpa::ProblemInfo;
using ncpa::WorkItem;

namespace {

constexpr double kPi = 3.141592653589793;
constexpr double kBisectTol = 1.0e-15;  // bracket width, units of S = h^2 A

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct ApiError : std::runtime_error {
    ncpa_status code;
    ApiError(ncpa_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CK(call)                                                                                    \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            throw CudaError(std::string(#call) + ": " + cudaGetErrorString(e_));                    \
    } while (0)

// owning device buffer on the stream-ordered allocator (pooled, so the
// per-solve temporaries cost no cudaMalloc round trips after warm-up)
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaStream_t st = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes), st(o.st) {
        o.p = nullptr;
        o.bytes = 0;
    }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            bytes = o.bytes;
            st = o.st;
            o.p = nullptr;
            o.bytes = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFreeAsync(p, st);
        p = nullptr;
        bytes = 0;
    }
    void alloc(size_t b, cudaStream_t stream) {
        if (b <= bytes && p) return;
        release();
        st = stream;
        if (b == 0) b = 16;
        cudaError_t e = cudaMallocAsync(&p, b, st);
        if (e != cudaSuccess) {
            p = nullptr;
            throw ApiError(NCPA_ENOMEM, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
        }
        bytes = b;
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

template <class T>
void upload(DevBuf& d, const std::vector<T>& h, cudaStream_t st) {
    d.alloc(h.size() * sizeof(T), st);
    if (!h.empty()) CK(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
}
template <class T>
void upload(DevBuf& d, const T* h, size_t n, cudaStream_t st) {
    d.alloc(n * sizeof(T), st);
    if (n) CK(cudaMemcpyAsync(d.p, h, n * sizeof(T), cudaMemcpyHostToDevice, st));
}

}  // namespace

struct ncpa_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    long long launches = 0;
    int num_sms = 148;
    DevBuf d_err;                  // device status word
    DevBuf ck1, ck2, cke;          // eigenvector checkpoint scratch
    std::map<int, DevBuf> twiddle; // per nfft
    DevBuf bb_out;                 // waveforms kept in HBM (NULL host buffer)
    DevBuf ms_img, ms_q, ms_tab, ms_raw, ms_vz, ms_idx, ms_re, ms_im;  // modal-sum scratch (grow-only)
    DevBuf ms_spart, ms_b64, ms_tp64, ms_a64, ms_fix, ms_fixcnt;        // guarded sum: bounds, FP64 tables, flags
    long long ms_last_points = 0;  // receivers x ranges of the last guarded modal sum
    double ms_last_eps = 0.0, ms_last_tau = 0.0;  // its error bound and flag threshold (relative to S)
    // modal-sum schedule autotuner: (format, groups, chunks, tiles) -> the
    // fastest ring-depth variant of the tensor-core kernel; NCPA_MS_TUNE=0
    // keeps variant 0
    bool ms_tune = true;
    std::map<std::array<long long, 4>, int> ms_choice;
    int ms_last_variant = 0, ms_last_fmt = 0;
    std::vector<double> ms_last_times;  // per variant, ms, of the last tuning run
    int item_override = 0;         // eigenvalues per bisection item (0: chosen per solve); NCPA_BISECT_ITEM
    // bisection items listed by estimated cost and spread over the warp
    // schedulers (heaviest first); NCPA_BISECT_ORDER=0 keeps problem order and
    // round-robin warps.  Results do not depend on it.
    bool bis_order = true;
    int bis_workers = ncpa::kSchedWorkers;  // bisection warps per warp scheduler; NCPA_BISECT_WORKERS
    // fused launch: only the bisection warps take eigenvector items (as their
    // bisection ends), the others leave them to the k_eigvec launch that
    // follows; NCPA_FUSE_EV_WORKERS=0 lets every warp of the launch take them
    bool fuse_ev_workers = true;
    // modal sum of ncpa_tl_2d (the front ends' tloss_2d.nm): NCPA_SUM_FP64,
    // or NCPA_SUM_TC_GUARDED with NCPA_TL2D_SUM=3
    int tl2d_method = NCPA_SUM_FP64;
    // isolation scan trimmed to a whole number of units per warp scheduler;
    // NCPA_SCAN_TRIM=0 keeps every problem's own estimate
    bool scan_trim = true;
    bool fuse_solve = true;        // fused bisection + eigenvector launch; NCPA_FUSE_SOLVE=0 turns it off
    // how long a consumer of the fused launch waits for an empty queue slot
    // before leaving the item to the following launch; NCPA_FUSE_WAIT_NS
    unsigned long long fuse_wait_ns = 1000000000ull;
    double* h_pin = nullptr;       // small pinned host buffer for scalars read back per solve
    int* h_tot = nullptr;          // pinned: item and mode totals of a device-built solve
    size_t h_pin_n = 0;
    DevBuf d_stats;                // device counters (Sturm sequences)
    bool timing = false;           // NCPA_TIMING=1: per-phase times on stderr
    bool stats = false;            // ncpa_ctx_set_timing: accumulate per phase
    bool stats_fused = false;      // ncpa_ctx_set_timing(ctx, 2): ... keeping the fused launch
    std::map<std::string, std::pair<double, long long>> phase;
    std::map<std::string, std::array<int, 3>> tune_cache;  // plan shape -> tuned launch shapes
    void count(int n) { launches += n; }
};

namespace {
// per-phase timing with CUDA events on the context stream (diagnostics)
struct PhaseTimer {
    ncpa_ctx* ctx;
    std::vector<std::pair<std::string, cudaEvent_t>> ev;
    explicit PhaseTimer(ncpa_ctx* c) : ctx(c) {}
    void mark(const char* name) {
        if (!ctx->timing && !ctx->stats) return;
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, ctx->stream);
        ev.emplace_back(name, e);
    }
    ~PhaseTimer() {
        if (ev.size() > 1) {
            cudaEventSynchronize(ev.back().second);
            for (size_t i = 1; i < ev.size(); ++i) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, ev[i - 1].second, ev[i].second);
                if (ctx->timing) std::fprintf(stderr, "[ncpa] %-14s %9.3f ms\n", ev[i].first.c_str(), ms);
                if (ctx->stats) {
                    auto& acc = ctx->phase[ev[i].first];
                    acc.first += ms;
                    acc.second += 1;
                }
            }
        }
        for (auto& e : ev) cudaEventDestroy(e.second);
    }
};
}  // namespace

struct ncpa_profile {
    ncpa_ctx* ctx = nullptr;
    int n = 0;
    DevBuf z, u, v, t, p, rho, c0, ws, wd, pcoef, rcoef, attn;
    bool has_attn = false;
    double z0 = 0.0;
    int has_z0 = 0;
    double z_lo = 0.0, z_hi = 0.0;
    int plan_refs = 0;  // plans whose graphs read this profile's arrays
};

struct ncpa_modes {
    ncpa_ctx* ctx = nullptr;
    int P = 0, nf = 0, na = 0;
    int nz_max = 0;  // largest grid of the batch (each problem's own grid is in info[p])
    ncpa_ess_params prm{};
    std::vector<double> freqs, az;
    std::vector<double> rho_src_p, rho_rcv_p;  // rho at the source / receiver grid points, per problem
    bool multi_job = false;                     // built by ncpa_ess_solve_jobs (one profile per job)
    bool plan_owned = false;                    // the arrays are a plan's graph buffers
    std::vector<ProblemInfo> info;
    int Mtot = 0;
    DevBuf d_pinfo, d_kr, d_ki, d_vs, d_vr, d_vg, d_vfull, d_vfull_off;
    mutable DevBuf tl_re, tl_im, tl_inc;  // 1-D TL kept in HBM
    mutable bool host_valid = false;      // host copies of the mode arrays
    mutable std::vector<double> kr, ki, vs, vr, vg;
    std::vector<long long> vfull_off;
};

namespace {

ncpa_status fail(ncpa_ctx* ctx, ncpa_status s, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return s;
}

template <class F>
ncpa_status guarded(ncpa_ctx* ctx, F&& f) {
    try {
        return f();
    } catch (const ApiError& e) {
        return fail(ctx, e.code, e.what());
    } catch (const ncpa::ParseError& e) {
        return fail(ctx, NCPA_EPARSE, e.what());
    } catch (const CudaError& e) {
        return fail(ctx, NCPA_ECUDA, e.what());
    } catch (const std::bad_alloc&) {
        return fail(ctx, NCPA_ENOMEM, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(ctx, NCPA_EINVAL, e.what());
    }
}

void check_launch(ncpa_ctx* ctx, int n) {
    if (n < 0) throw ApiError(NCPA_EINVAL, "kernel launch rejected its arguments");
    ctx->count(n);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw CudaError(std::string("kernel launch: ") + cudaGetErrorString(e));
}

void check_device_status(ncpa_ctx* ctx) {
    unsigned h = 0;
    CK(cudaMemcpyAsync(&h, ctx->d_err.p, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (h) {
        CK(cudaMemsetAsync(ctx->d_err.p, 0, sizeof(unsigned), ctx->stream));
        if (h & ncpa::kErrTimeout) throw ApiError(NCPA_ETIMEDOUT, "a bounded device wait gave up");
        if (h & ncpa::kErrBracket) throw ApiError(NCPA_ECUDA, "bisection bracket inconsistent with Sturm counts");
        if (h & ncpa::kErrWkb) throw ApiError(NCPA_ECUDA, "WKB window search exceeded its trial count");
    }
}

const double* twiddle(ncpa_ctx* ctx, int nfft) {
    auto it = ctx->twiddle.find(nfft);
    if (it != ctx->twiddle.end()) return it->second.as<double>();
    DevBuf b;
    b.alloc((size_t)2 * nfft * sizeof(double), ctx->stream);
    check_launch(ctx, ncpa::launch_twiddle(ctx->stream, nfft, b.as<double>()));
    const double* p = b.as<double>();
    ctx->twiddle.emplace(nfft, std::move(b));
    return p;
}

// copy the mode arrays of a solve to its host mirror (stream-ordered)
void fetch_modes(const ncpa_modes* M) {
    cudaStream_t st = M->ctx->stream;
    M->kr.resize(M->Mtot);
    M->ki.resize(M->Mtot);
    M->vs.resize(M->Mtot);
    M->vr.resize(M->Mtot);
    M->vg.resize(M->Mtot);
    if (M->Mtot > 0) {
        CK(cudaMemcpyAsync(M->kr.data(), M->d_kr.p, M->Mtot * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(M->ki.data(), M->d_ki.p, M->Mtot * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(M->vs.data(), M->d_vs.p, M->Mtot * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(M->vr.data(), M->d_vr.p, M->Mtot * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(M->vg.data(), M->d_vg.p, M->Mtot * 8, cudaMemcpyDeviceToHost, st));
    }
    M->host_valid = true;
}

}  // namespace

namespace {

// pinned host scratch of at least n doubles (grow-only; the stream must be
// idle when it grows, which holds at the start of a solve)
double* pinned(ncpa_ctx* ctx, size_t n) {
    if (n > ctx->h_pin_n) {
        CK(cudaStreamSynchronize(ctx->stream));
        if (ctx->h_pin) cudaFreeHost(ctx->h_pin);
        ctx->h_pin = nullptr;
        ctx->h_pin_n = 0;
        const size_t m = std::max<size_t>(n, 256);
        CK(cudaHostAlloc((void**)&ctx->h_pin, m * sizeof(double), cudaHostAllocDefault));
        ctx->h_pin_n = m;
    }
    return ctx->h_pin;
}

// grid geometry of ESSModeSolver.cpp:39-41, 144-151, 212-220, 314
struct Geometry {
    double z_min, dz_grid, dz;
    int isrc, ircv;
};

void check_ess_params(const ncpa_ess_params* prm) {
    if (prm->nz_grid < 10) throw ApiError(NCPA_EINVAL, "Nz_grid must be >= 10");
    if (prm->method != NCPA_METHOD_ESS && prm->method != NCPA_METHOD_WMOD)
        throw ApiError(NCPA_EINVAL, "unknown method");
    if (prm->wvnum_filter && !(prm->c_min > 0.0 && prm->c_max > 0.0))
        throw ApiError(NCPA_EINVAL, "wvnum_filter needs c_min > 0 and c_max > 0");
}

Geometry grid_geometry(const ncpa_profile* prof, const ncpa_ess_params* prm, int nz) {
    Geometry g{};
    double z_min = prm->zground_km * 1000.0;
    double maxheight = prm->maxheight_km * 1000.0;
    if (maxheight >= prof->z_hi) maxheight = prof->z_hi - 1e-6;
    g.dz_grid = (maxheight - z_min) / (nz - 1);
    if (prof->has_z0 && z_min < prof->z0) z_min = prof->z0;
    g.dz = (maxheight - z_min) / (nz - 1);
    if (!(g.dz > 0.0)) throw ApiError(NCPA_EINVAL, "maxheight must lie above the ground");
    g.z_min = z_min;
    g.isrc = (int)std::ceil(prm->sourceheight_km * 1000.0 / g.dz);
    g.ircv = (int)std::ceil(prm->receiverheight_km * 1000.0 / g.dz);
    if (g.isrc < 0 || g.isrc >= nz || g.ircv < 0 || g.ircv >= nz)
        throw ApiError(NCPA_EINVAL, "source/receiver height outside the grid");
    return g;
}

// One group of problems: one profile on one solver grid, n_freq x n_az
// problems numbered frequency-major from p0.  Its rows start at s_base in
// s, g and kz2 (nz_pad apart) and at w_base in w (one row per frequency).
struct Group {
    const ncpa_profile* prof;
    Geometry geo;
    int nz, nz_pad;
    const double* freqs;
    int n_freq;
    const double* az;
    int n_az;
    int p0;
    long long s_base, w_base;
};

Group make_group(const ncpa_profile* prof, const ncpa_ess_params* prm, int nz, const double* freqs, int n_freq,
                 const double* az, int n_az) {
    Group g{};
    g.prof = prof;
    g.geo = grid_geometry(prof, prm, nz);
    g.nz = nz;
    g.nz_pad = ((nz + ncpa::kChunk - 1) / ncpa::kChunk) * ncpa::kChunk;
    g.freqs = freqs;
    g.n_freq = n_freq;
    g.az = az;
    g.n_az = n_az;
    return g;
}

// Ground admittance of the Lamb-wave condition, -rho'(z0) / (2 rho(z0)), from
// one point of the profile's rho spline and its slope (scalar set-up, as in
// ESSModeSolver.cpp:347-349).  Synchronises the stream.
double lamb_admittance(ncpa_ctx* ctx, const ncpa_profile* prof, double z_min) {
    cudaStream_t st = ctx->stream;
    const int nk = prof->n;
    std::vector<double> hz(nk), hc(4 * (nk - 1)), hr(nk);
    CK(cudaMemcpyAsync(hz.data(), prof->z.p, nk * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hr.data(), prof->rho.p, nk * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hc.data(), prof->rcoef.p, hc.size() * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double zq = z_min, val, der;
    if (zq > hz[nk - 1] || zq < hz[0]) {
        val = zq > hz[nk - 1] ? hr[nk - 1] : hr[0];
        der = 0.0;
    } else {
        int lo = 0, hi = nk - 1;
        while (hi > lo + 1) {
            int mid = (lo + hi) / 2;
            if (hz[mid] > zq) hi = mid; else lo = mid;
        }
        const double* c = &hc[4 * lo];
        double t = zq - hz[lo];
        val = c[3] + t * (c[2] + t * (c[1] + t * c[0]));
        der = c[2] + t * (2.0 * c[1] + t * 3.0 * c[0]);
    }
    return -der / val / 2.0;
}

// Device buffers of one group's knot-level and grid-level stages.
struct GroupBufs {
    DevBuf freqs, az, ceffk, ceffc, alpha, alphac, rho_g, ct_g;
    double admittance = 0.0;
};

// Allocates a group's buffers, uploads its frequencies and azimuths and, with
// the Lamb-wave condition, computes the ground admittance (host work that
// stays outside any captured graph).
void prepare_group(ncpa_ctx* ctx, const ncpa_ess_params* prm, const Group& g, GroupBufs& b) {
    cudaStream_t st = ctx->stream;
    const int nk = g.prof->n;
    upload(b.freqs, g.freqs, g.n_freq, st);
    upload(b.az, g.az, g.n_az, st);
    b.ceffk.alloc((size_t)g.n_az * nk * 8, st);
    b.ceffc.alloc((size_t)g.n_az * 4 * (nk - 1) * 8, st);
    b.alpha.alloc((size_t)g.n_freq * nk * 8, st);
    b.alphac.alloc((size_t)g.n_freq * 4 * (nk - 1) * 8, st);
    b.rho_g.alloc((size_t)g.nz * 8, st);
    b.ct_g.alloc((size_t)g.nz * 8, st);
    b.admittance = prm->lamb_wave_bc ? lamb_admittance(ctx, g.prof, g.geo.z_min) : 0.0;
}

// Knot-level fields, grid fields and matrices of one group's problems: only
// kernel launches, device copies and memsets, plus one copy of rho at the
// source and receiver grid points to rho_pair[0..1] (pinned host memory when
// captured).  d_pinfo, s, w, gs, kz2 point at the group's first problem / row.
void enqueue_group(ncpa_ctx* ctx, PhaseTimer& tm, const Group& g, GroupBufs& b, bool wkb, ProblemInfo* d_pinfo,
                   double* s, double* w, double* gs, double* kz2, double* rho_pair) {
    cudaStream_t st = ctx->stream;
    const ncpa_profile* prof = g.prof;
    const int nk = prof->n;
    const int P = g.n_freq * g.n_az;
    check_launch(ctx, ncpa::launch_ceff_knots(st, nk, g.n_az, b.az.as<double>(), prof->c0.as<double>(),
                                              prof->ws.as<double>(), prof->wd.as<double>(), b.ceffk.as<double>()));
    check_launch(ctx, ncpa::launch_steffen(st, nk, prof->z.as<double>(), b.ceffk.as<double>(), g.n_az, nk,
                                           b.ceffc.as<double>(), 4 * (nk - 1)));
    if (prof->has_attn) {
        for (int f = 0; f < g.n_freq; ++f)
            CK(cudaMemcpyAsync(b.alpha.as<double>() + (size_t)f * nk, prof->attn.p, nk * 8, cudaMemcpyDeviceToDevice,
                               st));
    } else {
        check_launch(ctx, ncpa::launch_alpha_knots(st, nk, g.n_freq, b.freqs.as<double>(), prof->z.as<double>(),
                                                   prof->t.as<double>(), prof->p.as<double>(),
                                                   prof->rho.as<double>(), b.alpha.as<double>()));
    }
    check_launch(ctx, ncpa::launch_steffen(st, nk, prof->z.as<double>(), b.alpha.as<double>(), g.n_freq, nk,
                                           b.alphac.as<double>(), 4 * (nk - 1)));
    // ---- grid fields ----
    CK(cudaMemsetAsync(w, 0, (size_t)g.n_freq * g.nz_pad * 8, st));
    check_launch(ctx, ncpa::launch_grid_common(st, nk, prof->z.as<double>(), prof->rho.as<double>(),
                                               prof->rcoef.as<double>(), prof->p.as<double>(),
                                               prof->pcoef.as<double>(), g.nz, g.geo.z_min, g.geo.dz_grid,
                                               b.rho_g.as<double>(), b.ct_g.as<double>()));
    check_launch(ctx, ncpa::launch_attn_weight(st, nk, prof->z.as<double>(), b.alpha.as<double>(),
                                               b.alphac.as<double>(), g.n_freq, b.freqs.as<double>(), g.nz,
                                               g.geo.z_min, g.geo.dz_grid, b.ct_g.as<double>(), w, g.nz_pad));
    CK(cudaMemcpyAsync(rho_pair, b.rho_g.as<double>() + g.geo.isrc, 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(rho_pair + 1, b.rho_g.as<double>() + g.geo.ircv, 8, cudaMemcpyDeviceToHost, st));
    tm.mark("knots+grid");
    // ---- K1 matrix ----
    check_launch(ctx, ncpa::launch_build_matrix(st, nk, prof->z.as<double>(), b.ceffk.as<double>(),
                                                b.ceffc.as<double>(), g.n_az, P, d_pinfo, g.nz, g.nz_pad,
                                                g.geo.z_min, g.geo.dz_grid, g.geo.dz, b.admittance, s,
                                                wkb ? kz2 : nullptr, gs));
    tm.mark("matrix");
}

// Launch shapes of the device-driven eigen-solve (the autotuner's knobs).
struct Tuning {
    int bis_item = ncpa::kWItem;  // eigenvalues per bisection work item (<= 32)
    int bis_ctas = 0;             // bisection CTAs per SM (0: as many as fit)
    int ev_ctas = 0;              // eigenvector CTAs per SM (0: as many as fit)
};

// Buffers of the device-driven eigen-solve.  The eigenvector checkpoint
// scratch is the context's (grown on demand) unless own_ck is set (a
// captured graph must keep its addresses for good).
struct SolveBufs {
    DevBuf counts, bis, ev, tot, mu, counter, sched;
    DevBuf pstat, fq;  // fused launch: per-problem readiness; ready queue, done flags, queue counters
    DevBuf ck1, ck2, cke;
    bool own_ck = false;
    int bis_cap = 0, ev_cap = 0;
};

ncpa::EigvecArgs eigvec_args(ncpa_ctx* ctx, ncpa_modes* M, const ncpa_ess_params* prm, double* s, double* w,
                             double* gs, SolveBufs& b) {
    ncpa::EigvecArgs ea{};
    ea.pinfo = M->d_pinfo.as<ProblemInfo>();
    ea.s = s;
    ea.w = w;
    ea.g = prm->want_group_speed ? gs : nullptr;
    ea.items = b.ev.as<WorkItem>();
    ea.n_items = 0;
    ea.n_items_dev = b.tot.as<int>() + 1;
    ea.counter = b.counter.as<int>() + 1;
    ea.mu = b.mu.as<double>();
    ea.kr = M->d_kr.as<double>();
    ea.ki = M->d_ki.as<double>();
    ea.vs = M->d_vs.as<double>();
    ea.vr = M->d_vr.as<double>();
    ea.vg = M->d_vg.as<double>();
    ea.err = ctx->d_err.as<unsigned>();
    return ea;
}

int eigvec_grid(ncpa_ctx* ctx, const ncpa::EigvecArgs& ea, int ev_cap, int ctas_per_sm) {
    const int fit = ncpa::eigvec_ctas_per_sm(ea);
    const int per_sm = ctas_per_sm > 0 ? std::min(ctas_per_sm, fit) : fit;
    return std::max(1, std::min(ev_cap / ncpa::kEvWarpsPerCta + 1, ctx->num_sms * per_sm));
}

// Allocates the eigen-solve's buffers and the mode arrays (max_modes per
// problem) and sizes the eigenvector checkpoint scratch for the largest grid
// any of the given tunings launches.  min_bis_item sizes the bisection item
// list for the smallest item size that will run.
void prepare_solve(ncpa_ctx* ctx, ncpa_modes* M, const ncpa_ess_params* prm, int min_bis_item, SolveBufs& b,
                   double* s, double* w, double* gs) {
    cudaStream_t st = ctx->stream;
    const int P = M->P;
    const int cap_modes = M->prm.max_modes;
    const size_t mcap = (size_t)P * cap_modes;
    b.counts.alloc((size_t)P * ncpa::kScanMax * 4, st);
    b.bis_cap = P * ((cap_modes + min_bis_item - 1) / min_bis_item);
    b.ev_cap = P * ((cap_modes + ncpa::kEvItem - 1) / ncpa::kEvItem);
    b.bis.alloc((size_t)b.bis_cap * sizeof(WorkItem), st);
    b.ev.alloc((size_t)b.ev_cap * sizeof(WorkItem), st);
    b.tot.alloc(4 * sizeof(int), st);
    b.pstat.alloc((size_t)3 * P * sizeof(int), st);
    b.fq.alloc(((size_t)2 * b.ev_cap + 2) * sizeof(int), st);
    b.mu.alloc(mcap * 8, st);
    b.counter.alloc(2 * sizeof(int), st);
    b.sched.alloc(ncpa::kSchedInts * sizeof(int), st);
    M->d_kr.alloc(mcap * 8, st);
    M->d_ki.alloc(mcap * 8, st);
    M->d_vs.alloc(mcap * 8, st);
    M->d_vr.alloc(mcap * 8, st);
    M->d_vg.alloc(mcap * 8, st);
    const ncpa::EigvecArgs ea = eigvec_args(ctx, M, prm, s, w, gs, b);
    const int grid_e = eigvec_grid(ctx, ea, b.ev_cap, 0);  // the largest grid
    const long long slot = ncpa::ck_slot_elems(M->nz_max);
    const size_t need = (size_t)grid_e * ncpa::kEvWarpsPerCta * slot;
    DevBuf& c1 = b.own_ck ? b.ck1 : ctx->ck1;
    DevBuf& c2 = b.own_ck ? b.ck2 : ctx->ck2;
    DevBuf& ce = b.own_ck ? b.cke : ctx->cke;
    if (c1.bytes < need * 8) {
        c1.alloc(need * 8, st);
        c2.alloc(need * 8, st);
        ce.alloc(need * 4, st);
    }
}

// Window, Sturm scan, device-built work items, bisection and eigenvectors
// over all problems of M, then copies of the item/mode totals, the problem
// warp schedulers of the device for the scan trim (0: no trim)
int scan_slots(const ncpa_ctx* ctx) { return ctx->scan_trim ? 4 * ctx->num_sms : 0; }

// records and the device status word to tot_dst, info_dst and err_dst.  No
// host synchronisation: the whole sequence can be captured in a CUDA graph.
void enqueue_solve(ncpa_ctx* ctx, PhaseTimer& tm, ncpa_modes* M, const ncpa_ess_params* prm, bool wkb, double* s,
                   double* w, double* gs, double* kz2, SolveBufs& b, const Tuning& t, bool count_steps,
                   int* tot_dst, ProblemInfo* info_dst, unsigned* err_dst) {
    cudaStream_t st = ctx->stream;
    const int P = M->P;
    ProblemInfo* d_pinfo = M->d_pinfo.as<ProblemInfo>();
    unsigned* err = ctx->d_err.as<unsigned>();
    // ---- K2 window ----
    check_launch(ctx, ncpa::launch_window(st, P, d_pinfo, wkb ? kz2 : nullptr, wkb ? 1 : 0, prm->wvnum_filter,
                                          prm->c_min, prm->c_max, err));
    tm.mark("window");
    // ---- K3a scan ----
    // the scan's units claimed per warp scheduler through the item scheduler's
    // state (zeroed again below before the bisection uses it)
    int* scan_sched = nullptr;
    if (scan_slots(ctx) > 0) {
        scan_sched = b.sched.as<int>();
        CK(cudaMemsetAsync(scan_sched, 0, ncpa::kSchedInts * sizeof(int), st));
    }
    check_launch(ctx, ncpa::launch_scan(st, P, d_pinfo, s, b.counts.as<int>(), err, scan_slots(ctx), scan_sched));
    tm.mark("scan");
    // fused bisection + eigenvectors (one launch, eigenvectors of finished
    // problems overlapping the others' bisection), unless per-phase timing or
    // step counts ask for the kernels alone, or group speeds are wanted
    const bool fuse = ctx->fuse_solve && !ctx->timing && (!ctx->stats || ctx->stats_fused) && !count_steps &&
                      !prm->want_group_speed;
    check_launch(ctx, ncpa::launch_make_items(st, P, d_pinfo, b.counts.as<int>(), M->prm.max_modes, t.bis_item,
                                              b.bis.as<WorkItem>(), b.bis_cap, b.ev.as<WorkItem>(), b.ev_cap,
                                              b.tot.as<int>(), err, fuse ? b.pstat.as<int>() : nullptr,
                                              ctx->bis_order ? 1 : 0));
    CK(cudaMemsetAsync(b.counter.p, 0, 2 * sizeof(int), st));
    int* sched = nullptr;
    if (ctx->bis_order) {
        sched = b.sched.as<int>();
        CK(cudaMemsetAsync(sched, 0, ncpa::kSchedInts * sizeof(int), st));
    }
    tm.mark("host-items");
    const int fit_b = ncpa::bisect_ctas_per_sm();
    const int grid_b = ctx->num_sms * (t.bis_ctas > 0 ? std::min(t.bis_ctas, fit_b) : fit_b);
    ncpa::EigvecArgs ea = eigvec_args(ctx, M, prm, s, w, gs, b);
    const int grid_e = eigvec_grid(ctx, ea, b.ev_cap, t.ev_ctas);
    ea.ck_q1 = (b.own_ck ? b.ck1 : ctx->ck1).as<double>();
    ea.ck_q2 = (b.own_ck ? b.ck2 : ctx->ck2).as<double>();
    ea.ck_e = (b.own_ck ? b.cke : ctx->cke).as<int>();
    ea.ck_slot_stride = ncpa::ck_slot_elems(M->nz_max);
    if (fuse) {
        int* fq = b.fq.as<int>();
        CK(cudaMemsetAsync(fq, 0, ((size_t)2 * b.ev_cap + 2) * sizeof(int), st));
        ncpa::FusedArgs fa{};
        fa.P = P;
        fa.pinfo = d_pinfo;
        fa.s = s;
        fa.counts = b.counts.as<int>();
        fa.bis = b.bis.as<WorkItem>();
        fa.n_bis_dev = b.tot.as<int>();
        fa.tol = kBisectTol;
        fa.mu = b.mu.as<double>();
        fa.err = err;
        fa.pstat = b.pstat.as<int>();
        fa.queue = fq;
        fa.ev_done = fq + b.ev_cap;
        fa.wait_ns = ctx->fuse_wait_ns;
        fa.sched = sched;
        fa.workers = ctx->bis_workers;
        fa.ev_workers_only = ctx->fuse_ev_workers && sched ? 1 : 0;
        fa.q_head = fq + 2 * b.ev_cap;
        fa.q_tail = fq + 2 * b.ev_cap + 1;
        fa.ea = ea;
        // no more warps than the checkpoint scratch has slots (sized for grid_e)
        const int fit_f = ncpa::fused_ctas_per_sm();
        const int grid_f =
            std::min(grid_e, ctx->num_sms * (t.bis_ctas > 0 ? std::min(t.bis_ctas, fit_f) : fit_f));
        check_launch(ctx, ncpa::launch_bisect_eigvec(st, grid_f, fa));
        tm.mark("bisect+eigvec");
        ea.ev_done = fa.ev_done;  // the items the fused launch did not finish
        check_launch(ctx, ncpa::launch_eigvec(st, grid_e, ea));
        tm.mark("eigvec-rest");
    } else {
        // ---- K3 bisection ----
        check_launch(ctx, ncpa::launch_bisect(st, grid_b, d_pinfo, s, b.counts.as<int>(), b.bis.as<WorkItem>(), 0,
                                              b.counter.as<int>(), kBisectTol, b.mu.as<double>(), err,
                                              count_steps ? ctx->d_stats.as<unsigned long long>() : nullptr,
                                              b.tot.as<int>(), sched, ctx->bis_workers));
        tm.mark("bisect");
        // ---- K4 eigenvectors ----
        check_launch(ctx, ncpa::launch_eigvec(st, grid_e, ea));
        tm.mark("eigvec");
    }
    CK(cudaMemcpyAsync(tot_dst, b.tot.p, 3 * sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(info_dst, d_pinfo, P * sizeof(ProblemInfo), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(err_dst, err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
}

// After enqueue_solve: waits for the stream, reports a problem above
// max_modes and device errors, records the mode total and fetches the modes
// to the host mirror unless they stay on the device.
void finish_solve(ncpa_ctx* ctx, PhaseTimer& tm, ncpa_modes* M, const int* tot, const unsigned* err) {
    cudaStream_t st = ctx->stream;
    CK(cudaStreamSynchronize(st));
    if (*err & ncpa::kErrTooMany) {
        CK(cudaMemsetAsync(ctx->d_err.p, 0, sizeof(unsigned), st));
        int worst = 0;
        for (int p = 0; p < M->P; ++p)
            if (M->info[p].c_hi - M->info[p].c_lo > M->info[worst].c_hi - M->info[worst].c_lo) worst = p;
        char buf[160];
        std::snprintf(buf, sizeof buf, "problem %d (f=%g Hz, az=%g) has %d modes > max_modes %d", worst,
                      M->info[worst].freq, M->info[worst].az, M->info[worst].c_hi - M->info[worst].c_lo,
                      M->prm.max_modes);
        throw ApiError(NCPA_ETOOMANY, buf);
    }
    M->Mtot = tot[2];
    M->host_valid = false;
    if (!M->prm.keep_on_device) fetch_modes(M);
    check_device_status(ctx);
    tm.mark("fetch");
}

// Window, Sturm scan, work items, bisection and eigenvectors over all
// problems of M (their matrices built; each problem's rows of s, w, g and kz2
// at the offsets in its ProblemInfo).
void solve_core(ncpa_ctx* ctx, PhaseTimer& tm, ncpa_modes* M, const ncpa_ess_params* prm, bool wkb, DevBuf& s,
                DevBuf& w, DevBuf& g, DevBuf& kz2) {
    cudaStream_t st = ctx->stream;
    const int P = M->P;
    ProblemInfo* d_pinfo = M->d_pinfo.as<ProblemInfo>();
    if (!prm->want_vectors) {  // device-built work items, one host wait at the end
        Tuning t;
        if (ctx->item_override > 0) t.bis_item = std::min(ctx->item_override, ncpa::kWItem);
        SolveBufs b;
        prepare_solve(ctx, M, prm, t.bis_item, b, s.as<double>(), w.as<double>(), g.as<double>());
        unsigned h_err = 0;
        enqueue_solve(ctx, tm, M, prm, wkb, s.as<double>(), w.as<double>(), g.as<double>(), kz2.as<double>(), b, t,
                      ctx->stats && !ctx->stats_fused, ctx->h_tot, M->info.data(), &h_err);
        finish_solve(ctx, tm, M, ctx->h_tot, &h_err);
        return;
    }
    // ---- K2 window ----
    check_launch(ctx, ncpa::launch_window(st, P, d_pinfo, wkb ? kz2.as<double>() : nullptr, wkb ? 1 : 0,
                                          prm->wvnum_filter, prm->c_min, prm->c_max, ctx->d_err.as<unsigned>()));
    tm.mark("window");
    // ---- K3a scan ----
    DevBuf counts;
    counts.alloc((size_t)P * ncpa::kScanMax * 4, st);
    check_launch(ctx, ncpa::launch_scan(st, P, d_pinfo, s.as<double>(), counts.as<int>(), ctx->d_err.as<unsigned>(),
                                        scan_slots(ctx)));
    tm.mark("scan");
    std::vector<int> hcounts((size_t)P * ncpa::kScanMax);
    CK(cudaMemcpyAsync(hcounts.data(), counts.p, hcounts.size() * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(M->info.data(), d_pinfo, P * sizeof(ProblemInfo), cudaMemcpyDeviceToHost, st));
    check_device_status(ctx);
    // ---- modes per problem, offsets, work items ----
    std::vector<WorkItem> items;
    int off = 0;
    for (int p = 0; p < P; ++p) {
        ProblemInfo& pi = M->info[p];
        pi.c_lo = hcounts[(size_t)p * ncpa::kScanMax];
        pi.c_hi = hcounts[(size_t)p * ncpa::kScanMax + pi.n_scan - 1];
        pi.M = std::max(0, pi.c_hi - pi.c_lo);
        if (pi.M > M->prm.max_modes) {
            char buf[160];
            std::snprintf(buf, sizeof buf, "problem %d (f=%g Hz, az=%g) has %d modes > max_modes %d", p, pi.freq,
                          pi.az, pi.M, M->prm.max_modes);
            throw ApiError(NCPA_ETOOMANY, buf);
        }
        pi.off = off;
        off += pi.M;
    }
    // eigenvalues per bisection item: 32 (one per lane).  Smaller items give
    // each eigenvalue more shifts per round but cost more Sturm sequences in
    // total, which measured slower on the 256-frequency workload (16: +26 %,
    // 8: +100 %); NCPA_BISECT_ITEM overrides it for tuning.
    const int item_sz = ctx->item_override > 0 ? ctx->item_override : ncpa::kWItem;
    for (int p = 0; p < P; ++p) {
        const ProblemInfo& pi = M->info[p];
        const int nit = (pi.M + item_sz - 1) / item_sz;
        for (int k = 0; k < nit; ++k) {
            int j0 = (int)((long long)pi.M * k / nit), j1 = (int)((long long)pi.M * (k + 1) / nit);
            items.push_back(WorkItem{p, j0, j1 - j0, 0});
        }
    }
    M->Mtot = off;
    // largest items first: they need the most multisection rounds
    std::stable_sort(items.begin(), items.end(), [](const WorkItem& a, const WorkItem& b) { return a.m > b.m; });
    CK(cudaMemcpyAsync(d_pinfo, M->info.data(), P * sizeof(ProblemInfo), cudaMemcpyHostToDevice, st));
    const int Mt = std::max(1, M->Mtot);
    DevBuf mu, d_items, d_counter;
    mu.alloc((size_t)Mt * 8, st);
    M->d_kr.alloc((size_t)Mt * 8, st);
    M->d_ki.alloc((size_t)Mt * 8, st);
    M->d_vs.alloc((size_t)Mt * 8, st);
    M->d_vr.alloc((size_t)Mt * 8, st);
    M->d_vg.alloc((size_t)Mt * 8, st);
    if (prm->want_vectors) {
        M->vfull_off.resize(P);
        long long acc = 0;
        for (int p = 0; p < P; ++p) {
            M->vfull_off[p] = acc;
            acc += (long long)M->info[p].M * M->info[p].nz;
        }
        M->d_vfull.alloc((size_t)std::max(1LL, acc) * 8, st);
        upload(M->d_vfull_off, M->vfull_off, st);
    }
    const int n_items = (int)items.size();
    if (n_items > 0) {
        upload(d_items, items, st);
        d_counter.alloc(2 * sizeof(int), st);
        CK(cudaMemsetAsync(d_counter.p, 0, 2 * sizeof(int), st));
        // ---- K3 bisection ----
        const int wpc = 4;  // warps per bisection CTA
        int grid_b = std::min((n_items + wpc - 1) / wpc, ctx->num_sms * ncpa::bisect_ctas_per_sm());
        tm.mark("host-items");
        check_launch(ctx, ncpa::launch_bisect(st, grid_b, d_pinfo, s.as<double>(), counts.as<int>(),
                                              d_items.as<WorkItem>(), n_items, d_counter.as<int>(), kBisectTol,
                                              mu.as<double>(), ctx->d_err.as<unsigned>(),
                                              ctx->stats ? ctx->d_stats.as<unsigned long long>() : nullptr));
        tm.mark("bisect");
        // ---- K4 eigenvectors: items of <= kEvItem eigenvalues ----
        std::vector<WorkItem> ev_items;
        for (int p = 0; p < P; ++p) {
            const int Mp = M->info[p].M;
            for (int j0 = 0; j0 < Mp; j0 += ncpa::kEvItem)
                ev_items.push_back(WorkItem{p, j0, std::min(ncpa::kEvItem, Mp - j0), 0});
        }
        DevBuf d_ev_items;
        upload(d_ev_items, ev_items, st);
        const int n_ev = (int)ev_items.size();
        ncpa::EigvecArgs ea{};
        ea.pinfo = d_pinfo;
        ea.s = s.as<double>();
        ea.w = w.as<double>();
        ea.g = prm->want_group_speed ? g.as<double>() : nullptr;
        ea.items = d_ev_items.as<WorkItem>();
        ea.n_items = n_ev;
        ea.counter = d_counter.as<int>() + 1;
        ea.mu = mu.as<double>();
        ea.kr = M->d_kr.as<double>();
        ea.ki = M->d_ki.as<double>();
        ea.vs = M->d_vs.as<double>();
        ea.vr = M->d_vr.as<double>();
        ea.vg = M->d_vg.as<double>();
        ea.vfull = prm->want_vectors ? M->d_vfull.as<double>() : nullptr;
        ea.vfull_off = prm->want_vectors ? M->d_vfull_off.as<long long>() : nullptr;
        const int ewpc = ncpa::kEvWarpsPerCta;
        const int grid_e = std::min((n_ev + ewpc - 1) / ewpc, ctx->num_sms * ncpa::eigvec_ctas_per_sm(ea));
        const long long slot = ncpa::ck_slot_elems(M->nz_max);
        const size_t need = (size_t)grid_e * ewpc * slot;
        if (ctx->ck1.bytes < need * 8) {
            ctx->ck1.alloc(need * 8, st);
            ctx->ck2.alloc(need * 8, st);
            ctx->cke.alloc(need * 4, st);
        }
        ea.ck_q1 = ctx->ck1.as<double>();
        ea.ck_q2 = ctx->ck2.as<double>();
        ea.ck_e = ctx->cke.as<int>();
        ea.ck_slot_stride = slot;
        ea.err = ctx->d_err.as<unsigned>();
        check_launch(ctx, ncpa::launch_eigvec(st, grid_e, ea));
    }
    tm.mark("eigvec");
    // ---- results to host ----
    if (!prm->keep_on_device) fetch_modes(M);
    check_device_status(ctx);
    tm.mark("fetch");
}

void init_modes(ncpa_modes* M, ncpa_ctx* ctx, const ncpa_ess_params* prm, int P) {
    M->ctx = ctx;
    M->prm = *prm;
    if (M->prm.max_modes <= 0) M->prm.max_modes = 4000;
    M->P = P;
    M->info.assign(P, ProblemInfo{});
    M->rho_src_p.assign(P, 1.0);
    M->rho_rcv_p.assign(P, 1.0);
}

bool wants_wkb(const ncpa_ess_params* prm);

// Lays the groups out in one batch (problem records, row offsets), builds
// every group's matrices and runs the window, scan, bisection and
// eigenvector kernels once over all problems.
// Numbers the groups' problems, fills their records (grid, row offsets) and
// returns the doubles needed by s (and g, kz2) and by w.
void layout_groups(ncpa_modes* M, std::vector<Group>& groups, long long& s_tot, long long& w_tot) {
    s_tot = 0;
    w_tot = 0;
    int p = 0;
    M->nz_max = 0;
    for (Group& g : groups) {
        g.p0 = p;
        g.s_base = s_tot;
        g.w_base = w_tot;
        for (int f = 0; f < g.n_freq; ++f)
            for (int a = 0; a < g.n_az; ++a, ++p) {
                ProblemInfo& pi = M->info[p];
                pi.freq = g.freqs[f];
                pi.omega = 2 * kPi * g.freqs[f];
                pi.az = g.az[a];
                pi.ceffmin_bits = 0x7ff0000000000000ull;
                pi.ceffmax_bits = 0ull;
                pi.dz = g.geo.dz;
                pi.nz = g.nz;
                pi.isrc = g.geo.isrc;
                pi.ircv = g.geo.ircv;
                pi.s_off = g.s_base + (long long)(f * g.n_az + a) * g.nz_pad;
                pi.w_off = g.w_base + (long long)f * g.nz_pad;
            }
        s_tot += (long long)g.n_freq * g.n_az * g.nz_pad;
        w_tot += (long long)g.n_freq * g.nz_pad;
        M->nz_max = std::max(M->nz_max, g.nz);
    }
}

void solve_groups(ncpa_ctx* ctx, ncpa_modes* M, const ncpa_ess_params* prm, std::vector<Group>& groups) {
    cudaStream_t st = ctx->stream;
    PhaseTimer tm(ctx);
    tm.mark("start");
    long long s_tot = 0, w_tot = 0;
    layout_groups(M, groups, s_tot, w_tot);
    upload(M->d_pinfo, M->info, st);
    const bool wkb = wants_wkb(prm);
    DevBuf s, w, gs, kz2;
    s.alloc((size_t)s_tot * 8, st);
    w.alloc((size_t)w_tot * 8, st);
    if (wkb) kz2.alloc((size_t)s_tot * 8, st);
    if (prm->want_group_speed) gs.alloc((size_t)s_tot * 8, st);
    double* rho_pairs = pinned(ctx, 2 * groups.size());
    ProblemInfo* d_pinfo = M->d_pinfo.as<ProblemInfo>();
    std::vector<GroupBufs> gb(groups.size());
    for (size_t gi = 0; gi < groups.size(); ++gi) prepare_group(ctx, prm, groups[gi], gb[gi]);
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        const Group& g = groups[gi];
        enqueue_group(ctx, tm, g, gb[gi], wkb, d_pinfo + g.p0, s.as<double>() + g.s_base, w.as<double>() + g.w_base,
                      prm->want_group_speed ? gs.as<double>() + g.s_base : nullptr,
                      wkb ? kz2.as<double>() + g.s_base : nullptr, rho_pairs + 2 * gi);
    }
    solve_core(ctx, tm, M, prm, wkb, s, w, gs, kz2);
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        const Group& g = groups[gi];
        const int np = g.n_freq * g.n_az;
        for (int k = 0; k < np; ++k) {
            M->rho_src_p[g.p0 + k] = rho_pairs[2 * gi];
            M->rho_rcv_p[g.p0 + k] = rho_pairs[2 * gi + 1];
        }
    }
}

// ---------------------------------------------------------------------------
// WMod (wide-angle) solve: WModeSolver::solve (WModeSolver.cpp:257-486)
// ---------------------------------------------------------------------------
constexpr double kWmodTol = 1.0e-15;  // relative to kappa_max = h k_max

// the matrix spacing of WModeSolver::solve, (maxheight - z_min) / Nz_grid
// (WModeSolver.cpp:281; the sampling grid keeps setParams' spacing), and the
// source / receiver rows on it
void wmod_geometry(Group& g, const ncpa_ess_params* prm) {
    double maxheight = prm->maxheight_km * 1000.0;
    if (maxheight >= g.prof->z_hi) maxheight = g.prof->z_hi - 1e-6;
    g.geo.dz = (maxheight - g.geo.z_min) / g.nz;
    if (!(g.geo.dz > 0.0)) throw ApiError(NCPA_EINVAL, "maxheight must lie above the ground");
    g.geo.isrc = (int)std::ceil(prm->sourceheight_km * 1000.0 / g.geo.dz);
    g.geo.ircv = (int)std::ceil(prm->receiverheight_km * 1000.0 / g.geo.dz);
    if (g.geo.isrc < 0 || g.geo.isrc >= g.nz || g.geo.ircv < 0 || g.geo.ircv >= g.nz)
        throw ApiError(NCPA_EINVAL, "source/receiver height outside the grid");
}

struct WmodBufs {
    GroupBufs gb;           // frequencies, azimuths, c_eff and alpha knots, grid fields
    DevBuf wck, wcc, c0c;   // wind component knots and splines, c0 spline
};

// knot-level fields, attenuation weights and coefficient rows of one group
void enqueue_wmod_group(ncpa_ctx* ctx, PhaseTimer& tm, const Group& g, WmodBufs& wb, bool wkb, ProblemInfo* d_pinfo,
                        double* rows, double* w, double* kz2, double* rho_pair) {
    cudaStream_t st = ctx->stream;
    const ncpa_profile* prof = g.prof;
    const int nk = prof->n;
    GroupBufs& b = wb.gb;
    check_launch(ctx, ncpa::launch_ceff_knots(st, nk, g.n_az, b.az.as<double>(), prof->c0.as<double>(),
                                              prof->ws.as<double>(), prof->wd.as<double>(), b.ceffk.as<double>()));
    check_launch(ctx, ncpa::launch_steffen(st, nk, prof->z.as<double>(), b.ceffk.as<double>(), g.n_az, nk,
                                           b.ceffc.as<double>(), 4 * (nk - 1)));
    check_launch(ctx, ncpa::launch_wc_knots(st, nk, g.n_az, b.az.as<double>(), prof->ws.as<double>(),
                                            prof->wd.as<double>(), wb.wck.as<double>()));
    check_launch(ctx, ncpa::launch_steffen(st, nk, prof->z.as<double>(), wb.wck.as<double>(), g.n_az, nk,
                                           wb.wcc.as<double>(), 4 * (nk - 1)));
    check_launch(ctx, ncpa::launch_steffen(st, nk, prof->z.as<double>(), prof->c0.as<double>(), 1, nk,
                                           wb.c0c.as<double>(), 4 * (nk - 1)));
    if (prof->has_attn) {
        for (int f = 0; f < g.n_freq; ++f)
            CK(cudaMemcpyAsync(b.alpha.as<double>() + (size_t)f * nk, prof->attn.p, nk * 8, cudaMemcpyDeviceToDevice,
                               st));
    } else {
        check_launch(ctx, ncpa::launch_alpha_knots(st, nk, g.n_freq, b.freqs.as<double>(), prof->z.as<double>(),
                                                   prof->t.as<double>(), prof->p.as<double>(),
                                                   prof->rho.as<double>(), b.alpha.as<double>()));
    }
    check_launch(ctx, ncpa::launch_steffen(st, nk, prof->z.as<double>(), b.alpha.as<double>(), g.n_freq, nk,
                                           b.alphac.as<double>(), 4 * (nk - 1)));
    CK(cudaMemsetAsync(w, 0, (size_t)g.n_freq * g.nz_pad * 8, st));
    check_launch(ctx, ncpa::launch_grid_common(st, nk, prof->z.as<double>(), prof->rho.as<double>(),
                                               prof->rcoef.as<double>(), prof->p.as<double>(),
                                               prof->pcoef.as<double>(), g.nz, g.geo.z_min, g.geo.dz_grid,
                                               b.rho_g.as<double>(), b.ct_g.as<double>()));
    check_launch(ctx, ncpa::launch_attn_weight(st, nk, prof->z.as<double>(), b.alpha.as<double>(),
                                               b.alphac.as<double>(), g.n_freq, b.freqs.as<double>(), g.nz,
                                               g.geo.z_min, g.geo.dz_grid, b.ct_g.as<double>(), w, g.nz_pad));
    CK(cudaMemcpyAsync(rho_pair, b.rho_g.as<double>() + g.geo.isrc, 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(rho_pair + 1, b.rho_g.as<double>() + g.geo.ircv, 8, cudaMemcpyDeviceToHost, st));
    tm.mark("knots+grid");
    check_launch(ctx, ncpa::launch_wmod_build(st, nk, prof->z.as<double>(), prof->c0.as<double>(),
                                              wb.c0c.as<double>(), wb.wck.as<double>(), wb.wcc.as<double>(),
                                              b.ceffk.as<double>(), b.ceffc.as<double>(), g.n_az,
                                              g.n_freq * g.n_az, d_pinfo, g.nz, g.nz_pad, g.geo.z_min,
                                              g.geo.dz_grid, g.geo.dz, b.admittance, rows, wkb ? kz2 : nullptr));
    tm.mark("matrix");
}

void solve_wmod(ncpa_ctx* ctx, ncpa_modes* M, const ncpa_ess_params* prm, std::vector<Group>& groups) {
    cudaStream_t st = ctx->stream;
    PhaseTimer tm(ctx);
    tm.mark("start");
    for (Group& g : groups) wmod_geometry(g, prm);
    long long s_tot = 0, w_tot = 0;
    layout_groups(M, groups, s_tot, w_tot);
    upload(M->d_pinfo, M->info, st);
    const bool wkb = wants_wkb(prm);
    DevBuf rows, w, kz2;
    rows.alloc((size_t)s_tot * 16, st);
    w.alloc((size_t)w_tot * 8, st);
    if (wkb) kz2.alloc((size_t)s_tot * 8, st);
    double* rho_pairs = pinned(ctx, 2 * groups.size());
    ProblemInfo* d_pinfo = M->d_pinfo.as<ProblemInfo>();
    std::vector<WmodBufs> wbs(groups.size());
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        const Group& g = groups[gi];
        prepare_group(ctx, prm, g, wbs[gi].gb);
        const int nk = g.prof->n;
        wbs[gi].wck.alloc((size_t)g.n_az * nk * 8, st);
        wbs[gi].wcc.alloc((size_t)g.n_az * 4 * (nk - 1) * 8, st);
        wbs[gi].c0c.alloc((size_t)4 * (nk - 1) * 8, st);
    }
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        const Group& g = groups[gi];
        enqueue_wmod_group(ctx, tm, g, wbs[gi], wkb, d_pinfo + g.p0, rows.as<double>() + 2 * g.s_base,
                           w.as<double>() + g.w_base, wkb ? kz2.as<double>() + g.s_base : nullptr, rho_pairs + 2 * gi);
    }
    const int P = M->P;
    unsigned* err = ctx->d_err.as<unsigned>();
    check_launch(ctx, ncpa::launch_window(st, P, d_pinfo, wkb ? kz2.as<double>() : nullptr, wkb ? 1 : 0,
                                          prm->wvnum_filter, prm->c_min, prm->c_max, err));
    tm.mark("window");
    DevBuf counts, bis, ev, tot;
    counts.alloc((size_t)P * ncpa::kScanMax * 4, st);
    check_launch(ctx, ncpa::launch_wscan(st, P, d_pinfo, rows.as<double>(), counts.as<int>(), err));
    tm.mark("scan");
    const int cap_modes = M->prm.max_modes;
    const int bis_cap = P * ((cap_modes + ncpa::kWItem - 1) / ncpa::kWItem);
    const int ev_cap = P * ((cap_modes + ncpa::kEvItem - 1) / ncpa::kEvItem);
    bis.alloc((size_t)bis_cap * sizeof(WorkItem), st);
    ev.alloc((size_t)ev_cap * sizeof(WorkItem), st);
    tot.alloc(4 * sizeof(int), st);
    // fused bisection + eigenvector launch, as on the ESS path (full vectors
    // excepted; kernels alone under per-phase timing)
    const bool fuse = ctx->fuse_solve && !ctx->timing && (!ctx->stats || ctx->stats_fused) && !prm->want_vectors;
    DevBuf pstat, fq, sched_buf;
    if (fuse) pstat.alloc((size_t)3 * P * sizeof(int), st);
    int* sched = nullptr;
    if (ctx->bis_order) {
        sched_buf.alloc(ncpa::kSchedInts * sizeof(int), st);
        sched = sched_buf.as<int>();
        CK(cudaMemsetAsync(sched, 0, ncpa::kSchedInts * sizeof(int), st));
    }
    check_launch(ctx, ncpa::launch_make_items(st, P, d_pinfo, counts.as<int>(), cap_modes, ncpa::kWItem,
                                              bis.as<WorkItem>(), bis_cap, ev.as<WorkItem>(), ev_cap,
                                              tot.as<int>(), err, fuse ? pstat.as<int>() : nullptr,
                                              ctx->bis_order ? 1 : 0));
    // mode counts to the host (sizes of the outputs and of the vectors)
    int* h_tot = ctx->h_tot;
    unsigned h_err = 0;
    CK(cudaMemcpyAsync(h_tot, tot.p, 3 * sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(M->info.data(), d_pinfo, P * sizeof(ProblemInfo), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&h_err, err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (h_err & ncpa::kErrTooMany) {
        CK(cudaMemsetAsync(ctx->d_err.p, 0, sizeof(unsigned), st));
        throw ApiError(NCPA_ETOOMANY, "a problem has more wide-angle modes than max_modes");
    }
    check_device_status(ctx);
    tm.mark("host-items");
    const int n_bis = h_tot[0], n_ev = h_tot[1];
    M->Mtot = h_tot[2];
    const size_t mt = (size_t)std::max(1, M->Mtot);
    DevBuf mu;
    mu.alloc(mt * 8, st);
    for (DevBuf* b : {&M->d_kr, &M->d_ki, &M->d_vs, &M->d_vr, &M->d_vg}) b->alloc(mt * 8, st);
    if (prm->want_vectors) {
        M->vfull_off.resize(P);
        long long acc = 0;
        for (int p = 0; p < P; ++p) {
            M->vfull_off[p] = acc;
            acc += (long long)M->info[p].M * M->info[p].nz;
        }
        M->d_vfull.alloc((size_t)std::max(1LL, acc) * 8, st);
        upload(M->d_vfull_off, M->vfull_off, st);
    }
    ncpa::EigvecArgs ea{};
    ea.pinfo = d_pinfo;
    ea.s = rows.as<double>();
    ea.w = w.as<double>();
    ea.g = nullptr;
    ea.items = ev.as<WorkItem>();
    ea.n_items = 0;
    ea.n_items_dev = tot.as<int>() + 1;
    ea.mu = mu.as<double>();
    ea.kr = M->d_kr.as<double>();
    ea.ki = M->d_ki.as<double>();
    ea.vs = M->d_vs.as<double>();
    ea.vr = M->d_vr.as<double>();
    ea.vg = M->d_vg.as<double>();
    ea.vfull = prm->want_vectors ? M->d_vfull.as<double>() : nullptr;
    ea.vfull_off = prm->want_vectors ? M->d_vfull_off.as<long long>() : nullptr;
    ea.err = err;
    const int fit = ncpa::eigvec_wmod_ctas_per_sm(ea);
    const int grid_e = std::max(1, std::min((n_ev + ncpa::kEvWarpsPerCta - 1) / ncpa::kEvWarpsPerCta,
                                            ctx->num_sms * fit));
    const bool fused = fuse && n_ev > 0;
    // the fused launch runs on every SM (idle warps take eigenvector items from
    // the start), so the checkpoint scratch has a slot for each of its warps
    const int grid_f = fused ? ctx->num_sms * ncpa::fused_wmod_ctas_per_sm() : 0;
    const long long slot = ncpa::ck_slot_elems(M->nz_max);
    const size_t need = (size_t)std::max(grid_e, grid_f) * ncpa::kEvWarpsPerCta * slot;
    if (n_ev > 0 && ctx->ck1.bytes < need * 8) {
        ctx->ck1.alloc(need * 8, st);
        ctx->ck2.alloc(need * 8, st);
        ctx->cke.alloc(need * 4, st);
    }
    ea.ck_q1 = ctx->ck1.as<double>();
    ea.ck_q2 = ctx->ck2.as<double>();
    ea.ck_e = ctx->cke.as<int>();
    ea.ck_slot_stride = slot;
    if (fused) {
        fq.alloc(((size_t)2 * ev_cap + 2) * sizeof(int), st);
        CK(cudaMemsetAsync(fq.p, 0, ((size_t)2 * ev_cap + 2) * sizeof(int), st));
        ncpa::FusedArgs fa{};
        fa.P = P;
        fa.pinfo = d_pinfo;
        fa.s = rows.as<double>();
        fa.counts = counts.as<int>();
        fa.bis = bis.as<WorkItem>();
        fa.n_bis_dev = tot.as<int>();
        fa.tol = kWmodTol;
        fa.mu = mu.as<double>();
        fa.err = err;
        fa.pstat = pstat.as<int>();
        fa.queue = fq.as<int>();
        fa.ev_done = fq.as<int>() + ev_cap;
        fa.wait_ns = ctx->fuse_wait_ns;
        fa.sched = sched;
        fa.workers = ctx->bis_workers;
        fa.ev_workers_only = ctx->fuse_ev_workers && sched ? 1 : 0;
        fa.q_head = fq.as<int>() + 2 * ev_cap;
        fa.q_tail = fq.as<int>() + 2 * ev_cap + 1;
        fa.ea = ea;
        check_launch(ctx, ncpa::launch_bisect_eigvec_wmod(st, grid_f, fa));
        tm.mark("bisect+eigvec");
        ea.ev_done = fa.ev_done;  // the items the fused launch did not finish
        check_launch(ctx, ncpa::launch_eigvec_wmod(st, grid_e, ea));
    } else {
        if (n_bis > 0) {
            const int grid_b = ctx->num_sms * ncpa::bisect_wmod_ctas_per_sm();
            check_launch(ctx, ncpa::launch_bisect_wmod(st, grid_b, d_pinfo, rows.as<double>(), counts.as<int>(),
                                                       bis.as<WorkItem>(), kWmodTol, mu.as<double>(), err,
                                                       ctx->stats ? ctx->d_stats.as<unsigned long long>() : nullptr,
                                                       tot.as<int>(), sched, ctx->bis_workers));
        }
        tm.mark("bisect");
        if (n_ev > 0) check_launch(ctx, ncpa::launch_eigvec_wmod(st, grid_e, ea));
    }
    tm.mark(fused ? "eigvec-rest" : "eigvec");
    M->host_valid = false;
    if (!prm->keep_on_device) fetch_modes(M);
    check_device_status(ctx);
    tm.mark("fetch");
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        const Group& g = groups[gi];
        for (int k = 0; k < g.n_freq * g.n_az; ++k) {
            M->rho_src_p[g.p0 + k] = rho_pairs[2 * gi];
            M->rho_rcv_p[g.p0 + k] = rho_pairs[2 * gi + 1];
        }
    }
}

bool wants_wkb(const ncpa_ess_params* prm) {
    return !prm->turnoff_wkb && std::fabs(prm->sourceheight_km * 1000.0) < 1.0e-3 &&
           std::fabs(prm->receiverheight_km * 1000.0) < 1.0e-3;
}


// Plan: buffers, pinned staging and the instantiated graph of one captured
// batched solve.
struct PlanData {
    ncpa_ctx* ctx = nullptr;
    std::unique_ptr<ncpa_modes> M;
    ncpa_ess_params prm{};
    std::vector<std::vector<double>> freqs, azs;  // host copies the groups point at
    std::vector<Group> groups;
    std::vector<GroupBufs> gb;
    DevBuf s, w, gs, kz2, pinfo_init;
    SolveBufs sb;
    Tuning tuning;
    bool wkb = false, with_tl = false, ran = false;
    ncpa_tl_params tp{};
    ProblemInfo* h_info = nullptr;  // pinned staging written by the graph
    int* h_tot = nullptr;
    unsigned* h_err = nullptr;
    double* h_rho = nullptr;
    cudaGraphExec_t exec = nullptr;
    long long kernels = 0;  // kernel launches in one replay
    int fit_e = 1;          // eigenvector CTAs per SM that fit
    double tuned_ms = 0.0;
};

// The device sequence of a plan (captured into its graph).
void enqueue_plan(PlanData& pl, const Tuning& t) {
    ncpa_ctx* ctx = pl.ctx;
    cudaStream_t st = ctx->stream;
    ncpa_modes* M = pl.M.get();
    PhaseTimer tm(ctx);  // records nothing: timing is off while capturing
    ProblemInfo* d_pinfo = M->d_pinfo.as<ProblemInfo>();
    CK(cudaMemcpyAsync(d_pinfo, pl.pinfo_init.p, (size_t)M->P * sizeof(ProblemInfo), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemsetAsync(ctx->d_err.p, 0, sizeof(unsigned), st));
    const bool grp = pl.prm.want_group_speed != 0;
    for (size_t gi = 0; gi < pl.groups.size(); ++gi) {
        const Group& g = pl.groups[gi];
        enqueue_group(ctx, tm, g, pl.gb[gi], pl.wkb, d_pinfo + g.p0, pl.s.as<double>() + g.s_base,
                      pl.w.as<double>() + g.w_base, grp ? pl.gs.as<double>() + g.s_base : nullptr,
                      pl.wkb ? pl.kz2.as<double>() + g.s_base : nullptr, pl.h_rho + 2 * gi);
    }
    enqueue_solve(ctx, tm, M, &pl.prm, pl.wkb, pl.s.as<double>(), pl.w.as<double>(), grp ? pl.gs.as<double>() : nullptr,
                  pl.kz2.as<double>(), pl.sb, t, false, pl.h_tot, pl.h_info, pl.h_err);
    if (pl.with_tl)
        check_launch(ctx, ncpa::launch_tl1d(st, M->P, d_pinfo, M->d_kr.as<double>(), M->d_ki.as<double>(),
                                            M->d_vs.as<double>(), M->d_vr.as<double>(), pl.tp.n_ranges, pl.tp.dr_m,
                                            pl.tp.lossless, M->tl_re.as<double>(), M->tl_im.as<double>(),
                                            M->tl_inc.as<double>()));
}

// Captures the plan's sequence with launch shapes t and instantiates it.
cudaGraphExec_t capture_plan(PlanData& pl, const Tuning& t) {
    ncpa_ctx* ctx = pl.ctx;
    cudaStream_t st = ctx->stream;
    const bool timing = ctx->timing, stats = ctx->stats;
    const long long l0 = ctx->launches;
    ctx->timing = ctx->stats = false;
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    try {
        enqueue_plan(pl, t);
    } catch (...) {
        cudaStreamEndCapture(st, &graph);
        if (graph) cudaGraphDestroy(graph);
        ctx->timing = timing;
        ctx->stats = stats;
        ctx->launches = l0;
        throw;
    }
    ctx->timing = timing;
    ctx->stats = stats;
    pl.kernels = ctx->launches - l0;  // counted per replay instead
    ctx->launches = l0;
    CK(cudaStreamEndCapture(st, &graph));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) throw CudaError(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    return exec;
}

// After a replay: one wait, then the records, totals and errors.
void finish_plan(PlanData& pl) {
    ncpa_ctx* ctx = pl.ctx;
    ncpa_modes* M = pl.M.get();
    CK(cudaStreamSynchronize(ctx->stream));
    std::memcpy(M->info.data(), pl.h_info, (size_t)M->P * sizeof(ProblemInfo));
    PhaseTimer tm(ctx);
    finish_solve(ctx, tm, M, pl.h_tot, pl.h_err);
    for (size_t gi = 0; gi < pl.groups.size(); ++gi) {
        const Group& g = pl.groups[gi];
        for (int k = 0; k < g.n_freq * g.n_az; ++k) {
            M->rho_src_p[g.p0 + k] = pl.h_rho[2 * gi];
            M->rho_rcv_p[g.p0 + k] = pl.h_rho[2 * gi + 1];
        }
    }
    pl.ran = true;
}

// Replays exec reps times (after one untimed replay) and returns ms per replay.
double time_graph(PlanData& pl, cudaGraphExec_t exec, int reps) {
    cudaStream_t st = pl.ctx->stream;
    CK(cudaGraphLaunch(exec, st));
    pl.ctx->launches += pl.kernels;
    finish_plan(pl);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, st));
    for (int r = 0; r < reps; ++r) CK(cudaGraphLaunch(exec, st));
    pl.ctx->launches += pl.kernels * reps;
    CK(cudaEventRecord(e1, st));
    finish_plan(pl);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return (double)ms / reps;
}

}  // namespace

extern "C" {

const char* ncpa_status_str(ncpa_status s) {
    switch (s) {
        case NCPA_OK: return "ok";
        case NCPA_EINVAL: return "invalid argument";
        case NCPA_ENOMEM: return "out of memory";
        case NCPA_ECUDA: return "CUDA error";
        case NCPA_EPARSE: return "parse error";
        case NCPA_ETOOMANY: return "too many modes";
        case NCPA_EIO: return "I/O error";
        case NCPA_ETIMEDOUT: return "device wait timed out";
        case NCPA_ENODEV: return "no CUDA device";
    }
    return "unknown status";
}

const char* ncpa_last_error(const ncpa_ctx* ctx) { return ctx ? ctx->err.c_str() : ""; }

long long ncpa_kernel_launches(const ncpa_ctx* ctx) { return ctx ? ctx->launches : 0; }

void* ncpa_ctx_stream(ncpa_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

ncpa_status ncpa_ctx_set_timing(ncpa_ctx* ctx, int on) {
    if (!ctx || on < 0 || on > 2) return NCPA_EINVAL;
    ctx->stats = on != 0;
    ctx->stats_fused = on == 2;
    return NCPA_OK;
}

ncpa_status ncpa_ctx_reset_stats(ncpa_ctx* ctx) {
    if (!ctx) return NCPA_EINVAL;
    ctx->phase.clear();
    return guarded(ctx, [&]() -> ncpa_status {
        CK(cudaMemsetAsync(ctx->d_stats.p, 0, 4 * sizeof(unsigned long long), ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        return NCPA_OK;
    });
}

ncpa_status ncpa_ctx_phase_stats(const ncpa_ctx* ctx, const char* phase, double* total_ms, long long* calls) {
    if (!ctx || !phase) return NCPA_EINVAL;
    auto it = ctx->phase.find(phase);
    if (total_ms) *total_ms = it == ctx->phase.end() ? 0.0 : it->second.first;
    if (calls) *calls = it == ctx->phase.end() ? 0 : it->second.second;
    return NCPA_OK;
}

ncpa_status ncpa_ctx_sturm_steps(ncpa_ctx* ctx, long long* steps) {
    if (!ctx || !steps) return NCPA_EINVAL;
    return guarded(ctx, [&]() -> ncpa_status {
        unsigned long long h = 0;
        CK(cudaMemcpyAsync(&h, ctx->d_stats.p, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        *steps = (long long)h;
        return NCPA_OK;
    });
}

ncpa_status ncpa_ctx_bisect_steps(ncpa_ctx* ctx, long long* steps, long long* deriv_steps) {
    if (!ctx || !steps || !deriv_steps) return NCPA_EINVAL;
    return guarded(ctx, [&]() -> ncpa_status {
        unsigned long long h[2] = {0, 0};
        CK(cudaMemcpyAsync(h, ctx->d_stats.p, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        *steps = (long long)h[0];
        *deriv_steps = (long long)h[1];
        return NCPA_OK;
    });
}

ncpa_status ncpa_ctx_sum_fixups(ncpa_ctx* ctx, long long* recomputed, long long* points) {
    if (!ctx || !recomputed || !points) return NCPA_EINVAL;
    return guarded(ctx, [&]() -> ncpa_status {
        int h = 0;
        if (ctx->ms_fixcnt.p) {
            CK(cudaMemcpyAsync(&h, ctx->ms_fixcnt.p, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
        }
        *recomputed = h;
        *points = ctx->ms_last_points;
        return NCPA_OK;
    });
}

ncpa_status ncpa_ctx_sum_guard(ncpa_ctx* ctx, double* eps, double* tau, int* tile_ranges) {
    if (!ctx || !eps || !tau) return NCPA_EINVAL;
    *eps = ctx->ms_last_eps;
    *tau = ctx->ms_last_tau;
    if (tile_ranges) *tile_ranges = ncpa::ms_tile_ranges();
    return NCPA_OK;
}

ncpa_status ncpa_ctx_sum_schedule(ncpa_ctx* ctx, int* t_stages, int* g_stages, int* variants, double* times_ms) {
    if (!ctx || !t_stages || !g_stages) return NCPA_EINVAL;
    ncpa::ms_tc_variant_shape(ctx->ms_last_fmt, ctx->ms_last_variant, t_stages, g_stages);
    if (variants) *variants = ncpa::ms_tc_variants();
    if (times_ms)
        for (size_t v = 0; v < ctx->ms_last_times.size(); ++v) times_ms[v] = ctx->ms_last_times[v];
    return NCPA_OK;
}

ncpa_status ncpa_probe_fp64_peak(ncpa_ctx* ctx, double* tflops) {
    if (!ctx || !tflops) return NCPA_EINVAL;
    return guarded(ctx, [&]() -> ncpa_status {
        CK(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        DevBuf out;
        out.alloc(8, st);
        const int block = 256, grid = ctx->num_sms * 8;
        cudaEvent_t a, b;
        CK(cudaEventCreate(&a));
        CK(cudaEventCreate(&b));
        int iters = 1 << 12;
        float ms = 0.f;
        for (int rep = 0; rep < 8; ++rep) {  // grow until ~50 ms
            CK(cudaEventRecord(a, st));
            check_launch(ctx, ncpa::launch_fp64_probe(st, grid, block, iters, out.as<double>()));
            CK(cudaEventRecord(b, st));
            CK(cudaEventSynchronize(b));
            CK(cudaEventElapsedTime(&ms, a, b));
            if (ms > 40.f) break;
            iters *= 2;
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        const double flops = 2.0 * 8.0 * (double)iters * grid * block;
        *tflops = flops / (ms * 1e-3) / 1e12;
        return NCPA_OK;
    });
}

ncpa_status ncpa_ctx_create(ncpa_ctx** out, const ncpa_ctx_opts* opts) {
    if (!out) return NCPA_EINVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return NCPA_ENODEV;
    auto ctx = std::make_unique<ncpa_ctx>();
    ctx->device = opts ? opts->device : 0;
    if (ctx->device < 0 || ctx->device >= ndev) return NCPA_EINVAL;
    ncpa_status s = guarded(ctx.get(), [&]() -> ncpa_status {
        CK(cudaSetDevice(ctx->device));
        cudaDeviceProp prop;
        CK(cudaGetDeviceProperties(&prop, ctx->device));
        if (prop.major < 10) throw ApiError(NCPA_ENODEV, "this library is built for sm_100a (B200)");
        ctx->num_sms = prop.multiProcessorCount;
        CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        // keep freed blocks of the stream-ordered allocator cached in the pool
        cudaMemPool_t pool;
        CK(cudaDeviceGetDefaultMemPool(&pool, ctx->device));
        unsigned long long thr = ~0ull;
        CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
        ctx->d_err.alloc(sizeof(unsigned), ctx->stream);
        CK(cudaMemsetAsync(ctx->d_err.p, 0, sizeof(unsigned), ctx->stream));
        ctx->d_stats.alloc(4 * sizeof(unsigned long long), ctx->stream);
        CK(cudaMemsetAsync(ctx->d_stats.p, 0, 4 * sizeof(unsigned long long), ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        CK(cudaHostAlloc((void**)&ctx->h_tot, 64, cudaHostAllocDefault));
        const char* tv = std::getenv("NCPA_TIMING");
        ctx->timing = tv && tv[0] == '1';
        if (const char* fv = std::getenv("NCPA_FUSE_SOLVE")) ctx->fuse_solve = fv[0] != '0';
        if (const char* wv = std::getenv("NCPA_FUSE_WAIT_NS")) ctx->fuse_wait_ns = std::strtoull(wv, nullptr, 10);
        if (const char* mv = std::getenv("NCPA_MS_TUNE")) ctx->ms_tune = mv[0] != '0';
        if (const char* ov = std::getenv("NCPA_BISECT_ORDER")) ctx->bis_order = ov[0] != '0';
        if (const char* ev = std::getenv("NCPA_FUSE_EV_WORKERS")) ctx->fuse_ev_workers = ev[0] != '0';
        if (const char* sv = std::getenv("NCPA_SCAN_TRIM")) ctx->scan_trim = sv[0] != '0';
        if (const char* tv2 = std::getenv("NCPA_TL2D_SUM"))
            ctx->tl2d_method = std::atoi(tv2) == NCPA_SUM_TC_GUARDED ? NCPA_SUM_TC_GUARDED : NCPA_SUM_FP64;
        if (const char* wv = std::getenv("NCPA_BISECT_WORKERS")) {
            const int v = std::atoi(wv);
            if (v >= 1 && v <= 16) ctx->bis_workers = v;
        }
        // tuning override of the eigenvalues per bisection item (1..32)
        if (const char* iv = std::getenv("NCPA_BISECT_ITEM")) {
            const int v = std::atoi(iv);
            if (v >= 1 && v <= 32) ctx->item_override = v;
        }
        return NCPA_OK;
    });
    if (s != NCPA_OK) return s;
    *out = ctx.release();
    return NCPA_OK;
}

ncpa_status ncpa_ctx_destroy(ncpa_ctx* ctx) {
    if (!ctx) return NCPA_EINVAL;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->twiddle.clear();
    ctx->bb_out.release();
    ctx->d_stats.release();
    ctx->ck1.release();
    ctx->ck2.release();
    ctx->cke.release();
    ctx->d_err.release();
    for (DevBuf* b : {&ctx->ms_img, &ctx->ms_q, &ctx->ms_tab, &ctx->ms_raw, &ctx->ms_vz, &ctx->ms_idx, &ctx->ms_re,
                      &ctx->ms_im, &ctx->ms_spart, &ctx->ms_b64, &ctx->ms_tp64, &ctx->ms_a64, &ctx->ms_fix,
                      &ctx->ms_fixcnt})
        b->release();  // stream-ordered frees need the stream alive
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->h_pin) cudaFreeHost(ctx->h_pin);
    if (ctx->h_tot) cudaFreeHost(ctx->h_tot);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return NCPA_OK;
}

ncpa_status ncpa_ctx_synchronize(ncpa_ctx* ctx) {
    if (!ctx) return NCPA_EINVAL;
    return guarded(ctx, [&]() -> ncpa_status {
        CK(cudaStreamSynchronize(ctx->stream));
        return NCPA_OK;
    });
}

// ---------------------------------------------------------------------------
// profiles
// ---------------------------------------------------------------------------
namespace {
// Copies the knot columns into the profile's allocated arrays and derives
// the pressure / density splines, c0 and wind speed / direction on the
// device.  No synchronisation: pageable uploads are staged before the copy
// calls return, and everything later is ordered on the stream.
void fill_profile(ncpa_ctx* ctx, ncpa_profile* P, const ncpa_profile_desc* d) {
    cudaStream_t st = ctx->stream;
    const int n = P->n;
    const std::pair<DevBuf*, const double*> cols[] = {{&P->z, d->z}, {&P->u, d->u}, {&P->v, d->v},
                                                      {&P->t, d->t}, {&P->p, d->p}, {&P->rho, d->rho}};
    for (const auto& c : cols) CK(cudaMemcpyAsync(c.first->p, c.second, n * sizeof(double), cudaMemcpyHostToDevice, st));
    if (d->c0) CK(cudaMemcpyAsync(P->c0.p, d->c0, n * sizeof(double), cudaMemcpyHostToDevice, st));
    if (d->attn) CK(cudaMemcpyAsync(P->attn.p, d->attn, n * sizeof(double), cudaMemcpyHostToDevice, st));
    check_launch(ctx, ncpa::launch_steffen(st, n, P->z.as<double>(), P->p.as<double>(), 1, n, P->pcoef.as<double>(),
                                           4 * (n - 1)));
    check_launch(ctx, ncpa::launch_steffen(st, n, P->z.as<double>(), P->rho.as<double>(), 1, n,
                                           P->rcoef.as<double>(), 4 * (n - 1)));
    check_launch(ctx, ncpa::launch_profile_derived(st, n, P->z.as<double>(), P->u.as<double>(), P->v.as<double>(),
                                                   P->p.as<double>(), P->rho.as<double>(), P->pcoef.as<double>(),
                                                   P->rcoef.as<double>(), d->c0 ? 1 : 0, P->c0.as<double>(),
                                                   P->ws.as<double>(), P->wd.as<double>()));
}
}  // namespace


ncpa_status ncpa_profile_create(ncpa_ctx* ctx, const ncpa_profile_desc* d, ncpa_profile** out) {
    if (!ctx || !d || !out) return NCPA_EINVAL;
    *out = nullptr;
    return guarded(ctx, [&]() -> ncpa_status {
        const int n = d->n_knots;
        if (n < 3) throw ApiError(NCPA_EINVAL, "profile needs at least 3 knots");
        if (!d->z || !d->u || !d->v || !d->t || !d->p || !d->rho)
            throw ApiError(NCPA_EINVAL, "profile arrays z, u, v, t, p, rho are required");
        for (int i = 1; i < n; ++i)
            if (!(d->z[i] > d->z[i - 1])) throw ApiError(NCPA_EINVAL, "profile altitudes must increase strictly");
        CK(cudaSetDevice(ctx->device));
        auto P = std::make_unique<ncpa_profile>();
        P->ctx = ctx;
        P->n = n;
        cudaStream_t st = ctx->stream;
        for (DevBuf* b : {&P->z, &P->u, &P->v, &P->t, &P->p, &P->rho, &P->c0, &P->ws, &P->wd})
            b->alloc(n * sizeof(double), st);
        P->pcoef.alloc(4 * (n - 1) * sizeof(double), st);
        P->rcoef.alloc(4 * (n - 1) * sizeof(double), st);
        if (d->attn) {
            P->attn.alloc(n * sizeof(double), st);
            P->has_attn = true;
        }
        fill_profile(ctx, P.get(), d);
        P->z0 = d->z0_m;
        P->has_z0 = d->has_z0;
        P->z_lo = d->z[0];
        P->z_hi = d->z[n - 1];
        // no synchronisation: pageable uploads are staged before the copy
        // calls return, and everything later is ordered on the stream
        *out = P.release();
        return NCPA_OK;
    });
}

ncpa_status ncpa_profile_load(ncpa_ctx* ctx, const char* path, const char* header_path, ncpa_profile** out) {
    if (!ctx || !path || !out) return NCPA_EINVAL;
    *out = nullptr;
    ncpa::SiProfile S;
    ncpa_status s = guarded(ctx, [&]() -> ncpa_status {
        auto parsed = ncpa::read_profile(path, header_path ? header_path : "");
        S = ncpa::to_si_profile(parsed);
        return NCPA_OK;
    });
    if (s != NCPA_OK) return s;
    ncpa_profile_desc d{};
    d.n_knots = (int)S.z.size();
    d.z = S.z.data();
    d.u = S.u.data();
    d.v = S.v.data();
    d.t = S.t.data();
    d.p = S.p.data();
    d.rho = S.rho.data();
    d.c0 = S.has_c0 ? S.c0.data() : nullptr;
    d.attn = nullptr;
    d.z0_m = S.z0;
    d.has_z0 = S.has_z0;
    return ncpa_profile_create(ctx, &d, out);
}

namespace {
ncpa_status create_from_si(ncpa_ctx* ctx, const ncpa::SiProfile& S, ncpa_profile** out) {
    ncpa_profile_desc d{};
    d.n_knots = (int)S.z.size();
    d.z = S.z.data();
    d.u = S.u.data();
    d.v = S.v.data();
    d.t = S.t.data();
    d.p = S.p.data();
    d.rho = S.rho.data();
    d.c0 = S.has_c0 ? S.c0.data() : nullptr;
    d.attn = nullptr;
    d.z0_m = S.z0;
    d.has_z0 = S.has_z0;
    return ncpa_profile_create(ctx, &d, out);
}
}  // namespace

ncpa_status ncpa_g2s_convert(const char* g2s_path, const char* ncpa_path, double* lat, double* lon) {
    if (!g2s_path || !ncpa_path) return NCPA_EINVAL;
    return guarded(nullptr, [&]() -> ncpa_status {
        double la, lo;
        const ncpa::ParsedProfile P = ncpa::read_g2s_profile(g2s_path, la, lo);
        ncpa::write_ncpa_profile(P, {"U", "V", "T", "RHO", "P"}, ncpa_path);
        if (lat) *lat = la;
        if (lon) *lon = lo;
        return NCPA_OK;
    });
}

ncpa_status ncpa_profile_load_g2s(ncpa_ctx* ctx, const char* path, ncpa_profile** out) {
    if (!ctx || !path || !out) return NCPA_EINVAL;
    *out = nullptr;
    ncpa::SiProfile S;
    ncpa_status s = guarded(ctx, [&]() -> ncpa_status {
        double la, lo;
        S = ncpa::to_si_profile(ncpa::read_g2s_profile(path, la, lo));
        return NCPA_OK;
    });
    if (s != NCPA_OK) return s;
    return create_from_si(ctx, S, out);
}

ncpa_status ncpa_profile_set_attn(ncpa_profile* prof, const double* z_km, const double* attn, int n) {
    if (!prof || !z_km || !attn || n < 2) return NCPA_EINVAL;
    if (prof->plan_refs > 0) return fail(prof->ctx, NCPA_EINVAL, "profile is used by a plan");
    ncpa_ctx* ctx = prof->ctx;
    return guarded(ctx, [&]() -> ncpa_status {
        for (int i = 1; i < n; ++i)
            if (!(z_km[i] > z_km[i - 1])) throw ApiError(NCPA_EINVAL, "attenuation heights must increase strictly");
        CK(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        // extend the table to the profile's range with its end values, in
        // km like the reference (Atmosphere1D.cpp:365-396)
        std::vector<double> hz(prof->n);
        CK(cudaMemcpyAsync(hz.data(), prof->z.p, prof->n * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (auto& z : hz) z = z * 0.001;
        std::vector<double> za(z_km, z_km + n), aa(attn, attn + n);
        if (za.front() > hz.front()) {
            za.insert(za.begin(), hz.front());
            aa.insert(aa.begin(), aa.front());
        }
        if (za.back() < hz.back()) {
            za.push_back(hz.back());
            aa.push_back(aa.back());
        }
        const int na = (int)za.size();
        DevBuf dza, daa, dcoef, dq;
        upload(dza, za, st);
        upload(daa, aa, st);
        upload(dq, hz, st);
        dcoef.alloc((size_t)4 * (na - 1) * 8, st);
        check_launch(ctx, ncpa::launch_steffen(st, na, dza.as<double>(), daa.as<double>(), 1, na, dcoef.as<double>(),
                                               4 * (na - 1)));
        prof->attn.alloc((size_t)prof->n * 8, st);
        check_launch(ctx, ncpa::launch_spline_eval(st, na, dza.as<double>(), daa.as<double>(), dcoef.as<double>(),
                                                   prof->n, dq.as<double>(), prof->attn.as<double>()));
        prof->has_attn = true;
        CK(cudaStreamSynchronize(st));
        return NCPA_OK;
    });
}

ncpa_status ncpa_profile_load_attn(ncpa_profile* prof, const char* path) {
    if (!prof || !path) return NCPA_EINVAL;
    std::vector<double> zk, a;
    ncpa_status s = guarded(prof->ctx, [&]() -> ncpa_status {
        ncpa::read_attn_file(path, zk, a);
        return NCPA_OK;
    });
    if (s != NCPA_OK) return s;
    return ncpa_profile_set_attn(prof, zk.data(), a.data(), (int)zk.size());
}

ncpa_status ncpa_profile_knots(ncpa_profile* prof, double az_deg, double* z, double* u, double* v, double* t,
                               double* p, double* rho, double* c0, double* ceff) {
    if (!prof) return NCPA_EINVAL;
    ncpa_ctx* ctx = prof->ctx;
    return guarded(ctx, [&]() -> ncpa_status {
        CK(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        const int n = prof->n;
        DevBuf daz, dce;
        if (ceff) {
            upload(daz, &az_deg, 1, st);
            dce.alloc((size_t)n * 8, st);
            check_launch(ctx, ncpa::launch_ceff_knots(st, n, 1, daz.as<double>(), prof->c0.as<double>(),
                                                      prof->ws.as<double>(), prof->wd.as<double>(),
                                                      dce.as<double>()));
        }
        const std::pair<double*, const DevBuf*> cols[] = {{z, &prof->z},   {u, &prof->u},     {v, &prof->v},
                                                          {t, &prof->t},   {p, &prof->p},     {rho, &prof->rho},
                                                          {c0, &prof->c0}, {ceff, &dce}};
        for (const auto& c : cols)
            if (c.first) CK(cudaMemcpyAsync(c.first, c.second->p, n * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return NCPA_OK;
    });
}

ncpa_status ncpa_profile_z0(const ncpa_profile* prof, double* z0_m, int* has_z0) {
    if (!prof) return NCPA_EINVAL;
    if (z0_m) *z0_m = prof->z0;
    if (has_z0) *has_z0 = prof->has_z0;
    return NCPA_OK;
}

ncpa_status ncpa_profile_destroy(ncpa_profile* prof) {
    if (!prof) return NCPA_EINVAL;
    if (prof->plan_refs > 0) return fail(prof->ctx, NCPA_EINVAL, "profile is used by a plan; destroy the plan first");
    cudaSetDevice(prof->ctx->device);
    cudaStreamSynchronize(prof->ctx->stream);
    delete prof;
    return NCPA_OK;
}

ncpa_status ncpa_profile_info(const ncpa_profile* prof, int* n, double* z_lo, double* z_hi) {
    if (!prof) return NCPA_EINVAL;
    if (n) *n = prof->n;
    if (z_lo) *z_lo = prof->z_lo;
    if (z_hi) *z_hi = prof->z_hi;
    return NCPA_OK;
}

// ---------------------------------------------------------------------------
// batched ESS solve
// ---------------------------------------------------------------------------
void ncpa_ess_params_default(ncpa_ess_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->nz_grid = 20000;
    p->maxheight_km = 150.0;
    p->max_modes = 4000;
}

ncpa_status ncpa_ess_solve(ncpa_ctx* ctx, const ncpa_profile* prof, const ncpa_ess_params* prm,
                           const double* freqs, int n_freq, const double* az_deg, int n_az, ncpa_modes** out) {
    if (!ctx || !prof || !prm || !freqs || !az_deg || !out) return NCPA_EINVAL;
    *out = nullptr;
    return guarded(ctx, [&]() -> ncpa_status {
        if (n_freq < 1 || n_az < 1) throw ApiError(NCPA_EINVAL, "need at least one frequency and azimuth");
        check_ess_params(prm);
        for (int i = 0; i < n_freq; ++i)
            if (!(freqs[i] > 0.0)) throw ApiError(NCPA_EINVAL, "frequencies must be positive");
        CK(cudaSetDevice(ctx->device));
        std::vector<Group> groups{make_group(prof, prm, prm->nz_grid, freqs, n_freq, az_deg, n_az)};
        auto M = std::make_unique<ncpa_modes>();
        init_modes(M.get(), ctx, prm, n_freq * n_az);
        M->nf = n_freq;
        M->na = n_az;
        M->freqs.assign(freqs, freqs + n_freq);
        M->az.assign(az_deg, az_deg + n_az);
        if (prm->method == NCPA_METHOD_WMOD) solve_wmod(ctx, M.get(), prm, groups);
        else solve_groups(ctx, M.get(), prm, groups);
        *out = M.release();
        return NCPA_OK;
    });
}

ncpa_status ncpa_ess_solve_jobs(ncpa_ctx* ctx, const ncpa_ess_job* jobs, int n_jobs, const ncpa_ess_params* prm,
                                ncpa_modes** out) {
    if (!ctx || !jobs || n_jobs < 1 || !prm || !out) return NCPA_EINVAL;
    *out = nullptr;
    return guarded(ctx, [&]() -> ncpa_status {
        check_ess_params(prm);
        int P = 0;
        std::vector<Group> groups;
        groups.reserve(n_jobs);
        for (int j = 0; j < n_jobs; ++j) {
            const ncpa_ess_job& jb = jobs[j];
            if (!jb.profile || !jb.freqs || jb.n_freq < 1) throw ApiError(NCPA_EINVAL, "job without profile or frequencies");
            for (int i = 0; i < jb.n_freq; ++i)
                if (!(jb.freqs[i] > 0.0)) throw ApiError(NCPA_EINVAL, "frequencies must be positive");
            if (jb.profile->ctx != ctx) throw ApiError(NCPA_EINVAL, "profile belongs to another context");
            if (jb.n_az < 0 || (jb.n_az > 0 && !jb.az_list)) throw ApiError(NCPA_EINVAL, "job azimuth list missing");
            if (jb.nz_grid != 0 && jb.nz_grid < 10) throw ApiError(NCPA_EINVAL, "Nz_grid must be >= 10");
            const int n_az = jb.n_az > 0 ? jb.n_az : 1;
            groups.push_back(make_group(jb.profile, prm, jb.nz_grid > 0 ? jb.nz_grid : prm->nz_grid, jb.freqs,
                                        jb.n_freq, jb.n_az > 0 ? jb.az_list : &jb.az_deg, n_az));
            P += jb.n_freq * n_az;
        }
        CK(cudaSetDevice(ctx->device));
        auto M = std::make_unique<ncpa_modes>();
        init_modes(M.get(), ctx, prm, P);
        M->nf = P;
        M->na = 1;
        M->multi_job = true;
        for (const Group& g : groups)
            for (int f = 0; f < g.n_freq; ++f)
                for (int a = 0; a < g.n_az; ++a) M->freqs.push_back(g.freqs[f]);
        M->az.assign(1, groups[0].az[0]);
        if (prm->method == NCPA_METHOD_WMOD) solve_wmod(ctx, M.get(), prm, groups);
        else solve_groups(ctx, M.get(), prm, groups);
        *out = M.release();
        return NCPA_OK;
    });
}

ncpa_status ncpa_modes_destroy(ncpa_modes* m) {
    if (!m) return NCPA_EINVAL;
    if (m->plan_owned) return fail(m->ctx, NCPA_EINVAL, "these modes belong to a plan; destroy the plan");
    cudaSetDevice(m->ctx->device);
    cudaStreamSynchronize(m->ctx->stream);
    delete m;
    return NCPA_OK;
}

ncpa_status ncpa_modes_problems(const ncpa_modes* m, int* n) {
    if (!m || !n) return NCPA_EINVAL;
    *n = m->P;
    return NCPA_OK;
}

ncpa_status ncpa_modes_count(const ncpa_modes* m, int problem, int* n) {
    if (!m || !n || problem < 0 || problem >= m->P) return NCPA_EINVAL;
    *n = m->info[problem].M;
    return NCPA_OK;
}

ncpa_status ncpa_modes_info(const ncpa_modes* m, int problem, double* freq, double* az, double* dz, double* k_min,
                            double* k_max, double* rho_src, double* rho_rcv) {
    if (!m || problem < 0 || problem >= m->P) return NCPA_EINVAL;
    const ProblemInfo& pi = m->info[problem];
    if (freq) *freq = pi.freq;
    if (az) *az = pi.az;
    if (dz) *dz = pi.dz;
    if (k_min) *k_min = pi.k_min;
    if (k_max) *k_max = pi.k_max;
    if (rho_src) *rho_src = m->rho_src_p[problem];
    if (rho_rcv) *rho_rcv = m->rho_rcv_p[problem];
    return NCPA_OK;
}

ncpa_status ncpa_modes_get(const ncpa_modes* m, int problem, double* re_k, double* im_k, double* v_src,
                           double* v_rcv, double* v_group) {
    if (!m || problem < 0 || problem >= m->P) return NCPA_EINVAL;
    if (!m->host_valid) {
        ncpa_status s = guarded(m->ctx, [&]() -> ncpa_status {
            fetch_modes(m);
            CK(cudaStreamSynchronize(m->ctx->stream));
            return NCPA_OK;
        });
        if (s != NCPA_OK) return s;
    }
    const ProblemInfo& pi = m->info[problem];
    const size_t o = pi.off, n = pi.M;
    if (re_k) std::memcpy(re_k, m->kr.data() + o, n * 8);
    if (im_k) std::memcpy(im_k, m->ki.data() + o, n * 8);
    if (v_src) std::memcpy(v_src, m->vs.data() + o, n * 8);
    if (v_rcv) std::memcpy(v_rcv, m->vr.data() + o, n * 8);
    if (v_group) std::memcpy(v_group, m->vg.data() + o, n * 8);
    return NCPA_OK;
}

ncpa_status ncpa_modes_get_all(const ncpa_modes* m, int* mode_off, double* re_k, double* im_k, double* v_src,
                               double* v_rcv, double* v_group) {
    if (!m || !mode_off) return NCPA_EINVAL;
    for (int p = 0; p < m->P; ++p) mode_off[p] = m->info[p].off;
    mode_off[m->P] = m->Mtot;
    if (!re_k && !im_k && !v_src && !v_rcv && !v_group) return NCPA_OK;
    return guarded(m->ctx, [&]() -> ncpa_status {
        cudaStream_t st = m->ctx->stream;
        const size_t n = (size_t)m->Mtot * 8;
        if (n) {
            const std::pair<double*, const DevBuf*> cols[] = {
                {re_k, &m->d_kr}, {im_k, &m->d_ki}, {v_src, &m->d_vs}, {v_rcv, &m->d_vr}, {v_group, &m->d_vg}};
            for (const auto& c : cols)
                if (c.first) CK(cudaMemcpyAsync(c.first, c.second->p, n, cudaMemcpyDeviceToHost, st));
        }
        CK(cudaStreamSynchronize(st));
        return NCPA_OK;
    });
}

ncpa_status ncpa_modes_get_vectors(const ncpa_modes* m, int problem, double* v) {
    if (!m || !v || problem < 0 || problem >= m->P) return NCPA_EINVAL;
    if (!m->prm.want_vectors) return fail(m->ctx, NCPA_EINVAL, "solve was run without want_vectors");
    return guarded(m->ctx, [&]() -> ncpa_status {
        const size_t n = (size_t)m->info[problem].M * m->info[problem].nz;
        if (n) {
            CK(cudaMemcpyAsync(v, m->d_vfull.as<double>() + m->vfull_off[problem], n * 8, cudaMemcpyDeviceToHost,
                               m->ctx->stream));
            CK(cudaStreamSynchronize(m->ctx->stream));
        }
        return NCPA_OK;
    });
}

// ---------------------------------------------------------------------------
// transmission loss
// ---------------------------------------------------------------------------
ncpa_status ncpa_tl_1d(ncpa_ctx* ctx, const ncpa_modes* m, const ncpa_tl_params* tp, double* re, double* im,
                       double* incoh) {
    if (!ctx || !m || !tp) return NCPA_EINVAL;
    const bool keep = !re && !im && !incoh;
    if (!keep && (!re || !im || !incoh)) return NCPA_EINVAL;
    if (keep && m->plan_owned) return fail(ctx, NCPA_EINVAL, "TL of a plan's modes needs host buffers");
    return guarded(ctx, [&]() -> ncpa_status {
        if (tp->n_ranges < 1 || !(tp->dr_m > 0)) throw ApiError(NCPA_EINVAL, "bad range grid");
        CK(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        const size_t n = (size_t)m->P * tp->n_ranges;
        DevBuf tre, tim, tinc;  // a plan's TL buffers are written by its graph: never reallocated here
        DevBuf& dre = m->plan_owned ? tre : m->tl_re;
        DevBuf& dim = m->plan_owned ? tim : m->tl_im;
        DevBuf& dinc = m->plan_owned ? tinc : m->tl_inc;
        dre.alloc(n * 8, st);
        dim.alloc(n * 8, st);
        dinc.alloc(n * 8, st);
        check_launch(ctx, ncpa::launch_tl1d(st, m->P, m->d_pinfo.as<ProblemInfo>(), m->d_kr.as<double>(),
                                            m->d_ki.as<double>(), m->d_vs.as<double>(), m->d_vr.as<double>(),
                                            tp->n_ranges, tp->dr_m, tp->lossless, dre.as<double>(), dim.as<double>(),
                                            dinc.as<double>()));
        if (!keep) {
            CK(cudaMemcpyAsync(re, dre.p, n * 8, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(im, dim.p, n * 8, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(incoh, dinc.p, n * 8, cudaMemcpyDeviceToHost, st));
        }
        CK(cudaStreamSynchronize(st));
        return NCPA_OK;
    });
}

ncpa_status ncpa_tl_1d_range(ncpa_ctx* ctx, const ncpa_modes* m, int first, int count, const ncpa_tl_params* tp,
                             double* re, double* im, double* incoh) {
    if (!ctx || !m || !tp || !re || !im || !incoh || first < 0 || count < 1 || first + count > m->P)
        return NCPA_EINVAL;
    return guarded(ctx, [&]() -> ncpa_status {
        if (tp->n_ranges < 1 || !(tp->dr_m > 0)) throw ApiError(NCPA_EINVAL, "bad range grid");
        CK(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        const size_t n = (size_t)count * tp->n_ranges;
        DevBuf dre, dim, dinc;
        dre.alloc(n * 8, st);
        dim.alloc(n * 8, st);
        dinc.alloc(n * 8, st);
        // the problem records carry absolute mode offsets: start at `first`
        check_launch(ctx, ncpa::launch_tl1d(st, count, m->d_pinfo.as<ProblemInfo>() + first, m->d_kr.as<double>(),
                                            m->d_ki.as<double>(), m->d_vs.as<double>(), m->d_vr.as<double>(),
                                            tp->n_ranges, tp->dr_m, tp->lossless, dre.as<double>(), dim.as<double>(),
                                            dinc.as<double>()));
        CK(cudaMemcpyAsync(re, dre.p, n * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(im, dim.p, n * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(incoh, dinc.p, n * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return NCPA_OK;
    });
}

ncpa_status ncpa_modes_from_host(ncpa_ctx* ctx, int n_problems, const int* mode_off, const double* re_k,
                                 const double* im_k, const double* v_src, const double* v_rcv, ncpa_modes** out) {
    if (!ctx || !out || n_problems < 1 || !mode_off) return NCPA_EINVAL;
    *out = nullptr;
    if (mode_off[0] != 0) return fail(ctx, NCPA_EINVAL, "mode offsets must start at 0");
    for (int p = 0; p < n_problems; ++p)
        if (mode_off[p + 1] < mode_off[p]) return fail(ctx, NCPA_EINVAL, "mode offsets must not decrease");
    const int Mtot = mode_off[n_problems];
    if (Mtot > 0 && (!re_k || !im_k || !v_src || !v_rcv)) return NCPA_EINVAL;
    auto m = std::make_unique<ncpa_modes>();
    m->ctx = ctx;
    ncpa_status s = guarded(ctx, [&]() -> ncpa_status {
        CK(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        m->P = n_problems;
        m->nf = n_problems;
        m->na = 1;
        ncpa_ess_params_default(&m->prm);
        m->Mtot = Mtot;
        m->info.assign(n_problems, ProblemInfo{});
        for (int p = 0; p < n_problems; ++p) {
            m->info[p].off = mode_off[p];
            m->info[p].M = mode_off[p + 1] - mode_off[p];
        }
        m->rho_src_p.assign(n_problems, 1.0);
        m->rho_rcv_p.assign(n_problems, 1.0);
        m->kr.assign(re_k, re_k + Mtot);
        m->ki.assign(im_k, im_k + Mtot);
        m->vs.assign(v_src, v_src + Mtot);
        m->vr.assign(v_rcv, v_rcv + Mtot);
        m->vg.assign(Mtot, 0.0);
        m->host_valid = true;
        upload(m->d_pinfo, m->info, st);
        upload(m->d_kr, m->kr, st);
        upload(m->d_ki, m->ki, st);
        upload(m->d_vs, m->vs, st);
        upload(m->d_vr, m->vr, st);
        upload(m->d_vg, m->vg, st);
        CK(cudaStreamSynchronize(st));
        return NCPA_OK;
    });
    if (s != NCPA_OK) return s;
    *out = m.release();
    return NCPA_OK;
}

ncpa_status ncpa_tl_2d_heights(const ncpa_modes* m, int problem, int* n_heights) {
    if (!m || !n_heights || problem < 0 || problem >= m->P) return NCPA_EINVAL;
    const int nz = m->info[problem].nz;
    int stepj = nz / 500;
    if (stepj == 0) stepj = 10;
    *n_heights = (nz + stepj - 1) / stepj;
    return NCPA_OK;
}

namespace {

// The modal sum at grid rows idx (receiver-major [idx.size() x n_ranges]
// into ctx->ms_re / ms_im) by `method`; shared by ncpa_tl_multi and the
// tensor-core form of ncpa_tl_2d.
void modal_sum_rows(ncpa_ctx* ctx, const ncpa_modes* m, int problem, const std::vector<int>& idx,
                    const ncpa_tl_params* tp, int method) {
    cudaStream_t st = ctx->stream;
    PhaseTimer tm(ctx);
    tm.mark("start");
    const ProblemInfo& pi = m->info[problem];
    const int M = pi.M, nr = tp->n_ranges;
    const int n_rcv = (int)idx.size();
    const size_t nout = (size_t)n_rcv * nr;
    ctx->ms_re.alloc(nout * 8, st);
    ctx->ms_im.alloc(nout * 8, st);
    if (M == 0) {
        CK(cudaMemsetAsync(ctx->ms_re.p, 0, nout * 8, st));
        CK(cudaMemsetAsync(ctx->ms_im.p, 0, nout * 8, st));
    } else {
        // receiver indices through pinned memory: no host synchronisation
        int* hidx = reinterpret_cast<int*>(pinned(ctx, (size_t)(n_rcv + 1) / 2));
        std::memcpy(hidx, idx.data(), (size_t)n_rcv * 4);
        ctx->ms_idx.alloc((size_t)n_rcv * 4, st);
        CK(cudaMemcpyAsync(ctx->ms_idx.p, hidx, (size_t)n_rcv * 4, cudaMemcpyHostToDevice, st));
        const double* vfull = m->d_vfull.as<double>() + m->vfull_off[problem];
        const double* kr = m->d_kr.as<double>() + pi.off;
        const double* ki = m->d_ki.as<double>() + pi.off;
        const double* vs = m->d_vs.as<double>() + pi.off;
        if (method == NCPA_SUM_FP64) {
            ctx->ms_vz.alloc((size_t)n_rcv * M * 8, st);
            check_launch(ctx, ncpa::launch_ms_gather(st, n_rcv, M, ctx->ms_idx.as<int>(), vfull,
                                                     ctx->ms_vz.as<double>()));
            tm.mark("ms-prep");
            check_launch(ctx, ncpa::launch_tl2d_rcv_major(st, M, kr, ki, vs, ctx->ms_vz.as<double>(), n_rcv, nr,
                                                          tp->dr_m, tp->lossless, ctx->ms_re.as<double>(),
                                                          ctx->ms_im.as<double>()));
            tm.mark("ms-fp64");
        } else {
            const ncpa::MsPlan pl = ncpa::ms_plan(n_rcv, M, nr, ctx->num_sms);
            ctx->ms_img.alloc(pl.a_img_bytes, st);
            ctx->ms_q.alloc(pl.q_bytes, st);
            ctx->ms_tab.alloc(pl.tab_bytes, st);
            ctx->ms_raw.alloc(pl.raw_bytes, st);
            const bool guard = method == NCPA_SUM_TC_GUARDED;
            const int fmt = method == NCPA_SUM_TC_TF32 ? 1 : (guard ? 2 : 0);
            if (guard) {
                ctx->ms_spart.alloc(pl.s_part_bytes, st);
                ctx->ms_b64.alloc(pl.b64_bytes, st);
                ctx->ms_tp64.alloc(pl.tp64_bytes, st);
                ctx->ms_a64.alloc(pl.a64_bytes, st);
                ctx->ms_fix.alloc(pl.fix_list_bytes, st);
                ctx->ms_fixcnt.alloc(sizeof(int), st);
                CK(cudaMemsetAsync(ctx->ms_fixcnt.p, 0, sizeof(int), st));
                ctx->ms_last_points = (long long)n_rcv * nr;
                ctx->ms_last_eps = ncpa::ms_guard_eps(pl);
                ctx->ms_last_tau = ncpa::ms_guard_tau(pl);
            }
            check_launch(ctx, ncpa::launch_ms_prepare(st, pl, fmt, n_rcv, M, kr, ki, vs, ctx->ms_idx.as<int>(),
                                                      vfull, tp->dr_m, tp->lossless, ctx->ms_img.p, ctx->ms_q.p,
                                                      ctx->ms_tab.p, guard ? ctx->ms_b64.p : nullptr,
                                                      guard ? ctx->ms_tp64.p : nullptr,
                                                      guard ? ctx->ms_a64.p : nullptr));
            tm.mark("ms-prep");
            auto tc = [&](int variant) {
                check_launch(ctx, ncpa::launch_ms_tc(st, pl, fmt, nr, ctx->ms_img.p, ctx->ms_q.p, ctx->ms_tab.p,
                                                     ctx->ms_raw.as<float>(),
                                                     guard ? ctx->ms_spart.as<float>() : nullptr,
                                                     ctx->d_err.as<unsigned>(), variant));
            };
            // schedule: the fastest ring depths for this shape, timed
            // once per context (each variant computes the same sums)
            int variant = 0;
            if (ctx->ms_tune) {
                const std::array<long long, 4> key{fmt, pl.groups, pl.n_chunks, pl.n_tiles};
                auto it = ctx->ms_choice.find(key);
                if (it == ctx->ms_choice.end()) {
                    const int nv = ncpa::ms_tc_variants();
                    std::vector<double> best_ms(nv, 0.0);
                    cudaEvent_t e0, e1;
                    CK(cudaEventCreate(&e0));
                    CK(cudaEventCreate(&e1));
                    int best = 0;
                    for (int v = 0; v < nv; ++v) {
                        tc(v);  // warm-up (function attributes, caches)
                        CK(cudaEventRecord(e0, st));
                        for (int r = 0; r < 3; ++r) tc(v);
                        CK(cudaEventRecord(e1, st));
                        CK(cudaEventSynchronize(e1));
                        float ms = 0.f;
                        CK(cudaEventElapsedTime(&ms, e0, e1));
                        best_ms[v] = ms / 3.0;
                        if (best_ms[v] < best_ms[best]) best = v;
                    }
                    cudaEventDestroy(e0);
                    cudaEventDestroy(e1);
                    it = ctx->ms_choice.emplace(key, best).first;
                    ctx->ms_last_times = best_ms;
                }
                variant = it->second;
            }
            ctx->ms_last_variant = variant;
            ctx->ms_last_fmt = fmt;
            tc(variant);
            tm.mark("ms-tc");
            check_launch(ctx, ncpa::launch_ms_finish(st, pl, n_rcv, nr, tp->dr_m, ctx->ms_raw.as<float>(),
                                                     ctx->ms_re.as<double>(), ctx->ms_im.as<double>(),
                                                     guard ? ctx->ms_spart.as<float>() : nullptr,
                                                     guard ? ctx->ms_fixcnt.as<int>() : nullptr,
                                                     guard ? ctx->ms_fix.p : nullptr));
            tm.mark("ms-finish");
            if (guard) {
                check_launch(ctx, ncpa::launch_ms_fix(st, ctx->num_sms, M, pl.M_pad, nr, tp->dr_m,
                                                      ctx->ms_fixcnt.as<int>(), ctx->ms_fix.p, ctx->ms_a64.p,
                                                      ctx->ms_tp64.p, ctx->ms_b64.p, ctx->ms_re.as<double>(),
                                                      ctx->ms_im.as<double>()));
                tm.mark("ms-fix");
            }
        }
    }
}

}  // namespace

ncpa_status ncpa_tl_2d(ncpa_ctx* ctx, const ncpa_modes* m, int problem, const ncpa_tl_params* tp, double* z_out,
                       double* re, double* im) {
    if (!ctx || !m || !tp || !re || !im || problem < 0 || problem >= m->P) return NCPA_EINVAL;
    if (!m->prm.want_vectors) return fail(ctx, NCPA_EINVAL, "2-D TL needs a solve with want_vectors");
    return guarded(ctx, [&]() -> ncpa_status {
        CK(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        const ProblemInfo& pi = m->info[problem];
        const int Mm = pi.M, nz = pi.nz;
        int stepj = nz / 500;
        if (stepj == 0) stepj = 10;
        const int nzo = (nz + stepj - 1) / stepj;
        if (nzo > 1024) throw ApiError(NCPA_EINVAL, "too many output heights");
        if (ctx->tl2d_method == NCPA_SUM_TC_GUARDED) {
            // the guarded tensor-core sum at the sampled rows (receiver-major),
            // written out range-major as the FP64 kernel does
            std::vector<int> idx(nzo);
            for (int j = 0; j < nzo; ++j) {
                idx[j] = j * stepj;
                if (z_out) z_out[j] = (j * stepj) * pi.dz;
            }
            const int nr = tp->n_ranges;
            modal_sum_rows(ctx, m, problem, idx, tp, NCPA_SUM_TC_GUARDED);
            const size_t n = (size_t)nzo * nr;
            DevBuf tre, tim;
            tre.alloc(n * 8, st);
            tim.alloc(n * 8, st);
            check_launch(ctx, ncpa::launch_transpose(st, nzo, nr, ctx->ms_re.as<double>(), tre.as<double>()));
            check_launch(ctx, ncpa::launch_transpose(st, nzo, nr, ctx->ms_im.as<double>(), tim.as<double>()));
            CK(cudaMemcpyAsync(re, tre.p, n * 8, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(im, tim.p, n * 8, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            check_device_status(ctx);
            return NCPA_OK;
        }
        // rows of the sampled heights and the source row (last), gathered on
        // the device: the full vectors never leave HBM
        std::vector<int> rows(nzo + 1);
        for (int j = 0; j < nzo; ++j) {
            rows[j] = j * stepj;
            if (z_out) z_out[j] = (j * stepj) * pi.dz;
        }
        rows[nzo] = pi.isrc;
        DevBuf drows, dvz, dre, dim;
        upload(drows, rows, st);
        dvz.alloc((size_t)(nzo + 1) * std::max(Mm, 1) * 8, st);
        check_launch(ctx, ncpa::launch_ms_gather(st, nzo + 1, Mm, drows.as<int>(),
                                                 m->d_vfull.as<double>() + m->vfull_off[problem], dvz.as<double>()));
        const size_t n = (size_t)tp->n_ranges * nzo;
        dre.alloc(n * 8, st);
        dim.alloc(n * 8, st);
        check_launch(ctx, ncpa::launch_tl2d(st, Mm, m->d_kr.as<double>() + pi.off, m->d_ki.as<double>() + pi.off,
                                            dvz.as<double>() + (size_t)nzo * Mm, dvz.as<double>(), nzo, tp->n_ranges,
                                            tp->dr_m, tp->lossless, dre.as<double>(), dim.as<double>()));
        CK(cudaMemcpyAsync(re, dre.p, n * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(im, dim.p, n * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return NCPA_OK;
    });
}


ncpa_status ncpa_tl_multi(ncpa_ctx* ctx, const ncpa_modes* m, int problem, int n_rcv, const double* rcv_height_m,
                          const ncpa_tl_params* tp, int method, double* re, double* im) {
    if (!ctx || !m || !tp || !rcv_height_m || n_rcv < 1 || problem < 0 || problem >= m->P) return NCPA_EINVAL;
    if ((re == nullptr) != (im == nullptr)) return NCPA_EINVAL;
    if (method != NCPA_SUM_FP64 && method != NCPA_SUM_TC_BF16X3 && method != NCPA_SUM_TC_TF32 &&
        method != NCPA_SUM_TC_GUARDED)
        return NCPA_EINVAL;
    if (!m->prm.want_vectors) return fail(ctx, NCPA_EINVAL, "the modal sum at receivers needs want_vectors");
    return guarded(ctx, [&]() -> ncpa_status {
        if (tp->n_ranges < 1 || !(tp->dr_m > 0)) throw ApiError(NCPA_EINVAL, "bad range grid");
        if (method == NCPA_SUM_FP64 && n_rcv > 1024) throw ApiError(NCPA_EINVAL, "FP64 sum: at most 1024 receivers");
        CK(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        const ProblemInfo& pi = m->info[problem];
        const int nr = tp->n_ranges;
        // receiver grid points: ceil(z / dz) as ModeSolver.cpp:301 does
        std::vector<int> idx(n_rcv);
        for (int j = 0; j < n_rcv; ++j) {
            const int k = (int)std::ceil(rcv_height_m[j] / pi.dz);
            if (k < 0 || k >= pi.nz) throw ApiError(NCPA_EINVAL, "receiver height outside the grid");
            idx[j] = k;
        }
        const size_t nout = (size_t)n_rcv * nr;
        modal_sum_rows(ctx, m, problem, idx, tp, method);
        if (re) {
            CK(cudaMemcpyAsync(re, ctx->ms_re.p, nout * 8, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(im, ctx->ms_im.p, nout * 8, cudaMemcpyDeviceToHost, st));
        }
        check_device_status(ctx);
        return NCPA_OK;
    });
}

// ---------------------------------------------------------------------------
// broadband synthesis
// ---------------------------------------------------------------------------
namespace {
ncpa_status bb_common(ncpa_ctx* ctx, int nfreq, const double* d_f, const int* d_off, int n_modes, const double* d_rk,
                      const double* d_ik, const double* d_vs, const double* d_vr, double rho_ratio,
                      const ncpa_bb_params* bp, double* waveforms) {
    cudaStream_t st = ctx->stream;
    if (bp->n_ranges < 1 || !bp->ranges_m || bp->nfft < nfreq || !(bp->max_celerity > 0) || !bp->src_re ||
        !bp->src_im)
        throw ApiError(NCPA_EINVAL, "bad broadband parameters (need nfft >= n_freq, ranges, source spectrum)");
    const int nr = bp->n_ranges, nfft = bp->nfft;
    std::vector<double> t0(nr), src(2 * (size_t)nfreq);
    for (int i = 0; i < nr; ++i) t0[i] = 0.0 + bp->ranges_m[i] / bp->max_celerity;
    for (int i = 0; i < nfreq; ++i) {
        src[2 * i] = bp->src_re[i];
        src[2 * i + 1] = bp->src_im[i];
    }
    DevBuf dr, dt0, dsrc, dh, dfac;
    DevBuf& dout = ctx->bb_out;
    dfac.alloc((size_t)std::max(n_modes, 1) * 4 * 8, st);
    upload(dr, bp->ranges_m, nr, st);
    upload(dt0, t0, st);
    upload(dsrc, src, st);
    dh.alloc((size_t)nr * nfreq * 16, st);
    dout.alloc((size_t)nr * nfft * 8, st);
    const double* tw = twiddle(ctx, nfft);
    check_launch(ctx, ncpa::launch_bb_transfer(st, nfreq, d_off, d_rk, d_ik, d_vs, d_vr, rho_ratio, nr,
                                               dr.as<double>(), bp->zero_attn, n_modes, dfac.as<double>(),
                                               dh.as<double>()));
    check_launch(ctx, ncpa::launch_bb_pulse(st, nfreq, d_f, dsrc.as<double>(), dh.as<double>(), nr, dt0.as<double>(),
                                            nfft, tw, dout.as<double>()));
    if (waveforms) CK(cudaMemcpyAsync(waveforms, dout.p, (size_t)nr * nfft * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return NCPA_OK;
}
}  // namespace

ncpa_status ncpa_bb_synthesize(ncpa_ctx* ctx, const ncpa_dispersion_desc* d, const ncpa_bb_params* bp,
                               double* waveforms) {
    if (!ctx || !d || !bp) return NCPA_EINVAL;
    return guarded(ctx, [&]() -> ncpa_status {
        if (d->n_freq < 3 || !d->f || !d->mode_off) throw ApiError(NCPA_EINVAL, "dispersion needs >= 2 frequencies");
        CK(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        const int nf = d->n_freq;
        const int mt = d->mode_off[nf];
        DevBuf df, doff, drk, dik, dvs, dvr;
        upload(df, d->f, nf, st);
        upload(doff, d->mode_off, nf + 1, st);
        upload(drk, d->re_k, std::max(mt, 1), st);
        upload(dik, d->im_k, std::max(mt, 1), st);
        upload(dvs, d->v_src, std::max(mt, 1), st);
        upload(dvr, d->v_rcv, std::max(mt, 1), st);
        return bb_common(ctx, nf, df.as<double>(), doff.as<int>(), mt, drk.as<double>(), dik.as<double>(),
                         dvs.as<double>(), dvr.as<double>(), d->rho_rcv / d->rho_src, bp, waveforms);
    });
}

ncpa_status ncpa_bb_synthesize_modes(ncpa_ctx* ctx, const ncpa_modes* m, int az_index, const ncpa_bb_params* bp,
                                     double* waveforms) {
    if (!ctx || !m || !bp || az_index < 0 || az_index >= m->na) return NCPA_EINVAL;
    return guarded(ctx, [&]() -> ncpa_status {
        if (m->na != 1 || m->multi_job)
            throw ApiError(NCPA_EINVAL, "device-resident synthesis needs a single-azimuth, single-profile solve");
        CK(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        const int nf = m->nf + 1;  // DC slot first
        std::vector<double> f(nf);
        std::vector<int> off(nf + 1);
        f[0] = 0.0;
        off[0] = 0;
        off[1] = 0;
        for (int i = 0; i < m->nf; ++i) {
            f[i + 1] = m->freqs[i];
            off[i + 2] = m->info[i].off + m->info[i].M;
        }
        DevBuf df, doff;
        upload(df, f, st);
        upload(doff, off, st);
        return bb_common(ctx, nf, df.as<double>(), doff.as<int>(), m->Mtot, m->d_kr.as<double>(),
                         m->d_ki.as<double>(), m->d_vs.as<double>(), m->d_vr.as<double>(), m->rho_rcv_p[0] / m->rho_src_p[0],
                         bp, waveforms);
    });
}

ncpa_status ncpa_modal_starter(ncpa_ctx* ctx, const ncpa_modes* m, int problem, int* n_out, double* z_km,
                               double* re, double* im) {
    if (!ctx || !m || !n_out || problem < 0 || problem >= m->P) return NCPA_EINVAL;
    if (!m->prm.want_vectors) return fail(ctx, NCPA_EINVAL, "the modal starter needs a solve with want_vectors");
    return guarded(ctx, [&]() -> ncpa_status {
        const ProblemInfo& pi = m->info[problem];
        const double freq = pi.freq;
        int step = (int)((340.0 / freq) / 10 / pi.dz);  // ESSModeSolver.cpp:692-693
        if (step < 1) step = 1;
        const int nout = (pi.nz + step - 1) / step;
        if (!z_km || !re || !im) {
            *n_out = nout;
            return NCPA_OK;
        }
        if (*n_out < nout) throw ApiError(NCPA_EINVAL, "output arrays too short for the modal starter");
        CK(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        DevBuf dout;
        dout.alloc((size_t)nout * 8, st);
        const double k0 = 2 * kPi * freq / 340.0;
        check_launch(ctx, ncpa::launch_starter(st, pi.M, pi.nz, step, pi.isrc,
                                               m->d_vfull.as<double>() + m->vfull_off[problem],
                                               m->d_kr.as<double>() + pi.off, k0, dout.as<double>()));
        CK(cudaMemcpyAsync(re, dout.p, nout * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (int j = 0; j < nout; ++j) {
            z_km[j] = (j * step) * pi.dz / 1000.0;
            im[j] = 0.0;
        }
        *n_out = nout;
        return NCPA_OK;
    });
}

ncpa_status ncpa_source_waveform(ncpa_ctx* ctx, const double* f, int nfreq, const double* s_re, const double* s_im,
                                 int nfft, double* out) {
    if (!ctx || !f || !s_re || !s_im || !out || nfreq < 3 || nfft < nfreq) return NCPA_EINVAL;
    return guarded(ctx, [&]() -> ncpa_status {
        CK(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        std::vector<double> src(2 * (size_t)nfreq), t0(1, 0.0);
        for (int i = 0; i < nfreq; ++i) {
            src[2 * i] = s_re[i];
            src[2 * i + 1] = s_im[i];
        }
        DevBuf df, dsrc, dh, dt0, dout;
        upload(df, f, nfreq, st);
        upload(dsrc, src, st);
        upload(dt0, t0, st);
        dh.alloc((size_t)nfreq * 16, st);
        dout.alloc((size_t)nfft * 8, st);
        check_launch(ctx, ncpa::launch_fill_unit(st, nfreq, dh.as<double>()));
        const double* tw = twiddle(ctx, nfft);
        check_launch(ctx, ncpa::launch_bb_pulse(st, nfreq, df.as<double>(), dsrc.as<double>(), dh.as<double>(), 1,
                                                dt0.as<double>(), nfft, tw, dout.as<double>()));
        CK(cudaMemcpyAsync(out, dout.p, (size_t)nfft * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return NCPA_OK;
    });
}

ncpa_status ncpa_source_spectrum_builtin(ncpa_ctx* ctx, int kind, const double* f, int nfreq, double f_center,
                                         int nfft, double* s_re, double* s_im) {
    if (!ctx || !f || !s_re || !s_im || nfreq < 3 || kind < 0 || kind > 2) return NCPA_EINVAL;
    return guarded(ctx, [&]() -> ncpa_status {
        CK(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        const double fmax = f[nfreq - 1];
        double scale = 0.0;
        if (kind >= 1) {  // BroadbandPropagator.cpp:268-283
            double fc = f_center < 0.0 ? fmax / 5.0 : f_center;
            if (!(fc > 0 && fc <= fmax / 5.0 + 1.0E-16))
                throw ApiError(NCPA_EINVAL, "f_center is too large: the built-in pulse needs f_center <= f_max/5");
            scale = 1.0 / fc;
        }
        DevBuf df, ds;
        upload(df, f, nfreq, st);
        ds.alloc((size_t)2 * nfreq * 8, st);
        if (kind <= 1) {
            check_launch(ctx, ncpa::launch_src_builtin(st, kind, nfreq, df.as<double>(), scale, ds.as<double>()));
        } else {  // pulse2: transform of the sampled power-law pulse, dt = 1/(nfft df)
            if (nfft < nfreq) throw ApiError(NCPA_EINVAL, "nfft must be >= the number of frequencies");
            const double dt = 1.0 / ((double)nfft * (f[2] - f[1]));
            DevBuf dx;
            dx.alloc((size_t)nfft * 8, st);
            check_launch(ctx, ncpa::launch_src_pulse2(st, nfft, dt, scale, dx.as<double>()));
            const double* tw = twiddle(ctx, nfft);
            check_launch(ctx, ncpa::launch_src_dft(st, nfft, dx.as<double>(), dt, nfft, nfreq, tw, ds.as<double>()));
        }
        std::vector<double> h(2 * (size_t)nfreq);
        CK(cudaMemcpyAsync(h.data(), ds.p, h.size() * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (int k = 0; k < nfreq; ++k) {
            s_re[k] = h[2 * k];
            s_im[k] = h[2 * k + 1];
        }
        return NCPA_OK;
    });
}

ncpa_status ncpa_source_spectrum_waveform(ncpa_ctx* ctx, const double* x, int n, double dt, int nfft, int nfreq,
                                          double* s_re, double* s_im) {
    if (!ctx || !x || !s_re || !s_im || n < 1 || nfft < 1 || nfreq < 1) return NCPA_EINVAL;
    return guarded(ctx, [&]() -> ncpa_status {
        CK(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        DevBuf dx, ds;
        upload(dx, x, n, st);
        ds.alloc((size_t)2 * nfreq * 8, st);
        const double* tw = twiddle(ctx, nfft);
        check_launch(ctx, ncpa::launch_src_dft(st, n, dx.as<double>(), dt, nfft, nfreq, tw, ds.as<double>()));
        std::vector<double> h(2 * (size_t)nfreq);
        CK(cudaMemcpyAsync(h.data(), ds.p, h.size() * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (int k = 0; k < nfreq; ++k) {
            s_re[k] = h[2 * k];
            s_im[k] = h[2 * k + 1];
        }
        return NCPA_OK;
    });
}

// ---------------------------------------------------------------------------
// captured solves (plans)
// ---------------------------------------------------------------------------
ncpa_status ncpa_profile_update(ncpa_profile* prof, const ncpa_profile_desc* d) {
    if (!prof || !d) return NCPA_EINVAL;
    ncpa_ctx* ctx = prof->ctx;
    return guarded(ctx, [&]() -> ncpa_status {
        if (d->n_knots != prof->n) throw ApiError(NCPA_EINVAL, "profile update needs the same number of knots");
        if (!d->z || !d->u || !d->v || !d->t || !d->p || !d->rho)
            throw ApiError(NCPA_EINVAL, "profile arrays z, u, v, t, p, rho are required");
        if (d->z[0] != prof->z_lo || d->z[prof->n - 1] != prof->z_hi)
            throw ApiError(NCPA_EINVAL, "profile update needs the same altitude range");
        for (int i = 1; i < prof->n; ++i)
            if (!(d->z[i] > d->z[i - 1])) throw ApiError(NCPA_EINVAL, "profile altitudes must increase strictly");
        if (d->has_z0 != prof->has_z0 || (d->has_z0 && d->z0_m != prof->z0))
            throw ApiError(NCPA_EINVAL, "profile update needs the same ground height");
        if ((d->attn != nullptr) != prof->has_attn)
            throw ApiError(NCPA_EINVAL, "profile update needs an attenuation column exactly when the profile has one");
        CK(cudaSetDevice(ctx->device));
        fill_profile(ctx, prof, d);
        return NCPA_OK;
    });
}

}  // extern "C"

struct ncpa_plan {
    PlanData d;
    ~ncpa_plan() {
        if (d.ctx) {
            cudaSetDevice(d.ctx->device);
            cudaStreamSynchronize(d.ctx->stream);
        }
        if (d.exec) cudaGraphExecDestroy(d.exec);
        for (const Group& g : d.groups) const_cast<ncpa_profile*>(g.prof)->plan_refs--;
        if (d.h_info) cudaFreeHost(d.h_info);
        if (d.h_tot) cudaFreeHost(d.h_tot);
        if (d.h_err) cudaFreeHost(d.h_err);
        if (d.h_rho) cudaFreeHost(d.h_rho);
    }
};

extern "C" {

ncpa_status ncpa_ess_plan_create(ncpa_ctx* ctx, const ncpa_ess_job* jobs, int n_jobs, const ncpa_ess_params* prm,
                                 const ncpa_tl_params* tl, int tune, ncpa_plan** out) {
    if (!ctx || !jobs || n_jobs < 1 || !prm || !out) return NCPA_EINVAL;
    *out = nullptr;
    return guarded(ctx, [&]() -> ncpa_status {
        check_ess_params(prm);
        if (prm->method != NCPA_METHOD_ESS) throw ApiError(NCPA_EINVAL, "plans take the ESS method only");
        if (prm->want_vectors) throw ApiError(NCPA_EINVAL, "plans do not keep eigenvectors (want_vectors = 0)");
        if (prm->lamb_wave_bc) throw ApiError(NCPA_EINVAL, "plans do not take the Lamb-wave condition");
        if (tl && (tl->n_ranges < 1 || !(tl->dr_m > 0))) throw ApiError(NCPA_EINVAL, "bad range grid");
        CK(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        auto plan = std::make_unique<ncpa_plan>();
        PlanData& pl = plan->d;
        pl.prm = *prm;
        if (pl.prm.max_modes <= 0) pl.prm.max_modes = 4000;
        pl.freqs.reserve(n_jobs);
        pl.azs.reserve(n_jobs);
        int P = 0;
        for (int j = 0; j < n_jobs; ++j) {
            const ncpa_ess_job& jb = jobs[j];
            if (!jb.profile || !jb.freqs || jb.n_freq < 1) throw ApiError(NCPA_EINVAL, "job without profile or frequencies");
            for (int i = 0; i < jb.n_freq; ++i)
                if (!(jb.freqs[i] > 0.0)) throw ApiError(NCPA_EINVAL, "frequencies must be positive");
            if (jb.profile->ctx != ctx) throw ApiError(NCPA_EINVAL, "profile belongs to another context");
            if (jb.n_az < 0 || (jb.n_az > 0 && !jb.az_list)) throw ApiError(NCPA_EINVAL, "job azimuth list missing");
            if (jb.nz_grid != 0 && jb.nz_grid < 10) throw ApiError(NCPA_EINVAL, "Nz_grid must be >= 10");
            pl.freqs.emplace_back(jb.freqs, jb.freqs + jb.n_freq);
            if (jb.n_az > 0) pl.azs.emplace_back(jb.az_list, jb.az_list + jb.n_az);
            else pl.azs.emplace_back(1, jb.az_deg);
            const int n_az = (int)pl.azs.back().size();
            pl.groups.push_back(make_group(jb.profile, prm, jb.nz_grid > 0 ? jb.nz_grid : prm->nz_grid,
                                           pl.freqs.back().data(), jb.n_freq, pl.azs.back().data(), n_az));
            const_cast<ncpa_profile*>(jb.profile)->plan_refs++;  // released by ~ncpa_plan
            P += jb.n_freq * n_az;
        }
        pl.ctx = ctx;
        pl.M = std::make_unique<ncpa_modes>();
        ncpa_modes* M = pl.M.get();
        init_modes(M, ctx, &pl.prm, P);
        M->nf = P;
        M->na = 1;
        M->multi_job = true;
        M->plan_owned = true;
        for (const Group& g : pl.groups)
            for (int f = 0; f < g.n_freq; ++f)
                for (int a = 0; a < g.n_az; ++a) M->freqs.push_back(g.freqs[f]);
        M->az.assign(1, pl.groups[0].az[0]);
        long long s_tot = 0, w_tot = 0;
        layout_groups(M, pl.groups, s_tot, w_tot);
        upload(pl.pinfo_init, M->info, st);
        M->d_pinfo.alloc((size_t)P * sizeof(ProblemInfo), st);
        pl.wkb = wants_wkb(prm);
        pl.s.alloc((size_t)s_tot * 8, st);
        pl.w.alloc((size_t)w_tot * 8, st);
        if (pl.wkb) pl.kz2.alloc((size_t)s_tot * 8, st);
        if (prm->want_group_speed) pl.gs.alloc((size_t)s_tot * 8, st);
        CK(cudaHostAlloc((void**)&pl.h_info, (size_t)P * sizeof(ProblemInfo), cudaHostAllocDefault));
        CK(cudaHostAlloc((void**)&pl.h_tot, 4 * sizeof(int), cudaHostAllocDefault));
        CK(cudaHostAlloc((void**)&pl.h_err, sizeof(unsigned), cudaHostAllocDefault));
        CK(cudaHostAlloc((void**)&pl.h_rho, 2 * pl.groups.size() * sizeof(double), cudaHostAllocDefault));
        pl.gb.resize(pl.groups.size());
        for (size_t gi = 0; gi < pl.groups.size(); ++gi) prepare_group(ctx, prm, pl.groups[gi], pl.gb[gi]);
        const int kMinItem = 16;  // smallest bisection item the tuner tries
        double* gsp = prm->want_group_speed ? pl.gs.as<double>() : nullptr;
        pl.sb.own_ck = true;
        prepare_solve(ctx, M, &pl.prm, tune ? kMinItem : ncpa::kWItem, pl.sb, pl.s.as<double>(), pl.w.as<double>(),
                      gsp);
        if (tl) {
            pl.with_tl = true;
            pl.tp = *tl;
            const size_t n = (size_t)P * tl->n_ranges * 8;
            M->tl_re.alloc(n, st);
            M->tl_im.alloc(n, st);
            M->tl_inc.alloc(n, st);
        }
        ncpa::bisect_ctas_per_sm();  // sets the kernels' shared-memory attributes before any capture
        const int fit_e = ncpa::eigvec_ctas_per_sm(eigvec_args(ctx, M, &pl.prm, pl.s.as<double>(), pl.w.as<double>(),
                                                               gsp, pl.sb));
        pl.fit_e = fit_e;
        CK(cudaStreamSynchronize(st));
        char key[160];
        std::snprintf(key, sizeof key, "P%d s%lld w%lld nz%d m%d g%d t%d", P, s_tot, w_tot, M->nz_max,
                      pl.prm.max_modes, prm->want_group_speed ? 1 : 0, tl ? tl->n_ranges : 0);
        if (tune) {
            auto hit = ctx->tune_cache.find(key);
            if (hit != ctx->tune_cache.end()) {
                pl.tuning.bis_item = hit->second[0];
                pl.tuning.bis_ctas = hit->second[1];
                pl.tuning.ev_ctas = hit->second[2];
            } else {
                // coordinate search: item size, then bisection CTAs per SM, then
                // eigenvector CTAs per SM, each timed on its captured graph
                Tuning best;
                double best_ms = 1e300;
                auto consider = [&](const Tuning& t) {
                    cudaGraphExec_t e = capture_plan(pl, t);
                    double ms;
                    try {
                        ms = time_graph(pl, e, 2);
                    } catch (...) {
                        cudaGraphExecDestroy(e);
                        throw;
                    }
                    cudaGraphExecDestroy(e);
                    if (ms < best_ms) {
                        best_ms = ms;
                        best = t;
                    }
                };
                consider(Tuning{});
                for (int item : {24, kMinItem}) {
                    Tuning t = best;
                    t.bis_item = item;
                    consider(t);
                }
                const Tuning after_item = best;
                for (int c = 1; c < ncpa::bisect_ctas_per_sm(); ++c) {
                    Tuning t = after_item;
                    t.bis_ctas = c;
                    consider(t);
                }
                const Tuning after_bis = best;
                for (int c = 1; c < fit_e; ++c) {
                    Tuning t = after_bis;
                    t.ev_ctas = c;
                    consider(t);
                }
                pl.tuning = best;
                ctx->tune_cache[key] = {best.bis_item, best.bis_ctas, best.ev_ctas};
            }
        }
        pl.exec = capture_plan(pl, pl.tuning);
        if (tune) pl.tuned_ms = time_graph(pl, pl.exec, 3);
        *out = plan.release();
        return NCPA_OK;
    });
}

ncpa_status ncpa_ess_plan_run(ncpa_plan* plan) {
    if (!plan) return NCPA_EINVAL;
    PlanData& pl = plan->d;
    return guarded(pl.ctx, [&]() -> ncpa_status {
        CK(cudaSetDevice(pl.ctx->device));
        CK(cudaGraphLaunch(pl.exec, pl.ctx->stream));
        pl.ctx->launches += pl.kernels;
        finish_plan(pl);
        return NCPA_OK;
    });
}

ncpa_status ncpa_ess_plan_modes(ncpa_plan* plan, ncpa_modes** modes) {
    if (!plan || !modes) return NCPA_EINVAL;
    if (!plan->d.ran) return fail(plan->d.ctx, NCPA_EINVAL, "the plan has not run");
    *modes = plan->d.M.get();
    return NCPA_OK;
}

ncpa_status ncpa_ess_plan_tl(ncpa_plan* plan, double* re, double* im, double* incoh) {
    if (!plan || !re || !im || !incoh) return NCPA_EINVAL;
    PlanData& pl = plan->d;
    if (!pl.with_tl) return fail(pl.ctx, NCPA_EINVAL, "the plan has no TL range grid");
    if (!pl.ran) return fail(pl.ctx, NCPA_EINVAL, "the plan has not run");
    return guarded(pl.ctx, [&]() -> ncpa_status {
        cudaStream_t st = pl.ctx->stream;
        const size_t n = (size_t)pl.M->P * pl.tp.n_ranges * 8;
        CK(cudaMemcpyAsync(re, pl.M->tl_re.p, n, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(im, pl.M->tl_im.p, n, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(incoh, pl.M->tl_inc.p, n, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return NCPA_OK;
    });
}

ncpa_status ncpa_ess_plan_tuning(const ncpa_plan* plan, int* bis_item, int* bis_ctas_per_sm, int* ev_ctas_per_sm,
                                 double* ms) {
    if (!plan) return NCPA_EINVAL;
    const PlanData& pl = plan->d;
    if (bis_item) *bis_item = pl.tuning.bis_item;
    if (bis_ctas_per_sm) *bis_ctas_per_sm = pl.tuning.bis_ctas > 0 ? pl.tuning.bis_ctas : ncpa::bisect_ctas_per_sm();
    if (ev_ctas_per_sm) *ev_ctas_per_sm = pl.tuning.ev_ctas > 0 ? pl.tuning.ev_ctas : pl.fit_e;
    if (ms) *ms = pl.tuned_ms;
    return NCPA_OK;
}

ncpa_status ncpa_ess_plan_destroy(ncpa_plan* plan) {
    if (!plan) return NCPA_EINVAL;
    delete plan;
    return NCPA_OK;
}

}  // extern "C"
