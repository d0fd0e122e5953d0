// Serving loop over the C ABI (ncpa_server_* in ncpa_gpu.h).
//
// Requests (profile knots, frequencies, azimuth) are copied at submit and
// queued.  Each worker lane owns one library context (one device stream) and
// a host thread; a free lane takes the oldest queued request and every
// further queued request that fits the per-batch problem limit and the HBM
// budget, solves them in one ncpa_ess_solve_jobs call (requests whose
// profiles give different solver grids share the batch: every problem
// carries its own grid) plus one ncpa_tl_1d call, and hands each request its
// slice.  With two or more lanes, requests that arrive while a batch is
// on the device are admitted into the next batch on another lane, so their
// work overlaps on the GPU.  A batch that fails is re-run request by
// request so one bad request does not fail the others.
//
// Each request may carry its own 1-D TL range grid (a TL launch per run of
// requests with the same grid, over their slice of the batch) and ask for
// pulse waveforms (ModBB's synthesis on its own dispersion, built-in
// source spectrum).  With a cache budget, the modes of solved requests stay
// in HBM on a context of the cache, keyed by hashes of the profile's knot
// values and the exact frequencies and azimuth; a later request with the
// same key skips the eigen-solve and runs only its TL / synthesis on the
// cached modes.  Entries are reference counted, so an evicted entry that a
// lane still reads is freed after that lane is done with it.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <cstdint>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ncpa_gpu.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    unsigned long long id = 0;
    // copies of the caller's inputs
    int n_knots = 0;
    std::vector<double> z, u, v, t, p, rho, c0, attn;
    bool has_c0 = false, has_attn = false;
    double z0 = 0.0;
    int has_z0 = 0;
    std::vector<double> freqs;
    double az = 0.0;
    int n_ranges = 0;
    double dr = 0.0;
    std::vector<double> wave_ranges;
    double max_cel = 340.0;
    int nfft = 0, source = 1;
    double est_bytes = 0.0;
    uint64_t h1 = 0, h2 = 0;  // profile hashes (cache key with freqs and az)
    Clock::time_point t_submit;
    // results
    bool done = false;
    int status = NCPA_OK;
    std::vector<int> mode_off;
    std::vector<double> kr, ki, vs, vr, tl_re, tl_im, tl_inc, waves;
    double rho_s = 1.0, rho_r = 1.0;
    double latency_ms = 0.0;
    int batch_requests = 0;
    int from_cache = 0;
};

// one cached solve: the request's modes on the cache context (HBM) and their
// host copies
struct CacheEntry {
    uint64_t h1 = 0, h2 = 0;
    double az = 0.0;
    std::vector<double> freqs;
    ncpa_modes* modes = nullptr;
    std::vector<int> mode_off;
    std::vector<double> kr, ki, vs, vr;
    double rho_s = 1.0, rho_r = 1.0;
    double bytes = 0.0;
};

// two FNV-1a-style 64-bit hashes of the profile (different offsets and
// primes), so a key mismatch has to defeat both
void hash_bytes(uint64_t& a, uint64_t& b, const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) {
        a = (a ^ c[i]) * 0x100000001b3ull;
        b = (b ^ c[i]) * 0x00000100000001b3ull * 0x9e3779b97f4a7c15ull;
    }
}

}  // namespace

struct ncpa_server {
    ncpa_server_opts opts{};
    int nz_pad = 0;
    // mode cache: entries on cache_ctx, most recently used first.  Recursive:
    // an entry evicted under the lock may be destroyed (which locks) at once.
    std::recursive_mutex cache_mu;
    ncpa_ctx* cache_ctx = nullptr;
    std::list<std::shared_ptr<CacheEntry>> lru;
    double cache_used = 0.0;
    long long cache_hits = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> queue;
    std::map<unsigned long long, std::unique_ptr<Request>> all;
    unsigned long long next_id = 1;
    double admitted_bytes = 0.0, peak_admitted = 0.0;
    bool stop = false;
    long long submitted = 0, completed = 0, batches = 0, batched_requests = 0;
    std::vector<double> latencies;
    std::vector<std::thread> lanes;
    std::vector<ncpa_ctx*> ctxs;
};

namespace {

double estimate_bytes(const ncpa_server* s, const Request& r) {
    // per problem: matrix, weights, group speeds, WKB work row, scan counts,
    // modes (up to 2048 of 5 doubles), 1-D TL; plus the profile and waveforms
    const double per_problem = 4.0 * 8.0 * s->nz_pad + 256 * 4 + 2048.0 * 5 * 8 + 3.0 * 8 * r.n_ranges;
    const double waves = (double)r.wave_ranges.size() * 8.0 * std::max(r.nfft, 4 * ((int)r.freqs.size() + 1));
    return per_problem * (double)r.freqs.size() + 12.0 * 8 * r.n_knots + waves;
}

bool same_key(const CacheEntry& e, const Request& r) {
    return e.h1 == r.h1 && e.h2 == r.h2 && e.az == r.az && e.freqs == r.freqs;
}

// the cached entry of r, most recently used from now on, or null
std::shared_ptr<CacheEntry> cache_find(ncpa_server* s, const Request& r) {
    if (!(s->opts.cache_bytes > 0.0)) return nullptr;
    std::lock_guard<std::recursive_mutex> lk(s->cache_mu);
    for (auto it = s->lru.begin(); it != s->lru.end(); ++it) {
        if (same_key(**it, r)) {
            auto e = *it;
            s->lru.erase(it);
            s->lru.push_front(e);
            ++s->cache_hits;
            return e;
        }
    }
    return nullptr;
}

// keeps r's modes in HBM (a copy on the cache context), evicting the least
// recently used entries to stay within the cache budget
void cache_insert(ncpa_server* s, const Request& r) {
    if (!(s->opts.cache_bytes > 0.0) || r.status != NCPA_OK) return;
    const double bytes = (double)r.kr.size() * 4 * 8 + (double)r.freqs.size() * 160 + 256;
    if (bytes > s->opts.cache_bytes) return;
    std::lock_guard<std::recursive_mutex> lk(s->cache_mu);
    for (const auto& e : s->lru)
        if (same_key(*e, r)) return;  // solved twice in flight: keep the first
    while (!s->lru.empty() && s->cache_used + bytes > s->opts.cache_bytes) {
        s->cache_used -= s->lru.back()->bytes;
        s->lru.pop_back();  // freed when the last lane reading it lets go
    }
    ncpa_ctx* cctx = s->cache_ctx;
    std::recursive_mutex* mu = &s->cache_mu;
    // destroyed under the cache lock, which serialises every use of the cache
    // context; the last reference goes once no lane reads the modes any more
    std::shared_ptr<CacheEntry> e(new CacheEntry, [mu](CacheEntry* x) {
        if (x->modes) {
            std::lock_guard<std::recursive_mutex> l(*mu);
            ncpa_modes_destroy(x->modes);
        }
        delete x;
    });
    e->h1 = r.h1;
    e->h2 = r.h2;
    e->az = r.az;
    e->freqs = r.freqs;
    e->mode_off = r.mode_off;
    e->kr = r.kr;
    e->ki = r.ki;
    e->vs = r.vs;
    e->vr = r.vr;
    e->rho_s = r.rho_s;
    e->rho_r = r.rho_r;
    e->bytes = bytes;
    if (ncpa_modes_from_host(cctx, (int)r.freqs.size(), e->mode_off.data(), e->kr.data(), e->ki.data(),
                             e->vs.data(), e->vr.data(), &e->modes) != NCPA_OK)
        return;
    s->lru.push_front(e);
    s->cache_used += bytes;
}

// waveforms of a broadband request from its modes (host arrays): ModBB's
// synthesis with the built-in source spectrum (frequencies k df)
ncpa_status synthesize(ncpa_ctx* ctx, Request& r) {
    if (r.wave_ranges.empty()) return NCPA_OK;
    const int nf = (int)r.freqs.size();
    if (nf < 2) return NCPA_EINVAL;
    const double df = r.freqs[0];
    for (int k = 0; k < nf; ++k)
        if (std::fabs(r.freqs[k] - (k + 1) * df) > 1e-9 * (k + 1) * df) return NCPA_EINVAL;
    std::vector<double> f(nf + 1, 0.0);
    for (int k = 0; k < nf; ++k) f[k + 1] = r.freqs[k];
    std::vector<int> off(nf + 2, 0);
    for (int k = 0; k <= nf; ++k) off[k + 1] = r.mode_off[k];
    const int nfft = std::max(r.nfft, 4 * (nf + 1));
    std::vector<double> sre(nf + 1), sim(nf + 1);
    ncpa_status st = ncpa_source_spectrum_builtin(ctx, r.source, f.data(), nf + 1, -1.0, nfft, sre.data(), sim.data());
    if (st != NCPA_OK) return st;
    ncpa_dispersion_desc d{nf + 1, f.data(), off.data(), r.kr.data(), r.ki.data(), r.vs.data(), r.vr.data(),
                           r.rho_s, r.rho_r};
    ncpa_bb_params bp{(int)r.wave_ranges.size(), r.wave_ranges.data(), r.max_cel, nfft, sre.data(), sim.data(), 0};
    r.waves.assign(r.wave_ranges.size() * (size_t)nfft, 0.0);
    r.nfft = nfft;
    return ncpa_bb_synthesize(ctx, &d, &bp, r.waves.data());
}

// TL (and waveforms) of a request whose modes are cached: no eigen-solve
ncpa_status serve_cached(ncpa_ctx* ctx, Request& r, const CacheEntry& e) {
    const int nf = (int)r.freqs.size();
    r.mode_off = e.mode_off;
    r.kr = e.kr;
    r.ki = e.ki;
    r.vs = e.vs;
    r.vr = e.vr;
    r.rho_s = e.rho_s;
    r.rho_r = e.rho_r;
    const size_t n = (size_t)nf * r.n_ranges;
    r.tl_re.resize(n);
    r.tl_im.resize(n);
    r.tl_inc.resize(n);
    ncpa_tl_params tp{r.n_ranges, r.dr, 0};
    ncpa_status st = ncpa_tl_1d_range(ctx, e.modes, 0, nf, &tp, r.tl_re.data(), r.tl_im.data(), r.tl_inc.data());
    if (st == NCPA_OK) st = synthesize(ctx, r);
    r.status = st;
    r.from_cache = 1;
    r.batch_requests = 1;
    return st;
}

ncpa_status create_profile(ncpa_ctx* ctx, const Request& r, ncpa_profile** out) {
    ncpa_profile_desc d{};
    d.n_knots = r.n_knots;
    d.z = r.z.data();
    d.u = r.u.data();
    d.v = r.v.data();
    d.t = r.t.data();
    d.p = r.p.data();
    d.rho = r.rho.data();
    d.c0 = r.has_c0 ? r.c0.data() : nullptr;
    d.attn = r.has_attn ? r.attn.data() : nullptr;
    d.z0_m = r.z0;
    d.has_z0 = r.has_z0;
    return ncpa_profile_create(ctx, &d, out);
}

// one batched solve for the requests of a batch, then each run of requests
// with the same range grid gets one 1-D TL launch over its slice of the
// batch; fills their results (and waveforms) and caches their modes
ncpa_status run_batch(ncpa_server* s, ncpa_ctx* ctx, const std::vector<Request*>& batch) {
    std::vector<ncpa_profile*> profs(batch.size(), nullptr);
    ncpa_modes* m = nullptr;
    auto cleanup = [&]() {
        if (m) ncpa_modes_destroy(m);
        for (auto* p : profs)
            if (p) ncpa_profile_destroy(p);
    };
    ncpa_status st = NCPA_OK;
    std::vector<ncpa_ess_job> jobs(batch.size());
    for (size_t i = 0; i < batch.size() && st == NCPA_OK; ++i) {
        st = create_profile(ctx, *batch[i], &profs[i]);
        jobs[i] = ncpa_ess_job{profs[i], batch[i]->freqs.data(), (int)batch[i]->freqs.size(), batch[i]->az};
    }
    if (st == NCPA_OK) st = ncpa_ess_solve_jobs(ctx, jobs.data(), (int)jobs.size(), &s->opts.params, &m);
    int P = 0;
    if (st == NCPA_OK) st = ncpa_modes_problems(m, &P);
    // first problem of each request
    std::vector<int> first(batch.size() + 1, 0);
    for (size_t i = 0; i < batch.size(); ++i) first[i + 1] = first[i] + (int)batch[i]->freqs.size();
    for (size_t i = 0; i < batch.size() && st == NCPA_OK;) {
        size_t j = i + 1;
        while (j < batch.size() && batch[j]->n_ranges == batch[i]->n_ranges && batch[j]->dr == batch[i]->dr) ++j;
        const int nr = batch[i]->n_ranges, cnt = first[j] - first[i];
        std::vector<double> re((size_t)cnt * nr), im(re.size()), inc(re.size());
        ncpa_tl_params tp{nr, batch[i]->dr, 0};
        st = ncpa_tl_1d_range(ctx, m, first[i], cnt, &tp, re.data(), im.data(), inc.data());
        for (size_t k = i; k < j && st == NCPA_OK; ++k) {
            Request* r = batch[k];
            const size_t o = (size_t)(first[k] - first[i]) * nr, n = r->freqs.size() * (size_t)nr;
            r->tl_re.assign(re.begin() + o, re.begin() + o + n);
            r->tl_im.assign(im.begin() + o, im.begin() + o + n);
            r->tl_inc.assign(inc.begin() + o, inc.begin() + o + n);
        }
        i = j;
    }
    if (st != NCPA_OK) {
        cleanup();
        return st;
    }
    int p = 0;
    for (Request* r : batch) {
        const int nf = (int)r->freqs.size();
        r->mode_off.assign(1, 0);
        r->kr.clear();
        r->ki.clear();
        r->vs.clear();
        r->vr.clear();
        ncpa_modes_info(m, p, nullptr, nullptr, nullptr, nullptr, nullptr, &r->rho_s, &r->rho_r);
        for (int f = 0; f < nf; ++f, ++p) {
            int M = 0;
            ncpa_modes_count(m, p, &M);
            const size_t o = r->kr.size();
            r->kr.resize(o + M);
            r->ki.resize(o + M);
            r->vs.resize(o + M);
            r->vr.resize(o + M);
            if (M) ncpa_modes_get(m, p, &r->kr[o], &r->ki[o], &r->vs[o], &r->vr[o], nullptr);
            r->mode_off.push_back((int)r->kr.size());
        }
        r->status = synthesize(ctx, *r);
        r->batch_requests = (int)batch.size();
        r->from_cache = 0;
        cache_insert(s, *r);
    }
    cleanup();
    return NCPA_OK;
}

void lane_main(ncpa_server* s, int lane) {
    ncpa_ctx* ctx = s->ctxs[lane];
    for (;;) {
        std::vector<Request*> batch;
        double bytes = 0.0;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            // admission: the oldest request fits the budget, or nothing runs
            // the cache's HBM counts against the budget
            double budget = s->opts.hbm_budget_bytes;
            {
                std::lock_guard<std::recursive_mutex> cl(s->cache_mu);
                budget -= s->cache_used;
            }
            auto can_take = [&] {
                return !s->queue.empty() &&
                       (s->admitted_bytes == 0.0 || s->admitted_bytes + s->queue.front()->est_bytes <= budget);
            };
            s->cv_work.wait(lk, [&] { return (s->stop && s->queue.empty()) || can_take(); });
            if (s->queue.empty()) return;  // stopping; queued work is finished before a lane stops
            int problems = 0;
            for (auto it = s->queue.begin(); it != s->queue.end();) {
                Request* r = *it;  // taken in arrival order while the batch limits hold
                const bool fits_batch = batch.empty() || problems + (int)r->freqs.size() <= s->opts.max_batch_problems;
                const bool fits_mem = (s->admitted_bytes == 0.0 && batch.empty()) ||
                                      s->admitted_bytes + bytes + r->est_bytes <= budget;
                if (fits_batch && fits_mem) {
                    batch.push_back(r);
                    problems += (int)r->freqs.size();
                    bytes += r->est_bytes;
                    it = s->queue.erase(it);
                } else {
                    break;  // keep arrival order for what is left
                }
            }
            s->admitted_bytes += bytes;
            s->peak_admitted = std::max(s->peak_admitted, s->admitted_bytes);
        }
        // requests whose modes are cached skip the solve
        std::vector<Request*> solve;
        for (Request* r : batch) {
            auto e = cache_find(s, *r);
            if (e) serve_cached(ctx, *r, *e);
            else solve.push_back(r);
        }
        ncpa_status st = solve.empty() ? NCPA_OK : run_batch(s, ctx, solve);
        if (st != NCPA_OK) {
            if (solve.size() > 1) {
                for (Request* r : solve) {
                    const ncpa_status si = run_batch(s, ctx, std::vector<Request*>{r});
                    if (si != NCPA_OK) r->status = si;
                }
            } else {
                solve[0]->status = st;
            }
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            const auto now = Clock::now();
            for (Request* r : batch) {
                r->latency_ms = std::chrono::duration<double, std::milli>(now - r->t_submit).count();
                r->done = true;
                s->latencies.push_back(r->latency_ms);
                ++s->completed;
            }
            ++s->batches;
            s->batched_requests += (long long)batch.size();
            s->admitted_bytes -= bytes;
            if (s->admitted_bytes < 1.0) s->admitted_bytes = 0.0;
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
}

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t i = (size_t)pos;
    const double f = pos - (double)i;
    return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

}  // namespace

extern "C" {

void ncpa_server_opts_default(ncpa_server_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    ncpa_ess_params_default(&o->params);
    o->n_ranges = 2000;
    o->dr_m = 500.0;
    o->lanes = 2;
    o->max_batch_problems = 1024;
    o->hbm_budget_bytes = 8.0 * (1ull << 30);
    o->cache_bytes = 0.0;
}

ncpa_status ncpa_server_create(const ncpa_server_opts* opts, ncpa_server** out) {
    if (!opts || !out) return NCPA_EINVAL;
    *out = nullptr;
    if (opts->n_ranges < 1 || !(opts->dr_m > 0.0) || opts->params.nz_grid < 10) return NCPA_EINVAL;
    auto s = std::make_unique<ncpa_server>();
    s->opts = *opts;
    if (s->opts.lanes <= 0) s->opts.lanes = 2;
    if (s->opts.max_batch_problems <= 0) s->opts.max_batch_problems = 1024;
    if (!(s->opts.hbm_budget_bytes > 0.0)) s->opts.hbm_budget_bytes = 8.0 * (1ull << 30);
    s->opts.params.keep_on_device = 0;
    if (s->opts.cache_bytes < 0.0) s->opts.cache_bytes = 0.0;
    s->nz_pad = (s->opts.params.nz_grid + 1023) / 1024 * 1024;
    if (s->opts.cache_bytes > 0.0) {
        ncpa_ctx_opts co{opts->device};
        const ncpa_status st = ncpa_ctx_create(&s->cache_ctx, &co);
        if (st != NCPA_OK) return st;
    }
    for (int l = 0; l < s->opts.lanes; ++l) {
        ncpa_ctx* c = nullptr;
        ncpa_ctx_opts co{opts->device};
        const ncpa_status st = ncpa_ctx_create(&c, &co);
        if (st != NCPA_OK) {
            for (auto* x : s->ctxs) ncpa_ctx_destroy(x);
            if (s->cache_ctx) ncpa_ctx_destroy(s->cache_ctx);
            return st;
        }
        s->ctxs.push_back(c);
    }
    ncpa_server* raw = s.get();
    for (int l = 0; l < s->opts.lanes; ++l) s->lanes.emplace_back(lane_main, raw, l);
    *out = s.release();
    return NCPA_OK;
}

ncpa_status ncpa_server_submit(ncpa_server* s, const ncpa_request* req, unsigned long long* id) {
    if (!s || !req || !id || !req->freqs || req->n_freq < 1) return NCPA_EINVAL;
    const ncpa_profile_desc& d = req->profile;
    if (d.n_knots < 3 || !d.z || !d.u || !d.v || !d.t || !d.p || !d.rho) return NCPA_EINVAL;
    for (int i = 0; i < req->n_freq; ++i)
        if (!(req->freqs[i] > 0.0)) return NCPA_EINVAL;
    auto r = std::make_unique<Request>();
    const int n = d.n_knots;
    r->n_knots = n;
    r->z.assign(d.z, d.z + n);
    r->u.assign(d.u, d.u + n);
    r->v.assign(d.v, d.v + n);
    r->t.assign(d.t, d.t + n);
    r->p.assign(d.p, d.p + n);
    r->rho.assign(d.rho, d.rho + n);
    if (d.c0) {
        r->c0.assign(d.c0, d.c0 + n);
        r->has_c0 = true;
    }
    if (d.attn) {
        r->attn.assign(d.attn, d.attn + n);
        r->has_attn = true;
    }
    r->z0 = d.z0_m;
    r->has_z0 = d.has_z0;
    r->freqs.assign(req->freqs, req->freqs + req->n_freq);
    r->az = req->az_deg;
    r->n_ranges = req->n_ranges > 0 ? req->n_ranges : s->opts.n_ranges;
    r->dr = req->n_ranges > 0 ? req->dr_m : s->opts.dr_m;
    if (!(r->dr > 0.0)) return NCPA_EINVAL;
    if (req->n_wave_ranges > 0) {
        if (!req->wave_ranges_m || req->n_freq < 2 || req->source < 0 || req->source > 2 || req->nfft < 0)
            return NCPA_EINVAL;
        r->wave_ranges.assign(req->wave_ranges_m, req->wave_ranges_m + req->n_wave_ranges);
        r->max_cel = req->max_celerity > 0.0 ? req->max_celerity : 340.0;
        r->nfft = req->nfft;
        r->source = req->source;
    }
    // cache key: the profile's knot values (and which optional arrays it has)
    uint64_t h1 = 0xcbf29ce484222325ull, h2 = 0x84222325cbf29ce4ull;
    hash_bytes(h1, h2, &n, sizeof n);
    for (const auto* a : {&r->z, &r->u, &r->v, &r->t, &r->p, &r->rho, &r->c0, &r->attn})
        if (!a->empty()) hash_bytes(h1, h2, a->data(), a->size() * 8);
    const int flags[3] = {r->has_c0, r->has_attn, r->has_z0};
    hash_bytes(h1, h2, flags, sizeof flags);
    if (r->has_z0) hash_bytes(h1, h2, &r->z0, sizeof r->z0);
    r->h1 = h1;
    r->h2 = h2;
    r->est_bytes = estimate_bytes(s, *r);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->id = s->next_id++;
        r->t_submit = Clock::now();
        *id = r->id;
        s->queue.push_back(r.get());
        s->all.emplace(r->id, std::move(r));
        ++s->submitted;
    }
    s->cv_work.notify_one();
    return NCPA_OK;
}

ncpa_status ncpa_server_wait(ncpa_server* s, unsigned long long id, int timeout_ms, ncpa_result* out) {
    if (!s || !out) return NCPA_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return NCPA_EINVAL;
    Request* r = it->second.get();
    auto ready = [&] { return r->done; };
    if (timeout_ms < 0) s->cv_done.wait(lk, ready);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return NCPA_ETIMEDOUT;
    out->status = r->status;
    out->n_freq = (int)r->freqs.size();
    out->mode_off = r->mode_off.empty() ? nullptr : r->mode_off.data();
    out->re_k = r->kr.data();
    out->im_k = r->ki.data();
    out->v_src = r->vs.data();
    out->v_rcv = r->vr.data();
    out->tl_re = r->tl_re.data();
    out->tl_im = r->tl_im.data();
    out->tl_incoh = r->tl_inc.data();
    out->latency_ms = r->latency_ms;
    out->batch_requests = r->batch_requests;
    out->n_ranges = r->n_ranges;
    out->n_wave_ranges = r->waves.empty() ? 0 : (int)r->wave_ranges.size();
    out->nfft = r->waves.empty() ? 0 : r->nfft;
    out->waveforms = r->waves.empty() ? nullptr : r->waves.data();
    out->from_cache = r->from_cache;
    return NCPA_OK;
}

ncpa_status ncpa_server_release(ncpa_server* s, unsigned long long id) {
    if (!s) return NCPA_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end() || !it->second->done) return NCPA_EINVAL;
    s->all.erase(it);
    return NCPA_OK;
}

ncpa_status ncpa_server_stats_get(ncpa_server* s, ncpa_server_stats* o) {
    if (!s || !o) return NCPA_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    o->submitted = s->submitted;
    o->completed = s->completed;
    o->batches = s->batches;
    o->mean_batch_requests = s->batches ? (double)s->batched_requests / (double)s->batches : 0.0;
    o->p50_ms = percentile(s->latencies, 0.50);
    o->p99_ms = percentile(s->latencies, 0.99);
    o->max_ms = s->latencies.empty() ? 0.0 : *std::max_element(s->latencies.begin(), s->latencies.end());
    o->peak_admitted_bytes = s->peak_admitted;
    std::lock_guard<std::recursive_mutex> cl(s->cache_mu);
    o->cache_hits = s->cache_hits;
    o->cache_entries = (long long)s->lru.size();
    o->cache_used_bytes = s->cache_used;
    return NCPA_OK;
}

ncpa_status ncpa_server_destroy(ncpa_server* s) {
    if (!s) return NCPA_EINVAL;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->lanes) t.join();
    {
        std::lock_guard<std::recursive_mutex> cl(s->cache_mu);
        s->lru.clear();  // every lane has stopped: the entries go now
        s->cache_used = 0.0;
    }
    for (auto* c : s->ctxs) ncpa_ctx_destroy(c);
    if (s->cache_ctx) ncpa_ctx_destroy(s->cache_ctx);
    delete s;
    return NCPA_OK;
}

}  // extern "C"
