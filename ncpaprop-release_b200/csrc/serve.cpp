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
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
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
    double est_bytes = 0.0;
    Clock::time_point t_submit;
    // results
    bool done = false;
    int status = NCPA_OK;
    std::vector<int> mode_off;
    std::vector<double> kr, ki, vs, vr, tl_re, tl_im, tl_inc;
    double latency_ms = 0.0;
    int batch_requests = 0;
};

}  // namespace

struct ncpa_server {
    ncpa_server_opts opts{};
    int nz_pad = 0;
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
    // modes (up to 2048 of 5 doubles), 1-D TL; plus the profile
    const double per_problem = 4.0 * 8.0 * s->nz_pad + 256 * 4 + 2048.0 * 5 * 8 + 3.0 * 8 * s->opts.n_ranges;
    return per_problem * (double)r.freqs.size() + 12.0 * 8 * r.n_knots;
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

// one batched solve + 1-D TL for the requests of a batch; fills their results
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
    const int nr = s->opts.n_ranges;
    std::vector<double> re, im, inc;
    if (st == NCPA_OK) {
        re.resize((size_t)P * nr);
        im.resize(re.size());
        inc.resize(re.size());
        ncpa_tl_params tp{nr, s->opts.dr_m, 0};
        st = ncpa_tl_1d(ctx, m, &tp, re.data(), im.data(), inc.data());
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
        const size_t o = (size_t)(p - nf) * nr;
        r->tl_re.assign(re.begin() + o, re.begin() + o + (size_t)nf * nr);
        r->tl_im.assign(im.begin() + o, im.begin() + o + (size_t)nf * nr);
        r->tl_inc.assign(inc.begin() + o, inc.begin() + o + (size_t)nf * nr);
        r->status = NCPA_OK;
        r->batch_requests = (int)batch.size();
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
            auto can_take = [&] {
                return !s->queue.empty() &&
                       (s->admitted_bytes == 0.0 ||
                        s->admitted_bytes + s->queue.front()->est_bytes <= s->opts.hbm_budget_bytes);
            };
            s->cv_work.wait(lk, [&] { return (s->stop && s->queue.empty()) || can_take(); });
            if (s->queue.empty()) return;  // stopping; queued work is finished before a lane stops
            int problems = 0;
            for (auto it = s->queue.begin(); it != s->queue.end();) {
                Request* r = *it;  // taken in arrival order while the batch limits hold
                const bool fits_batch = batch.empty() || problems + (int)r->freqs.size() <= s->opts.max_batch_problems;
                const bool fits_mem = (s->admitted_bytes == 0.0 && batch.empty()) ||
                                      s->admitted_bytes + bytes + r->est_bytes <= s->opts.hbm_budget_bytes;
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
        ncpa_status st = run_batch(s, ctx, batch);
        if (st != NCPA_OK) {
            if (batch.size() > 1) {
                for (Request* r : batch) {
                    const ncpa_status si = run_batch(s, ctx, std::vector<Request*>{r});
                    if (si != NCPA_OK) r->status = si;
                }
            } else {
                batch[0]->status = st;
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
    s->nz_pad = (s->opts.params.nz_grid + 1023) / 1024 * 1024;
    for (int l = 0; l < s->opts.lanes; ++l) {
        ncpa_ctx* c = nullptr;
        ncpa_ctx_opts co{opts->device};
        const ncpa_status st = ncpa_ctx_create(&c, &co);
        if (st != NCPA_OK) {
            for (auto* x : s->ctxs) ncpa_ctx_destroy(x);
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
    for (auto* c : s->ctxs) ncpa_ctx_destroy(c);
    delete s;
    return NCPA_OK;
}

}  // extern "C"
