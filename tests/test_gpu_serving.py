"""Batched multi-profile solve and the serving loop on the GPU.

- ncpa_ess_solve_jobs over jobs with different profiles, frequencies and
  azimuths gives, problem by problem, exactly what ncpa_ess_solve gives for
  each job alone.
- Every served request's dispersion and 1-D TL are the same whether it was
  solved alone or in a batch with others (continuous batching), and the HBM
  admission limit serialises requests when it is tight.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NZ = 4000
NR, DR = 300, 2000.0


def _jobs(seed, n):
    import workloads

    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        prof = workloads.perturbed_profile(rng)
        if k % 3 == 1:
            nf = int(rng.integers(8, 24))
            freqs = 0.25 / nf * np.arange(1, nf + 1)
        else:
            freqs = np.array([np.exp(rng.uniform(np.log(0.05), np.log(0.6)))])
        out.append((prof, freqs, float(rng.uniform(0.0, 360.0))))
    return out


def _params(**kw):
    import ncpa_gpu

    return ncpa_gpu.default_params(nz_grid=NZ, **kw)


def _alone(gpu, prof, freqs, az):
    p = gpu.profile_from_arrays(*prof)
    m = gpu.solve(p, _params(), freqs, [az])
    probs = [m.problem(i) for i in range(m.P)]
    re, im, inc = m.tl1d(NR, DR)
    m.close()
    p.close()
    return probs, re, im, inc


def test_solve_jobs_equals_one_solve_per_job(gpu):
    jobs = _jobs(11, 5)
    profs = [gpu.profile_from_arrays(*j[0]) for j in jobs]
    m = gpu.solve_jobs([(p, f, az) for p, (_, f, az) in zip(profs, jobs)], _params())
    assert m.P == sum(len(j[1]) for j in jobs)
    re_b, im_b, _ = m.tl1d(NR, DR)
    off, kr, ki, vs, vr, _ = m.all_modes()  # bulk getter, CSR order
    # the same into caller buffers (larger than needed)
    n = m.total_modes()
    assert n == off[-1]
    bufs = [np.full(n + 7, np.nan) for _ in range(5)]
    off2, kr2, ki2, vs2, vr2, _ = m.all_modes(out=bufs)
    assert np.array_equal(off2, off) and np.array_equal(kr2, kr) and np.array_equal(vr2, vr)
    assert kr2.base is bufs[0] or np.shares_memory(kr2, bufs[0])
    assert np.isnan(bufs[0][n:]).all()
    for i in range(m.P):
        b = m.problem(i)
        assert off[i + 1] - off[i] == b.M
        assert np.array_equal(kr[off[i]:off[i + 1]], b.kr) and np.array_equal(vr[off[i]:off[i + 1]], b.vr)
    p0 = 0
    for prof, freqs, az in jobs:
        probs, re, im, _ = _alone(gpu, prof, freqs, az)
        for i, a in enumerate(probs):
            b = m.problem(p0 + i)
            assert b.M == a.M and b.freq == a.freq and b.az == a.az
            for k in ("kr", "ki", "vs", "vr"):
                assert np.array_equal(getattr(a, k), getattr(b, k)), k
            assert b.rho_src == a.rho_src and b.rho_rcv == a.rho_rcv
            assert np.array_equal(re[i], re_b[p0 + i]) and np.array_equal(im[i], im_b[p0 + i])
        p0 += len(freqs)
    m.close()
    for p in profs:
        p.close()


def test_served_results_equal_alone_and_in_the_mix(gpu):
    import ncpa_gpu

    jobs = _jobs(23, 12)
    with ncpa_gpu.Server(0, params=_params(), n_ranges=NR, dr_m=DR, lanes=2) as srv:
        ids = [srv.submit(*prof, freqs, az) for prof, freqs, az in jobs]
        res = [srv.wait(i, timeout_ms=120000) for i in ids]
        st = srv.stats()
    assert st["completed"] == len(jobs)
    assert max(r["batch_requests"] for r in res) >= 2  # some requests shared a batch
    for (prof, freqs, az), r in zip(jobs, res):
        assert r["status"] == 0
        probs, re, im, inc = _alone(gpu, prof, freqs, az)
        off = r["mode_off"]
        for i, a in enumerate(probs):
            sl = slice(off[i], off[i + 1])
            assert off[i + 1] - off[i] == a.M
            assert np.array_equal(r["re_k"][sl], a.kr) and np.array_equal(r["im_k"][sl], a.ki)
            assert np.array_equal(r["v_src"][sl] * r["v_rcv"][sl], a.vs * a.vr)
        assert np.array_equal(r["tl_re"], re) and np.array_equal(r["tl_im"], im)
        assert np.array_equal(r["tl_incoh"], inc)
    assert st["p99_ms"] >= st["p50_ms"] > 0


def test_tight_hbm_budget_admits_one_request_at_a_time(gpu):
    import ncpa_gpu

    jobs = _jobs(5, 6)
    with ncpa_gpu.Server(0, params=_params(), n_ranges=NR, dr_m=DR, lanes=2, hbm_budget_bytes=1.0) as srv:
        ids = [srv.submit(*prof, freqs, az) for prof, freqs, az in jobs]
        res = [srv.wait(i, timeout_ms=120000) for i in ids]
        st = srv.stats()
    assert all(r["status"] == 0 for r in res)
    assert all(r["batch_requests"] == 1 for r in res)
    assert st["batches"] == len(jobs)


def _alone_grid(gpu, prof, freqs, az, nr, dr):
    p = gpu.profile_from_arrays(*prof)
    m = gpu.solve(p, _params(), freqs, [az])
    re, im, inc = m.tl1d(nr, dr)
    return p, m, re, im, inc


def test_per_request_range_grids_and_waveforms(gpu):
    """Each request's own TL range grid, and waveforms for broadband
    requests, equal the same request solved alone (synthesis of the solve's
    own dispersion, ModBB's built-in pulse)."""
    import ncpa_gpu

    jobs = _jobs(31, 9)
    grids = [(0, 0.0), (150, 3000.0), (NR, DR), (420, 1000.0)]
    with ncpa_gpu.Server(0, params=_params(), n_ranges=NR, dr_m=DR, lanes=2) as srv:
        ids = []
        for k, (prof, freqs, az) in enumerate(jobs):
            nr, dr = grids[k % len(grids)]
            wr = np.array([80e3, 140e3]) if len(freqs) > 1 else None
            ids.append(srv.submit(*prof, freqs, az, n_ranges=nr, dr_m=dr, wave_ranges_m=wr, max_celerity=330.0))
        res = [srv.wait(i, timeout_ms=120000) for i in ids]
    n_wave = 0
    for k, ((prof, freqs, az), r) in enumerate(zip(jobs, res)):
        assert r["status"] == 0 and not r["from_cache"]
        nr, dr = grids[k % len(grids)]
        if nr == 0:
            nr, dr = NR, DR
        p, m, re, im, inc = _alone_grid(gpu, prof, freqs, az, nr, dr)
        assert r["tl_re"].shape == (len(freqs), nr)
        assert np.array_equal(r["tl_re"], re) and np.array_equal(r["tl_im"], im)
        assert np.array_equal(r["tl_incoh"], inc)
        if len(freqs) > 1:
            n_wave += 1
            f = np.concatenate([[0.0], freqs])
            nfft = 4 * len(f)
            sre, sim = gpu.source_spectrum_builtin("pulse1", f, nfft)
            w = m.bb_synthesize(np.array([80e3, 140e3]), 330.0, nfft, sre, sim)
            assert r["waveforms"].shape == w.shape
            assert np.linalg.norm(r["waveforms"] - w) <= 1e-12 * np.linalg.norm(w)
        else:
            assert "waveforms" not in r
        m.close()
        p.close()
    assert n_wave > 0


def test_mode_cache_skips_the_solve_and_equals_a_fresh_one(gpu):
    """With a cache, a repeated request is served from its modes kept in HBM
    (no eigen-solve) and gives the fresh result bit for bit, on its own range
    grid too; a changed profile is not a hit."""
    import ncpa_gpu

    jobs = _jobs(41, 6)
    with ncpa_gpu.Server(0, params=_params(), n_ranges=NR, dr_m=DR, lanes=2, cache_bytes=float(1 << 30)) as srv:
        first = [srv.wait(srv.submit(*prof, freqs, az), timeout_ms=120000) for prof, freqs, az in jobs]
        again = [srv.wait(srv.submit(*prof, freqs, az), timeout_ms=120000) for prof, freqs, az in jobs]
        grid = [srv.wait(srv.submit(*prof, freqs, az, n_ranges=77, dr_m=3500.0), timeout_ms=120000)
                for prof, freqs, az in jobs]
        prof, freqs, az = jobs[0]
        changed = list(prof)
        changed[3] = changed[3] + 0.5  # temperature
        other = srv.wait(srv.submit(*changed, freqs, az), timeout_ms=120000)
        st = srv.stats()
    assert all(not r["from_cache"] for r in first)
    assert all(r["from_cache"] for r in again) and all(r["from_cache"] for r in grid)
    assert not other["from_cache"]
    assert st["cache_hits"] == 2 * len(jobs) and st["cache_entries"] == len(jobs) + 1
    for a, b in zip(first, again):
        for k in ("mode_off", "re_k", "im_k", "v_src", "v_rcv", "tl_re", "tl_im", "tl_incoh"):
            assert np.array_equal(a[k], b[k]), k
    for (prof, freqs, az), r in zip(jobs, grid):
        p, m, re, im, inc = _alone_grid(gpu, prof, freqs, az, 77, 3500.0)
        assert np.array_equal(r["tl_re"], re) and np.array_equal(r["tl_im"], im)
        m.close()
        p.close()


def test_mode_cache_evicts_within_its_budget(gpu):
    import ncpa_gpu

    jobs = _jobs(43, 8)
    with ncpa_gpu.Server(0, params=_params(), n_ranges=NR, dr_m=DR, lanes=2, cache_bytes=60e3) as srv:
        res = [srv.wait(srv.submit(*prof, freqs, az), timeout_ms=120000) for prof, freqs, az in jobs]
        again = [srv.wait(srv.submit(*prof, freqs, az), timeout_ms=120000) for prof, freqs, az in jobs]
        st = srv.stats()
    assert st["cache_used_bytes"] <= 60e3
    assert st["cache_entries"] < len(jobs)
    for a, b in zip(res, again):
        assert b["status"] == 0
        assert np.array_equal(a["tl_re"], b["tl_re"]) and np.array_equal(a["re_k"], b["re_k"])
