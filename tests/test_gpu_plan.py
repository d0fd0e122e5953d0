"""Captured solves (plans): one CUDA graph per batch shape, autotuned launch
shapes, profile updates between replays.

- An untuned plan gives, replay after replay, exactly what ncpa_ess_solve_jobs
  plus ncpa_tl_1d give for the same jobs (same kernels, same launch shapes).
- After ncpa_profile_update a replay equals a fresh solve of the new profile.
- A tuned plan keeps the mode counts and agrees on k within the parity bound
  (another bisection item size only changes the bracketing) and on TL within
  1e-3 dB where TL > -140 dB.
- Plans refuse what needs host work inside the solve, and the objects a
  graph reads cannot be destroyed under it.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = np.finfo(float).eps
NR, DR = 300, 3000.0


def _params(**kw):
    import ncpa_gpu

    return ncpa_gpu.default_params(**kw)


def _jobs(prof):
    return [(prof, [0.1, 0.25], [0.0, 90.0, 180.0], 3000),
            (prof, [0.4], [45.0, 300.0], 6000),
            (prof, [0.05, 0.15, 0.2], 270.0, 0)]


def _same(a, b):
    for p in range(a.P):
        x, y = a.problem(p), b.problem(p)
        assert x.M == y.M and x.freq == y.freq and x.az == y.az and x.dz == y.dz
        for k in ("kr", "ki", "vs", "vr", "vg"):
            assert np.array_equal(getattr(x, k), getattr(y, k)), (p, k)
        assert x.rho_src == y.rho_src and x.rho_rcv == y.rho_rcv


def test_plan_equals_solve_jobs(gpu, analytic_profile):
    prof = gpu.load_profile(analytic_profile)
    jobs = _jobs(prof)
    prm = _params(nz_grid=4000, want_group_speed=1)
    ref = gpu.solve_jobs(jobs, prm)
    re0, im0, inc0 = ref.tl1d(NR, DR)
    l0 = gpu.launches
    with gpu.plan(jobs, prm, tl=(NR, DR)) as plan:
        assert gpu.launches == l0  # capture launches nothing
        for _ in range(2):  # replays are identical
            plan.run()
            assert gpu.launches > l0
            _same(ref, plan.modes())
            re, im, inc = plan.tl()
            assert np.array_equal(re, re0) and np.array_equal(im, im0) and np.array_equal(inc, inc0)
        t = plan.tuning()
        assert t["bis_item"] == 32 and t["ms"] == 0.0
    ref.close()
    prof.close()


def test_profile_update_between_replays(gpu):
    import workloads

    rng = np.random.default_rng(3)
    a = workloads.perturbed_profile(rng)
    b = workloads.perturbed_profile(rng)
    assert np.array_equal(a[0], b[0])
    prof = gpu.profile_from_arrays(*a)
    jobs = [(prof, [0.08, 0.3], [20.0, 200.0], 5000)]
    prm = _params()
    with gpu.plan(jobs, prm, tl=(NR, DR)) as plan:
        for arrays in (b, a, b):
            prof.update(*arrays)
            plan.run()
            fresh = gpu.profile_from_arrays(*arrays)
            ref = gpu.solve_jobs([(fresh, [0.08, 0.3], [20.0, 200.0], 5000)], prm)
            _same(ref, plan.modes())
            re0, im0, _ = ref.tl1d(NR, DR)
            re, im, _ = plan.tl()
            assert np.array_equal(re, re0) and np.array_equal(im, im0)
            ref.close()
            fresh.close()
    prof.close()


def test_tuned_plan(gpu, analytic_profile):
    prof = gpu.load_profile(analytic_profile)
    jobs = _jobs(prof)
    prm = _params(nz_grid=4000)
    ref = gpu.solve_jobs(jobs, prm)
    re0, im0, _ = ref.tl1d(NR, DR)
    with gpu.plan(jobs, prm, tl=(NR, DR), tune=True) as plan:
        t = plan.tuning()
        assert t["bis_item"] in (16, 24, 32) and t["bis_ctas_per_sm"] >= 1 and t["ev_ctas_per_sm"] >= 1
        assert t["ms"] > 0.0
        plan.run()
        m = plan.modes()
        for p in range(ref.P):
            x, y = ref.problem(p), m.problem(p)
            assert x.M == y.M
            tol = np.maximum(1e-9, 8 * EPS * (4.0 / x.dz ** 2) / (2 * x.kr ** 2))
            assert np.all(np.abs(x.kr - y.kr) / x.kr <= tol)
        re, im, _ = plan.tl()
        tl0 = 20 * np.log10(np.hypot(re0, im0))
        tl1 = 20 * np.log10(np.hypot(re, im))
        mask = tl0 > -140
        assert np.max(np.abs(tl1 - tl0)[mask]) <= 1e-3
    # the tuned shapes are cached per batch shape: a second plan reuses them
    with gpu.plan(jobs, prm, tl=(NR, DR), tune=True) as again:
        assert {k: v for k, v in again.tuning().items() if k != "ms"} == \
               {k: v for k, v in t.items() if k != "ms"}
    ref.close()
    prof.close()


def test_plan_guards(gpu, analytic_profile):
    import ncpa_gpu

    prof = gpu.load_profile(analytic_profile)
    jobs = [(prof, [0.1], 90.0, 2000)]
    for bad in (_params(want_vectors=1), _params(lamb_wave_bc=1)):
        with pytest.raises(ncpa_gpu.NcpaError):
            gpu.plan(jobs, bad)
    plan = gpu.plan(jobs, _params())
    with pytest.raises(ncpa_gpu.NcpaError):
        plan.modes()  # not run yet
    plan.run()
    m = plan.modes()
    assert ncpa_gpu.lib().ncpa_modes_destroy(m.h) != 0          # owned by the plan
    assert ncpa_gpu.lib().ncpa_profile_destroy(prof.h) != 0     # read by the plan's graph
    z_km, attn = np.array([0.0, 150.0]), np.array([1e-6, 1e-5])
    assert ncpa_gpu.lib().ncpa_profile_set_attn(prof.h, ncpa_gpu._p(z_km), ncpa_gpu._p(attn), 2) != 0
    re, im, inc = m.tl1d(10, 1000.0)  # host TL of plan-owned modes uses temporaries
    assert np.all(np.isfinite(re))
    plan.close()
    prof.close()
    assert not prof.h
