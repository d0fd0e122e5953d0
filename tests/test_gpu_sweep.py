"""Batches that mix solver grid sizes (the azimuth sweep with Nz per frequency).

- A batch of jobs with different grids, frequencies and azimuth lists gives,
  problem by problem, exactly what a separate ncpa_ess_solve on that grid
  gives (bit for bit: the kernels read each problem's own grid).
- A reduced azimuth sweep (8 log-spaced frequencies, Nz following the
  wavelength, several azimuths, one batch) against the oracle: mode counts
  identical, Re k within 1e-9 relative (or the conditioning floor), TL within
  0.05 dB where TL > -140 dB.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = np.finfo(float).eps


def _params(**kw):
    import ncpa_gpu

    return ncpa_gpu.default_params(**kw)


def test_mixed_grid_batch_equals_solo_solves(gpu, analytic_profile):
    import workloads

    rng = np.random.default_rng(7)
    prof = gpu.load_profile(analytic_profile)
    pert = gpu.profile_from_arrays(*workloads.perturbed_profile(rng))
    jobs = [
        (prof, [0.1, 0.2], [30.0, 90.0, 200.0], 3000),
        (prof, [0.35], [0.0, 120.0], 7000),
        (pert, [0.5], 45.0, 5000),
        (prof, [0.05, 0.15], 270.0, 0),  # 0: params' grid (4000)
    ]
    prm = _params(nz_grid=4000, want_group_speed=1)
    m = gpu.solve_jobs(jobs, prm)
    assert m.P == 6 + 2 + 1 + 2
    re_b, im_b, inc_b = m.tl1d(400, 2500.0)
    p = 0
    for pr, freqs, az, nz in jobs:
        azs = np.atleast_1d(az)
        solo = gpu.solve(pr, _params(nz_grid=nz or 4000, want_group_speed=1), freqs, azs)
        re, im, inc = solo.tl1d(400, 2500.0)
        for i in range(solo.P):
            a, b = solo.problem(i), m.problem(p)
            assert b.M == a.M and b.freq == a.freq and b.az == a.az and b.dz == a.dz
            for k in ("kr", "ki", "vs", "vr", "vg"):
                assert np.array_equal(getattr(a, k), getattr(b, k)), (p, k)
            assert b.rho_src == a.rho_src and b.rho_rcv == a.rho_rcv
            assert np.array_equal(re[i], re_b[p]) and np.array_equal(im[i], im_b[p])
            assert np.array_equal(inc[i], inc_b[p])
            p += 1
        solo.close()
    m.close()
    pert.close()
    prof.close()


def test_reduced_sweep_vs_oracle(gpu, analytic_profile):
    """8 frequencies 0.1-0.4 Hz log-spaced, Nz = 20 points per wavelength at
    300 m/s (at least 1000), 3 azimuths: one batch of 24 problems on 6 grids."""
    import workloads
    from oracle import oracle as O

    freqs = workloads.sweep_freqs(8, 0.1, 0.4)
    nzs = [workloads.sweep_nz(f, points_per_wavelength=20, nz_min=1000) for f in freqs]
    assert len(set(nzs)) >= 5
    azs = [0.0, 90.0, 250.0]
    prof = gpu.load_profile(analytic_profile)
    jobs = [(prof, [f], azs, nz) for f, nz in zip(freqs, nzs)]
    m = gpu.solve_jobs(jobs, _params(turnoff_wkb=1))
    re, im, _ = m.tl1d(500, 2000.0)
    op = O.read_profile(analytic_profile)
    p = 0
    for f, nz in zip(freqs, nzs):
        prm = O.EssParams(Nz_grid=nz, turnoff_WKB=True)
        pp = O.prepare(op, prm)
        for a in azs:
            g = m.problem(p)
            o = O.solve_problem(pp, prm, f, a)
            assert g.M == o.M, (f, a, g.M, o.M)
            assert abs(g.dz - o.dz) <= 1e-15 * o.dz
            tol = np.maximum(1e-9, 8 * EPS * (4.0 / o.dz ** 2) / (2 * o.kr ** 2))
            assert np.all(np.abs(g.kr - o.kr) / o.kr <= tol)
            ore, oim, _ = O.tl1d(o, 500, 2000.0)
            tl_g = 20 * np.log10(np.hypot(re[p], im[p]))
            tl_o = 20 * np.log10(np.hypot(ore, oim))
            mask = tl_o > -140
            assert np.max(np.abs(tl_g - tl_o)[mask]) <= 0.05
            p += 1
    m.close()
    prof.close()


def test_job_arguments_are_checked(gpu, analytic_profile):
    import ncpa_gpu

    prof = gpu.load_profile(analytic_profile)
    with pytest.raises(ncpa_gpu.NcpaError):
        gpu.solve_jobs([(prof, [0.1], 90.0, 5)], _params())  # grid too small
    prof.close()
