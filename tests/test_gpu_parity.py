"""GPU (C ABI) vs CPU oracle on the same inputs.

Tolerances (the reference's own numbers):
  * mode counts: identical;
  * Re k: |dk|/k <= max(1e-9, 8 eps |A| / (2 k^2)) -- the second term is the
    conditioning floor of the finite-difference eigenproblem, |A| ~ 4/dz^2;
  * TL: |dTL| <= 0.05 dB wherever TL > -140 dB;
  * V_s V_r and Im k: 1e-6 relative (eigenvector pieces agree far better);
  * waveforms: 1e-4 relative L2.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = np.finfo(float).eps


def _k_tol(k, dz):
    return np.maximum(1e-9, 8 * EPS * (4.0 / dz ** 2) / (2 * k ** 2))


def _oracle_modes(path, freq, az, **kw):
    from oracle import oracle as O

    prof = O.read_profile(path)
    prm = O.EssParams(**kw)
    pp = O.prepare(prof, prm)
    return O, pp, prm, O.solve_problem(pp, prm, freq, az, want_group=True)


def _check_modes(g, o):
    assert g.M == o.M, (g.M, o.M)
    tol = _k_tol(o.kr, o.dz)
    assert np.all(np.abs(g.kr - o.kr) / o.kr <= tol)
    assert np.allclose(g.ki, o.ki, rtol=1e-6, atol=1e-18)
    assert np.allclose(g.vs * g.vr, o.vs * o.vr, rtol=1e-6, atol=1e-12 * np.abs(o.vs * o.vr).max())


@pytest.mark.parametrize("freq,az,nowkb", [(0.1, 90.0, False), (0.1, 90.0, True), (0.37, 45.0, True)])
def test_single_problem_vs_oracle(gpu, analytic_profile, freq, az, nowkb):
    import ncpa_gpu

    O, pp, prm, o = _oracle_modes(analytic_profile, freq, az, turnoff_WKB=nowkb)
    prof = gpu.load_profile(analytic_profile)
    modes = gpu.solve(prof, ncpa_gpu.default_params(turnoff_wkb=int(nowkb), want_group_speed=1), [freq], [az])
    g = modes.problem(0)
    assert abs(g.k_min - o.k_min) <= 1e-14 * o.k_min
    assert abs(g.k_max - o.k_max) <= 1e-14 * o.k_max
    _check_modes(g, o)
    # group speeds
    assert np.allclose(g.vg, o.vg, rtol=1e-6)
    # 1-D TL, 1000 ranges to 1000 km
    re, im, inc = modes.tl1d(1000, 1000.0)
    ore, oim, oinc = O.tl1d(o, 1000, 1000.0)
    tl_g = 20 * np.log10(np.hypot(re[0], im[0]))
    tl_o = 20 * np.log10(np.hypot(ore, oim))
    mask = tl_o > -140
    assert np.max(np.abs(tl_g - tl_o)[mask]) <= 0.05
    assert np.allclose(inc[0], oinc, rtol=1e-6)
    modes.close()
    prof.close()


def test_batched_broadband_vs_oracle(gpu, analytic_profile):
    """A batch of frequencies (uneven mode counts) in one solve."""
    import ncpa_gpu
    from oracle import oracle as O

    freqs = np.array([0.005, 0.05, 0.12, 0.23, 0.31])
    prof = gpu.load_profile(analytic_profile)
    modes = gpu.solve(prof, ncpa_gpu.default_params(turnoff_wkb=1), freqs, [90.0])
    op = O.read_profile(analytic_profile)
    prm = O.EssParams(turnoff_WKB=True)
    pp = O.prepare(op, prm)
    for i, f in enumerate(freqs):
        _check_modes(modes.problem(i), O.solve_problem(pp, prm, f, 90.0))
    modes.close()
    prof.close()


def test_multi_azimuth_vs_oracle(gpu, canonical_profile):
    import ncpa_gpu
    from oracle import oracle as O

    azs = np.array([0.0, 90.0, 180.0, 270.0, 333.0])
    prof = gpu.load_profile(canonical_profile)
    modes = gpu.solve(prof, ncpa_gpu.default_params(), [0.1], azs)
    op = O.read_profile(canonical_profile)
    prm = O.EssParams()
    pp = O.prepare(op, prm)
    for i, a in enumerate(azs):
        _check_modes(modes.problem(i), O.solve_problem(pp, prm, 0.1, a))
    modes.close()
    prof.close()


def test_full_vectors_and_2d_tl(gpu, analytic_profile):
    import ncpa_gpu
    from oracle import oracle as O

    nz = 4000
    prof = gpu.load_profile(analytic_profile)
    modes = gpu.solve(prof, ncpa_gpu.default_params(nz_grid=nz, turnoff_wkb=1, want_vectors=1), [0.05], [90.0])
    g = modes.problem(0)
    V = modes.vectors(0, nz)
    op = O.read_profile(analytic_profile)
    prm = O.EssParams(Nz_grid=nz, turnoff_WKB=True)
    pp = O.prepare(op, prm)
    o = O.solve_problem(pp, prm, 0.05, 90.0, want_full=True)
    assert g.M == o.M
    # columns agree up to sign
    for m in range(o.M):
        a, b = V[:, m], o.vfull[:, m]
        s = np.sign(np.dot(a, b))
        assert np.max(np.abs(a - s * b)) <= 1e-6 * np.max(np.abs(b))
    # normalisation sum v^2 dz = 1
    assert np.allclose((V ** 2).sum(axis=0) * g.dz, 1.0, rtol=1e-9)
    z, re, im = modes.tl2d(0, 50, 2000.0)
    stepj = nz // 500
    vz = o.vfull[::stepj]
    ore, oim = np.empty((50, len(vz))), np.empty((50, len(vz)))
    O.lib().orc_tl2d(o.M, O._p(O._f64(o.kr)), O._p(O._f64(o.ki)), O._p(O._f64(o.vfull[o.isrc])),
                     O._p(O._f64(vz)), len(vz), 50, 2000.0, 0, O._p(ore), O._p(oim))
    amp_o = np.hypot(ore, oim)
    amp_g = np.hypot(re, im)
    mask = amp_o > 1e-7 * amp_o.max()
    tl_d = np.abs(20 * np.log10(amp_g[mask]) - 20 * np.log10(amp_o[mask]))
    assert tl_d.max() <= 0.05
    modes.close()
    prof.close()
