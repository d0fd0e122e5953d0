"""Wide-angle (WMod) normal modes on the GPU (C ABI, method = WMod) against
the oracle's restatement of WModeSolver::solve (WModeSolver.cpp:257-486) and
against the reference's shipped WMod output.

Tolerances as for the ESS path: mode counts identical; Re k within
max(1e-9, 8 eps |T h^2| / (2 k^2 h^2)) relative (the conditioning floor of
the finite-difference quadratic eigenproblem); Im k and V_s V_r 1e-6
relative; TL within 0.05 dB wherever TL > -140 dB.  Modes are ordered by
ascending Re k on both sides (the reference keeps SLEPc's convergence order,
WModeSolver.cpp:491-509, which no sum depends on).
"""
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

EPS = np.finfo(float).eps


def _k_tol(k, dz):
    return np.maximum(1e-9, 8 * EPS * (4.0 / dz ** 2) / (2 * k ** 2))


def _check_modes(g, o):
    assert g.M == o.M, (g.M, o.M)
    assert np.all(np.abs(g.kr - o.kr) / o.kr <= _k_tol(o.kr, o.dz))
    assert np.allclose(g.ki, o.ki, rtol=1e-6, atol=1e-18)
    assert np.allclose(g.vs * g.vr, o.vs * o.vr, rtol=1e-6, atol=1e-12 * np.abs(o.vs * o.vr).max())


def _check_tl(re_, im_, ms, nr, dr):
    from oracle import oracle as O

    ore, oim, _ = O.tl1d(ms, nr, dr)
    tl_g = 20 * np.log10(np.hypot(re_, im_))
    tl_o = 20 * np.log10(np.hypot(ore, oim))
    mask = tl_o > -140
    assert mask.sum() > nr // 2
    assert np.max(np.abs(tl_g - tl_o)[mask]) <= 0.05


def _wmod(**kw):
    import ncpa_gpu

    return ncpa_gpu.default_params(method=ncpa_gpu.METHOD_WMOD, **kw)


@pytest.mark.parametrize("freq,az,nowkb", [(0.1, 90.0, True), (0.1, 90.0, False), (0.25, 270.0, True)])
def test_single_problem_vs_oracle(gpu, canonical_profile, freq, az, nowkb):
    from oracle import oracle as O

    prm = O.EssParams(turnoff_WKB=nowkb)
    o = O.solve_problem_wmod(O.prepare(O.read_profile(canonical_profile), prm), prm, freq, az)
    prof = gpu.load_profile(canonical_profile)
    modes = gpu.solve(prof, _wmod(turnoff_wkb=int(nowkb)), [freq], [az])
    g = modes.problem(0)
    assert abs(g.k_min - o.k_min) <= 1e-14 * o.k_min
    assert abs(g.k_max - o.k_max) <= 1e-14 * o.k_max
    _check_modes(g, o)
    re_, im_, _ = modes.tl1d(1000, 1000.0)
    _check_tl(re_[0], im_[0], o, 1000, 1000.0)
    modes.close()
    prof.close()


def test_against_the_reference_output(gpu, canonical_profile):
    """wtloss_1d.nm of `WMod --singleprop --azimuth 90 --freq 0.1
    --write_2d_tloss` (pre-2.0.1 scaling, +60 dB): the GPU path must sit as
    close to it as the oracle does."""
    g = np.load(os.path.join(GOLDEN, "wmod_tloss_1d.npz"))["lossy"]
    prof = gpu.load_profile(canonical_profile)
    modes = gpu.solve(prof, _wmod(turnoff_wkb=1), [0.1], [90.0])
    assert modes.problem(0).M == 62
    re_, im_, inc = modes.tl1d(1000, 1000.0)
    d = np.abs(20 * np.log10(np.hypot(re_[0], im_[0])) - (20 * np.log10(np.hypot(g[:, 1], g[:, 2])) + 60.0))
    assert np.median(d) < 0.02
    assert np.percentile(d, 90) < 0.2
    di = np.abs(20 * np.log10(inc[0]) - (20 * np.log10(g[:, 3]) + 60.0))
    assert di.max() < 0.02
    modes.close()
    prof.close()


def test_batch_of_frequencies_and_azimuths(gpu, analytic_profile):
    """Uneven mode counts in one solve: 4 frequencies x 3 azimuths."""
    from oracle import oracle as O

    freqs = np.array([0.01, 0.07, 0.15, 0.3])
    azs = np.array([0.0, 90.0, 225.0])
    prof = gpu.load_profile(analytic_profile)
    modes = gpu.solve(prof, _wmod(turnoff_wkb=1), freqs, azs)
    prm = O.EssParams(turnoff_WKB=True)
    pp = O.prepare(O.read_profile(analytic_profile), prm)
    counts = modes.counts()
    assert len(set(counts)) > 3
    for fi, f in enumerate(freqs):
        for ai, a in enumerate(azs):
            _check_modes(modes.problem(fi * len(azs) + ai), O.solve_problem_wmod(pp, prm, f, a))
    modes.close()
    prof.close()


def test_eigenvectors_and_normalisation(gpu, canonical_profile):
    """Full vectors: equal to the oracle's up to one sign per mode, and
    sum v^2 dz = 1 / (1 + k^2) (SLEPc's unit-norm vectors of the linearised
    pencil [v; k v], EigenEngine.cpp:368-379)."""
    from oracle import oracle as O

    nz = 4000
    prm = O.EssParams(Nz_grid=nz, turnoff_WKB=True)
    o = O.solve_problem_wmod(O.prepare(O.read_profile(canonical_profile), prm), prm, 0.08, 90.0, want_full=True)
    prof = gpu.load_profile(canonical_profile)
    modes = gpu.solve(prof, _wmod(nz_grid=nz, turnoff_wkb=1, want_vectors=1), [0.08], [90.0])
    g = modes.problem(0)
    _check_modes(g, o)
    v = modes.vectors(0, nz)
    assert v.shape == o.vfull.shape
    for j in range(g.M):
        s = np.sign(np.dot(v[:, j], o.vfull[:, j]))
        assert np.allclose(s * v[:, j], o.vfull[:, j], rtol=0, atol=1e-7 * np.abs(o.vfull[:, j]).max())
        kr = g.kr[j]
        assert np.sum(v[:, j] ** 2) * g.dz == pytest.approx(1.0 / (1.0 + kr * kr), rel=1e-6)
    # the 2-D field runs on these vectors as on the ESS ones
    nzo = modes.tl2d(0, 50, 2000.0)[0].shape[0]
    assert nzo > 0
    modes.close()
    prof.close()


def test_jobs_mixed_grids_match_single_solves(gpu, canonical_profile, analytic_profile):
    """Wide-angle jobs on two profiles and two grids (one with an azimuth
    list) in one ncpa_ess_solve_jobs call: every problem bit-identical to the
    same problem solved alone."""
    pc = gpu.load_profile(canonical_profile)
    pa = gpu.load_profile(analytic_profile)
    m = gpu.solve_jobs([(pc, [0.05, 0.1], 90.0, 4000), (pa, [0.08], [0.0, 200.0], 6000)], _wmod(turnoff_wkb=1))
    s1 = gpu.solve(pc, _wmod(nz_grid=4000, turnoff_wkb=1), [0.05, 0.1], [90.0])
    s2 = gpu.solve(pa, _wmod(nz_grid=6000, turnoff_wkb=1), [0.08], [0.0, 200.0])
    singles = [s1.problem(0), s1.problem(1), s2.problem(0), s2.problem(1)]
    for p, o in enumerate(singles):
        g = m.problem(p)
        assert g.M == o.M > 0
        for f in ("kr", "ki", "vs", "vr"):
            assert np.array_equal(getattr(g, f), getattr(o, f)), (p, f)
        assert g.dz == o.dz
    for h in (m, s1, s2, pc, pa):
        h.close()


def test_plans_reject_wmod(gpu, canonical_profile):
    import ncpa_gpu

    prof = gpu.load_profile(canonical_profile)
    with pytest.raises(ncpa_gpu.NcpaError):
        gpu.plan([(prof, [0.1], 90.0)], _wmod())
    bad = _wmod()
    bad.method = 7
    with pytest.raises(ncpa_gpu.NcpaError):
        gpu.solve(prof, bad, [0.1], [90.0])
    prof.close()


def test_modbb_wmod_dispersion_file(canonical_profile, tmp_path):
    """`ModBB --dispersion --method wmod`: one line per frequency, the
    ESS file format (ModeSolver.cpp:569-589), with the wide-angle modes."""
    import subprocess

    from oracle import oracle as O

    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "ncpaprop-release_b200")
    nz = 6000
    args = ["--dispersion", "--method", "wmod", "--dispersion_file", "wdisp.dat", "--atmosfile", canonical_profile,
            "--azimuth", "90", "--f_min", "0.02", "--f_step", "0.02", "--f_max", "0.1", "--Nz_grid", str(nz)]
    p = subprocess.run([os.path.join(pkg, "bin", "ModBB")] + args, cwd=tmp_path, capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    lines = (tmp_path / "wdisp.dat").read_text().splitlines()
    assert len(lines) == 5
    prm = O.EssParams(Nz_grid=nz, turnoff_WKB=True)
    pp = O.prepare(O.read_profile(canonical_profile), prm)
    for i, ln in enumerate(lines):
        f = 0.02 + i * 0.02
        assert re.match(r"\d\.\d{7}e[+-]\d\d   \d+    \d\.\d{7}e[+-]\d\d   \d\.\d{7}e[+-]\d\d", ln), ln
        toks = ln.split()
        o = O.solve_problem_wmod(pp, prm, f, 90.0)
        assert float(toks[0]) == pytest.approx(f, rel=1e-7) and int(toks[1]) == o.M
        assert float(toks[2]) == pytest.approx(o.rho_s, rel=1e-7)
        v = np.array(toks[4:], dtype=float).reshape(o.M, 4)
        assert np.all(np.abs(v[:, 0] - o.kr) / o.kr <= _k_tol(o.kr, o.dz))
        assert np.allclose(v[:, 2] * v[:, 3], o.vs * o.vr, rtol=1e-6, atol=1e-12 * np.abs(o.vs * o.vr).max())
