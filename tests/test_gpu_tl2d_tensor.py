"""The 2-D transmission loss (ncpa_tl_2d, the front ends' tloss_2d.nm) on the
guarded tcgen05 modal sum (NCPA_TL2D_SUM=3) against the FP64 CUDA-core sum
and the CPU oracle.  The guarded sum recomputes in FP64 every point whose
|P| falls below its error bound, so |dTL| <= 0.05 dB must hold wherever
TL > -140 dB (ModeSolver.cpp:492-565 sums in FP64 on the CPU)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ctx(env):
    import ncpa_gpu

    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        return ncpa_gpu.Context(0)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _tl_db(re, im):
    return 20 * np.log10(np.maximum(np.hypot(re, im), 1e-300))


@pytest.mark.parametrize("freq,nz,n_ranges,dr", [(0.05, 4000, 50, 2000.0), (0.5, 20000, 1500, 500.0)])
def test_tl2d_guarded_tensor_sum(analytic_profile, freq, nz, n_ranges, dr):
    import ncpa_gpu

    out = {}
    for name, env in (("fp64", {}), ("tc", {"NCPA_TL2D_SUM": "3"})):
        ctx = _ctx(env)
        prof = ctx.load_profile(analytic_profile)
        m = ctx.solve(prof, ncpa_gpu.default_params(nz_grid=nz, turnoff_wkb=1, want_vectors=1), [freq], [90.0])
        z, re, im = m.tl2d(0, n_ranges, dr)
        out[name] = (z, re, im, m.problem(0).M, ctx.sum_guard() if name == "tc" else None)
        m.close()
        prof.close()
        ctx.close()
    z0, re0, im0, M0, _ = out["fp64"]
    z1, re1, im1, M1, guard = out["tc"]
    assert M0 == M1 and M0 > 0
    assert np.array_equal(z0, z1)
    assert re1.shape == re0.shape == (n_ranges, len(z0))
    tl0, tl1 = _tl_db(re0, im0), _tl_db(re1, im1)
    # heights above the duct lie below -140 dB at the top of the band
    mask = tl0 > -140.0
    assert mask.mean() > 0.5
    d = np.abs(tl1 - tl0)[mask]
    assert d.max() <= 0.05, (d.max(), np.median(d))
    eps, tau, _ = guard
    assert 0 < eps < tau


def test_tl2d_guarded_tensor_sum_against_oracle(analytic_profile):
    import ncpa_gpu
    from oracle import oracle as O

    nz, freq, nr, dr = 4000, 0.05, 50, 2000.0
    ctx = _ctx({"NCPA_TL2D_SUM": "3"})
    prof = ctx.load_profile(analytic_profile)
    m = ctx.solve(prof, ncpa_gpu.default_params(nz_grid=nz, turnoff_wkb=1, want_vectors=1), [freq], [90.0])
    z, re, im = m.tl2d(0, nr, dr)
    M = m.problem(0).M
    m.close()
    prof.close()
    ctx.close()
    prm = O.EssParams(Nz_grid=nz, turnoff_WKB=True)
    o = O.solve_problem(O.prepare(O.read_profile(analytic_profile), prm), prm, freq, 90.0, want_full=True)
    assert M == o.M
    stepj = nz // 500
    vz = o.vfull[::stepj]
    ore, oim = np.empty((nr, len(vz))), np.empty((nr, len(vz)))
    O.lib().orc_tl2d(o.M, O._p(O._f64(o.kr)), O._p(O._f64(o.ki)), O._p(O._f64(o.vfull[o.isrc])),
                     O._p(O._f64(vz)), len(vz), nr, dr, 0, O._p(ore), O._p(oim))
    tl_o = _tl_db(ore, oim)
    mask = tl_o > -140.0
    d = np.abs(_tl_db(re, im) - tl_o)[mask]
    assert d.max() <= 0.05, d.max()
