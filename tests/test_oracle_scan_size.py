"""The estimate that sizes the isolation scan (k_scan_size): the number of
eigenvalues of S (diagonal s_i, unit off-diagonals) below x is close to
sum_i theta_i / pi with cos theta_i = (s_i - x) / 2 clipped to [-1, 1], so
the mode count in the window [lo, hi] is about the difference at hi and lo.
Here the same formula (single precision after the FP64 difference, as the
kernel evaluates it) on the oracle's matrices, against the oracle's Sturm
counts (the reference's mode numbers): within one mode across the benchmark's
band.  The estimate only sizes the scan; the mode counts themselves always
come from the sequential Sturm counts."""
import ctypes
import math
import os

import numpy as np
import pytest


def _matrix(O, pp, prm, f, az=90.0):
    L = O.lib()
    ceffk = np.empty_like(pp.zk)
    L.orc_ceff_knots(len(pp.zk), O._p(pp.c0), O._p(pp.ws), O._p(pp.wd), float(az), O._p(ceffk))
    sp = O.Spline(pp.zk, ceffk)
    nz = prm.Nz_grid
    gp = O._GridParams(nz, pp.z_min, pp.dz_grid, pp.dz, f, pp.admittance, prm.sourceheight_km * 1000.0,
                       prm.receiverheight_km * 1000.0, 1, int(prm.wvnum_filter), prm.c_min, prm.c_max)
    hgt, ceff, diag, s = (np.empty(nz) for _ in range(4))
    res = O._GridResult()
    L.orc_build_grid(ctypes.byref(gp), len(pp.zk), O._p(pp.zk), O._p(ceffk), O._p(sp.coef), O._p(hgt), O._p(ceff),
                     O._p(diag), O._p(s), ctypes.byref(res))
    h2 = pp.dz * pp.dz
    return s, res.k_min ** 2 * h2, res.k_max ** 2 * h2


def _estimate(s, lo, hi):
    ch = np.clip(((s - hi) * 0.5).astype(np.float32), -1, 1)
    cl = np.clip(((s - lo) * 0.5).astype(np.float32), -1, 1)
    return max(float(np.sum(np.arccos(ch) - np.arccos(cl), dtype=np.float64)) / math.pi, 0.0)


@pytest.mark.parametrize("f", [0.002, 0.02, 0.08, 0.16, 0.25, 0.35, 0.43, 0.5])
def test_mode_count_estimate_within_one_mode(workdir, f):
    import workloads
    from oracle import oracle as O

    path = workloads.write_profile(os.path.join(str(workdir), "analytic_150km.dat"))
    prm = O.EssParams(Nz_grid=20000, turnoff_WKB=True)
    pp = O.prepare(O.read_profile(path), prm)
    s, lo, hi = _matrix(O, pp, prm, f)
    L = O.lib()
    m = L.orc_sturm_count(len(s), O._p(s), hi) - L.orc_sturm_count(len(s), O._p(s), lo)
    est = _estimate(s, lo, hi)
    assert abs(est - m) <= 1.0, (f, m, est)
