"""A G2S-style profile on the device: loaded directly, and through its NCPA
conversion, gives the same modes bit for bit, and the oracle's modes on the
converted file (counts identical, Re k within the parity bound)."""
import gzip
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

EPS = np.finfo(float).eps


def test_g2s_profile_solves_like_its_ncpa_conversion(gpu, tmp_path):
    import ncpa_gpu
    from oracle import oracle as O

    src = tmp_path / "g2sprofile.sample"
    with gzip.open(os.path.join(GOLDEN, "g2s_profile.sample.gz"), "rb") as fi:
        src.write_bytes(fi.read())
    conv = tmp_path / "converted.dat"
    ncpa_gpu.g2s_convert(src, conv)
    prm = ncpa_gpu.default_params(nz_grid=8000, turnoff_wkb=1)
    a = gpu.load_profile_g2s(src)
    b = gpu.load_profile(conv)
    ma = gpu.solve(a, prm, [0.1, 0.3], [90.0, 200.0])
    mb = gpu.solve(b, prm, [0.1, 0.3], [90.0, 200.0])
    for p in range(ma.P):
        x, y = ma.problem(p), mb.problem(p)
        assert x.M == y.M > 0
        for k in ("kr", "ki", "vs", "vr"):
            assert np.array_equal(getattr(x, k), getattr(y, k)), (p, k)
    oprm = O.EssParams(Nz_grid=8000, turnoff_WKB=True)
    pp = O.prepare(O.read_profile(str(conv)), oprm)
    o = O.solve_problem(pp, oprm, 0.1, 90.0)
    g = ma.problem(0)
    assert g.M == o.M
    tol = np.maximum(1e-9, 8 * EPS * (4.0 / o.dz ** 2) / (2 * o.kr ** 2))
    assert np.all(np.abs(g.kr - o.kr) / o.kr <= tol)
    for h in (ma, mb, a, b):
        h.close()
