"""The oracle's eigen-solve against LAPACK on the matrix the reference
assembles (EigenEngine.cpp:57-83: off-diagonal 1/h^2, row 0 carries the
ground condition, the last row repeats diag[n-2]).

dstebz (bisection) gives the eigenvalues in [k_min^2, k_max^2] and dstein
(inverse iteration) the eigenvectors.  Mode counts must be identical;
eigenvalues agree to 16 eps |A| (|A| ~ 4/h^2, the accuracy class of both
methods); V_s V_r and the attenuation integral to 1e-6 relative.
"""
import numpy as np
import pytest
from scipy.linalg import lapack


def _assemble(ms_s, dz):
    h2 = dz * dz
    d = (ms_s + 2.0) / h2 - 2.0 / h2  # diagonal of A from S = h^2 A
    e = np.full(len(d) - 1, 1.0 / h2)
    return d, e


@pytest.mark.parametrize("freq,az,prof", [(0.05, 90.0, "analytic"), (0.2, 270.0, "analytic"),
                                          (0.1, 90.0, "canonical")])
def test_against_dstebz_dstein(freq, az, prof, analytic_profile, canonical_profile):
    from oracle import oracle as O

    path = analytic_profile if prof == "analytic" else canonical_profile
    prm = O.EssParams(Nz_grid=8000, turnoff_WKB=True)
    pp = O.prepare(O.read_profile(path), prm)
    ms = O.solve_problem(pp, prm, freq, az, keep_matrix=True)
    dz = ms.dz
    d, e = _assemble(ms.s, dz)
    lo, hi = ms.k_min ** 2, ms.k_max ** 2
    m, w, iblock, isplit, info = lapack.dstebz(d, e, 1, lo, hi, 0, 0, 0.0, "E")
    assert info == 0
    assert m == ms.M
    lam = np.sort(w[:m])
    normA = 4.0 / dz ** 2
    assert np.max(np.abs(ms.mu / dz ** 2 - lam)) <= 16 * np.finfo(float).eps * normA
    z, info = lapack.dstein(d, e, w[:m], iblock, isplit)
    assert info == 0
    order = np.argsort(w[:m])
    z = z[:, order] / np.sqrt(dz)
    vs, vr = z[ms.isrc], z[ms.ircv]
    assert np.allclose(ms.vs * ms.vr, vs * vr, rtol=1e-6, atol=1e-9 * np.max(np.abs(vs * vr)))
    # perturbative attenuation sum dz v^2 w
    absorb = (z ** 2 * ms.w[:, None]).sum(axis=0) * dz
    kk = (np.sqrt(ms.mu / dz ** 2)) ** 2
    kp = np.sqrt(kk + 1j * absorb)
    assert np.allclose(ms.ki, kp.imag, rtol=1e-6)
