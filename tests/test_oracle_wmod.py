"""The WMod (wide-angle) restatement of the oracle.

- Against the reference's shipped WMod output: wtloss_1d.nm of
  `WMod --singleprop --azimuth 90 --freq 0.1 --write_2d_tloss` on the
  canonical profile (tests/golden/wmod_tloss_1d.npz, pre-2.0.1 scaling:
  +60 dB, as for the Modess golden).
- Against a dense solve of the reference's own linearisation: the 2N pencil
  A x = k B x of EigenEngine::doWideAngleCalculation (EigenEngine.cpp:
  226-296) solved by QZ on coarse grids; the Sturm counts in k must find
  exactly its real eigenvalues inside the window, to round-off.
"""
import os

import numpy as np
import pytest
import scipy.linalg as sl

from conftest import GOLDEN


def test_wmod_tl_against_the_reference_output(canonical_profile):
    from oracle import oracle as O

    g = np.load(os.path.join(GOLDEN, "wmod_tloss_1d.npz"))["lossy"]
    prm = O.EssParams(forces_no_wkb=True)  # --write_2d_tloss turns the WKB cut off
    ms = O.solve_problem_wmod(O.prepare(O.read_profile(canonical_profile), prm), prm, 0.1, 90.0)
    assert ms.M == 62
    re, im, inc = O.tl1d(ms, 1000, 1000.0)
    d = np.abs(20 * np.log10(np.hypot(re, im)) - (20 * np.log10(np.hypot(g[:, 1], g[:, 2])) + 60.0))
    assert np.median(d) < 0.02
    assert np.percentile(d, 90) < 0.2
    di = np.abs(20 * np.log10(inc) - (20 * np.log10(g[:, 3]) + 60.0))
    assert di.max() < 0.02


def _bisect_unperturbed(O, ms, j, nz):
    """Eigenvalue j (0-based inside the window) by bisection on the counts."""
    a2, a1, a0 = ms.coeffs
    L = O.lib()
    c_lo = L.orc_wmod_count(nz, O._p(a2), O._p(a1), O._p(a0), ms.k_min)
    lo, hi = ms.k_min, ms.k_max
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if mid <= lo or mid >= hi:
            break
        if L.orc_wmod_count(nz, O._p(a2), O._p(a1), O._p(a0), mid) > c_lo + j:
            hi = mid
        else:
            lo = mid
    return 0.5 * (lo + hi)


@pytest.mark.parametrize("nz,freq,az", [(400, 0.05, 90.0), (500, 0.08, 270.0), (450, 0.06, 30.0)])
def test_wmod_eigenvalues_against_the_linearised_pencil(canonical_profile, nz, freq, az):
    from oracle import oracle as O

    prm = O.EssParams(Nz_grid=nz, turnoff_WKB=True)
    ms = O.solve_problem_wmod(O.prepare(O.read_profile(canonical_profile), prm), prm, freq, az)
    a2, a1, a0 = ms.coeffs
    h2 = ms.dz ** 2
    M, C = np.diag(a2 / h2), np.diag(a1 / h2)
    D = np.diag(a0 / h2) + np.diag(np.ones(nz - 1) / h2, 1) + np.diag(np.ones(nz - 1) / h2, -1)
    Z = np.zeros((nz, nz))
    ev = sl.eigvals(np.block([[-D, Z], [Z, M]]), np.block([[C, M], [M, Z]]))
    ev = ev[np.isfinite(ev)]
    inw = (ev.real >= ms.k_min) & (ev.real <= ms.k_max)
    real = np.abs(ev.imag) < 1e-9 * np.abs(ev.real)
    assert not np.any(inw & ~real)  # no complex eigenvalue inside the window
    kq = np.sort(ev[inw & real].real)
    assert len(kq) == ms.M > 10
    kb = np.array([_bisect_unperturbed(O, ms, j, nz) for j in range(ms.M)])
    assert np.max(np.abs(kb - kq) / kq) < 1e-10
    # the attenuation perturbation moves Re k by far less than the mode spacing
    assert np.max(np.abs(ms.kr - kb) / kb) < 1e-4
