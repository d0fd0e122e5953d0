"""Unit checks of the oracle's building blocks against independent Python
restatements: Steffen (1990) monotone cubic, Sutherland-Bass absorption
(src/atmosphere/AtmosphericModel.cpp:86-219) and the profile reader
(src/atmosphere/Atmosphere1D.cpp:85-285)."""
import math
import os

import numpy as np
import pytest


def _steffen_py(x, y, xq):
    n = len(x)
    h = np.diff(x)
    s = np.diff(y) / h
    yp = np.empty(n)
    yp[0], yp[-1] = s[0], s[-1]
    for i in range(1, n - 1):
        p = (s[i - 1] * h[i] + s[i] * h[i - 1]) / (h[i - 1] + h[i])
        sg = (1.0 if s[i - 1] >= 0 else -1.0) + (1.0 if s[i] >= 0 else -1.0)
        yp[i] = sg * min(abs(s[i - 1]), abs(s[i]), 0.5 * abs(p))
    out = []
    for q in xq:
        if q > x[-1]:
            out.append(y[-1]); continue
        if q < x[0]:
            out.append(y[0]); continue
        i = min(max(np.searchsorted(x, q, side="right") - 1, 0), n - 2)
        t = q - x[i]
        a = (yp[i] + yp[i + 1] - 2 * s[i]) / h[i] ** 2
        b = (3 * s[i] - 2 * yp[i] - yp[i + 1]) / h[i]
        out.append(y[i] + t * (yp[i] + t * (b + t * a)))
    return np.array(out)


def test_steffen_matches_restatement_and_is_monotone():
    from oracle import oracle as O

    rng = np.random.default_rng(7)
    x = np.cumsum(rng.uniform(0.5, 2.0, 40))
    y = np.cumsum(rng.uniform(0.0, 1.0, 40))  # monotone data
    sp = O.Spline(x, y)
    xq = np.linspace(x[0] - 1, x[-1] + 1, 2001)
    v = sp(xq)
    assert np.allclose(v, _steffen_py(x, y, xq), rtol=1e-13, atol=1e-13)
    inside = (xq >= x[0]) & (xq <= x[-1])
    assert np.all(np.diff(v[inside]) >= -1e-12)  # no overshoot on monotone data
    assert np.allclose(sp(x), y, rtol=1e-14)
    lin = O.Spline(x, 3.0 * x + 1.0)
    assert np.allclose(lin(xq[inside]), 3.0 * xq[inside] + 1.0, rtol=1e-13)


def _sb_py(z, T, P, D, f):
    PI = 3.141592653589793
    mu_o, T_o, P_o, S = 18.192e-6, 293.15, 101325.0, 117.0
    c = math.sqrt(1.4 * P / D)
    mu = mu_o * math.sqrt(T / T_o) * ((1 + S / T_o) / (1 + S / T))
    nu = 8 * PI * f * mu / (3 * P)
    X = [0.0] * 7
    X[0] = 10 ** (49.296 - 1.5524 * z + 1.8714e-2 * z**2 - 1.1069e-4 * z**3 + 3.199e-7 * z**4
                  - 3.6211e-10 * z**5) if z > 90 else 10 ** -0.67887
    X[1] = 10 ** (1.3972e-1 - 5.6269e-3 * z + 3.9407e-5 * z**2 - 1.0737e-7 * z**3) if z > 76 else 10 ** -0.10744
    X[2] = 10 ** -3.3979
    X[3] = 10 ** (-4.234 - 3.0975e-2 * z) if z > 80 else 10 ** (-19.027 + 1.3093 * z - 4.6496e-2 * z**2
                                                                  + 7.8543e-4 * z**3 - 6.5169e-6 * z**4
                                                                  + 2.1343e-8 * z**5)
    X[4] = 10 ** (-3.2456 + 4.6642e-2 * z - 2.6894e-4 * z**2 + 5.264e-7 * z**3) if z > 95 else \
        10 ** (-11.195 + 1.5408e-1 * z - 1.4348e-3 * z**2 + 1.0166e-5 * z**3)
    X[5] = 10 ** (-53.746 + 1.5439 * z - 1.8824e-2 * z**2 + 1.1587e-4 * z**3 - 3.5399e-7 * z**4
                  + 4.2609e-10 * z**5)
    X[6] = 10 ** (-4.2563 + 7.6245e-2 * z - 2.1824e-3 * z**2 - 2.3010e-6 * z**3 + 2.4265e-7 * z**4
                  - 1.25e-9 * z**5) if z > 30 else 10 ** (-1.7491 + 4.4986e-2 * z - 6.8549e-2 * z**2
                                                           + 5.4639e-3 * z**3 - 1.5539e-4 * z**4
                                                           + 1.5063e-6 * z**5)
    XON = (X[0] + X[1]) / 0.9903
    Zr = 1 / (X[1] / (63.3 * math.exp(-16.7 * T ** (-1 / 3))) + X[0] / (54.1 * math.exp(-17.3 * T ** (-1 / 3))))
    sigma = 5 / math.sqrt(21)
    chi = 3 * (0.8 * math.sqrt(3 / 7) * Zr) * nu / 4
    cchi = 2.36 * chi
    k0 = 2 * PI * f / c
    a_cl = k0 * math.sqrt(0.5 * (math.sqrt(1 + nu**2) - 1) * (1 + cchi**2) / ((1 + nu**2) * (1 + (sigma * cchi)**2)))
    a_rot = k0 * XON * ((sigma**2 - 1) * chi / (2 * sigma)) * math.sqrt(
        0.5 * (math.sqrt(1 + nu**2) + 1) / ((1 + nu**2) * (1 + cchi**2)))
    Tr = (T / T_o) ** (-1 / 3) - 1
    A1 = (X[0] + X[1]) * 24 * math.exp(-9.16 * Tr)
    A2 = (X[4] + X[5]) * 2400
    B = 40400 * math.exp(10 * Tr)
    C = 0.02 * math.exp(-11.2 * Tr)
    Dd = 0.391 * math.exp(8.41 * Tr)
    E = 9 * math.exp(-19.9 * Tr)
    G = 28000 * math.exp(-4.17 * Tr)
    ZZ = 22000 * math.exp(-7.68 * Tr) * X[2] + 15100 * math.exp(-10.4 * Tr) * (X[0] + 0.5 * X[4]) + \
        11500 * math.exp(-9.17 * Tr) * (X[1] + 0.5 * X[5]) + 8.48e8 * math.exp(9.17 * Tr) * (X[6] + X[3])
    hu = 100 * (X[3] + X[6])
    pf = (P / P_o) * (mu_o / mu)
    fv = [pf * (A1 + A2 + B * hu * (C + hu) * (Dd + hu)), pf * (E + 60000 * X[3] + G * X[6]), pf * ZZ,
          pf * 1.2e5 * math.exp(-7.72 * Tr)]
    th, cv, cp = [2239.1, 3352.0, 915.0, 1037.0], [2.5, 2.5, 3, 3], [3.5, 3.5, 4, 4]
    a_vib = 0
    for m in range(4):
        CR = (th[m] / T) ** 2 * math.exp(-th[m] / T) / (1 - math.exp(-th[m] / T)) ** 2
        Am = X[m] * (PI / 2) * CR / (cp[m] * (cv[m] + CR))
        a_vib += (Am / c) * ((2 * f**2 / fv[m]) / (1 + (f / fv[m]) ** 2))
    return a_cl + a_rot + 0.003 * a_cl + a_vib


@pytest.mark.parametrize("z,T,f", [(0.0, 288.0, 0.1), (35.0, 240.0, 0.5), (85.0, 190.0, 1.0), (120.0, 400.0, 0.05)])
def test_sutherland_bass(z, T, f):
    from oracle import oracle as O

    D = 1.225 * math.exp(-z / 7.0)
    P = D * 287.0 * T
    a = O.lib().orc_attn_sutherland_bass(z, T, P, D, f)
    assert a > 0
    assert a == pytest.approx(_sb_py(z, T, P, D, f), rel=1e-12)


def test_profile_reader_units(tmp_path):
    from oracle import oracle as O

    p = tmp_path / "p.dat"
    p.write_text("#% 0, Z0, km, 0.5\n#% 1, Z, km\n#% 2, U, km/s\n#% 3, V, m/s\n#% 4, T, degC\n"
                 "#% 5, RHO, g/cm3\n#% 6, P, mbar\n# a comment\n\n"
                 "0 0.001 1 15 1.2e-3 1000\n1, 0.002, 2, 10, 1.1e-3, 900\n2\t0.003\t3\t5\t1.0e-3\t800\n")
    prof = O.read_profile(str(p))
    assert prof.z_units == "km"
    assert prof.scalars["Z0"] == (0.5, "km")
    pp = O.prepare(prof, O.EssParams(Nz_grid=10, maxheight_km=2.0))
    assert np.allclose(pp.U, [1.0, 2.0, 3.0])
    assert np.allclose(pp.T, [288.15, 283.15, 278.15])
    assert np.allclose(pp.RHO, [1.2, 1.1, 1.0])
    assert np.allclose(pp.P, [1e5, 9e4, 8e4])
    assert pp.z_min == 500.0                 # raised to Z0
    assert pp.maxheight == 2000.0 - 1e-6     # clamped below the profile top


@pytest.mark.parametrize("text,err", [
    ("#% 1, Z, km\n#% 2, U, furlongs\n0 1\n", "Unrecognized units"),
    ("#% 1, Z, km\n#% 2, U, m/s\n#% 2, U, m/s\n0 1\n", "not unique"),
    ("#% 1, Z, km\n#% 2, U, m/s\n0 1 2\n", "columns expected"),
    ("0 1\n", "No descriptive fields"),
])
def test_profile_reader_errors(tmp_path, text, err):
    from oracle import oracle as O

    p = tmp_path / "bad.dat"
    p.write_text(text)
    with pytest.raises(Exception, match=err):
        O.read_profile(str(p))
