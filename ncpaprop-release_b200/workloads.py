"""Synthetic inputs for the ESS normal-mode path.

The analytic stratified atmosphere used by the benchmark workloads (no public
dataset is involved): z = 0-150 km every 0.1 km, temperature piecewise linear
(288 K at 0 km, 217 K at 11-20 km, 271 K at 50 km, 187 K at 90 km, 700 K at
150 km), zonal wind 60 exp(-((z-60)/10)^2) + 20 exp(-((z-12)/3)^2) m/s, no
meridional wind, rho = 1.225 exp(-z/7 km) kg/m^3, p = rho 287 T.  Written in
the NCPA profile format the Modess/ModBB command lines read.

Also the source waveform of the broadband workload: a Gaussian-windowed
0.1 Hz Ricker pulse sampled at 1 Hz.
"""
from __future__ import annotations

import numpy as np

T_KNOTS_KM = np.array([0.0, 11.0, 20.0, 50.0, 90.0, 150.0])
T_KNOTS_K = np.array([288.0, 217.0, 217.0, 271.0, 187.0, 700.0])


def analytic_profile(top_km=150.0, dz_km=0.1, t_above_150="extend"):
    """Knot arrays (z km, u, v m/s, T K, rho kg/m3, p Pa).

    Above 150 km (only used by the tall-atmosphere workload) the temperature
    keeps the 90-150 km slope when ``t_above_150 == "extend"`` or is held at
    700 K when ``"hold"``.
    """
    n = int(round(top_km / dz_km)) + 1
    z = np.round(np.arange(n) * dz_km, 10)
    T = np.interp(z, T_KNOTS_KM, T_KNOTS_K)
    hi = z > 150.0
    if np.any(hi):
        slope = (700.0 - 187.0) / 60.0
        T[hi] = 700.0 + slope * (z[hi] - 150.0) if t_above_150 == "extend" else 700.0
    u = 60.0 * np.exp(-((z - 60.0) / 10.0) ** 2) + 20.0 * np.exp(-((z - 12.0) / 3.0) ** 2)
    v = np.zeros_like(z)
    rho = 1.225 * np.exp(-z / 7.0)
    p = rho * 287.0 * T
    return z, u, v, T, rho, p


def write_profile(path, top_km=150.0, dz_km=0.1, t_above_150="extend"):
    z, u, v, T, rho, p = analytic_profile(top_km, dz_km, t_above_150)
    with open(path, "w") as f:
        f.write("#% 0, Z0, m, 0.0\n#% 1, Z, km\n#% 2, U, m/s\n#% 3, V, m/s\n#% 4, T, K\n"
                "#% 5, RHO, kg/m3\n#% 6, P, Pa\n")
        for row in zip(z, u, v, T, rho, p):
            f.write(" ".join("%.12e" % x for x in row) + "\n")
    return path


def si_arrays(top_km=150.0, dz_km=0.1, t_above_150="extend"):
    """Same profile as SI knot arrays (z in m) for ncpa_profile_create."""
    z, u, v, T, rho, p = analytic_profile(top_km, dz_km, t_above_150)
    return z * 1000.0, u, v, T, p, rho


def ricker_waveform(f0=0.1, dt=1.0, n=256, t_center=30.0, sigma=40.0):
    """Gaussian-windowed Ricker pulse (time s, amplitude)."""
    t = np.arange(n) * dt
    a = (np.pi * f0 * (t - t_center)) ** 2
    x = (1.0 - 2.0 * a) * np.exp(-a) * np.exp(-0.5 * ((t - t_center) / sigma) ** 2)
    return t, x


def write_waveform(path, **kw):
    t, x = ricker_waveform(**kw)
    with open(path, "w") as f:
        for a, b in zip(t, x):
            f.write("%12.6f %15.6e\n" % (a, b))
    return path


def broadband_freqs(n=256, f_max=0.5):
    """f_min = f_step = f_max / n, n frequencies (Nfreq rule of
    ESSModeSolver.cpp:109)."""
    df = f_max / n
    nf = int(np.floor((f_max - df) / df)) + 1
    return df + np.arange(nf) * df


# ---------------------------------------------------------------------------
# azimuth sweep (one batch of mixed grid sizes)
# ---------------------------------------------------------------------------
def sweep_freqs(n=8, f_lo=0.1, f_hi=2.0):
    """Frequencies of the azimuth-sweep workload: n log-spaced in [f_lo, f_hi]."""
    return np.exp(np.linspace(np.log(f_lo), np.log(f_hi), n))


def sweep_nz(f, top_km=150.0, c=300.0, points_per_wavelength=60, nz_min=5000):
    """Grid size of the azimuth sweep: points_per_wavelength points per
    wavelength c / f over the atmosphere, at least nz_min.  With the defaults
    Nz runs from 5000 (0.1 Hz, floor) to 60000 (2 Hz)."""
    return max(nz_min, int(np.ceil(points_per_wavelength * top_km * 1000.0 * f / c)))


# ---------------------------------------------------------------------------
# served request stream
# ---------------------------------------------------------------------------
_GP_CHOL = {}


def _gp_factor(z_km, sigma_k=3.0, corr_km=5.0):
    key = (len(z_km), sigma_k, corr_km)
    if key not in _GP_CHOL:
        d = z_km[:, None] - z_km[None, :]
        cov = sigma_k ** 2 * np.exp(-0.5 * (d / corr_km) ** 2)
        cov[np.diag_indices_from(cov)] += 1e-6 * sigma_k ** 2
        _GP_CHOL[key] = np.linalg.cholesky(cov)
    return _GP_CHOL[key]


def perturbed_profile(rng, dz_km=0.1):
    """One served request's atmosphere as SI knot arrays (z m, u, v, T, p, rho):
    the analytic profile with the stratospheric jet's amplitude drawn from
    U(0, 80) m/s at a height from U(40, 70) km, the tropospheric jet's
    amplitude from U(0, 40) m/s, and Gaussian-process temperature noise
    (sigma 3 K, squared-exponential correlation of 5 km, Cholesky factor on the
    knot grid); p = rho 287 T is recomputed."""
    z, _, v, T, rho, _ = analytic_profile(150.0, dz_km)
    a_s, h_s, a_t = rng.uniform(0.0, 80.0), rng.uniform(40.0, 70.0), rng.uniform(0.0, 40.0)
    u = a_s * np.exp(-((z - h_s) / 10.0) ** 2) + a_t * np.exp(-((z - 12.0) / 3.0) ** 2)
    T = T + _gp_factor(z) @ rng.standard_normal(len(z))
    p = rho * 287.0 * T
    return z * 1000.0, u, v, T, p, rho


def request_stream(n, rate_hz, seed=0, dr_m=500.0):
    """n requests with Poisson arrivals at rate_hz: 80 % single frequency
    (log-uniform 0.05-2 Hz), 20 % broadband (32-256 frequencies, uniform
    spacing f_max/n up to 0.5 Hz); azimuth uniform in [0, 360).  Each request
    has its own range grid: dr_m spacing out to a maximum range uniform in
    100-1000 km; broadband requests also ask for pulse waveforms at a third,
    two thirds and all of that range.  Yields dicts with the arrival time [s],
    profile arrays, frequencies, azimuth, n_ranges and wave_ranges_m (None for
    single frequencies).  The grids come from a second generator, so the
    other draws are those of the stream without them."""
    rng = np.random.default_rng(seed)
    rng_grid = np.random.default_rng(seed + 7919)
    t = 0.0
    out = []
    for _ in range(n):
        t += rng.exponential(1.0 / rate_hz)
        if rng.uniform() < 0.8:
            freqs = np.array([np.exp(rng.uniform(np.log(0.05), np.log(2.0)))])
        else:
            nf = int(rng.integers(32, 257))
            freqs = 0.5 / nf * np.arange(1, nf + 1)
        az = rng.uniform(0.0, 360.0)
        r_max = rng_grid.uniform(100e3, 1000e3)
        nr = max(1, int(round(r_max / dr_m)))
        waves = np.array([1.0, 2.0, 3.0]) * (nr * dr_m / 3.0) if len(freqs) > 1 else None
        out.append({"t": t, "profile": perturbed_profile(rng), "freqs": freqs, "az": az, "n_ranges": nr,
                    "wave_ranges_m": waves})
    return out
