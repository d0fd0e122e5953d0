"""CPU oracle driver for the effective-sound-speed normal-mode path.

TEST INFRASTRUCTURE ONLY.  Used as the checker by tests/, by
``__graft_entry__.smoke()`` and as the ``cpu_baseline`` leg of ``bench.py``.
The product library never imports this module.

The numerics live in ``ncpa_oracle.c`` (loaded through ctypes); this file
restates the reference's orchestration:

* profile parsing        src/atmosphere/Atmosphere1D.cpp:85-285
* unit strings           src/common/units.cpp:120-260
* ESSModeSolver setup    src/libmodes/ESSModeSolver.cpp:30-240
* per-problem solve      src/libmodes/ESSModeSolver.cpp:320-466
* dispersion reader      src/libbroadband/ModalBroadbandPropagator.cpp:25-138
* pulse synthesis        src/libbroadband/ModalBroadbandPropagator.cpp:141-242,
                         src/libbroadband/BroadbandPropagator.cpp:244-476
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libncpa_oracle.so")
PI = 3.141592653589793  # src/common/util.h:13-14
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        c_int, c_double = ctypes.c_int, ctypes.c_double
        L.orc_steffen_init.argtypes = [c_int, dp, dp, dp]
        L.orc_spline_get.argtypes = [c_int, dp, dp, dp, c_double]
        L.orc_spline_get.restype = c_double
        L.orc_spline_deriv.argtypes = [c_int, dp, dp, c_double]
        L.orc_spline_deriv.restype = c_double
        L.orc_spline_get_many.argtypes = [c_int, dp, dp, dp, c_int, dp, dp]
        L.orc_attn_sutherland_bass.argtypes = [c_double] * 5
        L.orc_attn_sutherland_bass.restype = c_double
        L.orc_c0_from_p_rho.argtypes = [c_int, dp, dp, dp, dp]
        L.orc_c0_from_t.argtypes = [c_int, dp, dp, dp]
        L.orc_wind_speed_dir.argtypes = [c_int, dp, dp, dp, dp]
        L.orc_ceff_knots.argtypes = [c_int, dp, dp, dp, c_double, dp]
        L.orc_build_grid.argtypes = [ctypes.c_void_p, c_int, dp, dp, dp, dp, dp, dp, dp, ctypes.c_void_p]
        L.orc_sturm_count.argtypes = [c_int, dp, c_double]
        L.orc_sturm_count.restype = c_int
        L.orc_bisect.argtypes = [c_int, dp, c_double, c_double, c_int, c_int, c_double, dp]
        L.orc_eigvec.argtypes = [c_int, dp, c_double, c_double, dp, dp, c_int, c_int, dp, dp]
        L.orc_solve_modes.argtypes = [c_int, dp, c_double, c_double, c_double, c_double, c_double,
                                      dp, dp, c_int, c_int, c_double, c_int, dp, dp, dp, dp, dp, dp]
        L.orc_solve_modes.restype = c_int
        L.orc_wc_knots.argtypes = [c_int, dp, dp, c_double, dp]
        L.orc_wmod_coeffs.argtypes = [c_int, dp, dp, c_double, c_double, c_double, dp, dp, dp]
        L.orc_wmod_count.argtypes = [c_int, dp, dp, dp, c_double]
        L.orc_wmod_count.restype = c_int
        L.orc_wmod_solve.argtypes = [c_int, dp, dp, dp, c_double, c_double, c_double, dp, c_int, c_int, c_double,
                                     c_int, dp, dp, dp, dp, dp]
        L.orc_wmod_solve.restype = c_int
        L.orc_tl1d.argtypes = [c_int, dp, dp, dp, dp, c_int, c_double, c_int, dp, dp, dp]
        L.orc_tl2d.argtypes = [c_int, dp, dp, dp, dp, c_int, c_int, c_double, c_int, dp, dp]
        L.orc_bb_transfer.argtypes = [c_int, ip, dp, dp, dp, dp, c_double, c_double, c_double, dp, dp]
        L.orc_bb_pulse.argtypes = [c_int, dp, dp, dp, dp, dp, c_double, c_int, dp]
        L.orc_dft_source.argtypes = [c_int, dp, c_double, c_int, c_int, dp, dp]
        L.orc_num_threads.restype = c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class _GridParams(ctypes.Structure):
    _fields_ = [("nz", ctypes.c_int), ("z_min", ctypes.c_double), ("dz_grid", ctypes.c_double),
                ("dz", ctypes.c_double), ("freq", ctypes.c_double), ("admittance", ctypes.c_double),
                ("src_h", ctypes.c_double), ("rcv_h", ctypes.c_double), ("turnoff_wkb", ctypes.c_int),
                ("wvnum_filter", ctypes.c_int), ("c_min", ctypes.c_double), ("c_max", ctypes.c_double)]


class _GridResult(ctypes.Structure):
    _fields_ = [("k_min", ctypes.c_double), ("k_max", ctypes.c_double), ("ceffmin", ctypes.c_double),
                ("ceffmax", ctypes.c_double), ("used_wkb", ctypes.c_int)]


# --------------------------------------------------------------------------
# units (src/common/units.cpp:120-260): string -> (kind, factor-to-SI or func)
# --------------------------------------------------------------------------
_UNITS = {}
for _k in ("K", "DEGK", "DEG K", "DEGREES K", "KELVIN"):
    _UNITS[_k] = ("K", None)
for _k in ("C", "DEGC", "DEG C", "DEGREES C", "CELSIUS", "CENTIGRADE"):
    _UNITS[_k] = ("C", None)
for _k in ("F", "DEGF", "DEG F", "DEGREES F", "FAHRENHEIT"):
    _UNITS[_k] = ("F", None)
for _k in ("M", "METERS"):
    _UNITS[_k] = ("m", None)
for _k in ("KM", "KILOMETERS"):
    _UNITS[_k] = ("km", None)
for _k in ("M/S", "MPS", "MPERS", "M PER S", "METERS PER SECOND"):
    _UNITS[_k] = ("m/s", None)
for _k in ("KM/S", "KMPS", "KMPERS", "KM PER S", "KILOMETERS PER SECOND"):
    _UNITS[_k] = ("km/s", None)
for _k in ("PA", "PASCAL", "PASCALS"):
    _UNITS[_k] = ("Pa", None)
for _k in ("MBAR", "MILLIBAR", "MILLIBARS"):
    _UNITS[_k] = ("mbar", None)
for _k in ("HECTOPASCALS", "HPA"):
    _UNITS[_k] = ("hPa", None)
for _k in ("ATMOSPHERES", "ATM"):
    _UNITS[_k] = ("atm", None)
for _k in ("KG/M3", "KGPM3", "KILOGRAMS PER CUBIC METER"):
    _UNITS[_k] = ("kg/m3", None)
for _k in ("G/CM3", "GPCM3", "GRAMS PER CUBIC CENTIMETER"):
    _UNITS[_k] = ("g/cm3", None)
for _k in ("DEG", "DEGREES"):
    _UNITS[_k] = ("deg", None)
for _k in ("RAD", "RADIANS"):
    _UNITS[_k] = ("rad", None)
for _k in ("", "N/A"):
    _UNITS[_k] = ("", None)


def units_from_string(s: str) -> str:
    key = s.upper()
    if key not in _UNITS:
        raise ValueError("Unrecognized units string: " + s)
    return _UNITS[key][0]


def to_si(values, unit: str, target: str):
    """Conversions of units.cpp:132-172 (same operations, same order)."""
    v = np.asarray(values, dtype=np.float64)
    if unit == target:
        return v.copy()
    table = {
        ("km", "m"): lambda x: x * 1000.0,
        ("m", "km"): lambda x: x * 0.001,
        ("km/s", "m/s"): lambda x: x * 1000.0,
        ("mbar", "Pa"): lambda x: x * 100.0,
        ("hPa", "Pa"): lambda x: x * 100,
        ("atm", "Pa"): lambda x: x * 101325.0,
        ("g/cm3", "kg/m3"): lambda x: x * 1000.0,
        ("C", "K"): lambda x: x + 273.15,
        ("F", "K"): lambda x: ((x - 32.0) * 5.0 / 9.0) + 273.15,
    }
    if (unit, target) not in table:
        raise ValueError("no conversion from %s to %s" % (unit, target))
    return table[(unit, target)](v)


# --------------------------------------------------------------------------
# profile parser (Atmosphere1D.cpp:85-285)
# --------------------------------------------------------------------------
def _split(s, delims):
    out, cur = [], []
    for ch in s:
        if ch in delims:
            if cur:
                out.append("".join(cur))
                cur = []
        else:
            cur.append(ch)
    if cur:
        out.append("".join(cur))
    return out


@dataclass
class Profile:
    z: np.ndarray                       # altitude column as read
    z_units: str
    vectors: dict = field(default_factory=dict)   # key -> (values, units)
    scalars: dict = field(default_factory=dict)   # key -> (value, units)


def read_profile(path: str, header_path: str = "") -> Profile:
    hfile = header_path if header_path else path
    headerlines = []
    with open(hfile) as f:
        for line in f:
            line = line.strip()
            if line.startswith("#") and len(line) > 1 and line[1] == "%":
                headerlines.append(line[2:])
    datalines = []
    with open(path) as f:
        for line in f:
            line = line.strip()
            if not line or line.startswith("#"):
                continue
            datalines.append(line)
    if not headerlines:
        raise RuntimeError("Atmosphere1D - No descriptive fields found.")
    cols, keys, units, vals = [], [], [], []
    for h in headerlines:
        fields = _split(h.strip(), " ,")
        if len(fields) not in (3, 4):
            raise ValueError("Atmosphere1D - Error parsing descriptive line: " + h)
        cols.append(int(fields[0]))
        keys.append(fields[1].strip())
        units.append(units_from_string(fields[2].strip()))
        vals.append(float(fields[3]) if len(fields) == 4 else 0.0)
    if len(set(keys)) != len(keys):
        raise ValueError("Atmosphere1D: key values are not unique")
    ncols = max(cols)
    depunits = ""
    for c, u in zip(cols, units):
        if c == 1:
            depunits = u
    data = np.empty((len(datalines), ncols))
    for r, line in enumerate(datalines):
        fields = _split(line, " \t,")
        if len(fields) != ncols:
            raise ValueError("Error parsing data line: %s (%d columns expected, %d found)"
                             % (line, ncols, len(fields)))
        data[r] = [float(x) for x in fields]
    prof = Profile(z=data[:, 0].copy(), z_units=depunits)
    for c, k, u, v in zip(cols, keys, units, vals):
        if c == 0:
            prof.scalars[k] = (v, u)
        elif c > 1:
            prof.vectors[k] = (data[:, c - 1].copy(), u)
    return prof


# --------------------------------------------------------------------------
# spline helper
# --------------------------------------------------------------------------
class Spline:
    def __init__(self, x, y):
        self.x = _f64(x)
        self.y = _f64(y)
        self.n = len(self.x)
        self.coef = np.empty(4 * (self.n - 1))
        lib().orc_steffen_init(self.n, _p(self.x), _p(self.y), _p(self.coef))

    def __call__(self, xq):
        xq = _f64(np.atleast_1d(xq))
        out = np.empty_like(xq)
        lib().orc_spline_get_many(self.n, _p(self.x), _p(self.y), _p(self.coef), len(xq), _p(xq), _p(out))
        return out

    def deriv(self, xq):
        return lib().orc_spline_deriv(self.n, _p(self.x), _p(self.coef), float(xq))


# --------------------------------------------------------------------------
# ESSModeSolver set-up (ESSModeSolver.cpp:30-240)
# --------------------------------------------------------------------------
@dataclass
class EssParams:
    Nz_grid: int = 20000
    maxheight_km: float = 150.0
    zground_km: float = 0.0
    zground_found: bool = False
    sourceheight_km: float = 0.0
    receiverheight_km: float = 0.0
    maxrange_km: float = 1000.0
    Nrng_steps: int = 1000
    Lamb_wave_BC: bool = False
    turnoff_WKB: bool = False
    wvnum_filter: bool = False
    c_min: float = 0.0
    c_max: float = 0.0
    use_attn_file: str = ""
    write_speeds: bool = False
    # any of write_phase_speeds / write_speeds / write_2d_tloss / write_modes /
    # dispersion file forces turnoff_WKB (ESSModeSolver.cpp:78-81)
    forces_no_wkb: bool = False


@dataclass
class Prepared:
    zk: np.ndarray
    c0: np.ndarray
    ws: np.ndarray
    wd: np.ndarray
    T: np.ndarray
    P: np.ndarray
    RHO: np.ndarray
    U: np.ndarray
    V: np.ndarray
    z_min: float
    maxheight: float
    dz_grid: float
    dz: float
    hgt: np.ndarray
    rho_g: np.ndarray
    p_g: np.ndarray
    attn_knots_z_km: np.ndarray
    user_alpha: np.ndarray | None
    admittance: float


def prepare(prof: Profile, prm: EssParams) -> Prepared:
    if prof.z_units not in ("m", "km"):
        raise ValueError("altitude units must be a distance")
    z = to_si(prof.z, prof.z_units, "m")
    vec = {k: v for k, v in prof.vectors.items()}

    def si(key, target):
        vals, u = vec[key]
        return to_si(vals, u, target)

    z_min = prm.zground_km * 1000.0
    maxheight = prm.maxheight_km * 1000.0
    if maxheight >= z[-1]:
        maxheight = z[-1] - 1e-6
    dz_grid = (maxheight - z_min) / (prm.Nz_grid - 1)

    if "C0" in vec:
        c0 = si("C0", "m/s")
        if "T" not in vec:
            sp = Spline(z, c0)
            T = np.array([sp(zz)[0] ** 2 / 1.4 / 287.0 for zz in z])
            vec["T"] = (T, "K")
    elif "P" in vec and "RHO" in vec:
        c0 = np.empty_like(z)
        lib().orc_c0_from_p_rho(len(z), _p(z), _p(_f64(si("P", "Pa"))), _p(_f64(si("RHO", "kg/m3"))), _p(c0))
    elif "T" in vec:
        c0 = np.empty_like(z)
        lib().orc_c0_from_t(len(z), _p(z), _p(_f64(si("T", "K"))), _p(c0))
    else:
        raise RuntimeError("Can't calculate static sound speed, either temperature T or pressure P "
                           "and density RHO missing")
    for key in ("U", "V", "T", "P", "RHO"):
        if key not in vec:
            raise RuntimeError("%s vector not found in atmosphere file" % key)
    U, V = _f64(si("U", "m/s")), _f64(si("V", "m/s"))
    T, P, RHO = _f64(si("T", "K")), _f64(si("P", "Pa")), _f64(si("RHO", "kg/m3"))
    if "Z0" in prof.scalars:
        z0v, z0u = prof.scalars["Z0"]
        z0 = float(to_si(np.array([z0v]), z0u, "m")[0])
        if z_min < z0:
            z_min = z0
    ws, wd = np.empty_like(z), np.empty_like(z)
    lib().orc_wind_speed_dir(len(z), _p(U), _p(V), _p(ws), _p(wd))
    user_alpha = None
    if prm.use_attn_file:
        user_alpha = read_attn_file(prm.use_attn_file, z)
    hgt = z_min + np.arange(prm.Nz_grid) * dz_grid
    dz = (maxheight - z_min) / (prm.Nz_grid - 1)
    sp_rho = Spline(z, RHO)
    admittance = 0.0
    if prm.Lamb_wave_BC:
        admittance = -sp_rho.deriv(z_min) / sp_rho(z_min)[0] / 2.0
    return Prepared(zk=_f64(z), c0=_f64(c0), ws=ws, wd=wd, T=T, P=P, RHO=RHO, U=U, V=V, z_min=z_min,
                    maxheight=maxheight, dz_grid=dz_grid, dz=dz, hgt=_f64(hgt), rho_g=sp_rho(hgt),
                    p_g=Spline(z, P)(hgt), attn_knots_z_km=z * 0.001, user_alpha=user_alpha,
                    admittance=admittance)


def read_attn_file(path, zk_m):
    """Attenuation from a two-column file (height km, Np/m), interpolated onto
    the profile knots (Atmosphere1D.cpp:307-424)."""
    rows = []
    with open(path) as f:
        for line in f:
            line = line.strip()
            if not line or line.startswith("#"):
                continue
            fl = _split(line, " ,")
            if len(fl) != 2:
                raise ValueError("Atmosphere1D - Error parsing attenuation line: " + line)
            rows.append((float(fl[0]), float(fl[1])))
    za = np.array([r[0] for r in rows])
    aa = np.array([r[1] for r in rows])
    zk_km = zk_m * 0.001
    if za[0] > zk_km[0]:
        za = np.concatenate([[zk_km[0]], za])
        aa = np.concatenate([[aa[0]], aa])
    if za[-1] < zk_km[-1]:
        za = np.concatenate([za, [zk_km[-1]]])
        aa = np.concatenate([aa, [aa[-1]]])
    return Spline(za, aa)(zk_km)


def alpha_knots(pp: Prepared, freq: float) -> np.ndarray:
    if pp.user_alpha is not None:
        return pp.user_alpha
    L = lib()
    return np.array([L.orc_attn_sutherland_bass(float(zk), float(t), float(p), float(d), float(freq))
                     for zk, t, p, d in zip(pp.attn_knots_z_km, pp.T, pp.P, pp.RHO)])


@dataclass
class ModeSet:
    freq: float
    az: float
    M: int
    kr: np.ndarray
    ki: np.ndarray
    vs: np.ndarray
    vr: np.ndarray
    vg: np.ndarray | None
    k_min: float
    k_max: float
    rho_s: float
    rho_r: float
    dz: float
    isrc: int
    ircv: int
    mu: np.ndarray | None = None
    s: np.ndarray | None = None
    vfull: np.ndarray | None = None
    ceff: np.ndarray | None = None
    w: np.ndarray | None = None          # attenuation weights on the grid


BISECT_TOL = 1.0e-15  # absolute, in units of the scaled matrix h^2 A


def solve_problem(pp: Prepared, prm: EssParams, freq: float, az: float, want_group=False,
                  want_full=False, keep_matrix=False, max_modes=1 << 20) -> ModeSet:
    L = lib()
    ceffk = np.empty_like(pp.zk)
    L.orc_ceff_knots(len(pp.zk), _p(pp.c0), _p(pp.ws), _p(pp.wd), float(az), _p(ceffk))
    sp = Spline(pp.zk, ceffk)
    nz = prm.Nz_grid
    gp = _GridParams(nz, pp.z_min, pp.dz_grid, pp.dz, freq, pp.admittance, prm.sourceheight_km * 1000.0,
                     prm.receiverheight_km * 1000.0, int(prm.turnoff_WKB or prm.forces_no_wkb),
                     int(prm.wvnum_filter), prm.c_min, prm.c_max)
    hgt, ceff, diag, s = (np.empty(nz) for _ in range(4))
    res = _GridResult()
    L.orc_build_grid(ctypes.byref(gp), len(pp.zk), _p(pp.zk), _p(ceffk), _p(sp.coef), _p(hgt), _p(ceff),
                     _p(diag), _p(s), ctypes.byref(res))
    omega = 2 * PI * freq
    alpha = Spline(pp.zk, alpha_knots(pp, freq))(pp.hgt)
    cT = np.sqrt(1.4 * pp.p_g / pp.rho_g)
    w = _f64(((omega / cT) * alpha) * 2)
    g = _f64(1.0 / (ceff * ceff)) if want_group else None
    isrc = int(math.ceil(prm.sourceheight_km * 1000.0 / pp.dz))
    ircv = int(math.ceil(prm.receiverheight_km * 1000.0 / pp.dz))
    h2 = pp.dz * pp.dz
    cap = max_modes
    lo = (res.k_min * res.k_min) * h2
    hi = (res.k_max * res.k_max) * h2
    cap = min(cap, max(0, L.orc_sturm_count(nz, _p(s), hi) - L.orc_sturm_count(nz, _p(s), lo)))
    kr, ki, vs, vr, vg = (np.zeros(max(cap, 1)) for _ in range(5))
    vfull = np.zeros(nz * max(cap, 1)) if want_full else None
    M = L.orc_solve_modes(nz, _p(s), h2, pp.dz, res.k_min, res.k_max, omega, _p(w),
                          _p(g) if g is not None else None, isrc, ircv, BISECT_TOL, cap, _p(kr), _p(ki),
                          _p(vs), _p(vr), _p(vg), _p(vfull) if vfull is not None else None)
    if M < 0:
        raise RuntimeError("too many modes")
    ms = ModeSet(freq=freq, az=az, M=M, kr=kr[:M], ki=ki[:M], vs=vs[:M], vr=vr[:M],
                 vg=vg[:M] if want_group else None, k_min=res.k_min, k_max=res.k_max,
                 rho_s=float(pp.rho_g[isrc]), rho_r=float(pp.rho_g[ircv]), dz=pp.dz, isrc=isrc, ircv=ircv)
    if keep_matrix:
        ms.s = s
        ms.ceff = ceff
        ms.w = w
        lo_c = L.orc_sturm_count(nz, _p(s), lo)
        mu = np.empty(max(M, 1))
        L.orc_bisect(nz, _p(s), lo, hi, lo_c, M, BISECT_TOL, _p(mu))
        ms.mu = mu[:M]
    if want_full:
        ms.vfull = vfull[: nz * M].reshape(nz, M)
    return ms


WMOD_TOL = 1.0e-14  # relative bracket width in k


def solve_problem_wmod(pp: Prepared, prm: EssParams, freq: float, az: float, want_full=False,
                       max_modes=1 << 20) -> ModeSet:
    """One wide-angle (WMod) problem: WModeSolver::solve's grid (matrix
    spacing (maxheight - z_min) / Nz_grid, WModeSolver.cpp:281; sampling as
    setParams, :146-208), window of getModalTrace (:514-629: the ESS window
    on c_eff), the quadratic eigenproblem in k (EigenEngine.cpp:174-395) and
    doPerturb (ModeSolver.cpp:263-284)."""
    L = lib()
    nz = prm.Nz_grid
    dz = (pp.maxheight - pp.z_min) / nz
    ceffk, wck = np.empty_like(pp.zk), np.empty_like(pp.zk)
    L.orc_ceff_knots(len(pp.zk), _p(pp.c0), _p(pp.ws), _p(pp.wd), float(az), _p(ceffk))
    L.orc_wc_knots(len(pp.zk), _p(pp.ws), _p(pp.wd), float(az), _p(wck))
    sp = Spline(pp.zk, ceffk)
    gp = _GridParams(nz, pp.z_min, pp.dz_grid, dz, freq, pp.admittance, prm.sourceheight_km * 1000.0,
                     prm.receiverheight_km * 1000.0, int(prm.turnoff_WKB or prm.forces_no_wkb),
                     int(prm.wvnum_filter), prm.c_min, prm.c_max)
    hgt, ceff, diag, s = (np.empty(nz) for _ in range(4))
    res = _GridResult()
    L.orc_build_grid(ctypes.byref(gp), len(pp.zk), _p(pp.zk), _p(ceffk), _p(sp.coef), _p(hgt), _p(ceff),
                     _p(diag), _p(s), ctypes.byref(res))
    omega = 2 * PI * freq
    c0g = _f64(Spline(pp.zk, pp.c0)(pp.hgt))
    wcg = _f64(Spline(pp.zk, wck)(pp.hgt))
    a2, a1, a0 = (np.empty(nz) for _ in range(3))
    L.orc_wmod_coeffs(nz, _p(c0g), _p(wcg), omega, dz, pp.admittance, _p(a2), _p(a1), _p(a0))
    alpha = Spline(pp.zk, alpha_knots(pp, freq))(pp.hgt)
    cT = np.sqrt(1.4 * pp.p_g / pp.rho_g)
    w = _f64(((omega / cT) * alpha) * 2)
    isrc = int(math.ceil(prm.sourceheight_km * 1000.0 / dz))
    ircv = int(math.ceil(prm.receiverheight_km * 1000.0 / dz))
    cap = min(max_modes, max(0, L.orc_wmod_count(nz, _p(a2), _p(a1), _p(a0), res.k_max)
                             - L.orc_wmod_count(nz, _p(a2), _p(a1), _p(a0), res.k_min)))
    kr, ki, vs, vr = (np.zeros(max(cap, 1)) for _ in range(4))
    vfull = np.zeros(nz * max(cap, 1)) if want_full else None
    M = L.orc_wmod_solve(nz, _p(a2), _p(a1), _p(a0), dz, res.k_min, res.k_max, _p(w), isrc, ircv, WMOD_TOL, cap,
                         _p(kr), _p(ki), _p(vs), _p(vr), _p(vfull) if vfull is not None else None)
    if M < 0:
        raise RuntimeError("too many modes")
    ms = ModeSet(freq=freq, az=az, M=M, kr=kr[:M], ki=ki[:M], vs=vs[:M], vr=vr[:M], vg=None, k_min=res.k_min,
                 k_max=res.k_max, rho_s=float(pp.rho_g[isrc]), rho_r=float(pp.rho_g[ircv]), dz=dz, isrc=isrc,
                 ircv=ircv)
    ms.coeffs = (a2, a1, a0)
    if want_full:
        ms.vfull = vfull[: nz * M].reshape(nz, M)
    return ms


def tl1d(ms: ModeSet, nr: int, dr: float, lossless=False):
    re, im, inc = np.empty(nr), np.empty(nr), np.empty(nr)
    lib().orc_tl1d(ms.M, _p(_f64(ms.kr)), _p(_f64(ms.ki)), _p(_f64(ms.vs)), _p(_f64(ms.vr)), nr, float(dr),
                   int(lossless), _p(re), _p(im), _p(inc))
    return re, im, inc


# --------------------------------------------------------------------------
# ModBB propagation (ModalBroadbandPropagator.cpp:25-277)
# --------------------------------------------------------------------------
@dataclass
class Dispersion:
    f: np.ndarray          # includes the DC slot f[0] = 0
    mode_off: np.ndarray   # CSR offsets into the mode arrays (len nfreq + 1)
    re_k: np.ndarray
    im_k: np.ndarray
    ms: np.ndarray
    mr: np.ndarray
    rho_s: float
    rho_r: float


def read_dispersion(path) -> Dispersion:
    # slot 0 is the DC frequency with no modes (ModalBroadbandPropagator.cpp:114-116)
    f, off, rk, ik, vs, vr = [0.0], [0, 0], [], [], [], []
    rho_s = rho_r = 1.0
    with open(path) as fh:
        toks = fh.read().split()
    i = 0
    while i < len(toks):
        f.append(float(toks[i]))
        m = int(toks[i + 1])
        rho_s, rho_r = float(toks[i + 2]), float(toks[i + 3])
        i += 4
        for _ in range(m):
            rk.append(float(toks[i])); ik.append(float(toks[i + 1]))
            vs.append(float(toks[i + 2])); vr.append(float(toks[i + 3]))
            i += 4
        off.append(off[-1] + m)
    return Dispersion(np.array(f), np.array(off, dtype=np.int32), np.array(rk), np.array(ik),
                      np.array(vs), np.array(vr), rho_s, rho_r)


def dispersion_from_modesets(modesets) -> Dispersion:
    f, off = [0.0], [0, 0]
    rk, ik, vs, vr = [], [], [], []
    for m in modesets:
        f.append(m.freq)
        off.append(off[-1] + m.M)
        rk.extend(m.kr); ik.extend(m.ki); vs.extend(m.vs); vr.extend(m.vr)
    last = modesets[-1]
    return Dispersion(np.array(f), np.array(off, dtype=np.int32), np.array(rk), np.array(ik),
                      np.array(vs), np.array(vr), last.rho_s, last.rho_r)


def bb_transfer(d: Dispersion, rng: float):
    nf = len(d.f)
    hre, him = np.empty(nf), np.empty(nf)
    off = np.ascontiguousarray(d.mode_off, dtype=np.int32)
    lib().orc_bb_transfer(nf, off.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _p(_f64(d.re_k)),
                          _p(_f64(d.im_k)), _p(_f64(d.ms)), _p(_f64(d.mr)), d.rho_s, d.rho_r, float(rng),
                          _p(hre), _p(him))
    return hre, him


def source_spectrum(kind: str, f_vec, nfft: int, f_center=-1.0, waveform=None, spectrum=None):
    """BroadbandPropagator::get_source_spectrum (BroadbandPropagator.cpp:244-353)."""
    f_vec = _f64(f_vec)
    nf = len(f_vec)
    f_step = f_vec[2] - f_vec[1]
    fmx = nfft * f_step
    dt = 1.0 / fmx
    if kind == "impulse":
        ang = 2.0 * PI * f_vec * nf / 2.0
        return np.cos(ang), np.sin(ang)
    if kind in ("pulse1", "pulse2"):
        if f_center < 0.0:
            f_center = f_vec[-1] / 5.0
        if not (f_center > 0 and f_center <= f_vec[-1] / 5.0 + 1.0e-16):
            raise ValueError("f_center too large")
        scale = 1.0 / f_center
        if kind == "pulse1":
            fnorm = 0.780776406404415
            x = scale * fnorm * f_vec
            ans = x * np.exp((-x - x * x) / 2) * np.exp(1j * (-0.5 * PI)) * scale / 33.4336
            ans = 4.0 * PI * 5.0 * ans * np.exp(1j * 2.0 * PI * x * 0.01)
            sp = ans * np.exp(1j * 2.0 * PI * f_vec * scale) / 2.0
            return sp.real.copy(), sp.imag.copy()
        power = 8.0
        t = np.arange(nfft) * dt
        xx = 2.094 * (1.0 + power) * t / scale
        pulse = xx ** power * (1 - xx / (1.0 + power)) * np.exp(-xx) / 1.387566e+03
        sre, sim = np.empty(nf), np.empty(nf)
        lib().orc_dft_source(nfft, _p(_f64(pulse)), dt, nfft, nf, _p(sre), _p(sim))
        return sre, sim
    if kind == "spectrum":
        return _f64(spectrum[0]), _f64(spectrum[1])
    if kind == "waveform":
        t, x = waveform
        dtw = t[1] - t[0]
        sre, sim = np.empty(nf), np.empty(nf)
        lib().orc_dft_source(len(x), _p(_f64(x)), float(dtw), nfft, nf, _p(sre), _p(sim))
        return sre, sim
    raise ValueError(kind)


def bb_pulse(d: Dispersion, sre, sim, hre, him, t0, nfft):
    out = np.empty(nfft)
    lib().orc_bb_pulse(len(d.f), _p(_f64(d.f)), _p(_f64(sre)), _p(_f64(sim)), _p(_f64(hre)), _p(_f64(him)),
                       float(t0), int(nfft), _p(out))
    return out


def bb_nfft(nfreq: int, nfft_opt: int, waveform_lines: int | None):
    """NFFT rule of ModalBroadbandPropagator.cpp:71-84."""
    nfft = nfft_opt
    if nfft < 4 * nfreq:
        nfft = 4 * nfreq
    if waveform_lines is not None:
        while waveform_lines > nfft:
            nfft *= 2
    return nfft
