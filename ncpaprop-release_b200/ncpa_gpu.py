"""ctypes binding of the C ABI in include/ncpa_gpu.h (libncpa_gpu.so).

Thin Python view of the B200 library for tests, benchmarks and scripting:
every call goes straight to the CUDA library; nothing here computes on the
CPU.  Loading fails loudly if the shared library is missing.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libncpa_gpu.so")

_c_int, _c_double, _c_ll = ctypes.c_int, ctypes.c_double, ctypes.c_longlong
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p

EXPORTED = [
    "ncpa_ctx_create", "ncpa_ctx_destroy", "ncpa_status_str", "ncpa_last_error", "ncpa_ctx_synchronize",
    "ncpa_profile_create", "ncpa_profile_load", "ncpa_profile_destroy", "ncpa_profile_info",
    "ncpa_ess_params_default", "ncpa_ess_solve", "ncpa_modes_destroy", "ncpa_modes_problems", "ncpa_modes_count",
    "ncpa_modes_info", "ncpa_modes_get", "ncpa_modes_get_vectors", "ncpa_tl_1d", "ncpa_tl_2d_heights",
    "ncpa_tl_2d", "ncpa_bb_synthesize", "ncpa_bb_synthesize_modes", "ncpa_source_spectrum_waveform",
    "ncpa_kernel_launches", "ncpa_ctx_stream", "ncpa_ctx_set_timing", "ncpa_ctx_phase_stats",
    "ncpa_ctx_reset_stats", "ncpa_ctx_sturm_steps", "ncpa_probe_fp64_peak", "ncpa_source_spectrum_builtin",
    "ncpa_eigvec_static", "ncpa_profile_set_attn", "ncpa_profile_load_attn", "ncpa_profile_knots", "ncpa_profile_z0",
    "ncpa_modal_starter", "ncpa_source_waveform", "ncpa_tl_multi", "ncpa_ess_solve_jobs", "ncpa_server_opts_default", "ncpa_server_create",
    "ncpa_server_submit", "ncpa_server_wait", "ncpa_server_release", "ncpa_server_stats_get", "ncpa_server_destroy", "ncpa_modes_get_all",
    "ncpa_ess_plan_create", "ncpa_ess_plan_run", "ncpa_ess_plan_modes", "ncpa_ess_plan_tl", "ncpa_ess_plan_tuning",
    "ncpa_ess_plan_destroy", "ncpa_profile_update", "ncpa_g2s_convert", "ncpa_profile_load_g2s",
    "ncpa_dispersion_read", "ncpa_dispersion_desc_get", "ncpa_dispersion_destroy", "ncpa_ctx_sum_fixups",
    "ncpa_ctx_sum_guard", "ncpa_tl_1d_range", "ncpa_modes_from_host", "ncpa_ctx_sum_schedule", "ncpa_ctx_bisect_steps",
]


def read_dispersion(text_path, cache_path=None):
    """A ModBB dispersion file parsed by the library (host only), optionally
    through its binary cache: dict of f (DC slot first), mode_off, kr, ki,
    vs, vr, rho_src, rho_rcv, rows (newlines of the text), from_cache."""
    h = _vp()
    st = lib().ncpa_dispersion_read(str(text_path).encode(), str(cache_path).encode() if cache_path else None,
                                    ctypes.byref(h))
    if st != 0:
        raise NcpaError(st, "ncpa_dispersion_read")
    try:
        d, rows, fc = _DispDesc(), _c_int(), _c_int()
        lib().ncpa_dispersion_desc_get(h, ctypes.byref(d), ctypes.byref(rows), ctypes.byref(fc))
        nf = d.n_freq
        off = np.ctypeslib.as_array(d.mode_off, shape=(nf + 1,)).copy()
        n = int(off[-1])
        arr = lambda p, k: np.ctypeslib.as_array(p, shape=(k,)).copy() if k else np.empty(0)
        return {"f": arr(d.f, nf), "mode_off": off, "kr": arr(d.re_k, n), "ki": arr(d.im_k, n),
                "vs": arr(d.v_src, n), "vr": arr(d.v_rcv, n), "rho_src": d.rho_src, "rho_rcv": d.rho_rcv,
                "rows": rows.value, "from_cache": fc.value}
    finally:
        lib().ncpa_dispersion_destroy(h)


def g2s_convert(g2s_path, ncpa_path):
    """Writes the NCPA-format equivalent of a G2S-style profile; returns the
    (lat, lon) of its location line (NaN when absent).  Host only."""
    la, lo = _c_double(), _c_double()
    st = lib().ncpa_g2s_convert(str(g2s_path).encode(), str(ncpa_path).encode(), ctypes.byref(la), ctypes.byref(lo))
    if st != 0:
        raise NcpaError(st, "ncpa_g2s_convert")
    return la.value, lo.value


class NcpaError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s (status %d): %s" % (msg, status, _status_str(status)))
        self.status = status


class _CtxOpts(ctypes.Structure):
    _fields_ = [("device", _c_int)]


class _ProfileDesc(ctypes.Structure):
    _fields_ = [("n_knots", _c_int), ("z", _dp), ("u", _dp), ("v", _dp), ("t", _dp), ("p", _dp), ("rho", _dp),
                ("c0", _dp), ("attn", _dp), ("z0_m", _c_double), ("has_z0", _c_int)]


class _EssJob(ctypes.Structure):
    _fields_ = [("profile", _vp), ("freqs", _dp), ("n_freq", _c_int), ("az_deg", _c_double), ("nz_grid", _c_int),
                ("n_az", _c_int), ("az_list", _dp)]


class EssParams(ctypes.Structure):
    _fields_ = [("nz_grid", _c_int), ("maxheight_km", _c_double), ("zground_km", _c_double),
                ("sourceheight_km", _c_double), ("receiverheight_km", _c_double), ("lamb_wave_bc", _c_int),
                ("turnoff_wkb", _c_int), ("wvnum_filter", _c_int), ("c_min", _c_double), ("c_max", _c_double),
                ("want_group_speed", _c_int), ("want_vectors", _c_int), ("max_modes", _c_int),
                ("keep_on_device", _c_int), ("method", _c_int)]

METHOD_ESS, METHOD_WMOD = 0, 1


class _TlParams(ctypes.Structure):
    _fields_ = [("n_ranges", _c_int), ("dr_m", _c_double), ("lossless", _c_int)]


class _DispDesc(ctypes.Structure):
    _fields_ = [("n_freq", _c_int), ("f", _dp), ("mode_off", _ip), ("re_k", _dp), ("im_k", _dp), ("v_src", _dp),
                ("v_rcv", _dp), ("rho_src", _c_double), ("rho_rcv", _c_double)]


class _BbParams(ctypes.Structure):
    _fields_ = [("n_ranges", _c_int), ("ranges_m", _dp), ("max_celerity", _c_double), ("nfft", _c_int),
                ("src_re", _dp), ("src_im", _dp), ("zero_attn", _c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError("libncpa_gpu.so not built: run `make -C %s`" % _HERE)
        L = ctypes.CDLL(LIB_PATH)
        L.ncpa_ctx_create.argtypes = [ctypes.POINTER(_vp), ctypes.POINTER(_CtxOpts)]
        L.ncpa_ctx_destroy.argtypes = [_vp]
        L.ncpa_status_str.restype = ctypes.c_char_p
        L.ncpa_status_str.argtypes = [_c_int]
        L.ncpa_last_error.restype = ctypes.c_char_p
        L.ncpa_last_error.argtypes = [_vp]
        L.ncpa_ctx_synchronize.argtypes = [_vp]
        L.ncpa_profile_create.argtypes = [_vp, ctypes.POINTER(_ProfileDesc), ctypes.POINTER(_vp)]
        L.ncpa_profile_load.argtypes = [_vp, ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(_vp)]
        L.ncpa_profile_destroy.argtypes = [_vp]
        L.ncpa_profile_info.argtypes = [_vp, _ip, _dp, _dp]
        L.ncpa_ess_params_default.argtypes = [ctypes.POINTER(EssParams)]
        L.ncpa_ess_params_default.restype = None
        L.ncpa_profile_load_attn.argtypes = [_vp, ctypes.c_char_p]
        L.ncpa_ess_solve_jobs.argtypes = [_vp, ctypes.POINTER(_EssJob), _c_int, ctypes.POINTER(EssParams),
                                          ctypes.POINTER(_vp)]
        L.ncpa_ess_plan_create.argtypes = [_vp, ctypes.POINTER(_EssJob), _c_int, ctypes.POINTER(EssParams),
                                           ctypes.POINTER(_TlParams), _c_int, ctypes.POINTER(_vp)]
        L.ncpa_ess_plan_run.argtypes = [_vp]
        L.ncpa_ess_plan_modes.argtypes = [_vp, ctypes.POINTER(_vp)]
        L.ncpa_ess_plan_tl.argtypes = [_vp, _dp, _dp, _dp]
        L.ncpa_ess_plan_tuning.argtypes = [_vp, _ip, _ip, _ip, ctypes.POINTER(_c_double)]
        L.ncpa_ess_plan_destroy.argtypes = [_vp]
        L.ncpa_profile_update.argtypes = [_vp, ctypes.POINTER(_ProfileDesc)]
        L.ncpa_g2s_convert.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(_c_double),
                                       ctypes.POINTER(_c_double)]
        L.ncpa_profile_load_g2s.argtypes = [_vp, ctypes.c_char_p, ctypes.POINTER(_vp)]
        L.ncpa_dispersion_read.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(_vp)]
        L.ncpa_dispersion_desc_get.argtypes = [_vp, ctypes.POINTER(_DispDesc), _ip, _ip]
        L.ncpa_dispersion_destroy.argtypes = [_vp]
        L.ncpa_ess_solve.argtypes = [_vp, _vp, ctypes.POINTER(EssParams), _dp, _c_int, _dp, _c_int,
                                     ctypes.POINTER(_vp)]
        L.ncpa_modes_destroy.argtypes = [_vp]
        L.ncpa_modes_problems.argtypes = [_vp, _ip]
        L.ncpa_modes_count.argtypes = [_vp, _c_int, _ip]
        L.ncpa_modes_info.argtypes = [_vp, _c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.ncpa_modes_get.argtypes = [_vp, _c_int, _dp, _dp, _dp, _dp, _dp]
        L.ncpa_modes_get_vectors.argtypes = [_vp, _c_int, _dp]
        L.ncpa_modes_get_all.argtypes = [_vp, _ip, _dp, _dp, _dp, _dp, _dp]
        L.ncpa_tl_1d.argtypes = [_vp, _vp, ctypes.POINTER(_TlParams), _dp, _dp, _dp]
        L.ncpa_tl_2d_heights.argtypes = [_vp, _c_int, _ip]
        L.ncpa_tl_2d.argtypes = [_vp, _vp, _c_int, ctypes.POINTER(_TlParams), _dp, _dp, _dp]
        L.ncpa_tl_multi.argtypes = [_vp, _vp, _c_int, _c_int, _dp, ctypes.POINTER(_TlParams), _c_int, _dp, _dp]
        L.ncpa_bb_synthesize.argtypes = [_vp, ctypes.POINTER(_DispDesc), ctypes.POINTER(_BbParams), _dp]
        L.ncpa_bb_synthesize_modes.argtypes = [_vp, _vp, _c_int, ctypes.POINTER(_BbParams), _dp]
        L.ncpa_source_spectrum_waveform.argtypes = [_vp, _dp, _c_int, _c_double, _c_int, _c_int, _dp, _dp]
        L.ncpa_kernel_launches.argtypes = [_vp]
        L.ncpa_kernel_launches.restype = _c_ll
        L.ncpa_ctx_stream.argtypes = [_vp]
        L.ncpa_ctx_stream.restype = _vp
        L.ncpa_ctx_set_timing.argtypes = [_vp, _c_int]
        L.ncpa_ctx_phase_stats.argtypes = [_vp, ctypes.c_char_p, _dp, ctypes.POINTER(_c_ll)]
        L.ncpa_ctx_reset_stats.argtypes = [_vp]
        L.ncpa_ctx_sturm_steps.argtypes = [_vp, ctypes.POINTER(_c_ll)]
        L.ncpa_ctx_sum_fixups.argtypes = [_vp, ctypes.POINTER(_c_ll), ctypes.POINTER(_c_ll)]
        L.ncpa_ctx_sum_guard.argtypes = [_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(_c_int)]
        L.ncpa_ctx_sum_schedule.argtypes = [_vp, _ip, _ip, _ip, _dp]
        L.ncpa_ctx_bisect_steps.argtypes = [_vp, ctypes.POINTER(_c_ll), ctypes.POINTER(_c_ll)]
        L.ncpa_probe_fp64_peak.argtypes = [_vp, _dp]
        L.ncpa_source_spectrum_builtin.argtypes = [_vp, _c_int, _dp, _c_int, _c_double, _c_int, _dp, _dp]
        _lib = L
    return _lib


def _status_str(s):
    try:
        return lib().ncpa_status_str(int(s)).decode()
    except OSError:
        return "?"


def _p(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def default_params(**kw) -> EssParams:
    p = EssParams()
    lib().ncpa_ess_params_default(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class Context:
    def __init__(self, device=0):
        self.h = _vp()
        opts = _CtxOpts(device)
        st = lib().ncpa_ctx_create(ctypes.byref(self.h), ctypes.byref(opts))
        if st != 0:
            raise NcpaError(st, "ncpa_ctx_create")

    def check(self, st, what):
        if st != 0:
            msg = lib().ncpa_last_error(self.h).decode()
            raise NcpaError(st, "%s: %s" % (what, msg))

    def close(self):
        if self.h:
            lib().ncpa_ctx_destroy(self.h)
            self.h = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def synchronize(self):
        self.check(lib().ncpa_ctx_synchronize(self.h), "synchronize")

    @property
    def launches(self):
        return int(lib().ncpa_kernel_launches(self.h))

    @property
    def stream_ptr(self):
        return int(lib().ncpa_ctx_stream(self.h) or 0)

    def set_timing(self, on=True):
        """per-phase device times: on = True / 1 runs the bisection and
        eigenvector kernels apart, 2 keeps the fused launch ("bisect+eigvec")"""
        self.check(lib().ncpa_ctx_set_timing(self.h, int(on)), "ncpa_ctx_set_timing")

    def reset_stats(self):
        self.check(lib().ncpa_ctx_reset_stats(self.h), "ncpa_ctx_reset_stats")

    def phase_stats(self, phase):
        ms, n = _c_double(), _c_ll()
        self.check(lib().ncpa_ctx_phase_stats(self.h, phase.encode(), ctypes.byref(ms), ctypes.byref(n)),
                   "ncpa_ctx_phase_stats")
        return ms.value, n.value

    def sturm_steps(self):
        """Sturm recurrence steps run by the bisection kernel since the last
        reset (counted while per-phase timing is on)."""
        a = _c_ll()
        self.check(lib().ncpa_ctx_sturm_steps(self.h, ctypes.byref(a)), "ncpa_ctx_sturm_steps")
        return a.value

    def sum_fixups(self):
        """(points recomputed in FP64, receivers x ranges) of the last guarded
        tensor-core modal sum"""
        a, b = _c_ll(), _c_ll()
        self.check(lib().ncpa_ctx_sum_fixups(self.h, ctypes.byref(a), ctypes.byref(b)), "ncpa_ctx_sum_fixups")
        return a.value, b.value

    def sum_guard(self):
        """(eps, tau, tile_ranges) of the last guarded tensor-core modal sum:
        its error is at most eps S (S = sum of the magnitudes of a point's
        modal terms at the first range of its tile of tile_ranges ranges) and
        points with |P| < tau S were recomputed in FP64"""
        e, t, n = ctypes.c_double(), ctypes.c_double(), _c_int()
        self.check(lib().ncpa_ctx_sum_guard(self.h, ctypes.byref(e), ctypes.byref(t), ctypes.byref(n)),
                   "ncpa_ctx_sum_guard")
        return e.value, t.value, n.value

    def sum_schedule(self):
        """(TMA ring depth, operand ring depth, per-variant times in ms of the
        last tuning run) of the last tensor-core modal sum"""
        t, g, n = _c_int(), _c_int(), _c_int()
        times = np.zeros(16)
        self.check(lib().ncpa_ctx_sum_schedule(self.h, ctypes.byref(t), ctypes.byref(g), ctypes.byref(n),
                                               _p(times)), "ncpa_ctx_sum_schedule")
        return t.value, g.value, times[:n.value].copy()

    def bisect_steps(self):
        """(all Sturm chain steps, steps of the chains carrying derivatives)
        of the bisection kernel since the last reset (counted while per-phase
        timing is on)"""
        a, b = _c_ll(), _c_ll()
        self.check(lib().ncpa_ctx_bisect_steps(self.h, ctypes.byref(a), ctypes.byref(b)), "ncpa_ctx_bisect_steps")
        return a.value, b.value

    def fp64_peak_tflops(self):
        t = _c_double()
        self.check(lib().ncpa_probe_fp64_peak(self.h, ctypes.byref(t)), "ncpa_probe_fp64_peak")
        return t.value

    # profiles -------------------------------------------------------------
    def load_profile(self, path, header=""):
        h = _vp()
        self.check(lib().ncpa_profile_load(self.h, str(path).encode(), str(header).encode() if header else None,
                                           ctypes.byref(h)), "ncpa_profile_load")
        return Profile(self, h)

    def load_profile_g2s(self, path):
        """G2S-style profile file (location line + Z T U V P RHO columns)."""
        h = _vp()
        self.check(lib().ncpa_profile_load_g2s(self.h, str(path).encode(), ctypes.byref(h)), "ncpa_profile_load_g2s")
        return Profile(self, h)

    def profile_from_arrays(self, z, u, v, t, p, rho, c0=None, attn=None, z0=None):
        d, _keep = _profile_desc(z, u, v, t, p, rho, c0, attn, z0)
        h = _vp()
        self.check(lib().ncpa_profile_create(self.h, ctypes.byref(d), ctypes.byref(h)), "ncpa_profile_create")
        return Profile(self, h)

    # solve ----------------------------------------------------------------
    def solve(self, profile, params: EssParams, freqs, azimuths):
        f = _f64(np.atleast_1d(freqs))
        a = _f64(np.atleast_1d(azimuths))
        h = _vp()
        self.check(lib().ncpa_ess_solve(self.h, profile.h, ctypes.byref(params), _p(f), len(f), _p(a), len(a),
                                        ctypes.byref(h)), "ncpa_ess_solve")
        return Modes(self, h, f, a)

    def solve_jobs(self, jobs, params: EssParams):
        """One batched solve over jobs [(profile, freqs, azimuth_deg[, nz_grid]), ...].
        azimuth_deg is a number or a list of azimuths (the job sweeps them);
        nz_grid (optional, 0 = params.nz_grid) sets the job's own grid.
        Problems are numbered job by job, frequency-major then azimuth."""
        arr, keep, fr, az_all = _jobs_array(jobs)
        h = _vp()
        self.check(lib().ncpa_ess_solve_jobs(self.h, arr, len(jobs), ctypes.byref(params), ctypes.byref(h)),
                   "ncpa_ess_solve_jobs")
        return Modes(self, h, fr, az_all)

    def plan(self, jobs, params: EssParams, tl=None, tune=False):
        """A captured solve (CUDA graph) of the jobs of solve_jobs; tl =
        (n_ranges, dr_m[, lossless]) adds the 1-D TL to the graph; tune times
        launch shapes and keeps the fastest."""
        arr, keep, fr, az_all = _jobs_array(jobs)
        tp = _TlParams(int(tl[0]), float(tl[1]), int(tl[2]) if len(tl) > 2 else 0) if tl is not None else None
        h = _vp()
        self.check(lib().ncpa_ess_plan_create(self.h, arr, len(jobs), ctypes.byref(params),
                                              ctypes.byref(tp) if tp is not None else None, int(bool(tune)),
                                              ctypes.byref(h)), "ncpa_ess_plan_create")
        return Plan(self, h, fr, az_all, tl)

    SOURCES = {"impulse": 0, "pulse1": 1, "pulse2": 2}

    def source_spectrum_builtin(self, kind, f, nfft, f_center=-1.0):
        f = _f64(f)
        sre, sim = np.empty(len(f)), np.empty(len(f))
        self.check(lib().ncpa_source_spectrum_builtin(self.h, self.SOURCES[kind], _p(f), len(f), float(f_center),
                                                      int(nfft), _p(sre), _p(sim)), "ncpa_source_spectrum_builtin")
        return sre, sim

    def source_spectrum_waveform(self, x, dt, nfft, nfreq):
        x = _f64(x)
        sre, sim = np.empty(nfreq), np.empty(nfreq)
        self.check(lib().ncpa_source_spectrum_waveform(self.h, _p(x), len(x), float(dt), int(nfft), int(nfreq),
                                                       _p(sre), _p(sim)), "ncpa_source_spectrum_waveform")
        return sre, sim

    def bb_synthesize(self, f, mode_off, re_k, im_k, v_src, v_rcv, rho_src, rho_rcv, ranges_m, max_celerity, nfft,
                      src_re, src_im, zero_attn=False):
        f, re_k, im_k, v_src, v_rcv = (_f64(x) for x in (f, re_k, im_k, v_src, v_rcv))
        off = np.ascontiguousarray(mode_off, dtype=np.int32)
        rng, sre, sim = _f64(ranges_m), _f64(src_re), _f64(src_im)
        d = _DispDesc(len(f), _p(f), off.ctypes.data_as(_ip), _p(re_k), _p(im_k), _p(v_src), _p(v_rcv),
                      float(rho_src), float(rho_rcv))
        bp = _BbParams(len(rng), _p(rng), float(max_celerity), int(nfft), _p(sre), _p(sim), int(zero_attn))
        out = np.empty((len(rng), nfft))
        self.check(lib().ncpa_bb_synthesize(self.h, ctypes.byref(d), ctypes.byref(bp), _p(out)),
                   "ncpa_bb_synthesize")
        return out


def _profile_desc(z, u, v, t, p, rho, c0=None, attn=None, z0=None):
    arrs = [_f64(x) for x in (z, u, v, t, p, rho)]
    c0a = _f64(c0) if c0 is not None else None
    aa = _f64(attn) if attn is not None else None
    d = _ProfileDesc(len(arrs[0]), *[_p(a) for a in arrs], _p(c0a), _p(aa), float(z0 or 0.0), int(z0 is not None))
    return d, (arrs, c0a, aa)


def _jobs_array(jobs):
    keep, fr, az_all = [], [], []
    arr = (_EssJob * len(jobs))()
    for i, job in enumerate(jobs):
        prof, freqs, az = job[0], job[1], job[2]
        nz = int(job[3]) if len(job) > 3 else 0
        f = _f64(np.atleast_1d(freqs))
        keep.append(f)
        if np.ndim(az) == 0:
            arr[i] = _EssJob(prof.h.value, _p(f), len(f), float(az), nz, 0, None)
            fr.append(f)
            az_all.append(np.full(len(f), float(az)))
        else:
            a = _f64(np.atleast_1d(az))
            keep.append(a)
            arr[i] = _EssJob(prof.h.value, _p(f), len(f), float(a[0]), nz, len(a), _p(a))
            fr.append(np.repeat(f, len(a)))
            az_all.append(np.tile(a, len(f)))
    return arr, keep, np.concatenate(fr), np.concatenate(az_all)


class Profile:
    def __init__(self, ctx, h):
        self.ctx, self.h = ctx, h

    def info(self):
        n, lo, hi = _c_int(), _c_double(), _c_double()
        self.ctx.check(lib().ncpa_profile_info(self.h, ctypes.byref(n), ctypes.byref(lo), ctypes.byref(hi)),
                       "ncpa_profile_info")
        return n.value, lo.value, hi.value

    def load_attn(self, path):
        """User attenuation table (height km, Np/m), the --use_attn_file option."""
        self.ctx.check(lib().ncpa_profile_load_attn(self.h, str(path).encode()), "ncpa_profile_load_attn")

    def update(self, z, u, v, t, p, rho, c0=None, attn=None, z0=None):
        """New knot values in place (same knots, altitudes and ground height)."""
        d, _keep = _profile_desc(z, u, v, t, p, rho, c0, attn, z0)
        self.ctx.check(lib().ncpa_profile_update(self.h, ctypes.byref(d)), "ncpa_profile_update")

    def close(self):
        if self.h:
            lib().ncpa_profile_destroy(self.h)
            self.h = _vp()


@dataclass
class ProblemModes:
    freq: float
    az: float
    dz: float
    k_min: float
    k_max: float
    rho_src: float
    rho_rcv: float
    kr: np.ndarray
    ki: np.ndarray
    vs: np.ndarray
    vr: np.ndarray
    vg: np.ndarray

    @property
    def M(self):
        return len(self.kr)


class Modes:
    def __init__(self, ctx, h, freqs, azs, owned=True):
        self.ctx, self.h, self.owned = ctx, h, owned
        self.freqs, self.azs = freqs, azs
        n = _c_int()
        ctx.check(lib().ncpa_modes_problems(h, ctypes.byref(n)), "ncpa_modes_problems")
        self.P = n.value

    def count(self, p):
        n = _c_int()
        self.ctx.check(lib().ncpa_modes_count(self.h, p, ctypes.byref(n)), "ncpa_modes_count")
        return n.value

    def counts(self):
        return np.array([self.count(p) for p in range(self.P)])

    def total_modes(self):
        """modes of all problems together (host bookkeeping, no device wait)"""
        off = np.empty(self.P + 1, dtype=np.int32)
        self.ctx.check(lib().ncpa_modes_get_all(self.h, off.ctypes.data_as(_ip), None, None, None, None, None),
                       "ncpa_modes_get_all")
        return int(off[-1])

    def problem(self, p) -> ProblemModes:
        M = self.count(p)
        vals = [_c_double() for _ in range(7)]
        self.ctx.check(lib().ncpa_modes_info(self.h, p, *[ctypes.byref(v) for v in vals]), "ncpa_modes_info")
        kr, ki, vs, vr, vg = (np.empty(M) for _ in range(5))
        self.ctx.check(lib().ncpa_modes_get(self.h, p, _p(kr), _p(ki), _p(vs), _p(vr), _p(vg)), "ncpa_modes_get")
        return ProblemModes(*[v.value for v in vals], kr, ki, vs, vr, vg)

    def all_modes(self, out=None):
        """(mode_off, kr, ki, vs, vr, vg) of every problem in CSR order.  out:
        five float64 arrays of at least the total mode count to copy into
        (page-locked ones make the copies direct); the returned arrays are
        views of their first entries."""
        off = np.empty(self.P + 1, dtype=np.int32)
        self.ctx.check(lib().ncpa_modes_get_all(self.h, off.ctypes.data_as(_ip), None, None, None, None, None),
                       "ncpa_modes_get_all")
        n = int(off[-1])
        if out is None:
            arrs = [np.empty(n) for _ in range(5)]
        else:
            if len(out) != 5 or any(a.dtype != np.float64 or a.size < n or not a.flags.c_contiguous for a in out):
                raise ValueError("out: five contiguous float64 arrays of at least %d entries" % n)
            arrs = [a.reshape(-1)[:n] for a in out]
        self.ctx.check(lib().ncpa_modes_get_all(self.h, off.ctypes.data_as(_ip), *[_p(a) for a in arrs]),
                       "ncpa_modes_get_all")
        return (off, *arrs)

    def vectors(self, p, nz):
        M = self.count(p)
        v = np.empty(nz * M)
        self.ctx.check(lib().ncpa_modes_get_vectors(self.h, p, _p(v)), "ncpa_modes_get_vectors")
        return v.reshape(nz, M)

    def tl1d(self, n_ranges, dr_m, lossless=False, to_host=True, out=None):
        """1-D TL of every problem; out = (re, im, inc) C-contiguous float64
        arrays of shape (P, n_ranges) to fill (e.g. views of pinned memory)."""
        tp = _TlParams(int(n_ranges), float(dr_m), int(lossless))
        if not to_host:
            self.ctx.check(lib().ncpa_tl_1d(self.ctx.h, self.h, ctypes.byref(tp), None, None, None), "ncpa_tl_1d")
            return None
        if out is not None:
            re, im, inc = out
            for a in out:
                assert a.dtype == np.float64 and a.flags.c_contiguous and a.shape == (self.P, n_ranges)
        else:
            re, im, inc = (np.empty((self.P, n_ranges)) for _ in range(3))
        self.ctx.check(lib().ncpa_tl_1d(self.ctx.h, self.h, ctypes.byref(tp), _p(re), _p(im), _p(inc)),
                       "ncpa_tl_1d")
        return re, im, inc

    def tl2d(self, p, n_ranges, dr_m, lossless=False):
        n = _c_int()
        self.ctx.check(lib().ncpa_tl_2d_heights(self.h, p, ctypes.byref(n)), "ncpa_tl_2d_heights")
        z = np.empty(n.value)
        re, im = np.empty((n_ranges, n.value)), np.empty((n_ranges, n.value))
        tp = _TlParams(int(n_ranges), float(dr_m), int(lossless))
        self.ctx.check(lib().ncpa_tl_2d(self.ctx.h, self.h, p, ctypes.byref(tp), _p(z), _p(re), _p(im)),
                       "ncpa_tl_2d")
        return z, re, im

    SUM_FP64, SUM_TC_BF16X3, SUM_TC_TF32, SUM_TC_GUARDED = 0, 1, 2, 3

    def tl_multi(self, p, heights_m, n_ranges, dr_m, method=1, lossless=False, to_host=True):
        """Modal sum at many receivers: complex P [n_rcv x n_ranges]."""
        h = _f64(heights_m)
        tp = _TlParams(int(n_ranges), float(dr_m), int(lossless))
        re = np.empty((len(h), n_ranges)) if to_host else None
        im = np.empty((len(h), n_ranges)) if to_host else None
        self.ctx.check(lib().ncpa_tl_multi(self.ctx.h, self.h, p, len(h), _p(h), ctypes.byref(tp), int(method),
                                           _p(re), _p(im)), "ncpa_tl_multi")
        return (re + 1j * im) if to_host else None

    def bb_synthesize(self, ranges_m, max_celerity, nfft, src_re, src_im, zero_attn=False, to_host=True, out=None):
        rng, sre, sim = _f64(ranges_m), _f64(src_re), _f64(src_im)
        bp = _BbParams(len(rng), _p(rng), float(max_celerity), int(nfft), _p(sre), _p(sim), int(zero_attn))
        if out is not None:
            assert out.dtype == np.float64 and out.flags.c_contiguous and out.shape == (len(rng), nfft)
        elif to_host:
            out = np.empty((len(rng), nfft))
        self.ctx.check(lib().ncpa_bb_synthesize_modes(self.ctx.h, self.h, 0, ctypes.byref(bp), _p(out)),
                       "ncpa_bb_synthesize_modes")
        return out

    def close(self):
        if self.h:
            if self.owned:
                lib().ncpa_modes_destroy(self.h)
            self.h = _vp()


class Plan:
    """A captured batched solve (see Context.plan)."""

    def __init__(self, ctx, h, freqs, azs, tl):
        self.ctx, self.h, self.freqs, self.azs, self.tl_grid = ctx, h, freqs, azs, tl
        self.P = len(freqs)

    def run(self):
        self.ctx.check(lib().ncpa_ess_plan_run(self.h), "ncpa_ess_plan_run")

    def modes(self) -> Modes:
        """Result of the last run (valid until the next run; owned by the plan)."""
        h = _vp()
        self.ctx.check(lib().ncpa_ess_plan_modes(self.h, ctypes.byref(h)), "ncpa_ess_plan_modes")
        return Modes(self.ctx, h, self.freqs, self.azs, owned=False)

    def tl(self):
        n = int(self.tl_grid[0])
        re, im, inc = (np.empty((self.P, n)) for _ in range(3))
        self.ctx.check(lib().ncpa_ess_plan_tl(self.h, _p(re), _p(im), _p(inc)), "ncpa_ess_plan_tl")
        return re, im, inc

    def tuning(self):
        a, b, c, ms = _c_int(), _c_int(), _c_int(), _c_double()
        self.ctx.check(lib().ncpa_ess_plan_tuning(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
                                                  ctypes.byref(ms)), "ncpa_ess_plan_tuning")
        return {"bis_item": a.value, "bis_ctas_per_sm": b.value, "ev_ctas_per_sm": c.value, "ms": ms.value}

    def close(self):
        if self.h:
            lib().ncpa_ess_plan_destroy(self.h)
            self.h = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


# ---------------------------------------------------------------------------
# serving loop (ncpa_server_*)
# ---------------------------------------------------------------------------
class _ServerOpts(ctypes.Structure):
    _fields_ = [("device", _c_int), ("params", EssParams), ("n_ranges", _c_int), ("dr_m", _c_double),
                ("lanes", _c_int), ("max_batch_problems", _c_int), ("hbm_budget_bytes", _c_double),
                ("cache_bytes", _c_double)]


class _Request(ctypes.Structure):
    _fields_ = [("profile", _ProfileDesc), ("freqs", _dp), ("n_freq", _c_int), ("az_deg", _c_double),
                ("n_ranges", _c_int), ("dr_m", _c_double), ("n_wave_ranges", _c_int), ("wave_ranges_m", _dp),
                ("max_celerity", _c_double), ("nfft", _c_int), ("source", _c_int)]


class _Result(ctypes.Structure):
    _fields_ = [("status", _c_int), ("n_freq", _c_int), ("mode_off", _ip), ("re_k", _dp), ("im_k", _dp),
                ("v_src", _dp), ("v_rcv", _dp), ("tl_re", _dp), ("tl_im", _dp), ("tl_incoh", _dp),
                ("latency_ms", _c_double), ("batch_requests", _c_int), ("n_ranges", _c_int),
                ("n_wave_ranges", _c_int), ("nfft", _c_int), ("waveforms", _dp), ("from_cache", _c_int)]


class _ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong), ("batches", ctypes.c_longlong),
                ("mean_batch_requests", _c_double), ("p50_ms", _c_double), ("p99_ms", _c_double),
                ("max_ms", _c_double), ("peak_admitted_bytes", _c_double), ("cache_hits", ctypes.c_longlong),
                ("cache_entries", ctypes.c_longlong), ("cache_used_bytes", _c_double)]


_SERVER_SIGS = False


def _server_sigs():
    global _SERVER_SIGS
    if _SERVER_SIGS:
        return
    L = lib()
    L.ncpa_server_opts_default.argtypes = [ctypes.POINTER(_ServerOpts)]
    L.ncpa_server_opts_default.restype = None
    L.ncpa_server_create.argtypes = [ctypes.POINTER(_ServerOpts), ctypes.POINTER(_vp)]
    L.ncpa_server_submit.argtypes = [_vp, ctypes.POINTER(_Request), ctypes.POINTER(ctypes.c_ulonglong)]
    L.ncpa_server_wait.argtypes = [_vp, ctypes.c_ulonglong, _c_int, ctypes.POINTER(_Result)]
    L.ncpa_server_release.argtypes = [_vp, ctypes.c_ulonglong]
    L.ncpa_server_stats_get.argtypes = [_vp, ctypes.POINTER(_ServerStats)]
    L.ncpa_server_destroy.argtypes = [_vp]
    _SERVER_SIGS = True


class Server:
    """Serving loop: submit requests (profile knots in SI, frequencies,
    azimuth, optionally their own TL range grid and waveform ranges) at any
    time; each returns dispersion, 1-D TL and, when asked, waveforms.  With
    cache_bytes > 0 solved modes stay in HBM and repeated requests skip the
    eigen-solve."""

    SOURCES = {"impulse": 0, "pulse1": 1, "pulse2": 2}

    def __init__(self, device=0, params=None, n_ranges=2000, dr_m=500.0, lanes=2, max_batch_problems=1024,
                 hbm_budget_bytes=0.0, cache_bytes=0.0):
        _server_sigs()
        o = _ServerOpts()
        lib().ncpa_server_opts_default(ctypes.byref(o))
        o.device = device
        if params is not None:
            o.params = params
        o.n_ranges, o.dr_m, o.lanes = int(n_ranges), float(dr_m), int(lanes)
        o.max_batch_problems, o.hbm_budget_bytes = int(max_batch_problems), float(hbm_budget_bytes)
        o.cache_bytes = float(cache_bytes)
        self.n_ranges = int(n_ranges)
        self.h = _vp()
        st = lib().ncpa_server_create(ctypes.byref(o), ctypes.byref(self.h))
        if st != 0:
            raise NcpaError(st, "ncpa_server_create")

    def submit(self, z, u, v, t, p, rho, freqs, az_deg, z0=None, n_ranges=0, dr_m=0.0, wave_ranges_m=None,
               max_celerity=0.0, nfft=0, source="pulse1"):
        arrs = [_f64(x) for x in (z, u, v, t, p, rho)]
        f = _f64(np.atleast_1d(freqs))
        d = _ProfileDesc(len(arrs[0]), *[_p(a) for a in arrs], None, None, float(z0 or 0.0), int(z0 is not None))
        wr = _f64(wave_ranges_m) if wave_ranges_m is not None else None
        req = _Request(d, _p(f), len(f), float(az_deg), int(n_ranges), float(dr_m), len(wr) if wr is not None else 0,
                       _p(wr) if wr is not None else None, float(max_celerity), int(nfft), self.SOURCES[source])
        rid = ctypes.c_ulonglong()
        st = lib().ncpa_server_submit(self.h, ctypes.byref(req), ctypes.byref(rid))
        if st != 0:
            raise NcpaError(st, "ncpa_server_submit")
        return rid.value

    def wait(self, rid, timeout_ms=-1, release=True):
        r = _Result()
        st = lib().ncpa_server_wait(self.h, ctypes.c_ulonglong(rid), int(timeout_ms), ctypes.byref(r))
        if st != 0:
            raise NcpaError(st, "ncpa_server_wait")
        nf, nr = r.n_freq, r.n_ranges
        out = {"status": r.status, "latency_ms": r.latency_ms, "batch_requests": r.batch_requests,
               "from_cache": bool(r.from_cache)}
        if r.status == 0:
            off = np.ctypeslib.as_array(r.mode_off, shape=(nf + 1,)).copy()
            nm = int(off[-1])
            out["mode_off"] = off
            for k in ("re_k", "im_k", "v_src", "v_rcv"):
                ptr = getattr(r, k)
                out[k] = np.ctypeslib.as_array(ptr, shape=(nm,)).copy() if nm else np.empty(0)
            for k in ("tl_re", "tl_im", "tl_incoh"):
                out[k] = np.ctypeslib.as_array(getattr(r, k), shape=(nf * nr,)).copy().reshape(nf, nr)
            if r.n_wave_ranges > 0:
                out["waveforms"] = np.ctypeslib.as_array(r.waveforms, shape=(r.n_wave_ranges * r.nfft,)).copy() \
                    .reshape(r.n_wave_ranges, r.nfft)
        if release:
            lib().ncpa_server_release(self.h, ctypes.c_ulonglong(rid))
        return out

    def stats(self):
        s = _ServerStats()
        lib().ncpa_server_stats_get(self.h, ctypes.byref(s))
        return {k: getattr(s, k) for k, _ in _ServerStats._fields_}

    def close(self):
        if self.h:
            lib().ncpa_server_destroy(self.h)
            self.h = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
