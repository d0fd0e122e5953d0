"""The allocation-free eigenvector entry point (ncpa_eigvec_static).

Some callers cannot allocate device memory while they run (an application
that reserves all GPU memory up front, code inside a memory budget it does
not own).  ncpa_eigvec_static serves them: it takes device buffers from the
caller, allocates nothing, and uses one fixed scratch array inside the
library.  This test feeds it the scaled diagonal, attenuation weights and
eigenvalues of one problem (built by the CPU oracle, copied to the device)
and checks its wavenumbers and mode values against those of the allocating
entry point ncpa_ess_solve for the same problem, on two calls in a row (the
second call runs on the scratch the first one left behind).

Tolerances are the ones of the other GPU parity tests: Re k within the
k tolerance, Im k and V_s V_r within 1e-6 relative.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = np.finfo(float).eps


def test_static_eigvec_matches_solve(analytic_profile):
    import torch

    import ncpa_gpu
    from oracle import oracle as O

    freq, az = 0.12, 90.0
    with ncpa_gpu.Context(0) as ctx:
        prof = ctx.load_profile(analytic_profile)
        modes = ctx.solve(prof, ncpa_gpu.default_params(turnoff_wkb=1), [freq], [az])
        ref = modes.problem(0)
        modes.close()
        prof.close()

    prm = O.EssParams(turnoff_WKB=True)
    o = O.solve_problem(O.prepare(O.read_profile(analytic_profile), prm), prm, freq, az, keep_matrix=True)
    assert o.M == ref.M and o.M > 0
    dev = torch.device("cuda:0")
    d_s = torch.tensor(o.s, dtype=torch.float64, device=dev)
    d_w = torch.tensor(o.w, dtype=torch.float64, device=dev)
    d_mu = torch.tensor(o.mu, dtype=torch.float64, device=dev)
    outs = [torch.empty(o.M, dtype=torch.float64, device=dev) for _ in range(4)]
    L = ncpa_gpu.lib()
    fn = L.ncpa_eigvec_static
    dp = ctypes.c_void_p
    fn.argtypes = [dp, dp, ctypes.c_int, ctypes.c_double, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                   ctypes.c_double, dp, dp, dp, dp, dp]
    fn.restype = ctypes.c_int
    stream = torch.cuda.current_stream(dev).cuda_stream
    tol_k = np.maximum(1e-9, 8 * EPS * (4.0 / o.dz ** 2) / (2 * ref.kr ** 2))
    for call in range(2):
        for t in outs:
            t.fill_(float("nan"))
        st = fn(d_s.data_ptr(), d_w.data_ptr(), len(o.s), o.dz, d_mu.data_ptr(), o.M, o.isrc, o.ircv,
                2 * np.pi * freq, *(t.data_ptr() for t in outs), stream)
        assert st == 0, (call, st)
        torch.cuda.synchronize()
        kr, ki, vs, vr = (t.cpu().numpy() for t in outs)
        assert np.all(np.abs(kr - ref.kr) / ref.kr <= tol_k), call
        assert np.allclose(ki, ref.ki, rtol=1e-6, atol=1e-18), call
        vv, vref = vs * vr, ref.vs * ref.vr
        assert np.allclose(vv, vref, rtol=1e-6, atol=1e-12 * np.abs(vref).max()), call


def test_static_eigvec_rejects_oversize():
    import ncpa_gpu

    L = ncpa_gpu.lib()
    fn = L.ncpa_eigvec_static
    dp = ctypes.c_void_p
    fn.argtypes = [dp, dp, ctypes.c_int, ctypes.c_double, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                   ctypes.c_double, dp, dp, dp, dp, dp]
    fn.restype = ctypes.c_int
    fake = ctypes.c_void_p(16)  # never dereferenced: the size checks come first
    assert fn(fake, fake, 40000, 1.0, fake, 10, 0, 0, 1.0, fake, fake, fake, fake, None) == 1  # NCPA_EINVAL
    assert fn(fake, fake, 1000, 1.0, fake, 5000, 0, 0, 1.0, fake, fake, fake, fake, None) == 5  # NCPA_ETOOMANY
