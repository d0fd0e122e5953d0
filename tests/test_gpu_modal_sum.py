"""Modal sum at many receivers (ncpa_tl_multi): the FP64 CUDA-core sum and the
tcgen05 tensor-core sums against an FP64 NumPy sum of the same modes, and end
to end against the oracle's modes.

The guarded tensor-core sum (NCPA_SUM_TC_GUARDED: 6-term split-BF16, points
whose |P| is below its error bound recomputed in FP64) must give TL within
0.05 dB of the FP64 sum at EVERY point where TL > -140 dB, nulls included.

The unguarded tensor-core sums carry a stated error only: split-BF16 (3
terms) |P_tc - P| is at most 2e-4 of S = sum_m |A_jm e^{i k_m r}| (the modal
terms' magnitude), and TL is within 0.05 dB wherever TL > -140 dB and
|P| > 1e-3 S (outside deep cancellation nulls, where no fixed relative
precision suffices).  TF32 (10-bit mantissa operands): |P_tf32 - P| at most
2e-3 of S, TL within 0.1 dB where TL > -140 dB and |P| > 2e-2 S."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PI = np.pi


def _ref_sum(kr, ki, vs, vz, n_ranges, dr, lossless=False):
    k = kr + 1j * (0.0 if lossless else ki)
    A = vs[None, :] * vz / np.sqrt(k)[None, :]                 # [J, M]
    r = (np.arange(n_ranges) + 1) * dr
    E = np.exp(1j * np.outer(k, r))                              # [M, N]
    C = 1000.0 * 4 * PI * 1j * np.exp(-1j * PI / 4) / np.sqrt(8 * PI * r)
    P = (A @ E) * C[None, :]
    S = (np.abs(A) @ np.abs(E)) * np.abs(C)[None, :]
    return P, S


@pytest.fixture(scope="module")
def solved(gpu, analytic_profile):
    import ncpa_gpu

    prof = gpu.load_profile(analytic_profile)
    nz = 8000
    m = gpu.solve(prof, ncpa_gpu.default_params(nz_grid=nz, want_vectors=1, turnoff_wkb=1), [0.5], [90.0])
    g = m.problem(0)
    v = m.vectors(0, nz)
    yield m, g, v, nz
    m.close()
    prof.close()


def _heights(n, dz, top_m=10000.0):
    return np.linspace(0.0, top_m, n) // dz * dz  # on grid points


@pytest.mark.parametrize("n_rcv,n_ranges,dr", [(64, 1000, 500.0), (100, 700, 1000.0), (7, 300, 2000.0)])
def test_fp64_and_tensor_core_sums(solved, n_rcv, n_ranges, dr):
    m, g, v, nz = solved
    dz = g.dz
    h = _heights(n_rcv, dz)
    idx = np.ceil(h / dz).astype(int)
    P, S = _ref_sum(g.kr, g.ki, g.vs, v[idx, :], n_ranges, dr)
    p64 = m.tl_multi(0, h, n_ranges, dr, method=m.SUM_FP64)
    assert np.max(np.abs(p64 - P) / S) < 1e-10
    ptc = m.tl_multi(0, h, n_ranges, dr, method=m.SUM_TC_BF16X3)
    err = np.abs(ptc - P) / S
    assert np.max(err) < 2e-4, np.max(err)
    tl_ref = 20 * np.log10(np.abs(P))
    tl_tc = 20 * np.log10(np.abs(ptc))
    sel = (tl_ref > -140.0) & (np.abs(P) > 1e-3 * S)
    assert sel.mean() > 0.8
    assert np.max(np.abs(tl_tc[sel] - tl_ref[sel])) < 0.05


def test_tensor_core_lossless_and_ground_row_matches_1d(solved):
    m, g, v, nz = solved
    dr, n_ranges = 1000.0, 400
    h = np.array([0.0, 1000.0, 5000.0])
    ptc = m.tl_multi(0, h, n_ranges, dr, method=m.SUM_TC_BF16X3, lossless=True)
    idx = np.ceil(h / g.dz).astype(int)
    P, S = _ref_sum(g.kr, g.ki, g.vs, v[idx, :], n_ranges, dr, lossless=True)
    assert np.max(np.abs(ptc - P) / S) < 2e-4
    # ground receiver, lossy: the same numbers as the 1-D TL of the solve
    p0 = m.tl_multi(0, h[:1], n_ranges, dr, method=m.SUM_TC_BF16X3)[0]
    re, im, _ = m.tl1d(n_ranges, dr)
    p1 = re[0] + 1j * im[0]
    _, S0 = _ref_sum(g.kr, g.ki, g.vs, v[idx[:1], :], n_ranges, dr)
    assert np.max(np.abs(p0 - p1) / S0[0]) < 2e-4


def test_tensor_core_sum_against_oracle_modes(solved, analytic_profile):
    from oracle import oracle as O

    m, g, v, nz = solved
    prm = O.EssParams(Nz_grid=nz, turnoff_WKB=True)
    o = O.solve_problem(O.prepare(O.read_profile(analytic_profile), prm), prm, 0.5, 90.0, want_full=True)
    assert o.M == g.M
    h = _heights(64, g.dz)
    idx = np.ceil(h / g.dz).astype(int)
    P, S = _ref_sum(o.kr, o.ki, o.vs, o.vfull[idx, :], 1000, 500.0)
    ptc = m.tl_multi(0, h, 1000, 500.0, method=m.SUM_TC_BF16X3)
    tl_ref = 20 * np.log10(np.abs(P))
    sel = (tl_ref > -140.0) & (np.abs(P) > 1e-3 * S)
    assert np.max(np.abs(20 * np.log10(np.abs(ptc[sel])) - tl_ref[sel])) < 0.05


@pytest.mark.parametrize("n_rcv,n_ranges,dr", [(64, 1000, 500.0), (100, 700, 1000.0), (7, 300, 2000.0)])
def test_tf32_tensor_core_sum(solved, n_rcv, n_ranges, dr):
    m, g, v, nz = solved
    h = _heights(n_rcv, g.dz)
    idx = np.ceil(h / g.dz).astype(int)
    P, S = _ref_sum(g.kr, g.ki, g.vs, v[idx, :], n_ranges, dr)
    p32 = m.tl_multi(0, h, n_ranges, dr, method=m.SUM_TC_TF32)
    err = np.abs(p32 - P) / S
    assert np.max(err) < 2e-3, np.max(err)
    tl_ref = 20 * np.log10(np.abs(P))
    sel = (tl_ref > -140.0) & (np.abs(P) > 2e-2 * S)
    assert sel.mean() > 0.5
    assert np.max(np.abs(20 * np.log10(np.abs(p32[sel])) - tl_ref[sel])) < 0.1
    # the split-BF16 sum is the more accurate of the two
    ptc = m.tl_multi(0, h, n_ranges, dr, method=m.SUM_TC_BF16X3)
    assert np.max(np.abs(ptc - P) / S) < np.max(err)


@pytest.mark.parametrize("n_rcv,n_ranges,dr,lossless", [(64, 1000, 500.0, False), (100, 700, 1000.0, False),
                                                       (7, 300, 2000.0, False), (64, 600, 500.0, True)])
def test_guarded_tensor_core_sum_every_point(gpu, solved, n_rcv, n_ranges, dr, lossless):
    m, g, v, nz = solved
    h = _heights(n_rcv, g.dz)
    idx = np.ceil(h / g.dz).astype(int)
    P, S = _ref_sum(g.kr, g.ki, g.vs, v[idx, :], n_ranges, dr, lossless=lossless)
    pg = m.tl_multi(0, h, n_ranges, dr, method=m.SUM_TC_GUARDED, lossless=lossless)
    fixed, points = gpu.sum_fixups()
    eps, tau, tile = gpu.sum_guard()
    assert tile > 0
    assert points == n_rcv * n_ranges and 0 <= fixed < points
    # the guard's error model: |P_tc - P| <= eps S (S here at the point's own
    # range, which is at most the tile-start S the guard uses)
    err = np.abs(pg - P) / S
    assert 0 < eps < tau and np.max(err) < eps, (np.max(err), eps)
    tl_ref = 20 * np.log10(np.abs(P))
    sel = tl_ref > -140.0
    assert sel.mean() > 0.9
    assert np.max(np.abs(20 * np.log10(np.abs(pg[sel])) - tl_ref[sel])) <= 0.05


def test_guarded_sum_is_reproducible(solved):
    m, g, v, nz = solved
    h = _heights(64, g.dz)
    a = m.tl_multi(0, h, 800, 500.0, method=m.SUM_TC_GUARDED)
    b = m.tl_multi(0, h, 800, 500.0, method=m.SUM_TC_GUARDED)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("method", [1, 2, 3])
def test_schedule_autotuner_keeps_the_sums(solved, method, monkeypatch):
    """The first tensor-core call of a shape times every ring-depth schedule
    and keeps the fastest; whatever it picks, the sums equal those of a
    context that keeps the default schedule (NCPA_MS_TUNE=0), bit for bit."""
    import ncpa_gpu

    m, g, v, nz = solved
    h = _heights(70, g.dz)
    tuned = m.tl_multi(0, h, 900, 500.0, method=method)
    ts, gs, times = m.ctx.sum_schedule()
    assert len(times) >= 2 and np.all(times > 0) and ts >= 2 and gs >= 1
    monkeypatch.setenv("NCPA_MS_TUNE", "0")
    own = m.ctx
    with ncpa_gpu.Context(0) as plain_ctx:
        m.ctx = plain_ctx  # the same modes, summed on a context that does not tune
        try:
            plain = m.tl_multi(0, h, 900, 500.0, method=method)
            ts0, gs0, _ = plain_ctx.sum_schedule()
        finally:
            m.ctx = own
    assert (ts0, gs0) == ((3, 2) if method == 3 else (4, 3))
    assert np.array_equal(tuned, plain)
