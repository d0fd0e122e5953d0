"""The fused bisection + eigenvector launch (k_bisect_eigvec) against the two
kernels run one after the other, and its fallback: eigenvector items that a
consumer warp gives up on (empty queue slot after the wait limit) are run by
the k_eigvec launch that follows.  All three must give the same modes bit for
bit: the per-item code is shared, only who runs an item changes.

The switches are read when a context is created (NCPA_FUSE_SOLVE,
NCPA_FUSE_WAIT_NS), so each variant gets its own context."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solve(path, env, method=0):
    import ncpa_gpu

    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        ctx = ncpa_gpu.Context(0)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    prof = ctx.load_profile(path)
    freqs = np.linspace(0.01, 0.4, 24)
    m = ctx.solve(prof, ncpa_gpu.default_params(nz_grid=8000, turnoff_wkb=1, method=method), freqs, [90.0, 200.0])
    out = [m.problem(p) for p in range(m.P)]
    m.close()
    prof.close()
    ctx.close()
    return out


@pytest.mark.parametrize("method", [0, 1])
def test_fused_unfused_and_fallback_identical(analytic_profile, method):
    fused = _solve(analytic_profile, {"NCPA_FUSE_SOLVE": "1"}, method)
    plain = _solve(analytic_profile, {"NCPA_FUSE_SOLVE": "0"}, method)
    # consumers give up at once on an empty slot: the items are split
    # between the fused launch and the following one
    fallback = _solve(analytic_profile, {"NCPA_FUSE_SOLVE": "1", "NCPA_FUSE_WAIT_NS": "0"}, method)
    assert len(fused) == len(plain) == len(fallback) == 48
    assert sum(p.M for p in fused) > 1000
    for a, b, c in zip(fused, plain, fallback):
        assert a.M == b.M == c.M
        for f in ("kr", "ki", "vs", "vr"):
            assert np.array_equal(getattr(a, f), getattr(b, f))
            assert np.array_equal(getattr(a, f), getattr(c, f))


@pytest.mark.parametrize("method", [0, 1])
def test_timing_that_keeps_the_fused_launch(gpu, analytic_profile, method):
    """set_timing(2) times the fused launch as one phase ("bisect+eigvec") and
    gives the modes of an untimed solve bit for bit; set_timing(1) times the
    kernels apart ("bisect", "eigvec")."""
    import ncpa_gpu

    prof = gpu.load_profile(analytic_profile)
    freqs = np.linspace(0.01, 0.4, 24)
    prm = ncpa_gpu.default_params(nz_grid=8000, turnoff_wkb=1, method=method)

    def solve():
        m = gpu.solve(prof, prm, freqs, [90.0])
        out = [m.problem(p) for p in range(m.P)]
        m.close()
        return out

    ref = solve()
    for mode, phase, other in ((2, "bisect+eigvec", "bisect"), (1, "bisect", "bisect+eigvec")):
        gpu.reset_stats()
        gpu.set_timing(mode)
        got = solve()
        gpu.set_timing(False)
        ms, n = gpu.phase_stats(phase)
        assert n == 1 and ms > 0, (mode, phase, ms, n)
        assert gpu.phase_stats(other)[1] == 0, (mode, other)
        for a, b in zip(ref, got):
            assert a.M == b.M
            for k in ("kr", "ki", "vs", "vr"):
                assert np.array_equal(getattr(a, k), getattr(b, k)), (mode, k)
    prof.close()


@pytest.mark.parametrize("method", [0, 1])
def test_bisection_scheduling_modes_identical(analytic_profile, method):
    """The bisection item scheduler (cost-ordered items, two warps per warp
    scheduler taking items from the two ends of the list) decides only which
    warp runs an item: plain round-robin, other worker counts, and letting
    every warp of the fused launch take eigenvector items give the same modes
    bit for bit."""
    ref = _solve(analytic_profile, {}, method)
    variants = (
        {"NCPA_BISECT_ORDER": "0"},
        {"NCPA_BISECT_WORKERS": "1"},
        {"NCPA_BISECT_WORKERS": "3", "NCPA_FUSE_EV_WORKERS": "0"},
        {"NCPA_FUSE_SOLVE": "0"},
    )
    for env in variants:
        got = _solve(analytic_profile, env, method)
        assert len(got) == len(ref)
        for a, b in zip(ref, got):
            assert a.M == b.M, env
            for f in ("kr", "ki", "vs", "vr"):
                assert np.array_equal(getattr(a, f), getattr(b, f)), (env, f)


def test_scheduler_with_more_problems_than_the_ranking_covers(analytic_profile):
    """Above 4096 problems the item list stays in problem order (no cost
    ranking); the scheduler still runs every item once: same modes as plain
    round-robin."""
    import ncpa_gpu

    def solve(env):
        old = {k: os.environ.get(k) for k in env}
        os.environ.update(env)
        try:
            ctx = ncpa_gpu.Context(0)
        finally:
            for k, v in old.items():
                if v is None:
                    os.environ.pop(k, None)
                else:
                    os.environ[k] = v
        prof = ctx.load_profile(analytic_profile)
        freqs = np.linspace(0.005, 0.05, 41)
        az = np.linspace(0.0, 357.0, 101)
        m = ctx.solve(prof, ncpa_gpu.default_params(nz_grid=1500, turnoff_wkb=1, max_modes=200), freqs, az)
        assert m.P == 4141
        off, kr, ki, vs, vr, _ = m.all_modes()
        out = (off.copy(), kr.copy(), ki.copy(), vs.copy(), vr.copy())
        m.close()
        prof.close()
        ctx.close()
        return out

    a = solve({})
    b = solve({"NCPA_BISECT_ORDER": "0"})
    assert a[0][-1] > 4141
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_scan_trim_keeps_counts_and_modes(analytic_profile):
    """The isolation scan's batch-wide trim (whole units per warp scheduler,
    claimed per scheduler) only changes the bisection's starting brackets:
    on the 256-frequency job (1329 units trimmed to 1184) mode counts are
    identical and the modes agree with the untrimmed scan's within the
    bisection tolerance."""
    import ncpa_gpu
    import workloads

    def solve(env):
        old = {k: os.environ.get(k) for k in env}
        os.environ.update(env)
        try:
            ctx = ncpa_gpu.Context(0)
        finally:
            for k, v in old.items():
                if v is None:
                    os.environ.pop(k, None)
                else:
                    os.environ[k] = v
        prof = ctx.load_profile(analytic_profile)
        m = ctx.solve(prof, ncpa_gpu.default_params(nz_grid=20000, turnoff_wkb=1),
                      workloads.broadband_freqs(256, 0.5), [90.0])
        off, kr, ki, vs, vr, _ = m.all_modes()
        out = (off.copy(), kr.copy(), ki.copy(), vs * vr)
        m.close()
        prof.close()
        ctx.close()
        return out

    a = solve({})
    b = solve({"NCPA_SCAN_TRIM": "0"})
    assert np.array_equal(a[0], b[0]) and a[0][-1] > 30000
    # the bisection stops within 1e-15 (units of h^2 A) of each eigenvalue from
    # either set of brackets; the parity bound on k is 1e-9 relative
    assert np.max(np.abs(a[1] - b[1]) / b[1]) < 1e-9
    assert np.max(np.abs(a[2] - b[2]) / np.abs(b[2])) < 1e-6
    assert np.max(np.abs(a[3] - b[3])) < 1e-6 * np.max(np.abs(b[3]))
