"""The identity behind the bisection kernel's twisted Sturm sweeps (k_bisect,
warp_sweep_tw_mode): for a tridiagonal T with unit off-diagonal, the forward
recurrence p over rows [0, h) and the backward recurrence q over rows
[h, n) (q_n = 1, q_{n+1} = 0) give

    #eig(T) < x = SC(p_{-1} .. p_{h-1}) + SC(q_n .. q_{h+1}) + [gamma_h < 0],
    gamma_h = det / (p_{h-1} q_{h+1}),  det = p_{h-1} q_h - p_{h-2} q_{h+1},

(SC = sign changes) and det' by the product rule from the chains'
derivatives.  Checked here against LAPACK's eigenvalues and the sequential
recurrence on random matrices, every split point, and a row-0 term entering
as p_{-2} (the wide-angle ground condition)."""
import numpy as np
import pytest


def _chain(rows, x, p0=0.0):
    p1, cnt, prev, d0, d1 = 1.0, 0, 0, 0.0, 0.0
    for si in rows:
        a = si - x
        q = a * p1 - p0
        e = a * d1 - (p1 + d0)
        b = int(np.signbit(q))
        cnt += b ^ prev
        prev = b
        p0, p1, d0, d1 = p1, q, d1, e
    return cnt, p0, p1, d0, d1


def _twisted(s, x, h, p_init):
    cf, f0, f1, fd0, fd1 = _chain(s[:h], x, p_init)
    cb, b0, b1, bd0, bd1 = _chain(s[h:][::-1], x)
    det = f1 * b1 - f0 * b0
    dd = fd1 * b1 + f1 * bd1 - fd0 * b0 - f0 * bd0
    sb = lambda v: int(np.signbit(v))
    return cf + cb - (sb(b1) ^ sb(b0)) + (sb(det) ^ sb(f1) ^ sb(b0)), det, dd


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_twisted_count_equals_inertia(seed):
    rng = np.random.default_rng(seed)
    for trial in range(40):
        n = int(rng.integers(2, 40))
        s = rng.normal(-2.0, 0.4, n)
        p_init = float(rng.uniform(-1.0, 0.0)) if trial % 2 else 0.0
        T = np.diag(s) + np.diag(np.ones(n - 1), 1) + np.diag(np.ones(n - 1), -1)
        T[0, 0] -= p_init  # q_0 = t_0 - p_{-2}
        ev = np.linalg.eigvalsh(T)
        for x in rng.uniform(ev.min() - 0.5, ev.max() + 0.5, 6):
            exact = int(np.sum(ev < x))
            c_seq, _, p_seq, _, d_seq = _chain(s, x, p_init)
            assert c_seq == exact
            for h in range(1, n):
                c, det, dd = _twisted(s, x, h, p_init)
                assert c == exact, (n, h, x)
                assert det == pytest.approx(p_seq, rel=1e-9, abs=1e-12 * abs(p_seq))
                assert dd == pytest.approx(d_seq, rel=1e-8, abs=1e-10 * abs(d_seq))
