"""Dispersion files on the host (no device): the library's reader follows
ModalBroadbandPropagator::read_dispersion_file (ModalBroadbandPropagator.cpp:
98-138) -- DC slot first, densities of the last line, reading stops at the
first non-number -- and its binary cache returns the same arrays bit for bit,
is used only while its stamp matches the text file, and is rebuilt when the
text changes or the cache is damaged."""
import os

import numpy as np
import pytest

EPARSE = 4


def _write_dispersion(path, rng, n_freq=6):
    """Lines in the format of ModeSolver::writeDispersion (ModeSolver.cpp:569-600)."""
    rows = []
    with open(path, "w") as f:
        for i in range(n_freq):
            fr = 0.01 * (i + 1)
            m = int(rng.integers(0, 7))
            rs, rr = 1.225 - 0.001 * i, 1.2 + 0.002 * i
            kr = np.sort(rng.uniform(1e-3, 5e-3, m))
            vals = np.column_stack([kr, rng.uniform(0, 1e-6, m), rng.normal(size=m), rng.normal(size=m)])
            f.write("%.7e   %d    %.7e   %.7e" % (fr, m, rs, rr))
            for r in vals:
                f.write("   %.12e   %.12e   %.12e   %.12e" % tuple(r))
            f.write("\n")
            rows.append((fr, rs, rr, vals))
    return rows


def _expected(rows):
    """Arrays as parsed from the text (strtod of the printed digits)."""
    f = [0.0] + [float("%.7e" % r[0]) for r in rows]
    off = np.cumsum([0, 0] + [len(r[3]) for r in rows])
    v = np.vstack([np.array([[float("%.12e" % x) for x in row] for row in r[3]]).reshape(-1, 4) for r in rows])
    return np.array(f), off, v, float("%.7e" % rows[-1][1]), float("%.7e" % rows[-1][2])


def test_text_parse_matches_the_reference_rules(tmp_path):
    import ncpa_gpu

    rows = _write_dispersion(tmp_path / "d.dat", np.random.default_rng(1))
    d = ncpa_gpu.read_dispersion(tmp_path / "d.dat")
    f, off, v, rs, rr = _expected(rows)
    assert np.array_equal(d["f"], f) and np.array_equal(d["mode_off"], off)
    assert np.array_equal(np.column_stack([d["kr"], d["ki"], d["vs"], d["vr"]]), v)
    assert (d["rho_src"], d["rho_rcv"]) == (rs, rr) and d["rows"] == len(rows) and d["from_cache"] == 0
    # trailing text that is not a number ends the reading, as in the reference
    with open(tmp_path / "d.dat", "a") as fo:
        fo.write("end of file\n")
    d2 = ncpa_gpu.read_dispersion(tmp_path / "d.dat")
    assert np.array_equal(d2["kr"], d["kr"]) and len(d2["f"]) == len(d["f"])


def test_binary_cache_round_trip_and_invalidation(tmp_path):
    import ncpa_gpu

    txt, cache = tmp_path / "d.dat", tmp_path / "d.cache"
    _write_dispersion(txt, np.random.default_rng(2), n_freq=9)
    a = ncpa_gpu.read_dispersion(txt, cache)
    assert a["from_cache"] == 0 and cache.exists()
    b = ncpa_gpu.read_dispersion(txt, cache)
    assert b["from_cache"] == 1
    for k in ("f", "mode_off", "kr", "ki", "vs", "vr"):
        assert np.array_equal(a[k], b[k]), k
    assert (a["rho_src"], a["rho_rcv"], a["rows"]) == (b["rho_src"], b["rho_rcv"], b["rows"])
    # a changed text file is parsed again and the cache rewritten
    _write_dispersion(txt, np.random.default_rng(3), n_freq=4)
    c = ncpa_gpu.read_dispersion(txt, cache)
    assert c["from_cache"] == 0 and len(c["f"]) == 5
    assert ncpa_gpu.read_dispersion(txt, cache)["from_cache"] == 1
    # a damaged cache is ignored and replaced
    data = cache.read_bytes()
    cache.write_bytes(data[: len(data) // 2])
    d = ncpa_gpu.read_dispersion(txt, cache)
    assert d["from_cache"] == 0 and np.array_equal(d["kr"], c["kr"])
    assert ncpa_gpu.read_dispersion(txt, cache)["from_cache"] == 1


def test_malformed_and_missing_files(tmp_path):
    import ncpa_gpu

    bad = tmp_path / "bad.dat"
    bad.write_text("1.0e-02   2    1.2e+00   1.2e+00   1e-3 1e-9 0.5\n")  # a mode quadruple cut short
    with pytest.raises(ncpa_gpu.NcpaError) as e:
        ncpa_gpu.read_dispersion(bad)
    assert e.value.status == EPARSE
    with pytest.raises(ncpa_gpu.NcpaError) as e:
        ncpa_gpu.read_dispersion(tmp_path / "missing.dat")
    assert e.value.status == EPARSE
    assert not os.path.exists(tmp_path / "missing.cache")
