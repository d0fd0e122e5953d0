"""G2S-style profile ingestion (host side, no device): the reference's
samples/g2sprofile.sample layout -- a "Profile at (lat, lon)" line, then
Z [km] T [K] U V [m/s] P [mbar] RHO [g/cm3] -- converted to the NCPA profile
format that Atmosphere1D reads (Atmosphere1D.cpp:85-285), checked value for
value and through the oracle's own profile reader."""
import gzip
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN

EPARSE = 4


@pytest.fixture(scope="module")
def g2s_sample(tmp_path_factory):
    path = tmp_path_factory.mktemp("g2s") / "g2sprofile.sample"
    with gzip.open(os.path.join(GOLDEN, "g2s_profile.sample.gz"), "rb") as fi:
        path.write_bytes(fi.read())
    return path


def _columns(path):
    rows = [ln.split() for ln in open(path) if ln.strip() and ln.strip()[0].isdigit()]
    return np.array(rows, dtype=float)


def test_convert_keeps_every_value_and_the_location(g2s_sample, tmp_path):
    import ncpa_gpu

    out = tmp_path / "converted.dat"
    lat, lon = ncpa_gpu.g2s_convert(g2s_sample, out)
    assert (lat, lon) == (35.528, -90.146)
    src = _columns(g2s_sample)                       # Z T U V P RHO
    header = [ln for ln in open(out) if ln.startswith("#%")]
    assert header == ["#% 1, Z, km\n", "#% 2, U, m/s\n", "#% 3, V, m/s\n", "#% 4, T, K\n",
                      "#% 5, RHO, g/cm3\n", "#% 6, P, mbar\n"]
    got = np.loadtxt(out, comments="#")
    assert got.shape == (len(src), 6)
    for gcol, scol in ((0, 0), (1, 2), (2, 3), (3, 1), (4, 5), (5, 4)):
        assert np.array_equal(got[:, gcol], src[:, scol])


def test_converted_file_reads_through_the_oracle(g2s_sample, tmp_path):
    import ncpa_gpu
    from oracle import oracle as O

    out = tmp_path / "converted.dat"
    ncpa_gpu.g2s_convert(g2s_sample, out)
    prof = O.read_profile(str(out))
    src = _columns(g2s_sample)
    assert prof.z_units == "km" and np.array_equal(prof.z, src[:, 0])
    for key, col, unit, si_unit, scale in (("T", 1, "K", "K", 1.0), ("U", 2, "m/s", "m/s", 1.0),
                                           ("V", 3, "m/s", "m/s", 1.0), ("P", 4, "mbar", "Pa", 100.0),
                                           ("RHO", 5, "g/cm3", "kg/m3", 1000.0)):
        vals, units = prof.vectors[key]
        assert units == unit and np.array_equal(vals, src[:, col])
        assert np.array_equal(O.to_si(vals, units, si_unit), src[:, col] * scale)


def test_location_line_is_optional_and_bad_rows_fail(tmp_path):
    import ncpa_gpu

    good = tmp_path / "noloc.txt"
    good.write_text("# comment\n0.0 288 1 0 1013 0.001225\n1.0 281 2 0 900 0.0011\n2.0 275 3 0 800 0.001\n")
    lat, lon = ncpa_gpu.g2s_convert(good, tmp_path / "noloc.dat")
    assert math.isnan(lat) and math.isnan(lon)
    bad = tmp_path / "bad.txt"
    bad.write_text("Profile at (1.0, 2.0)\n0.0 288 1 0 1013\n1.0 281 2 0 900 0.0011\n2.0 275 3 0 800 0.001\n")
    with pytest.raises(ncpa_gpu.NcpaError) as e:
        ncpa_gpu.g2s_convert(bad, tmp_path / "bad.dat")
    assert e.value.status == EPARSE
