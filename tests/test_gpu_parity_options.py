"""GPU (C ABI) against the oracle for the reference's solver options and for
reduced shapes of the other workloads:

- ground impedance with the Lamb-wave condition, raised ground, lowered top;
- elevated source and receiver;
- wavenumber filter (c_min, c_max);
- user attenuation table (--use_attn_file);
- many azimuths x log-spaced frequencies in one solve (N x 2-D sweep shape);
- a tall atmosphere at higher frequency (the large-solve shape, reduced);
- the max_modes limit reports NCPA_ETOOMANY.

Tolerances as in test_gpu_parity.py: identical mode counts, Re k within
1e-9 relative (or the conditioning floor), TL within 0.05 dB where
TL > -140 dB, V_s V_r and Im k 1e-6 relative.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = np.finfo(float).eps


def _check(g, o, tl_g=None, tl_o=None):
    assert g.M == o.M, (g.M, o.M)
    if o.M:
        tol = np.maximum(1e-9, 8 * EPS * (4.0 / o.dz ** 2) / (2 * o.kr ** 2))
        assert np.all(np.abs(g.kr - o.kr) / o.kr <= tol)
        assert np.allclose(g.ki, o.ki, rtol=1e-6, atol=1e-18)
        prod = o.vs * o.vr
        assert np.allclose(g.vs * g.vr, prod, rtol=1e-6, atol=1e-12 * np.abs(prod).max())
    if tl_g is not None:
        a, b = 20 * np.log10(np.abs(tl_g)), 20 * np.log10(np.abs(tl_o))
        sel = b > -140.0
        assert np.max(np.abs(a[sel] - b[sel])) < 0.05


def _solve_both(gpu, path, freqs, azs, gkw, okw, attn=None, nr=400, dr=2000.0):
    import ncpa_gpu
    from oracle import oracle as O

    prof = gpu.load_profile(path)
    if attn:
        prof.load_attn(attn)
    m = gpu.solve(prof, ncpa_gpu.default_params(**gkw), freqs, azs)
    re, im, _ = m.tl1d(nr, dr)
    prm = O.EssParams(**okw, use_attn_file=attn or "")
    pp = O.prepare(O.read_profile(path), prm)
    p = 0
    for f in freqs:
        for a in azs:
            o = O.solve_problem(pp, prm, f, a)
            ore, oim, _ = O.tl1d(o, nr, dr)
            _check(m.problem(p), o, re[p] + 1j * im[p], ore + 1j * oim)
            p += 1
    m.close()
    prof.close()


@pytest.mark.parametrize("case", ["lamb", "ground_top", "elevated", "wvnum"])
def test_solver_options(gpu, analytic_profile, case):
    nz = 6000
    g = dict(nz_grid=nz, turnoff_wkb=1)
    o = dict(Nz_grid=nz, turnoff_WKB=True)
    if case == "lamb":
        g["lamb_wave_bc"] = 1
        o["Lamb_wave_BC"] = True
    elif case == "ground_top":
        g.update(zground_km=1.0, maxheight_km=120.0)
        o.update(zground_km=1.0, maxheight_km=120.0)
    elif case == "elevated":
        g.update(sourceheight_km=5.0, receiverheight_km=1.0)
        o.update(sourceheight_km=5.0, receiverheight_km=1.0)
    else:
        g.update(wvnum_filter=1, c_min=300.0, c_max=360.0)
        o.update(wvnum_filter=True, c_min=300.0, c_max=360.0)
    _solve_both(gpu, analytic_profile, [0.2], [90.0], g, o)


def test_user_attenuation_table(gpu, analytic_profile, tmp_path):
    z = np.arange(0.0, 151.0, 5.0)
    a = 1e-7 * np.exp(z / 20.0)
    path = tmp_path / "attn.dat"
    path.write_text("".join("%g %.6e\n" % row for row in zip(z, a)))
    nz = 6000
    _solve_both(gpu, analytic_profile, [0.15, 0.3], [90.0], dict(nz_grid=nz, turnoff_wkb=1),
                dict(Nz_grid=nz, turnoff_WKB=True), attn=str(path))


def test_many_azimuths_log_frequencies(gpu, canonical_profile):
    # the N x 2-D sweep shape, reduced: 12 azimuths x 3 log-spaced frequencies
    freqs = list(np.geomspace(0.1, 0.4, 3))
    azs = list(np.arange(0.0, 360.0, 30.0))
    nz = 5000
    _solve_both(gpu, canonical_profile, freqs, azs, dict(nz_grid=nz), dict(Nz_grid=nz), nr=200, dr=5000.0)


def test_tall_atmosphere_higher_frequency(gpu, workdir):
    # the large-solve shape, reduced: 1 Hz, top 180 km, Nz = 30000 (hundreds of modes)
    import os

    import workloads

    path = workloads.write_profile(os.path.join(str(workdir), "analytic_180km.dat"), top_km=180.0)
    nz = 30000
    _solve_both(gpu, path, [1.0], [90.0], dict(nz_grid=nz, maxheight_km=180.0, turnoff_wkb=1),
                dict(Nz_grid=nz, maxheight_km=180.0, turnoff_WKB=True), nr=300, dr=2000.0)


def test_max_modes_limit(gpu, analytic_profile):
    import ncpa_gpu

    prof = gpu.load_profile(analytic_profile)
    with pytest.raises(ncpa_gpu.NcpaError) as e:
        gpu.solve(prof, ncpa_gpu.default_params(nz_grid=4000, max_modes=5), [0.5], [90.0])
    assert e.value.status == 5  # NCPA_ETOOMANY
    # the context stays usable
    m = gpu.solve(prof, ncpa_gpu.default_params(nz_grid=4000), [0.5], [90.0])
    assert m.count(0) > 5
    m.close()
    prof.close()
