"""Modess / ModBB front ends: option handling (CPU) and the files they write
(GPU), checked against the oracle.

The front ends keep the reference's options, defaults, validation messages,
file names and fprintf formats (Modess_main.cpp, ModBB_main.cpp,
ModeSolver.cpp:292-641, ESSModeSolver.cpp:670-752,
ModalBroadbandPropagator.cpp:141-231, BroadbandPropagator.cpp:360-414)."""
import math
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "ncpaprop-release_b200")
BIN = os.path.join(PKG, "bin")
PI = math.pi


@pytest.fixture(scope="module")
def binaries():
    if not (os.path.exists(os.path.join(BIN, "Modess")) and os.path.exists(os.path.join(BIN, "ModBB"))):
        env = dict(os.environ)
        env.pop("CC", None)
        env.pop("CXX", None)
        subprocess.run(["make", "-s", "-C", PKG, "all"], check=True, env=env)
    return BIN


def run(binaries, prog, args, cwd, check_rc=None):
    p = subprocess.run([os.path.join(binaries, prog)] + args, cwd=cwd, capture_output=True, text=True,
                       timeout=600)
    if check_rc is not None:
        assert p.returncode == check_rc, p.stdout + p.stderr
    return p


# ---------------------------------------------------------------------------
# CPU: option parsing and validation (no GPU needed: validation fails first)
# ---------------------------------------------------------------------------
def test_help_returns_1(binaries, tmp_path):
    for prog in ("Modess", "ModBB"):
        p = run(binaries, prog, ["--help"], tmp_path)
        assert p.returncode == 1
        assert "--" in p.stdout


def test_modess_validation_messages(binaries, tmp_path):
    p = run(binaries, "Modess", [], tmp_path, check_rc=0)
    out = p.stdout
    assert "Parameter validation failed:" in out
    assert "atmosfile is not present." in out
    assert "freq is not present." in out
    assert "operation_mode: 0 of { singleprop, multiprop } are present; must be one and only one." in out
    p = run(binaries, "Modess", ["--singleprop", "--freq", "-1", "--atmosfile", "x", "--Nz_grid", "5",
                                 "--azimuth", "400", "--ground_impedence_model", "soft"], tmp_path, check_rc=0)
    out = p.stdout
    assert "freq (-1.000000) must be greater than 0.000000." in out
    assert "Nz_grid (5) must be greater than or equal to 10." in out
    assert "azimuth (400.000000) must be less than 360.000000." in out
    assert 'ground_impedence_model: "soft" is not in { rigid }.' in out
    p = run(binaries, "Modess", ["--multiprop", "--freq", "0.1", "--atmosfile", "x", "--wvnum_filter"], tmp_path,
            check_rc=0)
    for k in ("azimuth_start", "azimuth_end", "azimuth_step"):
        assert "One of { multiprop } is set, but %s is not set." % k in p.stdout
    for k in ("c_min", "c_max"):
        assert "One of { wvnum_filter } is set, but %s is not set." % k in p.stdout


def test_modbb_validation_messages(binaries, tmp_path):
    p = run(binaries, "ModBB", ["--dispersion", "--method", "foo"], tmp_path, check_rc=0)
    out = p.stdout
    assert 'method: "foo" is not in { modess, wmod }.' in out
    for k in ("dispersion_file", "azimuth", "f_min", "f_max", "f_step", "atmosfile"):
        assert "One of { dispersion } is set, but %s is not set." % k in out
    p = run(binaries, "ModBB", ["--propagation", "--source", "chirp", "--nfft", "-4"], tmp_path, check_rc=0)
    out = p.stdout
    assert 'source: "chirp" is not in { impulse, pulse1, pulse2, waveform, spectrum }.' in out
    assert "nfft (-4) must be greater than or equal to 0." in out
    for k in ("input_dispersion_file", "output_waveform_file"):
        assert "One of { propagation } is set, but %s is not set." % k in out


def test_param_file_and_unknown_option(binaries, tmp_path):
    # "key: value" lines in modess.param count as given; the command line is
    # parsed again afterwards, so it wins
    (tmp_path / "modess.param").write_text("# comment\nfreq: 0.3\natmosfile = prof.dat\nsingleprop\n"
                                           "azimuth 45\nNz_grid: 5\n")
    p = run(binaries, "Modess", ["--Nz_grid", "20"], tmp_path)
    assert "freq is not present" not in p.stdout
    assert "atmosfile is not present" not in p.stdout
    assert "Nz_grid (5)" not in p.stdout
    assert "operation_mode" not in p.stdout
    p = run(binaries, "Modess", ["--bogus", "3"], tmp_path, check_rc=0)
    assert "Unknown option '--bogus'." in p.stdout


# ---------------------------------------------------------------------------
# GPU: files written by the front ends against the oracle
# ---------------------------------------------------------------------------
NZ = 4000


def _tl_db(re_, im_):
    return 20 * np.log10(np.hypot(re_, im_))


def _check_tl(rows_re, rows_im, ore, oim):
    a, b = _tl_db(rows_re, rows_im), _tl_db(ore, oim)
    sel = b > -140.0
    assert sel.sum() > 0.5 * len(b)
    assert np.max(np.abs(a[sel] - b[sel])) < 0.05


@pytest.fixture(scope="module")
def modess_single(binaries, analytic_profile, tmp_path_factory):
    from oracle import oracle as O

    d = tmp_path_factory.mktemp("modess_single")
    args = ["--singleprop", "--atmosfile", analytic_profile, "--freq", "0.1", "--azimuth", "90",
            "--Nz_grid", str(NZ), "--maxrange_km", "500", "--Nrng_steps", "250", "--write_lossless",
            "--write_phase_speeds", "--write_speeds", "--write_modes", "--write_2d_tloss",
            "--modal_starter_file", "starter.nm", "--dispersion_file", "disp.dat", "--write_atm_profile",
            "--filetag", "run"]
    p = run(binaries, "Modess", args, d, check_rc=0)
    prm = O.EssParams(Nz_grid=NZ, turnoff_WKB=True)
    pp = O.prepare(O.read_profile(analytic_profile), prm)
    o = O.solve_problem(pp, prm, 0.1, 90.0, want_group=True, want_full=True)
    return d, o, p.stdout


@pytest.mark.gpu
def test_modess_tloss_1d_files(modess_single):
    from oracle import oracle as O

    d, o, _ = modess_single
    dr = 500e3 / 250
    for name, lossless in (("run.tloss_1d.nm", False), ("run.tloss_1d.lossless.nm", True)):
        lines = (d / name).read_text().splitlines()
        assert len(lines) == 250
        assert re.fullmatch(r"\d+\.\d{6}( +-?\d\.\d{12}e[+-]\d\d){3}", lines[0]), lines[0]
        a = np.loadtxt(d / name)
        assert np.allclose(a[:, 0], (np.arange(250) + 1) * dr / 1000.0)
        ore, oim, oinc = O.tl1d(o, 250, dr, lossless)
        _check_tl(a[:, 1], a[:, 2], ore, oim)
        assert np.max(np.abs(20 * np.log10(a[:, 3] / oinc))) < 0.05


@pytest.mark.gpu
def test_modess_mode_outputs(modess_single):
    d, o, _ = modess_single
    ph = np.loadtxt(d / "run.phasespeeds.nm", ndmin=2)
    assert ph.shape[0] == o.M
    assert np.array_equal(ph[:, 0], np.arange(o.M))
    assert np.max(np.abs(ph[:, 1] - 2 * PI * 0.1 / o.kr)) < 2e-6
    assert np.allclose(ph[:, 2], o.ki, rtol=1e-6, atol=1e-20)
    sp = np.loadtxt(d / "run.speeds.nm", ndmin=2)
    assert np.array_equal(sp[:, 0], np.arange(1, o.M + 1))
    assert np.max(np.abs(sp[:, 2] - o.vg)) < 2e-3
    first = (d / "run.speeds.nm").read_text().splitlines()[0]
    assert re.fullmatch(r" {0,3}\d+ +\d+\.\d{3} +\d+\.\d{3} +-?\d\.\d{8}e[+-]\d\d", first), first
    # eigenfunctions: one file per mode, Nz rows, unit norm, the oracle's up to sign
    for j in (0, o.M // 2, o.M - 1):
        m = np.loadtxt(d / ("run.mode_%d.nm" % j))
        assert m.shape == (NZ, 2)
        assert abs(np.sum(m[:, 1] ** 2) * o.dz - 1.0) < 1e-5
        ref = o.vfull[:, j]
        s = np.sign(np.dot(m[:, 1], ref))
        assert np.max(np.abs(s * m[:, 1] - ref)) < 1e-6 * np.max(np.abs(ref)) + 1e-7
    assert not (d / ("run.mode_%d.nm" % o.M)).exists()


@pytest.mark.gpu
def test_modess_dispersion_line(modess_single):
    d, o, _ = modess_single
    toks = (d / "disp.dat").read_text().split()
    assert float(toks[0]) == pytest.approx(0.1) and int(toks[1]) == o.M
    assert float(toks[2]) == pytest.approx(o.rho_s, rel=2e-7)
    v = np.array(toks[4:], dtype=float).reshape(o.M, 4)
    assert np.max(np.abs(v[:, 0] - o.kr) / o.kr) < 1e-9
    assert np.allclose(v[:, 1], o.ki, rtol=1e-6, atol=1e-20)
    assert np.max(np.abs(v[:, 2] * v[:, 3] - o.vs * o.vr)) < 1e-6 * np.max(np.abs(o.vs * o.vr))


@pytest.mark.gpu
def test_modess_2d_and_starter(modess_single):
    d, o, _ = modess_single
    stepj = NZ // 500
    blocks = (d / "run.tloss_2d.nm").read_text().strip("\n").split("\n\n")
    assert len(blocks) == 250
    a = np.array([[float(x) for x in ln.split()] for ln in blocks[99].splitlines()])
    r = 100 * 2000.0
    js = np.arange(0, NZ, stepj)
    assert a.shape == (len(js), 4)
    assert np.allclose(a[:, 1], js * o.dz / 1000.0, atol=1e-6)
    k = o.kr + 1j * o.ki
    terms = o.vs[None, :] * o.vfull[js, :] * np.exp(1j * k * r) / np.sqrt(k)
    ref = 1000.0 * (4 * PI * 1j * np.exp(-1j * PI / 4) / np.sqrt(8 * PI)) * terms.sum(axis=1) / np.sqrt(r)
    sel = np.abs(ref) > 1e-7 * np.abs(ref).max()
    _check_tl(a[sel, 2], a[sel, 3], ref.real[sel], ref.imag[sel])
    # modal starter (ESSModeSolver.cpp:670-723)
    st = np.loadtxt(d / "run.starter.nm")
    step = int((340.0 / 0.1) / 10 / o.dz)
    js = np.arange(0, NZ, step)
    ref = PI * np.sqrt(2 * PI * 0.1 / 340.0) * (o.vs[None, :] * o.vfull[js, :] / np.sqrt(o.kr)).sum(axis=1)
    assert st.shape == (len(js), 3)
    assert np.max(np.abs(st[:, 1] - ref)) < 1e-6 * np.max(np.abs(ref))
    assert np.all(st[:, 2] == 0.0)


@pytest.mark.gpu
def test_modess_2d_tloss_on_tensor_cores(modess_single, binaries, analytic_profile, tmp_path):
    """Modess --write_2d_tloss with NCPA_TL2D_SUM=3 writes tloss_2d.nm from the
    guarded tcgen05 modal sum: the same layout as the FP64 file and TL within
    0.05 dB of it wherever TL > -140 dB."""
    d, _, _ = modess_single
    args = ["--singleprop", "--atmosfile", analytic_profile, "--freq", "0.1", "--azimuth", "90",
            "--Nz_grid", str(NZ), "--maxrange_km", "500", "--Nrng_steps", "250", "--write_2d_tloss",
            "--filetag", "tc"]
    p = subprocess.run([os.path.join(binaries, "Modess")] + args, cwd=tmp_path, capture_output=True, text=True,
                       timeout=600, env=dict(os.environ, NCPA_TL2D_SUM="3"))
    assert p.returncode == 0, p.stdout + p.stderr
    ref = np.loadtxt(d / "run.tloss_2d.nm")
    got = np.loadtxt(tmp_path / "tc.tloss_2d.nm")
    assert got.shape == ref.shape
    assert np.array_equal(got[:, :2], ref[:, :2])
    tl_ref, tl_got = _tl_db(ref[:, 2], ref[:, 3]), _tl_db(got[:, 2], got[:, 3])
    sel = tl_ref > -140.0
    assert sel.mean() > 0.5
    assert np.max(np.abs(tl_got[sel] - tl_ref[sel])) < 0.05


@pytest.mark.gpu
def test_modess_atm_profile(modess_single, analytic_profile):
    from oracle import oracle as O

    d, _, _ = modess_single
    txt = (d / "run.atm_profile.nm").read_text().splitlines()
    assert txt[0] == "#% 0, Z0, m, 0" and txt[1] == "#% 0, AZ, deg CW from N, 90"
    assert txt[2:10] == ["#% 1, Z, m", "#% 2, U, m/s", "#% 3, V, m/s", "#% 4, T, K", "#% 5, RHO, kg/m3",
                         "#% 6, P, Pa", "#% 7, C0, m/s", "#% 8, CEFF, m/s"]
    a = np.loadtxt(d / "run.atm_profile.nm", comments="#")
    prof = O.read_profile(analytic_profile)
    assert a.shape[1] == 8  # Z U V T RHO P C0 CEFF
    assert np.allclose(a[:, 0], np.asarray(prof.z) * 1000.0, rtol=1e-6)
    c0 = np.sqrt(1.4 * a[:, 5] / a[:, 4])
    assert np.allclose(a[:, 6], c0, rtol=2e-6)
    assert np.allclose(a[:, 7], a[:, 6] + a[:, 1], rtol=2e-6, atol=1e-5)  # azimuth 90: c_eff = c0 + u


@pytest.mark.gpu
def test_modess_multiprop(binaries, analytic_profile, tmp_path):
    from oracle import oracle as O

    args = ["--multiprop", "--atmosfile", analytic_profile, "--freq", "0.1", "--azimuth_start", "0",
            "--azimuth_end", "90", "--azimuth_step", "45", "--Nz_grid", str(NZ), "--maxrange_km", "400",
            "--Nrng_steps", "200"]
    run(binaries, "Modess", args, tmp_path, check_rc=0)
    blocks = (tmp_path / "Nby2D_tloss_1d.nm").read_text().strip("\n").split("\n\n")
    assert len(blocks) == 3
    prm = O.EssParams(Nz_grid=NZ)
    pp = O.prepare(O.read_profile(analytic_profile), prm)
    for b, az in zip(blocks, (0.0, 45.0, 90.0)):
        lines = b.splitlines()
        assert re.fullmatch(r" +\d+\.\d{3} +\d+\.\d{3}( +-?\d\.\d{12}e[+-]\d\d){3}", lines[0]), lines[0]
        a = np.array([[float(x) for x in ln.split()] for ln in lines])
        assert np.all(a[:, 1] == az)
        o = O.solve_problem(pp, prm, 0.1, az)
        ore, oim, _ = O.tl1d(o, 200, 2000.0)
        _check_tl(a[:, 2], a[:, 3], ore, oim)


@pytest.fixture(scope="module")
def modbb_dispersion(binaries, analytic_profile, tmp_path_factory):
    d = tmp_path_factory.mktemp("modbb")
    args = ["--dispersion", "--method", "modess", "--dispersion_file", "disp.dat", "--atmosfile", analytic_profile,
            "--azimuth", "90",
            "--f_min", "0.01", "--f_step", "0.005", "--f_max", "0.085", "--Nz_grid", str(NZ)]
    (d / "disp.dat").write_text("stale line that --dispersion truncates\n")
    run(binaries, "ModBB", args, d, check_rc=0)
    return d


@pytest.mark.gpu
def test_modbb_dispersion_file(modbb_dispersion, analytic_profile):
    from oracle import oracle as O

    d = modbb_dispersion
    lines = (d / "disp.dat").read_text().splitlines()
    assert len(lines) == 16
    prm = O.EssParams(Nz_grid=NZ, turnoff_WKB=True)
    pp = O.prepare(O.read_profile(analytic_profile), prm)
    for i, ln in enumerate(lines):
        f = 0.01 + i * 0.005
        assert re.match(r"\d\.\d{7}e[+-]\d\d   \d+    \d\.\d{7}e[+-]\d\d   \d\.\d{7}e[+-]\d\d", ln), ln
        toks = ln.split()
        o = O.solve_problem(pp, prm, f, 90.0)
        assert float(toks[0]) == pytest.approx(f, rel=1e-7) and int(toks[1]) == o.M
        v = np.array(toks[4:], dtype=float).reshape(o.M, 4)
        assert np.max(np.abs(v[:, 0] - o.kr) / o.kr) < 1e-9
    # the last frequency's 1-D TL is what remains in tloss_1d.nm
    assert len((d / "tloss_1d.nm").read_text().splitlines()) == 1000


@pytest.mark.gpu
@pytest.mark.parametrize("source", ["pulse1", "waveform", "impulse"])
def test_modbb_propagation_files(binaries, modbb_dispersion, source, tmp_path):
    from oracle import oracle as O

    import workloads

    disp = str(modbb_dispersion / "disp.dat")
    args = ["--propagation", "--input_dispersion_file", disp, "--output_waveform_file", "wave.dat",
            "--receiver", "multiple", "--start_range_km", "100", "--end_range_km", "200", "--range_step_km", "50",
            "--source", source, "--max_celerity", "330"]
    wf = None
    if source == "waveform":
        wf = workloads.write_waveform(str(tmp_path / "ricker.dat"))
        args += ["--source_file", wf]
    run(binaries, "ModBB", args, tmp_path, check_rc=0)
    d = O.read_dispersion(disp)
    nf = len(d.f)
    f_step = d.f[2] - d.f[1]
    lines_wf = None
    if wf:
        tw, xw = np.loadtxt(wf, unpack=True)
        lines_wf = len(tw)
    nfft = O.bb_nfft(nf, 0, lines_wf)
    if wf:
        sre, sim = O.source_spectrum("waveform", d.f, nfft, waveform=(tw, xw))
    else:
        sre, sim = O.source_spectrum(source, d.f, nfft)
    spec = np.loadtxt(tmp_path / "source_spectrum_input.dat")
    assert spec.shape == (nf, 3)
    assert np.allclose(spec[:, 0], d.f, atol=1e-9)
    s = sre + 1j * sim
    assert np.max(np.abs(spec[:, 1] + 1j * spec[:, 2] - s)) < 1e-5 * np.max(np.abs(s))
    src = np.loadtxt(tmp_path / "source_waveform_input.dat")
    assert src.shape == (nfft // 2, 2)
    fmx = nfft * f_step
    assert np.allclose(src[:, 0], np.arange(nfft // 2) / fmx, atol=1e-6)
    if wf:
        ref = np.zeros(nfft)
        ref[: len(xw)] = xw
    else:
        pad = np.zeros(nfft, complex)
        pad[:nf] = s
        ref = 2.0 * (f_step * np.fft.fft(pad)).real
    ref = ref[: nfft // 2]
    assert np.linalg.norm(src[:, 1] - ref) <= 1e-4 * np.linalg.norm(ref)
    blocks = (tmp_path / "wave.dat").read_text().strip("\n").split("\n\n")
    assert len(blocks) == 3
    for b, r in zip(blocks, (100e3, 150e3, 200e3)):
        lines = b.splitlines()
        assert len(lines) == nfft
        assert re.fullmatch(r" +\d+\.\d{3} +-?\d+\.\d{6} +-?\d\.\d{6}e[+-]\d\d", lines[0]), lines[0]
        a = np.array([[float(x) for x in ln.split()] for ln in lines])
        t0 = r / 330.0
        assert np.allclose(a[:, 1], np.arange(nfft) / fmx + t0, atol=2e-6)
        hre, him = O.bb_transfer(d, r)
        ref = O.bb_pulse(d, sre, sim, hre, him, t0, nfft)
        assert np.linalg.norm(a[:, 2] - ref) <= 1e-4 * np.linalg.norm(ref)


@pytest.mark.gpu
def test_modbb_propagation_with_dispersion_cache(binaries, modbb_dispersion, tmp_path):
    """--dispersion_cache: the first run writes the binary cache, the second
    reads it; both write the same waveform file byte for byte as a run
    without the option."""
    disp = str(modbb_dispersion / "disp.dat")
    base = ["--propagation", "--input_dispersion_file", disp, "--output_waveform_file", "wave.dat",
            "--receiver", "single", "--range_km", "150", "--source", "pulse1", "--max_celerity", "330"]
    outs = []
    for i, extra in enumerate(([], ["--dispersion_cache", str(tmp_path / "disp.cache")],
                               ["--dispersion_cache", str(tmp_path / "disp.cache")])):
        d = tmp_path / ("run%d" % i)
        d.mkdir()
        p = run(binaries, "ModBB", base + extra, d, check_rc=0)
        outs.append(((d / "wave.dat").read_bytes(), p.stdout))
    assert outs[0][0] == outs[1][0] == outs[2][0]
    assert "dispersion cache" not in outs[1][1] and "dispersion cache" in outs[2][1]


@pytest.mark.gpu
def test_modbb_propagation_reference_example(binaries, tmp_path):
    """ModBB --propagation on the reference's example dispersion file with the
    built-in pulse, 220-300 km every 20 km, max_celerity 320, 16384-point
    transform, against the shipped mywavf_grid.dat (older release: times
    without t0, pulse scale 1.6191256 / 2, taper one bin lower -> ~5e-5)."""
    z = np.load(os.path.join(ROOT, "tests", "golden", "modbb_synthesis.npz"))
    disp = tmp_path / "myDispersionFile.dat"
    md = z["disp_modes"]
    rho_s, rho_r = z["disp_rho"]
    with open(disp, "w") as f:
        k = 0
        for fr, m in zip(z["disp_f"], z["disp_M"]):
            f.write("%.7e   %d    %.7e   %.7e" % (fr, m, rho_s, rho_r))
            for row in md[k:k + m]:
                f.write("   %.12e   %.12e   %.12e   %.12e" % tuple(row))
            f.write("\n")
            k += m
    args = ["--propagation", "--input_dispersion_file", str(disp), "--output_waveform_file", "wave.dat",
            "--receiver", "multiple", "--start_range_km", "220", "--end_range_km", "300", "--range_step_km", "20",
            "--source", "pulse1", "--max_celerity", "320", "--nfft", "16384"]
    run(binaries, "ModBB", args, tmp_path, check_rc=0)
    blocks = (tmp_path / "wave.dat").read_text().strip("\n").split("\n\n")
    assert len(blocks) == 5
    for i, b in enumerate(blocks):
        a = np.array([[float(x) for x in ln.split()] for ln in b.splitlines()])
        assert a.shape == (16384, 3)
        r_km = z["grid_r_km"][i]
        assert np.allclose(a[:, 0], r_km)
        t0 = r_km * 1e3 / 320.0
        assert np.allclose(a[:, 1] - t0, z["grid_t"][0] + z["grid_t"][1] * np.arange(16384), atol=2e-6)
        ref = z["grid_amp"][i].astype(float)
        g = a[:, 2] * (1.6191256 / 2.0)
        assert np.linalg.norm(g - ref) <= 1e-4 * np.linalg.norm(ref)


@pytest.mark.gpu
def test_solver_class_takes_the_callers_atmosphere(binaries, canonical_profile, tmp_path):
    """ESSModeSolver(Params*, Atmosphere1D*) -- the reference's
    ESSModeSolver(ParameterSet*, Atmosphere1D*) (ESSModeSolver.h:53-80): a
    profile changed in memory gives the same files as the same profile
    written out and read back, and not those of the unchanged profile."""
    obj = os.path.join(PKG, "_obj")
    exe = str(tmp_path / "solver_atmosphere")
    cmd = ["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(PKG, "csrc"),
           os.path.join(ROOT, "tests", "cpp", "solver_atmosphere.cpp")]
    cmd += [os.path.join(obj, o) for o in ("cli_params.o", "cli_common.o", "cli_ess.o", "cli_bb.o", "solvers.o")]
    cmd += ["-L" + os.path.join(PKG, "lib"), "-lncpa_gpu", "-Wl,-rpath," + os.path.join(PKG, "lib"), "-o", exe]
    subprocess.run(cmd, check=True)
    p = subprocess.run([exe, canonical_profile, str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    for name in ("tloss_1d.nm", "tloss_2d.nm"):
        mem = (tmp_path / ("mem." + name)).read_bytes()
        assert mem == (tmp_path / ("file." + name)).read_bytes(), name
        assert mem != (tmp_path / ("orig." + name)).read_bytes(), name
