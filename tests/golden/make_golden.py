"""Regenerates the golden fixtures of this directory from the reference tree.

Reads the reference's shipped example outputs and sample profile (run once,
where the reference checkout is available) and writes compact copies:

  canonical_profile.dat.gz   samples/NCPA_canonical_profile_zuvwtdp.dat
  g2s_profile.sample.gz      samples/g2sprofile.sample (G2S layout: a
                             "Profile at (lat, lon)" line, then Z T U V P RHO)
  modess_tloss_1d.npz        docs/.../modess_gp_files/code_outputs/tloss_1d.nm
                             and tloss_1d.lossless.nm (Modess, 0.1 Hz, az 90,
                             pre-2.0.1 TL scaling: +60 dB vs the current code)
  wmod_tloss_1d.npz          docs/.../wmod_gp_files/code_outputs/wtloss_1d.nm and
                             wtloss_1d.lossless.nm (WMod, 0.1 Hz, az 90, with
                             --write_2d_tloss, pre-2.0.1 TL scaling)
  dispersion_goldens.npz     per-frequency mode counts, plus Re k / Im k /
                             V_s V_r at a few frequencies, of
                             samples/disp_256freqs_0p5hz_NCPA_canonic.dat and
                             docs/.../modbb_gp_files/code_outputs/myDispersionFile.dat
  modbb_synthesis.npz        the ModBB pulse-propagation example of the manual
                             (docs/.../modbb_gp_files/code_outputs, prop.sh):
                             the whole myDispersionFile.dat (input), the
                             source_spectrum.dat of the built-in pulse, the
                             single-range waveform mywavf.dat (270 km) and the
                             grid mywavf_grid.dat (220-300 km every 20 km),
                             all with --max_celerity 320 and 16384-point
                             transforms; time columns stored as (first, step)

Usage: python tests/golden/make_golden.py <reference_root>
"""
import gzip
import os
import sys

import numpy as np

if len(sys.argv) != 2:
    sys.exit("usage: make_golden.py <reference_root>")
REF = sys.argv[1]
OUT = os.path.dirname(os.path.abspath(__file__))


def read_dispersion(path):
    toks = open(path).read().split()
    i, rows = 0, []
    while i < len(toks):
        f, m = float(toks[i]), int(toks[i + 1])
        i += 4
        vals = np.array([float(x) for x in toks[i:i + 4 * m]]).reshape(m, 4)
        i += 4 * m
        rows.append((f, vals))
    return rows


def main():
    prof = os.path.join(REF, "samples", "NCPA_canonical_profile_zuvwtdp.dat")
    for src, dst in ((prof, "canonical_profile.dat.gz"),
                     (os.path.join(REF, "samples", "g2sprofile.sample"), "g2s_profile.sample.gz")):
        with open(src, "rb") as fi, open(os.path.join(OUT, dst), "wb") as raw, \
                gzip.GzipFile(fileobj=raw, mode="wb", compresslevel=9, mtime=0) as fo:
            fo.write(fi.read())
    co = os.path.join(REF, "docs", "ncpaprop_run_manual_TeX", "figs", "modess_gp_files", "code_outputs")
    lossy = np.loadtxt(os.path.join(co, "tloss_1d.nm"))
    lossless = np.loadtxt(os.path.join(co, "tloss_1d.lossless.nm"))
    np.savez_compressed(os.path.join(OUT, "modess_tloss_1d.npz"), lossy=lossy, lossless=lossless)
    wo = os.path.join(REF, "docs", "ncpaprop_run_manual_TeX", "figs", "wmod_gp_files", "code_outputs")
    np.savez_compressed(os.path.join(OUT, "wmod_tloss_1d.npz"), lossy=np.loadtxt(os.path.join(wo, "wtloss_1d.nm")),
                        lossless=np.loadtxt(os.path.join(wo, "wtloss_1d.lossless.nm")))
    sets = {
        "s256": os.path.join(REF, "samples", "disp_256freqs_0p5hz_NCPA_canonic.dat"),
        "manual": os.path.join(REF, "docs", "ncpaprop_run_manual_TeX", "figs", "modbb_gp_files", "code_outputs",
                               "myDispersionFile.dat"),
    }
    out = {}
    for key, path in sets.items():
        rows = read_dispersion(path)
        out[key + "_f"] = np.array([r[0] for r in rows])
        out[key + "_M"] = np.array([len(r[1]) for r in rows])
        pick = [0, len(rows) // 5, len(rows) // 2, len(rows) - 1]
        out[key + "_pick"] = np.array(pick)
        for j in pick:
            out["%s_modes_%d" % (key, j)] = rows[j][1]
    np.savez_compressed(os.path.join(OUT, "dispersion_goldens.npz"), **out)

    # ModBB pulse propagation example
    bo = os.path.join(REF, "docs", "ncpaprop_run_manual_TeX", "figs", "modbb_gp_files", "code_outputs")
    rows = read_dispersion(os.path.join(bo, "myDispersionFile.dat"))
    head = open(os.path.join(bo, "myDispersionFile.dat")).readline().split()
    modes = np.concatenate([r[1] for r in rows])
    spec = np.loadtxt(os.path.join(bo, "source_spectrum.dat"))
    single = np.loadtxt(os.path.join(bo, "mywavf.dat"))
    grid = np.loadtxt(os.path.join(bo, "mywavf_grid.dat"))

    def regular(t):
        step = (t[-1] - t[0]) / (len(t) - 1)
        assert np.max(np.abs(t - (t[0] + step * np.arange(len(t))))) < 1e-5
        return np.array([t[0], step])

    g_r = np.unique(grid[:, 0])
    g_amp = np.stack([grid[grid[:, 0] == r][:, 2] for r in g_r])
    np.savez_compressed(
        os.path.join(OUT, "modbb_synthesis.npz"),
        disp_f=np.array([r[0] for r in rows]), disp_M=np.array([len(r[1]) for r in rows], dtype=np.int32),
        disp_rho=np.array([float(head[2]), float(head[3])]), disp_modes=modes,
        spec_f=spec[:, 0], spec_re=spec[:, 1], spec_im=spec[:, 2],
        single_t=regular(single[:, 0]), single_re=single[:, 1].astype(np.float32),
        single_im=single[:, 2].astype(np.float32),
        grid_r_km=g_r, grid_t=regular(grid[grid[:, 0] == g_r[0]][:, 1]), grid_amp=g_amp.astype(np.float32))


if __name__ == "__main__":
    main()
