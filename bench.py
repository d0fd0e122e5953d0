"""Benchmark of the B200 ESS normal-mode path (ModBB broadband workload).

One step = the whole ModBB job of the 256-frequency case on the analytic
0-150 km atmosphere: the batched dispersion solve (256 frequencies
df = 0.5/256 Hz, Nz = 20000, one azimuth), the 1-D transmission loss of every
frequency on 1000 ranges to 1000 km (ModBB --dispersion writes it per
frequency), then pulse synthesis at 200-300 km every 10 km from a
Gaussian-windowed 0.1 Hz Ricker waveform sampled at 1 Hz.

The line also carries "modal_sum": the tensor-core modal sum at 64
receivers x 20000 ranges of a 2 Hz, Nz = 100000 solve (timed separately,
not part of the step), with its roofline against the measured bf16 peak,
and "serving": a seeded request stream replayed in real time through the
serving loop and through the plain one-request-at-a-time path (p50 / p99
latency, throughput), and "sweep": 360 azimuths x 8 frequencies with Nz per
frequency (5000-60000) as one batched solve, and "wmod": the same
256-frequency dispersion + 1-D TL with the wide-angle solver (ModBB
--method wmod), with its bisection roofline and its own CPU baseline.

  value  freq-solves/s with the profile resident in HBM and results left in
         HBM (device-timed with CUDA events on the library's stream; L2
         flushed between steps by writing a 256 MiB buffer)
  e2e    the same through the C ABI with host buffers: profile knots and the
         source waveform go up, dispersion, TL and waveforms come back, every
         step

Multi-GPU (torchrun): every rank solves its own independent 256-frequency
job (weak scaling, no data-path collective); time = max over ranks.

--impl reference times the CPU restatement of the reference algorithm (the
reference itself cannot be built here: PETSc/SLEPc/GSL/FFTW are absent) on
the host cores, on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "ncpaprop-release_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

import workloads  # noqa: E402

METRIC = "freq-solves/s"
NZ = 20000
NFREQ = 256
RANGES_KM = np.arange(200.0, 300.0 + 1e-9, 10.0)
MAX_CEL = 340.0
N_TL = 1000
DR_TL = 1000.0


def _dist():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def _nfft(nfreq_with_dc, n_wave):
    nfft = 4 * nfreq_with_dc
    while n_wave > nfft:
        nfft *= 2
    return nfft


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed
    region: NVML polled every 2 ms from a thread (the same counters
    nvidia-smi reports), or nvidia-smi -lms 20 where NVML is unavailable.
    Read-only: nothing here changes a GPU setting."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []
        self.samples = []  # (sm MHz, max sm MHz, set of reason names)
        self.source = None

    def _nvml_handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        u = str(torch.cuda.get_device_properties(self.device).uuid)
        return pynvml, pynvml.nvmlDeviceGetHandleByUUID(u if u.startswith("GPU-") else "GPU-" + u)

    def _poll_nvml(self, nv, h):
        bits = ((nv.nvmlClocksEventReasonHwSlowdown, "hw_slowdown"),
                (nv.nvmlClocksEventReasonHwThermalSlowdown, "hw_thermal_slowdown"),
                (nv.nvmlClocksEventReasonSwThermalSlowdown, "sw_thermal_slowdown"),
                (nv.nvmlClocksEventReasonSwPowerCap, "sw_power_cap"))
        smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        while not self.halt.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            except Exception:
                break
            self.samples.append((sm, smax, {nm for b, nm in bits if r & b}))
            self.halt.wait(0.002)

    def start(self):
        self.halt = threading.Event()
        try:
            nv, h = self._nvml_handle()
            self.t = threading.Thread(target=self._poll_nvml, args=(nv, h), daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.samples and time.time() - t0 < 5.0 and self.t.is_alive():
                time.sleep(0.001)
            if self.samples:
                self.source = "nvml, 2 ms"
                return
            self.halt.set()
        except Exception:
            pass
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # sampling is live before the timed region starts
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.005)
            self.n_before = len(self.lines)
            self.source = "nvidia-smi -lms 20"
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.source and self.source.startswith("nvml"):
            self.halt.set()
            self.t.join(timeout=5)
            got = self.samples[1:] or self.samples
        elif self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            got = []
            for ln in self.lines[getattr(self, "n_before", 0):] or self.lines[-1:]:
                f = [x.strip() for x in ln.split(",")]
                if len(f) < 9:
                    continue
                try:
                    got.append((float(f[1]), float(f[2]),
                                {nm for nm, v in zip(self.NAMES, f[5:9]) if v.lower() == "active"}))
                except ValueError:
                    continue
        else:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        sm = [g[0] for g in got]
        reasons = set().union(*(g[2] for g in got)) if got else set()
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_min_mhz": min(sm) if sm else None,
                "sm_max_mhz": max(g[1] for g in got) if got else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": self.source}


def reduce_max(values):
    """Element-wise max over the ranks of the initialised process group (the
    slowest rank's device time is the job's time)."""
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor(values, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    import ncpa_gpu

    rank, world, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize()

    ctx = ncpa_gpu.Context(local)
    tmp = tempfile.mkdtemp(prefix="ncpa_bench_")
    prof_path = workloads.write_profile(os.path.join(tmp, "analytic_150km.dat"))
    z, u, v, t, p, rho = workloads.si_arrays()
    t_w, x_w = workloads.ricker_waveform()
    freqs = workloads.broadband_freqs(NFREQ, 0.5)
    az = [(90.0 + 10.0 * rank) % 360.0]
    ranges_m = RANGES_KM * 1000.0
    nf_dc = len(freqs) + 1
    nfft = _nfft(nf_dc, len(x_w))
    prof = ctx.load_profile(prof_path)
    params_dev = ncpa_gpu.default_params(nz_grid=NZ, turnoff_wkb=1, keep_on_device=1)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    # pinned host buffers for the end-to-end leg
    pin = {k: torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for k, a in
           dict(z=z, u=u, v=v, t=t, p=p, rho=rho, x=x_w, f=freqs).items()}
    # pinned host buffers the results of the end-to-end leg land in
    pin_tl = [torch.empty((NFREQ, N_TL), dtype=torch.float64).pin_memory().numpy() for _ in range(3)]
    pin_wav = torch.empty((len(RANGES_KM), nfft), dtype=torch.float64).pin_memory().numpy()
    # pinned buffers for the modes (k, attenuation, source / receiver values,
    # group speeds), sized after the first end-to-end step
    pin_modes = []

    def step_device():
        sre, sim = ctx.source_spectrum_waveform(x_w, t_w[1] - t_w[0], nfft, nf_dc)
        m = ctx.solve(prof, params_dev, freqs, az)
        m.tl1d(N_TL, DR_TL, to_host=False)
        m.bb_synthesize(ranges_m, MAX_CEL, nfft, sre, sim, to_host=False)
        m.close()

    h2d = [0]
    d2h = [0]

    def step_e2e():
        pr = ctx.profile_from_arrays(*(pin[k].numpy() for k in ("z", "u", "v", "t", "p", "rho")))
        xw = pin["x"].numpy()
        sre, sim = ctx.source_spectrum_waveform(xw, t_w[1] - t_w[0], nfft, nf_dc)
        m = ctx.solve(pr, params_dev, pin["f"].numpy(), az)
        if not pin_modes or pin_modes[0].size < m.total_modes():
            pin_modes[:] = [torch.empty(m.total_modes(), dtype=torch.float64).pin_memory().numpy() for _ in range(5)]
        disp = m.all_modes(out=pin_modes)  # CSR offsets + k, attenuation, source / receiver values, group speeds
        tl = m.tl1d(N_TL, DR_TL, out=pin_tl)
        wav = m.bb_synthesize(ranges_m, MAX_CEL, nfft, sre, sim, out=pin_wav)
        nm = int(disp[0][-1])
        h2d[0] = 6 * len(z) * 8 + len(xw) * 8 + len(freqs) * 8
        d2h[0] = nm * 5 * 8 + sum(a.nbytes for a in tl) + wav.nbytes + 2 * nf_dc * 8
        m.close()
        pr.close()

    def timed(fn, k):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
        barrier()
        for i in range(k):
            flush.zero_()
            torch.cuda.synchronize()
            ev[i][0].record(stream)
            fn()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        barrier()
        return sum(a.elapsed_time(b) for a, b in ev)

    for _ in range(args.warmup):
        step_device()
    if not args.quick:
        for _ in range(max(1, min(args.warmup, 2))):
            step_e2e()
    # timed device-resident leg (clocks sampled throughout)
    l0 = ctx.launches
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    ms_dev = timed(step_device, args.steps)
    launches = (ctx.launches - l0) // args.steps
    # per-phase kernel times from CUDA events, in separate untimed steps
    n_ph = max(2, min(args.steps, 5))
    ctx.reset_stats()
    ctx.set_timing(True)
    for _ in range(n_ph):
        flush.zero_()
        step_device()
    torch.cuda.synchronize()
    ctx.set_timing(False)
    bis_ms, bis_n = ctx.phase_stats("bisect")
    sturm_steps, deriv_steps = ctx.bisect_steps()
    phases = {ph: ctx.phase_stats(ph)[0] / n_ph for ph in
              ("knots+grid", "matrix", "window", "scan", "host-items", "bisect", "eigvec", "fetch")}
    # the fused bisection + eigenvector launch the timed steps run, timed alone
    ctx.reset_stats()
    ctx.set_timing(2)
    for _ in range(n_ph):
        flush.zero_()
        step_device()
    torch.cuda.synchronize()
    ctx.set_timing(False)
    fused_ms, fused_n = ctx.phase_stats("bisect+eigvec")
    phases["bisect+eigvec (fused)"] = fused_ms / max(fused_n, 1)
    phases["eigvec-rest"] = ctx.phase_stats("eigvec-rest")[0] / n_ph
    m_cnt = ctx.solve(prof, params_dev, freqs, az)
    modes_total = m_cnt.total_modes()
    m_cnt.close()
    if args.quick:
        if sampler:
            sampler.stop()
        print(json.dumps({"quick": True, "ms_per_step": ms_dev / args.steps,
                          "phases_ms": {k: round(v, 4) for k, v in phases.items()}}), flush=True)
        prof.close()
        ctx.close()
        return
    ms_e2e = timed(step_e2e, args.steps)
    if sampler:
        clocks = sampler.stop()
    # plain per-frequency GPU path: one ncpa_ess_solve per frequency
    plain_freqs = freqs[::16]
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for f in plain_freqs:
        m = ctx.solve(prof, params_dev, [f], az)
        m.tl1d(N_TL, DR_TL, to_host=False)
        m.close()
    ev1.record(stream)
    torch.cuda.synchronize()
    plain_rate = len(plain_freqs) / (ev0.elapsed_time(ev1) / 1e3)

    if world > 1:
        ms_dev, ms_e2e = reduce_max([ms_dev, ms_e2e])
    fp64_peak = ctx.fp64_peak_tflops() if rank == 0 else None
    ms_leg = modal_sum_leg(ctx, stream, _bf16_peak()) if rank == 0 and not args.no_modal_sum else None
    sv_leg = serving_leg(ctx) if rank == 0 and not args.no_serving else None
    sw_leg = sweep_leg(ctx, stream) if rank == 0 and not args.no_sweep else None
    wm_leg = wmod_leg(ctx, stream, prof, freqs, az, fp64_peak, flush, args.cpu_seconds) \
        if rank == 0 and not args.no_wmod else None
    if rank == 0:
        solves = NFREQ * args.steps * world
        value = solves / (ms_dev / 1e3)
        e2e_value = solves / (ms_e2e / 1e3)
        # bisection kernel roofline, steps counted by the kernel: 3 FP64 flops
        # per step of a count-only chain (subtract + fused multiply-add), 10
        # per step of a Laguerre chain (p, p', p'': subtract, four FMAs, one add)
        flops = 3.0 * (sturm_steps - deriv_steps) + 10.0 * deriv_steps  # over the bis_n timed launches
        achieved = flops / (bis_ms / 1e3) / 1e12 if bis_ms > 0 else None
        # the fused launch: the same bisection work plus the reduction-only
        # eigenvector items, 7 flops per row and pass (square, add, multiply-
        # add with the weight, subtract, multiply-add of the recurrence), two
        # passes per mode
        ev_flops = 14.0 * NZ * modes_total
        fused_flops = (flops / bis_n if bis_n else 0.0) + ev_flops
        fused_launch_ms = fused_ms / max(fused_n, 1)
        fused_achieved = fused_flops / (fused_launch_ms / 1e3) / 1e12 if fused_ms > 0 else None
        cpu = cpu_baseline(freqs, max_seconds=args.cpu_seconds)
        cpu_lapack = lapack_baseline(freqs) if not args.no_lapack else None
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_dev / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "ModBB 256-frequency dispersion + 1-D TL + pulse synthesis",
                       "profile": "analytic 0-150 km (T piecewise linear, 60+20 m/s jets)", "nz_grid": NZ,
                       "n_freq": NFREQ, "df_hz": 0.5 / NFREQ, "azimuth_deg": az[0], "tl_ranges": N_TL,
                       "synthesis_ranges_km": "200-300/10", "nfft": nfft, "l2": "flushed (256 MiB write) between steps",
                       "eigen_solve": "fused bisection + eigenvector launch in the timed steps; phases_ms and the "
                                      "roofline time k_bisect and k_eigvec alone (per-phase timing runs them "
                                      "separately) and the fused launch alone (roofline.fused)",
                       "parallelism": "replicas (one 256-frequency job per GPU)"},
            "e2e": {"value": round(e2e_value, 2), "unit": METRIC, "h2d_bytes_per_step": int(h2d[0]),
                    "d2h_bytes_per_step": int(d2h[0])},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "roofline": {"kernel": "k_bisect (Sturm multisection)", "bound": "fp64",
                         "achieved": round(achieved, 3) if achieved else None, "peak": round(fp64_peak, 3),
                         "unit": "TFLOP/s", "frac": round(achieved / fp64_peak, 4) if achieved else None,
                         "peak_source": "measured in this run (dependent-FMA probe on all SMs)",
                         "traffic": None, "traffic_source": "not measured by this run (DRAM counters need ncu)",
                         "avg_launch_ms": round(bis_ms / max(bis_n, 1), 4),
                         "flops_per_launch": flops / bis_n if bis_n else None,
                         "flops": "3 per count-chain step, 10 per Laguerre-chain step (p, p', p'')",
                         "chain_steps_per_launch": sturm_steps / bis_n if bis_n else None,
                         "laguerre_chain_steps_per_launch": deriv_steps / bis_n if bis_n else None,
                         "fused": {"kernel": "k_bisect_eigvec (the launch the timed steps run)",
                                   "avg_launch_ms": round(fused_launch_ms, 4),
                                   "flops_per_launch": fused_flops,
                                   "achieved": round(fused_achieved, 3) if fused_achieved else None,
                                   "frac": round(fused_achieved / fp64_peak, 4) if fused_achieved else None,
                                   "flops": "the bisection's counted flops + 14 per grid row per mode for the "
                                            "two eigenvector passes (%d modes)" % modes_total}},
            "phases_ms": {k: round(v, 4) for k, v in phases.items()},
            "plain_gpu": {"value": round(plain_rate, 2), "unit": METRIC,
                          "what": "one ncpa_ess_solve + TL per frequency, same workload"},
            "cpu_baseline": cpu,
            "cpu_lapack": cpu_lapack,
            "modal_sum": ms_leg,
            "serving": sv_leg,
            "sweep": sw_leg,
            "wmod": wm_leg,
        }
        print(json.dumps(line), flush=True)
    for h in (prof,):
        h.close()
    ctx.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# modal sum at 64 receivers on the tensor cores (tall-atmosphere workload)
# ---------------------------------------------------------------------------
MS_NZ, MS_FREQ, MS_TOP_KM, MS_NR, MS_DR, MS_RCV = 100000, 2.0, 180.0, 20000, 100.0, 64


def _tl2d_at_scale(m, path, n_ranges=2000, dr=1000.0, reps=3):
    """The 2-D TL of ncpa_tl_2d (the reference's tloss_2d.nm: every
    Nz/500-th height) on the same 2 Hz, Nz = 100000 modes: the FP64
    CUDA-core sum of m's context against the guarded tensor-core sum of a
    context created with NCPA_TL2D_SUM=3 (its own solve, untimed).  Times are
    whole calls (results copied to host memory)."""
    import ncpa_gpu

    def timed(mm):
        mm.tl2d(0, n_ranges, dr)
        t0 = time.perf_counter()
        for _ in range(reps):
            out = mm.tl2d(0, n_ranges, dr)
        return (time.perf_counter() - t0) * 1e3 / reps, out

    ms64, (z, re64, im64) = timed(m)
    old = os.environ.get("NCPA_TL2D_SUM")
    os.environ["NCPA_TL2D_SUM"] = "3"
    try:
        ctx2 = ncpa_gpu.Context(0)
    finally:
        if old is None:
            os.environ.pop("NCPA_TL2D_SUM", None)
        else:
            os.environ["NCPA_TL2D_SUM"] = old
    prof2 = ctx2.load_profile(path)
    m2 = ctx2.solve(prof2, ncpa_gpu.default_params(nz_grid=MS_NZ, maxheight_km=MS_TOP_KM, want_vectors=1,
                                                   turnoff_wkb=1), [MS_FREQ], [90.0])
    mstc, (_, retc, imtc) = timed(m2)
    m2.close()
    prof2.close()
    ctx2.close()
    tl64 = 20 * np.log10(np.maximum(np.hypot(re64, im64), 1e-300))
    tltc = 20 * np.log10(np.maximum(np.hypot(retc, imtc), 1e-300))
    sel = tl64 > -140.0
    return {"workload": "ncpa_tl_2d (tloss_2d.nm): %d heights x %d ranges x %d km, same modes" %
                        (len(z), n_ranges, int(dr / 1000)),
            "ms_per_call_fp64": round(ms64, 3), "ms_per_call_tc_guarded": round(mstc, 3),
            "tl_db_max": float(np.abs(tltc - tl64)[sel].max()),
            "where": "every point with TL > -140 dB (%d of %d)" % (int(sel.sum()), sel.size)}


def modal_sum_leg(ctx, stream, bf16, k=10):
    """Solve the 2 Hz, 180 km, Nz = 100000 problem once (untimed), then time
    the modal sum at 64 receivers (0-10 km) x 20000 ranges (0.1 km to 2000 km)
    through ncpa_tl_multi: the guarded tensor-core sum (6-term split-BF16 with
    FP64 recomputation of the points its error bound flags), the unguarded
    3-term split-BF16 and TF32 sums, and the FP64 CUDA-core sum; errors of
    each against the FP64 sum over the whole grid."""
    import torch
    import ncpa_gpu

    bf16_peak, peak_source = bf16
    tmp = tempfile.mkdtemp(prefix="ncpa_ms_")
    path = workloads.write_profile(os.path.join(tmp, "analytic_180km.dat"), top_km=MS_TOP_KM)
    prof = ctx.load_profile(path)
    m = ctx.solve(prof, ncpa_gpu.default_params(nz_grid=MS_NZ, maxheight_km=MS_TOP_KM, want_vectors=1,
                                                turnoff_wkb=1), [MS_FREQ], [90.0])
    M = m.count(0)
    h = np.linspace(0.0, 10000.0, MS_RCV)
    G, X3, T32, F64 = m.SUM_TC_GUARDED, m.SUM_TC_BF16X3, m.SUM_TC_TF32, m.SUM_FP64

    def timed(method, reps):
        for _ in range(2):
            m.tl_multi(0, h, MS_NR, MS_DR, method=method, to_host=False)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(reps):
            m.tl_multi(0, h, MS_NR, MS_DR, method=method, to_host=False)
        ev1.record(stream)
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1) / reps

    def kernel_ms(method):
        """ms of the tensor-core kernel per call, and of each phase"""
        ctx.reset_stats()
        ctx.set_timing(True)
        for _ in range(k):
            m.tl_multi(0, h, MS_NR, MS_DR, method=method, to_host=False)
        ctx.set_timing(False)
        ph = {n: ctx.phase_stats(n) for n in ("ms-prep", "ms-tc", "ms-finish", "ms-fix")}
        per = {n: round(t / max(c, 1), 4) for n, (t, c) in ph.items() if c > 0}
        return per["ms-tc"], per

    ms_call_g = timed(G, k)
    sched_ts, sched_gs, sched_times = ctx.sum_schedule()
    ms_call = timed(X3, k)
    ms_call_tf32 = timed(T32, k)
    ms_fp64 = timed(F64, 2)
    ms_kernel_g, phases_g = kernel_ms(G)
    ms_kernel, phases = kernel_ms(X3)
    ms_kernel_tf32, phases_tf32 = kernel_ms(T32)
    p_64 = m.tl_multi(0, h, MS_NR, MS_DR, method=F64)
    p_g = m.tl_multi(0, h, MS_NR, MS_DR, method=G)
    fixed, points = ctx.sum_fixups()
    p_tc = m.tl_multi(0, h, MS_NR, MS_DR, method=X3)
    p_32 = m.tl_multi(0, h, MS_NR, MS_DR, method=T32)
    tl2d = _tl2d_at_scale(m, path)
    m.close()
    prof.close()
    alg = 8.0 * MS_RCV * M * MS_NR          # complex multiply-adds x 8 flops
    tl64 = 20 * np.log10(np.abs(p_64))
    sel = tl64 > -140.0

    def err(p):
        d = np.abs(20 * np.log10(np.abs(p)) - tl64)[sel]
        rel = np.abs(p - p_64).max(axis=1) / np.abs(p_64).max(axis=1)
        return {"max_abs_over_max_P": float(rel.max()), "tl_db_median": float(np.median(d)),
                "tl_db_p99_9": float(np.percentile(d, 99.9)), "tl_db_max": float(d.max()),
                "where": "every point with TL > -140 dB (%d of %d)" % (int(sel.sum()), sel.size)}

    tensor_g = 6.0 * alg                     # six bf16 products per term
    achieved_g = tensor_g / (ms_kernel_g / 1e3) / 1e12
    tensor3 = 3.0 * alg
    achieved3 = tensor3 / (ms_kernel / 1e3) / 1e12
    return {
        "workload": "2 Hz, analytic 0-180 km, Nz=100000, %d modes; 64 receivers 0-10 km x 20000 ranges to 2000 km"
                    % M,
        "modes": int(M),
        "ms_per_call": round(ms_call_g, 4), "ms_kernel": round(ms_kernel_g, 4),
        "ms_fp64_cuda_cores": round(ms_fp64, 3), "phases_ms": phases_g,
        "recomputed_fp64": {"points": int(fixed), "of": int(points), "frac": fixed / max(points, 1)},
        "schedule": {"tma_ring": int(sched_ts), "operand_ring": int(sched_gs),
                     "variant_ms": [round(float(t), 4) for t in sched_times],
                     "what": "ring depths picked by the autotuner (first call of the shape times every variant)"},
        "roofline": {"kernel": "k_ms_tc<guarded> (tcgen05 6-term split-BF16)", "bound": "tensor",
                     "achieved": round(achieved_g, 1), "peak": bf16_peak, "unit": "TFLOP/s",
                     "frac": round(achieved_g / bf16_peak, 4),
                     "frac_whole_call": round(tensor_g / (ms_call_g / 1e3) / 1e12 / bf16_peak, 4),
                     "peak_source": peak_source,
                     "flops_per_launch": tensor_g, "algorithmic_flops_per_launch": alg, "traffic": None,
                     "traffic_source": "not measured by this run (DRAM counters need ncu)"},
        "error_vs_fp64": err(p_g),
        "tl2d": tl2d,
        "bf16x3": {"ms_per_call": round(ms_call, 4), "ms_kernel": round(ms_kernel, 4), "phases_ms": phases,
                   "achieved_tflops": round(achieved3, 1), "frac": round(achieved3 / bf16_peak, 4),
                   "note": "unguarded: stated error only", "error_vs_fp64": err(p_tc)},
        "tf32": {"ms_per_call": round(ms_call_tf32, 4), "ms_kernel": round(ms_kernel_tf32, 4), "phases_ms": phases_tf32,
                 "algorithmic_tflops": round(alg / (ms_kernel_tf32 / 1e3) / 1e12, 1),
                 "frac_of_tf32_peak": round(alg / (ms_kernel_tf32 / 1e3) / 1e12 / (bf16_peak / 2.0), 4),
                 "peak_note": "tf32 dense rate taken as half the measured bf16 peak",
                 "note": "unguarded: stated error only", "error_vs_fp64": err(p_32)},
    }


# ---------------------------------------------------------------------------
# azimuth sweep: 360 azimuths x 8 frequencies, Nz per frequency, one batch
# ---------------------------------------------------------------------------
SW_NAZ, SW_NR, SW_DR = 360, 2000, 500.0


def sweep_leg(ctx, stream, reps=2):
    """The N x 2-D sweep: 360 azimuths (1 deg) x 8 frequencies log-spaced
    0.1-2 Hz on the analytic profile, Nz = 60 points per wavelength at 300 m/s
    (at least 5000: 5000-60000), ground source and receiver, 1-D TL on 2000
    ranges every 0.5 km.  Timed (CUDA events) as ONE batched solve over all
    2880 problems on their 7 grids plus one TL launch, against one solve per
    frequency (one grid each)."""
    import torch
    import ncpa_gpu

    prof = ctx.profile_from_arrays(*workloads.si_arrays())
    freqs = workloads.sweep_freqs()
    nzs = [workloads.sweep_nz(f) for f in freqs]
    azs = np.arange(SW_NAZ, dtype=np.float64)
    P = len(freqs) * SW_NAZ

    def batched():
        m = ctx.solve_jobs([(prof, [f], azs, nz) for f, nz in zip(freqs, nzs)],
                           ncpa_gpu.default_params(keep_on_device=1))
        m.tl1d(SW_NR, SW_DR, to_host=False)
        return m

    def per_grid():
        for f, nz in zip(freqs, nzs):
            m = ctx.solve(prof, ncpa_gpu.default_params(nz_grid=nz, keep_on_device=1), [f], azs)
            m.tl1d(SW_NR, SW_DR, to_host=False)
            m.close()

    def timed(fn, n):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(n):
            r = fn()
            if r is not None:
                r.close()
        ev1.record(stream)
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1) / n

    m = batched()  # warm-up; mode counts from this solve
    off = m.all_modes()[0]
    counts = np.diff(off)
    m.close()
    ms_b = timed(batched, reps)
    per_grid()
    ms_g = timed(per_grid, 1)
    # the same batch as one captured graph with autotuned launch shapes
    plan = ctx.plan([(prof, [f], azs, nz) for f, nz in zip(freqs, nzs)], ncpa_gpu.default_params(keep_on_device=1),
                    tl=(SW_NR, SW_DR), tune=True)
    tuning = plan.tuning()
    plan.run()
    ms_p = timed(plan.run, reps)
    plan.close()
    prof.close()
    return {
        "workload": "360 azimuths x 8 frequencies 0.1-2 Hz (log), Nz = max(5000, 60 points per wavelength at "
                    "300 m/s) = %s, ground source/receiver, 1-D TL at 2000 ranges x 0.5 km" % nzs,
        "problems": P, "modes_min": int(counts.min()), "modes_max": int(counts.max()),
        "modes_total": int(counts.sum()),
        "batched_ms": round(ms_b, 2), "batched_freq_solves_per_s": round(P / (ms_b / 1e3), 1),
        "per_grid_ms": round(ms_g, 2), "per_grid_freq_solves_per_s": round(P / (ms_g / 1e3), 1),
        "plan_ms": round(ms_p, 2), "plan_freq_solves_per_s": round(P / (ms_p / 1e3), 1), "plan_tuning": tuning,
        "what": "batched = one ncpa_ess_solve_jobs over all grids + one TL launch; per_grid = one "
                "ncpa_ess_solve + TL per frequency; plan = the batch replayed as one captured CUDA graph "
                "(launch shapes autotuned)",
    }


# ---------------------------------------------------------------------------
# wide-angle (WMod) dispersion: ModBB --dispersion --method wmod
# ---------------------------------------------------------------------------
def wmod_leg(ctx, stream, prof, freqs, az, fp64_peak, flush, cpu_seconds, k=5):
    """The 256-frequency dispersion + 1-D TL of the main step solved with the
    wide-angle solver (WKB off, as --dispersion_file forces), device-resident,
    L2 flushed before each timed solve; phases and the bisection roofline
    (3 FMA per counted chain step) from separate untimed solves; the oracle's
    WMod restatement on every 32nd frequency as the CPU baseline."""
    import torch
    import ncpa_gpu

    params = ncpa_gpu.default_params(nz_grid=NZ, turnoff_wkb=1, keep_on_device=1, method=ncpa_gpu.METHOD_WMOD)

    def step():
        m = ctx.solve(prof, params, freqs, az)
        m.tl1d(N_TL, DR_TL, to_host=False)
        return m

    for _ in range(2):
        step().close()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
    modes = 0
    for i in range(k):
        flush.zero_()
        torch.cuda.synchronize()
        ev[i][0].record(stream)
        m = step()
        ev[i][1].record(stream)
        torch.cuda.synchronize()
        modes = int(m.counts().sum())
        m.close()
    ms = sum(a.elapsed_time(b) for a, b in ev) / k
    n_ph = 3
    ctx.reset_stats()
    ctx.set_timing(True)
    for _ in range(n_ph):
        flush.zero_()
        step().close()
    torch.cuda.synchronize()
    ctx.set_timing(False)
    bis_ms, bis_n = ctx.phase_stats("bisect")
    steps, dsteps = ctx.bisect_steps()
    phases = {ph: round(ctx.phase_stats(ph)[0] / n_ph, 4) for ph in
              ("knots+grid", "matrix", "window", "scan", "host-items", "bisect", "eigvec", "fetch")}
    flops = 6.0 * (steps - dsteps) + 12.0 * dsteps
    achieved = flops / (bis_ms / 1e3) / 1e12 if bis_ms > 0 else None
    # CPU: the oracle's WMod restatement on a stratified sample
    O, pp, prm = _oracle_setup()
    t0 = time.perf_counter()
    done = 0
    for f in freqs[::32]:
        ms_o = O.solve_problem_wmod(pp, prm, float(f), az[0])
        O.tl1d(ms_o, N_TL, DR_TL)
        done += 1
        if time.perf_counter() - t0 > cpu_seconds / 2:
            break
    el = time.perf_counter() - t0
    return {
        "workload": "ModBB --dispersion --method wmod: 256 frequencies df = 0.5/256 Hz, Nz = %d, WKB off, "
                    "1-D TL at %d ranges x %g km, analytic 0-150 km profile" % (NZ, N_TL, DR_TL / 1e3),
        "modes_total": modes, "ms_per_step": round(ms, 4), "value": round(NFREQ / (ms / 1e3), 2), "unit": METRIC,
        "phases_ms": phases,
        "roofline": {"kernel": "k_bisect<WmodRows> (Sturm multisection in kappa)", "bound": "fp64",
                     "achieved": round(achieved, 3) if achieved else None,
                     "peak": round(fp64_peak, 3) if fp64_peak else None, "unit": "TFLOP/s",
                     "frac": round(achieved / fp64_peak, 4) if achieved and fp64_peak else None,
                     "flops": "6 per count-chain step (3 FMA), 12 per Newton-chain step (with the derivative)",
                     "avg_launch_ms": round(bis_ms / max(bis_n, 1), 4)},
        "cpu_baseline": {"value": round(done / el, 3), "unit": METRIC, "cores": O.lib().orc_num_threads(),
                         "kind": "port",
                         "sample": "%d of the 256 frequencies (every 32nd), Nz=%d, WMod eigen-solve + 1-D TL each"
                                   % (done, NZ)},
    }


SV_N, SV_NR, SV_DR, SV_SEED, SV_LOAD, SV_LANES = 200, 2000, 500.0, 2024, 0.8, 3
SV_CEL, SV_CACHE = 340.0, 4.0 * (1 << 30)


def serving_leg(ctx, n=SV_N):
    """Served request stream (seeded Poisson arrivals, per-request perturbed
    profiles, 80 % single frequency 0.05-2 Hz, 20 % 32-256 frequencies up to
    0.5 Hz with pulse waveforms at three ranges, uniform azimuth, per-request
    range grids every 0.5 km out to 100-1000 km, Nz = 20000) replayed in real
    time twice: through the serving loop (3 lanes, continuous batching) and
    through the plain path (one request at a time on one context: profile
    upload, solve, 1-D TL to the host, waveforms).  The arrival rate is set to
    load the plain path to 80 % of its measured capacity.  Latency =
    completion - arrival.  Then, with the mode cache on, the stream is
    submitted twice more: the second pass repeats every request (same
    profiles), which the cache serves without an eigen-solve."""
    import ncpa_gpu

    prm = ncpa_gpu.default_params(nz_grid=NZ)
    reqs = workloads.request_stream(n, 1.0, SV_SEED, dr_m=SV_DR)  # arrival times rescaled below

    def plain_one(r):
        p = ctx.profile_from_arrays(*r["profile"])
        m = ctx.solve(p, prm, r["freqs"], [r["az"]])
        m.tl1d(r["n_ranges"], SV_DR)
        for i in range(m.P):
            m.problem(i)
        if r["wave_ranges_m"] is not None:
            f = np.concatenate([[0.0], r["freqs"]])
            nfft = 4 * len(f)
            sre, sim = ctx.source_spectrum_builtin("pulse1", f, nfft)
            m.bb_synthesize(r["wave_ranges_m"], SV_CEL, nfft, sre, sim)
        m.close()
        p.close()

    def submit(srv, r):
        return srv.submit(*r["profile"], r["freqs"], r["az"], n_ranges=r["n_ranges"], dr_m=SV_DR,
                          wave_ranges_m=r["wave_ranges_m"], max_celerity=SV_CEL)

    for r in reqs[:5]:
        plain_one(r)  # warm-up
    t0 = time.perf_counter()
    for r in reqs[:40]:
        plain_one(r)
    service = (time.perf_counter() - t0) / 40
    rate = SV_LOAD / service
    arrivals = np.array([r["t"] for r in reqs]) / rate  # unit-rate times -> rate
    n_fs = sum(len(r["freqs"]) for r in reqs)

    # plain path, real-time replay
    lat = []
    start = time.perf_counter()
    for r, ta in zip(reqs, arrivals):
        now = time.perf_counter() - start
        if now < ta:
            time.sleep(ta - now)
        plain_one(r)
        lat.append((time.perf_counter() - start - ta) * 1e3)
    plain_wall = time.perf_counter() - start
    plain = {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
             "requests_per_s": n / plain_wall, "freq_solves_per_s": n_fs / plain_wall}

    # served, real-time replay from a submitting thread
    srv = ncpa_gpu.Server(0, params=prm, n_ranges=SV_NR, dr_m=SV_DR, lanes=SV_LANES)
    # capacity first (the whole stream submitted at once), twice: the first
    # pass is the warm-up, in which every lane meets the largest batches of
    # the stream, so its stream-ordered pool and scratch reach their working
    # size before anything is timed
    for _ in range(2):
        start = time.perf_counter()
        ids = [submit(srv, r) for r in reqs]
        res = [srv.wait(i) for i in ids]
        cap_wall = time.perf_counter() - start
    cap_batch = float(np.mean([r["batch_requests"] for r in res]))
    ids = [None] * n

    def submitter():
        st0 = time.perf_counter()
        for i, (r, ta) in enumerate(zip(reqs, arrivals)):
            now = time.perf_counter() - st0
            if now < ta:
                time.sleep(ta - now)
            ids[i] = submit(srv, r)

    start = time.perf_counter()
    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    res = [srv.wait(i) for i in ids]
    served_wall = time.perf_counter() - start
    slat = [r["latency_ms"] for r in res]
    served = {"p50_ms": float(np.percentile(slat, 50)), "p99_ms": float(np.percentile(slat, 99)),
              "requests_per_s": n / served_wall, "freq_solves_per_s": n_fs / served_wall,
              "mean_batch_requests": float(np.mean([r["batch_requests"] for r in res])),
              "failed": int(sum(r["status"] != 0 for r in res)),
              "waveform_requests": int(sum("waveforms" in r for r in res))}
    served["capacity_requests_per_s"] = n / cap_wall
    served["capacity_freq_solves_per_s"] = n_fs / cap_wall
    served["capacity_mean_batch_requests"] = cap_batch
    plain["capacity_requests_per_s"] = 1.0 / service
    plain["capacity_freq_solves_per_s"] = n_fs / (service * n)
    srv.close()

    # repeated stream with the mode cache: pass 1 fills it, pass 2 repeats
    # every request and is served from HBM-resident modes
    srv = ncpa_gpu.Server(0, params=prm, n_ranges=SV_NR, dr_m=SV_DR, lanes=SV_LANES, cache_bytes=SV_CACHE,
                          hbm_budget_bytes=SV_CACHE + 8.0 * (1 << 30))
    walls = []
    for _ in range(2):
        start = time.perf_counter()
        ids = [submit(srv, r) for r in reqs]
        res_c = [srv.wait(i) for i in ids]
        walls.append(time.perf_counter() - start)
    st = srv.stats()
    srv.close()
    cached = {"first_pass_s": round(walls[0], 4), "repeat_pass_s": round(walls[1], 4),
              "repeat_capacity_freq_solves_per_s": n_fs / walls[1],
              "repeat_from_cache": int(sum(r["from_cache"] for r in res_c)), "cache_entries": st["cache_entries"],
              "cache_used_bytes": st["cache_used_bytes"],
              "what": "the same 200 requests submitted twice with a %.0f GiB mode cache; the repeat pass skips "
                      "every eigen-solve (TL and waveforms still computed)" % (SV_CACHE / (1 << 30))}
    return {"workload": "%d requests, seed %d, Poisson at %.1f req/s (80%% of the plain path's capacity), Nz=%d, "
                        "per-request range grids every %.1f km to 100-1000 km, waveforms at 3 ranges for broadband "
                        "requests" % (n, SV_SEED, rate, NZ, SV_DR / 1000.0),
            "freq_solves": int(n_fs), "plain_service_ms": round(service * 1e3, 3), "plain": plain, "served": served,
            "p99_speedup": plain["p99_ms"] / served["p99_ms"] if served["p99_ms"] > 0 else None,
            "cache": cached}


def _bf16_peak():
    """(dense bf16 TFLOP/s, where the figure comes from)"""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "MEASURED_PEAKS.json bf16_tflops (burst), of measured"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback 1590 TFLOP/s (earlier burst measurement on this pool; MEASURED_PEAKS.json absent)"


# ---------------------------------------------------------------------------
# CPU (oracle) legs
# ---------------------------------------------------------------------------
def _oracle_setup():
    from oracle import oracle as O

    tmp = tempfile.mkdtemp(prefix="ncpa_cpu_")
    path = workloads.write_profile(os.path.join(tmp, "analytic_150km.dat"))
    prof = O.read_profile(path)
    prm = O.EssParams(Nz_grid=NZ, turnoff_WKB=True)
    pp = O.prepare(prof, prm)
    return O, pp, prm


def _oracle_freq_solve(O, pp, prm, f, az):
    ms = O.solve_problem(pp, prm, float(f), az)
    O.tl1d(ms, N_TL, DR_TL)
    return ms


def cpu_baseline(freqs, max_seconds=20.0, az=90.0):
    """Oracle on the host cores over a stratified sample of the frequencies
    (every 16th, i.e. the same mix of small and large mode counts)."""
    O, pp, prm = _oracle_setup()
    sample = freqs[::16]
    t0 = time.perf_counter()
    done = 0
    for f in sample:
        _oracle_freq_solve(O, pp, prm, f, az)
        done += 1
        if time.perf_counter() - t0 > max_seconds:
            break
    el = time.perf_counter() - t0
    return {"value": round(done / el, 3), "unit": METRIC, "cores": O.lib().orc_num_threads(), "kind": "port",
            "sample": "%d of the 256 frequencies (every 16th), Nz=20000, eigen-solve + 1-D TL each" % done}


def _lapack_eigen(job):
    """dstebz (bisection, eigenvalues in the window) + dstein (inverse
    iteration, eigenvectors) on one problem's matrix A = S / h^2."""
    from scipy.linalg import lapack

    d, e, lo, hi = job
    m, w, iblock, isplit, info = lapack.dstebz(d, e, 1, lo, hi, 0, 0, 0.0, "E")
    if info != 0:
        return -1
    z, info = lapack.dstein(d, e, w[:m], iblock, isplit)
    return int(m) if info == 0 else -1


def _lapack_ready(_):
    from scipy.linalg import lapack  # noqa: F401  (import cost outside the timed region)

    return 0


def lapack_baseline(freqs, max_seconds=20.0, az=90.0, every=32):
    """LAPACK on the host cores: the matrices of every 32nd frequency are
    assembled by the oracle (untimed), then dstebz + dstein run one problem per
    process of a spawn-started pool (no TL); value = problems per second."""
    import multiprocessing as mp

    O, pp, prm = _oracle_setup()
    jobs, modes = [], 0
    for f in freqs[::every]:
        ms = O.solve_problem(pp, prm, float(f), az, keep_matrix=True)
        h2 = ms.dz * ms.dz
        jobs.append((ms.s / h2, np.full(len(ms.s) - 1, 1.0 / h2), ms.k_min ** 2, ms.k_max ** 2))
        modes += ms.M
    n_proc = max(1, min(len(jobs), os.cpu_count() or 1))
    # one BLAS/OpenMP thread per worker: the pool supplies the parallelism
    # (threaded BLAS in every worker oversubscribes the cores ~100x)
    saved = {k: os.environ.get(k) for k in ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS")}
    os.environ.update({k: "1" for k in saved})
    try:
        with mp.get_context("spawn").Pool(n_proc) as pool:
            pool.map(_lapack_ready, range(n_proc))
            t0 = time.perf_counter()
            res = pool.map(_lapack_eigen, jobs, chunksize=1)
            el = time.perf_counter() - t0
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    return {"value": round(len(jobs) / el, 3), "unit": METRIC, "cores": n_proc, "kind": "lapack",
            "sample": "%d of the 256 frequencies (one in %d), Nz=%d, %d modes: scipy dstebz + dstein per problem, "
                      "one problem per process, no TL%s" % (len(jobs), every, NZ, modes,
                                                            "" if min(res) >= 0 else " (LAPACK reported an error)"),
            "seconds": round(el, 3), "lapack_modes": int(sum(res)), "oracle_modes": int(modes)}


def run_reference(args):
    rank, world, local = _dist()
    if rank != 0:
        return
    O, pp, prm = _oracle_setup()
    freqs = workloads.broadband_freqs(NFREQ, 0.5)
    per_step = 8  # bounded sample per step: 8 frequencies spread over the band
    order = np.concatenate([freqs[i::32] for i in range(32)])
    k = 0
    for _ in range(args.warmup):
        for f in order[k:k + per_step]:
            _oracle_freq_solve(O, pp, prm, f, 90.0)
        k = (k + per_step) % len(order)
    t0 = time.perf_counter()
    n = 0
    for _ in range(args.steps):
        for f in order[k:k + per_step]:
            _oracle_freq_solve(O, pp, prm, f, 90.0)
            n += 1
        k = (k + per_step) % len(order)
    el = time.perf_counter() - t0
    value = n / el
    cores = O.lib().orc_num_threads()
    line = {"metric": METRIC, "value": round(value, 3), "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(el * 1e3 / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": "ModBB 256-frequency dispersion + 1-D TL + pulse synthesis", "nz_grid": NZ,
                       "n_freq": NFREQ},
            "cpu_baseline": {"value": round(value, 3), "unit": METRIC, "cores": cores, "kind": "port",
                             "sample": "%d frequencies per step spread over the 256-frequency band, eigen-solve "
                                       "+ 1-D TL each (reference binary unbuildable here: PETSc/SLEPc/GSL/FFTW "
                                       "absent)" % per_step},
            "e2e": {"value": round(value, 3), "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--quick", action="store_true",
                    help="device-resident leg only (no e2e, plain-path or CPU legs); for profiler runs")
    ap.add_argument("--no-modal-sum", action="store_true", help="skip the tensor-core modal-sum leg")
    ap.add_argument("--no-serving", action="store_true", help="skip the served request-stream leg")
    ap.add_argument("--no-sweep", action="store_true", help="skip the 360-azimuth mixed-grid sweep leg")
    ap.add_argument("--no-wmod", action="store_true", help="skip the wide-angle (WMod) dispersion leg")
    ap.add_argument("--no-lapack", action="store_true", help="skip the LAPACK (dstebz/dstein) CPU leg")
    ap.add_argument("--only-lapack", action="store_true", help="run only the LAPACK CPU leg and print its JSON")
    ap.add_argument("--only-wmod", action="store_true",
                    help="run only the wide-angle dispersion leg and print its JSON (for profiler runs)")
    ap.add_argument("--only-modal-sum", action="store_true",
                    help="run only the tensor-core modal-sum leg and print its JSON (for profiler runs)")
    ap.add_argument("--only-serving", action="store_true",
                    help="run only the served request-stream leg and print its JSON")
    ap.add_argument("--only-sweep", action="store_true",
                    help="run only the mixed-grid sweep leg and print its JSON (for profiler runs)")
    args = ap.parse_args()
    if args.only_serving:
        import ncpa_gpu

        ctx = ncpa_gpu.Context(0)
        print(json.dumps(serving_leg(ctx)), flush=True)
        ctx.close()
        return
    if args.only_sweep:
        import torch
        import ncpa_gpu

        ctx = ncpa_gpu.Context(0)
        print(json.dumps(sweep_leg(ctx, torch.cuda.ExternalStream(ctx.stream_ptr), reps=1)), flush=True)
        ctx.close()
        return
    if args.only_lapack:
        print(json.dumps(lapack_baseline(workloads.broadband_freqs(NFREQ, 0.5))), flush=True)
        return
    if args.only_wmod:
        import torch
        import ncpa_gpu

        ctx = ncpa_gpu.Context(0)
        tmp = tempfile.mkdtemp(prefix="ncpa_bench_")
        prof = ctx.load_profile(workloads.write_profile(os.path.join(tmp, "analytic_150km.dat")))
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        print(json.dumps(wmod_leg(ctx, torch.cuda.ExternalStream(ctx.stream_ptr), prof,
                                  workloads.broadband_freqs(NFREQ, 0.5), [90.0], ctx.fp64_peak_tflops(), flush,
                                  args.cpu_seconds)), flush=True)
        prof.close()
        ctx.close()
        return
    if args.only_modal_sum:
        import torch
        import ncpa_gpu

        ctx = ncpa_gpu.Context(0)
        print(json.dumps(modal_sum_leg(ctx, torch.cuda.ExternalStream(ctx.stream_ptr), _bf16_peak(), k=3)),
              flush=True)
        ctx.close()
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
