#!/usr/bin/env python
"""Benchmark: CG-SENSE ms per reconstruction on one B200 (the headline
metric), with the NUFFT forward+adjoint throughput as a secondary figure.

Workload (2D radial CG-SENSE): 256x256 phantom (20 random ellipses), 16
coils with Gaussian-bump sensitivities, 96 golden-angle spokes x 512 samples
(49152 samples), oversampling 2 (512x512 grid), Kaiser-Bessel width 5.5, ramp
density compensation (sqrt passed to the operator), data = E x + 1% complex
noise, 10 CG iterations with tolerance 0 (exactly 10).  Synthetic, seeded.

A step is one reconstruction (cgSolver::solve).  `value` times it with all
inputs resident in HBM and the operator preprocessed; `e2e` times the whole
per-job call through the public API from pinned host buffers (H2D of data,
trajectory, weights and coil maps, preprocess, solve, D2H of the image).  The
L2 cache (126 MB) is flushed by writing a 256 MB buffer before every timed
step, outside the timed events.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (one per GPU; the path has no data
exchange) under torchrun; timing is the max over ranks.  `--impl reference`
times the reference's CPU reconstruction path in its own float arithmetic
(hoGriddingConvolution's convolution matrix with OpenMP over coils, a
complex64 FFT on every host thread, the cgSolver iteration) on the host
cores; it loads no CUDA library.  At N = 1 the headline line also carries
the NUFFT throughput, the preprocess time, the batched-vs-per-frame figure
and the reference's own GPU path timed on the same device
(headline_extras).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

CFG = dict(N=256, alpha=2, W=5.5, coils=16, spokes=96, samples=512, iterations=10, noise=0.01, seed=1234)
METRIC = "CG-SENSE ms/recon (2D radial 256^2, 16 coils, 96x512 samples, 10 CG iterations)"
UNIT = "ms/recon"


def make_workload(cfg=CFG):
    from gadgetron_b200 import synthetic as S
    N = cfg["N"]
    mos = N * cfg["alpha"]
    traj = S.radial_golden_angle_2d(cfg["spokes"], cfg["samples"])
    dcw = S.ramp_dcw(traj)
    sq = np.sqrt(dcw).astype(np.float32)
    csm = S.gaussian_bump_csm((N, N), cfg["coils"])
    ph = S.ellipse_phantom((N, N), 20, cfg["seed"])[None]
    return dict(N=(N, N), mos=(mos, mos), W=cfg["W"], traj=traj, sqrt_dcw=sq, csm=csm, phantom=ph)


def synth_data_gpu(wl, dev):
    """k-space = E x + 1% RMS complex noise, computed with the GPU operator."""
    import torch
    import gadgetron_b200 as gb
    E = gb.cuNonCartesianSenseOperator(2)
    E.setup(wl["N"], wl["mos"], wl["W"])
    E.set_csm(torch.from_numpy(wl["csm"]).to(dev))
    E.set_dcw(torch.from_numpy(wl["sqrt_dcw"]).to(dev))
    E.preprocess(torch.from_numpy(wl["traj"]).to(dev))
    C = wl["csm"].shape[0]
    y = torch.empty((C, wl["traj"].shape[0]), dtype=torch.complex64, device=dev)
    E.mult_M(torch.from_numpy(wl["phantom"]).to(dev), y)
    rng = np.random.default_rng(CFG["seed"] + 1)
    yc = y.cpu().numpy()
    rms = np.sqrt(np.mean(np.abs(yc) ** 2))
    noise = CFG["noise"] * rms * (rng.standard_normal(yc.shape) + 1j * rng.standard_normal(yc.shape)) / np.sqrt(2)
    return (yc + noise).astype(np.complex64)


# ------------------------------------------------------------------ clocks ---

class ClockSampler:
    """SM clock, max clock, power and clock-event reasons of this rank's GPU,
    polled through NVML every ~2 ms while the timed region runs (the timed
    region is tens of milliseconds, too short for nvidia-smi's sampling).
    Read-only: nothing is set on the GPU.  Samples go to `path` as CSV."""

    REASONS = (("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20), ("hw_thermal_slowdown", 0x40),
               ("sw_power_cap", 0x4))

    def __init__(self, device_index: int, path, period_s: float = 0.002):
        import threading
        self.path = path
        self.samples = []
        self.h = None
        self._stop = threading.Event()
        self._thread = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            self.nv = pynvml
            try:   # match the CUDA device by PCI address (CUDA_VISIBLE_DEVICES may renumber)
                pr = torch.cuda.get_device_properties(device_index)
                bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
                self.h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
                self.h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
        except Exception:
            self.h = None
            return

        def poll():
            nv = self.nv
            while not self._stop.is_set():
                try:
                    sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                    try:
                        rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                    except Exception:
                        rs = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                    pw = nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0
                    self.samples.append((time.perf_counter(), float(sm), int(rs), pw))
                except Exception:
                    pass
                self._stop.wait(period_s)

        self._thread = threading.Thread(target=poll, daemon=True)
        self._thread.start()

    def stop(self):
        if self._thread is None:
            return None
        self._stop.set()
        self._thread.join(timeout=5)
        try:
            if self.path is None:
                raise OSError("no sample file")
            with open(self.path, "w") as f:
                f.write("t_s,sm_mhz,max_mhz,reasons_mask,power_w\n")
                for t, sm, rs, pw in self.samples:
                    f.write("%.6f,%.0f,%.0f,0x%x,%.1f\n" % (t, sm, self.max_mhz, rs, pw))
        except OSError:
            pass
        if not self.samples:
            return None
        reasons = sorted({nm for _, _, rs, _ in self.samples for nm, bit in self.REASONS if rs & bit})
        return {"sm_mhz": float(np.median([sm for _, sm, _, _ in self.samples])), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples), "source": "NVML, 2 ms polling"}


def traffic_for(kname):
    """DRAM bytes (read + write) per launch of the named kernel from the ncu
    capture summarised in profiles/roofline_traffic.json (same workload, caches
    flushed before the launch as in the timed loop), or None."""
    try:
        t = json.load(open(os.path.join(ROOT, "profiles", "roofline_traffic.json")))
        return int(t["kernels"][kname.split()[0]]["dram_bytes_per_launch"])
    except Exception:
        return None


def reduce_max_over_ranks(vals, device):
    """Element-wise max of a float64 vector over all ranks (timings: the job
    is as slow as its slowest replica).  Identity when not distributed."""
    import torch
    import torch.distributed as dist
    vals = np.asarray(vals, np.float64)
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return vals
    t = torch.from_numpy(vals.copy()).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.cpu().numpy()


# ------------------------------------------------------------ our arm -------

def run_ours(args, rank, world, local_rank):
    import torch
    import gadgetron_b200 as gb
    from gadgetron_b200._lib import lib
    dev = torch.device("cuda:%d" % local_rank)
    torch.cuda.set_device(dev)
    wl = make_workload()
    d_host = synth_data_gpu(wl, dev)
    C = wl["csm"].shape[0]
    M = wl["traj"].shape[0]
    N = wl["N"]

    # Resident inputs.
    traj_d = torch.from_numpy(wl["traj"]).to(dev)
    csm_d = torch.from_numpy(wl["csm"]).to(dev)
    sq_d = torch.from_numpy(wl["sqrt_dcw"]).to(dev)
    sqrt_w = wl["sqrt_dcw"].reshape(1, -1)
    d_dev = torch.from_numpy((d_host * sqrt_w).astype(np.complex64)).to(dev)   # data pre-weighted by sqrt(w)
    E = gb.cuNonCartesianSenseOperator(2)
    E.setup(N, wl["mos"], wl["W"])
    E.set_csm(csm_d)
    E.set_dcw(sq_d)
    E.preprocess(traj_d)
    cg = gb.cuCgSolver()
    cg.set_encoding_operator(E)
    cg.set_max_iterations(CFG["iterations"])
    cg.set_tc_tolerance(0.0)
    cg.set_use_graph(True)
    x_out = torch.empty((1, N[1], N[0]), dtype=torch.complex64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()

    for _ in range(args.warmup):
        cg.solve(d_dev, x_out)
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    clk = ClockSampler(local_rank, (args.clocks_csv % rank) if args.clocks_csv else None)
    launches0 = lib.gb_kernel_launch_count()
    barrier()
    torch.cuda.synchronize()
    total_ms = 0.0
    for _ in range(args.steps):
        flush.fill_(1.0)
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record(stream)
        cg.solve(d_dev, x_out)
        e.record(stream)
        e.synchronize()
        total_ms += s.elapsed_time(e)
    torch.cuda.synchronize()
    barrier()
    launches = lib.gb_kernel_launch_count() - launches0
    clocks = clk.stop() if clk else None

    # e2e through the public API from pinned host buffers.
    h_d = torch.from_numpy((d_host * sqrt_w).astype(np.complex64)).pin_memory()
    h_traj = torch.from_numpy(wl["traj"]).pin_memory()
    h_sq = torch.from_numpy(wl["sqrt_dcw"]).pin_memory()
    h_csm = torch.from_numpy(wl["csm"]).pin_memory()
    h_x = torch.empty((1, N[1], N[0]), dtype=torch.complex64).pin_memory()
    g_d = torch.empty_like(d_dev)
    g_traj = torch.empty_like(traj_d)
    g_sq = torch.empty_like(sq_d)
    g_csm = torch.empty_like(csm_d)
    E2 = gb.cuNonCartesianSenseOperator(2)
    E2.setup(N, wl["mos"], wl["W"])
    cg2 = gb.cuCgSolver()
    cg2.set_max_iterations(CFG["iterations"])
    cg2.set_tc_tolerance(0.0)
    cg2.set_use_graph(True)

    # The trajectory goes first on the solve's stream; the data, weights and
    # coil maps (21 MB) cross on a second stream while the trajectory is
    # preprocessed (preprocess reads only the trajectory), and the solve
    # waits for them.
    side = torch.cuda.Stream(device=dev)
    copied = torch.cuda.Event()

    def e2e_step():
        g_traj.copy_(h_traj, non_blocking=True)
        side.wait_stream(stream)
        with torch.cuda.stream(side):
            g_d.copy_(h_d, non_blocking=True)
            g_sq.copy_(h_sq, non_blocking=True)
            g_csm.copy_(h_csm, non_blocking=True)
            copied.record(side)
        E2.set_csm(g_csm)
        E2.set_dcw(g_sq)
        E2.preprocess(g_traj)
        stream.wait_event(copied)
        cg2.set_encoding_operator(E2)
        cg2.solve(g_d, x_out)
        h_x.copy_(x_out, non_blocking=True)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    torch.cuda.synchronize()
    barrier()
    e2e_ms = 0.0
    for _ in range(args.steps):
        flush.fill_(1.0)
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record(stream)
        e2e_step()
        e.record(stream)
        e.synchronize()
        e2e_ms += s.elapsed_time(e)
    barrier()
    h2d = h_d.numel() * 8 + h_traj.numel() * 4 + h_sq.numel() * 4 + h_csm.numel() * 8
    d2h = h_x.numel() * 8

    # Kernel roofline: the gridding and degridding kernels timed alone on the
    # same plan (16 coils), L2 flushed before each launch.
    plan = E.get_plan()
    grid = torch.empty((C, 1, wl["mos"][1], wl["mos"][0]), dtype=torch.complex64, device=dev)
    samp = torch.empty((C, M), dtype=torch.complex64, device=dev)
    rng = np.random.default_rng(7)
    samp.copy_(torch.from_numpy((rng.standard_normal((C, M)) + 1j * rng.standard_normal((C, M))).astype(np.complex64)))

    def time_kernel(fn, reps=20):
        for _ in range(3):
            fn()
        ms = 0.0
        for _ in range(reps):
            flush.fill_(1.0)
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record(stream)
            fn()
            e.record(stream)
            e.synchronize()
            ms += s.elapsed_time(e)
        return ms / reps

    t_grid = time_kernel(lambda: plan.convolve(samp, grid, gb.NFFT_conv_mode.NC2C))
    t_degrid = time_kernel(lambda: plan.convolve(grid, samp, gb.NFFT_conv_mode.C2NC))
    # the two convolutions as E^H E runs them inside the timed solve (its
    # own kernels and workspace layouts), L2 flushed before every launch
    t_grid_n, t_degrid_n = plan.time_normal_convolutions(C, sq_d, reps=20, flush=flush)
    G = wl["mos"][0] * wl["mos"][1]
    bytes_grid = C * (8 * M + 8 * G) + 4 * 2 * M          # NC2C: samples in, grid out, coordinates
    bytes_degrid = C * (8 * G + 8 * M) + 4 * 2 * M        # C2NC: grid in, samples out, coordinates

    # Reduce timings over ranks (max).
    vals = reduce_max_over_ranks([total_ms, e2e_ms, t_grid, t_degrid, t_grid_n, t_degrid_n], dev)
    total_ms, e2e_ms, t_grid, t_degrid, t_grid_n, t_degrid_n = [float(v) for v in vals]
    if rank != 0:
        return None

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    # the dominant kernel of the timed region: the slower of E^H E's gridding
    # (k_grid_rows_ws on this workload) and degridding (k_degrid_table)
    if t_grid_n >= t_degrid_n:
        kname, kms, kbytes = "k_grid_rows_ws (gridding inside E^H E, 16 coils)", t_grid_n, bytes_grid
    else:
        kname, kms, kbytes = "k_degrid_table (degridding inside E^H E, 16 coils)", t_degrid_n, bytes_degrid
    achieved = kbytes / (kms * 1e-3) / 1e9

    ms_per_step = total_ms / args.steps
    value = ms_per_step / world
    result = {
        "metric": METRIC,
        "value": round(value, 4),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 4),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c64 (fp32), fp64 CG reductions",
        "data": "synthetic (seeded phantom, golden-angle radial trajectory, Gaussian-bump coil maps)",
        "config": {"workload": "cg-sense-2d-radial", "matrix": 256, "matrix_os": 512, "W": CFG["W"],
                   "coils": C, "spokes": CFG["spokes"], "samples_per_spoke": CFG["samples"],
                   "iterations": CFG["iterations"], "tc_tolerance": 0.0, "cuda_graph": True,
                   "l2": "flushed (256 MB write) before every timed step", "parallelism": "replicas%d" % world},
        "e2e": {"value": round(e2e_ms / args.steps / world, 4), "unit": UNIT,
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "includes": "H2D (pinned) of data/trajectory/dcw/csm (data, dcw and csm on a second stream, "
                            "overlapping the preprocess), preprocess, CG solve, D2H image"},
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": round(achieved, 1), "peak": hbm_peak,
                     "unit": "GB/s", "frac": round(achieved / hbm_peak, 4), "peak_source": peak_src,
                     "traffic": traffic_for(kname), "algorithmic_bytes": int(kbytes), "ms_per_launch": round(kms, 5),
                     "other_kernel_ms": {"grid_in_normal_op": round(t_grid_n, 5),
                                         "degrid_in_normal_op": round(t_degrid_n, 5),
                                         "grid_standalone_convolve": round(t_grid, 5),
                                         "degrid_standalone_convolve": round(t_degrid, 5)}},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    return result, wl, d_host, x_out


def cpu_cg_sample(wl, d_host, iters_timed=3):
    """Times the reference's CPU path in its float arithmetic
    (oracle.HoSenseFloat) on this host: one E^H d and `iters_timed` CG
    iterations, scaled to 10 iterations; the convolution-matrix build
    (preprocess) is not part of the recon time."""
    from oracle import oracle as O
    ncpu = os.cpu_count() or 1
    H = O.HoSenseFloat(wl["N"], wl["mos"], wl["W"], wl["traj"], wl["csm"], wl["sqrt_dcw"], workers=ncpu)
    d = (d_host * wl["sqrt_dcw"].reshape(1, -1)).astype(np.complex64)
    t0 = time.perf_counter()
    rhs = H.mult_MH(d)
    t_rhs = time.perf_counter() - t0
    r = rhs.copy()
    p = r.copy()
    x = np.zeros_like(rhs)
    rq = np.float32(np.real(np.vdot(r, r)))
    times = []
    for _ in range(iters_timed):
        t0 = time.perf_counter()
        q = H.mult_MH_M(p)
        alpha = np.complex64(rq / np.vdot(p, q))
        x += alpha * p
        r -= alpha * q
        rq2 = np.float32(np.real(np.vdot(r, r)))
        p = p * np.float32(rq2 / rq) + r
        rq = rq2
        times.append(time.perf_counter() - t0)
    t_iter = float(np.mean(times))
    ms = (t_rhs + CFG["iterations"] * t_iter) * 1e3
    return ms, ncpu, t_rhs, t_iter


def make_noisy_data_cpu(wl):
    """The workload's k-space on the host: FP64 oracle forward operator plus
    1% RMS complex noise (the same seed as the GPU arm's data)."""
    from oracle import oracle as O
    P = O.OraclePlan(wl["N"], wl["mos"], wl["W"])
    P.preprocess(wl["traj"][None])
    E = O.OracleSense(P, wl["csm"], wl["sqrt_dcw"].reshape(1, -1))
    d = E.mult_M(wl["phantom"]).astype(np.complex128)
    rng = np.random.default_rng(CFG["seed"] + 1)
    rms = np.sqrt(np.mean(np.abs(d) ** 2))
    d = d + CFG["noise"] * rms * (rng.standard_normal(d.shape) + 1j * rng.standard_normal(d.shape)) / np.sqrt(2)
    return E, d


def run_reference(args):
    """The reference arm: the reference's CPU reconstruction path in its own
    float arithmetic (oracle.HoSenseFloat: hoGriddingConvolution's
    per-sample convolution matrix and its transpose, complext<float> sums,
    OpenMP over coils; complex64 FFT on every host thread; the cgSolver
    iteration in complex64), timed on the host cores.  Each step is one CG
    iteration of the full workload (E^H E p and the vector updates); the
    recon time is one measured E^H d plus 10 x the mean iteration time.  The
    convolution-matrix build (the reference's preprocess) is timed on its
    own.  Loads no CUDA library."""
    from oracle import oracle as O
    wl = make_workload()
    ncpu = os.cpu_count() or 1
    E64, d64 = make_noisy_data_cpu(wl)
    d = d64.reshape(CFG["coils"], -1).astype(np.complex64)
    t0 = time.perf_counter()
    H = O.HoSenseFloat(wl["N"], wl["mos"], wl["W"], wl["traj"], wl["csm"], wl["sqrt_dcw"], workers=ncpu)
    t_prep = time.perf_counter() - t0
    t0 = time.perf_counter()
    rhs = H.mult_MH(d)
    t_rhs = time.perf_counter() - t0
    x = np.zeros_like(rhs)
    r = rhs.copy()
    p = r.copy()
    rq = np.float32(np.real(np.vdot(r, r)))
    state = {"x": x, "r": r, "p": p, "rq": rq, "it": 0, "x10": None}

    def step():
        q = H.mult_MH_M(state["p"])
        alpha = np.complex64(state["rq"] / np.vdot(state["p"], q))
        state["x"] += alpha * state["p"]
        state["r"] -= alpha * q
        rq2 = np.float32(np.real(np.vdot(state["r"], state["r"])))
        state["p"] = state["p"] * np.float32(rq2 / state["rq"]) + state["r"]
        state["rq"] = rq2
        state["it"] += 1
        if state["it"] == CFG["iterations"]:
            state["x10"] = state["x"].copy()

    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    t_iter = float(np.mean(times))
    value = (t_rhs + CFG["iterations"] * t_iter) * 1e3
    acc = None
    if state["x10"] is not None:
        xr = O.cg_solve(E64, d64, iterations=CFG["iterations"], tc_tolerance=0.0)
        acc = O.rel_l2(state["x10"], xr)
    sample = ("%d timed CG iterations (E^H E + updates) of the full workload; recon = one measured E^H d "
              "+ %d x mean iteration; float CSR gridding (OpenMP over %d coils), complex64 pocketfft FFT on "
              "%d threads standing in for FFTW" % (args.steps, CFG["iterations"], CFG["coils"], ncpu))
    return {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t_iter * 1e3, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64 (fp32, complext<float> as the reference)",
        "data": "synthetic (seeded)", "impl": "reference",
        "config": {"workload": "cg-sense-2d-radial", "matrix": 256, "matrix_os": 512, "W": CFG["W"],
                   "coils": CFG["coils"], "spokes": CFG["spokes"], "samples_per_spoke": CFG["samples"],
                   "iterations": CFG["iterations"], "tc_tolerance": 0.0, "parallelism": "host cores"},
        "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": ncpu, "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "preprocess_ms": round(t_prep * 1e3, 2),
        "recon_rel_l2_vs_fp64_oracle_cg": acc,
    }


# ------------------------------------------------------ other workloads ------

def _timed(fn, steps, warmup, flush, stream):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    total = 0.0
    for _ in range(steps):
        if flush is not None:
            flush.fill_(1.0)
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record(stream)
        fn()
        e.record(stream)
        e.synchronize()
        total += s.elapsed_time(e)
    return total / steps


def run_nufft(args, dims):
    """NUFFT forward (C2NC) + adjoint (NC2C, ramp dcw) throughput.
    2D: 128^2, 1 coil, 128 golden-angle spokes x 256 (32768 samples), alpha 2, W 5.5.
    3D: 128^3, 32 coils (Gaussian-bump coil images), 20000 golden-means
    spokes x 256 (5.12M samples), alpha 1.5 (192^3), W 4.
    --size small (profiling case, 3D only): 64^3, 16 coils, 2500 spokes x 128,
    alpha 1.5 (96^3), W 4."""
    import torch
    import gadgetron_b200 as gb
    from gadgetron_b200 import synthetic as S
    from gadgetron_b200._lib import lib
    from oracle import oracle as O
    dev = torch.device("cuda:0")
    if dims == 2:
        N, mos, W, C = (128, 128), (256, 256), 5.5, 1
        traj = S.radial_golden_angle_2d(128, 256)
        img = S.gaussian_image((C, 1, 128, 128), 11)
    elif getattr(args, "size", "full") == "small":
        N, mos, W, C = (64, 64, 64), (96, 96, 96), 4.0, 16
        traj = S.kooshball_golden_means_3d(2500, 128)
        x = S.gaussian_image((64, 64, 64), 6)
        img = (S.gaussian_bump_csm((64, 64, 64), C) * x[None])[:, None].astype(np.complex64)
    else:
        N, mos, W, C = (128, 128, 128), (192, 192, 192), 4.0, 32
        traj = S.kooshball_golden_means_3d(20000, 256)
        x = S.gaussian_image((128, 128, 128), 12)
        img = (S.gaussian_bump_csm((128, 128, 128), C) * x[None])[:, None].astype(np.complex64)
    M = traj.shape[0]
    dcw = S.ramp_dcw(traj)
    plan = gb.NFFT.make_plan(N, mos, W)
    t_prep0 = time.perf_counter()
    traj_d = torch.from_numpy(traj).to(dev)
    plan.preprocess(traj_d)
    torch.cuda.synchronize()
    t_prep = (time.perf_counter() - t_prep0) * 1e3
    x_d = torch.from_numpy(img).to(dev)
    dcw_d = torch.from_numpy(dcw).to(dev)
    y_d = torch.empty((C, M), dtype=torch.complex64, device=dev)
    xb_d = torch.empty_like(x_d)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()

    def step():
        plan.compute(x_d, y_d, None, gb.NFFT_comp_mode.FORWARDS_C2NC)
        plan.compute(y_d, xb_d, dcw_d, gb.NFFT_comp_mode.BACKWARDS_NC2C)

    l0 = lib.gb_kernel_launch_count()
    ms = _timed(step, args.steps, args.warmup, flush, stream)
    launches = (lib.gb_kernel_launch_count() - l0) // (args.steps + args.warmup) * args.steps
    t_fwd = _timed(lambda: plan.compute(x_d, y_d, None, gb.NFFT_comp_mode.FORWARDS_C2NC), 5, 2, flush, stream)
    t_adj = _timed(lambda: plan.compute(y_d, xb_d, dcw_d, gb.NFFT_comp_mode.BACKWARDS_NC2C), 5, 2, flush, stream)
    value = M * C / (ms * 1e-3) / 1e6
    # accuracy: forward vs FP64 direct NDFT on a subset of samples (coil 0)
    idx = np.random.default_rng(5).choice(M, 1024 if dims == 3 else 4096, replace=False)
    O.set_fft_workers(os.cpu_count() or 1)
    yn = O.ndft_forward(img[0, 0][None], traj[idx], mos)
    err_ndft = O.rel_l2(y_d[0].cpu().numpy()[idx], yn[0])
    res = {
        "metric": "NUFFT fwd+adj Msample-coils/s (%dD)" % dims, "value": round(value, 2),
        "unit": "Msample-coils/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64 (fp32)", "data": "synthetic",
        "config": {"workload": "nufft-%dd" % dims + ("-small" if N[0] == 64 and dims == 3 else ""), "matrix": N[0], "matrix_os": mos[0], "W": W, "coils": C,
                   "samples": M, "l2": "flushed before every timed step"},
        "ms_forward": round(t_fwd, 4), "ms_adjoint": round(t_adj, 4), "ms_preprocess_wall": round(t_prep, 2),
        "forward_rel_l2_vs_fp64_ndft": err_ndft, "gpu_launches": int(launches),
    }
    if dims == 2:
        P = O.OraclePlan(N, mos, W)
        P.preprocess(traj[None])
        yr = P.forward_c2nc(img)
        xr = P.backwards_nc2c(yr, dcw[None])
        res["forward_rel_l2_vs_oracle"] = O.rel_l2(y_d.cpu().numpy(), yr)
        res["adjoint_rel_l2_vs_oracle"] = O.rel_l2(xb_d.cpu().numpy(), xr)
        t0 = time.perf_counter()
        for _ in range(3):
            yr = P.forward_c2nc(img)
            P.backwards_nc2c(yr, dcw[None])
        cpu_ms = (time.perf_counter() - t0) / 3 * 1e3
        res["cpu_baseline"] = {"value": round(M * C / (cpu_ms * 1e-3) / 1e6, 3), "unit": "Msample-coils/s",
                               "cores": os.cpu_count(), "kind": "port", "sample": "3 fwd+adj pairs"}
    else:
        res["fd_gradient"] = fd_gradient_check_3d(plan, x_d, traj, dcw_d, N, mos, W)
    return res


def fd_gradient_check_3d(plan, x_d, traj, dcw_d, N, mos, W, n_check=64, h=1e-4):
    """Trajectory gradient through the autograd wrapper against central
    differences (step h in k units) on n_check random samples whose tap ranges
    do not change within +-h."""
    import torch
    import gadgetron_b200 as gb
    from gadgetron_b200.autograd import nufft_forward
    dev = x_d.device
    rng = np.random.default_rng(9)
    M = traj.shape[0]
    C = x_d.shape[0]
    traj = (traj.astype(np.float64) * 0.999).astype(np.float32)
    p = gb.NFFT.make_plan(N, mos, W)
    t_d = torch.from_numpy(traj).to(dev).requires_grad_(True)
    p.preprocess(t_d.detach())
    v = torch.from_numpy((rng.standard_normal((C, M)) + 1j * rng.standard_normal((C, M))).astype(np.complex64)).to(dev)
    x_g = x_d.clone().requires_grad_(True)
    y = nufft_forward(x_g, t_d, p, dcw_d)
    (v.conj() * y).real.sum().backward()
    g_ad = t_d.grad.cpu().numpy().astype(np.float64)
    r = W / 2
    ok = np.ones(M, bool)
    for d in range(3):
        lo = (traj[:, d].astype(np.float64) - h) * mos[d] + mos[d] / 2
        hi = (traj[:, d].astype(np.float64) + h) * mos[d] + mos[d] / 2
        for sgn in (-1.0, 1.0):
            ok &= np.ceil(lo + sgn * r - 1e-3) == np.ceil(hi + sgn * r + 1e-3)
            ok &= np.floor(lo + sgn * r - 1e-3) == np.floor(hi + sgn * r + 1e-3)
    pick = rng.choice(np.nonzero(ok)[0], n_check, replace=False)
    g_fd = np.zeros((n_check, 3))
    out = torch.empty((C, M), dtype=torch.complex64, device=dev)
    for d in range(3):
        vals = []
        for sg in (1.0, -1.0):
            tp = traj.copy()
            tp[:, d] = (tp[:, d].astype(np.float64) + sg * h).astype(np.float32)
            p2 = gb.NFFT.make_plan(N, mos, W)
            p2.preprocess(torch.from_numpy(tp).to(dev))
            p2.compute(x_d, out, dcw_d, gb.NFFT_comp_mode.FORWARDS_C2NC)
            vals.append((v.conj() * out).real.double().sum(0).cpu().numpy()[pick])
            del p2
        dk = ((traj[pick, d].astype(np.float64) + h).astype(np.float32).astype(np.float64) -
              (traj[pick, d].astype(np.float64) - h).astype(np.float32).astype(np.float64))
        g_fd[:, d] = (vals[0] - vals[1]) / dk
    err = float(np.linalg.norm(g_ad[pick] - g_fd) / np.linalg.norm(g_fd))
    return {"samples": n_check, "step_k": h, "rel_err": err, "valid_fraction": float(ok.mean())}


def run_batched(args):
    """64 frames of 192^2, frame f has 13 + (f*37 mod 77) golden-angle spokes of
    384 samples; 12 coils; alpha 2, W 5.5 (not stated by the workload; chosen);
    15 CG iterations.  Batched: one operator over all frames (uneven sample
    counts), per-frame CG scalars, one CUDA graph for the whole solve.  Plain:
    one operator + solve per frame, no graph, default tiling.
    --size small (profiling case): the first 16 frames."""
    import torch
    import gadgetron_b200 as gb
    from gadgetron_b200 import synthetic as S
    from gadgetron_b200._lib import lib
    dev = torch.device("cuda:0")
    F, N, mos, W, C, S_per, iters = 64, 192, 384, 5.5, 12, 384, 15
    if getattr(args, "size", "full") == "small":
        F = 16
    spokes = S.uneven_frame_spokes(F)
    trajs = [S.radial_golden_angle_2d(s, S_per, profile_offset=sum(spokes[:f])) for f, s in enumerate(spokes)]
    offs = np.cumsum([0] + [t.shape[0] for t in trajs]).tolist()
    traj = np.concatenate(trajs, 0)
    sq = np.concatenate([np.sqrt(S.ramp_dcw(t)) for t in trajs]).astype(np.float32)
    csm = S.gaussian_bump_csm((N, N), C)
    base = S.ellipse_phantom((N, N), 20, 77)
    amp = np.random.default_rng(78).uniform(0.9, 1.1, F)
    ph = (base[None] * amp[:, None, None]).astype(np.complex64)
    csm_d = torch.from_numpy(csm).to(dev)
    E = gb.cuNonCartesianSenseOperator(2)
    E.setup((N, N), (mos, mos), W)
    E.set_csm(csm_d)
    sq_d = torch.from_numpy(sq).to(dev)
    E.set_dcw(sq_d)
    E.preprocess(torch.from_numpy(traj).to(dev), frame_offsets=offs)
    if getattr(args, "tiling", None):
        tx, ty, cgr = (int(v) for v in args.tiling.split(","))
        E.get_plan().set_tiling((tx, ty), cgr)
    else:
        E.autotune()   # tile shape and coil group for this trajectory set
    if getattr(args, "schedule", None) is not None:
        E.get_plan().set_grid_schedule(args.schedule)
    tiling = E.get_plan().get_tiling()
    schedule = E.get_plan().get_grid_schedule()
    y = torch.empty((C, offs[-1]), dtype=torch.complex64, device=dev)
    E.mult_M(torch.from_numpy(ph).to(dev), y)
    rms = float(y.abs().pow(2).mean().sqrt())
    rng = np.random.default_rng(79)
    noise = torch.from_numpy((0.01 * rms * (rng.standard_normal(y.shape) + 1j * rng.standard_normal(y.shape)) /
                              np.sqrt(2)).astype(np.complex64)).to(dev)
    d = (y + noise).contiguous()
    cg = gb.cuCgSolver()
    cg.set_encoding_operator(E)
    cg.set_max_iterations(iters)
    cg.set_tc_tolerance(0.0)
    cg.set_frame_independent(True)
    cg.set_use_graph(True)
    xb = torch.empty((F, N, N), dtype=torch.complex64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()
    l0 = lib.gb_kernel_launch_count()
    ms_b = _timed(lambda: cg.solve(d, xb), args.steps, args.warmup, flush, stream)
    launches = (lib.gb_kernel_launch_count() - l0) // (args.steps + args.warmup)
    # plain per-frame form
    ops, solvers, ds, xs = [], [], [], []
    for f in range(F):
        Ef = gb.cuNonCartesianSenseOperator(2)
        Ef.setup((N, N), (mos, mos), W)
        Ef.set_csm(csm_d)
        Ef.set_dcw(sq_d[offs[f]:offs[f + 1]].contiguous())
        Ef.preprocess(torch.from_numpy(trajs[f]).to(dev))
        cf = gb.cuCgSolver()
        cf.set_encoding_operator(Ef)
        cf.set_max_iterations(iters)
        cf.set_tc_tolerance(0.0)
        ops.append(Ef)
        solvers.append(cf)
        ds.append(d[:, offs[f]:offs[f + 1]].contiguous())
        xs.append(torch.empty((1, N, N), dtype=torch.complex64, device=dev))

    def plain():
        for f in range(F):
            solvers[f].solve(ds[f], xs[f])

    ms_p = _timed(plain, max(2, args.steps // 4), 2, flush, stream)
    xp = torch.cat(xs, 0)
    err = float((xb - xp).abs().pow(2).sum().sqrt() / xp.abs().pow(2).sum().sqrt())
    return {
        "metric": "batched CG-SENSE ms/batch (%d uneven frames, 192^2, 12 coils, 15 it)" % F,
        "value": round(ms_b, 3), "unit": "ms/batch", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_b, 3), "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64 (fp32), fp64 CG reductions", "data": "synthetic",
        "config": {"workload": "batched-uneven-cg-sense", "frames": F, "matrix": N, "matrix_os": mos, "W": W,
                   "coils": C, "samples_total": offs[-1], "iterations": iters, "alpha_W": "chosen: 2.0, 5.5"},
        "plain_per_frame_ms": round(ms_p, 3), "speedup_vs_plain": round(ms_p / ms_b, 2),
        "batched_vs_plain_rel_l2": err, "gpu_launches_per_batch": int(launches),
        "tiling_after_autotune": {"tile": list(tiling[0]), "coil_group": tiling[1]},
        "grid_schedule": schedule,
    }


def run_precision(args):
    """512^2 ellipse phantom, 24 variable-density Archimedean interleaves x 4096
    (density 4x at the centre to 1x at the edge), 32 coils, alpha 1.25 (640^2),
    W 4; compensated gridding, FP64 CG reductions, 3 refinements x 8 CG
    iterations.  Errors vs FP64 direct NDFT (4096-sample subset) and vs the
    oracle."""
    import torch
    import gadgetron_b200 as gb
    from gadgetron_b200 import synthetic as S
    from oracle import oracle as O
    dev = torch.device("cuda:0")
    N, mos, W, C = 512, 640, 4.0, 32
    traj = S.spiral_archimedean_2d(24, 4096, N, 4.0)
    M = traj.shape[0]
    sq = np.sqrt(S.ramp_dcw(traj)).astype(np.float32)
    csm = S.gaussian_bump_csm((N, N), C)
    ph = S.ellipse_phantom((N, N), 20, 91)[None]
    res = {"metric": "precision study (spiral 512^2, 32 coils, 3x8 refinement)", "unit": "ms/recon",
           "higher_is_better": False, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "config": {"workload": "precision-spiral", "matrix": N, "matrix_os": mos, "W": W, "coils": C,
                      "samples": M, "refinements": 3, "iterations_each": 8}}
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    csm_d = torch.from_numpy(csm).to(dev)
    sq_d = torch.from_numpy(sq).to(dev)
    traj_d = torch.from_numpy(traj).to(dev)
    out = {}
    for flags, name in ((gb.FLAG_COMPENSATED, "compensated"), (0, "plain")):
        E = gb.cuNonCartesianSenseOperator(2, flags=flags)
        E.setup((N, N), (mos, mos), W)
        E.set_csm(csm_d)
        E.set_dcw(sq_d)
        E.preprocess(traj_d)
        y = torch.empty((C, M), dtype=torch.complex64, device=dev)
        E.mult_M(torch.from_numpy(ph).to(dev), y)
        cg = gb.cuCgSolver()
        cg.set_encoding_operator(E)
        cg.set_max_iterations(8)
        cg.set_tc_tolerance(0.0)
        cg.set_refinements(3)
        cg.set_use_graph(True)
        x = torch.empty((1, N, N), dtype=torch.complex64, device=dev)
        ms = _timed(lambda: cg.solve(y, x), args.steps, args.warmup, flush, stream)
        out[name] = (ms, y.cpu().numpy(), x.cpu().numpy())
    ms, y, x = out["compensated"]
    res["value"] = round(ms, 3)
    res["ms_plain_accumulation"] = round(out["plain"][0], 3)
    O.set_fft_workers(os.cpu_count() or 1)
    idx = np.random.default_rng(4).choice(M, 4096, replace=False)
    coil_imgs = csm[:4] * ph
    yn = O.ndft_forward(coil_imgs, traj[idx], (mos, mos), dcw=sq[idx])
    res["forward_rel_l2_vs_fp64_ndft_4096"] = O.rel_l2(y[:4][:, idx], yn)
    P = O.OraclePlan((N, N), (mos, mos), W)
    P.preprocess(traj[None])
    yr = P.forward_c2nc(coil_imgs[:, None], sq[None])
    res["forward_rel_l2_vs_oracle"] = O.rel_l2(y[:4], yr.reshape(4, -1))
    res["forward_rel_l2_vs_oracle_plain_accumulation"] = O.rel_l2(out["plain"][1][:4], yr.reshape(4, -1))
    res["recon_rel_l2_vs_phantom"] = O.rel_l2(x, ph)
    res["recon_rel_l2_compensated_vs_plain"] = O.rel_l2(x, out["plain"][2])
    return res


def run_regularized(args):
    """The gpuCgSenseGadget solve on the headline workload (256^2, 16 coils,
    96 x 512 radial samples, 10 iterations): image regulariser of weight kappa
    computed from the adjoint reconstruction, preconditioner
    1/sqrt(sum |csm|^2 + kappa R), CG on (E^H E + kappa R^H R) x = E^H d.
    value = the solve (graph replay); the regulariser and preconditioner
    setup is reported beside it.  Accuracy vs the oracle's FP64 CG."""
    import torch
    import gadgetron_b200 as gb
    from oracle import oracle as O
    dev = torch.device("cuda:0")
    wl = make_workload()
    d_host = synth_data_gpu(wl, dev)
    N, C = wl["N"], wl["csm"].shape[0]
    kappa = 0.05
    csm_d = torch.from_numpy(wl["csm"]).to(dev)
    sq_d = torch.from_numpy(wl["sqrt_dcw"]).to(dev)
    d_np = (d_host * wl["sqrt_dcw"].reshape(1, -1)).astype(np.complex64)
    d_dev = torch.from_numpy(d_np).to(dev)
    E = gb.cuNonCartesianSenseOperator(2)
    E.setup(N, wl["mos"], wl["W"])
    E.set_csm(csm_d)
    E.set_dcw(sq_d)
    E.preprocess(torch.from_numpy(wl["traj"]).to(dev))
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    reg = torch.empty((1, N[1], N[0]), dtype=torch.complex64, device=dev)
    E.mult_MH(d_dev, reg)
    R = gb.cuImageOperator()
    D = gb.cuCgPreconditioner()

    def setup():
        R.compute(reg)
        D.set_weights(gb.sense_precond_weights(E, R.get(), kappa))

    setup_ms = _timed(setup, args.steps, args.warmup, None, stream)
    # the gadget's other inputs generated on the device: golden-ratio
    # trajectory and its Voronoi density compensation (same shape)
    from gadgetron_b200 import radial as RU
    gen_ms = _timed(lambda: (RU.compute_radial_trajectory_golden_ratio_2d(CFG["samples"], CFG["spokes"], device=dev),
                             RU.compute_radial_dcw_golden_ratio_2d(CFG["samples"], CFG["spokes"], 2.0, 0.5,
                                                                   device=dev)),
                    args.steps, args.warmup, None, stream)
    t0 = time.perf_counter()
    O.radial_dcw_2d(CFG["samples"], CFG["spokes"], 2.0, 0.5)
    gen_cpu_ms = (time.perf_counter() - t0) * 1e3
    # density compensation estimate of the headline trajectory (Jinc kernel,
    # width 5.5, oversampling 2, 10 iterations)
    from gadgetron_b200 import sdc as SDC
    traj_d = torch.from_numpy(wl["traj"]).to(dev)
    sdc_ms = _timed(lambda: SDC.estimate_dcw(traj_d, N, 2.0, 10, 5.5), max(2, args.steps // 5), 1, None, stream)
    w_sdc = SDC.estimate_dcw(traj_d, N, 2.0, 10, 5.5)
    t0 = time.perf_counter()
    w_sdc_o = O.estimate_dcw(wl["traj"], N, 2.0, 10, 5.5)
    sdc_cpu_ms = (time.perf_counter() - t0) * 1e3
    # coil sensitivities from the coil images of the workload's phantom
    from gadgetron_b200 import b1map as B1
    rng_b1 = np.random.default_rng(12)
    coil_np = (wl["csm"] * wl["phantom"] + 0.01 * (rng_b1.standard_normal(wl["csm"].shape) +
                                                   1j * rng_b1.standard_normal(wl["csm"].shape))).astype(np.complex64)
    coil_d = torch.from_numpy(coil_np).to(dev)
    b1_ms = _timed(lambda: B1.estimate_b1_map(coil_d, 2), max(2, args.steps // 5), 1, None, stream)
    b1_d = B1.estimate_b1_map(coil_d, 2)
    t0 = time.perf_counter()
    b1_o = O.estimate_b1_map(coil_np, 2)
    b1_cpu_ms = (time.perf_counter() - t0) * 1e3
    R.set_weight(kappa)
    cg = gb.cuCgSolver()
    cg.set_encoding_operator(E)
    cg.add_regularization_operator(R)
    cg.set_preconditioner(D)
    cg.set_max_iterations(CFG["iterations"])
    cg.set_tc_tolerance(0.0)
    cg.set_use_graph(True)
    x = torch.empty((1, N[1], N[0]), dtype=torch.complex64, device=dev)
    l0 = gb.lib.gb_kernel_launch_count()
    ms = _timed(lambda: cg.solve(d_dev, x), args.steps, args.warmup, flush, stream)
    launches = (gb.lib.gb_kernel_launch_count() - l0) // (args.steps + args.warmup)
    O.set_fft_workers(os.cpu_count() or 1)
    plan = O.OraclePlan(N, wl["mos"], wl["W"])
    plan.preprocess(wl["traj"][None])
    orc = O.OracleSense(plan, wl["csm"], wl["sqrt_dcw"][None])
    R_o, off_o = O.image_operator_compute(reg.cpu().numpy())
    w_o = O.sense_precond_weights(wl["csm"], R_o[0], kappa)
    xr = O.cg_solve(orc, d_np[:, None, :], iterations=CFG["iterations"], tc_tolerance=0.0,
                    precond_weights=w_o[None], regularization=[(kappa, R_o)])
    return {
        "metric": "regularised CG-SENSE ms/recon (gadget form: image regulariser + preconditioner; 256^2, 16 coils, "
                  "96x512 samples, 10 CG iterations)",
        "value": round(ms, 4), "unit": "ms/recon", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 4), "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64 (fp32), fp64 CG reductions", "data": "synthetic (seeded)",
        "config": {"workload": "cg-sense-2d-regularised", "kappa": kappa, "regularisation_image": "E^H d",
                   "l2_flush": "256 MB write before every timed step"},
        "setup_ms_regulariser_and_preconditioner": round(setup_ms, 4),
        "setup_ms_trajectory_and_dcw_96x512": round(gen_ms, 4),
        "cpu_oracle_ms_dcw_96x512": round(gen_cpu_ms, 1),
        "sdc_ms_96x512_os2_10it": round(sdc_ms, 3), "cpu_oracle_ms_sdc": round(sdc_cpu_ms, 1),
        "sdc_rel_l2_vs_oracle": O.rel_l2(w_sdc.cpu().numpy(), w_sdc_o),
        "b1_map_ms_256x256x16": round(b1_ms, 3), "cpu_oracle_ms_b1_map": round(b1_cpu_ms, 1),
        "b1_map_rel_l2_vs_oracle": O.rel_l2(b1_d.cpu().numpy(), b1_o),
        "regulariser_offset": R.offset_, "regulariser_offset_oracle": off_o,
        "recon_rel_l2_vs_oracle_fp64_cg": O.rel_l2(x.cpu().numpy(), xr),
        "gpu_launches": int(launches),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="headline line without the NUFFT/preprocess/batched/reference-GPU figures")
    ap.add_argument("--workload", default="cg-sense-2d",
                    choices=["cg-sense-2d", "nufft-2d", "nufft-3d", "batched", "precision", "regularised"])
    ap.add_argument("--clocks-csv", default=None,
                    help="also write the raw clock samples of the timed region to this CSV path "
                         "(%%d = rank)")
    ap.add_argument("--size", default="full", choices=["full", "small"],
                    help="profiling cases: nufft-3d small = 64^3; batched small = 16 frames")
    ap.add_argument("--tiling", default=None,
                    help="batched workload: fixed tile and coil group 'tx,ty,cg' instead of the "
                         "autotuner's choice (profiling runs, whose launch timings the profiler skews)")
    ap.add_argument("--schedule", type=int, default=None, choices=[0, 1, 2],
                    help="batched workload: gridding schedule of the normal operator (0 by launch depth, "
                         "1 one CTA per work item, 2 persistent work queue); default 0")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return 0

    if args.workload != "cg-sense-2d":
        fn = {"nufft-2d": lambda: run_nufft(args, 2), "nufft-3d": lambda: run_nufft(args, 3),
              "batched": lambda: run_batched(args), "precision": lambda: run_precision(args),
              "regularised": lambda: run_regularized(args)}[args.workload]
        if rank == 0:
            print(json.dumps(fn()), flush=True)
        return 0

    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda:%d" % local_rank))
    out = run_ours(args, rank, world, local_rank)
    if rank == 0 and out is not None:
        result, wl, d_host, x_out = out
        # Accuracy of this run's reconstruction against the oracle CG (FP64)
        # and the operator's error against the direct NDFT on a sample subset.
        if world == 1 and not args.no_cpu_baseline:
            ms, ncpu, t_rhs, t_iter = cpu_cg_sample(wl, d_host)
            result["cpu_baseline"] = {"value": round(ms, 2), "unit": UNIT, "cores": ncpu, "kind": "port",
                                      "sample": "one E^H d + 3 CG iterations of the full workload on the reference's "
                                                "CPU path restated in float (CSR gridding, OpenMP over coils; "
                                                "complex64 pocketfft threads), scaled to 10 iterations"}
        try:
            result["accuracy"] = accuracy_report(wl, d_host, x_out)
        except Exception as e:  # accuracy is reported, never gates the timing
            result["accuracy"] = {"error": str(e)}
        if world == 1 and not args.no_extras:
            try:
                result.update(headline_extras(args, wl, d_host, x_out))
            except Exception as e:  # reported, never gates the timing
                result["extras_error"] = str(e)
        print(json.dumps(result), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


def _copy_args(args, **kw):
    a = argparse.Namespace(**vars(args))
    for k, v in kw.items():
        setattr(a, k, v)
    return a


def headline_extras(args, wl, d_host, x_out):
    """Figures the headline line carries besides the CG-SENSE time (N = 1
    only; computed after the timed region, never inside it):

    preprocess_ms  -- the SENSE operator's preprocess of the 49152-sample
                      trajectory alone (device time, CUDA events, L2 flushed);
    nufft_2d       -- the metric's first half: NUFFT forward C2NC + adjoint
                      NC2C throughput on 128^2, one coil, 128 golden-angle
                      spokes x 256 samples, alpha 2, W 5.5, with its error
                      against the reference's own cuNFFT and the FP64 NDFT;
    batched        -- 64 uneven frames (192^2, 12 coils, 15 iterations):
                      batched graph-captured solve vs the plain per-frame form;
    nufft_3d       -- the 3D kooshball NUFFT (128^3 -> 192^3, 5.12M samples, 32
                      coils, W 4): forward + adjoint throughput and the trajectory
                      gradient against central finite differences (64 samples);
    reference_gpu  -- the reference's own GPU path (built from its sources)
                      on the same B200: cuCgSolver ms/recon on this workload
                      and cuNFFT on the 2D NUFFT case, and the product's
                      per-iteration rel-L2 against the reference's iterates."""
    import torch
    import gadgetron_b200 as gb
    from gadgetron_b200 import synthetic as S
    from oracle import oracle as O
    from oracle import ref as R
    dev = x_out.device
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    out = {}
    # --- preprocess alone
    traj_d = torch.from_numpy(wl["traj"]).to(dev)
    E3 = gb.cuNonCartesianSenseOperator(2)
    E3.setup(wl["N"], wl["mos"], wl["W"])
    out["preprocess_ms"] = round(_timed(lambda: E3.preprocess(traj_d), 10, 3, flush, stream), 4)

    # --- NUFFT 2D forward + adjoint (single coil)
    N2, mos2, W2 = (128, 128), (256, 256), 5.5
    traj2 = S.radial_golden_angle_2d(128, 256)
    dcw2 = S.ramp_dcw(traj2)
    img2 = S.gaussian_image((1, 1, 128, 128), 11)
    M2 = traj2.shape[0]
    plan2 = gb.NFFT.make_plan(N2, mos2, W2)
    plan2.preprocess(torch.from_numpy(traj2).to(dev))
    x2 = torch.from_numpy(img2).to(dev)
    w2 = torch.from_numpy(dcw2).to(dev)
    y2 = torch.empty((1, M2), dtype=torch.complex64, device=dev)
    xb2 = torch.empty_like(x2)
    t_f = _timed(lambda: plan2.compute(x2, y2, None, gb.NFFT_comp_mode.FORWARDS_C2NC), 20, 3, flush, stream)
    t_a = _timed(lambda: plan2.compute(y2, xb2, w2, gb.NFFT_comp_mode.BACKWARDS_NC2C), 20, 3, flush, stream)
    nu = {"value": round(M2 / ((t_f + t_a) * 1e-3) / 1e6, 2), "unit": "Msample-coils/s",
          "ms_forward": round(t_f, 4), "ms_adjoint": round(t_a, 4),
          "config": {"workload": "nufft-2d-radial", "matrix": 128, "matrix_os": 256, "W": 5.5, "coils": 1,
                     "samples": M2, "l2": "flushed before every timed call"}}
    idx = np.random.default_rng(5).choice(M2, 4096, replace=False)
    yn = O.ndft_forward(img2[0, 0][None], traj2[idx], mos2)
    nu["forward_rel_l2_vs_fp64_ndft"] = O.rel_l2(y2[0].cpu().numpy()[idx], yn[0])
    ref_gpu = {}
    if R.available():
        y_ref = R.nfft_compute(N2, mos2, W2, traj2, 1, img2, None, "FORWARDS_C2NC")
        x_ref = R.nfft_compute(N2, mos2, W2, traj2, 1, y2.cpu().numpy(), dcw2, "BACKWARDS_NC2C")
        nu["forward_rel_l2_vs_reference"] = O.rel_l2(y2.cpu().numpy(), y_ref)
        nu["adjoint_rel_l2_vs_reference"] = O.rel_l2(xb2.cpu().numpy(), x_ref)
        rf, ra, rp = R.time_nfft(N2, mos2, W2, traj2, 1, img2, dcw2, 1, reps=10)
        ref_gpu["nufft_2d"] = {"ms_forward": round(rf, 4), "ms_adjoint": round(ra, 4),
                               "ms_preprocess": round(rp, 4),
                               "value": round(M2 / ((rf + ra) * 1e-3) / 1e6, 2), "unit": "Msample-coils/s"}
    out["nufft_2d"] = nu

    # --- batched uneven frames vs the plain per-frame form
    try:
        b = run_batched(_copy_args(args, steps=5, warmup=3, size="full", tiling=None))
        out["batched"] = {k: b[k] for k in ("value", "unit", "plain_per_frame_ms", "speedup_vs_plain",
                                            "batched_vs_plain_rel_l2", "tiling_after_autotune",
                                            "grid_schedule", "gpu_launches_per_batch")}
        out["batched"]["config"] = b["config"]
    except Exception as e:  # reported, never gates the headline
        out["batched"] = {"error": str(e)}

    # --- the reference's own GPU path on this workload
    if R.available():
        sq = wl["sqrt_dcw"]
        d = (d_host * sq.reshape(1, -1)).astype(np.complex64)
        ms_ref = R.time_cg_sense(wl["N"], wl["mos"], wl["W"], wl["traj"], 1, wl["csm"], sq, d,
                                 CFG["iterations"], reps=5)
        ref_gpu["cg_sense_ms_per_recon"] = round(ms_ref, 3)
        x_ref, its = R.cg_sense(wl["N"], wl["mos"], wl["W"], wl["traj"], 1, wl["csm"], sq, d,
                                CFG["iterations"], 0.0, keep_iterates=True)
        E = gb.cuNonCartesianSenseOperator(2)
        E.setup(wl["N"], wl["mos"], wl["W"])
        E.set_csm(torch.from_numpy(wl["csm"]).to(dev))
        E.set_dcw(torch.from_numpy(sq).to(dev))
        E.preprocess(traj_d)
        cg = gb.cuCgSolver()
        cg.set_encoding_operator(E)
        cg.set_tc_tolerance(0.0)
        d_t = torch.from_numpy(d).to(dev)
        per_it = []
        for k in range(1, CFG["iterations"] + 1):
            cg.set_max_iterations(k)
            per_it.append(O.rel_l2(cg.solve(d_t).cpu().numpy(), its[k - 1]))
        ref_gpu["recon_rel_l2_vs_reference"] = O.rel_l2(x_out.cpu().numpy(), x_ref)
        ref_gpu["per_iteration_rel_l2_vs_reference"] = [float("%.3g" % e) for e in per_it]
        ref_gpu["note"] = ("reference cuNFFT/cuNonCartesianSenseOperator/cuCgSolver compiled from its sources "
                           "for sm_100a, timed on this GPU with CUDA events (operator preprocessed, inputs "
                           "resident)")
    else:
        ref_gpu["unavailable"] = "oracle/_ref/libgbref.so not built"
    out["reference_gpu"] = ref_gpu

    # --- 3D kooshball NUFFT with the trajectory gradient (128^3 -> 192^3,
    # 20000 x 256 samples, 32 coils, W 4): throughput and the central
    # finite-difference check of the gradient on 64 samples
    try:
        n3 = run_nufft(_copy_args(args, steps=3, warmup=3, size="full"), 3)
        out["nufft_3d"] = {k: n3[k] for k in ("value", "unit", "ms_forward", "ms_adjoint", "config",
                                              "forward_rel_l2_vs_fp64_ndft", "fd_gradient")}
    except Exception as e:  # reported, never gates the headline
        out["nufft_3d"] = {"error": str(e)}
    return out


def accuracy_report(wl, d_host, x_out, n_sub=2048):
    """rel-L2 of the GPU recon vs the oracle CG (FP64), and of the GPU forward
    operator vs the FP64 direct NDFT on n_sub samples of every coil."""
    import torch
    import gadgetron_b200 as gb
    from oracle import oracle as O
    O.set_fft_workers(os.cpu_count() or 1)
    P = O.OraclePlan(wl["N"], wl["mos"], wl["W"])
    P.preprocess(wl["traj"][None])
    sq = wl["sqrt_dcw"].reshape(1, -1)
    E = O.OracleSense(P, wl["csm"], sq)
    d = (d_host * sq)[:, None, :]
    xr = O.cg_solve(E, d, iterations=CFG["iterations"], tc_tolerance=0.0)
    err_cg = O.rel_l2(x_out.cpu().numpy(), xr)
    # operator vs NDFT on a subset
    dev = x_out.device
    Eg = gb.cuNonCartesianSenseOperator(2)
    Eg.setup(wl["N"], wl["mos"], wl["W"])
    Eg.set_csm(torch.from_numpy(wl["csm"]).to(dev))
    Eg.preprocess(torch.from_numpy(wl["traj"]).to(dev))
    C, M = wl["csm"].shape[0], wl["traj"].shape[0]
    y = torch.empty((C, M), dtype=torch.complex64, device=dev)
    Eg.mult_M(torch.from_numpy(wl["phantom"]).to(dev), y)
    idx = np.random.default_rng(3).choice(M, n_sub, replace=False)
    coil_imgs = wl["csm"] * wl["phantom"]
    yn = O.ndft_forward(coil_imgs, wl["traj"][idx], wl["mos"])
    err_ndft = O.rel_l2(y.cpu().numpy()[:, idx], yn)
    return {"recon_rel_l2_vs_oracle_cg": err_cg, "forward_rel_l2_vs_fp64_ndft": err_ndft,
            "ndft_subset_samples": n_sub}


if __name__ == "__main__":
    sys.exit(main())
