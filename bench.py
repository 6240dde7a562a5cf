"""Benchmark of the space-charge tracking step (one JSON line on stdout).

Workload (default): one Gaussian electron bunch of 1,000,000 macro-particles
on a 64^3 mesh (128^3 doubled grid), 1 nC, dt = 1 ps, plain FP64 form --
the single-GPU configuration the reference metric is quoted on.  A "step" is
one ParallelTTracker step: half drift, space-charge fields (deposit, Hockney
FFT convolution with the integrated Green's function, gather), Boris kick,
half drift, reference-frame update.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--precision fp64|mixed]

value    particle-steps/s, device time (CUDA events) of K steps, the bunch
         resident in HBM; L2 flushed before every timed step.
e2e      the same metric through the C ABI with host buffers: every step
         uploads R, P from pinned host memory, runs scgpu_track(1) and
         downloads R, P (the DKS offload seam of the reference,
         ParallelTTracker.h:514-562).
Multi-GPU: independent replicas (one bunch per rank); no data-path collective.
"""
from __future__ import annotations

import argparse
import datetime
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DT = 1e-12
# name -> (particles, mesh cells per axis, uniform B_z [T], description)
WORKLOADS = {
    "c2": (1_000_000, 64, 0.0, "gaussian bunch 1e6 e-, 64^3 mesh (128^3 doubled), 1 nC, dt 1 ps, drift"),
    "c3": (10_000_000, 128, 0.2, "gaussian bunch 1e7 e-, 128^3 mesh (256^3 doubled), 1 nC, dt 1 ps, "
                                 "uniform solenoid B_z = 0.2 T"),
}
N_PARTICLES, MESH, BZ, WORKLOAD = WORKLOADS["c2"]
REORDER_EVERY = 32  # the library's default cell-reorder interval


def algorithmic_bytes(N, n, precision):
    """Per-step algorithmic HBM bytes of the whole step and of each phase.
    FP64 step model: 96 N + 32 M + 48 S + 16 G3 (M = n^3, S = (n+1)(2n)^2,
    G3 = (n+1)^3); mixed halves the grid terms except the FP64 G build."""
    M = n ** 3
    S = (n + 1) * (2 * n) ** 2
    G3 = (n + 1) ** 3
    r = 8 if precision == "fp64" else 4
    step = 96 * N + 4 * r * M + 6 * r * S + 16 * G3
    phases = {
        "drift_bounds": 72 * N,                    # read R, P; write R (beam frame)
        "deposit": 24 * N + 16 * M,                # read R; 128-bit node accumulators
        "assemble_rho": 16 * M + r * M,            # node accumulators in, rho out
        "green": 16 * G3,                          # G write + read
        "convolution": 2 * r * M + 6 * r * S,      # rho in, phi out, spectrum traffic
        "grad": r * M + 3 * r * M,                 # phi in, 3-component E out
        "gather_kick_push": 96 * N + 3 * r * M,    # R, P in and out; E read
        "reorder": 0,                              # amortised cell-order sort (no algorithmic bytes)
    }
    return step, phases


SINGLE_KERNEL_PHASES = ("drift_bounds", "deposit", "assemble_rho", "grad", "gather_kick_push")


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic(kernel, workload, precision):
    """DRAM bytes per launch of a kernel from the committed ncu summary of
    the same workload and precision (None when that capture does not exist)."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        t = json.load(f)
    v = t.get(f"{workload}/{precision}", {}).get(kernel)
    return None if v is None else float(v)


def reorder_cost_ms(ctx, stream, flush, every, steps_done, rounds=2, plain=3):
    """Extra device time of a step that also puts the particles in cell
    order: a reorder step against the plain steps that follow it, L2 flushed
    before each, averaged over `rounds` reorder intervals.  Returns (ms,
    steps advanced)."""
    import torch

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    extra, advanced = [], 0
    for _ in range(rounds):
        k = (-(steps_done + advanced)) % every
        if k:
            ctx.track(k)
            advanced += k
        t = []
        for _ in range(1 + plain):
            flush.zero_()
            ev[0].record(stream)
            ctx.track(1)
            ev[1].record(stream)
            ev[1].synchronize()
            t.append(ev[0].elapsed_time(ev[1]))
            advanced += 1
        extra.append(t[0] - sum(t[1:]) / plain)
    return max(0.0, sum(extra) / rounds), advanced


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = str(device_index)
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        if not self.lines:
            # a timed region shorter than the sampling period: one sample as it ends
            try:
                out = subprocess.run(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits"],
                                     capture_output=True, text=True, timeout=10).stdout
                self.lines.extend(l.strip() for l in out.splitlines() if l.strip())
            except (OSError, subprocess.TimeoutExpired):
                pass
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9 or parts[0] != self.idx:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args, world, rank):
    """The reference's CPU path (the oracle restatement with the reference's own
    FFTPACK engine), all host threads, on the same workload."""
    if rank != 0:
        return
    from oracle import oracle as O
    from src_b200.bunch import config_bunch

    threads = O.lib().sco_max_threads()
    O.lib().sco_set_threads(threads)
    if O.reference_fft_available():
        O.use_reference_fft(True)
    b = config_bunch("c2")
    tr = O.OracleTracker(O.make_params(b["nr"], b["dT"]), b["Q"])
    R, P = b["R"].copy(), b["P"].copy()
    t0 = time.perf_counter()
    tr.track(R, P, args.warmup)
    per_step = (time.perf_counter() - t0) / args.warmup
    # bound the run to about two minutes of host time
    timed = max(1, min(args.steps, int(120.0 / max(per_step, 1e-6))))
    t0 = time.perf_counter()
    tr.track(R, P, timed)
    el = time.perf_counter() - t0
    value = b["N"] * timed / el
    sample = (f"{timed} of {args.steps} requested full tracking steps of the 1e6-particle / 64^3 workload, "
              f"{threads} host threads ({'reference FFTPACK' if not O.fft_engine_is_own() else 'oracle FFT'} engine)")
    el = el * args.steps / timed
    line = {
        "impl": "reference", "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "particles": b["N"], "mesh": MESH, "precision": "fp64",
                   "l2": "n/a (host)"},
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline_single(target_s=12.0):
    """Oracle port, 1 thread, bounded sample of the same workload."""
    from oracle import oracle as O
    from src_b200.bunch import config_bunch

    O.lib().sco_set_threads(1)
    if O.reference_fft_available():
        O.use_reference_fft(True)
    b = config_bunch("c2")
    tr = O.OracleTracker(O.make_params(b["nr"], b["dT"]), b["Q"])
    R, P = b["R"].copy(), b["P"].copy()
    t0 = time.perf_counter()
    tr.track(R, P, 1)
    one = time.perf_counter() - t0
    steps = max(1, int(target_s / max(one, 1e-3)))
    t0 = time.perf_counter()
    tr.track(R, P, steps)
    el = time.perf_counter() - t0
    return {"value": b["N"] * steps / el, "unit": "particle-steps/s", "cores": 1, "kind": "port",
            "sample": f"{steps} full tracking steps of the 1e6-particle / 64^3 workload on 1 core "
                      f"({'reference FFTPACK' if not O.fft_engine_is_own() else 'oracle FFT'} engine)"}


def cpu_baseline_c1(target_s=6.0):
    """The CPU figures of the 1e5-particle / 32^3 workload (c1): the oracle
    port with the reference's FFTPACK on 1 core and on all host threads,
    bounded samples of the 100-step run."""
    from oracle import oracle as O
    from src_b200.bunch import config_bunch

    if O.reference_fft_available():
        O.use_reference_fft(True)
    b = config_bunch("c1")
    out = {}
    for label, threads in (("1_core", 1), ("all_cores", O.lib().sco_max_threads())):
        O.lib().sco_set_threads(threads)
        tr = O.OracleTracker(O.make_params(b["nr"], b["dT"]), b["Q"])
        R, P = b["R"].copy(), b["P"].copy()
        t0 = time.perf_counter()
        tr.track(R, P, 1)
        one = time.perf_counter() - t0
        steps = max(1, min(b["steps"] - 1, int(target_s / max(one, 1e-3))))
        t0 = time.perf_counter()
        tr.track(R, P, steps)
        el = time.perf_counter() - t0
        out[label] = {"value": b["N"] * steps / el, "unit": "particle-steps/s", "cores": threads, "kind": "port",
                      "sample": f"steps 2-{steps + 1} of the 100-step 1e5-particle / 32^3 run "
                                f"({'reference FFTPACK' if not O.fft_engine_is_own() else 'oracle FFT'} engine)"}
    O.lib().sco_set_threads(1)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS),
                    help="c2: 1e6 particles / 64^3 (the default bench line); c3: 1e7 / 128^3 with B_z = 0.2 T")
    ap.add_argument("--compare-precision", action="store_true",
                    help="run the plain and the mixed form on the same bunch for --steps steps and report "
                         "the mixed form's field and emittance error against FP64 (one JSON line)")
    ap.add_argument("--batched", action="store_true",
                    help="batched form: 64 bunches of mixed sizes and meshes in one batch (one JSON line)")
    ap.add_argument("--serve", action="store_true",
                    help="serving loop: Poisson arrivals at 50 jobs/s for --serve-seconds (one JSON line)")
    ap.add_argument("--serve-seconds", type=float, default=60.0)
    ap.add_argument("--serve-rate", type=float, default=50.0, help="Poisson arrival rate of the serving loop [jobs/s]")
    ap.add_argument("--binned", action="store_true",
                    help="photoinjector mode: energy bins with image charges (one JSON line)")
    ap.add_argument("--nbins", type=int, default=10)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    global N_PARTICLES, MESH, BZ, WORKLOAD
    N_PARTICLES, MESH, BZ, WORKLOAD = WORKLOADS[args.workload]
    world, rank, local = dist_setup()
    if args.compare_precision:
        compare_precision(args, local)
        return
    if args.batched:
        batched(args, local)
        return
    if args.serve:
        serve(args, local)
        return
    if args.binned:
        binned(args, local)
        return

    if args.impl == "reference":
        run_reference(args, world, rank)
        return

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    from src_b200 import scgpu
    from src_b200.bunch import gaussian_bunch

    prec = scgpu.PLAIN_FP64 if args.precision == "fp64" else scgpu.MIXED
    R, P = gaussian_bunch(N_PARTICLES, bunch_id=rank)
    Q = -1e-9 / N_PARTICLES
    mass = 0.51099892e-03 * 1.0e9
    ctx = scgpu.Context((MESH, MESH, MESH), precision=prec, device=local)
    stream = torch.cuda.current_stream(dev)
    ctx.set_stream(stream.cuda_stream)
    ctx.set_reorder_interval(REORDER_EVERY)
    ctx.upload(R, P, DT, Q, mass, bz_ext=BZ)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

    # warm-up (also builds the step's CUDA graph)
    ctx.track(args.warmup)
    kernels = ctx.kernels_per_step()
    torch.cuda.synchronize(dev)

    # ---- timed region: K steps, device time, L2 flushed before each step
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    launched0 = ctx.launch_count()
    wall0 = time.perf_counter()
    for k in range(args.steps):
        flush.zero_()
        starts[k].record(stream)
        ctx.track(1)
        ends[k].record(stream)
    torch.cuda.synchronize(dev)
    wall = time.perf_counter() - wall0
    launched = ctx.launch_count() - launched0  # reorder steps' extra kernels included
    clk = clocks.stop()
    if world > 1:
        dist.barrier()
    ms_measured = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    # The cell reorder runs every REORDER_EVERY steps counted from the
    # upload; a window of K steps holds K / REORDER_EVERY of them on average
    # but may hold none or one.  The whole job's rate counts the average:
    # the window's own reorders are exchanged for K / REORDER_EVERY times
    # the measured cost of one.
    in_window = sum(1 for k in range(args.warmup, args.warmup + args.steps) if k % REORDER_EVERY == 0)
    reorder_ms, _ = reorder_cost_ms(ctx, stream, flush, REORDER_EVERY, args.warmup + args.steps)
    ms = ms_measured + (args.steps / REORDER_EVERY - in_window) * reorder_ms
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * N_PARTICLES * args.steps / (ms_max * 1e-3)

    # ---- per-phase device times (serialised phases), the dominant kernel's roofline
    nprof = min(max(args.steps // 10, 20), 200)
    phases = ctx.profile(nprof)
    step_bytes, phase_bytes = algorithmic_bytes(N_PARTICLES, MESH, args.precision)
    peak, peak_kind = measured_peaks()
    # the dominant kernel: the longest phase that is one kernel (the Green's
    # function and the convolution phases are several short launches each)
    dom = max((k for k in phases if k in SINGLE_KERNEL_PHASES), key=phases.get)
    dom_ms = phases[dom] / nprof
    achieved = phase_bytes[dom] / (dom_ms * 1e-3) / 1e9
    traffic = committed_traffic(dom, args.workload, args.precision)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                "algorithmic_bytes": phase_bytes[dom], "avg_launch_ms": dom_ms}
    step_ms = ms_max / args.steps
    step_roofline = {"achieved": step_bytes / (step_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": step_bytes / (step_ms * 1e-3) / 1e9 / peak, "algorithmic_bytes": step_bytes}

    # ---- e2e through the C ABI with host buffers (per-step offload)
    e2e_steps = max(5, min(args.steps // 20, 50))
    Rh = torch.empty((N_PARTICLES, 3), dtype=torch.float64, pin_memory=True).numpy()
    Ph = torch.empty((N_PARTICLES, 3), dtype=torch.float64, pin_memory=True).numpy()
    Rh[:] = R
    Ph[:] = P
    st = ctx.tracker_state()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    e0.record(stream)
    for _ in range(e2e_steps):
        ctx.upload(Rh, Ph, DT, Q, mass, t=st["t"], path_length=st["path_length"], ref_R=st["ref_R"],
                   ref_P=st["ref_P"], bz_ext=BZ)
        ctx.track(1)
        ctx.download(Rh, Ph)
        st = ctx.tracker_state()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = e0.elapsed_time(e1)
    t = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_value = world * N_PARTICLES * e2e_steps / (float(t.item()) * 1e-3)

    # ---- e2e of a resident tracking job: upload once, per-step statistics
    # records to pinned host memory, download at the end
    job_steps = max(10, min(args.steps // 5, 200))
    stats = torch.empty((job_steps, scgpu.NSTATS), dtype=torch.float64, pin_memory=True).numpy()
    torch.cuda.synchronize(dev)
    e0.record(stream)
    ctx.upload(Rh, Ph, DT, Q, mass, bz_ext=BZ)
    ctx.track(job_steps, stats)
    ctx.download(Rh, Ph)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    job_value = N_PARTICLES * job_steps / (e0.elapsed_time(e1) * 1e-3)

    ctx.close()
    cpu = cpu_c1 = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload == "c2":
        cpu = cpu_baseline_single()
        cpu_c1 = cpu_baseline_c1()
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "particles": N_PARTICLES * world, "particles_per_gpu": N_PARTICLES,
                   "mesh": MESH, "precision": args.precision, "parallelism": f"replicas x{world}",
                   "l2": "flushed before every timed step (256 MiB write)"},
        "e2e": {"value": e2e_value, "unit": "particle-steps/s", "h2d_bytes_per_step": 48 * N_PARTICLES,
                "d2h_bytes_per_step": 48 * N_PARTICLES + 8 * 13, "steps": e2e_steps,
                "mode": "per-step upload / scgpu_track(1) / download of R, P (pinned host)"},
        "e2e_resident_job": {"value": job_value, "unit": "particle-steps/s", "steps": job_steps,
                             "h2d_bytes_per_step": 48 * N_PARTICLES / job_steps,
                             "d2h_bytes_per_step": 8 * scgpu.NSTATS + 48 * N_PARTICLES / job_steps},
        "roofline": roofline,
        "step_roofline": step_roofline,
        "phases_ms_per_step": {k: v / nprof for k, v in phases.items()},
        "gpu_launches": launched,
        "kernels_per_step": kernels,
        "clocks": clk,
        "wall_s_timed_region": wall,
        "reorder": {"interval": REORDER_EVERY, "in_window": in_window, "cost_ms": reorder_ms,
                    "ms_per_step_measured": ms_measured / args.steps,
                    "note": "value counts K / interval reorders at the measured cost in place of the window's own"},
        "cpu_baseline": cpu,
        "cpu_baseline_c1": cpu_c1,
    }
    print(json.dumps(line), flush=True)


def compare_precision(args, local):
    """Mixed form against the plain FP64 form on the same bunch: the field
    error of the first solve (identical inputs), the field error after
    --steps steps, and the largest relative difference of the normalised rms
    emittances over all steps (per-step statistics records)."""
    import torch

    from src_b200 import scgpu
    from src_b200.bunch import gaussian_bunch

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    R0, P0 = gaussian_bunch(N_PARTICLES, bunch_id=0)
    Q = -1e-9 / N_PARTICLES
    mass = 0.51099892e-03 * 1.0e9
    out = {}
    for name, prec in (("fp64", scgpu.PLAIN_FP64), ("mixed", scgpu.MIXED)):
        with scgpu.Context((MESH, MESH, MESH), precision=prec, device=local) as c:
            stream = torch.cuda.current_stream(dev)
            c.set_stream(stream.cuda_stream)
            c.upload(R0, P0, DT, Q, mass, bz_ext=BZ)
            first = np.zeros((1, scgpu.NSTATS))
            c.track(1, first)
            E1 = c.field(scgpu.FIELD_E)
            stats = np.zeros((args.steps, scgpu.NSTATS))
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            c.track(args.steps, stats)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            ms = e0.elapsed_time(e1)
            E = c.field(scgpu.FIELD_E)
            R, P = c.download()
            eps = np.array([scgpu.beam_parameters_from_stats(r, N_PARTICLES)["eps_norm"] for r in stats])
            out[name] = dict(E1=E1, E=E, R=R, P=P, eps=eps, ms_per_step=ms / args.steps)

    def rel(a, b):
        return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))

    d, m = out["fp64"], out["mixed"]
    drift = np.abs(m["eps"] - d["eps"]) / np.abs(d["eps"])
    line = {
        "metric": "mixed-form error vs FP64", "workload": WORKLOAD, "steps": args.steps + 1,
        "field_rel_err_first_solve": rel(m["E1"], d["E1"]),
        "field_rel_err_final": rel(m["E"], d["E"]),
        "emittance_rel_drift_max": float(drift.max()),
        "emittance_rel_drift_final": [float(v) for v in drift[-1]],
        "eps_norm_final_fp64": [float(v) for v in d["eps"][-1]],
        "R_rel_err_final": rel(m["R"], d["R"]), "P_rel_err_final": rel(m["P"], d["P"]),
        "ms_per_step": {"fp64": d["ms_per_step"], "mixed": m["ms_per_step"]},
        "speedup_mixed_over_fp64": d["ms_per_step"] / m["ms_per_step"],
        "bounds": {"field": 1e-5, "emittance_drift": 1e-6},
        "norms": "max|mixed - fp64| / max|fp64| over all mesh points (E) or particles (R, P)",
    }
    print(json.dumps(line), flush=True)


def batched(args, local):
    """64 bunches (particle counts log-uniform in [1e4, 5e5], meshes from
    {16, 32, 48, 64}^3, sigma, charge and beta*gamma drawn per bunch) in one
    batch: autotuned launch shapes, then --steps (200 unless given) timed
    batched steps.  Beside it, the same bunches one after another in
    single-bunch contexts (a probe of a few steps each, scaled), the way one
    tracker per design point would run them."""
    import torch

    from src_b200 import scgpu
    from src_b200.serving import MasterBunches
    from src_b200.workloads import DT as WDT, MASS_EV, batched_jobs

    torch.cuda.set_device(local)
    prec = scgpu.PLAIN_FP64 if args.precision == "fp64" else scgpu.MIXED
    steps = args.steps if args.steps != 1000 else 200
    jobs = batched_jobs(steps=steps)
    masters = MasterBunches(count=4, size=max(j.particles for j in jobs))
    data = [masters.bunch(j) for j in jobs]
    total_particles = sum(j.particles for j in jobs)
    with scgpu.Batch(precision=prec, device=local) as bt:
        for j, (R, P) in zip(jobs, data):
            bt.add((j.mesh,) * 3, R, P, WDT, j.q_macro, MASS_EV, ref_P=j.ref_P)
        tuned_steps = bt.autotune(3)
        tuning = {L: bt.tuning(L) for L in (32, 64, 96, 128)}
        bt.track(args.warmup)
        clocks = ClockSampler(local)
        clocks.start()
        ms = bt.track(steps)
        clk = clocks.stop()
    value = total_particles * steps / (ms * 1e-3)
    seq_ms = 0.0
    probe = 10
    for j, (R, P) in zip(jobs, data):
        with scgpu.Context((j.mesh,) * 3, precision=prec, device=local) as c:
            c.upload(R, P, WDT, j.q_macro, MASS_EV, ref_P=j.ref_P)
            c.track(3)
            seq_ms += c.track(probe) / probe * steps
    line = {
        "metric": "batched particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": 1,
        "steps": steps, "warmup": args.warmup, "ms_per_step": ms / steps, "higher_is_better": True,
        "precision": args.precision, "bunches": len(jobs), "particles_total": total_particles,
        "meshes": {str(m): sum(1 for j in jobs if j.mesh == m) for m in (16, 32, 48, 64)},
        "autotune": {"steps_taken": tuned_steps, "choices": {str(k): v for k, v in tuning.items()}},
        "sequential_single_contexts": {"value": total_particles * steps / (seq_ms * 1e-3), "ms": seq_ms,
                                       "note": f"each bunch alone, {probe}-step probe scaled to {steps} steps"},
        "speedup_vs_sequential": seq_ms / ms,
        "clocks": clk, "data": "synthetic (seeded)",
    }
    print(json.dumps(line), flush=True)


def binned(args, local):
    """Photoinjector mode: the energy-bin loop with image charges
    (ParallelTTracker.cpp:567-578, PartBunch::computeSelfFields(int bin)):
    a 1e6-particle bunch near the cathode with --nbins energy bins (seeded
    photoinjector_bunch) on a 64^3 mesh; per step and bin two Green's
    functions and two convolutions.  --steps (100 unless given) timed steps,
    device time, bunch resident; L2 flushed before each step.  Beside it the
    oracle's binned step on the host (one core, 1e5 particles / 32^3, one
    step) as the CPU reference of this mode."""
    import torch

    from src_b200 import scgpu
    from src_b200.bunch import photoinjector_bunch

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    prec = scgpu.PLAIN_FP64 if args.precision == "fp64" else scgpu.MIXED
    steps = args.steps if args.steps != 1000 else 100
    N, mesh, nb = N_PARTICLES, MESH, args.nbins
    R, P, bins = photoinjector_bunch(N, nbins=nb)
    Q = -1e-9 / N
    mass = 0.51099892e-03 * 1.0e9
    with scgpu.Context((mesh,) * 3, precision=prec, device=local) as c:
        stream = torch.cuda.current_stream(dev)
        c.set_stream(stream.cuda_stream)
        c.upload(R, P, DT, Q, mass, ref_P=(0.0, 0.0, 1.0))
        c.set_energy_bins(bins, nb)
        c.track(args.warmup)
        kernels = c.kernels_per_step()
        flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        torch.cuda.synchronize(dev)
        clocks = ClockSampler(local)
        clocks.start()
        launched0 = c.launch_count()
        for k in range(steps):
            flush.zero_()
            starts[k].record(stream)
            c.track(1)
            ends[k].record(stream)
        torch.cuda.synchronize(dev)
        clk = clocks.stop()
        launched = c.launch_count() - launched0
        ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends))
        gam, cnt = c.bin_gammas()
        bp = c.beam_parameters()
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        O.lib()
        Rc, Pc, bc = photoinjector_bunch(100_000, nbins=nb, bunch_id=1)
        tr = O.OracleTracker(O.make_params((32, 32, 32), DT, ref_pz=1.0), -1e-9 / 100_000)
        t0 = time.perf_counter()
        tr.track(Rc, Pc, 1, bins=bc, nbins=nb)
        cs = time.perf_counter() - t0
        cpu = {"value": 100_000 / cs, "unit": "particle-steps/s", "cores": 1, "kind": "port",
               "sample": f"oracle binned step, 1e5 particles, 32^3, {nb} bins, 1 step ({cs:.2f} s)"}
    line = {
        "metric": "particle-steps/s (energy bins + image charges)", "value": N * steps / (ms * 1e-3),
        "unit": "particle-steps/s", "n_gpus": 1, "steps": steps, "warmup": args.warmup,
        "ms_per_step": ms / steps, "higher_is_better": True, "precision": args.precision,
        "config": {"workload": f"photoinjector bunch {N} e-, {mesh}^3 mesh, {nb} energy bins, image charges",
                   "l2": "flushed before every timed step (256 MiB write)"},
        "ms_per_bin": ms / steps / nb, "kernels_per_step": kernels, "gpu_launches": launched,
        "bin_gammas": [float(g) for g in gam], "eps_norm": [float(v) for v in bp["eps_norm"]],
        "clocks": clk, "cpu_baseline": cpu, "data": "synthetic (seeded)",
    }
    print(json.dumps(line), flush=True)


def serve(args, local):
    """Serving loop: jobs arrive by a Poisson process at 50 jobs/s for
    --serve-seconds; each is admitted by HBM footprint into the running batch
    and advanced with the others; reports throughput and p50/p99 latency."""
    import torch

    from src_b200 import scgpu
    from src_b200.serving import MasterBunches, Server, latency_summary
    from src_b200.workloads import Job, serving_jobs

    torch.cuda.set_device(local)
    prec = scgpu.PLAIN_FP64 if args.precision == "fp64" else scgpu.MIXED
    jobs = serving_jobs(rate_hz=args.serve_rate, duration_s=args.serve_seconds)
    masters = MasterBunches(count=4, size=max(j.particles for j in jobs))
    srv = Server(precision=prec, masters=masters)
    cal = [Job(100000 + i, 0.0, 200_000, m, (1e-3, 1e-3, 2e-3), 10.0, 1.0, 10)
           for i, m in enumerate(sorted({j.mesh for j in jobs}))]
    tuning = srv.calibrate(cal)
    clocks = ClockSampler(local)
    clocks.start()
    try:
        res = srv.run(jobs, realtime=True)
    finally:
        srv.close()
    clk = clocks.stop()
    lat = latency_summary(res)
    line = {
        "metric": "serving p50/p99 job latency and throughput", "precision": args.precision,
        "arrival_rate_hz": args.serve_rate, "window_s": args.serve_seconds, "jobs": len(res),
        "device_busy_frac": srv.time["track_gpu_s"] / srv.makespan_s,
        "throughput": {"value": srv.particle_steps / srv.makespan_s, "unit": "particle-steps/s"},
        "particle_steps": srv.particle_steps, "latency_s": lat, "makespan_s": srv.makespan_s,
        "rounds": srv.rounds, "host_time": srv.time, "hbm_budget_gb": srv.budget / 1e9,
        "tuning": {str(k): v for k, v in tuning.items()},
        "clocks": clk, "data": "synthetic (seeded Poisson arrivals, log-uniform 1e4..2e6 particles, 16..128^3)",
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
