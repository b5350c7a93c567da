"""Benchmark of the 2D2V Vlasov-Poisson Strang step on B200.

Workload (default): the bandwidth-roofline configuration, 2D2V linear Landau
damping on a 128^4 grid (268,435,456 cells), FP32 storage of f, amplitude
0.05, k = 0.5 (Lx = Ly = 4 pi), v in [-6, 6], dt = 0.1. A "step" is one full
Strang step (x, y + rho, FP64 Poisson, vx + vy kick, y, x, diagnostics).
Metric: cell-updates/s = Nx*Ny*Nvx*Nvy * steps / seconds. Inputs are
synthetic (the initial condition is generated, nothing is downloaded);
f is 1 GiB, far above the 126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--dtype float32|bfloat16|float64] [--size 128]

--impl reference times the CPU restatement of the reference's algorithm
(the oracle: C + OpenMP over all host threads) on a bounded sample of the
same workload; the reference itself is Python that is not present on the
GPU host.
"""
from __future__ import annotations

import argparse
import ctypes
import importlib
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAK_FALLBACK_GBS = 6650.0
LX = 4.0 * math.pi
VMAX = 6.0
DT = 0.1
EPS = 0.05
KMODE = 0.5

PHASES = ("drift_x1", "drift_y1_rho", "field", "kick_vx_vy", "drift_y2", "drift_x2", "diag")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--dtype", choices=["float32", "bfloat16", "float64"], default="float32")
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU work for cpu_baseline")
    return ap.parse_args()


def workload_name(n, dtype):
    return f"2D2V Landau {n}x{n}x{n}x{n} {dtype} storage, eps={EPS}, k={KMODE}, v in [-6,6], dt={DT}"


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return PEAK_FALLBACK_GBS, "fallback"


def ncu_traffic(kernel_tag):
    """dram bytes per launch from a committed ncu summary (profiles/*.txt with a
    'dram_bytes_per_launch: <n>' line), or None."""
    p = os.path.join(ROOT, "profiles", f"traffic_{kernel_tag}.txt")
    try:
        with open(p) as fh:
            for line in fh:
                if line.startswith("dram_bytes_per_launch:"):
                    return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU side (the oracle): cpu_baseline and --impl reference
# ---------------------------------------------------------------------------
def cpu_sample(n, dtype_name, budget_s, min_steps=1):
    """Time the oracle's Strang step on (n, n, m, m) with m <= n chosen so the
    timed steps take about budget_s. Returns (cells_per_step, steps, seconds, m)."""
    import numpy as np

    from oracle import core as O

    npdt = np.float64 if dtype_name == "float64" else np.float32
    # calibrate on a small grid
    g = O.make_grid2d(n, n, 16, 16, LX, LX, VMAX, VMAX, dtype=npdt)
    st = O.Stepper2D(g, DT, window=1)
    f = O.landau_2d(g, EPS, KMODE)
    st.step(f)
    t0 = time.perf_counter()
    st.step(f)
    rate = (n * n * 256) / (time.perf_counter() - t0)
    m = 16
    for cand in (n, 96, 64, 48, 32, 24, 16):
        if cand <= n and (n * n * cand * cand) / rate * min_steps <= budget_s:
            m = cand
            break
    g = O.make_grid2d(n, n, m, m, LX, LX, VMAX, VMAX, dtype=npdt)
    st = O.Stepper2D(g, DT, window=1)
    f = O.landau_2d(g, EPS, KMODE)
    f = st.step(f).f  # warm-up
    steps = max(min_steps, int(budget_s / ((n * n * m * m) / rate)))
    t0 = time.perf_counter()
    for _ in range(steps):
        f = st.step(f).f
    sec = time.perf_counter() - t0
    return n * n * m * m, steps, sec, m


def run_reference(args):
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return 0
    from oracle import core as O

    n = args.size
    cores = O.num_threads()
    # each step is one Strang step of a bounded sample of the workload: the
    # whole --warmup + --steps run is kept to about three minutes
    per_step_budget = max(1.0, 150.0 / max(1, args.steps + args.warmup))
    cells, _, sec, m = cpu_sample(n, args.dtype, per_step_budget)
    import numpy as np

    npdt = np.float64 if args.dtype == "float64" else np.float32
    g = O.make_grid2d(n, n, m, m, LX, LX, VMAX, VMAX, dtype=npdt)
    st = O.Stepper2D(g, DT, window=1)
    f = O.landau_2d(g, EPS, KMODE)
    for _ in range(args.warmup):
        f = st.step(f).f
    t0 = time.perf_counter()
    for _ in range(args.steps):
        f = st.step(f).f
    sec = time.perf_counter() - t0
    value = cells * args.steps / sec
    sample = (f"oracle Strang step (C+OpenMP restatement of vlasov_step_gather_free) on a "
              f"{n}x{n}x{m}x{m} sample of the workload, {args.steps} steps after {args.warmup} warm-up")
    line = {
        "impl": "reference", "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.dtype != "float64"
        else "f64", "data": "synthetic",
        "config": {"workload": workload_name(n, args.dtype), "sample_grid": [n, n, m, m]},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU side
# ---------------------------------------------------------------------------
def run_ours(args):
    import torch

    vp = importlib.import_module("jax-pytorch-vlasov_b200")
    from importlib import import_module

    dist = import_module("jax-pytorch-vlasov_b200.dist")
    v2 = import_module("jax-pytorch-vlasov_b200.vlasov2d2v")
    L = vp._lib

    rank, local, world = dist.init()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.size
    dtype = {"float32": torch.float32, "bfloat16": torch.bfloat16, "float64": torch.float64}[args.dtype]
    esz = {torch.float32: 4, torch.bfloat16: 2, torch.float64: 8}[dtype]
    cells = n ** 4

    st = vp.Stepper2D(n, n, n, n, LX, LX, VMAX, VMAX, DT, dtype=dtype, device=dev, physics_mode=True, window=1,
                      diagnostics=True)
    # Landau initial condition, built on the device (not timed); each rank runs
    # an independent replica with its own amplitude
    gdt = torch.float64
    x = torch.linspace(0, LX, n + 1, dtype=gdt, device=dev)[:-1]
    v = torch.linspace(-VMAX, VMAX, n, dtype=gdt, device=dev)
    eps = EPS * (1.0 + 0.01 * rank)
    sp = 1.0 + eps * (torch.cos(KMODE * x)[:, None] + torch.cos(KMODE * x)[None, :])
    fv = torch.exp(-0.5 * (v[:, None] ** 2 + v[None, :] ** 2)) / (2.0 * math.pi)
    f = (sp.float()[:, :, None, None] * fv.float()[None, None]).to(dtype).contiguous()
    del sp, fv
    b = st.empty_f()
    diag = torch.zeros((max(args.steps, 1), L.DIAG_COUNT), dtype=torch.float64, device=dev)

    # per-phase timing events recorded by the library inside each step
    nph = len(PHASES)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(2 * nph)] for _ in range(args.steps)]
    for row in evs:  # materialise the CUDA events
        for e in row:
            e.record()
    torch.cuda.synchronize(dev)
    ev_arrays = [(ctypes.c_void_p * (2 * nph))(*[e.cuda_event for e in row]) for row in evs]

    def step(a, bb, i, timed):
        d = st._desc(a, bb, diag[i] if timed else diag[0])
        if timed:
            d.events = ctypes.cast(ev_arrays[i], ctypes.c_void_p)
        L.call("vp_step2d", ctypes.byref(d), ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))

    a = f
    for i in range(args.warmup):
        step(a, b, 0, False)
        a, b = b, a
    torch.cuda.synchronize(dev)
    dist.barrier()
    torch.cuda.synchronize(dev)
    launches0 = L.load().vp_launch_count()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        t_start.record()
        for i in range(args.steps):
            step(a, b, i, True)
            a, b = b, a
        t_end.record()
        torch.cuda.synchronize(dev)
    launches = L.load().vp_launch_count() - launches0
    dist.barrier()
    torch.cuda.synchronize(dev)
    ms = t_start.elapsed_time(t_end)
    ms_max = dist.max_over_ranks(ms)
    value = world * cells * args.steps / (ms_max / 1e3)

    # phase durations (ms), averaged over the timed steps
    ph = {p: 0.0 for p in PHASES}
    for row in evs:
        for j, p in enumerate(PHASES):
            ph[p] += row[2 * j].elapsed_time(row[2 * j + 1]) / args.steps
    sweep_bytes = 2.0 * esz * cells  # read f once + write f once per sweep
    phase_gbs = {p: (sweep_bytes / (ph[p] * 1e-3) / 1e9 if ph[p] > 0 and p not in ("field", "diag") else None)
                 for p in PHASES}
    # dominant kernel: the x drift (two launches per step) or the largest phase
    groups = {"drift_x": ph["drift_x1"] + ph["drift_x2"], "drift_y_rho": ph["drift_y1_rho"],
              "kick_vx_vy": ph["kick_vx_vy"], "drift_y": ph["drift_y2"]}
    dom = max(groups, key=groups.get)
    dom_launch_ms = groups[dom] / (2 if dom == "drift_x" else 1)
    peak, peak_kind = measured_peak()
    achieved = sweep_bytes / (dom_launch_ms * 1e-3) / 1e9
    traffic = ncu_traffic(f"{dom}_{n}x{n}x{n}x{n}_{args.dtype}")

    hist = diag[: args.steps].cpu()
    we = hist[:, 0]
    finite = bool(torch.isfinite(hist[:, :2]).all())  # field energy and mass (level-1 diagnostics)

    # end to end through the public API with pinned host buffers: every step
    # copies its input f host->device, runs the drop-in step function and
    # copies the resulting f and diagnostics back
    e2e = None
    if args.e2e_steps > 0:
        g = v2.Grid.create(n, n, n, n, LX, LX, VMAX, VMAX, device=dev,
                           dtype=torch.float64 if dtype == torch.float64 else torch.float32)
        h_in = a.cpu().pin_memory()
        h_out = torch.empty_like(h_in).pin_memory()
        h_rho = torch.empty((n, n), dtype=torch.float64 if dtype == torch.float64 else torch.float32).pin_memory()
        d_in = torch.empty_like(a)
        f0 = torch.zeros((n, n), device=dev)

        def e2e_step():
            d_in.copy_(h_in, non_blocking=True)
            fo, rho, phi = v2.vlasov_step_gather_free(
                d_in, f0, DT, g.x, g.y, g.vx, g.vy, g.kx, g.ky, g.inv_ksq, g.x_indices, g.y_indices, g.vx_indices,
                g.vy_indices, g.stencil_offsets, g.dx, g.dy, g.dvx, g.dvy, g.Nx, g.Ny, True, 1)
            h_out.copy_(fo, non_blocking=True)
            h_rho.copy_(rho, non_blocking=True)

        e2e_step()
        torch.cuda.synchronize(dev)
        dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.e2e_steps):
            e2e_step()
        e1.record()
        torch.cuda.synchronize(dev)
        ems = dist.max_over_ranks(e0.elapsed_time(e1))
        e2e = {"value": world * cells * args.e2e_steps / (ems / 1e3), "unit": "cell-updates/s",
               "h2d_bytes_per_step": h_in.numel() * h_in.element_size(),
               "d2h_bytes_per_step": h_out.numel() * h_out.element_size() + h_rho.numel() * h_rho.element_size(),
               "steps": args.e2e_steps, "path": "vlasov2d2v.vlasov_step_gather_free with pinned host f in/out"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import core as O

        c_cells, c_steps, c_sec, m = cpu_sample(n, args.dtype, args.cpu_budget)
        cpu = {"value": c_cells * c_steps / c_sec, "unit": "cell-updates/s", "cores": O.num_threads(),
               "kind": "port",
               "sample": f"oracle Strang step on a {n}x{n}x{m}x{m} sample, {c_steps} step(s), {c_sec:.1f} s"}

    if rank == 0:
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"float32": "f32", "bfloat16": "bf16", "float64": "f64"}[args.dtype], "data": "synthetic",
            "config": {"workload": workload_name(n, args.dtype), "grid": [n, n, n, n], "global_batch": world,
                       "parallelism": f"{world} independent replicas" if world > 1 else "single run",
                       "l2_flush": "not needed: f is 1 GiB per buffer, 8x the L2"
                       if n >= 128 else "inputs smaller than L2"},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                         "algorithmic_bytes_per_launch": sweep_bytes},
            "phases_ms": ph, "phases_gbs": phase_gbs,
            "step_gbs_5pass": 5 * sweep_bytes / (ms_max / args.steps * 1e-3) / 1e9,
            "gpu_launches": int(launches),
            "e2e": e2e,
            "cpu_baseline": cpu,
            "diagnostics": {"field_energy_first": float(we[0]), "field_energy_last": float(we[-1]),
                            "mass_drift_rel": float((hist[-1, 1] - hist[0, 1]) / hist[0, 1]),
                            "finite": finite},
        }
        clk_s = clk.summary()
        if clk_s:
            line["clocks"] = clk_s
        print(json.dumps(line), flush=True)
    dist.finalize()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
