"""Benchmark of the Vlasov-Poisson Strang step on B200.

Default workload (the headline line): the bandwidth-roofline configuration,
2D2V linear Landau damping on a 128^4 grid (268,435,456 cells), FP32 storage
of f, amplitude 0.05, k = 0.5 (Lx = Ly = 4 pi), v in [-6, 6], dt = 0.1. A
"step" is one full Strang step (x, y + rho, FP64 Poisson, vx + vy kick, y, x,
field-energy and mass diagnostics; in FP32 each pair of position drifts runs
as one fused pass, so the step reads and writes f three times, reported as
passes_over_f). Metric: cell-updates/s = cells * steps / seconds. The input
is synthetic (the initial condition is generated on the device); f is 1 GiB
per buffer, 8x the 126 MB L2, so no flush is needed. --sweeps-only runs one
sweep per axis for comparison.

Other workloads (--workload): c1 (Landau 32^4 FP64), c2 (two-stream 64^4
FP32), oned (1D1V Landau 4096 x 4096 FP32, the reference's 1D benchmark
grid). These are small enough to be launch-bound and run as CUDA graphs.
c4: 64 seeded independent runs of uneven size advanced by the batched step
(one launch per substep for all runs), graph-replayed; 272M cells in all.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload c3|c1|c2|c4|oned] [--dtype float32|bfloat16|float64]

--impl reference times the CPU restatement of the reference's algorithm (the
oracle: C + OpenMP over all host threads) on a bounded sample of the same
workload: the reference itself is Python that is not present on the GPU host.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAK_FALLBACK_GBS = 6650.0
PHASES = ("drift_x1", "drift_y1_rho", "field", "kick_vx_vy", "drift_y2", "drift_x2", "diag")

WORKLOADS = {
    # name: (kind, grid, L, vmax, dt, ic, ic parameters, default dtype, description)
    "c3": ("2d", (128, 128, 128, 128), 4 * math.pi, 6.0, 0.1, "landau", (0.05, 0.5), "float32",
           "2D2V Landau 128^4, eps=0.05, k=0.5, v in [-6,6], dt=0.1"),
    "c1": ("2d", (32, 32, 32, 32), 4 * math.pi, 6.0, 0.1, "landau", (0.01, 0.5), "float64",
           "2D2V Landau 32^4, eps=0.01, k=0.5, v in [-6,6], dt=0.1"),
    "c2": ("2d", (64, 64, 64, 64), 10 * math.pi, 8.0, 0.05, "two_stream", (0.001, 0.2, 2.4), "float32",
           "2D2V two-stream 64^4, eps=0.001, k=0.2, v0=2.4, v in [-8,8], dt=0.05"),
    "oned": ("1d", (4096, 4096), 4 * math.pi, 5.0, 0.05, "landau", (0.001, 0.5), "float32",
             "1D1V Landau 4096x4096, eps=0.001, k=0.5, v in [-5,5], dt=0.05"),
    "c5": ("learned", (32, 32, 32, 32), 4 * math.pi, 6.0, 0.1, None, None, "float32",
           "learned kick correction on a 32^4 grid (L = 4 pi, v in [-6,6], dt = 0.1): trained on seeded "
           "coarse / 2x-refined pairs of Landau and two-stream runs, evaluated on held-out seeds against plain 32^4 "
           "and plain 2x-refined runs, errors against a 4x-refined run"),
    "c4": ("batch", None, None, None, 0.05, None, None, "float32",
           "64 independent 2D2V runs of uneven size (seed 20261203: Nx=Ny in {16,24,32,48,64}, Nvx=Nvy in "
           "{32,48,64}, eps~U[0.001,0.05], k~U[0.3,1], v0~U[0,3], Landau or two-stream), dt=0.05"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="c3")
    ap.add_argument("--dtype", choices=["float32", "bfloat16", "float64"], default=None)
    ap.add_argument("--size", type=int, default=None, help="override N of a 2D2V workload (N^4 grid)")
    ap.add_argument("--grid", default=None,
                    help="override the grid of a 2D2V workload: NX,NY,NVX,NVY (small cases for profiling)")
    ap.add_argument("--diagnostics", type=int, default=1, help="0 none, 1 field energy + mass, 2 + L2/kinetic")
    ap.add_argument("--e2e-steps", type=int, default=100)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-history-check", action="store_true",
                    help="skip the 20-step comparison with the reference's FP64 run (128^4 Landau only)")
    ap.add_argument("--sweeps-only", action="store_true",
                    help="2D2V and the batch: one sweep per axis even where the fused (x, y) plane passes apply")
    ap.add_argument("--split", action="store_true",
                    help="2D2V: store the perturbation of the initial condition's velocity equilibrium "
                         "(g = f - A(vx) B(vy)) with float64-evaluated drift tables")
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU work for cpu_baseline")
    ap.add_argument("--train-ics", type=int, default=125, help="learned workload: training initial conditions")
    ap.add_argument("--train-iters", type=int, default=1500, help="learned workload: Adam steps")
    ap.add_argument("--eval-ics", type=int, default=4, help="learned workload: held-out initial conditions")
    ap.add_argument("--tiles", choices=["default", "auto", "tune"], default="auto",
                    help="batched workload: default tile shapes, the autotuner's cache, or tune now")
    a = ap.parse_args()
    a.grid_override = a.grid
    wl = WORKLOADS[a.workload]
    a.kind, a.grid, a.L, a.vmax, a.dt, a.ic, a.icp, dflt, a.desc = wl
    a.dtype = a.dtype or dflt
    if a.kind in ("batch", "learned") and a.size:
        raise SystemExit("--size does not apply to the batched workload")
    if a.split and a.kind != "2d":
        raise SystemExit("--split applies to 2D2V workloads")
    if a.size:
        if a.kind != "2d":
            raise SystemExit("--size applies to 2D2V workloads")
        a.grid = (a.size,) * 4
        a.desc = a.desc.replace("128^4", f"{a.size}^4")
    if a.grid_override:
        if a.kind != "2d":
            raise SystemExit("--grid applies to 2D2V workloads")
        a.grid = tuple(int(v) for v in a.grid_override.split(","))
        if len(a.grid) != 4 or a.grid[2] != a.grid[3] or a.grid[0] < 1 or a.grid[1] < 1:
            raise SystemExit("--grid takes NX,NY,NV,NV (equal velocity sizes)")
        a.desc = a.desc.replace("128^4", "x".join(map(str, a.grid)))
    return a


def short_dtype(name):
    return {"float32": "f32", "bfloat16": "bf16", "float64": "f64"}[name]


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return PEAK_FALLBACK_GBS, "fallback"


def ncu_traffic(tag):
    """DRAM bytes per launch from a committed ncu summary (a line
    'dram_bytes_per_launch: <n>' in profiles/traffic_<tag>.txt), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", f"traffic_{tag}.txt")) as fh:
            for line in fh:
                if line.startswith("dram_bytes_per_launch:"):
                    return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 50 ms, stamped with the
    host clock so that the summary covers the timed window."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.samples = []
        self.window = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append((time.monotonic(), line.strip()))

    def ready(self, timeout=5.0):
        """Wait (bounded) for nvidia-smi's first sample, so that the timed
        region that follows is covered from its start."""
        t = time.monotonic()
        while self.proc is not None and not self.samples and time.monotonic() - t < timeout:
            time.sleep(0.02)

    def mark(self, t0, t1):
        self.window = (t0, t1)

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

        def parse(lines):
            sm, mx, reasons = [], None, set()
            for _, ln in lines:
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
            return sm, mx, reasons

        window = "timed"
        lines = self.samples
        if self.window:
            t0, t1 = self.window
            inwin = [s for s in self.samples if t0 - 0.05 <= s[0] <= t1 + 0.05]
            if len(inwin) >= 3:
                lines = inwin
            else:
                window = "run (the timed region is shorter than three samples)"
        sm, mx, reasons = parse(lines)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "window": window}


# ---------------------------------------------------------------------------
# CPU side (the oracle): cpu_baseline and --impl reference
# ---------------------------------------------------------------------------
def _oracle_setup(a, grid):
    import numpy as np

    from oracle import core as O

    npdt = np.float64 if a.dtype == "float64" else np.float32
    if a.kind == "1d":
        g = O.make_grid1d(grid[0], grid[1], a.L, a.vmax, dtype=npdt)
        return O.Stepper1D(g, a.dt, window=1), O.landau_1d(g, a.icp[0], a.icp[1])
    g = O.make_grid2d(*grid, a.L, a.L, a.vmax, a.vmax, dtype=npdt)
    f = O.landau_2d(g, *a.icp) if a.ic == "landau" else O.two_stream_2d(g, *a.icp)
    return O.Stepper2D(g, a.dt, window=1), f


def cpu_sample_grid(a, budget_s):
    """The largest sample of the workload (velocity dims reduced for 2D2V)
    whose one step fits in budget_s on the host, from a small calibration."""
    if a.kind == "1d":
        return a.grid
    n = a.grid[0]
    st, f = _oracle_setup(a, (n, n, 16, 16))
    st.step(f)
    t0 = time.perf_counter()
    st.step(f)
    rate = (n * n * 256) / (time.perf_counter() - t0)
    for m in (a.grid[2], 96, 64, 48, 32, 24, 16):
        if m <= a.grid[2] and (n * n * m * m) / rate <= budget_s:
            return (n, n, m, m)
    return (n, n, 16, 16)


def time_oracle(a, grid, steps, warmup):
    st, f = _oracle_setup(a, grid)
    for _ in range(warmup):
        f = st.step(f).f
    t0 = time.perf_counter()
    for _ in range(steps):
        f = st.step(f).f
    return time.perf_counter() - t0


def run_reference(a):
    if int(os.environ.get("RANK", 0)) != 0:
        return 0
    from oracle import core as O

    # a bounded sample of the workload per step, so that --warmup + --steps
    # stays within about three minutes
    per_step = max(0.5, 150.0 / max(1, a.steps + a.warmup))
    grid = cpu_sample_grid(a, per_step)
    cells = math.prod(grid)
    sec = time_oracle(a, grid, a.steps, a.warmup)
    value = cells * a.steps / sec
    sample = (f"oracle Strang step (C + OpenMP restatement of the reference's vlasov_step_gather_free) on a "
              f"{'x'.join(map(str, grid))} sample of the workload, {a.steps} steps after {a.warmup} warm-up")
    line = {
        "impl": "reference", "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
        "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * sec / a.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": short_dtype(a.dtype),
        "data": "synthetic", "config": {"workload": a.desc + f", {a.dtype} storage", "grid": list(a.grid),
                                        "cpu_sample_grid": list(grid)},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": O.num_threads(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU side
# ---------------------------------------------------------------------------
def _equilibrium(a, torch):
    """The velocity equilibrium A(vx), B(vy) of a 2D2V workload's initial
    condition (float64, on the host): unit Maxwellians for Landau, the two
    beams times a Maxwellian for two-stream."""
    nv = a.grid[2]
    v = torch.linspace(-a.vmax, a.vmax, nv, dtype=torch.float64)
    M = lambda u: torch.exp(-0.5 * u * u) / math.sqrt(2 * math.pi)  # noqa: E731
    if a.ic == "landau":
        return M(v), M(v)
    return 0.5 * (M(v - a.icp[2]) + M(v + a.icp[2])), M(v)


def _initial_f(a, dev, dtype, rank, torch):
    """Initial condition built on the device (not timed)."""
    gdt = torch.float64
    eps = a.icp[0] * (1.0 + 0.01 * rank)  # each rank runs its own replica
    if a.kind == "1d":
        nx, nv = a.grid
        x = torch.linspace(0, a.L, nx + 1, dtype=gdt, device=dev)[:-1]
        v = torch.linspace(-a.vmax, a.vmax, nv, dtype=gdt, device=dev)
        ops = importlib.import_module("jax-pytorch-vlasov_b200.ops")
        return ops.init_product(1.0 + eps * torch.cos(a.icp[1] * x), torch.exp(-0.5 * v * v) / math.sqrt(2 * math.pi),
                                dtype)
    nx, ny, nv, _ = a.grid
    x = torch.linspace(0, a.L, nx + 1, dtype=gdt, device=dev)[:-1]
    y = torch.linspace(0, a.L, ny + 1, dtype=gdt, device=dev)[:-1]
    v = torch.linspace(-a.vmax, a.vmax, nv, dtype=gdt, device=dev)
    k = a.icp[1]
    sp = 1.0 + eps * (torch.cos(k * x)[:, None] + torch.cos(k * y)[None, :])
    M = lambda u: torch.exp(-0.5 * u * u) / math.sqrt(2 * math.pi)  # noqa: E731
    if a.ic == "landau":
        fv = M(v)[:, None] * M(v)[None, :]
    else:
        fv = (0.5 * (M(v - a.icp[2]) + M(v + a.icp[2])))[:, None] * M(v)[None, :]
    # one FP64 product per element, rounded once (the library's IC kernel)
    return importlib.import_module("jax-pytorch-vlasov_b200.ops").init_product(sp, fv, dtype)


def reference_history(a, vp, dev, dtype, torch):
    """Errors of the first 20 steps against the reference solver's own FP64
    run of the 128^4 Landau configuration (tests/golden/history_c3.npz, made
    by tests/golden/make_golden.py): field energy and mass after every step,
    relative to their largest magnitude, and the mid-step density fluctuation
    at steps 10 and 20, for the storage type (and split) this bench timed.
    None for other workloads."""
    path = os.path.join(ROOT, "tests", "golden", "history_c3.npz")
    if (a.kind != "2d" or tuple(a.grid) != (128, 128, 128, 128) or a.ic != "landau" or
            tuple(a.icp[:2]) != (0.05, 0.5) or a.dt != 0.1 or a.vmax != 6.0 or abs(a.L - 4 * math.pi) > 1e-12 or
            not os.path.exists(path)):
        return None
    H = np.load(path)
    n = a.grid[0]
    st = vp.Stepper2D(n, n, n, n, a.L, a.L, a.vmax, a.vmax, a.dt, dtype=dtype, device=dev, window=1,
                      fuse_drifts=not a.sweeps_only, equilibrium="maxwellian" if a.split else None,
                      precise_tables=a.split)
    # the golden run's initial condition: the FP64 product of the spatial
    # profile and the 2D Maxwellian on the reference's grids, rounded once
    g = vp.vlasov2d2v.Grid.create(n, n, n, n, a.L, a.L, a.vmax, a.vmax, device="cpu", dtype=torch.float64)
    sp = 1.0 + 0.05 * (torch.cos(0.5 * g.x)[:, None] + torch.cos(0.5 * g.y)[None, :])
    fv = torch.exp(-0.5 * (g.vx[:, None] ** 2 + g.vy[None, :] ** 2)) / (2.0 * math.pi)
    if a.split:
        f64 = vp.ops.init_product(sp.to(dev), fv.to(dev), torch.float64)
        x = st.split(f64)
        del f64
    else:
        x = vp.ops.init_product(sp.to(dev), fv.to(dev), dtype)
    h = torch.zeros((20, vp._lib.DIAG_COUNT), dtype=torch.float64, device=dev)
    x = st.run(x, 10, history=h[:10], graph=True)
    d10 = st.drho.clone()
    x = st.run(x, 10, history=h[10:], graph=True)
    torch.cuda.synchronize(dev)
    st.check()
    h, d10, d20 = h.cpu().numpy(), d10.cpu().numpy(), st.drho.cpu().numpy()
    rel = lambda got, ref: float(np.abs(got - ref).max() / np.abs(ref).max())  # noqa: E731
    out = {"steps": 20, "W_E": rel(h[:, 0], H["W_E"]), "mass": rel(h[:, 1], H["mass"]),
           "drho_10": rel(d10, H["drho_10"]), "drho_20": rel(d20, H["drho_20"]),
           "reference": "tests/golden/history_c3.npz: the reference solver in FP64 on the CPU"}
    del st, x
    torch.cuda.empty_cache()
    return out


def run_ours(a):
    import torch

    vp = importlib.import_module("jax-pytorch-vlasov_b200")
    dist = importlib.import_module("jax-pytorch-vlasov_b200.dist")
    L = vp._lib

    rank, local, world = dist.init()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dtype = {"float32": torch.float32, "bfloat16": torch.bfloat16, "float64": torch.float64}[a.dtype]
    esz = {torch.float32: 4, torch.bfloat16: 2, torch.float64: 8}[dtype]
    cells = math.prod(a.grid)
    big = cells * esz > 256 * 2 ** 20
    if a.kind == "1d":
        st = vp.Stepper1D(*a.grid, a.L, a.vmax, a.dt, dtype=dtype, device=dev, window=1, diagnostics=a.diagnostics)
        n_sweeps = 3
    else:
        st = vp.Stepper2D(*a.grid, a.L, a.L, a.vmax, a.vmax, a.dt, dtype=dtype, device=dev, window=1,
                          diagnostics=a.diagnostics, fuse_drifts=not a.sweeps_only,
                          equilibrium=_equilibrium(a, torch) if a.split else None, precise_tables=a.split)
    if a.split:
        # the state is g = f - feq, formed from the FP64 initial condition
        f = st.split(_initial_f(a, dev, torch.float64, rank, torch))
        torch.cuda.empty_cache()
    else:
        f = _initial_f(a, dev, dtype, rank, torch)
    b = st.empty_f()
    planar = False
    if a.kind != "1d":
        n_sweeps, planar = st.passes(f, b)
    K = max(a.steps, 1)
    hist = torch.zeros((K, L.DIAG_COUNT), dtype=torch.float64, device=dev)
    use_events = a.kind == "2d" and big  # per-phase events on the big grid; graphs for the small ones

    nph = len(PHASES)
    if use_events:
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(2 * nph)] for _ in range(K)]
        for row in evs:  # materialise the CUDA events before handing them to the library
            for e in row:
                e.record()
        torch.cuda.synchronize(dev)
        ev_arrays = [(ctypes.c_void_p * (2 * nph))(*[e.cuda_event for e in row]) for row in evs]

    def step(x, y, i, timed):
        d = st._desc(x, y, hist[i] if timed else hist[0])
        if timed and use_events:
            d.events = ctypes.cast(ev_arrays[i], ctypes.c_void_p)
        name = "vp_step1d" if a.kind == "1d" else "vp_step2d"
        L.call(name, ctypes.byref(d), ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))

    with ClockSampler(local) as clk:
        x, y = f, b
        # kernels one step launches (graph replays bypass the library's host
        # launch counter, so replayed steps are counted as this many each)
        c0 = L.load().vp_launch_count()
        step(x, y, 0, False)
        per_step_launches = L.load().vp_launch_count() - c0
        step(y, x, 0, False)
        if use_events or a.kind == "1d":
            for i in range(a.warmup):
                step(x, y, 0, False)
                x, y = y, x
        else:
            # an even number of steps returns the state to x, the buffer the
            # graph captured here expects at the start of the timed run
            x = st.run(x, max(20, 2 * (a.warmup // 2)), graph=True, graph_chunk=10)
        torch.cuda.synchronize(dev)
        clk.ready()
        dist.barrier()
        torch.cuda.synchronize(dev)
        launches0 = L.load().vp_launch_count()
        t_start = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        h0 = time.monotonic()
        t_start.record()
        if use_events or a.kind == "1d":
            for i in range(K):
                step(x, y, i, True)
                x, y = y, x
        else:
            x = st.run(x, K, history=hist, graph=True, graph_chunk=10)
        t_end.record()
        torch.cuda.synchronize(dev)
        clk.mark(h0, time.monotonic())
        launches = L.load().vp_launch_count() - launches0
        if not (use_events or a.kind == "1d"):
            launches = per_step_launches * K
    dist.barrier()
    torch.cuda.synchronize(dev)
    ms = t_start.elapsed_time(t_end)
    ms_max = dist.max_over_ranks(ms)
    value = world * cells * K / (ms_max / 1e3)
    sweep_bytes = 2.0 * esz * cells  # read f once + write f once per sweep
    peak, peak_kind = measured_peak()
    ms_step = ms_max / K

    ph = None
    phase_gbs = None
    if use_events:
        ph = {p: 0.0 for p in PHASES}
        for row in evs:
            for j, p in enumerate(PHASES):
                ph[p] += row[2 * j].elapsed_time(row[2 * j + 1]) / K
        # empty phases (the y phases of a fused step) have no bandwidth
        busy = 0.05 * max(ph.values())
        phase_gbs = {p: (sweep_bytes / (ph[p] * 1e-3) / 1e9 if ph[p] > busy and p not in ("field", "diag") else None)
                     for p in PHASES}
        if planar:
            # x then y (with the density partials) and y then x each make one
            # pass over f; their phases carry the x names. The y1 phase is the
            # separate kernel that sums the density partials (no pass over f).
            phase_gbs["drift_y1_rho"] = phase_gbs["drift_y2"] = None
            groups = {"plane_xy_rho": ph["drift_x1"], "kick_vx_vy": ph["kick_vx_vy"], "plane_yx": ph["drift_x2"]}
            dom = max(groups, key=groups.get)
            dom_ms = groups[dom]
        else:
            groups = {"drift_x": ph["drift_x1"] + ph["drift_x2"], "drift_y_rho": ph["drift_y1_rho"],
                      "kick_vx_vy": ph["kick_vx_vy"], "drift_y": ph["drift_y2"]}
            dom = max(groups, key=groups.get)
            dom_ms = groups[dom] / (2 if dom == "drift_x" else 1)
        achieved = sweep_bytes / (dom_ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": ncu_traffic(f"{dom}_{'x'.join(map(str, a.grid))}_{a.dtype}"),
                "algorithmic_bytes_per_launch": sweep_bytes}
        if planar:
            roof["density_partials_sum_ms"] = ph["drift_y1_rho"]
    else:
        # graph-replayed small grids: whole-step bandwidth (the f-sized sweeps
        # dominate; the grid fits the L2, so this may exceed the HBM figure)
        achieved = n_sweeps * sweep_bytes / (ms_step * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": "whole step (graph replay)", "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                "algorithmic_bytes_per_launch": n_sweeps * sweep_bytes,
                "note": "f fits the 126 MB L2" if cells * esz * 3 < 126e6 else ""}

    h = hist[:K].cpu()
    finite = bool(torch.isfinite(h[:, :2]).all())

    # end to end through the public API with pinned host buffers: every step
    # copies its input f host->device, runs the drop-in step function, and
    # copies the resulting f and mid-step density back
    e2e = None
    if a.e2e_steps > 0:
        e2e = run_e2e(a, x, dev, dtype, world, dist, torch, vp, stepper=st if a.split else None)
    ref_hist = reference_history(a, vp, dev, dtype, torch) if rank == 0 and not a.no_history_check else None

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        from oracle import core as O

        grid = cpu_sample_grid(a, a.cpu_budget / 2)
        # one warm-up step sets how many timed steps fill half the budget
        t_one = time_oracle(a, grid, 1, 0)
        c_steps = max(2, min(50, int(a.cpu_budget / 2 / max(t_one, 1e-3))))
        sec = time_oracle(a, grid, c_steps, 1)
        cpu = {"value": math.prod(grid) * c_steps / sec, "unit": "cell-updates/s", "cores": O.num_threads(),
               "kind": "port",
               "sample": f"oracle Strang step on a {'x'.join(map(str, grid))} sample, {c_steps} steps, {sec:.1f} s"}

    if rank == 0:
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": K, "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": short_dtype(a.dtype), "data": "synthetic",
            "config": {"workload": a.desc + f", {a.dtype} storage" + (
                           " of the perturbation g = f - A(vx) B(vy) (equilibrium split), float64-evaluated "
                           "drift tables" if a.split else ""), "grid": list(a.grid), "global_batch": world,
                       "parallelism": f"{world} independent replicas" if world > 1 else "single run",
                       "l2_flush": "not needed: f exceeds the L2 several times" if big
                       else "none: the whole state is L2-resident (launch/latency-bound size)",
                       "diagnostics_level": a.diagnostics},
            "roofline": roof,
            "step_gbs": n_sweeps * sweep_bytes / (ms_step * 1e-3) / 1e9,
            "gpu_launches": int(launches),
            "e2e": e2e,
            "cpu_baseline": cpu,
            "diagnostics": {"field_energy_first": float(h[0, 0]), "field_energy_last": float(h[-1, 0]),
                            "mass_drift_rel": float((h[-1, 1] - h[0, 1]) / h[0, 1]), "finite": finite},
        }
        if ref_hist is not None:
            line["diagnostics"]["vs_reference_history"] = ref_hist
        if ph is not None:
            line["phases_ms"] = ph
            line["phases_gbs"] = phase_gbs
        if a.kind != "1d":
            line["passes_over_f"] = n_sweeps
            line["fused_plane_drifts"] = planar
        clk_s = clk.summary()
        if clk_s:
            line["clocks"] = clk_s
        print(json.dumps(line), flush=True)
    dist.finalize()
    return 0


def run_e2e(a, f_dev, dev, dtype, world, dist, torch, vp, stepper=None):
    cells = math.prod(a.grid)
    gdt = torch.float64 if dtype == torch.float64 else torch.float32
    h_in = f_dev.cpu().pin_memory()
    if stepper is not None:
        # the split state has no reference signature: the library's own
        # public step, with its mid-step density fluctuation as the result read back
        h_rho0 = torch.empty(a.grid[:2], dtype=torch.float64)

        def call(d_in):
            out = stepper.step(d_in)
            return out, stepper.drho.clone(), None  # the next step overwrites drho
        path = "Stepper2D.step (equilibrium split) with pinned host g in/out"
    elif a.kind == "1d":
        m = importlib.import_module("jax-pytorch-vlasov_b200.vlasov1d1v")
        g = m.Grid.create(*a.grid, a.L, a.vmax, device=dev, dtype=gdt)
        h_rho0 = torch.empty(a.grid[0], dtype=gdt)

        def call(d_in):
            return m.vlasov_step_gather_free(d_in, a.dt, g.v, g.inv_kx, g.inv_kx_sq, g.x_indices, g.v_indices,
                                             g.x_batch_offsets, g.v_batch_offsets, g.stencil_offsets, g.dx, g.dv,
                                             g.V_max, True, 1)
        path = "vlasov1d1v.vlasov_step_gather_free with pinned host f in/out"
    else:
        m = importlib.import_module("jax-pytorch-vlasov_b200.vlasov2d2v")
        g = m.Grid.create(*a.grid, a.L, a.L, a.vmax, a.vmax, device=dev, dtype=gdt)
        h_rho0 = torch.empty(a.grid[:2], dtype=gdt)
        f0 = torch.zeros(a.grid[2:], dtype=gdt, device=dev)

        def call(d_in):
            return m.vlasov_step_gather_free(d_in, f0, a.dt, g.x, g.y, g.vx, g.vy, g.kx, g.ky, g.inv_ksq,
                                             g.x_indices, g.y_indices, g.vx_indices, g.vy_indices,
                                             g.stencil_offsets, g.dx, g.dy, g.dvx, g.dvy, g.Nx, g.Ny, True, 1)
        path = "vlasov2d2v.vlasov_step_gather_free with pinned host f in/out"

    # Consecutive steps overlap: step i+1's input copies in on one stream
    # while step i computes and step i-1's result copies out on another
    # (PCIe carries both directions at once). Inputs rotate through three
    # device buffers, results through two pinned host buffers.
    comp = torch.cuda.current_stream(dev)
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    d_in = [torch.empty_like(f_dev) for _ in range(3)]
    h_out = [torch.empty_like(h_in).pin_memory() for _ in range(2)]
    h_rho = [torch.empty_like(h_rho0).pin_memory() for _ in range(2)]
    read_done = [None] * 3

    def e2e_step(i):
        j = i % 3
        if read_done[j] is not None:
            s_in.wait_event(read_done[j])
        with torch.cuda.stream(s_in):
            d_in[j].copy_(h_in, non_blocking=True)
        loaded = torch.cuda.Event()
        loaded.record(s_in)
        comp.wait_event(loaded)
        fo, rho, _ = call(d_in[j])
        done = torch.cuda.Event()
        done.record(comp)
        read_done[j] = done
        s_out.wait_event(done)
        with torch.cuda.stream(s_out):
            h_out[i % 2].copy_(fo, non_blocking=True)
            h_rho[i % 2].copy_(rho, non_blocking=True)
        fo.record_stream(s_out)
        rho.record_stream(s_out)

    for i in range(3):
        e2e_step(i)
    torch.cuda.synchronize(dev)
    dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s_in)
    for i in range(a.e2e_steps):
        e2e_step(i)
    e1.record(s_out)
    torch.cuda.synchronize(dev)
    ems = dist.max_over_ranks(e0.elapsed_time(e1))
    return {"value": world * cells * a.e2e_steps / (ems / 1e3), "unit": "cell-updates/s",
            "h2d_bytes_per_step": h_in.numel() * h_in.element_size(),
            "d2h_bytes_per_step": h_out[0].numel() * h_out[0].element_size() + h_rho[0].numel() * h_rho[0].element_size(),
            "steps": a.e2e_steps, "path": path + ", steps pipelined over copy-in / compute / copy-out streams"}


# ---------------------------------------------------------------------------
# the batched workload (64 uneven runs, one launch per substep for all)
# ---------------------------------------------------------------------------
def _batch_oracle_sample(budget_s):
    """The oracle on runs of the batch in their drawn order, one step each,
    until budget_s of host time is spent: (cells stepped, seconds, runs used)."""
    from oracle import core as O

    wl = importlib.import_module("jax-pytorch-vlasov_b200.workloads")
    runs = wl.batch_runs()
    done = 0
    spent = 0.0
    used = 0
    for p in runs:
        g = O.make_grid2d(p["Nx"], p["Ny"], p["Nvx"], p["Nvy"], p["Lx"], p["Ly"], p["Vx_max"], p["Vy_max"],
                          dtype=np.float32)
        if p["kind"] == "landau":
            f = O.landau_2d(g, p["eps"], p["k"])
        else:
            f = O.two_stream_2d(g, p["eps"], p["k"], p["v0"])
        st = O.Stepper2D(g, p["dt"], window=1)
        st.step(f)  # warm-up
        t0 = time.perf_counter()
        st.step(f)
        spent += time.perf_counter() - t0
        done += p["Nx"] * p["Ny"] * p["Nvx"] * p["Nvy"]
        used += 1
        if spent >= budget_s:
            break
    return done, spent, used


def run_batch_reference(a):
    if int(os.environ.get("RANK", 0)) != 0:
        return 0
    from oracle import core as O

    per_step = max(0.5, 150.0 / max(1, a.steps + a.warmup))
    cells = 0
    sec = 0.0
    used = 0
    for i in range(a.warmup + a.steps):
        c, t, u = _batch_oracle_sample(per_step)
        if i >= a.warmup:
            cells += c
            sec += t
            used = u
    value = cells / sec
    all_runs = importlib.import_module("jax-pytorch-vlasov_b200.workloads").batch_runs()
    sample = (f"oracle Strang step (C + OpenMP restatement of the reference's vlasov_step_gather_free) over the "
              f"first {used} runs of the batch per step, {a.steps} steps after {a.warmup} warm-up")
    line = {
        "impl": "reference", "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
        "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * sec / a.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": short_dtype(a.dtype),
        "data": "synthetic", "config": {"workload": a.desc + f", {a.dtype} storage", "runs": len(all_runs),
                                        "cells": sum(p["Nx"] * p["Ny"] * p["Nvx"] * p["Nvy"] for p in all_runs),
                                        "cpu_sample_runs": used},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": O.num_threads(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_batch(a):
    import torch

    vp = importlib.import_module("jax-pytorch-vlasov_b200")
    dist = importlib.import_module("jax-pytorch-vlasov_b200.dist")
    wl = importlib.import_module("jax-pytorch-vlasov_b200.workloads")
    L = vp._lib

    rank, local, world = dist.init()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dtype = {"float32": torch.float32, "bfloat16": torch.bfloat16, "float64": torch.float64}[a.dtype]
    esz = {torch.float32: 4, torch.bfloat16: 2, torch.float64: 8}[dtype]
    runs = wl.batch_runs()
    diag = 1 if a.diagnostics else 0
    st = vp.BatchStepper2D(runs, dtype=dtype, device=dev, window=1, diagnostics=diag, graph_slots=10,
                           tiles=None if a.tiles == "default" else "auto", fuse_drifts=not a.sweeps_only)
    if a.tiles == "tune":  # on a scratch state, before the initial condition is set
        at = importlib.import_module("jax-pytorch-vlasov_b200.autotune")
        for r, p in enumerate(runs):
            st.set_state(r, wl.initial_2d(p["kind"], p["Nx"], p["Ny"], p["Nvx"], p["Nvy"], p["Lx"], p["Ly"],
                                          p["Vx_max"], p["Vy_max"], p["eps"], p["k"], p["v0"], dtype=dtype,
                                          device=dev))
        at.tune(st)  # writes the cache ($VLASOV_B200_TUNE_CACHE or the package's tune_b200.json)
    for r, p in enumerate(runs):  # each rank advances its own replica of the batch
        st.set_state(r, wl.initial_2d(p["kind"], p["Nx"], p["Ny"], p["Nvx"], p["Nvy"], p["Lx"], p["Ly"],
                                      p["Vx_max"], p["Vy_max"], p["eps"] * (1.0 + 0.01 * rank), p["k"], p["v0"],
                                      dtype=dtype, device=dev))
    cells = st.cells
    n = len(runs)
    K = max(a.steps, 1)
    hist = torch.zeros((K, n, L.DIAG_COUNT), dtype=torch.float64, device=dev)
    nph = len(PHASES)
    with ClockSampler(local) as clk:
        c0 = L.load().vp_launch_count()
        st.step(0)
        per_step_launches = L.load().vp_launch_count() - c0
        st.run(max(a.warmup, 3) + 10, graph=True)  # captures the graph, then replays it
        torch.cuda.synchronize(dev)
        clk.ready()
        dist.barrier()
        torch.cuda.synchronize(dev)
        t_start = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        h0 = time.monotonic()
        t_start.record()
        st.run(K, history=hist, graph=True)
        t_end.record()
        torch.cuda.synchronize(dev)
        clk.mark(h0, time.monotonic())
        # per-substep times from eager steps with events (after the timed region)
        n_ev = 5
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(2 * nph)] for _ in range(n_ev)]
        for row in evs:
            for e in row:
                e.record()
        torch.cuda.synchronize(dev)
        for row in evs:
            arr = (ctypes.c_void_p * (2 * nph))(*[e.cuda_event for e in row])
            st.step(0, events=arr)
        torch.cuda.synchronize(dev)
    dist.barrier()
    ms = t_start.elapsed_time(t_end)
    ms_max = dist.max_over_ranks(ms)
    value = world * cells * K / (ms_max / 1e3)
    ms_step = ms_max / K
    sweep_bytes = 2.0 * esz * cells
    fused_cells = sum(math.prod(sh) for sh, fu in zip(st.shapes, st.fused) if fu)
    # the x phases and the kick move every run's f once; the y phases only
    # the runs on single-axis sweeps (the fused runs' y drifts ride in the x
    # phases' plane passes)
    phase_bytes = {"drift_x1": sweep_bytes, "drift_y1_rho": 2.0 * esz * (cells - fused_cells),
                   "kick_vx_vy": sweep_bytes, "drift_y2": 2.0 * esz * (cells - fused_cells), "drift_x2": sweep_bytes}
    peak, peak_kind = measured_peak()
    ph = {p: sum(row[2 * j].elapsed_time(row[2 * j + 1]) for row in evs) / n_ev for j, p in enumerate(PHASES)}
    dom = max(phase_bytes, key=lambda p: ph[p])
    achieved = phase_bytes[dom] / (ph[dom] * 1e-3) / 1e9
    dom_name = {"drift_x1": "x1 phase: x-then-y plane pass of the fused runs, x sweep of the others",
                "drift_x2": "x2 phase: y-then-x plane pass of the fused runs, x sweep of the others",
                "kick_vx_vy": "fused vx+vy kick", "drift_y1_rho": "y drift + rho partials (swept runs)",
                "drift_y2": "y drift (swept runs)"}[dom]
    roof = {"bound": "hbm", "kernel": dom_name + " (batched)", "achieved": achieved, "peak": peak,
            "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
            "traffic": ncu_traffic(f"batch_{dom}_{a.dtype}"), "algorithmic_bytes_per_launch": phase_bytes[dom]}
    phase_gbs = {p: (phase_bytes[p] / (ph[p] * 1e-3) / 1e9 if p in phase_bytes and ph[p] > 0 and phase_bytes[p] > 0
                     else None) for p in PHASES}
    h = hist.cpu()
    finite = bool(torch.isfinite(h[:, :, :2]).all())

    e2e = None
    if a.e2e_steps > 0:
        # end to end through the public API: every step copies every run's f
        # from pinned host memory, steps the batch, and copies f and the
        # diagnostics back
        # The stepper advances its runs in place in one arena, so steps
        # overlap through staging buffers: step i+1's input copies in on one
        # stream while step i computes (staging -> arena, step, arena ->
        # staging) and step i-1's result copies out on another.
        arena = st._arenas[0]
        h_in = arena.cpu().pin_memory()
        h_out = [torch.empty_like(h_in).pin_memory() for _ in range(2)]
        h_diag = [torch.empty((n, L.DIAG_COUNT), dtype=torch.float64).pin_memory() for _ in range(2)]
        stage_in = [torch.empty_like(arena) for _ in range(2)]
        stage_out = [torch.empty_like(arena) for _ in range(2)]
        diag_out = [torch.empty((n, L.DIAG_COUNT), dtype=torch.float64, device=dev) for _ in range(2)]
        comp = torch.cuda.current_stream(dev)
        s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
        consumed = [None, None]  # compute event that last read stage_in[k]
        shipped = [None, None]   # copy-out event that last read stage_out[k]

        def e2e_step(i):
            k = i % 2
            if consumed[k] is not None:
                s_in.wait_event(consumed[k])
            with torch.cuda.stream(s_in):
                stage_in[k].copy_(h_in, non_blocking=True)
            loaded = torch.cuda.Event()
            loaded.record(s_in)
            comp.wait_event(loaded)
            arena.copy_(stage_in[k], non_blocking=True)
            st.step(0)
            if shipped[k] is not None:
                comp.wait_event(shipped[k])
            stage_out[k].copy_(arena, non_blocking=True)
            diag_out[k].copy_(st.stage[0], non_blocking=True)
            done = torch.cuda.Event()
            done.record(comp)
            consumed[k] = done
            s_out.wait_event(done)
            with torch.cuda.stream(s_out):
                h_out[k].copy_(stage_out[k], non_blocking=True)
                h_diag[k].copy_(diag_out[k], non_blocking=True)
            out = torch.cuda.Event()
            out.record(s_out)
            shipped[k] = out

        for i in range(3):
            e2e_step(i)
        torch.cuda.synchronize(dev)
        dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s_in)
        for i in range(a.e2e_steps):
            e2e_step(i)
        e1.record(s_out)
        torch.cuda.synchronize(dev)
        e_ms = dist.max_over_ranks(e0.elapsed_time(e1))
        e2e = {"value": world * cells * a.e2e_steps / (e_ms / 1e3), "unit": "cell-updates/s",
               "h2d_bytes_per_step": int(arena.numel()), "d2h_bytes_per_step": int(arena.numel() + n * L.DIAG_COUNT * 8),
               "steps": a.e2e_steps,
               "path": "BatchStepper2D.step with every run's f copied from/to pinned host memory, steps pipelined "
                       "over copy-in / compute / copy-out streams through device staging buffers"}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        from oracle import core as O

        c, t, used = _batch_oracle_sample(a.cpu_budget / 2)
        cpu = {"value": c / t, "unit": "cell-updates/s", "cores": O.num_threads(), "kind": "port",
               "sample": f"oracle Strang step over the first {used} runs of the batch, one step each, {t:.1f} s"}

    if rank == 0:
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": K, "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": short_dtype(a.dtype), "data": "synthetic",
            "config": {"workload": a.desc + f", {a.dtype} storage", "runs": n, "cells": cells,
                       "global_batch": n * world,
                       "parallelism": f"{world} independent replicas of the batch" if world > 1 else "one batch",
                       "l2_flush": "not needed: the batch state (all runs) exceeds the L2 several times",
                       "diagnostics_level": diag, "graph": "10 steps per CUDA graph, replayed",
                       "tiles": {k: v for k, v in (st.tiles or {}).items() if k != "run_segments"},
                       "tiles_source": a.tiles,
                       "fused_runs": int(sum(st.fused)), "fused_cells": int(fused_cells)},
            "roofline": roof,
            "step_gbs": sum(phase_bytes.values()) / (ms_step * 1e-3) / 1e9,
            "gpu_launches": int(per_step_launches * K),
            "e2e": e2e,
            "cpu_baseline": cpu,
            "diagnostics": {"mass_drift_rel_max": float(((h[-1, :, 1] - h[0, :, 1]) / h[0, :, 1]).abs().max()),
                            "finite": finite},
            "phases_ms": ph,
            "phases_gbs": phase_gbs,
        }
        clk_s = clk.summary()
        if clk_s:
            line["clocks"] = clk_s
        print(json.dumps(line), flush=True)
    dist.finalize()
    return 0


# ---------------------------------------------------------------------------
# the learned corrector: training on coarse / refined pairs, held-out runs
# ---------------------------------------------------------------------------
def run_learned(a):
    import torch

    vp = importlib.import_module("jax-pytorch-vlasov_b200")
    C = vp.corrector
    L = vp._lib
    rank, local, world = importlib.import_module("jax-pytorch-vlasov_b200.dist").init()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    N, _, Nv, _ = a.grid
    Lb, V, dt = a.L, a.vmax, a.dt
    K = max(a.steps, 10)
    # the plain 2x-refined run and the 4x-refined truth (the nested grids with
    # Nv = 2 Nv - 1 only serve the training pairs)
    fine_shape = (2 * N, 2 * N, 2 * Nv, 2 * Nv)
    truth_shape = (4 * N, 4 * N, 4 * Nv, 4 * Nv)

    def stepper(shape):
        return vp.Stepper2D(*shape, Lb, Lb, V, V, dt, dtype=torch.float32, device=dev, window=-1, diagnostics=1,
                            precise_tables=True)

    with ClockSampler(local) as clk:
        # training pairs: seeded initial conditions, 8 snapshots of the refined run each, two kicks per snapshot
        t0 = time.perf_counter()
        src = C.PairSource(N, N, Nv, Nv, Lb, Lb, V, V, dt, device=dev)
        rng = np.random.default_rng(20261203)
        ics = [C.draw_ic(rng, Lb) for _ in range(a.train_ics)]
        pairs = C.collect_kick_pairs(src, ics, tuple(range(10, 81, 10)), Lb, V)
        torch.cuda.synchronize(dev)
        t_pairs = time.perf_counter() - t0
        net = C.Corrector(dev, seed=0)
        t0 = time.perf_counter()
        losses = C.train_kicks(net, pairs, src.coarse, iters=a.train_iters, batch=16, lr=1e-3)
        w3_scale = net.w3_scale
        torch.cuda.synchronize(dev)
        t_train = time.perf_counter() - t0
        cells_trained = a.train_iters * 16 * math.prod(a.grid)
        del pairs
        # held-out runs: E-energy histories against the 4x-refined run
        erng = np.random.default_rng(20261204)
        eval_ics = [C.draw_ic(erng, Lb) for _ in range(a.eval_ics)]
        coarse, fine, truth = stepper(a.grid), stepper(fine_shape), stepper(truth_shape)
        learned = C.LearnedStepper2D(net, N, N, Nv, Nv, Lb, Lb, V, V, dt, device=dev)
        zero = C.LearnedStepper2D(C.Corrector(dev), N, N, Nv, Nv, Lb, Lb, V, V, dt, device=dev)
        res = []
        for ic in eval_ics:
            hist = {}
            for name, st, shape in (("truth", truth, truth_shape), ("plain_coarse", coarse, a.grid),
                                    ("plain_refined", fine, fine_shape)):
                h = torch.zeros((K, L.DIAG_COUNT), dtype=torch.float64, device=dev)
                st.run(C.initial(ic, shape, Lb, V, dev), K, history=h, graph=True)
                hist[name] = h[:, :2].cpu().numpy()
            for name, st in (("learned_coarse", learned), ("plain_coarse_separate_kicks", zero)):
                h = torch.zeros((K, 2), dtype=torch.float64, device=dev)
                st.run(C.initial(ic, a.grid, Lb, V, dev), K, history=h, graph=True)
                hist[name] = h.cpu().numpy()
            ref = hist["truth"][:, 0]
            t = dt * np.arange(1, K + 1)
            row = {"ic": ic}
            for name, h in hist.items():
                we = h[:, 0]
                row[name] = {"we_err": float(np.abs(we - ref).max() / np.abs(ref).max()),
                             "we_err_rms_log": float(np.sqrt(np.mean(np.log(np.maximum(we, 1e-300) / ref) ** 2))),
                             "rate": float(np.polyfit(t, 0.5 * np.log(np.maximum(we, 1e-300)), 1)[0]),
                             "mass_drift": float(h[-1, 1] / h[0, 1] - 1)}
            res.append(row)
        # device time per step, graph-replayed, after warm-up
        def timed(run, steps):
            run(steps)  # captures the graphs of this buffer
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            run(steps)
            e1.record()
            torch.cuda.synchronize(dev)
            return e0.elapsed_time(e1) / steps

        f_c = C.initial(eval_ics[0], a.grid, Lb, V, dev)
        f_f = C.initial(eval_ics[0], fine_shape, Lb, V, dev)
        ms = {"plain_coarse": timed(lambda k: coarse.run(f_c, k, graph=True), K),
              "learned_coarse": timed(lambda k: learned.run(f_c, k, graph=True), K),
              "plain_refined": timed(lambda k: fine.run(f_f, k, graph=True), K)}
        # the corrected kick alone (tensor-core roofline)
        Ex = coarse.ex
        out = torch.empty_like(f_c)
        net.kick(f_c, Ex, 2, dt, coarse.dvx, out=out)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 20
        e0.record()
        for _ in range(reps):
            net.kick(f_c, Ex, 2, dt, coarse.dvx, out=out)
        e1.record()
        torch.cuda.synchronize(dev)
        kick_ms = e0.elapsed_time(e1) / reps
        c0 = L.load().vp_launch_count()
        learned.step(f_c, out)
        launches_per_step = L.load().vp_launch_count() - c0
        torch.cuda.synchronize(dev)
        net.check()

    def mean(key, field):
        return float(np.mean([r[key][field] for r in res]))

    err = {k: mean(k, "we_err") for k in ("plain_coarse", "learned_coarse", "plain_refined",
                                           "plain_coarse_separate_kicks")}
    err_log = {k: mean(k, "we_err_rms_log") for k in ("plain_coarse", "learned_coarse", "plain_refined")}
    rate_err = {k: float(np.mean([abs(r[k]["rate"] - r["truth"]["rate"]) for r in res]))
                for k in ("plain_coarse", "learned_coarse", "plain_refined")}
    ratio = ms["learned_coarse"] / ms["plain_refined"]
    flops_cell = 2 * (16 * 64 + 80 * 64 + 80 * 16)  # one forward pass, padded shapes
    achieved = flops_cell * math.prod(a.grid) / (kick_ms * 1e-3) / 1e12
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peak, pk = float(json.load(fh)["bf16_tflops"]), "measured"
    except Exception:
        peak, pk = 1590.0, "fallback"
    if rank == 0:
        line = {
            "metric": "wall time per step, learned 32^4 / plain 2x-refined (lower is better; meaningful where "
                      "the learned E-energy error reaches the refined run's)",
            "value": ratio, "unit": "ratio", "n_gpus": world, "steps": K, "warmup": 4,
            "ms_per_step": ms["learned_coarse"], "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 state, bf16 network (fp32 accumulate)", "data": "synthetic",
            "config": {"workload": a.desc, "grid": list(a.grid), "refined_grid": list(fine_shape),
                       "truth_grid": list(truth_shape), "pair_grid": [2 * N, 2 * N, 2 * Nv - 1, 2 * Nv - 1],
                       "train_ics": a.train_ics, "train_pairs": 16 * a.train_ics,
                       "train_iters": a.train_iters, "batch_pairs": 16, "eval_ics": a.eval_ics,
                       "steps_per_eval_run": K},
            "errors_we_vs_truth": err, "errors_rms_log_we_vs_truth": err_log, "rate_error_vs_truth": rate_err,
            "learned_reaches_refined_error": bool(err["learned_coarse"] <= err["plain_refined"]),
            "learned_improves_on_plain_coarse": bool(err["learned_coarse"] < err["plain_coarse"]),
            "ms_per_step_each": ms,
            "training": {"pairs_s": t_pairs, "train_s": t_train, "loss_first": losses[0],
                         "loss_last_20_mean": float(np.mean(losses[-20:])), "w3_scale": w3_scale,
                         "cell_samples": cells_trained},
            "eval_runs": res,
            "roofline": {"bound": "tensor", "kernel": "corrected kick (forward network per cell)",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "peak_kind": pk, "traffic": None, "kick_ms": kick_ms,
                         "flops_per_launch": flops_cell * math.prod(a.grid)},
            "gpu_launches": int(launches_per_step * K),
            "e2e": None, "cpu_baseline": None,
        }
        clk_s = clk.summary()
        if clk_s:
            line["clocks"] = clk_s
        print(json.dumps(line), flush=True)
    return 0


def main():
    a = parse()
    if a.kind == "learned":
        if a.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no learned interpolation "
                              "corrector (its interpolation is plain Lagrange only)"}), flush=True)
            return 0
        return run_learned(a)
    if a.kind == "batch":
        return run_batch_reference(a) if a.impl == "reference" else run_batch(a)
    if a.impl == "reference":
        return run_reference(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
