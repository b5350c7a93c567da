"""Autotuner of the batched sweeps' tile shapes, with a JSON cache.

What is tuned (all measured on the device with CUDA events around the
substeps of eager batched steps, see BatchStepper2D.phase_ms):
  * per launch and sweep kind (x drifts, y drifts, fused kick): the tile
    width (128 or 256 threads, i.e. 512 or 1024 FP32 columns per CTA) and the
    number of persistent CTAs per SM (1 or 2);
  * per run shape and drift axis: the CTAs per line (1, 2 or 4 segments;
    each extra segment re-reads the 5-row interpolation halo of the line).
    Segments are tuned inside the batch they serve, one shape class at a
    time (coordinate descent), because a run's best split depends on how
    much parallelism the other runs already supply.

Cache entries (one JSON object):
  "segments:<kind>:<N_axis>:<N_contig>:<dtype>" -> 1 | 2 | 4
      kind x: N_axis = Nx, N_contig = Ny*Nvx*Nvy; kind y: N_axis = Ny,
      N_contig = Nvx*Nvy
  "launch:<dtype>:<signature of the batch's shapes>" -> {"block": [3], "ctas_per_sm": [3]}
The default cache file is tune_b200.json beside this module (overridden by
$VLASOV_B200_TUNE_CACHE).
"""
from __future__ import annotations

import hashlib
import json
import os
import statistics

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_CACHE = os.path.join(HERE, "tune_b200.json")
BLOCKS = (128, 256)
CTAS = (1, 2)
SEGMENTS = (1, 2, 4)


def cache_path() -> str:
    return os.environ.get("VLASOV_B200_TUNE_CACHE", DEFAULT_CACHE)


def load_cache(path: str | None = None) -> dict:
    path = path or cache_path()
    try:
        with open(path) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def save_cache(cache: dict, path: str | None = None) -> None:
    path = path or cache_path()
    tmp = path + ".tmp"
    with open(tmp, "w") as fh:
        json.dump(cache, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _dt(dtype) -> str:
    return str(dtype).replace("torch.", "")


def segment_key(kind: str, shape, dtype) -> str:
    nx, ny, nvx, nvy = shape
    if kind == "x":
        return f"segments:x:{nx}:{ny * nvx * nvy}:{_dt(dtype)}"
    return f"segments:y:{ny}:{nvx * nvy}:{_dt(dtype)}"


def launch_key(shapes, dtype) -> str:
    sig = ",".join("x".join(map(str, s)) for s in sorted(tuple(s) for s in shapes))
    return f"launch:{_dt(dtype)}:{hashlib.sha1(sig.encode()).hexdigest()[:16]}"


def cached_tiles(shapes, dtype, cache: dict | None = None) -> dict:
    """Tile shapes for a batch from the cache (defaults where it has none)."""
    cache = load_cache() if cache is None else cache
    launch = cache.get(launch_key(shapes, dtype), {})
    segs = [(int(cache.get(segment_key("x", s, dtype), 1)), int(cache.get(segment_key("y", s, dtype), 1)))
            for s in shapes]
    return {"block": list(launch.get("block", (256, 256, 256))),
            "ctas_per_sm": list(launch.get("ctas_per_sm", (0, 0, 0))),
            "segments": [1, 1, 1], "run_segments": segs}


def _kind_ms(stepper, reps: int, steps: int) -> dict:
    """Median over reps of the per-kind times: x (both x drifts), y (both y
    drifts), kick."""
    xs, ys, ks = [], [], []
    for _ in range(reps):
        ph = stepper.phase_ms(steps)
        xs.append(ph["drift_x1"] + ph["drift_x2"])
        ys.append(ph["drift_y1_rho"] + ph["drift_y2"])
        ks.append(ph["kick"])
    return {"x": statistics.median(xs), "y": statistics.median(ys), "kick": statistics.median(ks)}


def tune(stepper, reps: int = 3, steps: int = 3, min_gain: float = 0.01, cache_file: str | None = None,
         log=None) -> dict:
    """Tune a BatchStepper2D in place (its state advances while it is timed)
    and record the choices in the cache. Returns the chosen tiles dict."""
    shapes = [tuple(s) for s in stepper.shapes]
    n = len(shapes)
    say = log or (lambda *a: None)
    # 1. launch shapes per kind, whole lines everywhere
    best_t = {}
    for b in BLOCKS:
        for c in CTAS:
            tiles = {"block": [b] * 3, "ctas_per_sm": [c] * 3, "segments": [1, 1, 1], "run_segments": [(1, 1)] * n}
            stepper.retile(tiles)
            stepper.phase_ms(1)  # first launch of each kernel variant outside the timing
            t = _kind_ms(stepper, reps, steps)
            say(f"launch block={b} ctas={c}: {t}")
            for kind, v in t.items():
                if kind not in best_t or v < best_t[kind][0]:
                    best_t[kind] = (v, b, c)
    kinds = ("x", "y", "kick")
    block = [best_t[k][1] for k in kinds]
    ctas = [best_t[k][2] for k in kinds]
    # 2. segments per shape class and drift axis, by coordinate descent
    classes = sorted(set(shapes))
    segs = {s: [1, 1] for s in classes}

    def tiles_now():
        return {"block": block, "ctas_per_sm": ctas, "segments": [1, 1, 1],
                "run_segments": [tuple(segs[s]) for s in shapes]}

    stepper.retile(tiles_now())
    cur = _kind_ms(stepper, reps, steps)
    for cls in classes:
        for axis, kind in ((0, "x"), (1, "y")):
            best_v, best_s = cur[kind], segs[cls][axis]
            for sg in SEGMENTS:
                if sg == segs[cls][axis]:
                    continue
                old = segs[cls][axis]
                segs[cls][axis] = sg
                stepper.retile(tiles_now())
                v = _kind_ms(stepper, reps, steps)[kind]
                segs[cls][axis] = old
                if v < best_v * (1.0 - min_gain):
                    best_v, best_s = v, sg
            if best_s != segs[cls][axis]:
                say(f"class {cls} axis {kind}: segments {segs[cls][axis]} -> {best_s} ({cur[kind]:.4f} -> {best_v:.4f} ms)")
                segs[cls][axis] = best_s
                cur[kind] = best_v
    tiles = tiles_now()
    stepper.retile(tiles)
    cache = load_cache(cache_file)
    cache[launch_key(shapes, stepper.dtype)] = {"block": block, "ctas_per_sm": ctas}
    for cls in classes:
        cache[segment_key("x", cls, stepper.dtype)] = segs[cls][0]
        cache[segment_key("y", cls, stepper.dtype)] = segs[cls][1]
    save_cache(cache, cache_file)
    return tiles


def main(argv=None):
    """Tune the seeded 64-run batch on this GPU and write the cache."""
    import argparse
    import importlib

    ap = argparse.ArgumentParser()
    ap.add_argument("--dtype", default="float32", choices=["float32", "bfloat16", "float64"])
    ap.add_argument("--cache", default=None)
    a = ap.parse_args(argv)
    pkg = importlib.import_module(__package__)
    wl = importlib.import_module(__package__ + ".workloads")
    dtype = getattr(torch, a.dtype)
    runs = wl.batch_runs()
    st = pkg.BatchStepper2D(runs, dtype=dtype, window=1)
    for r, p in enumerate(runs):
        st.set_state(r, wl.initial_2d(p["kind"], p["Nx"], p["Ny"], p["Nvx"], p["Nvy"], p["Lx"], p["Ly"],
                                      p["Vx_max"], p["Vy_max"], p["eps"], p["k"], p["v0"], dtype=dtype))
    tiles = tune(st, cache_file=a.cache, log=print)
    print(json.dumps({k: v for k, v in tiles.items() if k != "run_segments"}))


if __name__ == "__main__":
    main()
