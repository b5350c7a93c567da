"""Batched uneven runs (vp_batch2d_*): every run of a batch follows the
single-run step exactly. With the default tile shapes the batch reproduces
Stepper2D bit for bit (same item bodies, same reduction order): the runs whose
drift pairs the batch fuses against a Stepper2D with the fused passes, the
others against one sweep per axis; other tile shapes only reorder the FP64
charge sums."""
import math

import numpy as np
import pytest
import torch

from oracle import core as O

pytestmark = pytest.mark.gpu

RUNS = [
    dict(Nx=16, Ny=24, Nvx=32, Nvy=48, Lx=4 * math.pi, Ly=4 * math.pi, Vx_max=6.0, Vy_max=6.0, dt=0.1),
    dict(Nx=32, Ny=56, Nvx=48, Nvy=32, Lx=10 * math.pi, Ly=6 * math.pi, Vx_max=8.0, Vy_max=7.0, dt=0.05),
    dict(Nx=24, Ny=64, Nvx=64, Nvy=64, Lx=2 * math.pi / 0.7, Ly=2 * math.pi / 0.7, Vx_max=7.5, Vy_max=7.5,
         dt=0.05),
    dict(Nx=8, Ny=8, Nvx=16, Nvy=12, Lx=4 * math.pi, Ly=4 * math.pi, Vx_max=6.0, Vy_max=5.0, dt=0.3),
    dict(Nx=12, Ny=40, Nvx=20, Nvy=24, Lx=8.0, Ly=9.0, Vx_max=5.0, Vy_max=6.0, dt=0.2),
]


def _ic(vp, p, r, dtype):
    kind = "landau" if r % 2 == 0 else "two_stream"
    return vp.workloads.initial_2d(kind, p["Nx"], p["Ny"], p["Nvx"], p["Nvy"], p["Lx"], p["Ly"], p["Vx_max"],
                                   p["Vy_max"], 0.05, 2 * math.pi / p["Lx"], 1.5, dtype=dtype)


def _single(vp, p, dtype, fused):
    # the same drift passes as the batch's run: fused pairs or one sweep per
    # axis (the two sum the density in different orders)
    return vp.Stepper2D(p["Nx"], p["Ny"], p["Nvx"], p["Nvy"], p["Lx"], p["Ly"], p["Vx_max"], p["Vy_max"], p["dt"],
                        dtype=dtype, window=-1, diagnostics=1, fuse_drifts=fused)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32, torch.bfloat16])
def test_batch_equals_single_runs(vp, dtype):
    b = vp.BatchStepper2D(RUNS, dtype=dtype, window=-1, diagnostics=1)
    assert b.fused == ([False, True, True, False, False] if dtype == torch.float32 else [False] * len(RUNS))
    ref = []
    for r, p in enumerate(RUNS):
        f0 = _ic(vp, p, r, dtype)
        b.set_state(r, f0)
        st = _single(vp, p, dtype, b.fused[r])
        assert st.passes(st.empty_f(), st.empty_f())[1] == b.fused[r]
        ref.append((st, f0.clone()))
    hist = []
    for s in range(3):
        b.step(0)
        hist.append(b.stage[0].clone())
        for r, (st, f) in enumerate(ref):
            ref[r] = (st, st.step(f))
            assert torch.equal(b.f[r], ref[r][1]), (r, s)
            assert torch.equal(b.drho[r], st.drho) and torch.equal(b.phi[r], st.phi)
            d = hist[-1][r].cpu().numpy()
            np.testing.assert_array_equal(d[[0, 1, 5]], st.diag.cpu().numpy()[[0, 1, 5]])


@pytest.mark.parametrize("physics", [True, False])
def test_batch_fused_and_sweeps(vp, physics):
    """The fused drift pairs of a batch against one sweep per axis: the same
    f to FP32 rounding of the density's summation order, the same density."""
    dtype = torch.float32
    a = vp.BatchStepper2D(RUNS, dtype=dtype, physics_mode=physics, diagnostics=1 if physics else 0)
    b = vp.BatchStepper2D(RUNS, dtype=dtype, physics_mode=physics, diagnostics=1 if physics else 0,
                          fuse_drifts=False)
    assert any(a.fused) and not any(b.fused)
    for r, p in enumerate(RUNS):
        f0 = _ic(vp, p, r, dtype)
        a.set_state(r, f0)
        b.set_state(r, f0)
    for _ in range(3):
        a.step(0)
        b.step(0)
    torch.cuda.synchronize()
    for r in range(len(RUNS)):
        if physics:
            np.testing.assert_allclose(a.drho[r].cpu().numpy(), b.drho[r].cpu().numpy(), rtol=0, atol=1e-9)
            scale = b.f[r].abs().max().item()
            assert (a.f[r] - b.f[r]).abs().max().item() <= 1e-5 * scale
        else:
            assert torch.equal(a.f[r], b.f[r])  # drifts only: the same bits


def test_batch_tile_shapes(vp):
    """Other tile shapes: 128-thread tiles, split lines, one CTA per SM. The
    drifts and kicks are unchanged; only the FP64 charge sums are reordered."""
    dtype = torch.float64
    a = vp.BatchStepper2D(RUNS, dtype=dtype)
    b = vp.BatchStepper2D(RUNS, dtype=dtype, tiles=dict(block=(128, 128, 128), ctas_per_sm=(1, 1, 1),
                                                        segments=(2, 4, 1)))
    c = vp.BatchStepper2D(RUNS, dtype=dtype, tiles=dict(block=(256, 256, 256), ctas_per_sm=(2, 1, 2),
                                                        segments=(4, 2, 1)))
    for r, p in enumerate(RUNS):
        f0 = _ic(vp, p, r, dtype)
        for s in (a, b, c):
            s.set_state(r, f0)
    for _ in range(3):
        a.step(0)
        b.step(0)
        c.step(0)
    torch.cuda.synchronize()
    for r in range(len(RUNS)):
        scale = a.f[r].abs().max().item()
        assert (b.f[r] - a.f[r]).abs().max().item() <= 1e-13 * scale
        assert torch.equal(c.f[r], a.f[r])  # same tiles width: identical sums
    np.testing.assert_allclose(b.stage[0].cpu().numpy()[:, :2], a.stage[0].cpu().numpy()[:, :2], rtol=1e-12)


def test_batch_graph_history(vp):
    """A graph-captured run equals eager steps, history included."""
    dtype = torch.float32
    a = vp.BatchStepper2D(RUNS, dtype=dtype, graph_slots=4)
    b = vp.BatchStepper2D(RUNS, dtype=dtype, graph_slots=4)
    for r, p in enumerate(RUNS):
        f0 = _ic(vp, p, r, dtype)
        a.set_state(r, f0)
        b.set_state(r, f0)
    n = 11
    ha = torch.zeros((n, len(RUNS), 8), dtype=torch.float64, device="cuda")
    hb = torch.zeros_like(ha)
    a.run(n, history=ha, graph=True)
    b.run(n, history=hb, graph=False)
    torch.cuda.synchronize()
    for r in range(len(RUNS)):
        assert torch.equal(a.f[r], b.f[r])
    assert torch.equal(ha[:, :, :2], hb[:, :, :2])
    a.run(5, graph=True)  # replays the cached graph, then eager steps
    b.run(5, graph=False)
    for r in range(len(RUNS)):
        assert torch.equal(a.f[r], b.f[r])


def test_batch_against_oracle_fp64(vp):
    """Two runs of the batch against the CPU oracle's step (FP64)."""
    runs = [RUNS[0], RUNS[3]]
    b = vp.BatchStepper2D(runs, dtype=torch.float64, window=-1)
    fs = []
    for r, p in enumerate(runs):
        g = O.make_grid2d(p["Nx"], p["Ny"], p["Nvx"], p["Nvy"], p["Lx"], p["Ly"], p["Vx_max"], p["Vy_max"],
                          dtype=np.float64)
        f = O.landau_2d(g, 0.1, 2 * math.pi / p["Lx"])
        b.set_state(r, torch.from_numpy(f).cuda())
        fs.append((g, f))
    b.step(0)
    torch.cuda.synchronize()
    for r, (g, f) in enumerate(fs):
        fo = O.Stepper2D(g, runs[r]["dt"], window=-1).step(f).f
        err = np.abs(b.f[r].cpu().numpy() - fo).max() / np.abs(fo).max()
        assert err <= 1e-12, (r, err)


def test_batch_seeded_draws(vp):
    """The 64 seeded uneven runs: two batched steps equal four of the runs
    stepped alone, and every run keeps its mass."""
    runs = vp.workloads.batch_runs()
    b = vp.BatchStepper2D(runs, dtype=torch.float32)
    for r, p in enumerate(runs):
        b.set_state(r, vp.workloads.initial_2d(p["kind"], p["Nx"], p["Ny"], p["Nvx"], p["Nvy"], p["Lx"], p["Ly"],
                                               p["Vx_max"], p["Vy_max"], p["eps"], p["k"], p["v0"]))
    pick = [0, 17, 40, 63] + [r for r in range(len(runs)) if runs[r]["Nvy"] % 32][:2]  # fused and not
    singles = {r: (_single(vp, runs[r], torch.float32, b.fused[r]), b.f[r].clone()) for r in pick}
    h = torch.zeros((2, len(runs), 8), dtype=torch.float64, device="cuda")
    b.run(2, history=h, graph=False)
    for r, (st, f) in singles.items():
        f = st.step(st.step(f))
        assert torch.equal(b.f[r], f), r
    m = h[:, :, 1].cpu().numpy()
    np.testing.assert_allclose(m[1], m[0], rtol=1e-5)
    assert np.isfinite(h[:, :, 0].cpu().numpy()).all()


def test_autotune_small_batch(vp, tmp_path):
    """The autotuner runs on a small batch, records its choices, and the tuned
    batch computes the same steps (FP64: only the charge sums reorder)."""
    at = vp.autotune
    dtype = torch.float64
    a = vp.BatchStepper2D(RUNS, dtype=dtype)
    t = vp.BatchStepper2D(RUNS, dtype=dtype)
    for r, p in enumerate(RUNS):
        t.set_state(r, _ic(vp, p, r, dtype))
    cache = str(tmp_path / "tune.json")
    tiles = at.tune(t, reps=1, steps=1, cache_file=cache)
    assert len(tiles["run_segments"]) == len(RUNS)
    saved = at.load_cache(cache)
    assert at.launch_key(t.shapes, dtype) in saved
    assert at.cached_tiles(t.shapes, dtype, cache=saved)["run_segments"] == [tuple(s) for s in tiles["run_segments"]]
    for r, p in enumerate(RUNS):
        f0 = _ic(vp, p, r, dtype)
        a.set_state(r, f0)
        t.set_state(r, f0)
    for _ in range(2):
        a.step(0)
        t.step(0)
    torch.cuda.synchronize()
    for r in range(len(RUNS)):
        assert (t.f[r] - a.f[r]).abs().max().item() <= 1e-13 * a.f[r].abs().max().item()


def test_batch_beyond_64_runs(vp):
    """66 runs, fused ones at run indices on both sides of 64 (the plane
    records, fused runs only, map back to their runs): each equals the run
    stepped alone. More than 64 fused runs per launch class:
    test_batch_chained_plane_launches."""
    small = dict(Nx=8, Ny=8, Nvx=16, Nvy=16, Lx=4 * math.pi, Ly=4 * math.pi, Vx_max=6.0, Vy_max=6.0, dt=0.1)
    big = dict(Nx=32, Ny=32, Nvx=16, Nvy=32, Lx=4 * math.pi, Ly=4 * math.pi, Vx_max=6.0, Vy_max=5.0, dt=0.1)
    runs = [dict(big) if r in (1, 64, 65) else dict(small) for r in range(66)]
    b = vp.BatchStepper2D(runs, dtype=torch.float32, window=-1, diagnostics=1)
    assert [r for r in range(66) if b.fused[r]] == [1, 64, 65]
    ref = {}
    for r, p in enumerate(runs):
        f0 = _ic(vp, p, r, torch.float32)
        b.set_state(r, f0)
        if r in (0, 1, 63, 64, 65):
            ref[r] = (_single(vp, p, torch.float32, b.fused[r]), f0.clone())
    for _ in range(2):
        b.step(0)
        for r, (st, f) in ref.items():
            ref[r] = (st, st.step(f))
            assert torch.equal(b.f[r], ref[r][1]), r
            assert torch.equal(b.drho[r], st.drho), r


@pytest.mark.parametrize("physics", [True, False])
def test_batch_chained_plane_launches(vp, physics):
    """More than 64 fused runs in each box class (two launches per class and
    pass, the 64-run parameter chunks) and runs on sweeps: the plane passes'
    four launches and the sweep after them follow each other as programmatic
    dependents. Every run against the same batch on one sweep per axis:
    bit-identical drifts, and with the field the density to 1e-9 (its
    summation order differs)."""
    base = dict(Nx=32, Ny=32, Lx=4 * math.pi, Ly=4 * math.pi, Vx_max=6.0, Vy_max=6.0, dt=0.1)
    whole = dict(base, Nvx=16, Nvy=32)
    half = dict(base, Nvx=16, Nvy=48)
    swept = dict(base, Nx=16, Ny=16, Nvx=16, Nvy=32)
    runs = [dict(whole) for _ in range(66)] + [dict(half) for _ in range(66)] + [dict(swept) for _ in range(3)]
    # interleave the classes, so that the plan's ordering is exercised too
    order = [r for trio in zip(range(0, 66), range(66, 132)) for r in trio] + [132, 133, 134]
    runs = [runs[r] for r in order]
    dtype = torch.float32
    a = vp.BatchStepper2D(runs, dtype=dtype, physics_mode=physics, diagnostics=1 if physics else 0)
    b = vp.BatchStepper2D(runs, dtype=dtype, physics_mode=physics, diagnostics=1 if physics else 0,
                          fuse_drifts=False)
    assert sum(a.fused) == 132 and not any(b.fused)
    for r, p in enumerate(runs):
        f0 = _ic(vp, p, r, dtype)
        a.set_state(r, f0)
        b.set_state(r, f0)
    for _ in range(2):
        a.step(0)
        b.step(0)
    torch.cuda.synchronize()
    a.check()
    for r in range(len(runs)):
        if physics:
            np.testing.assert_allclose(a.drho[r].cpu().numpy(), b.drho[r].cpu().numpy(), rtol=0, atol=1e-9)
            assert (a.f[r] - b.f[r]).abs().max().item() <= 1e-5 * b.f[r].abs().max().item(), r
        else:
            assert torch.equal(a.f[r], b.f[r]), r


@pytest.mark.parametrize("physics", [True, False])
def test_batch_half_box_runs(vp, physics):
    """Runs whose 32-column groups span two vx (nvy = 48, 80): the fused
    passes load each half group at its own x row. Against one sweep per axis:
    the drifts alone are bit-identical, with the field the density's summation
    order differs (f to FP32 rounding)."""
    runs = [dict(Nx=32, Ny=32, Nvx=32, Nvy=48, Lx=4 * math.pi, Ly=4 * math.pi, Vx_max=6.0, Vy_max=6.0, dt=0.1),
            dict(Nx=24, Ny=48, Nvx=16, Nvy=48, Lx=6 * math.pi, Ly=5 * math.pi, Vx_max=7.0, Vy_max=6.0, dt=0.08),
            dict(Nx=16, Ny=40, Nvx=8, Nvy=80, Lx=4 * math.pi, Ly=4 * math.pi, Vx_max=5.0, Vy_max=8.0, dt=0.2),
            dict(Nx=16, Ny=32, Nvx=16, Nvy=64, Lx=4 * math.pi, Ly=4 * math.pi, Vx_max=6.0, Vy_max=6.0, dt=0.1)]
    dtype = torch.float32
    a = vp.BatchStepper2D(runs, dtype=dtype, physics_mode=physics, diagnostics=1 if physics else 0)
    b = vp.BatchStepper2D(runs, dtype=dtype, physics_mode=physics, diagnostics=1 if physics else 0,
                          fuse_drifts=False)
    assert a.fused == [True] * 4 and not any(b.fused)
    for r, p in enumerate(runs):
        f0 = _ic(vp, p, r, dtype)
        a.set_state(r, f0)
        b.set_state(r, f0)
    for _ in range(3):
        a.step(0)
        b.step(0)
    torch.cuda.synchronize()
    a.check()
    for r in range(len(runs)):
        if physics:
            np.testing.assert_allclose(a.drho[r].cpu().numpy(), b.drho[r].cpu().numpy(), rtol=0, atol=1e-9)
            assert (a.f[r] - b.f[r]).abs().max().item() <= 1e-5 * b.f[r].abs().max().item(), r
        else:
            assert torch.equal(a.f[r], b.f[r]), r
