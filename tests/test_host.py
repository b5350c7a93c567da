"""Host-side logic that needs no GPU: static drift tables, argument checks of
the tensor API, velocity-layout classification, snapshot files, and the
multi-process plumbing on gloo (world size 2)."""
import importlib
import math
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from conftest import PACKAGE, ROOT


@pytest.mark.parametrize("tag", ["c1", "c2", "c3", "ref128", "oned4096"])
@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_drift_tables_match_reference(vp, golden, tag, dt):
    """The library's drift tables equal precompute_x_drift's bit for bit."""
    t = golden("tables")
    n, vmax, dx, half_dt = t[f"{tag}_{dt}_meta"]
    tdt = torch.float64 if dt == "f64" else torch.float32
    s, W = vp.ops.drift_table_np(torch.from_numpy(t[f"{tag}_{dt}_v"]), half_dt, dx, tdt)
    np.testing.assert_array_equal(s, t[f"{tag}_{dt}_shift"])
    np.testing.assert_array_equal(W, t[f"{tag}_{dt}_W"])
    v2 = importlib.import_module(PACKAGE + ".vlasov2d2v")
    blocks, Wt = v2.precompute_x_drift(torch.from_numpy(t[f"{tag}_{dt}_v"]), half_dt, dx, tdt)
    np.testing.assert_array_equal(v2._blocks_to_shift(blocks, int(n)), t[f"{tag}_{dt}_shift"])
    np.testing.assert_array_equal(Wt.numpy(), t[f"{tag}_{dt}_W"])


@pytest.mark.parametrize("tag", ["c1", "c2", "c3"])
def test_precise_tables_are_rounded_f64_tables(vp, golden, tag):
    """precise_tables: shifts of the float64 table, weights of the float64
    table rounded once to float32."""
    t = golden("tables")
    n, vmax, dx, half_dt = t[f"{tag}_f64_meta"]
    precise = vp.ops.DriftTable.from_velocity(torch.from_numpy(t[f"{tag}_f64_v"]), half_dt, dx, torch.float32,
                                              "cpu", precise=True)
    plain = vp.ops.DriftTable.from_velocity(torch.from_numpy(t[f"{tag}_f32_v"]), half_dt, dx, torch.float32, "cpu")
    np.testing.assert_array_equal(precise.shift.numpy(), t[f"{tag}_f64_shift"])
    np.testing.assert_array_equal(precise.W.numpy(), t[f"{tag}_f64_W"].astype(np.float32))
    np.testing.assert_array_equal(plain.W.numpy(), t[f"{tag}_f32_W"])
    assert precise.W.dtype == plain.W.dtype == torch.float32


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_lagrange_weights_host(vp, golden, dt):
    t = golden("tables")
    a = t["alpha"].astype(np.float64 if dt == "f64" else np.float32)
    np.testing.assert_array_equal(vp.ops.lagrange5_weights_np(a), t[f"lag5_{dt}"])


def test_tensor_api_rejects_cpu_tensors(vp):
    f = torch.zeros(4, 4, 4, 4)
    table = type("T", (), {"n": 4, "shift": torch.zeros(4, dtype=torch.int32), "W": torch.zeros(6, 4)})()
    with pytest.raises(ValueError, match="CUDA"):
        vp.ops.drift(f, table, 0, 2)
    with pytest.raises(ValueError, match="CUDA"):
        vp.ops.kick(f, torch.zeros(4, 4), 0.1, 0.1, 2)
    with pytest.raises(ValueError, match="CUDA"):
        vp.ops.velocity_moment(f, 1.0, 1.0, 2)
    with pytest.raises(TypeError):
        vp._lib.dtype_code(torch.int32)


def test_stepper_requires_cuda(vp):
    with pytest.raises(ValueError):
        vp.Stepper2D(4, 4, 4, 4, 1.0, 1.0, 1.0, 1.0, 0.1, device="cpu")


def test_velocity_layout_classification(vp):
    v2 = importlib.import_module(PACKAGE + ".vlasov2d2v")
    f = torch.zeros(3, 4, 5, 6)
    k = v2._line_velocity_structure(f, torch.arange(5.0)[None, :, None], 0)
    assert k[0] == "drift" and k[1] == 2 and k[2].numel() == 5
    k = v2._line_velocity_structure(f, torch.arange(6.0)[None, None, :], 1)
    assert k[0] == "drift" and k[1] == 3
    k = v2._line_velocity_structure(f, torch.zeros(3, 4)[:, :, None], 2)
    assert k[0] == "kick" and tuple(k[1].shape) == (3, 4)
    k = v2._line_velocity_structure(f, torch.zeros(3, 4)[:, :, None], 3)
    assert k[0] == "kick" and tuple(k[1].shape) == (3, 4, 5)
    assert v2._line_velocity_structure(f, torch.zeros(4, 5, 6), 0) is None


def test_stencil_offsets_checked(vp):
    v2 = importlib.import_module(PACKAGE + ".vlasov2d2v")
    v2._check_offsets(torch.arange(-2, 4))
    with pytest.raises(NotImplementedError):
        v2._check_offsets(torch.arange(-3, 3))


def test_snapshot_raw_round_trip(vp, tmp_path):
    snap = importlib.import_module(PACKAGE + ".snapshot")
    a = np.random.default_rng(0).random((3, 4, 5)).astype(np.float32)
    snap.write_raw(tmp_path, 7, fn=a, rho=a[0])
    b = snap.read_raw(tmp_path / "fn_000007.bin", a.shape, np.float32)
    np.testing.assert_array_equal(a, b)
    assert (tmp_path / "rho_000007.bin").stat().st_size == a[0].nbytes


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import sys

    sys.path.insert(0, ROOT)
    dist = importlib.import_module(PACKAGE + ".dist")
    r, _, w = dist.init(backend="gloo", timeout_s=60)
    dist.barrier()
    mx = dist.max_over_ranks(10.0 + r)
    sm = dist.sum_over_ranks(1.0)
    out[r] = (w, mx, sm)
    dist.finalize()


def test_dist_gloo_world2():
    """bench.py's multi-rank timing: max over ranks, sum, barrier (gloo, CPU)."""
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == (2, 11.0, 2.0) and out[1] == (2, 11.0, 2.0)


def test_autotune_cache_keys(vp, tmp_path):
    """Cache entries per (kind, N_axis, N_contig, dtype) and per batch
    signature; missing entries fall back to the default tile shapes."""
    at = importlib.import_module(PACKAGE + ".autotune")
    shapes = [(16, 16, 32, 32), (64, 64, 48, 48), (16, 16, 32, 32)]
    assert at.segment_key("x", shapes[1], torch.float32) == "segments:x:64:147456:float32"
    assert at.segment_key("y", shapes[1], torch.float32) == "segments:y:64:2304:float32"
    assert at.launch_key(shapes, torch.float32) == at.launch_key(shapes[::-1], torch.float32)
    t = at.cached_tiles(shapes, torch.float32, cache={})
    assert t["block"] == [256, 256, 256] and t["run_segments"] == [(1, 1)] * 3
    cache = {at.segment_key("y", shapes[1], torch.float32): 2,
             at.launch_key(shapes, torch.float32): {"block": [128, 256, 128], "ctas_per_sm": [1, 2, 2]}}
    path = tmp_path / "tune.json"
    at.save_cache(cache, str(path))
    t = at.cached_tiles(shapes, torch.float32, cache=at.load_cache(str(path)))
    assert t["block"] == [128, 256, 128] and t["ctas_per_sm"] == [1, 2, 2]
    assert t["run_segments"] == [(1, 1), (1, 2), (1, 1)]


def test_corrector_packing_matches_oracle(vp):
    """The packed BF16 network (W1, W2, W3, W3T, W2T) has the layout the
    kernels and the oracle use."""
    C = importlib.import_module(PACKAGE + ".corrector")
    from oracle import corrector as OC

    net = C.Corrector("cpu", seed=5, out_scale=0.1)
    bits = net.net.view(torch.int16).numpy().view(np.uint16)
    ref = OC.pack_net(net.W1.numpy(), net.W2.numpy(), net.W3.numpy())
    np.testing.assert_array_equal(bits, ref)
    assert bits.size == C.NET_ELEMS


def test_corrector_oracle_line_projection():
    """The oracle's line projection: power-of-two lines keep the plain
    sweep's sums, the projected dL/dy has zero line sums, and other line
    lengths are left unprojected."""
    from oracle import corrector as OC

    rng = np.random.default_rng(3)
    shape = (3, 8, 4)
    lines = OC.lines_of(shape, 1)
    assert lines == (3, 8, 4) and OC.lines_of((3, 6, 4), 1) is None and OC.lines_of((3, 8, 5), 1) is None
    N = int(np.prod(shape))
    F = rng.random((N, 6), dtype=np.float32)
    w = rng.standard_normal((N, 6)).astype(np.float32) * np.float32(0.2)
    al = rng.random(N, dtype=np.float32)
    W1 = rng.standard_normal((OC.HID, OC.K1)).astype(np.float32) * np.float32(0.3)
    W2 = rng.standard_normal((OC.HID, OC.K2)).astype(np.float32) * np.float32(0.1)
    W3 = rng.standard_normal((OC.NO, OC.K2)).astype(np.float32) * np.float32(0.1)
    W3[6:] = 0
    y, _ = OC.forward_cells(F, w, al, W1, W2, W3, lines=lines)
    yu, _ = OC.forward_cells(F, w, al, W1, W2, W3)
    p = OC.plain_cells(F, w)
    ls = lambda v: np.asarray(v, np.float64).reshape(shape).sum(axis=1)  # noqa: E731
    np.testing.assert_allclose(ls(y), ls(p), rtol=0, atol=1e-5)
    assert np.abs(ls(yu) - ls(p)).max() > 1e-3
    # the projection's transpose: with residuals of zero line mean the
    # projected loss and gradients are the unprojected ones of the same
    # residuals (sum_l (gy_l - mean gy) dy_l = sum_l gy_l dy_l)
    target = y + rng.standard_normal(N).astype(np.float32) * np.float32(0.01)
    target = (target - OC.line_mean(target - y, lines)).astype(np.float32)
    a = OC.train_cells(F, w, al, target, W1, W2, W3, 1.0, lines=lines)
    b = OC.train_cells(F, w, al, (target + (yu - y)).astype(np.float32), W1, W2, W3, 1.0)
    assert abs(a[0] - b[0]) <= 1e-4 * a[0]
    for ga, gb in zip(a[1:], b[1:]):
        assert np.linalg.norm(ga - gb) <= 2e-2 * np.linalg.norm(gb)
