"""Parity of every sweep kernel with the CPU oracle on seeded inputs."""
import math

import numpy as np
import pytest
import torch

from oracle import core as O

pytestmark = pytest.mark.gpu

SHAPES = [(8, 6, 10, 12), (16, 16, 16, 16), (12, 20, 24, 36), (5, 7, 9, 11)]
NP = {torch.float32: np.float32, torch.float64: np.float64}
# FMA-vs-separate rounding of a 6-term sum of O(1) data
TOL = {torch.float64: 1e-14, torch.float32: 2e-6, torch.bfloat16: 1.6e-2}


def seeded(seed, shape, dtype):
    return np.random.default_rng(seed).random(shape).astype(NP.get(dtype, np.float32))


def to_dev(a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda").to(dtype)


def relerr(got, want):
    got = got.float().cpu().numpy() if got.dtype == torch.bfloat16 else got.cpu().numpy()
    return float(np.abs(got.astype(np.float64) - want).max() / max(np.abs(want).max(), 1e-300))


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32, torch.bfloat16])
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("axis", [0, 1])
@pytest.mark.parametrize("fac", [0.3, 2.7, 6.0])
def test_drift(vp, dtype, shape, axis, fac):
    ref_dt = torch.float64 if dtype == torch.float64 else torch.float32
    g = O.make_grid2d(*shape, 2 * math.pi, 3.0, 4.0, 5.0, dtype=NP[ref_dt])
    f = seeded(1, shape, ref_dt)
    if dtype == torch.bfloat16:  # start from bf16-representable data
        f = to_dev(f, dtype).float().cpu().numpy()
    dx = g.dx if axis == 0 else g.dy
    v = (g.vx / 4.0 if axis == 0 else g.vy / 5.0) * NP[ref_dt](fac * dx / 0.1)
    s, W = O.precompute_drift(v, 0.1, dx, NP[ref_dt])
    want = O.drift_static(f.astype(NP[ref_dt]), s, W, axis, axis + 2)
    table = vp.ops.DriftTable(s, W, dtype, torch.device("cuda"))
    got = vp.ops.drift(to_dev(f, dtype), table, axis, axis + 2)
    assert relerr(got, want) < TOL[dtype]


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32, torch.bfloat16])
@pytest.mark.parametrize("shape", SHAPES)
def test_drift_rho(vp, dtype, shape):
    ref_dt = torch.float64 if dtype == torch.float64 else torch.float32
    g = O.make_grid2d(*shape, 2 * math.pi, 3.0, 4.0, 5.0, dtype=NP[ref_dt])
    f = seeded(2, shape, ref_dt)
    s, W = O.precompute_drift(g.vy, 0.05, g.dy, NP[ref_dt])
    table = vp.ops.DriftTable(s, W, dtype, torch.device("cuda"))
    out, rho = vp.ops.drift_rho(to_dev(f, dtype), table, 1, 3, g.dvx * g.dvy)
    out64 = out.double().cpu().numpy()
    # rho is the FP64 sum of the stored values of the drift output
    want = out64.sum(axis=(2, 3)) * (g.dvx * g.dvy)
    np.testing.assert_allclose(rho.cpu().numpy(), want, rtol=1e-13, atol=0)
    want_f = O.drift_static(f, s, W, 1, 3)
    assert relerr(out, want_f) < TOL[dtype]


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("axis", [2, 3])
@pytest.mark.parametrize("fac,window", [(0.3, -1), (1.5, -1), (4.2, -1), (1.5, 1), (0.7, 0)])
def test_kick(vp, dtype, shape, axis, fac, window):
    g = O.make_grid2d(*shape, 2 * math.pi, 3.0, 4.0, 5.0, dtype=NP[dtype])
    f = seeded(3, shape, dtype)
    dv = g.dvx if axis == 2 else g.dvy
    T = NP[dtype]
    E = (T(fac * dv / 0.1) * (np.sin(2 * np.pi * np.arange(shape[0]) / shape[0])[:, None]
                              * np.cos(2 * np.pi * np.arange(shape[1]) / shape[1])[None, :])).astype(T)
    want = O.kick_static(f, E, 0.1, dv, axis, window=window)
    got = vp.ops.kick(to_dev(f, dtype), to_dev(E, dtype), 0.1, dv, axis, window=window)
    assert relerr(got, want) < TOL[dtype]


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32, torch.bfloat16])
@pytest.mark.parametrize("shape", SHAPES + [(4, 4, 32, 128), (3, 2, 64, 64), (2, 3, 16, 48)])
@pytest.mark.parametrize("window", [-1, 1])
def test_kick2d(vp, dtype, shape, window):
    ref_dt = torch.float64 if dtype == torch.float64 else torch.float32
    T = NP[ref_dt]
    g = O.make_grid2d(*shape, 2 * math.pi, 3.0, 4.0, 5.0, dtype=T)
    f = seeded(4, shape, ref_dt)
    if dtype == torch.bfloat16:
        f = to_dev(f, dtype).float().cpu().numpy()
    rng = np.random.default_rng(9)
    Ex = rng.uniform(-2.5, 2.5, shape[:2]) * g.dvx / 0.1
    Ey = rng.uniform(-2.5, 2.5, shape[:2]) * g.dvy / 0.1
    mid = O.kick_static(f, Ex.astype(T) if ref_dt == torch.float32 else Ex, 0.1, g.dvx, 2, window=window)
    if dtype == torch.bfloat16:
        mid = to_dev(mid, dtype).float().cpu().numpy()
    want = O.kick_static(mid, Ey.astype(T) if ref_dt == torch.float32 else Ey, 0.1, g.dvy, 3, window=window)
    Exd = torch.from_numpy(Ex).cuda()
    Eyd = torch.from_numpy(Ey).cuda()
    mom = torch.zeros((shape[0] * shape[1], 4), dtype=torch.float64, device="cuda")
    vx = torch.from_numpy(np.asarray(g.vx, np.float64)).cuda()
    vy = torch.from_numpy(np.asarray(g.vy, np.float64)).cuda()
    got = vp.ops.kick2d(to_dev(f, dtype), Exd, Eyd, 0.1, g.dvx, g.dvy, window=window, vx=vx, vy=vy, moments=mom)
    # the oracle evaluates the kick weights from E rounded to float32 for an
    # FP32 field; the kernel from the FP64 field: allow the weight rounding
    tol = {torch.float64: 1e-14, torch.float32: 1e-5, torch.bfloat16: 2e-2}[dtype]
    assert relerr(got, want) < tol
    out = got.double().cpu().numpy()
    v2 = np.asarray(g.vx, np.float64)[:, None] ** 2 + np.asarray(g.vy, np.float64)[None, :] ** 2
    m = mom.cpu().numpy().reshape(shape[0], shape[1], 4)
    np.testing.assert_allclose(m[..., 1], np.einsum("xyab,ab->xy", out, v2), rtol=1e-12)
    np.testing.assert_allclose(m[..., 2], np.einsum("xyab,xyab->xy", out, out), rtol=1e-12)
    np.testing.assert_allclose(m[..., 3], out.sum(axis=(2, 3)), rtol=1e-12)
    fin = to_dev(f, dtype).double().cpu().numpy()
    np.testing.assert_allclose(m[..., 0], np.einsum("xyab,ab->xy", fin, v2), rtol=1e-12)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32, torch.bfloat16])
@pytest.mark.parametrize("shape", [(4, 4, 32, 128), (2, 2, 30, 128), (3, 2, 13, 128), (2, 3, 9, 64)])
def test_kick2d_without_moments(vp, dtype, shape):
    """The step's form of the fused kick (no moment epilogue), including the
    4-row chunks of 4 doubles per lane and plane rows that end mid-chunk."""
    ref_dt = torch.float64 if dtype == torch.float64 else torch.float32
    T = NP[ref_dt]
    g = O.make_grid2d(*shape, 2 * math.pi, 3.0, 4.0, 5.0, dtype=T)
    f = seeded(5, shape, ref_dt)
    if dtype == torch.bfloat16:
        f = to_dev(f, dtype).float().cpu().numpy()
    rng = np.random.default_rng(11)
    Ex = rng.uniform(-2.5, 2.5, shape[:2]) * g.dvx / 0.1
    Ey = rng.uniform(-2.5, 2.5, shape[:2]) * g.dvy / 0.1
    mid = O.kick_static(f, Ex.astype(T) if ref_dt == torch.float32 else Ex, 0.1, g.dvx, 2, window=-1)
    if dtype == torch.bfloat16:
        mid = to_dev(mid, dtype).float().cpu().numpy()
    want = O.kick_static(mid, Ey.astype(T) if ref_dt == torch.float32 else Ey, 0.1, g.dvy, 3, window=-1)
    got = vp.ops.kick2d(to_dev(f, dtype), torch.from_numpy(Ex).cuda(), torch.from_numpy(Ey).cuda(), 0.1, g.dvx,
                        g.dvy, window=-1)
    tol = {torch.float64: 1e-14, torch.float32: 1e-5, torch.bfloat16: 2e-2}[dtype]
    assert relerr(got, want) < tol


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("axis", [0, 1, 2, 3])
@pytest.mark.parametrize("shape", [(8, 6, 10, 12), (7, 9, 5, 6)])
def test_gather_bitwise(vp, dtype, axis, shape):
    """The per-element sweep rounds every operation like the reference
    (explicit round-to-nearest, no contraction): bit-identical to the oracle."""
    g = O.make_grid2d(*shape, 2 * math.pi, 3.0, 4.0, 5.0, dtype=NP[dtype])
    f = seeded(5, shape, dtype)
    T = NP[dtype]
    hx = {0: g.dx, 1: g.dy, 2: g.dvx, 3: g.dvy}
    vel = {
        0: g.vx[None, :, None] * T(1.7),
        1: g.vy[None, None, :] * T(-2.3),
        2: np.linspace(-3, 3, shape[0] * shape[1]).astype(T).reshape(shape[0], shape[1])[:, :, None],
        3: np.linspace(4, -4, shape[0] * shape[1]).astype(T).reshape(shape[0], shape[1])[:, :, None],
    }[axis]
    want = O.advect_gather(f, vel, axis, 0.1, hx[axis], periodic=axis < 2)
    got = vp.ops.advect_gather(to_dev(f, dtype), to_dev(np.asarray(vel), dtype), axis, 0.1, hx[axis], axis < 2)
    np.testing.assert_array_equal(got.cpu().numpy(), want)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32, torch.bfloat16])
def test_rho(vp, dtype):
    f = seeded(6, (9, 7, 11, 13), torch.float32)
    fd = to_dev(f, dtype)
    rho = vp.ops.velocity_moment(fd, 0.3, 0.7, 2)
    want = (fd.double().cpu().numpy().sum(axis=(2, 3)) * 0.3) * 0.7
    np.testing.assert_allclose(rho.cpu().numpy(), want, rtol=1e-14)


def test_contiguous_kick_long_rows(vp):
    """1D1V v kick: rows of 4096 elements (Nv of the reference's 1D benchmark)."""
    f = seeded(7, (6, 4096), torch.float64)
    E = np.linspace(-3, 3, 6)
    dv = 10.0 / 4095
    for window in (-1, 1):
        want = O.kick_static(f, E, 0.05, dv, 1, window=window)
        got = vp.ops.kick(to_dev(f, torch.float64), to_dev(E, torch.float64), 0.05, dv, 1, window=window)
        assert relerr(got, want) < 1e-14


@pytest.mark.parametrize("dtype", [torch.float32, torch.bfloat16])
@pytest.mark.parametrize("n", [4, 12, 48, 256, 4096, 8192])
@pytest.mark.parametrize("window", [-1, 0, 1])
def test_contiguous_kick_vector_rows_equal_scalar_rows(vp, dtype, n, window):
    """Rows of a multiple of 4 elements at 16-byte (8-byte for BF16) aligned
    addresses take the 4-wide kernel; the same rows one element off that
    alignment take the one-element-per-thread kernel. Both apply the 6 taps in
    the same order with zero fill, so the results agree bit for bit."""
    rows = 37
    f = to_dev(seeded(8, (rows, n), torch.float32) + 0.25, dtype)
    dv = 10.0 / (n - 1) if n > 1 else 1.0
    # shifts from a fraction of a cell to several times the row length
    E = to_dev(np.linspace(-1.0, 1.0, rows) * (3.0 * n * dv / 0.05) * np.geomspace(1e-3, 1.0, rows), torch.float32)
    want = vp.ops.kick(f, E, 0.05, dv, 1, window=window)
    flat = torch.empty(rows * n + 1, dtype=dtype, device="cuda")
    off = flat[1:].view(rows, n)
    off.copy_(f)
    out_flat = torch.empty(rows * n + 1, dtype=dtype, device="cuda")
    got = vp.ops.kick(off, E, 0.05, dv, 1, window=window, out=out_flat[1:].view(rows, n))
    assert torch.equal(got.view(torch.int16 if dtype == torch.bfloat16 else torch.int32),
                       want.view(torch.int16 if dtype == torch.bfloat16 else torch.int32))
