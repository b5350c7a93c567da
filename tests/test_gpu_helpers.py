"""The reference modules' smaller public helpers, against outputs of the
reference itself (tests/golden/helpers.npz, made by make_golden.py from the
same seeded inputs): block_roll, build_v_tap_weights, the batched 2D sweep
advect_1d_vectorized, advect_1d_matrix_diag_core with its roll and
banded-weight helpers, and the 1D1V forms (vlasov2D2V.py:287-353, 526-589,
717-753, 822-865; vlasov1D1V.py:258-296, 389-406, 450-476)."""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TD = {"f64": torch.float64, "f32": torch.float32}
SMALL = dict(Nx=8, Ny=6, Nvx=10, Nvy=12, Lx=2.0 * math.pi, Ly=3.0, Vx_max=4.0, Vy_max=5.0)
# per-element departure / kick kernels against the reference's gather and
# roll forms: bit-identical where the arithmetic is the same, else round-off
SWEEP_REL = {"f64": 1e-13, "f32": 2e-6}


def rng_f(seed, shape, dt):
    return torch.from_numpy(np.random.default_rng(seed).random(shape)).to(TD[dt]).cuda()


def close(got, want, rel):
    got = got.double().cpu().numpy()
    scale = max(np.abs(want).max(), 1e-300)
    assert np.abs(got - want).max() <= rel * scale


@pytest.fixture(scope="module")
def H(golden):
    return golden("helpers")


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_block_roll(vp, H, dt):
    v2 = vp.vlasov2d2v
    g = v2.Grid.create(**SMALL, device="cuda", dtype=TD[dt])
    f = rng_f(21, (g.Nx, g.Ny, g.Nvx, g.Nvy), dt)
    for axis, vel in ((0, g.vx), (1, g.vy)):
        h = g.dx if axis == 0 else g.dy
        blocks, _ = v2.precompute_x_drift(vel * 3.1, 0.1, h, TD[dt])
        got = v2.block_roll(f, blocks, axis, axis + 2)
        np.testing.assert_array_equal(got.cpu().numpy(), H[f"broll_{dt}_a{axis}"])
    # no block moves: the input itself comes back
    assert v2.block_roll(f, [(0, g.Nvx, 0)], 0, 2) is f


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_build_v_tap_weights(vp, H, dt):
    v2 = vp.vlasov2d2v
    g = v2.Grid.create(**SMALL, device="cuda", dtype=TD[dt])
    T = TD[dt]
    E = (0.7 * torch.sin(torch.arange(g.Nx * g.Ny, dtype=T).reshape(g.Nx, g.Ny))).to(T).cuda()
    for S in (1, 2):
        got = v2.build_v_tap_weights(E, 0.1, g.dvx, S, g.stencil_offsets)
        np.testing.assert_array_equal(got.cpu().numpy(), H[f"vtap_{dt}_S{S}"])


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_batched_sweeps(vp, H, dt):
    v2 = vp.vlasov2d2v
    T = TD[dt]
    B, N = 7, 19
    fb = rng_f(22, (B, N), dt)
    vb = torch.linspace(-3.0, 4.0, B, dtype=T).cuda()
    ve = (2.5 * torch.cos(torch.arange(B * N, dtype=T) * 0.37).reshape(B, N)).to(T).cuda()
    so = torch.arange(-2, 4, dtype=torch.int64)
    for per in (True, False):
        tag = "p" if per else "d"
        # the per-element departure kernel reproduces the reference's gather bit for bit
        np.testing.assert_array_equal(v2.advect_1d_vectorized(fb, vb, 0.1, 0.25, periodic=per).cpu().numpy(),
                                      H[f"avec_{dt}_rows_{tag}"])
        np.testing.assert_array_equal(v2.advect_1d_vectorized(fb, ve, 0.1, 0.25, periodic=per).cpu().numpy(),
                                      H[f"avec_{dt}_elem_{tag}"])
        close(v2.advect_1d_matrix_diag_core(fb, vb, 0.1, 0.25, so, periodic=per), H[f"mdcore_{dt}_{tag}"],
              SWEEP_REL[dt])


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_roll_and_banded_weights(vp, H, dt):
    v2, v1 = vp.vlasov2d2v, vp.vlasov1d1v
    T = TD[dt]
    B, N = 7, 19
    fb = rng_f(22, (B, N), dt)
    sh = torch.tensor([-3, 0, 2, 5, -7, 19, 40], dtype=torch.int64).cuda()
    np.testing.assert_array_equal(v2._roll_batch(fb, sh).cpu().numpy(), H[f"rollb_{dt}"])
    al = torch.linspace(0.05, 0.95, B, dtype=T).cuda()
    so = torch.arange(-2, 4, dtype=torch.int64).cuda()
    np.testing.assert_array_equal(v2.build_diag_weights(so, sh, al, N).cpu().numpy(), H[f"dw_{dt}"])
    f1 = rng_f(23, (24, 20), dt)
    shc = (torch.arange(20, dtype=torch.int64) - 9).cuda()
    shr = (torch.arange(24, dtype=torch.int64) * 3 - 30).cuda()
    np.testing.assert_array_equal(v1._roll_columns(f1, shc).cpu().numpy(), H[f"rollc1_{dt}"])
    np.testing.assert_array_equal(v1._roll_rows(f1, shr).cpu().numpy(), H[f"rollr1_{dt}"])
    al1 = torch.linspace(0.1, 0.9, 24, dtype=T).cuda()
    np.testing.assert_array_equal(v1.build_v_diag_weights(so, shr, al1, 20).cpu().numpy(), H[f"vdw1_{dt}"])


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_oned_block_roll_and_taps(vp, H, dt):
    v1 = vp.vlasov1d1v
    T = TD[dt]
    g1 = v1.Grid.create(24, 20, 4.0 * math.pi, 5.0, device="cuda", dtype=T)
    f1 = rng_f(23, (24, 20), dt)
    blocks1, _ = v1.precompute_x_drift(g1.v * 2.3, 0.1, g1.dx, T)
    np.testing.assert_array_equal(v1.block_roll(f1, blocks1).cpu().numpy(), H[f"broll1_{dt}"])
    E1 = (0.9 * torch.sin(torch.arange(24, dtype=T))).to(T).cuda()
    np.testing.assert_array_equal(v1.build_v_tap_weights(E1, 0.1, g1.dv, 1, g1.stencil_offsets).cpu().numpy(),
                                  H[f"vtap1_{dt}"])
