"""The fused (x, y) drift passes of the 2D2V step against the single-axis
sweeps: f bit for bit, the charge density to FP64 summation order."""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

# (Nx, Ny, Nvx, Nvy): Ny not a multiple of 8, Ny = 1, Nx below the stencil
# width, groups of 32 columns inside wider vy rows, the 128-row maximum
SHAPES = [(16, 16, 32, 32), (8, 6, 16, 64), (12, 100, 4, 32), (5, 3, 2, 32), (33, 128, 8, 64), (7, 1, 3, 32),
          (64, 128, 16, 128),
          # fused edge cases: x lines shorter than the stencil (window rows
          # repeat), two vx, the 16-row minimum, 17 rows (a part-filled warp)
          (3, 16, 2, 32), (2, 24, 2, 64), (5, 17, 3, 32), (9, 64, 2, 32), (4, 65, 2, 32),
          # x first with the register window (more than 112 rows): a part-filled
          # last warp, and the 113-row minimum
          (6, 120, 2, 32), (5, 113, 3, 64)]


def seeded(shape, seed):
    g = np.random.default_rng(seed)
    return torch.from_numpy(1.0 + 0.25 * g.standard_normal(shape)).float().cuda()


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("dt", [0.1, 1.3])
def test_plane_pairs_equal_sweeps(vp, shape, dt):
    Nx, Ny, Nvx, Nvy = shape
    st = vp.Stepper2D(Nx, Ny, Nvx, Nvy, 4 * math.pi, 3.0, 6.0, 5.0, dt, dtype=torch.float32, physics_mode=False)
    f = seeded(shape, 7)
    got = st.step(f)
    a = vp.ops.drift(f, st.tx, 0, 2)
    b = vp.ops.drift(a, st.ty, 1, 3)
    c = vp.ops.drift(b, st.ty, 1, 3)
    want = vp.ops.drift(c, st.tx, 0, 2)
    assert torch.equal(got, want)


@pytest.mark.parametrize("shape", [(16, 16, 32, 32), (12, 100, 4, 32), (64, 128, 16, 128), (3, 16, 2, 32),
                                   (5, 17, 3, 32), (4, 65, 2, 32), (6, 120, 2, 32), (5, 113, 3, 64)])
def test_plane_density(vp, shape):
    Nx, Ny, Nvx, Nvy = shape
    st = vp.Stepper2D(Nx, Ny, Nvx, Nvy, 4 * math.pi, 3.0, 6.0, 5.0, 0.4, dtype=torch.float32, physics_mode=True)
    f = seeded(shape, 11)
    st.step(f)
    a = vp.ops.drift(f, st.tx, 0, 2)
    _, rho = vp.ops.drift_rho(a, st.ty, 1, 3, st.dvx * st.dvy)
    np.testing.assert_allclose(st.drho.cpu().numpy(), rho.cpu().numpy() - 1.0, rtol=0, atol=1e-12)


SPLIT_SHAPES = [(16, 16, 32, 32), (12, 100, 4, 32), (64, 128, 16, 128), (5, 17, 3, 32), (4, 65, 2, 32),
                (6, 120, 2, 32), (5, 113, 3, 64)]


@pytest.mark.parametrize("shape", SPLIT_SHAPES)
def test_plane_pairs_equal_sweeps_split(vp, shape):
    """Equilibrium split (the state holds g = f - A(vx) B(vy)): the fused
    passes add each column's split constant exactly as the single-axis
    sweeps do, so the drifts of g are the same bits."""
    Nx, Ny, Nvx, Nvy = shape
    args = (Nx, Ny, Nvx, Nvy, 4 * math.pi, 3.0, 6.0, 5.0, 0.7)
    a = vp.Stepper2D(*args, dtype=torch.float32, physics_mode=False, equilibrium="maxwellian")
    b = vp.Stepper2D(*args, dtype=torch.float32, physics_mode=False, equilibrium="maxwellian", fuse_drifts=False)
    g = 0.01 * seeded(shape, 9)
    assert a.passes(g, a.empty_f()) == (2, True)
    assert b.passes(g, b.empty_f()) == (4, False)
    assert torch.equal(a.step(g), b.step(g))


@pytest.mark.parametrize("shape", [(16, 32, 8, 64), (8, 128, 4, 128)])
def test_fused_and_sweeps_only_split_steps(vp, shape):
    """A physics step of the split state: fused and single-axis drifts give
    the same density (the equilibrium's included) to FP64 summation order,
    and f to FP32 rounding."""
    args = (*shape, 4 * math.pi, 4 * math.pi, 6.0, 6.0, 0.3)
    a = vp.Stepper2D(*args, dtype=torch.float32, equilibrium="maxwellian")
    b = vp.Stepper2D(*args, dtype=torch.float32, equilibrium="maxwellian", fuse_drifts=False)
    g = 0.01 * seeded(shape, 13)
    assert a.passes(g, a.empty_f()) == (3, True)
    ga, gb = a.step(g), b.step(g)
    np.testing.assert_allclose(a.drho.cpu().numpy(), b.drho.cpu().numpy(), rtol=0, atol=1e-13)
    np.testing.assert_allclose(ga.cpu().numpy(), gb.cpu().numpy(), rtol=0, atol=1e-7)


def test_plane_graph_replay(vp):
    """Captured steps (the TMA descriptors live in the kernel parameters)
    replay to the eager result."""
    shape = (32, 64, 8, 64)
    st = vp.Stepper2D(*shape, 4 * math.pi, 4 * math.pi, 6.0, 6.0, 0.2, dtype=torch.float32)
    f = seeded(shape, 3)
    fa = st.run(f.clone(), 12, graph=False)
    fb = st.run(f.clone(), 12, graph=True, graph_chunk=4)
    assert torch.equal(fa, fb)


@pytest.mark.parametrize("dtype,physics,want", [(torch.float32, True, (3, True)), (torch.float32, False, (2, True)),
                                                (torch.float64, True, (5, False)), (torch.bfloat16, True, (5, False))])
def test_step_passes(vp, dtype, physics, want):
    """vp_step2d_passes: passes over f and whether the drifts are fused."""
    shape = (16, 16, 32, 32)
    st = vp.Stepper2D(*shape, 4 * math.pi, 4 * math.pi, 6.0, 6.0, 0.1, dtype=dtype, physics_mode=physics)
    f = st.empty_f()
    assert st.passes(f, st.empty_f()) == want
    # ny above 128, or fusion turned off, keeps the single-axis sweeps
    wide = vp.Stepper2D(4, 136, 2, 32, 4 * math.pi, 4 * math.pi, 6.0, 6.0, 0.1, dtype=torch.float32)
    assert wide.passes(wide.empty_f(), wide.empty_f()) == (3 + 2, False)
    off = vp.Stepper2D(*shape, 4 * math.pi, 4 * math.pi, 6.0, 6.0, 0.1, dtype=dtype, physics_mode=physics,
                       fuse_drifts=False)
    assert off.passes(f, off.empty_f()) == (want[0] + (2 if want[1] else 0), False)


def test_fused_and_sweeps_only_steps(vp):
    """Fused and single-axis drifts give the same f and density to FP64
    summation order over a physics step."""
    shape = (16, 32, 8, 64)
    args = (*shape, 4 * math.pi, 4 * math.pi, 6.0, 6.0, 0.3)
    a = vp.Stepper2D(*args, dtype=torch.float32)
    b = vp.Stepper2D(*args, dtype=torch.float32, fuse_drifts=False)
    f = seeded(shape, 5)
    fa, fb = a.step(f), b.step(f)
    np.testing.assert_allclose(a.drho.cpu().numpy(), b.drho.cpu().numpy(), rtol=0, atol=1e-13)
    np.testing.assert_allclose(fa.cpu().numpy(), fb.cpu().numpy(), rtol=0, atol=1e-6)
