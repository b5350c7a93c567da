"""The reference's own test families, restated against the drop-in modules
on the GPU: interpolation exactness (simulations/vlasov2d_2v/pytorch/tests/
test_interpolation.py), analytic shifts and cross-kernel equality
(test_advection.py), full-step cross-checks, the real / complex Poisson
paths of 1D1V (vlasov1d_1v/pytorch/tests/test_poisson.py) and the grid
(test_grid.py). Same tolerances as the reference's tests."""
import importlib
import math

import numpy as np
import pytest
import torch

from conftest import PACKAGE

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def v2():
    return importlib.import_module(PACKAGE + ".vlasov2d2v")


@pytest.fixture(scope="module")
def v1():
    return importlib.import_module(PACKAGE + ".vlasov1d1v")


NODES = torch.arange(-2, 4, dtype=torch.float64)


# ---- interpolation -----------------------------------------------------------
@pytest.mark.parametrize("deg", range(6))
def test_interp_sum_exact_for_polynomials(v2, deg):
    alpha = torch.tensor([[0.0, 0.1, 0.25, 0.5, 0.75, 0.9, 1.0]], dtype=torch.float64)
    vals = (NODES ** deg).view(1, 1, 6).expand(1, alpha.shape[1], 6)
    got = v2.lagrange5_interp_sum(alpha.cuda(), vals.cuda()).cpu()
    np.testing.assert_allclose(got[0].numpy(), (alpha[0] ** deg).numpy(), atol=1e-10)


def test_interp_at_nodes_and_partition_of_unity(v2):
    g = torch.Generator().manual_seed(0)
    vals = torch.randn(5, 6, generator=g, dtype=torch.float64)
    zero = torch.zeros(5, dtype=torch.float64)
    np.testing.assert_allclose(v2.lagrange5_interp_sum(zero.cuda(), vals.cuda()).cpu().numpy(),
                               vals[:, 2].numpy(), atol=1e-12)
    alpha = torch.rand(7, 9, generator=g, dtype=torch.float64)
    w = v2.get_lagrange5_weights(alpha.cuda()).cpu()
    assert w.shape == (7, 9, 6)
    np.testing.assert_allclose(w.sum(-1).numpy(), 1.0, atol=1e-12)
    nodes_w = v2.get_lagrange5_weights(NODES.cuda()).cpu()  # alpha at a node: one-hot
    np.testing.assert_allclose(nodes_w.numpy(), np.eye(6), atol=1e-12)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_interp_helpers_bitwise(v2, dtype):
    """Both helpers round every operation as the reference's eager formulas
    do: equal to a CPU evaluation of those formulas bit for bit."""
    g = torch.Generator().manual_seed(1)
    a = torch.rand(1000, generator=g, dtype=torch.float64).to(dtype)
    vals = torch.randn(1000, 6, generator=g, dtype=torch.float64).to(dtype)
    a2 = a * a
    a3 = a2 * a
    a4 = a3 * a
    a5 = a4 * a
    w = [(a / 20.0) - (a2 / 24.0) - (a3 / 24.0) + (a4 / 24.0) - (a5 / 120.0),
         -(a / 2.0) + (2.0 * a2 / 3.0) - (a3 / 24.0) - (a4 / 6.0) + (a5 / 24.0),
         1.0 - (a / 3.0) - (5.0 * a2 / 4.0) + (5.0 * a3 / 12.0) + (a4 / 4.0) - (a5 / 12.0),
         a + (2.0 * a2 / 3.0) - (7.0 * a3 / 12.0) - (a4 / 6.0) + (a5 / 12.0),
         -(a / 4.0) - (a2 / 24.0) + (7.0 * a3 / 24.0) + (a4 / 24.0) - (a5 / 24.0),
         (a / 30.0) - (a3 / 24.0) + (a5 / 120.0)]
    want = w[0] * vals[:, 0]
    for k in range(1, 6):
        want = want + w[k] * vals[:, k]
    assert torch.equal(v2.lagrange5_interp_sum(a.cuda(), vals.cuda()).cpu(), want)
    nodes = NODES.to(dtype)
    pw = []
    for j in range(6):
        wj = torch.ones_like(a)
        for m in range(6):
            if m != j:
                wj = wj * (a - nodes[m]) / (nodes[j] - nodes[m])
        pw.append(wj)
    assert torch.equal(v2.get_lagrange5_weights(a.cuda()).cpu(), torch.stack(pw, -1))


# ---- advection: analytic shifts of a Gaussian (FP32, 16^4, L = 2 pi, V = 4) --------
N, LBOX, VMAX = 16, 2 * math.pi, 4.0


@pytest.fixture(scope="module")
def grid32(v2):
    return v2.Grid.create(N, N, N, N, LBOX, LBOX, VMAX, VMAX, dtype=torch.float32)


def _gauss(u, c, s):
    return torch.exp(-0.5 * ((u - c) / s) ** 2)


def _periodic_gauss(u, c, s, L):
    return sum(_gauss(u + m * L, c, s) for m in (-1, 0, 1))


@pytest.mark.parametrize("axis", [0, 1])
@pytest.mark.parametrize("cells", [0.3, 1.0, 2.5, 4.2])
def test_periodic_shift_analytic(v2, grid32, axis, cells):
    g = grid32
    coord = (g.x if axis == 0 else g.y).double().cpu()
    d = (g.dx if axis == 0 else g.dy)
    dt = 0.1
    v = cells * d / dt
    shape = [1, 1, 1, 1]
    shape[axis] = N
    s = LBOX / 10
    f = _periodic_gauss(coord, LBOX / 2, s, LBOX).view(shape).expand(N, N, N, N).float().contiguous().cuda()
    want = _periodic_gauss(coord, LBOX / 2 + v * dt, s, LBOX).view(shape).expand(N, N, N, N).float()
    # one velocity per column of the other velocity axis (all equal here)
    vel = torch.full((N,), v, dtype=torch.float32, device="cuda").view(*([1] * (2 - axis)), N, *([1] * axis))
    outs = {"advect_1d": v2.advect_1d(f, vel, axis, dt, d, True, stencil_offsets=g.stencil_offsets),
            "advect_1d_matrix_diag": v2.advect_1d_matrix_diag(f, vel, axis, dt, d, True,
                                                               stencil_offsets=g.stencil_offsets)}
    blocks, W = v2.precompute_x_drift(torch.full((N,), v), dt, d, torch.float32)
    outs["advect_x_static"] = v2.advect_x_static(f, W.cuda(), blocks, g.stencil_offsets, axis)
    for name, out in outs.items():
        err = (out.cpu() - want).abs().max().item()
        assert err < 1e-2, (name, err)


@pytest.mark.parametrize("axis", [2, 3])
@pytest.mark.parametrize("cells", [0.3, 1.0, 2.5, 4.2])
def test_dirichlet_shift_analytic(v2, grid32, axis, cells):
    g = grid32
    vgrid = (g.vx if axis == 2 else g.vy).double().cpu()
    dv = g.dvx if axis == 2 else g.dvy
    dt = 0.1
    E = cells * dv / dt
    shape = [1, 1, 1, 1]
    shape[axis] = N
    s = 0.8
    f = _gauss(vgrid, -0.5, s).view(shape).expand(N, N, N, N).float().contiguous().cuda()
    want = _gauss(vgrid, -0.5 + E * dt, s).view(shape).expand(N, N, N, N).float()
    field = torch.full((N, N), E, dtype=torch.float32, device="cuda")  # E(x, y), as the step passes it
    outs = {"advect_1d": v2.advect_1d(f, field[:, :, None], axis, dt, dv, False, stencil_offsets=g.stencil_offsets),
            "advect_1d_matrix_diag": v2.advect_1d_matrix_diag(f, field[:, :, None], axis, dt, dv, False,
                                                               stencil_offsets=g.stencil_offsets),
            "advect_v_static": v2.advect_v_static(f, field, dt, dv, 5, g.stencil_offsets, axis)}
    for name, out in outs.items():
        err = (out.cpu() - want).abs().max().item()
        assert err < 1e-2, (name, err)


# ---- advection: the kernels agree with the per-element sweep (FP64) ------------------
@pytest.fixture(scope="module")
def grid64(v2):
    return v2.Grid.create(16, 12, 10, 14, LBOX, 1.5 * LBOX, VMAX, 3.0, dtype=torch.float64)


@pytest.mark.parametrize("axis", [0, 1, 2, 3])
def test_matrix_diag_equals_gather(v2, grid64, axis):
    g = grid64
    f = torch.rand((16, 12, 10, 14), generator=torch.Generator().manual_seed(0), dtype=torch.float64).cuda()
    if axis < 2:
        vel = g.vx[None, :, None] if axis == 0 else g.vy[None, None, :]
        d, periodic = (g.dx if axis == 0 else g.dy), True
    else:
        E = torch.randn((16, 12), generator=torch.Generator().manual_seed(1), dtype=torch.float64).cuda()
        vel = E[:, :, None]
        d, periodic = (g.dvx if axis == 2 else g.dvy), False
    a = v2.advect_1d(f, vel, axis, 0.1, d, periodic, stencil_offsets=g.stencil_offsets)
    b = v2.advect_1d_matrix_diag(f, vel, axis, 0.1, d, periodic, stencil_offsets=g.stencil_offsets)
    assert (a - b).abs().max().item() < 1e-10


@pytest.mark.parametrize("fac", [0.3, 1.0, 2.5, 4.2, 6.0])
def test_static_kernels_equal_gather(v2, grid64, fac):
    g = grid64
    f = torch.rand((16, 12, 10, 14), generator=torch.Generator().manual_seed(2), dtype=torch.float64).cuda()
    dt = fac * g.dx / VMAX
    blocks, W = v2.precompute_x_drift(g.vx.cpu(), dt, g.dx, torch.float64)
    a = v2.advect_x_static(f, W.cuda(), blocks, g.stencil_offsets, 0)
    b = v2.advect_1d(f, g.vx[None, :, None], 0, dt, g.dx, True, stencil_offsets=g.stencil_offsets)
    assert (a - b).abs().max().item() < 1e-10
    E = torch.full((16, 12), fac * g.dvx / 0.1, dtype=torch.float64, device="cuda")
    S = int(math.ceil(fac)) + 1
    c = v2.advect_v_static(f, E, 0.1, g.dvx, S, g.stencil_offsets, 2)
    d = v2.advect_1d(f, E[:, :, None], 2, 0.1, g.dvx, False, stencil_offsets=g.stencil_offsets)
    assert (c - d).abs().max().item() < 1e-10


# ---- full steps: solvers 1 and 2 against solver 0 (FP64, Landau eps = 0.05) -----------
@pytest.mark.parametrize("physics", [True, False])
def test_steps_agree_across_solvers(v2, physics):
    g = v2.Grid.create(16, 16, 16, 16, 4 * math.pi, 4 * math.pi, 6.0, 6.0, dtype=torch.float64)
    x, y = g.x.cpu(), g.y.cpu()
    vx, vy = g.vx.cpu(), g.vy.cpu()
    sp = 1 + 0.05 * (torch.cos(0.5 * x)[:, None] + torch.cos(0.5 * y)[None, :])
    fv = torch.exp(-0.5 * (vx[:, None] ** 2 + vy[None, :] ** 2)) / (2 * math.pi)
    f = (sp[:, :, None, None] * fv[None, None]).contiguous().cuda()
    f0 = fv.cuda()
    args = (g.x, g.y, g.vx, g.vy, g.kx, g.ky, g.inv_ksq, g.x_indices, g.y_indices, g.vx_indices, g.vy_indices,
            g.stencil_offsets, g.dx, g.dy, g.dvx, g.dvy, g.Nx, g.Ny, physics)
    ref = v2.vlasov_step_impl(f, f0, 0.1, *args)
    rho = v2.compute_rho(f, g.dvx, g.dvy)
    Ex, Ey, _, _ = v2.compute_poisson_real(rho, g.kx, g.ky, g.inv_ksq)
    assert max(v2.check_v_window(Ex, 0.1, g.dvx, 1), v2.check_v_window(Ey, 0.1, g.dvy, 1)) < 1
    for step in (v2.vlasov_step_matrix_diag, v2.vlasov_step_gather_free):
        out = step(f, f0, 0.1, *args)
        for a, b in zip(out, ref):
            assert (a - b).abs().max().item() <= 1e-9 * max(b.abs().max().item(), 1.0)


# ---- Poisson: the complex and real-valued 1D1V paths agree -------------------------
def test_poisson1d_complex_and_real_paths(v1):
    g = v1.Grid.create(64, 48, 4 * math.pi, 5.0, dtype=torch.float64)
    x, v = g.x.cpu(), g.v.cpu()
    f = ((1 + 0.01 * torch.cos(0.5 * x))[:, None] * torch.exp(-0.5 * v[None, :] ** 2) / math.sqrt(2 * math.pi))
    f = f.contiguous().cuda()
    a = v1.solve_poisson(f, g.inv_kx, g.dv)
    b = v1.solve_poisson_real(f, g.inv_kx, g.inv_kx_sq, g.dv)
    for p, q in zip(a, b):
        np.testing.assert_allclose(p.cpu().numpy(), q.cpu().numpy(), atol=1e-12)
    # the single mode rho = eps cos(kx) gives E = (eps / k) sin(kx) (dE/dx = rho)
    np.testing.assert_allclose(b[0].cpu().numpy(), 0.01 / 0.5 * np.sin(0.5 * x.numpy()), atol=1e-5)


# ---- grid ------------------------------------------------------------------------------
def test_grid_properties(v2):
    g = v2.Grid.create(12, 10, 9, 7, 4 * math.pi, 3.0, 5.0, 2.0, dtype=torch.float64)
    assert g.dx == pytest.approx(4 * math.pi / 12) and g.dy == pytest.approx(3.0 / 10)
    assert g.dvx == pytest.approx(10.0 / 8) and g.dvy == pytest.approx(4.0 / 6)
    assert g.x[0].item() == 0.0 and g.x[-1].item() == pytest.approx(4 * math.pi - g.dx)
    assert g.vx[0].item() == -5.0 and g.vx[-1].item() == 5.0
    assert tuple(g.kx.shape) == (12, 1) and tuple(g.ky.shape) == (1, 6)
    assert g.inv_ksq[0, 0].item() == 0.0 and tuple(g.inv_ksq.shape) == (12, 6)
    assert g.x.is_cuda and g.stencil_offsets.tolist() == [-2, -1, 0, 1, 2, 3]
