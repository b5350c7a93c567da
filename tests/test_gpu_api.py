"""The drop-in modules (reference function names and signatures) against the
reference's own golden outputs, and the Vlasov drivers."""
import importlib
import math
import os

import numpy as np
import pytest
import torch

from conftest import PACKAGE

pytestmark = pytest.mark.gpu

SMALL = dict(Nx=8, Ny=6, Nvx=10, Nvy=12, Lx=2.0 * math.pi, Ly=3.0, Vx_max=4.0, Vy_max=5.0)
STEP = dict(Nx=8, Ny=8, Nvx=16, Nvy=12, Lx=4.0 * math.pi, Ly=4.0 * math.pi, Vx_max=6.0, Vy_max=5.0)
TD = {"f64": torch.float64, "f32": torch.float32}


@pytest.fixture(scope="module")
def v2():
    return importlib.import_module(PACKAGE + ".vlasov2d2v")


@pytest.fixture(scope="module")
def v1():
    return importlib.import_module(PACKAGE + ".vlasov1d1v")


def seeded(seed, shape, dt):
    return torch.from_numpy(np.random.default_rng(seed).random(shape)).to(TD[dt]).cuda()


def close(got, want, rel):
    got = got.double().cpu().numpy()
    assert np.abs(got - want).max() <= rel * max(np.abs(want).max(), 1e-300)


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_sweeps_against_reference(v2, golden, dt):
    G = golden("sweeps2d")
    g = v2.Grid.create(**SMALL, dtype=TD[dt])
    f = seeded(11, (g.Nx, g.Ny, g.Nvx, g.Nvy), dt)
    rel = 1e-14 if dt == "f64" else 2e-6
    for axis in (0, 1):
        dx = g.dx if axis == 0 else g.dy
        for fac in (0.3, 2.7, 6.0):
            key = f"drift_{dt}_a{axis}_{fac}"
            v = torch.from_numpy(G[key + "_v"]).cuda()
            blocks, W = v2.precompute_x_drift(v, 0.1, dx, TD[dt])
            close(v2.advect_x_static(f, W, blocks, g.stencil_offsets, axis), G[key], rel)
    for axis in (2, 3):
        dv = g.dvx if axis == 2 else g.dvy
        for fac in (0.3, 1.5, 4.2):
            key = f"kick_{dt}_a{axis}_{fac}"
            E = torch.from_numpy(G[key + "_E"]).cuda()
            close(v2.advect_v_static(f, E, 0.1, dv, int(G[key + "_S"]), g.stencil_offsets, axis), G[key], rel)
            close(v2.advect_v_static(f, E, 0.1, dv, 1, g.stencil_offsets, axis), G[key + "_S1"], rel)
    vel = {
        0: g.vx[None, :, None] * 1.7,
        1: g.vy[None, None, :] * -2.3,
        2: torch.linspace(-3, 3, g.Nx * g.Ny, dtype=TD[dt]).reshape(g.Nx, g.Ny)[:, :, None].cuda(),
        3: torch.linspace(4, -4, g.Nx * g.Ny, dtype=TD[dt]).reshape(g.Nx, g.Ny)[:, :, None].cuda(),
    }
    hx = {0: g.dx, 1: g.dy, 2: g.dvx, 3: g.dvy}
    idx = {0: g.x_indices, 1: g.y_indices, 2: g.vx_indices, 3: g.vy_indices}
    for axis in range(4):
        got = v2.advect_1d(f, vel[axis], axis, 0.1, hx[axis], periodic=axis < 2, point_indices=idx[axis],
                           stencil_offsets=g.stencil_offsets)
        # per-element departure sweep: bit-identical to the reference
        np.testing.assert_array_equal(got.cpu().numpy(), G[f"gather_{dt}_a{axis}"])
        got = v2.advect_1d_matrix_diag(f, vel[axis], axis, 0.1, hx[axis], periodic=axis < 2,
                                       point_indices=idx[axis], stencil_offsets=g.stencil_offsets)
        close(got, G[f"diag_{dt}_a{axis}"], rel * 10)
    close(v2.compute_rho(f, g.dvx, g.dvy), G[f"rho_{dt}"], 1e-14 if dt == "f64" else 3e-7)


@pytest.mark.parametrize("shape", [(16, 12), (15, 9), (9, 15), (8, 10)])
def test_poisson_against_reference(v2, golden, shape):
    nx, ny = shape
    G = golden("poisson2d")
    g = v2.Grid.create(nx, ny, 4, 4, 4.0 * math.pi, 3.3, 1.0, 1.0, dtype=torch.float64)
    rho = torch.from_numpy(1.0 + 0.01 * np.random.default_rng(nx * 100 + ny).standard_normal((nx, ny))).cuda()
    Ex, Ey, drho, phi = v2.compute_poisson_real(rho, g.kx, g.ky, g.inv_ksq)
    for name, v in (("Ex", Ex), ("Ey", Ey), ("drho", drho), ("phi", phi)):
        close(v, G[f"p{nx}x{ny}_f64_{name}"], 1e-13)


def landau_ref(g, eps, k):
    """The golden script's initial condition, evaluated the same way."""
    x, y = g.x.cpu().double(), g.y.cpu().double()
    vx, vy = g.vx.cpu().double(), g.vy.cpu().double()
    sp = 1.0 + eps * (torch.cos(k * x)[:, None] + torch.cos(k * y)[None, :])
    fv = torch.exp(-0.5 * (vx[:, None] ** 2 + vy[None, :] ** 2)) / (2.0 * math.pi)
    return (sp[:, :, None, None] * fv[None, None]).cuda()


@pytest.mark.parametrize("phys", [True, False])
def test_steps_against_reference(v2, golden, phys):
    """Three steps of each solver's drop-in against the reference's own."""
    G = golden("steps2d")
    g = v2.Grid.create(**STEP, dtype=torch.float64)
    f0 = torch.zeros(g.Nvx, g.Nvy, dtype=torch.float64, device="cuda")
    args = (f0, 0.1, g.x, g.y, g.vx, g.vy, g.kx, g.ky, g.inv_ksq, g.x_indices, g.y_indices, g.vx_indices,
            g.vy_indices, g.stencil_offsets, g.dx, g.dy, g.dvx, g.dvy, g.Nx, g.Ny, phys)
    tag = "phys" if phys else "free"
    for s, fn in ((0, v2.vlasov_step_impl), (1, v2.vlasov_step_matrix_diag), (2, v2.vlasov_step_gather_free)):
        f = landau_ref(g, 0.05, 0.5)
        for i in range(3):
            f, drho, phi = fn(f, *args)
            close(drho, G[f"s{s}_{tag}_n{i + 1}_drho"], 1e-13)
            close(phi, G[f"s{s}_{tag}_n{i + 1}_phi"], 1e-12)
        close(f, G[f"s{s}_{tag}_f"], 1e-13)


def test_gather_free_impl_against_reference(v2, golden):
    G = golden("steps2d")
    g = v2.Grid.create(**STEP, dtype=torch.float64)
    bx, Wx = v2.precompute_x_drift(g.vx, 0.05, g.dx, torch.float64)
    by, Wy = v2.precompute_x_drift(g.vy, 0.05, g.dy, torch.float64)
    offs = v2.static_stencil_offsets(g.stencil_offsets)
    f = landau_ref(g, 0.05, 0.5)
    for _ in range(3):
        f, drho, phi = v2.vlasov_step_gather_free_impl(f, 0.1, Wx, Wy, bx, by, offs, g.kx, g.ky, g.inv_ksq,
                                                       g.dvx, g.dvy, g.Nx, g.Ny, True, 1)
    close(f, G["s2_phys_f"], 1e-13)


def test_vlasov_driver_2d(v2, tmp_path):
    sim = v2.Vlasov(Nx=16, Ny=16, Nvx=32, Nvy=32, Lx=4 * math.pi, Ly=4 * math.pi, nbiter=24, diag_steps=12,
                    dt=0.1, physics_mode=True, epsilon=0.05, dtype="float64", solver=2,
                    out_dir=str(tmp_path))
    state = sim.initialize()
    g = sim.grid
    # the reference's initial condition (vlasov2D2V.py:1328-1333)
    x, y = g.x[:, None, None, None], g.y[None, :, None, None]
    fM = (1.0 / math.sqrt(2 * math.pi)) * torch.exp(-0.5 * (g.vx[:, None] ** 2 + g.vy[None, :] ** 2))
    want = (1.0 + 0.05 * torch.cos(0.5 * x) * torch.cos(0.5 * y)) * fM[None, None]
    assert torch.allclose(state.variables.fn, want, atol=1e-12)
    f_init = state.variables.fn.clone()
    state = sim.run(state)
    assert state.step == 24 and abs(state.t - 2.4) < 1e-12
    assert sorted(os.listdir(tmp_path)) == ["field_000000.npz", "field_000012.npz", "field_000024.npz"]
    snap = np.load(tmp_path / "field_000024.npz")
    assert snap["f"].shape == (1, 16, 16, 32, 32) and int(snap["step"]) == 24
    # the driver's graph-captured loop equals plain drop-in steps
    f = f_init
    args = (state.variables.f0, 0.1, g.x, g.y, g.vx, g.vy, g.kx, g.ky, g.inv_ksq, g.x_indices, g.y_indices,
            g.vx_indices, g.vy_indices, g.stencil_offsets, g.dx, g.dy, g.dvx, g.dvy, g.Nx, g.Ny, True)
    for _ in range(24):
        f, _, _ = v2.vlasov_step_gather_free(f, *args)
    assert torch.equal(f, state.variables.fn)
    h = sim.history.cpu().numpy()
    assert h.shape == (24, 8) and np.isfinite(h[:, :2]).all()
    assert abs(h[-1, 1] / h[0, 1] - 1.0) < 1e-8  # mass


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_oned_against_reference(v1, golden, dt):
    G = golden("oned")
    g = v1.Grid.create(24, 20, 4.0 * math.pi, 5.0, dtype=TD[dt])
    f = seeded(5, (24, 20), dt)
    rel = 1e-14 if dt == "f64" else 2e-6
    for fac in (0.4, 3.3):
        v = torch.from_numpy(G[f"drift_{dt}_{fac}_v"]).cuda()
        blocks, W = v1.precompute_x_drift(v, 0.1, g.dx, TD[dt])
        close(v1.advect_x_static(f, W, blocks, g.stencil_offsets), G[f"drift_{dt}_{fac}"], rel)
    for fac in (0.3, 2.2):
        E = torch.from_numpy(G[f"kick_{dt}_{fac}_E"]).cuda()
        close(v1.advect_v_static(f, E, 0.1, g.dv, 8, g.stencil_offsets), G[f"kick_{dt}_{fac}"], rel)
    # the gather sweep on a transposed view, as the reference's vlasov_step calls it
    got = v1.advect_1d_vectorized(f.T, g.v * 1.3, 0.1, g.x_indices, g.x_batch_offsets, g.stencil_offsets, g.dx,
                                  periodic=True).T
    np.testing.assert_array_equal(got.cpu().numpy(), G[f"gx_{dt}"])
    Ev = torch.linspace(-2, 2, 24, dtype=TD[dt]).cuda()
    got = v1.advect_1d_vectorized(f, Ev, 0.1, g.v_indices, g.v_batch_offsets, g.stencil_offsets, g.dv,
                                  periodic=False)
    np.testing.assert_array_equal(got.cpu().numpy(), G[f"gv_{dt}"])
    x, v = g.x.cpu(), g.v.cpu()
    fl = ((1.0 + 0.01 * torch.cos(2 * torch.pi / g.L * x))[:, None] * torch.exp(-0.5 * v ** 2)[None, :]
          / math.sqrt(2 * math.pi)).to(TD[dt]).cuda()
    E, rho, phi = v1.solve_poisson_real(fl, g.inv_kx, g.inv_kx_sq, g.dv)
    tol = 1e-15 if dt == "f64" else 6e-7
    for name, val in (("E", E), ("rho", rho), ("phi", phi)):
        np.testing.assert_allclose(val.double().cpu().numpy(), G[f"pois_{dt}_{name}"], rtol=0,
                                   atol=tol * (10 if name == "phi" else 1))
    for s, fn in ((0, v1.vlasov_step), (2, v1.vlasov_step_gather_free)):
        fs = fl
        for i in range(3):
            fs, rho, phi = fn(fs, 0.1, g.v, g.inv_kx, g.inv_kx_sq, g.x_indices, g.v_indices, g.x_batch_offsets,
                              g.v_batch_offsets, g.stencil_offsets, g.dx, g.dv, g.V_max, True)
            np.testing.assert_allclose(rho.double().cpu().numpy(), G[f"s{s}_{dt}_n{i + 1}_rho"], rtol=0, atol=tol)
        np.testing.assert_allclose(fs.double().cpu().numpy(), G[f"s{s}_{dt}_f"], rtol=0,
                                   atol=tol if dt == "f64" else 2e-6)


def test_vlasov_driver_1d(v1, tmp_path):
    sim = v1.Vlasov(Nx=64, Nv=64, L=4 * math.pi, V_max=6.0, nbiter=20, diag_steps=10, dt=0.1, physics_mode=True,
                    epsilon=0.05, dtype="float64", solver=2, out_dir=str(tmp_path))
    state = sim.initialize()
    f = state.variables.fn.clone()
    state = sim.run(state)
    g = sim.grid
    for _ in range(20):
        f, _, _ = v1.vlasov_step_gather_free(f, 0.1, g.v, g.inv_kx, g.inv_kx_sq, g.x_indices, g.v_indices,
                                             g.x_batch_offsets, g.v_batch_offsets, g.stencil_offsets, g.dx, g.dv,
                                             g.V_max, True)
    assert torch.equal(f, state.variables.fn)
    assert sorted(os.listdir(tmp_path)) == ["field_000000.npz", "field_000010.npz", "field_000020.npz"]


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_fused_step_returns_fresh_fields(v1, v2, dt):
    """rho and phi returned by one fused step stay as they were after the
    next call (the reference computes new tensors each call)."""
    g = v2.Grid.create(**STEP, dtype=TD[dt])
    f = seeded(3, (g.Nx, g.Ny, g.Nvx, g.Nvy), dt)
    f0 = torch.zeros((g.Nvx, g.Nvy), dtype=TD[dt], device="cuda")
    args = (0.1, g.x, g.y, g.vx, g.vy, g.kx, g.ky, g.inv_ksq, g.x_indices, g.y_indices, g.vx_indices,
            g.vy_indices, g.stencil_offsets, g.dx, g.dy, g.dvx, g.dvy, g.Nx, g.Ny, True)
    f1, rho1, phi1 = v2.vlasov_step_gather_free(f, f0, *args)
    keep = rho1.clone(), phi1.clone()
    f2, rho2, phi2 = v2.vlasov_step_gather_free(f1, f0, *args)
    assert rho1.data_ptr() != rho2.data_ptr() and phi1.data_ptr() != phi2.data_ptr()
    assert torch.equal(rho1, keep[0]) and torch.equal(phi1, keep[1])
    assert not torch.equal(rho1, rho2)
    g1 = v1.Grid.create(24, 20, 4.0 * math.pi, 5.0, dtype=TD[dt])
    fl = seeded(4, (24, 20), dt)
    a1 = (0.1, g1.v, g1.inv_kx, g1.inv_kx_sq, g1.x_indices, g1.v_indices, g1.x_batch_offsets, g1.v_batch_offsets,
          g1.stencil_offsets, g1.dx, g1.dv, g1.V_max, True)
    s1, r1, p1 = v1.vlasov_step_gather_free(fl, *a1)
    keep = r1.clone(), p1.clone()
    s2, r2, p2 = v1.vlasov_step_gather_free(s1, *a1)
    assert r1.data_ptr() != r2.data_ptr() and p1.data_ptr() != p2.data_ptr()
    assert torch.equal(r1, keep[0]) and torch.equal(p1, keep[1])


@pytest.mark.parametrize("dt", [torch.float64, torch.float32, torch.bfloat16])
@pytest.mark.parametrize("shape", [((8, 6), (10, 12)), ((33,), (17,)), ((4, 4), (3, 5)), ((0, 3), (4, 4))])
def test_init_product(vp, dt, shape):
    """vp_init_product: the same bits as torch's broadcast product rounded
    by .to(dtype), vectorised (v a multiple of 4) and scalar paths."""
    g = np.random.default_rng(9)
    space = torch.from_numpy(1.0 + 0.1 * g.standard_normal(shape[0])).cuda()
    vel = torch.from_numpy(np.exp(-g.random(shape[1]) * 3)).cuda()
    got = vp.ops.init_product(space, vel, dt)
    want = (space.reshape(space.shape + (1,) * vel.dim()) * vel).to(dt)
    assert got.shape == want.shape and torch.equal(got, want)


def test_initialize_matches_reference_formula(v1, v2):
    """The drivers' initial conditions through the IC kernel equal the
    reference's broadcast expressions (vlasov2D2V.py:1328-1333,
    vlasov1D1V.py:890-896) bit for bit."""
    for dt in ("float64", "float32"):
        sim = v2.Vlasov(Nx=8, Ny=12, Nvx=16, Nvy=20, nbiter=1, physics_mode=True, epsilon=0.05, dtype=dt,
                        write_snapshots=False)
        g = sim.grid
        x, y = g.x[:, None, None, None].double(), g.y[None, :, None, None].double()
        vx, vy = g.vx[:, None].double(), g.vy[None, :].double()
        f0 = (1.0 / math.sqrt(2.0 * math.pi)) * torch.exp(-0.5 * (vx ** 2 + vy ** 2))
        want = ((1.0 + 0.05 * torch.cos(2 * math.pi / g.Lx * x) * torch.cos(2 * math.pi / g.Ly * y)) * f0[None, None])
        assert torch.equal(sim.initialize().variables.fn, want.to(sim.dtype))
        s1 = v1.Vlasov(Nx=24, Nv=20, nbiter=1, physics_mode=True, epsilon=0.05, dtype=dt, write_snapshots=False)
        h = s1.grid
        maxw = (1.0 / math.sqrt(2.0 * math.pi)) * torch.exp(-0.5 * h.v.double()[None, :] ** 2)
        want1 = (1.0 + 0.05 * torch.cos(2.0 * math.pi / h.L * h.x.double()[:, None])) * maxw
        assert torch.equal(s1.initialize().variables.fn, want1.to(s1.dtype))
