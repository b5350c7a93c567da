"""Pins the CPU oracle against golden outputs of the reference solver itself
(tests/golden/make_golden.py). CPU only."""
import math

import numpy as np
import pytest

from oracle import core as O

SMALL = dict(Nx=8, Ny=6, Nvx=10, Nvy=12, Lx=2.0 * math.pi, Ly=3.0, Vx_max=4.0, Vy_max=5.0)
STEP = dict(Nx=8, Ny=8, Nvx=16, Nvy=12, Lx=4.0 * math.pi, Ly=4.0 * math.pi, Vx_max=6.0, Vy_max=5.0)
DT = {"f64": np.float64, "f32": np.float32}
# FP64: round-off; FP32: a few ulps of O(1) data (the reference sums with
# torch's vectorised kernels, the oracle with scalar C loops)
TOL = {"f64": 1e-13, "f32": 2e-6}


def seeded(seed, shape, dt):
    return np.random.default_rng(seed).random(shape).astype(DT[dt])


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_lagrange_weights_bitwise(golden, dt):
    t = golden("tables")
    a = t["alpha"].astype(DT[dt])
    w = O.lagrange5_weights(a)
    np.testing.assert_array_equal(w, t[f"lag5_{dt}"])


@pytest.mark.parametrize("tag", ["c1", "c2", "c3", "ref128", "oned4096"])
@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_drift_tables_bitwise(golden, tag, dt):
    """Integer shifts and weights equal precompute_x_drift bit for bit."""
    t = golden("tables")
    n, vmax, dx, half_dt = t[f"{tag}_{dt}_meta"]
    s, W = O.precompute_drift(t[f"{tag}_{dt}_v"], half_dt, dx, DT[dt])
    np.testing.assert_array_equal(s, t[f"{tag}_{dt}_shift"])
    np.testing.assert_array_equal(W, t[f"{tag}_{dt}_W"])


@pytest.mark.parametrize("dt", ["f64", "f32"])
@pytest.mark.parametrize("axis", [0, 1])
@pytest.mark.parametrize("fac", [0.3, 2.7, 6.0])
def test_drift_static(golden, dt, axis, fac):
    g = O.make_grid2d(**SMALL, dtype=DT[dt])
    G = golden("sweeps2d")
    f = seeded(11, (g.Nx, g.Ny, g.Nvx, g.Nvy), dt)
    key = f"drift_{dt}_a{axis}_{fac}"
    dx = g.dx if axis == 0 else g.dy
    s, W = O.precompute_drift(G[key + "_v"], 0.1, dx, DT[dt])
    out = O.drift_static(f, s, W, axis=axis, vel_axis=axis + 2)
    # same weights, same order, multiply-then-add: bit-exact
    np.testing.assert_array_equal(out, G[key])


@pytest.mark.parametrize("dt", ["f64", "f32"])
@pytest.mark.parametrize("axis", [2, 3])
@pytest.mark.parametrize("fac", [0.3, 1.5, 4.2])
def test_kick_static(golden, dt, axis, fac):
    g = O.make_grid2d(**SMALL, dtype=DT[dt])
    G = golden("sweeps2d")
    f = seeded(11, (g.Nx, g.Ny, g.Nvx, g.Nvy), dt)
    key = f"kick_{dt}_a{axis}_{fac}"
    dv = g.dvx if axis == 2 else g.dvy
    E = G[key + "_E"]
    out = O.kick_static(f, E, 0.1, dv, axis, window=int(G[key + "_S"]))
    np.testing.assert_array_equal(out, G[key])
    # the exact (unwindowed) kick equals the windowed one whenever S covers |d|
    np.testing.assert_array_equal(O.kick_static(f, E, 0.1, dv, axis, window=-1), G[key])
    # S = 1 drops the taps outside [-3, 3] once |E dt/dv| >= 1
    np.testing.assert_array_equal(O.kick_static(f, E, 0.1, dv, axis, window=1), G[key + "_S1"])


@pytest.mark.parametrize("dt", ["f64", "f32"])
@pytest.mark.parametrize("axis", [0, 1, 2, 3])
def test_gather_and_diag_sweeps(golden, dt, axis):
    g = O.make_grid2d(**SMALL, dtype=DT[dt])
    G = golden("sweeps2d")
    f = seeded(11, (g.Nx, g.Ny, g.Nvx, g.Nvy), dt)
    T = DT[dt]
    vel = {
        0: g.vx[None, :, None] * T(1.7),
        1: g.vy[None, None, :] * T(-2.3),
        2: np.linspace(-3, 3, g.Nx * g.Ny).astype(T).reshape(g.Nx, g.Ny)[:, :, None],
        3: np.linspace(4, -4, g.Nx * g.Ny).astype(T).reshape(g.Nx, g.Ny)[:, :, None],
    }
    import torch  # the reference builds these velocities with torch.linspace

    td = torch.float64 if dt == "f64" else torch.float32
    vel[2] = torch.linspace(-3, 3, g.Nx * g.Ny, dtype=td).reshape(g.Nx, g.Ny)[:, :, None].numpy()
    vel[3] = torch.linspace(4, -4, g.Nx * g.Ny, dtype=td).reshape(g.Nx, g.Ny)[:, :, None].numpy()
    hx = {0: g.dx, 1: g.dy, 2: g.dvx, 3: g.dvy}
    out = O.advect_gather(f, vel[axis], axis, 0.1, hx[axis], periodic=axis < 2)
    np.testing.assert_array_equal(out, G[f"gather_{dt}_a{axis}"])
    # the roll/diag solver is the same interpolant with per-line weights
    np.testing.assert_allclose(out, G[f"diag_{dt}_a{axis}"], rtol=0, atol=TOL[dt] * 10)


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_rho(golden, dt):
    g = O.make_grid2d(**SMALL, dtype=DT[dt])
    f = seeded(11, (g.Nx, g.Ny, g.Nvx, g.Nvy), dt)
    rho = O.compute_rho(f, g.dvx, g.dvy)
    np.testing.assert_allclose(rho, golden("sweeps2d")[f"rho_{dt}"], rtol=TOL[dt], atol=0)


@pytest.mark.parametrize("shape", [(16, 12), (15, 9), (9, 15), (8, 10)])
@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_poisson(golden, shape, dt):
    nx, ny = shape
    g = O.make_grid2d(nx, ny, 4, 4, 4.0 * math.pi, 3.3, 1.0, 1.0, dtype=DT[dt])
    rho = (1.0 + 0.01 * np.random.default_rng(nx * 100 + ny).standard_normal((nx, ny))).astype(DT[dt])
    Ex, Ey, drho, phi = O.compute_poisson_real(rho, g.kx, g.ky, g.inv_ksq)
    G = golden("poisson2d")
    key = f"p{nx}x{ny}_{dt}"
    scale = {"f64": 1e-14, "f32": 1e-6}[dt]
    for name, v in (("Ex", Ex), ("Ey", Ey), ("drho", drho), ("phi", phi)):
        ref = G[f"{key}_{name}"]
        np.testing.assert_allclose(v, ref, rtol=0, atol=scale * max(1.0, np.abs(ref).max()), err_msg=name)


@pytest.mark.parametrize("phys", [True, False])
def test_steps_solver2_and_0(golden, phys):
    g = O.make_grid2d(**STEP, dtype=np.float64)
    G = golden("steps2d")
    f0 = O.landau_2d(g, 0.05, 0.5)
    tag = "phys" if phys else "free"
    st = O.Stepper2D(g, 0.1, window=1)
    f = f0
    for i in range(3):
        r = st.step(f, phys)
        f = r.f
        np.testing.assert_allclose(r.drho, G[f"s2_{tag}_n{i + 1}_drho"], rtol=0, atol=1e-14)
        np.testing.assert_allclose(r.phi, G[f"s2_{tag}_n{i + 1}_phi"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(f, G[f"s2_{tag}_f"], rtol=0, atol=1e-15)
    # solver 0 (per-element departure) and solver 1 (roll/diag) agree with
    # solver 2 to round-off, in the oracle as in the reference
    f = f0
    for i in range(3):
        r = O.step_gather_2d(f, g, 0.1, phys)
        f = r.f
    np.testing.assert_allclose(f, G[f"s0_{tag}_f"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(G[f"s1_{tag}_f"], G[f"s0_{tag}_f"], rtol=0, atol=1e-12)


def test_history_c1(golden):
    """Configuration C1 (Landau, 32^4, FP64, 100 steps): the oracle's field
    energy history equals the reference's to 1e-10 relative."""
    H = golden("history_c1")
    g = O.make_grid2d(32, 32, 32, 32, 4 * math.pi, 4 * math.pi, 6.0, 6.0, dtype=np.float64)
    st = O.Stepper2D(g, 0.1, window=1)
    f = O.landau_2d(g, 0.01, 0.5)
    we = []
    for i in range(100):
        r = st.step(f)
        f = r.f
        we.append(O.field_energy_2d(r.Ex, r.Ey, g.dx, g.dy))
        if (i + 1) % 25 == 0:
            np.testing.assert_allclose(r.drho, H[f"drho_{i + 1}"], rtol=0, atol=1e-14)
    we = np.array(we)
    rel = np.abs(we - H["W_E"]) / np.abs(H["W_E"])
    assert rel.max() < 1e-10, rel.max()


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_oned_sweeps_and_steps(golden, dt):
    G = golden("oned")
    g = O.make_grid1d(24, 20, 4.0 * math.pi, 5.0, dtype=DT[dt])
    f = seeded(5, (24, 20), dt)
    for fac in (0.4, 3.3):
        s, W = O.precompute_drift(G[f"drift_{dt}_{fac}_v"], 0.1, g.dx, DT[dt])
        np.testing.assert_array_equal(O.drift_static(f, s, W, 0, 1), G[f"drift_{dt}_{fac}"])
    for fac in (0.3, 2.2):
        E = G[f"kick_{dt}_{fac}_E"]
        np.testing.assert_array_equal(O.kick_static(f, E, 0.1, g.dv, 1, window=-1), G[f"kick_{dt}_{fac}"])
    T = DT[dt]
    np.testing.assert_array_equal(
        O.advect_gather(f, g.v * T(1.3), 0, 0.1, g.dx, periodic=True), G[f"gx_{dt}"])
    import torch

    Ev = torch.linspace(-2, 2, 24, dtype=torch.float64 if dt == "f64" else torch.float32).numpy()
    np.testing.assert_array_equal(O.advect_gather_rows(f, Ev, 0.1, g.dv, periodic=False), G[f"gv_{dt}"])
    tol = {"f64": 1e-15, "f32": 6e-7}[dt]  # FP32 sums: a few ulps of rho ~ 1
    x = np.asarray(g.x)
    fl = ((1.0 + 0.01 * np.cos(2 * np.pi / g.L * x))[:, None] * np.exp(-0.5 * np.asarray(g.v) ** 2)[None, :]
          / math.sqrt(2 * math.pi)).astype(T)
    # the reference builds this IC in the run dtype; compare the Poisson on its own input
    import torch as _t

    tx = _t.from_numpy(np.asarray(g.x))
    tv = _t.from_numpy(np.asarray(g.v))
    fl = ((1.0 + 0.01 * _t.cos(2 * _t.pi / g.L * tx))[:, None] * _t.exp(-0.5 * tv ** 2)[None, :]
          / math.sqrt(2 * math.pi)).numpy().astype(T)
    E, rho, phi = O.solve_poisson_1d(fl, g.inv_kx, g.inv_kx_sq, g.dv)
    np.testing.assert_allclose(E, G[f"pois_{dt}_E"], rtol=0, atol=tol)
    np.testing.assert_allclose(rho, G[f"pois_{dt}_rho"], rtol=0, atol=tol)
    np.testing.assert_allclose(phi, G[f"pois_{dt}_phi"], rtol=0, atol=tol * 10)
    st = O.Stepper1D(g, 0.1, window=1)
    fs, f0s = fl, fl
    for i in range(3):
        r = st.step(fs)
        fs = r.f
        np.testing.assert_allclose(r.drho, G[f"s2_{dt}_n{i + 1}_rho"], rtol=0, atol=tol)
        r0 = O.step_gather_1d(f0s, g, 0.1)
        f0s = r0.f
        np.testing.assert_allclose(r0.drho, G[f"s0_{dt}_n{i + 1}_rho"], rtol=0, atol=tol)
    np.testing.assert_allclose(fs, G[f"s2_{dt}_f"], rtol=0, atol=tol)
    np.testing.assert_allclose(f0s, G[f"s0_{dt}_f"], rtol=0, atol=tol)


def test_history_oned_landau(golden):
    H = golden("history_oned_landau")
    nx, nv, L, vmax, eps, dt, steps = H["params"]
    g = O.make_grid1d(int(nx), int(nv), L, vmax, dtype=np.float64)
    st = O.Stepper1D(g, dt, window=1)
    f = O.landau_1d(g, eps, 2 * np.pi / L)
    for i in range(int(steps)):
        r = st.step(f)
        f = r.f
        np.testing.assert_allclose(r.drho, H["rho"][i], rtol=0, atol=1e-14)
