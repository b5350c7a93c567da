"""Parity of the field solves and of whole Strang steps with the CPU oracle,
and of multi-step histories with the reference's own runs (golden files)."""
import importlib
import math

import numpy as np
import pytest
import torch

from oracle import core as O

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("shape", [(16, 12), (15, 9), (9, 15), (8, 10), (128, 128), (24, 48), (1, 6), (7, 5)])
def test_poisson2d(vp, shape):
    nx, ny = shape
    g = O.make_grid2d(nx, ny, 4, 4, 4.0 * math.pi, 3.3, 1.0, 1.0, dtype=np.float64)
    rho = 1.0 + 0.01 * np.random.default_rng(nx * 100 + ny).standard_normal((nx, ny))
    Ex, Ey, drho, phi = O.compute_poisson_real(rho, g.kx, g.ky, g.inv_ksq)
    kx, ky, inv = vp.ops.spectral_2d(nx, ny, 4.0 * math.pi, 3.3, "cuda")
    ex, ey, dr, ph, en = vp.ops.poisson2d(dev(rho), kx, ky, inv, g.dx, g.dy, want_energy=True)
    for got, want in ((ex, Ex), (ey, Ey), (dr, drho), (ph, phi)):
        scale = max(np.abs(want).max(), 1e-300)
        assert np.abs(got.cpu().numpy() - want).max() <= 1e-13 * scale
    we = 0.5 * np.sum(Ex ** 2 + Ey ** 2) * g.dx * g.dy
    assert abs(float(en[0]) - we) <= 1e-12 * we
    assert abs(float(en[1]) - rho.sum() * g.dx * g.dy) <= 1e-13 * rho.sum() * g.dx * g.dy


@pytest.mark.parametrize("mode", [1, 2, 3])
def test_poisson2d_analytic(vp, mode):
    """The reference's test_poisson.py check: single cos.cos mode, analytic
    phi, Ex, Ey to 1e-5 (here to 1e-12 in FP64)."""
    nx = ny = 16
    L = 2.0 * 3.14159265358979
    g = O.make_grid2d(nx, ny, 16, 16, L, L, 4.0, 4.0, dtype=np.float64)
    k0 = mode * 2.0 * np.pi / L
    x, y = g.x[:, None], g.y[None, :]
    pert = 0.01 * np.cos(k0 * x) * np.cos(k0 * y)
    kx, ky, inv = vp.ops.spectral_2d(nx, ny, L, L, "cuda")
    ex, ey, dr, ph = vp.ops.poisson2d(dev(pert + 1.0), kx, ky, inv)
    phi_a = 0.01 / (2 * k0 * k0) * np.cos(k0 * x) * np.cos(k0 * y)
    ex_a = 0.01 * k0 / (2 * k0 * k0) * np.sin(k0 * x) * np.cos(k0 * y)
    ey_a = 0.01 * k0 / (2 * k0 * k0) * np.cos(k0 * x) * np.sin(k0 * y)
    np.testing.assert_allclose(ph.cpu().numpy(), phi_a, atol=1e-12)
    np.testing.assert_allclose(ex.cpu().numpy(), ex_a, atol=1e-12)
    np.testing.assert_allclose(ey.cpu().numpy(), ey_a, atol=1e-12)


@pytest.mark.parametrize("nx", [2, 4, 8, 16, 32, 64, 128, 256, 512, 2048, 4096, 8192, 24, 48, 1000])
def test_poisson1d(vp, nx):
    L = 4.0 * math.pi
    g = O.make_grid1d(nx, 16, L, 5.0, dtype=np.float64)
    n = 1.0 + 0.01 * np.random.default_rng(nx).standard_normal(nx)
    rk = np.fft.rfft(n - 1.0)
    E_ref = np.fft.irfft((rk.imag * g.inv_kx) + 1j * (-rk.real * g.inv_kx), n=nx)
    phi_ref = np.fft.irfft((rk.real * g.inv_kx_sq) + 1j * (rk.imag * g.inv_kx_sq), n=nx)
    inv, inv2 = vp.ops.spectral_1d(nx, L, "cuda")
    e, rho, phi, en = vp.ops.poisson1d(dev(n), inv, inv2, g.dx, want_energy=True)
    assert np.abs(e.cpu().numpy() - E_ref).max() <= 1e-12 * np.abs(E_ref).max()
    assert np.abs(phi.cpu().numpy() - phi_ref).max() <= 1e-12 * np.abs(phi_ref).max()
    np.testing.assert_allclose(rho.cpu().numpy(), n - 1.0, rtol=0, atol=0)
    we = 0.5 * np.sum(E_ref ** 2) * g.dx
    assert abs(float(en[0]) - we) <= 1e-11 * we


SHAPES = [(8, 8, 16, 12), (16, 16, 16, 16), (12, 10, 24, 20), (9, 7, 10, 6), (8, 8, 32, 128)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("physics", [True, False])
@pytest.mark.parametrize("window", [-1, 1])
def test_step2d_fp64(vp, shape, physics, window):
    Nx, Ny, Nvx, Nvy = shape
    Lx, Ly = 4.0 * math.pi, 4.0 * math.pi
    g = O.make_grid2d(Nx, Ny, Nvx, Nvy, Lx, Ly, 6.0, 5.0, dtype=np.float64)
    f = O.landau_2d(g, 0.3, 0.5)  # strong field: |E dt/dv| exceeds 1 somewhere
    st_o = O.Stepper2D(g, 0.5, window=window)
    st = vp.Stepper2D(Nx, Ny, Nvx, Nvy, Lx, Ly, 6.0, 5.0, 0.5, dtype=torch.float64, physics_mode=physics,
                      window=window)
    fd = dev(f)
    for i in range(3):
        f_prev = f
        r = st_o.step(f, physics)
        f = r.f
        fd = st.step(fd)
        torch.cuda.synchronize()
        err = np.abs(fd.cpu().numpy() - f).max() / np.abs(f).max()
        assert err < 1e-12, (i, err)
        np.testing.assert_allclose(st.drho.cpu().numpy(), r.drho, rtol=0, atol=1e-13)
        np.testing.assert_allclose(st.phi.cpu().numpy(), r.phi, rtol=0, atol=1e-12)
    d = st.diag.cpu().numpy()
    if physics:
        we = O.field_energy_2d(r.Ex, r.Ey, g.dx, g.dy)
        assert abs(d[0] - we) <= 1e-10 * we
        shift = max(np.abs(r.Ex).max() * 0.5 / g.dvx, np.abs(r.Ey).max() * 0.5 / g.dvy)
        assert abs(d[5] - shift) <= 1e-12 * shift
    # mid-step mass: the periodic drifts conserve the mass of the step's input
    m = O.moments_2d(f_prev, g)
    assert abs(d[1] - m["mass"]) <= 1e-10 * m["mass"]


def test_step2d_diag_moments(vp):
    """L2 and kinetic energy of f right after the kicks, against the oracle."""
    shape = (8, 8, 16, 12)
    g = O.make_grid2d(*shape, 4 * math.pi, 4 * math.pi, 6.0, 5.0, dtype=np.float64)
    f = O.landau_2d(g, 0.1, 0.5)
    st_o = O.Stepper2D(g, 0.2, window=-1)
    st = vp.Stepper2D(*shape, 4 * math.pi, 4 * math.pi, 6.0, 5.0, 0.2, dtype=torch.float64, diagnostics=2)
    # oracle: state right after the kicks of the first step
    a = st_o.drift_y(st_o.drift_x(f))
    Ex, Ey, _, _ = O.solve_poisson_real(a, g)
    k = O.kick_static(O.kick_static(a, Ex, 0.2, g.dvx, 2), Ey, 0.2, g.dvy, 3)
    st.step(dev(f))
    d = st.diag.cpu().numpy()
    mk, ma = O.moments_2d(k, g), O.moments_2d(a, g)
    assert abs(d[2] - mk["l2"]) <= 1e-12 * mk["l2"]
    assert abs(d[3] - mk["kinetic"]) <= 1e-12 * mk["kinetic"]
    assert abs(d[4] - ma["kinetic"]) <= 1e-12 * ma["kinetic"]


@pytest.mark.parametrize("dtype,tol", [(torch.float32, 5e-6), (torch.bfloat16, 3e-2)])
def test_step2d_reduced_precision(vp, dtype, tol):
    shape = (16, 16, 32, 32)
    g = O.make_grid2d(*shape, 4 * math.pi, 4 * math.pi, 6.0, 6.0, dtype=np.float64)
    f = O.landau_2d(g, 0.05, 0.5)
    st_o = O.Stepper2D(g, 0.1, window=-1)
    st = vp.Stepper2D(*shape, 4 * math.pi, 4 * math.pi, 6.0, 6.0, 0.1, dtype=dtype)
    fd = dev(f).to(dtype)
    for _ in range(5):
        f = st_o.step(f).f
        fd = st.step(fd)
    err = np.abs(fd.double().cpu().numpy() - f).max() / np.abs(f).max()
    assert err < tol, err


def test_history_c1_against_reference(vp, golden):
    """C1 (Landau 32^4, FP64, 100 steps): the field-energy history of the
    library equals the reference solver's own (golden) to 1e-10 relative."""
    H = golden("history_c1")
    n = 32
    L = 4 * math.pi
    g = O.make_grid2d(n, n, n, n, L, L, 6.0, 6.0, dtype=np.float64)
    st = vp.Stepper2D(n, n, n, n, L, L, 6.0, 6.0, 0.1, dtype=torch.float64, window=1)
    f = dev(O.landau_2d(g, 0.01, 0.5))
    hist = torch.zeros((100, 8), dtype=torch.float64, device="cuda")
    f = st.run(f, 100, history=hist, graph=True)
    we = hist[:, 0].cpu().numpy()
    rel = np.abs(we - H["W_E"]) / np.abs(H["W_E"])
    assert rel.max() < 1e-10, rel.max()
    # the Landau damping rate, as the reference's post-processing checks it
    R = importlib.import_module("jax-pytorch-vlasov_b200.rates")
    t = 0.1 * np.arange(1, 101)
    rate = R.damping_rate(t, we)
    assert abs(rate - R.damping_rate(t, H["W_E"])) <= 1e-6 * rate
    assert abs(rate - R.LANDAU_RATE_K05) <= 0.02 * R.LANDAU_RATE_K05
    mass = hist[:, 1].cpu().numpy()
    np.testing.assert_allclose(mass, H["mass"], rtol=1e-12)
    np.testing.assert_allclose(st.drho.cpu().numpy(), H["drho_final"], rtol=0, atol=1e-13)


@pytest.mark.parametrize("shape", [(64, 48), (24, 20), (256, 128), (4096, 64)])
@pytest.mark.parametrize("physics", [True, False])
def test_step1d_fp64(vp, shape, physics):
    Nx, Nv = shape
    L = 4.0 * math.pi
    g = O.make_grid1d(Nx, Nv, L, 6.0, dtype=np.float64)
    f = O.landau_1d(g, 0.2, 0.5)
    so = O.Stepper1D(g, 0.3, window=-1)
    st = vp.Stepper1D(Nx, Nv, L, 6.0, 0.3, dtype=torch.float64, physics_mode=physics)
    fd = dev(f)
    for _ in range(3):
        r = so.step(f, physics)
        f = r.f
        fd = st.step(fd)
    err = np.abs(fd.cpu().numpy() - f).max() / np.abs(f).max()
    assert err < 1e-12, err
    np.testing.assert_allclose(st.rho.cpu().numpy(), r.drho, rtol=0, atol=1e-13)
    if physics:
        we = O.field_energy_1d(r.Ex, g.dx)
        assert abs(float(st.diag[0]) - we) <= 1e-10 * we
        # power-of-two Nx: the field solve writes the diagnostics itself
        d = st.diag.cpu().numpy()
        np.testing.assert_allclose(d[1], (r.drho + 1.0).sum() * g.dx, rtol=1e-12)
        assert np.isnan(d[2]) and np.isnan(d[3]) and np.isnan(d[4])
        np.testing.assert_allclose(d[5], np.abs(r.Ex).max() * 0.3 / g.dv, rtol=1e-12)
        assert d[6] == 0.0 and d[7] == 0.0


def test_history_oned_against_reference(vp, golden):
    H = golden("history_oned_landau")
    nx, nv, L, vmax, eps, dt, steps = H["params"]
    nx, nv, steps = int(nx), int(nv), int(steps)
    g = O.make_grid1d(nx, nv, L, vmax, dtype=np.float64)
    st = vp.Stepper1D(nx, nv, L, vmax, dt, dtype=torch.float64, window=1)
    f = dev(O.landau_1d(g, eps, 2 * np.pi / L))
    for i in range(steps):
        f = st.step(f)
        if i % 20 == 19 or i == steps - 1:
            np.testing.assert_allclose(st.rho.cpu().numpy(), H["rho"][i], rtol=0, atol=1e-13)


def test_graph_replay_matches_eager(vp):
    shape = (8, 8, 16, 16)
    g = O.make_grid2d(*shape, 4 * math.pi, 4 * math.pi, 6.0, 6.0, dtype=np.float64)
    f0 = dev(O.landau_2d(g, 0.05, 0.5)).float()
    a = vp.Stepper2D(*shape, 4 * math.pi, 4 * math.pi, 6.0, 6.0, 0.1, diagnostics=2)
    b = vp.Stepper2D(*shape, 4 * math.pi, 4 * math.pi, 6.0, 6.0, 0.1, diagnostics=2)
    ha = torch.zeros((23, 8), dtype=torch.float64, device="cuda")
    hb = torch.zeros_like(ha)
    fa = a.run(f0.clone(), 23, history=ha, graph=False)
    fb = b.run(f0.clone(), 23, history=hb, graph=True, graph_chunk=6)
    assert torch.equal(fa, fb)
    assert torch.equal(ha, hb)


@pytest.mark.parametrize("nx", [16384, 4600])
def test_poisson1d_beyond_one_block_is_rejected(vp, nx):
    """Power-of-two lengths above 8192 and other lengths above 4522 do not fit
    the one-block solvers: a clear error, no launch."""
    n = torch.ones(nx, dtype=torch.float64, device="cuda")
    inv, inv2 = vp.ops.spectral_1d(nx, 4.0 * math.pi, "cuda")
    with pytest.raises(vp._lib.VlasovError, match="too large|power-of-two"):
        vp.ops.poisson1d(n, inv, inv2)
