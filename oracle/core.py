"""CPU oracle of the Vlasov-Poisson Strang step (2D2V and 1D1V).

TEST INFRASTRUCTURE ONLY. This module is the checker that the CUDA library is
compared against, and the CPU baseline that bench.py times; the product never
imports it. It restates the reference's PyTorch solver
(simulations/vlasov2d_2v/pytorch/src/vlasov2D2V.py,
simulations/vlasov1d_1v/pytorch/src/vlasov1D1V.py) in numpy plus a small C
library (vp_oracle.c, OpenMP) for the O(N^4) sweeps. Grid vectors come from
the same torch factory calls the reference uses (linspace, fftfreq), so both
sides see bit-identical coordinates.

Parity is pinned by tests/golden/*.npz, produced by running the reference
itself (tests/golden/make_golden.py).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

OFFSETS = (-2, -1, 0, 1, 2, 3)  # Grid.stencil_offsets, vlasov2D2V.py:169


def build() -> str:
    """Compile libvp_oracle.so in place (make) and return its path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "libvp_oracle.so")


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libvp_oracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P, I, D = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double
        for sfx in ("f32", "f64"):
            getattr(L, f"or_drift_static_{sfx}").argtypes = [P, P, I, I, I, I, I, P, P]
            getattr(L, f"or_kick_static_{sfx}").argtypes = [P, P, I, I, I, P, I, D, D, I]
            getattr(L, f"or_advect_gather_{sfx}").argtypes = [P, P, I, I, I, P, I, I, I, D, D, ctypes.c_int]
            getattr(L, f"or_rho_{sfx}").argtypes = [P, I, I, D, D, P]
            getattr(L, f"or_lagrange5_weights_{sfx}").argtypes = [P, I, P]
        L.or_num_threads.restype = ctypes.c_int
        L.or_set_num_threads.argtypes = [ctypes.c_int]
        _LIB = L
    return _LIB


def _sfx(dtype) -> str:
    dt = np.dtype(dtype)
    if dt == np.float64:
        return "f64"
    if dt == np.float32:
        return "f32"
    raise TypeError(f"oracle supports float32/float64, got {dt}")


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def num_threads() -> int:
    return lib().or_num_threads()


def set_num_threads(n: int) -> None:
    lib().or_set_num_threads(int(n))


# --------------------------------------------------------------------------
# grids
# --------------------------------------------------------------------------
@dataclass
class Grid2D:
    """Grid of the 2D2V solver; fields follow Grid, vlasov2D2V.py:87-173."""
    Nx: int
    Ny: int
    Nvx: int
    Nvy: int
    Lx: float
    Ly: float
    Vx_max: float
    Vy_max: float
    dx: float
    dy: float
    dvx: float
    dvy: float
    x: np.ndarray
    y: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    kx: np.ndarray       # (Nx, 1)
    ky: np.ndarray       # (1, Ny//2+1)
    inv_ksq: np.ndarray  # (Nx, Ny//2+1)
    dtype: np.dtype


def make_grid2d(Nx, Ny, Nvx, Nvy, Lx, Ly, Vx_max, Vy_max, dtype=np.float64) -> Grid2D:
    """Grid.create, vlasov2D2V.py:146-173 (torch factories on the CPU)."""
    import torch

    tdt = torch.float64 if np.dtype(dtype) == np.float64 else torch.float32
    dx, dy = Lx / Nx, Ly / Ny
    dvx, dvy = 2 * Vx_max / (Nvx - 1), 2 * Vy_max / (Nvy - 1)
    x = torch.linspace(0, Lx, Nx + 1, dtype=tdt)[:-1]
    y = torch.linspace(0, Ly, Ny + 1, dtype=tdt)[:-1]
    vx = torch.linspace(-Vx_max, Vx_max, Nvx, dtype=tdt)
    vy = torch.linspace(-Vy_max, Vy_max, Nvy, dtype=tdt)
    kx = 2 * math.pi * torch.fft.fftfreq(Nx, d=dx, dtype=tdt).unsqueeze(1)
    ky = 2 * math.pi * torch.fft.rfftfreq(Ny, d=dy, dtype=tdt).unsqueeze(0)
    ksq = kx ** 2 + ky ** 2
    inv = torch.where(ksq == 0, torch.tensor(0.0, dtype=tdt), 1.0 / ksq)
    return Grid2D(Nx, Ny, Nvx, Nvy, Lx, Ly, Vx_max, Vy_max, dx, dy, dvx, dvy,
                  x.numpy(), y.numpy(), vx.numpy(), vy.numpy(), kx.numpy(), ky.numpy(),
                  inv.numpy(), np.dtype(dtype))


@dataclass
class Grid1D:
    """Grid of the 1D1V solver; fields follow Grid, vlasov1D1V.py:76-122."""
    Nx: int
    Nv: int
    L: float
    V_max: float
    dx: float
    dv: float
    x: np.ndarray
    v: np.ndarray
    inv_kx: np.ndarray
    inv_kx_sq: np.ndarray
    dtype: np.dtype


def make_grid1d(Nx, Nv, L, V_max, dtype=np.float64) -> Grid1D:
    """Grid.create, vlasov1D1V.py:94-122."""
    import torch

    tdt = torch.float64 if np.dtype(dtype) == np.float64 else torch.float32
    dx = L / Nx
    dv = 2 * V_max / (Nv - 1)
    x = torch.linspace(0, L, Nx + 1, dtype=tdt)[:-1]
    v = torch.linspace(-V_max, V_max, Nv, dtype=tdt)
    kx = 2 * math.pi * torch.fft.rfftfreq(Nx, d=dx, dtype=tdt)
    inv = torch.where(kx == 0, torch.tensor(0.0, dtype=tdt), 1.0 / kx)
    return Grid1D(Nx, Nv, L, V_max, dx, dv, x.numpy(), v.numpy(), inv.numpy(),
                  (inv * inv).numpy(), np.dtype(dtype))


# --------------------------------------------------------------------------
# interpolation weights and static drift tables
# --------------------------------------------------------------------------
def lagrange5_weights(alpha: np.ndarray) -> np.ndarray:
    """lagrange5_weights, vlasov2D2V.py:263-285; returns (6, *alpha.shape)."""
    a = np.ascontiguousarray(alpha)
    out = np.empty((6,) + a.shape, dtype=a.dtype)
    getattr(lib(), f"or_lagrange5_weights_{_sfx(a.dtype)}")(_ptr(a), a.size, _ptr(out))
    return out


def precompute_drift(v: np.ndarray, dt: float, dx: float, dtype) -> tuple[np.ndarray, np.ndarray]:
    """precompute_x_drift, vlasov2D2V.py:670-714: per-velocity integer shift
    s = floor((v*dt)/dx) and Lagrange weights of the fraction, all in the run
    dtype. Returns (shift int64 (Nv,), W (6, Nv))."""
    T = np.dtype(dtype).type
    d = (np.asarray(v).astype(T) * T(dt)) / T(dx)
    s = np.floor(d)
    alpha = d - s
    return s.astype(np.int64), lagrange5_weights(alpha.astype(T))


# --------------------------------------------------------------------------
# sweeps
# --------------------------------------------------------------------------
def _olc(shape, axis):
    n_outer = int(np.prod(shape[:axis], dtype=np.int64))
    n_inner = int(np.prod(shape[axis + 1:], dtype=np.int64))
    return n_outer, int(shape[axis]), n_inner


def drift_static(f: np.ndarray, shift: np.ndarray, W: np.ndarray, axis: int, vel_axis: int) -> np.ndarray:
    """advect_x_static, vlasov2D2V.py:756-819: periodic drift along `axis`
    whose per-column shift/weights are indexed by `vel_axis` (> axis)."""
    f = np.ascontiguousarray(f)
    n_outer, n_line, n_inner = _olc(f.shape, axis)
    sel_div = int(np.prod(f.shape[vel_axis + 1:], dtype=np.int64))
    sel_mod = int(f.shape[vel_axis])
    out = np.empty_like(f)
    sh = np.ascontiguousarray(shift, dtype=np.int64)
    Wc = np.ascontiguousarray(W, dtype=f.dtype)
    getattr(lib(), f"or_drift_static_{_sfx(f.dtype)}")(
        _ptr(f), _ptr(out), n_outer, n_line, n_inner, sel_div, sel_mod, _ptr(sh), _ptr(Wc))
    return out


def kick_static(f: np.ndarray, E: np.ndarray, dt: float, dv: float, axis: int, window: int = -1) -> np.ndarray:
    """advect_v_static, vlasov2D2V.py:868-913 (1D: vlasov1D1V.py:479-501).
    E has the shape of the leading dims that precede the velocity dims
    ((Nx, Ny) in 2D2V, (Nx,) in 1D1V). window = S of the reference; a
    negative window keeps every tap (the exact kick)."""
    f = np.ascontiguousarray(f)
    n_outer, n_line, n_inner = _olc(f.shape, axis)
    Ef = np.ascontiguousarray(E, dtype=f.dtype).reshape(-1)
    e_div = n_outer // Ef.size
    out = np.empty_like(f)
    getattr(lib(), f"or_kick_static_{_sfx(f.dtype)}")(
        _ptr(f), _ptr(out), n_outer, n_line, n_inner, _ptr(Ef), e_div, float(dt), float(dv), int(window))
    return out


def advect_gather(f: np.ndarray, velocities: np.ndarray, axis: int, dt: float, dx: float,
                  periodic: bool = True) -> np.ndarray:
    """advect_1d, vlasov2D2V.py:356-413 with advect_1d_vectorized :287-353.
    `velocities` broadcasts to the batch shape (every dim except `axis`)."""
    f = np.ascontiguousarray(f)
    n_outer, n_line, n_inner = _olc(f.shape, axis)
    batch = f.shape[:axis] + f.shape[axis + 1:]
    v = np.ascontiguousarray(np.broadcast_to(np.asarray(velocities, dtype=f.dtype), batch))
    out = np.empty_like(f)
    getattr(lib(), f"or_advect_gather_{_sfx(f.dtype)}")(
        _ptr(f), _ptr(out), n_outer, n_line, n_inner, _ptr(v), n_inner, 0, 1,
        float(dt), float(dx), 1 if periodic else 0)
    return out


def advect_gather_rows(f_batch: np.ndarray, velocities: np.ndarray, dt: float, dx: float,
                       periodic: bool = True) -> np.ndarray:
    """advect_1d_vectorized of vlasov1D1V.py:212-256 on a [B, N] batch with
    per-row ([B]) or per-element ([B, N]) velocities."""
    f = np.ascontiguousarray(f_batch)
    B, N = f.shape
    v = np.ascontiguousarray(np.asarray(velocities, dtype=f.dtype))
    vso, vsl = (N, 1) if v.ndim == 2 else (1, 0)
    out = np.empty_like(f)
    # view [B][N] as outer=B, line=N, inner=1
    getattr(lib(), f"or_advect_gather_{_sfx(f.dtype)}")(
        _ptr(f), _ptr(out), B, N, 1, _ptr(v), vso, vsl, 0, float(dt), float(dx), 1 if periodic else 0)
    return out


def compute_rho(f: np.ndarray, dvx: float, dvy: float = 1.0, n_v_dims: int = 2) -> np.ndarray:
    """compute_rho, vlasov2D2V.py:416-431 (1D1V: n = sum(f, 1)*dv, :521)."""
    f = np.ascontiguousarray(f)
    lead = f.shape[: f.ndim - n_v_dims]
    n_v = int(np.prod(f.shape[f.ndim - n_v_dims:], dtype=np.int64))
    rho = np.empty(lead, dtype=f.dtype)
    getattr(lib(), f"or_rho_{_sfx(f.dtype)}")(_ptr(f), rho.size, n_v, float(dvx), float(dvy), _ptr(rho))
    return rho


# --------------------------------------------------------------------------
# Poisson
# --------------------------------------------------------------------------
def compute_poisson_real(rho: np.ndarray, kx: np.ndarray, ky: np.ndarray, inv_ksq: np.ndarray):
    """compute_poisson_real, vlasov2D2V.py:488-517, with numpy's pocketfft in
    place of torch.fft: delta = rho - 1, phi_k = rho_k * inv_ksq,
    E_k = -i k phi_k, three irfft2 of size (Nx, Ny). Returns (Ex, Ey, delta, phi)."""
    T = rho.dtype.type
    Nx, Ny = rho.shape
    delta = rho - T(1)
    rk = np.fft.rfft2(delta)
    pr = rk.real * inv_ksq
    pi = rk.imag * inv_ksq
    ex_k = (pi * kx) + 1j * (-pr * kx)
    ey_k = (pi * ky) + 1j * (-pr * ky)
    phi = np.fft.irfft2(pr + 1j * pi, s=(Nx, Ny)).astype(rho.dtype)
    Ex = np.fft.irfft2(ex_k.astype(rk.dtype), s=(Nx, Ny)).astype(rho.dtype)
    Ey = np.fft.irfft2(ey_k.astype(rk.dtype), s=(Nx, Ny)).astype(rho.dtype)
    return Ex, Ey, delta, phi


def solve_poisson_real(f, grid: Grid2D):
    rho = compute_rho(f, grid.dvx, grid.dvy)
    return compute_poisson_real(rho, grid.kx, grid.ky, grid.inv_ksq)


def solve_poisson_1d(f: np.ndarray, inv_kx: np.ndarray, inv_kx_sq: np.ndarray, dv: float):
    """solve_poisson_real, vlasov1D1V.py:538-572: n = sum(f,1)*dv, rho = n-1,
    E_k = -i rho_k inv_kx, phi_k = rho_k inv_kx^2. Returns (E, rho, phi)."""
    T = f.dtype.type
    n = compute_rho(f, dv, 1.0, n_v_dims=1)
    rho = n - T(1)
    rk = np.fft.rfft(rho)
    ek = (rk.imag * inv_kx) + 1j * (-rk.real * inv_kx)
    pk = (rk.real * inv_kx_sq) + 1j * (rk.imag * inv_kx_sq)
    Nx = rho.shape[0]
    E = np.fft.irfft(ek.astype(rk.dtype), n=Nx).astype(f.dtype)
    phi = np.fft.irfft(pk.astype(rk.dtype), n=Nx).astype(f.dtype)
    return E, rho, phi


# --------------------------------------------------------------------------
# Strang steps
# --------------------------------------------------------------------------
@dataclass
class StepOut:
    f: np.ndarray
    drho: np.ndarray
    phi: np.ndarray
    Ex: np.ndarray | None = None
    Ey: np.ndarray | None = None


class Stepper2D:
    """The solver-2 step of the reference (vlasov_step_gather_free_impl,
    vlasov2D2V.py:1043-1083) with the drift tables hoisted as in
    Vlasov.__init__ (:1277-1303). window = S of the kick (reference default
    1; negative = exact kick)."""

    def __init__(self, grid: Grid2D, dt: float, window: int = 1):
        self.g = grid
        self.dt = dt
        self.window = window
        T = grid.dtype
        self.sx, self.Wx = precompute_drift(grid.vx, dt / 2.0, grid.dx, T)
        self.sy, self.Wy = precompute_drift(grid.vy, dt / 2.0, grid.dy, T)

    def drift_x(self, f):
        return drift_static(f, self.sx, self.Wx, axis=0, vel_axis=2)

    def drift_y(self, f):
        return drift_static(f, self.sy, self.Wy, axis=1, vel_axis=3)

    def step(self, f: np.ndarray, physics_mode: bool = True) -> StepOut:
        g = self.g
        f = self.drift_x(f)
        f = self.drift_y(f)
        if physics_mode:
            Ex, Ey, drho, phi = solve_poisson_real(f, g)
        else:
            z = np.zeros((g.Nx, g.Ny), dtype=f.dtype)
            Ex, Ey, drho, phi = z, z.copy(), z.copy(), z.copy()
        f = kick_static(f, Ex, self.dt, g.dvx, axis=2, window=self.window)
        f = kick_static(f, Ey, self.dt, g.dvy, axis=3, window=self.window)
        f = self.drift_y(f)
        f = self.drift_x(f)
        return StepOut(f, drho, phi, Ex, Ey)


def step_gather_2d(f: np.ndarray, grid: Grid2D, dt: float, physics_mode: bool = True) -> StepOut:
    """The solver-0 step of the reference (vlasov_step_impl, vlasov2D2V.py:943-998)."""
    g = grid
    f = advect_gather(f, g.vx[None, :, None], 0, dt / 2.0, g.dx, periodic=True)
    f = advect_gather(f, g.vy[None, None, :], 1, dt / 2.0, g.dy, periodic=True)
    if physics_mode:
        Ex, Ey, drho, phi = solve_poisson_real(f, g)
    else:
        z = np.zeros((g.Nx, g.Ny), dtype=f.dtype)
        Ex, Ey, drho, phi = z, z.copy(), z.copy(), z.copy()
    f = advect_gather(f, Ex[:, :, None], 2, dt, g.dvx, periodic=False)
    f = advect_gather(f, Ey[:, :, None], 3, dt, g.dvy, periodic=False)
    f = advect_gather(f, g.vy[None, None, :], 1, dt / 2.0, g.dy, periodic=True)
    f = advect_gather(f, g.vx[None, :, None], 0, dt / 2.0, g.dx, periodic=True)
    return StepOut(f, drho, phi, Ex, Ey)


class Stepper1D:
    """The solver-2 step of the 1D1V reference (vlasov_step_gather_free_impl,
    vlasov1D1V.py:668-701)."""

    def __init__(self, grid: Grid1D, dt: float, window: int = 1):
        self.g = grid
        self.dt = dt
        self.window = window
        self.s, self.W = precompute_drift(grid.v, dt / 2.0, grid.dx, grid.dtype)

    def drift(self, f):
        return drift_static(f, self.s, self.W, axis=0, vel_axis=1)

    def step(self, f: np.ndarray, physics_mode: bool = True) -> StepOut:
        g = self.g
        f = self.drift(f)
        if physics_mode:
            E, rho, phi = solve_poisson_1d(f, g.inv_kx, g.inv_kx_sq, g.dv)
        else:
            E = np.zeros(g.Nx, dtype=f.dtype)
            rho, phi = E.copy(), E.copy()
        f = kick_static(f, E, self.dt, g.dv, axis=1, window=self.window)
        f = self.drift(f)
        return StepOut(f, rho, phi, E, None)


def step_gather_1d(f: np.ndarray, grid: Grid1D, dt: float, physics_mode: bool = True) -> StepOut:
    """The solver-0 step of the 1D1V reference (vlasov_step, vlasov1D1V.py:574-622)."""
    g = grid
    f = advect_gather(f, g.v, 0, dt / 2.0, g.dx, periodic=True)
    if physics_mode:
        E, rho, phi = solve_poisson_1d(f, g.inv_kx, g.inv_kx_sq, g.dv)
    else:
        E = np.zeros(g.Nx, dtype=f.dtype)
        rho, phi = E.copy(), E.copy()
    f = advect_gather(f, E, 1, dt, g.dv, periodic=False)
    f = advect_gather(f, g.v, 0, dt / 2.0, g.dx, periodic=True)
    return StepOut(f, rho, phi, E, None)


# --------------------------------------------------------------------------
# diagnostics (no reference counterpart; FP64)
# --------------------------------------------------------------------------
def field_energy_2d(Ex, Ey, dx, dy) -> float:
    """W_E = 1/2 sum(Ex^2 + Ey^2) dx dy."""
    Ex = np.asarray(Ex, dtype=np.float64)
    Ey = np.asarray(Ey, dtype=np.float64)
    return float(0.5 * np.sum(Ex * Ex + Ey * Ey) * dx * dy)


def field_energy_1d(E, dx) -> float:
    E = np.asarray(E, dtype=np.float64)
    return float(0.5 * np.sum(E * E) * dx)


def moments_2d(f: np.ndarray, g: Grid2D) -> dict:
    """mass, L2 and kinetic energy of f in FP64."""
    f64 = np.asarray(f, dtype=np.float64)
    dV = g.dx * g.dy * g.dvx * g.dvy
    v2 = (np.asarray(g.vx, np.float64)[:, None] ** 2 + np.asarray(g.vy, np.float64)[None, :] ** 2)
    return {
        "mass": float(f64.sum() * dV),
        "l2": float(np.sum(f64 * f64) * dV),
        "kinetic": float(0.5 * np.einsum("xyab,ab->", f64, v2) * dV),
    }


# --------------------------------------------------------------------------
# initial conditions of the benchmark configurations
# --------------------------------------------------------------------------
def landau_2d(g: Grid2D, eps: float, k: float) -> np.ndarray:
    """(1 + eps (cos kx + cos ky)) exp(-(vx^2+vy^2)/2) / (2 pi), FP64 then cast."""
    x = np.asarray(g.x, np.float64)
    y = np.asarray(g.y, np.float64)
    vx = np.asarray(g.vx, np.float64)
    vy = np.asarray(g.vy, np.float64)
    sp = 1.0 + eps * (np.cos(k * x)[:, None] + np.cos(k * y)[None, :])
    fv = np.exp(-0.5 * (vx[:, None] ** 2 + vy[None, :] ** 2)) / (2.0 * np.pi)
    return (sp[:, :, None, None] * fv[None, None]).astype(g.dtype)


def two_stream_2d(g: Grid2D, eps: float, k: float, v0: float) -> np.ndarray:
    """(1 + eps (cos kx + cos ky)) 1/2[M(vx-v0)+M(vx+v0)] M(vy), M the unit Maxwellian."""
    x = np.asarray(g.x, np.float64)
    y = np.asarray(g.y, np.float64)
    vx = np.asarray(g.vx, np.float64)
    vy = np.asarray(g.vy, np.float64)
    M = lambda u: np.exp(-0.5 * u * u) / np.sqrt(2.0 * np.pi)  # noqa: E731
    sp = 1.0 + eps * (np.cos(k * x)[:, None] + np.cos(k * y)[None, :])
    fv = (0.5 * (M(vx - v0) + M(vx + v0)))[:, None] * M(vy)[None, :]
    return (sp[:, :, None, None] * fv[None, None]).astype(g.dtype)


def landau_1d(g: Grid1D, eps: float, k: float) -> np.ndarray:
    x = np.asarray(g.x, np.float64)
    v = np.asarray(g.v, np.float64)
    f = (1.0 + eps * np.cos(k * x))[:, None] * (np.exp(-0.5 * v * v) / np.sqrt(2.0 * np.pi))[None, :]
    return f.astype(g.dtype)
