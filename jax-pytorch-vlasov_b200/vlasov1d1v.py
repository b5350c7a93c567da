"""Drop-in counterpart of the reference's PyTorch 1D1V solver module
(simulations/vlasov1d_1v/pytorch/src/vlasov1D1V.py), computed by the
sm_100a CUDA library. f is (Nx, Nv) with v contiguous.
"""
from __future__ import annotations

import math
import pathlib
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from . import ops
from .engine import Stepper1D
from . import vlasov2d2v as _v2
from .vlasov2d2v import (STENCIL_OFFSETS, _blocks_to_shift, _check_offsets, build_v_tap_weights,  # noqa: F401
                         check_v_window, get_lagrange5_weights, lagrange5_interp_sum, lagrange5_weights,
                         precompute_x_drift, static_stencil_offsets)


def _default_device():
    return torch.device("cuda", torch.cuda.current_device())


@dataclass
class Grid:
    """Grid of the 1D1V solver (vlasov1D1V.py:76-134), built on the CPU with
    the reference's torch factories, then moved to `device`."""
    Nx: int
    Nv: int
    L: float
    V_max: float
    dx: float
    dv: float
    x: torch.Tensor
    v: torch.Tensor
    inv_kx: torch.Tensor
    inv_kx_sq: torch.Tensor
    x_indices: torch.Tensor
    v_indices: torch.Tensor
    x_batch_offsets: torch.Tensor
    v_batch_offsets: torch.Tensor
    stencil_offsets: torch.Tensor

    @classmethod
    def create(cls, Nx, Nv, L, V_max, device=None, dtype=torch.float32):
        device = _default_device() if device is None else torch.device(device)
        gdt = torch.float64 if dtype == torch.float64 else torch.float32
        dx = L / Nx
        dv = 2 * V_max / (Nv - 1)
        x = torch.linspace(0, L, Nx + 1, dtype=gdt)[:-1]
        v = torch.linspace(-V_max, V_max, Nv, dtype=gdt)
        kx = 2 * math.pi * torch.fft.rfftfreq(Nx, d=dx, dtype=gdt)
        inv = torch.where(kx == 0, torch.tensor(0.0, dtype=gdt), 1.0 / kx)
        t = [x, v, inv, inv * inv, torch.arange(Nx, dtype=gdt), torch.arange(Nv, dtype=gdt),
             (torch.arange(Nv, dtype=torch.int64) * Nx).view(Nv, 1, 1),
             (torch.arange(Nx, dtype=torch.int64) * Nv).view(Nx, 1, 1),
             torch.arange(-2, 4, dtype=torch.int64)]
        t = [a.to(device) for a in t]
        return cls(Nx, Nv, L, V_max, dx, dv, *t)

    def to(self, device) -> "Grid":
        for name in ("x", "v", "inv_kx", "inv_kx_sq", "x_indices", "v_indices", "x_batch_offsets",
                     "v_batch_offsets", "stencil_offsets"):
            setattr(self, name, getattr(self, name).to(device))
        return self


@dataclass
class Field:
    rho: torch.Tensor
    phi: torch.Tensor


@dataclass
class Variables:
    fn: torch.Tensor
    f0: torch.Tensor


@dataclass
class SimulationState:
    field: Field
    variables: Variables
    t: float
    step: int


def _out_dtype(t):
    return torch.float64 if t.dtype == torch.float64 else torch.float32


# ---------------------------------------------------------------------------
# sweeps
# ---------------------------------------------------------------------------
def advect_1d_vectorized(f_batch, velocities, dt, point_indices, batch_offsets, stencil_offsets, dx, periodic=True):
    """Sweep along the last dim of f_batch [B, N] with per-row ([B]) or
    per-element ([B, N]) velocities (vlasov1D1V.py:212-256). A transposed
    view of a contiguous (N, B) array (the reference passes f.T) is swept in
    place along its strided axis, and the result is returned as the same
    kind of view, so that `.T` gives the contiguous (N, B) result."""
    _check_offsets(stencil_offsets)
    B, N = f_batch.shape
    v = velocities
    if f_batch.is_contiguous():
        if v.dim() == 1:
            return ops.advect_gather(f_batch, v, 1, dt, dx, periodic, vel_strides=(1, 0, 0))
        return ops.advect_gather(f_batch, v, 1, dt, dx, periodic, vel_strides=(N, 1, 0))
    base = f_batch.T
    if not base.is_contiguous():
        f_batch = f_batch.contiguous()
        return advect_1d_vectorized(f_batch, velocities, dt, point_indices, batch_offsets, stencil_offsets, dx,
                                    periodic)
    # base is (N, B) contiguous: axis 0 of base, velocity per column c = b
    if v.dim() == 1:
        out = ops.advect_gather(base, v, 0, dt, dx, periodic, vel_strides=(0, 0, 1))
    else:
        out = ops.advect_gather(base, v.contiguous(), 0, dt, dx, periodic, vel_strides=(0, 1, N))
    return out.T


def advect_1d_matrix_diag(f_batch, velocities, dt, dx, stencil_offsets, periodic=True):
    """Per-line shift + banded weights (vlasov1D1V.py:298-337): periodic
    branch drifts along dim 0 with one velocity per column, Dirichlet branch
    kicks along dim 1 with one field value per row."""
    _check_offsets(stencil_offsets)
    if periodic:
        table = ops.DriftTable.from_velocity(velocities, dt, dx, f_batch.dtype, f_batch.device)
        return ops.drift(f_batch.contiguous(), table, 0, 1)
    return ops.kick(f_batch.contiguous(), velocities, dt, dx, 1, window=-1)


def _roll_columns(x, shifts):
    """out[i, j] = x[(i - shifts[j]) % N, j] for x [N, M] (_roll_columns,
    vlasov1D1V.py:258-267): a periodic sweep along dim 0 whose departure
    points are whole cells (unit weight on the zero-offset tap, so finite
    values move unchanged). Floating-point x only."""
    if x.dim() != 2:
        raise ValueError("x must be [N, M]")
    v = shifts.to(L.compute_dtype(x.dtype))
    return ops.advect_gather(x.contiguous(), v, 0, 1.0, 1.0, True, vel_strides=(0, 0, 1))


def _roll_rows(x, shifts):
    """out[i, j] = x[i, (j - shifts[i]) % M] (_roll_rows, vlasov1D1V.py:269-277)."""
    return _v2._roll_batch(x, shifts)


def build_v_diag_weights(stencil_offsets, shifts, alpha, n_points):
    """Banded Dirichlet weights [6, Nx, Nv] of the v sweep
    (build_v_diag_weights, vlasov1D1V.py:279-296)."""
    return _v2.build_diag_weights(stencil_offsets, shifts, alpha, n_points)


def block_roll(f, blocks):
    """Roll each column block (start, stop, shift) of precompute_x_drift
    along x (block_roll, vlasov1D1V.py:389-406), by the drift kernel with a
    unit weight on the zero-offset tap."""
    return _v2.block_roll(f, blocks, 0, 1)


def advect_x_static(f, W_x, blocks, stencil_offsets):
    """Periodic x drift with static shifts (vlasov1D1V.py:408-448)."""
    _check_offsets(stencil_offsets)
    shift = _blocks_to_shift(blocks, f.shape[1])
    Wn = W_x.detach().cpu().numpy() if torch.is_tensor(W_x) else np.asarray(W_x)
    table = ops.DriftTable(shift, Wn, f.dtype, f.device)
    return ops.drift(f, table, 0, 1)


def advect_v_static(f, E, dt, dv, S, stencil_offsets):
    """Dirichlet v kick with static window S (vlasov1D1V.py:479-501)."""
    _check_offsets(stencil_offsets)
    return ops.kick(f, E, dt, dv, 1, window=int(S))


# ---------------------------------------------------------------------------
# field
# ---------------------------------------------------------------------------
def solve_poisson_real(f, inv_kx, inv_kx_sq, dv):
    """(E, rho, phi) from f (vlasov1D1V.py:538-572): n = sum(f,1)*dv in FP64,
    FP64 spectral solve, results in f's precision."""
    n = ops.velocity_moment(f, dv, 1.0, 1, out_dtype=torch.float64)
    e, rho, phi = ops.poisson1d(n, inv_kx, inv_kx_sq)
    dt = _out_dtype(f)
    return e.to(dt), rho.to(dt), phi.to(dt)


def solve_poisson(f, inv_kx, dv):
    """vlasov1D1V.py:514-536 (same result as solve_poisson_real)."""
    inv = inv_kx.to(torch.float64)
    return solve_poisson_real(f, inv, inv ** 2, dv)


# ---------------------------------------------------------------------------
# steps
# ---------------------------------------------------------------------------
def vlasov_step(f, dt, grid_v, grid_inv_kx, grid_inv_kx_sq, x_indices, v_indices, x_batch_offsets,
                v_batch_offsets, stencil_offsets, grid_dx, grid_dv, grid_V_max, physics_mode):
    """Strang step with per-element departure sweeps (vlasov1D1V.py:574-622)."""
    _check_offsets(stencil_offsets)
    f = ops.advect_gather(f, grid_v, 0, dt / 2.0, grid_dx, True)
    cdt = _out_dtype(f)
    if physics_mode:
        n = ops.velocity_moment(f, grid_dv, 1.0, 1, out_dtype=torch.float64)
        E, rho, phi = ops.poisson1d(n, grid_inv_kx, grid_inv_kx_sq)
    else:
        E = torch.zeros(f.shape[0], dtype=torch.float64, device=f.device)
        rho, phi = E.clone(), E.clone()
    f = ops.advect_gather(f, E.to(cdt), 1, dt, grid_dv, False)
    f = ops.advect_gather(f, grid_v, 0, dt / 2.0, grid_dx, True)
    return f, rho.to(cdt), phi.to(cdt)


_PLANS: dict = {}


def _fused(f, dt, table, grid_inv_kx, grid_inv_kx_sq, grid_dx, grid_dv, physics_mode, S, key):
    L.require_cuda(f)
    st = _PLANS.get(key)
    if st is None:
        st = Stepper1D.__new__(Stepper1D)
        st.device = f.device
        st.shape = tuple(f.shape)
        st.L = float(grid_dx) * f.shape[0]
        st.dx, st.dv, st.dt = float(grid_dx), float(grid_dv), float(dt)
        st.dtype = f.dtype
        st.physics_mode = bool(physics_mode)
        st.window = int(S)
        st.diagnostics = False
        st.table = table
        st.inv_kx = grid_inv_kx.reshape(-1).to(device=f.device, dtype=torch.float64).contiguous()
        st.inv_kx_sq = grid_inv_kx_sq.reshape(-1).to(device=f.device, dtype=torch.float64).contiguous()
        st.v64 = torch.zeros(1, dtype=torch.float64, device=f.device)
        nb = L.query("vp_step1d_workspace_bytes", *st.shape)
        st.ws = torch.empty(nb, dtype=torch.uint8, device=f.device)
        st.f_tmp = torch.empty_like(f)
        st.rho = torch.zeros(f.shape[0], dtype=torch.float64, device=f.device)
        st.phi = torch.zeros_like(st.rho)
        st.e = torch.zeros_like(st.rho)
        st.diag = None
        st._graphs = {}
        st._bufs = [None, None]
        st.eq, st.eq_moment = None, 0.0
        st.status = torch.zeros(1, dtype=torch.int32, device=f.device)
        st.test_stall = 0
        if len(_PLANS) > 16:
            _PLANS.clear()
        _PLANS[key] = st
    st.physics_mode = bool(physics_mode)
    out = st.step(f, torch.empty_like(f))
    cdt = _out_dtype(f)
    return out, st.rho.to(cdt, copy=True), st.phi.to(cdt, copy=True)


def vlasov_step_gather_free(f, dt, grid_v, grid_inv_kx, grid_inv_kx_sq, x_indices, v_indices, x_batch_offsets,
                            v_batch_offsets, stencil_offsets, grid_dx, grid_dv, grid_V_max, physics_mode, S=1):
    """Solver-2 step (vlasov1D1V.py:703-755): x(dt/2) fused with n, Poisson,
    v(dt), x(dt/2) in one launch sequence."""
    _check_offsets(stencil_offsets)
    key = (tuple(f.shape), f.dtype, f.device, float(dt), grid_v.data_ptr(), grid_v._version, float(grid_dx),
           float(grid_dv), int(S), grid_inv_kx.data_ptr())
    table = None if key in _PLANS else ops.DriftTable.from_velocity(grid_v, dt / 2.0, grid_dx, f.dtype, f.device)
    return _fused(f, dt, table, grid_inv_kx, grid_inv_kx_sq, grid_dx, grid_dv, physics_mode, S, key)


def vlasov_step_gather_free_impl(f, dt, W_x, blocks, stencil_offsets, grid_inv_kx, grid_inv_kx_sq, grid_dv,
                                 physics_mode, S):
    """Solver-2 step with precomputed tables (vlasov1D1V.py:668-701)."""
    _check_offsets(stencil_offsets)
    key = ("impl", W_x.data_ptr(), W_x._version, tuple(map(tuple, blocks)), tuple(f.shape), f.dtype, f.device,
           float(dt), float(grid_dv), int(S), grid_inv_kx.data_ptr())
    table = None
    if key not in _PLANS:
        table = ops.DriftTable(_blocks_to_shift(blocks, f.shape[1]), W_x.detach().cpu().numpy(), f.dtype, f.device)
    return _fused(f, dt, table, grid_inv_kx, grid_inv_kx_sq, 1.0, grid_dv, physics_mode, S, key)


def vlasov_step_matrix_diag(f, dt, grid_v, grid_inv_kx, grid_inv_kx_sq, x_indices, v_indices, x_batch_offsets,
                            v_batch_offsets, stencil_offsets, grid_dx, grid_dv, grid_V_max, physics_mode):
    """Solver-1 step (vlasov1D1V.py:624-666): per-line shifts, exact kick."""
    return vlasov_step_gather_free(f, dt, grid_v, grid_inv_kx, grid_inv_kx_sq, x_indices, v_indices,
                                   x_batch_offsets, v_batch_offsets, stencil_offsets, grid_dx, grid_dv, grid_V_max,
                                   physics_mode, S=-1)


class Vlasov:
    """Driver with the reference's constructor arguments (vlasov1D1V.py:770-876).
    Extra keyword arguments: device, window (S of solver 2), write_snapshots."""

    def __init__(self, Nx=128, Nv=128, L=2.0 * math.pi, V_max=6.0, nbiter=10, diag_steps=10, dt=0.05,
                 out_dir="data", physics_mode=False, epsilon=0.001, dtype="float32", solver=0, device=None,
                 window=1, write_snapshots=True):
        self.output_log = ""
        self.dtype = {"float32": torch.float32, "float64": torch.float64, "bfloat16": torch.bfloat16}[dtype]
        self.device = _default_device() if device is None else torch.device(device)
        gdt = torch.float64 if self.dtype == torch.float64 else torch.float32
        self.grid = Grid.create(Nx, Nv, L, V_max, device=self.device, dtype=gdt)
        self.nbiter, self.diag_steps, self.dt = nbiter, diag_steps, dt
        self.out_dir, self.physics_mode, self.epsilon = out_dir, physics_mode, epsilon
        self.solver = solver
        self.solver_type = {0: "vlasov_step", 1: "vlasov_step_matrix_diag", 2: "vlasov_step_gather_free"}[solver]
        self.write_snapshots = write_snapshots
        self.stepper = Stepper1D(Nx, Nv, L, V_max, dt, dtype=self.dtype, device=self.device,
                                 physics_mode=physics_mode, window=(window if solver == 2 else -1),
                                 v=self.grid.v.cpu())
        self.history = None
        if write_snapshots:
            pathlib.Path(out_dir).mkdir(parents=True, exist_ok=True)
        self.output_log += (f"Starting simulation on {self.device} with {self.dtype} storage, solver "
                            f"{self.solver_type}\nGrid: {Nx}x{Nv}, Steps: {nbiter}, diag_freq: {diag_steps}\n")

    def initialize(self) -> SimulationState:
        """vlasov1D1V.py:881-911: Landau (physics_mode) or Gaussian pulse."""
        g = self.grid
        x = g.x.double()[:, None]
        v = g.v.double()[None, :]
        if self.physics_mode:
            maxw = (1.0 / math.sqrt(2.0 * math.pi)) * torch.exp(-0.5 * v ** 2)
            f = ops.init_product((1.0 + self.epsilon * torch.cos(2.0 * math.pi / g.L * x))[:, 0], maxw[0],
                                 self.dtype)
            f0 = maxw.squeeze(0)
        else:
            sx, sv = g.L / 10.0, g.V_max / 4.0
            f = torch.exp(-0.5 * ((x - g.L / 2.0) ** 2 / sx ** 2 + v ** 2 / sv ** 2))
            f0 = torch.zeros(g.Nv, dtype=torch.float64, device=self.device)
        f = f.to(self.dtype).contiguous()
        n = ops.velocity_moment(f, g.dv, 1.0, 1)
        _, rho, phi = ops.poisson1d(n, g.inv_kx, g.inv_kx_sq)
        state = SimulationState(Field(rho, phi), Variables(f, f0.to(_out_dtype(f))), 0.0, 0)
        self.save_diag(state)
        return state

    def save_diag(self, state):
        if not self.write_snapshots:
            return
        from .snapshot import write_snapshot_1d
        write_snapshot_1d(pathlib.Path(self.out_dir) / f"field_{int(state.step):06d}.npz", state, self)

    def run(self, state):
        g = self.grid
        f = state.variables.fn.contiguous()
        hist = torch.zeros((self.nbiter, L.DIAG_COUNT), dtype=torch.float64, device=self.device)
        done = 0
        while done < self.nbiter:
            n = min(self.diag_steps, self.nbiter - done)
            if self.solver == 0:
                for _ in range(n):
                    f, rho, phi = vlasov_step(f, self.dt, g.v, g.inv_kx, g.inv_kx_sq, g.x_indices, g.v_indices,
                                              g.x_batch_offsets, g.v_batch_offsets, g.stencil_offsets, g.dx, g.dv,
                                              g.V_max, self.physics_mode)
            else:
                f = self.stepper.run(f, n, history=hist[done: done + n])
                rho = self.stepper.rho.to(_out_dtype(f), copy=True)
                phi = self.stepper.phi.to(_out_dtype(f), copy=True)
            done += n
            state = SimulationState(Field(rho, phi), Variables(f, state.variables.f0), state.t + n * self.dt,
                                    state.step + n)
            if n == self.diag_steps:
                self.save_diag(state)
        torch.cuda.synchronize(self.device)
        self.history = hist
        return state
