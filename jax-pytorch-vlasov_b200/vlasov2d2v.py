"""Drop-in counterpart of the reference's PyTorch 2D2V solver module
(simulations/vlasov2d_2v/pytorch/src/vlasov2D2V.py): the same names,
signatures and return values, computed by the sm_100a CUDA library.

Inputs are CUDA tensors; outputs are new CUDA tensors (the reference's
functional convention). Everything O(N^4) runs in the library's kernels; the
host side only builds the small static tables (drift shifts and weights,
wave numbers) once per configuration.
"""
from __future__ import annotations

import math
import os
import pathlib
from dataclasses import dataclass
from typing import Tuple

import numpy as np
import torch

from . import _lib as L
from . import ops
from .engine import Stepper2D

STENCIL_OFFSETS = (-2, -1, 0, 1, 2, 3)


def _default_device():
    return torch.device("cuda", torch.cuda.current_device())


# ---------------------------------------------------------------------------
# state containers (vlasov2D2V.py:87-208)
# ---------------------------------------------------------------------------
@dataclass
class Grid:
    """Grid of the 2D2V solver (vlasov2D2V.py:87-188). Coordinates and wave
    numbers are built on the CPU with the same torch factories as the
    reference (so they are bit-identical to it) and then moved to `device`."""
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
    x: torch.Tensor
    y: torch.Tensor
    vx: torch.Tensor
    vy: torch.Tensor
    kx: torch.Tensor
    ky: torch.Tensor
    inv_ksq: torch.Tensor
    x_indices: torch.Tensor
    y_indices: torch.Tensor
    vx_indices: torch.Tensor
    vy_indices: torch.Tensor
    stencil_offsets: torch.Tensor

    @classmethod
    def create(cls, Nx, Ny, Nvx, Nvy, Lx, Ly, Vx_max, Vy_max, device=None, dtype=torch.float32):
        device = _default_device() if device is None else torch.device(device)
        gdt = torch.float64 if dtype == torch.float64 else torch.float32
        dx, dy = Lx / Nx, Ly / Ny
        dvx, dvy = 2 * Vx_max / (Nvx - 1), 2 * Vy_max / (Nvy - 1)
        x = torch.linspace(0, Lx, Nx + 1, dtype=gdt)[:-1]
        y = torch.linspace(0, Ly, Ny + 1, dtype=gdt)[:-1]
        vx = torch.linspace(-Vx_max, Vx_max, Nvx, dtype=gdt)
        vy = torch.linspace(-Vy_max, Vy_max, Nvy, dtype=gdt)
        kx = 2 * math.pi * torch.fft.fftfreq(Nx, d=dx, dtype=gdt).unsqueeze(1)
        ky = 2 * math.pi * torch.fft.rfftfreq(Ny, d=dy, dtype=gdt).unsqueeze(0)
        ksq = kx ** 2 + ky ** 2
        inv = torch.where(ksq == 0, torch.tensor(0.0, dtype=gdt), 1.0 / ksq)
        t = [x, y, vx, vy, kx, ky, inv,
             torch.arange(Nx, dtype=gdt), torch.arange(Ny, dtype=gdt),
             torch.arange(Nvx, dtype=gdt), torch.arange(Nvy, dtype=gdt),
             torch.arange(-2, 4, dtype=torch.int64)]
        t = [v.to(device) for v in t]
        return cls(Nx, Ny, Nvx, Nvy, Lx, Ly, Vx_max, Vy_max, dx, dy, dvx, dvy, *t)

    def to(self, device) -> "Grid":
        for name in ("x", "y", "vx", "vy", "kx", "ky", "inv_ksq", "x_indices", "y_indices", "vx_indices",
                     "vy_indices", "stencil_offsets"):
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


# ---------------------------------------------------------------------------
# interpolation helpers (host side; the kernels evaluate the same weights)
# ---------------------------------------------------------------------------
def lagrange5_weights(alpha):
    """Weights of the 6-point Lagrange stencil (vlasov2D2V.py:263-285),
    returned as (6, *alpha.shape) on alpha's device. Used for the static
    drift tables; evaluated on the host (a few hundred values at most)."""
    a = alpha.detach().cpu().numpy() if torch.is_tensor(alpha) else np.asarray(alpha)
    w = ops.lagrange5_weights_np(a)
    out = torch.from_numpy(w)
    return out.to(alpha.device) if torch.is_tensor(alpha) else out


def _lagrange_dtype(*ts):
    dt = torch.result_type(*ts) if len(ts) > 1 else ts[0].dtype
    if dt not in (torch.float32, torch.float64):
        raise TypeError(f"Lagrange helpers take float32 or float64 tensors, not {dt}")
    return dt


def lagrange5_interp_sum(alpha, gather_vals):
    """The 6-point interpolation sum (lagrange5_interp_sum,
    vlasov2D2V.py:238-260): sum_k w_k(alpha) * gather_vals[..., k] with the
    closed-form weights, computed on the device by vp_lagrange_interp with
    the reference's rounding (bit-identical to its eager evaluation)."""
    L.require_cuda(alpha, gather_vals)
    if gather_vals.shape[-1] != 6:
        raise ValueError("gather_vals must have 6 values in its last dimension")
    dt = _lagrange_dtype(alpha, gather_vals)
    shape = torch.broadcast_shapes(alpha.shape, gather_vals.shape[:-1])
    a = alpha.to(dt).expand(shape).contiguous()
    v = gather_vals.to(dt).expand(*shape, 6).contiguous()
    out = torch.empty(shape, dtype=dt, device=a.device)
    L.call("vp_lagrange_interp", L.ptr(a), L.ptr(v), L.ptr(out), L.dtype_code(dt), a.numel(), L.stream_of(a))
    return out


def get_lagrange5_weights(alpha):
    """Product-form Lagrange weights of the nodes -2..3
    (get_lagrange5_weights, vlasov2D2V.py:210-235), shape (*alpha.shape, 6),
    computed on the device by vp_lagrange_weights."""
    L.require_cuda(alpha)
    dt = _lagrange_dtype(alpha)
    a = alpha.contiguous()
    out = torch.empty((*a.shape, 6), dtype=dt, device=a.device)
    L.call("vp_lagrange_weights", L.ptr(a), L.ptr(out), L.dtype_code(dt), a.numel(), L.stream_of(a))
    return out


def static_stencil_offsets(stencil_offsets) -> Tuple[int, ...]:
    """vlasov2D2V.py:644-667."""
    if isinstance(stencil_offsets, torch.Tensor):
        return tuple(int(o) for o in stencil_offsets.tolist())
    return tuple(int(o) for o in stencil_offsets)


def _check_offsets(stencil_offsets):
    if stencil_offsets is not None and static_stencil_offsets(stencil_offsets) != STENCIL_OFFSETS:
        raise NotImplementedError("the kernels implement the 6-point stencil with offsets -2..3 only")


def precompute_x_drift(v, dt, dx, dtype):
    """vlasov2D2V.py:670-714: static shift blocks (start, stop, shift) and the
    (6, Nv) weights, computed in `dtype`'s precision as the reference does."""
    s, W = ops.drift_table_np(v, dt, dx, dtype)
    edges = np.flatnonzero(np.diff(s)) + 1
    starts = np.concatenate(([0], edges))
    stops = np.concatenate((edges, [len(s)]))
    blocks = [(int(a), int(b), int(s[a])) for a, b in zip(starts, stops)]
    dev = v.device if torch.is_tensor(v) else None
    return blocks, torch.as_tensor(W, dtype=dtype if dtype != torch.bfloat16 else torch.float32, device=dev)


def _blocks_to_shift(blocks, n):
    s = np.zeros(n, dtype=np.int64)
    for a, b, sh in blocks:
        s[a:b] = sh
    return s


# ---------------------------------------------------------------------------
# sweeps
# ---------------------------------------------------------------------------
def advect_1d(f_data, velocities, axis, dt, dx, periodic=True, point_indices=None, stencil_offsets=None):
    """Semi-Lagrangian sweep along `axis` with a per-element departure point
    (advect_1d + advect_1d_vectorized, vlasov2D2V.py:287-413), without the
    reference's permute copies: the kernel addresses the strided axis directly."""
    _check_offsets(stencil_offsets)
    return ops.advect_gather(f_data, velocities, axis, dt, dx, periodic)


def advect_1d_vectorized(f_batch, velocities, dt, dx, point_indices=None, stencil_offsets=None, periodic=True):
    """Batched sweep along the last dim of f_batch [B, N] with per-row ([B])
    or per-element ([B, N]) velocities (advect_1d_vectorized,
    vlasov2D2V.py:287-353), by the per-element departure kernel. The grid
    points are 0 .. N-1 (the reference's default point_indices, the only ones
    its callers pass)."""
    _check_offsets(stencil_offsets)
    if f_batch.dim() != 2:
        raise ValueError("f_batch must be [batch, n_points]")
    B, N = f_batch.shape
    if point_indices is not None and tuple(point_indices.shape) != (N,):
        raise ValueError("point_indices must be the N grid indices 0 .. N-1")
    f_batch = f_batch.contiguous()
    v = velocities
    if v.dim() == 1:
        return ops.advect_gather(f_batch, v, 1, dt, dx, periodic, vel_strides=(1, 0, 0))
    return ops.advect_gather(f_batch, v.expand(B, N), 1, dt, dx, periodic, vel_strides=(N, 1, 0))


def _roll_batch(x, shifts):
    """out[i, j] = x[i, (j - shifts[i]) % N] for x [B, N] (_roll_batch,
    vlasov2D2V.py:526-535): a periodic sweep whose departure points are whole
    cells. At a zero fraction the Lagrange weights are exactly (0, 0, 1, 0,
    0, 0), so every finite value moves unchanged. Floating-point x only."""
    if x.dim() != 2:
        raise ValueError("x must be [batch, n_points]")
    v = shifts.to(L.compute_dtype(x.dtype))
    return ops.advect_gather(x.contiguous(), v, 1, 1.0, 1.0, True, vel_strides=(1, 0, 0))


def build_diag_weights(stencil_offsets, shifts, alpha, n_points):
    """Banded weights [6, B, n_points] of the Dirichlet per-row sweep
    (build_diag_weights, vlasov2D2V.py:538-555): tap k of row b carries
    w_k(alpha_b) at the points j whose source j - shifts[b] - o_k lies inside
    the line, zero elsewhere."""
    offs = torch.as_tensor(static_stencil_offsets(stencil_offsets), dtype=torch.int64, device=alpha.device)
    W = lagrange5_weights(alpha)                                   # [6, B]
    j = torch.arange(n_points, device=alpha.device)
    src = j[None, None, :] - (offs[:, None] + shifts.to(torch.int64)[None, :])[..., None]
    inside = (src >= 0) & (src < n_points)
    return torch.where(inside, W[..., None], torch.zeros((), dtype=W.dtype, device=W.device))


def advect_1d_matrix_diag_core(f_batch, velocities, dt, dx, stencil_offsets, periodic=True):
    """Per-row sweep of f_batch [B, N] with one velocity per row
    (advect_1d_matrix_diag_core, vlasov2D2V.py:558-589): shift s = floor(d)
    and fraction of d = v dt / dx per row. Dirichlet rows (zero outside) run
    the kick kernel, which uses exactly this shift and fraction; periodic rows
    run the per-element departure kernel (the same interpolant, round-off
    apart)."""
    _check_offsets(stencil_offsets)
    if f_batch.dim() != 2:
        raise ValueError("f_batch must be [batch, n_points]")
    f_batch = f_batch.contiguous()
    if periodic:
        return ops.advect_gather(f_batch, velocities.reshape(-1), 1, dt, dx, True, vel_strides=(1, 0, 0))
    return ops.kick(f_batch, velocities.reshape(-1), dt, dx, 1, window=-1)


def _line_velocity_structure(f_data, velocities, axis):
    """If velocities (broadcast to the batch shape) depend on a single dim
    of f after `axis` (a drift) or only on the dims before `axis` (a kick),
    return ('drift', vel_axis, 1D values) or ('kick', field over the
    leading dims); else None."""
    nd = f_data.dim()
    v = velocities
    vshape = list(v.shape)
    batch_dims = [d for d in range(nd) if d != axis]
    # pad to len(batch_dims)
    vshape = [1] * (len(batch_dims) - len(vshape)) + vshape
    v = v.reshape(vshape)
    varying = [batch_dims[i] for i, s in enumerate(vshape) if s != 1]
    if len(varying) == 1 and varying[0] > axis:
        return ("drift", varying[0], v.reshape(-1))
    if all(d < axis for d in varying):
        lead = tuple(f_data.shape[:axis])
        return ("kick", v.reshape(vshape[:axis] if axis > 0 else []).expand(lead) if axis > 0 else v.reshape(()))
    return None


def advect_1d_matrix_diag(f_data, velocities, axis, dt, dx, periodic=True, point_indices=None, stencil_offsets=None):
    """Per-line shift + banded weights (advect_1d_matrix_diag,
    vlasov2D2V.py:526-641): the interpolant of each line uses one
    displacement d = v*dt/dx, its floor and its fraction. Drifts whose
    velocity varies along one later dim and kicks whose field varies over the
    leading dims run the static-table kernels; other velocity layouts fall
    back to the per-element sweep (same interpolant, round-off apart)."""
    _check_offsets(stencil_offsets)
    st = _line_velocity_structure(f_data, velocities, axis)
    if st is not None and st[0] == "drift" and periodic:
        _, vel_axis, v1 = st
        table = ops.DriftTable.from_velocity(v1, dt, dx, f_data.dtype, f_data.device)
        return ops.drift(f_data, table, axis, vel_axis)
    if st is not None and st[0] == "kick" and not periodic and axis > 0:
        return ops.kick(f_data, st[1].contiguous(), dt, dx, axis, window=-1)
    return ops.advect_gather(f_data, velocities, axis, dt, dx, periodic)


def _unit_table(blocks, n, dtype, device):
    """Drift table of whole-cell shifts: weight 1 on the tap at offset 0."""
    W = np.zeros((6, n), dtype=np.float64)
    W[STENCIL_OFFSETS.index(0)] = 1.0
    return ops.DriftTable(_blocks_to_shift(blocks, n), W, dtype, device)


def block_roll(f_data, blocks, axis, vel_axis):
    """Roll each velocity block (start, stop, shift) of precompute_x_drift by
    its whole-cell shift along the spatial `axis` (block_roll,
    vlasov2D2V.py:717-753): the periodic drift kernel with a unit weight on
    the zero-offset tap, so every finite value moves unchanged. Returns f_data
    itself when no shift moves anything, as the reference does."""
    if vel_axis <= axis:
        raise ValueError("the velocity axis of the blocks must come after the rolled axis")
    if all(sh % f_data.shape[axis] == 0 for _, _, sh in blocks):
        return f_data
    table = _unit_table(blocks, f_data.shape[vel_axis], f_data.dtype, f_data.device)
    return ops.drift(f_data.contiguous(), table, axis, vel_axis)


def build_v_tap_weights(E, dt, dv, S, stencil_offsets):
    """Tap weights of the static kick window (build_v_tap_weights,
    vlasov2D2V.py:822-865; vlasov1D1V.py:450-476): shape (2S+5, *E.shape),
    row m + S + 2 holding w_k(alpha) where floor(E dt / dv) + o_k = m. Each
    row takes at most one weight, so the table is exact. The small table is
    built on the host with correctly rounded division (a CUDA tensor divided
    by a Python number is multiplied by its reciprocal instead, which can
    move the fraction by one unit in the last place); the weights are the
    reference's closed form."""
    Eh = E.detach().cpu()
    d = (Eh * dt) / dv
    s = torch.floor(d)
    alpha = d - s
    s = s.to(torch.int64)
    W6 = lagrange5_weights(alpha)
    offs = static_stencil_offsets(stencil_offsets)
    zero = torch.zeros((), dtype=W6.dtype)
    rows = []
    for m in range(-(S + 2), S + 3):
        row = torch.zeros_like(alpha)
        for k, o in enumerate(offs):
            row = torch.where(s == m - o, W6[k], row)
        rows.append(torch.where(row == 0, zero, row))
    return torch.stack(rows, dim=0).to(E.device)


def advect_x_static(f_data, W, blocks, stencil_offsets, axis):
    """Periodic x/y drift with static shifts (advect_x_static,
    vlasov2D2V.py:756-819). W: (6, Nv) weights, blocks from precompute_x_drift."""
    _check_offsets(stencil_offsets)
    vel_axis = axis + 2
    n = f_data.shape[vel_axis]
    shift = _blocks_to_shift(blocks, n)
    Wn = W.detach().cpu().numpy() if torch.is_tensor(W) else np.asarray(W)
    table = ops.DriftTable(shift, Wn, f_data.dtype, f_data.device)
    return ops.drift(f_data, table, axis, vel_axis)


def advect_v_static(f_data, E, dt, dv, S, stencil_offsets, axis):
    """Dirichlet vx/vy kick (advect_v_static, vlasov2D2V.py:868-913), with
    the reference's static window S (taps with |s+o| > S+2 dropped; exact
    while |E dt/dv| < S)."""
    _check_offsets(stencil_offsets)
    return ops.kick(f_data, E, dt, dv, axis, window=int(S))


def check_v_window(E, dt, dv, S):
    """max |E dt/dv| in cells (vlasov2D2V.py:916-941)."""
    return float((E * dt / dv).abs().max())


# ---------------------------------------------------------------------------
# moments and field
# ---------------------------------------------------------------------------
def _out_dtype(t):
    return torch.float64 if t.dtype == torch.float64 else torch.float32


def compute_rho(f_data, dvx, dvy):
    """sum(f, dim=(2,3)) * dvx * dvy (vlasov2D2V.py:416-431), FP64 accumulation."""
    return ops.velocity_moment(f_data, dvx, dvy, 2, out_dtype=_out_dtype(f_data))


def compute_poisson_real(rho, kx, ky, inv_ksq):
    """(Ex, Ey, delta_rho, phi) of rho (vlasov2D2V.py:488-517), solved in FP64
    and returned in rho's precision."""
    ex, ey, drho, phi = ops.poisson2d(rho.to(torch.float64), kx, ky, inv_ksq)
    dt = _out_dtype(rho)
    return ex.to(dt), ey.to(dt), drho.to(dt), phi.to(dt)


compute_poisson = compute_poisson_real  # vlasov2D2V.py:434-465: same result


def solve_poisson_real(f_data, kx, ky, inv_ksq, dvx, dvy):
    """vlasov2D2V.py:520-523."""
    rho = ops.velocity_moment(f_data, dvx, dvy, 2, out_dtype=torch.float64)
    ex, ey, drho, phi = ops.poisson2d(rho, kx, ky, inv_ksq)
    dt = _out_dtype(f_data)
    return ex.to(dt), ey.to(dt), drho.to(dt), phi.to(dt)


solve_poisson = solve_poisson_real  # vlasov2D2V.py:468-485


# ---------------------------------------------------------------------------
# steps
# ---------------------------------------------------------------------------
def vlasov_step_impl(f, f0, dt, grid_x, grid_y, grid_vx, grid_vy, grid_kx, grid_ky, grid_inv_ksq,
                     grid_x_indices, grid_y_indices, grid_vx_indices, grid_vy_indices, grid_stencil_offsets,
                     grid_dx, grid_dy, grid_dvx, grid_dvy, grid_Nx, grid_Ny, physics_mode):
    """Strang step with per-element departure sweeps (vlasov_step_impl,
    vlasov2D2V.py:943-998). Returns (f, delta_rho, phi)."""
    _check_offsets(grid_stencil_offsets)
    f = ops.advect_gather(f, grid_vx[None, :, None], 0, dt / 2.0, grid_dx, True)
    f = ops.advect_gather(f, grid_vy[None, None, :], 1, dt / 2.0, grid_dy, True)
    cdt = _out_dtype(f)
    if physics_mode:
        rho = ops.velocity_moment(f, grid_dvx, grid_dvy, 2, out_dtype=torch.float64)
        Ex, Ey, drho, phi = ops.poisson2d(rho, grid_kx, grid_ky, grid_inv_ksq)
    else:
        Ex = torch.zeros((grid_Nx, grid_Ny), dtype=torch.float64, device=f.device)
        Ey, drho, phi = Ex.clone(), Ex.clone(), Ex.clone()
    f = ops.advect_gather(f, Ex.to(cdt)[:, :, None], 2, dt, grid_dvx, False)
    f = ops.advect_gather(f, Ey.to(cdt)[:, :, None], 3, dt, grid_dvy, False)
    f = ops.advect_gather(f, grid_vy[None, None, :], 1, dt / 2.0, grid_dy, True)
    f = ops.advect_gather(f, grid_vx[None, :, None], 0, dt / 2.0, grid_dx, True)
    return f, drho.to(cdt), phi.to(cdt)


_PLANS: dict = {}


def _plan_key(f, dt, grid_vx, grid_vy, grid_kx, grid_dx, grid_dy, grid_dvx, grid_dvy, S):
    def tk(t):
        return (t.data_ptr(), t._version, tuple(t.shape), t.dtype) if torch.is_tensor(t) else repr(t)
    return (tuple(f.shape), f.dtype, f.device, float(dt), tk(grid_vx), tk(grid_vy), tk(grid_kx), float(grid_dx),
            float(grid_dy), float(grid_dvx), float(grid_dvy), int(S))


def _fused_step(f, dt, tables, spectral, grid_dx, grid_dy, grid_dvx, grid_dvy, physics_mode, S, key):
    """One vp_step2d call; tables = (tx, ty) DriftTables, spectral =
    (kx, ky, inv_ksq) float64 on f's device."""
    L.require_cuda(f)
    plan = _PLANS.get(key)
    if plan is None:
        Nx, Ny, Nvx, Nvy = f.shape
        st = Stepper2D.__new__(Stepper2D)
        st.device = f.device
        st.shape = tuple(f.shape)
        st.dx, st.dy, st.dvx, st.dvy = float(grid_dx), float(grid_dy), float(grid_dvx), float(grid_dvy)
        st.dt = float(dt)
        st.dtype = f.dtype
        st.physics_mode = bool(physics_mode)
        st.window = int(S)
        st.diagnostics = False
        st.tx, st.ty = tables
        st.kx, st.ky, st.inv_ksq = spectral
        st.vx64 = st.vy64 = torch.zeros(1, dtype=torch.float64, device=f.device)
        nb = L.query("vp_step2d_workspace_bytes", Nx, Ny, Nvx, Nvy)
        st.ws = torch.empty(nb, dtype=torch.uint8, device=f.device)
        st.f_tmp = torch.empty_like(f)
        z = lambda: torch.zeros((Nx, Ny), dtype=torch.float64, device=f.device)  # noqa: E731
        st.drho, st.phi, st.ex, st.ey = z(), z(), z(), z()
        st.diag = None
        st._graphs = {}
        st._bufs = [None, None]
        st.eq, st.eq_moment = None, 0.0
        st.status = torch.zeros(1, dtype=torch.int32, device=f.device)
        st.test_stall = 0
        if len(_PLANS) > 16:
            _PLANS.clear()
        _PLANS[key] = plan = st
    plan.physics_mode = bool(physics_mode)
    out = plan.step(f, torch.empty_like(f))
    cdt = _out_dtype(f)
    return out, plan.drho.to(cdt, copy=True), plan.phi.to(cdt, copy=True)


def _spectral(grid_kx, grid_ky, grid_inv_ksq, device):
    return (grid_kx.reshape(-1).to(device=device, dtype=torch.float64).contiguous(),
            grid_ky.reshape(-1).to(device=device, dtype=torch.float64).contiguous(),
            grid_inv_ksq.to(device=device, dtype=torch.float64).contiguous())


def vlasov_step_gather_free_impl(f, dt, W_x, W_y, blocks_x, blocks_y, stencil_offsets, grid_kx, grid_ky,
                                 grid_inv_ksq, grid_dvx, grid_dvy, grid_Nx, grid_Ny, physics_mode, S):
    """Solver-2 step with precomputed tables (vlasov2D2V.py:1043-1083), as one
    fused launch sequence: x, y+rho, Poisson, vx+vy, y, x."""
    _check_offsets(stencil_offsets)
    Nvx, Nvy = f.shape[2], f.shape[3]
    key = ("impl", W_x.data_ptr(), W_x._version, W_y.data_ptr(), W_y._version, tuple(map(tuple, blocks_x)),
           tuple(map(tuple, blocks_y)), tuple(f.shape), f.dtype, f.device, float(dt), float(grid_dvx),
           float(grid_dvy), int(S))
    tables = spectral = None
    if key not in _PLANS:
        tables = (ops.DriftTable(_blocks_to_shift(blocks_x, Nvx), W_x.detach().cpu().numpy(), f.dtype, f.device),
                  ops.DriftTable(_blocks_to_shift(blocks_y, Nvy), W_y.detach().cpu().numpy(), f.dtype, f.device))
        spectral = _spectral(grid_kx, grid_ky, grid_inv_ksq, f.device)
    # dx, dy only enter the diagnostics, which this entry point does not return
    return _fused_step(f, dt, tables, spectral, 1.0, 1.0, grid_dvx, grid_dvy, physics_mode, S, key)


def vlasov_step_gather_free(f, f0, dt, grid_x, grid_y, grid_vx, grid_vy, grid_kx, grid_ky, grid_inv_ksq,
                            grid_x_indices, grid_y_indices, grid_vx_indices, grid_vy_indices, grid_stencil_offsets,
                            grid_dx, grid_dy, grid_dvx, grid_dvy, grid_Nx, grid_Ny, physics_mode, S=1):
    """Solver-2 Strang step (vlasov_step_gather_free, vlasov2D2V.py:1086-1132).
    Returns (f, delta_rho, phi) at the reference's mid-step time level."""
    _check_offsets(grid_stencil_offsets)
    key = _plan_key(f, dt, grid_vx, grid_vy, grid_kx, grid_dx, grid_dy, grid_dvx, grid_dvy, S)
    plan = _PLANS.get(key)
    tables = None if plan is not None else (
        ops.DriftTable.from_velocity(grid_vx, dt / 2.0, grid_dx, f.dtype, f.device),
        ops.DriftTable.from_velocity(grid_vy, dt / 2.0, grid_dy, f.dtype, f.device))
    spectral = None if plan is not None else _spectral(grid_kx, grid_ky, grid_inv_ksq, f.device)
    return _fused_step(f, dt, tables, spectral, grid_dx, grid_dy, grid_dvx, grid_dvy, physics_mode, S, key)


def vlasov_step_matrix_diag(f, f0, dt, grid_x, grid_y, grid_vx, grid_vy, grid_kx, grid_ky, grid_inv_ksq,
                            grid_x_indices, grid_y_indices, grid_vx_indices, grid_vy_indices, grid_stencil_offsets,
                            grid_dx, grid_dy, grid_dvx, grid_dvy, grid_Nx, grid_Ny, physics_mode):
    """Solver-1 step (vlasov2D2V.py:1001-1040): per-line shifts and weights
    with exact (unwindowed) kicks, i.e. the fused step with S unbounded."""
    return vlasov_step_gather_free(f, f0, dt, grid_x, grid_y, grid_vx, grid_vy, grid_kx, grid_ky, grid_inv_ksq,
                                   grid_x_indices, grid_y_indices, grid_vx_indices, grid_vy_indices,
                                   grid_stencil_offsets, grid_dx, grid_dy, grid_dvx, grid_dvy, grid_Nx, grid_Ny,
                                   physics_mode, S=-1)


# ---------------------------------------------------------------------------
# driver (vlasov2D2V.py:1223-1435)
# ---------------------------------------------------------------------------
class Vlasov:
    """Driver with the reference's constructor arguments (vlasov2D2V.py:1236-1240).

    Extra keyword arguments: device, window (kick window S of solver 2;
    default 1 as in the reference, -1 = exact kick), graph (capture the step
    loop in CUDA graphs), dtype may also be "bfloat16" (BF16 storage with
    FP32 arithmetic). After run(), `history` holds one row of diagnostics
    per step (field energy, mass, L2, kinetic energy, ...; see
    include/vlasov_b200.h VP_DIAG_*).
    """

    def __init__(self, Nx=32, Ny=32, Nvx=32, Nvy=32, Lx=2.0 * math.pi, Ly=2.0 * math.pi, Vx_max=6.0, Vy_max=6.0,
                 nbiter=10, diag_steps=10, dt=0.05, out_dir="data", physics_mode=False, epsilon=0.001,
                 dtype: str = "float32", solver: int = 0, device=None, window: int = 1, graph: bool = True,
                 write_snapshots: bool = True):
        self.output_log = ""
        self.dtype = {"float32": torch.float32, "float64": torch.float64, "bfloat16": torch.bfloat16}[dtype]
        self.device = _default_device() if device is None else torch.device(device)
        grid_dtype = torch.float64 if self.dtype == torch.float64 else torch.float32
        self.grid = Grid.create(Nx, Ny, Nvx, Nvy, Lx, Ly, Vx_max, Vy_max, device=self.device, dtype=grid_dtype)
        self.nbiter = nbiter
        self.diag_steps = diag_steps
        self.dt = dt
        self.out_dir = out_dir
        self.physics_mode = physics_mode
        self.epsilon = epsilon
        self.solver = solver
        self.solver_type = {0: "vlasov_step_impl", 1: "vlasov_step_matrix_diag", 2: "vlasov_step_gather_free"}[solver]
        self.graph = graph
        self.write_snapshots = write_snapshots
        self.history = None
        self.stepper = Stepper2D(Nx, Ny, Nvx, Nvy, Lx, Ly, Vx_max, Vy_max, dt, dtype=self.dtype, device=self.device,
                                 physics_mode=physics_mode, window=(window if solver == 2 else -1), diagnostics=True,
                                 vx=self.grid.vx.cpu(), vy=self.grid.vy.cpu())
        if write_snapshots:
            pathlib.Path(self.out_dir).mkdir(parents=True, exist_ok=True)
        self._append_log(f"vlasov_b200 {L.load().vp_version().decode()}; torch {torch.__version__}")
        self._append_log(f"Starting simulation on {self.device} with {self.dtype} storage "
                         + ("with Poisson solver" if physics_mode else "without Poisson solver")
                         + f" and solver type {self.solver_type}.")
        self._append_log(f"Grid: {Nx}x{Ny}x{Nvx}x{Nvy}, Steps: {nbiter}, diag_freq: {diag_steps}")

    def _append_log(self, message: str) -> None:
        self.output_log += f"{message}\n"

    def initialize(self) -> SimulationState:
        """Initial state (vlasov2D2V.py:1319-1355): Landau (1 + eps cos kx cos ky)
        e^{-v^2/2}/sqrt(2 pi) with physics_mode, else the Gaussian pulse."""
        g = self.grid
        x = g.x[:, None, None, None].double()
        y = g.y[None, :, None, None].double()
        vx = g.vx[:, None].double()
        vy = g.vy[None, :].double()
        if self.physics_mode:
            kxm, kym = 2.0 * math.pi / g.Lx, 2.0 * math.pi / g.Ly
            f0 = (1.0 / math.sqrt(2.0 * math.pi)) * torch.exp(-0.5 * (vx ** 2 + vy ** 2))
            space = (1.0 + self.epsilon * torch.cos(kxm * x) * torch.cos(kym * y))[:, :, 0, 0]
            f = ops.init_product(space, f0, self.dtype)
        else:
            sx, sv = g.Lx / 10.0, g.Vx_max / 4.0
            f = torch.exp(-0.5 * ((x - g.Lx / 2) ** 2 / sx ** 2 + (y - g.Ly / 2) ** 2 / sx ** 2
                                  + vx[None, None] ** 2 / sv ** 2 + vy[None, None] ** 2 / sv ** 2))
            f0 = torch.zeros((g.Nvx, g.Nvy), dtype=torch.float64, device=self.device)
        f = f.to(self.dtype).contiguous()
        rho = ops.velocity_moment(f, g.dvx, g.dvy, 2)
        kx, ky, inv = _spectral(g.kx, g.ky, g.inv_ksq, self.device)
        _, _, drho, phi = ops.poisson2d(rho, kx, ky, inv)
        state = SimulationState(Field(drho, phi), Variables(f, f0.to(_out_dtype(f))), 0.0, 0)
        self.save_diag(state)
        return state

    def save_diag(self, state: SimulationState) -> None:
        """Snapshot of f, f0, rho, phi with coordinates and attributes, as
        field_{step:06d}.npz (the reference writes the same variables to netCDF)."""
        if not self.write_snapshots:
            return
        from .snapshot import write_snapshot_2d
        write_snapshot_2d(pathlib.Path(self.out_dir) / f"field_{int(state.step):06d}.npz", state, self)

    def run(self, state: SimulationState) -> SimulationState:
        """Advance nbiter steps (vlasov2D2V.py:1392-1435), writing a snapshot
        every diag_steps. Solver 2 (and 1) run the fused step, captured in
        CUDA graphs between snapshots; solver 0 runs the per-element sweeps."""
        g = self.grid
        st = self.stepper
        f = state.variables.fn.contiguous()
        hist = torch.zeros((self.nbiter, L.DIAG_COUNT), dtype=torch.float64, device=self.device)
        done = 0
        while done < self.nbiter:
            n = min(self.diag_steps, self.nbiter - done)
            if self.solver == 0:
                for i in range(n):
                    f, drho, phi = vlasov_step_impl(
                        f, state.variables.f0, self.dt, g.x, g.y, g.vx, g.vy, g.kx, g.ky, g.inv_ksq, g.x_indices,
                        g.y_indices, g.vx_indices, g.vy_indices, g.stencil_offsets, g.dx, g.dy, g.dvx, g.dvy,
                        g.Nx, g.Ny, self.physics_mode)
                rho_out, phi_out = drho, phi
            else:
                f = st.run(f, n, history=hist[done: done + n], graph=self.graph and n >= 4)
                rho_out = st.drho.to(_out_dtype(f), copy=True)
                phi_out = st.phi.to(_out_dtype(f), copy=True)
            done += n
            state = SimulationState(Field(rho_out, phi_out), Variables(f, state.variables.f0),
                                    state.t + n * self.dt, state.step + n)
            if n == self.diag_steps:
                self.save_diag(state)
        torch.cuda.synchronize(self.device)
        self.history = hist
        return state
