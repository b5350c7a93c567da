"""Tensor-level wrappers of the C ABI: every function here launches the
library's CUDA kernels on the current torch stream of its inputs' device.

Shapes follow the reference solver: f is (Nx, Ny, Nvx, Nvy) for 2D2V and
(Nx, Nv) for 1D1V, contiguous; a sweep along `axis` views f as
[n_outer][n_line][n_inner] (see include/vlasov_b200.h).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib as L

# ---------------------------------------------------------------------------
# scratch memory owned by the host side (the library never allocates)
# ---------------------------------------------------------------------------
_WS: dict = {}


def workspace(device: torch.device, nbytes: int, tag: str = "default") -> torch.Tensor:
    """A cached uint8 scratch buffer of at least nbytes on device for the
    current stream. Calls on one stream are ordered, so they may share it."""
    key = (device, torch.cuda.current_stream(device).cuda_stream, tag)
    buf = _WS.get(key)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
        _WS[key] = buf
    return buf


def _olc(shape, axis):
    n_outer = int(np.prod(shape[:axis], dtype=np.int64))
    n_inner = int(np.prod(shape[axis + 1:], dtype=np.int64))
    return n_outer, int(shape[axis]), n_inner


# ---------------------------------------------------------------------------
# drift tables (precompute_x_drift, vlasov2D2V.py:670-714)
# ---------------------------------------------------------------------------
def lagrange5_weights_np(alpha: np.ndarray) -> np.ndarray:
    """The 6-point Lagrange weights of fraction alpha, with the closed-form
    polynomials and operation order of lagrange5_weights
    (vlasov2D2V.py:263-285), in alpha's own precision. Returns (6, n)."""
    a = np.asarray(alpha)
    T = a.dtype.type
    a2 = a * a
    a3 = a2 * a
    a4 = a3 * a
    a5 = a4 * a
    w0 = (a / T(20.0)) - (a2 / T(24.0)) - (a3 / T(24.0)) + (a4 / T(24.0)) - (a5 / T(120.0))
    w1 = -(a / T(2.0)) + (T(2.0) * a2 / T(3.0)) - (a3 / T(24.0)) - (a4 / T(6.0)) + (a5 / T(24.0))
    w2 = T(1.0) - (a / T(3.0)) - (T(5.0) * a2 / T(4.0)) + (T(5.0) * a3 / T(12.0)) + (a4 / T(4.0)) - (a5 / T(12.0))
    w3 = a + (T(2.0) * a2 / T(3.0)) - (T(7.0) * a3 / T(12.0)) - (a4 / T(6.0)) + (a5 / T(12.0))
    w4 = -(a / T(4.0)) - (a2 / T(24.0)) + (T(7.0) * a3 / T(24.0)) + (a4 / T(24.0)) - (a5 / T(24.0))
    w5 = (a / T(30.0)) - (a3 / T(24.0)) + (a5 / T(120.0))
    return np.stack([w0, w1, w2, w3, w4, w5]).astype(a.dtype)


def drift_table_np(v, dt: float, dx: float, dtype: torch.dtype):
    """Integer shift s = floor((v*dt)/dx) and weights of the fraction, in the
    precision of `dtype` (float64 for float64 runs, else float32)."""
    np_t = np.float64 if dtype == torch.float64 else np.float32
    T = np.dtype(np_t).type
    vn = (v.detach().cpu().numpy() if torch.is_tensor(v) else np.asarray(v)).astype(np_t)
    d = (vn * T(dt)) / T(dx)
    s = np.floor(d)
    alpha = d - s
    return s.astype(np.int64), lagrange5_weights_np(alpha.astype(np_t))


def group_spread(shift: np.ndarray, group: int = 4) -> int:
    """max(shift) - min(shift) over aligned groups of `group` entries, or -1
    when the table does not split into such groups (vp_drift's shift_spread)."""
    s = np.asarray(shift, dtype=np.int64)
    if s.size == 0 or s.size % group:
        return -1
    g = s.reshape(-1, group)
    return int((g.max(axis=1) - g.min(axis=1)).max())


class DriftTable:
    """Device copy of one drift table: shift int32[Nv], W compute-type [6][Nv]."""

    def __init__(self, shift: np.ndarray, W: np.ndarray, dtype: torch.dtype, device):
        if np.abs(shift).max(initial=0) >= 2 ** 30:
            raise ValueError("drift shift out of range")
        self.n = int(shift.shape[0])
        self.spread = group_spread(shift)
        self.shift = torch.as_tensor(shift.astype(np.int32), device=device)
        self.W = torch.as_tensor(np.ascontiguousarray(W), device=device).to(L.compute_dtype(dtype)).contiguous()

    @classmethod
    def from_velocity(cls, v, dt, dx, dtype, device, precise=False):
        """precise: evaluate shift and weights in float64 and round only the
        weights to the compute type (the reference evaluates them in the run
        precision, which for float32 also rounds the velocity grid)."""
        s, W = drift_table_np(v, dt, dx, torch.float64 if precise else dtype)
        return cls(s, W, dtype, device)


# ---------------------------------------------------------------------------
# sweeps
# ---------------------------------------------------------------------------
def drift(f: torch.Tensor, table: DriftTable, axis: int, vel_axis: int, out: torch.Tensor | None = None):
    """Periodic drift of f along `axis`; column shifts indexed by `vel_axis`."""
    L.require_cuda(f)
    out = torch.empty_like(f) if out is None else out
    n_outer, n_line, n_inner = _olc(f.shape, axis)
    sel_div = int(np.prod(f.shape[vel_axis + 1:], dtype=np.int64))
    sel_mod = int(f.shape[vel_axis])
    if table.n != sel_mod:
        raise ValueError(f"drift table has {table.n} entries, axis {vel_axis} has {sel_mod}")
    L.call("vp_drift", L.ptr(f), L.ptr(out), L.dtype_code(f.dtype), n_outer, n_line, n_inner, sel_div, sel_mod,
           L.ptr(table.shift), table.spread, L.ptr(table.W), L.stream_of(f))
    return out


def drift_rho(f: torch.Tensor, table: DriftTable, axis: int, vel_axis: int, scale: float,
              out: torch.Tensor | None = None, rho: torch.Tensor | None = None):
    """drift() fused with rho[o, l] = scale * sum over the trailing dims (FP64)."""
    L.require_cuda(f)
    out = torch.empty_like(f) if out is None else out
    n_outer, n_line, n_inner = _olc(f.shape, axis)
    sel_div = int(np.prod(f.shape[vel_axis + 1:], dtype=np.int64))
    sel_mod = int(f.shape[vel_axis])
    if rho is None:
        rho = torch.empty(f.shape[: axis + 1], dtype=torch.float64, device=f.device)
    nb = L.query("vp_drift_rho_workspace_bytes", n_outer, n_line, n_inner)
    ws = workspace(f.device, nb)
    L.call("vp_drift_rho", L.ptr(f), L.ptr(out), L.dtype_code(f.dtype), n_outer, n_line, n_inner, sel_div, sel_mod,
           L.ptr(table.shift), table.spread, L.ptr(table.W), float(scale), L.ptr(rho), L.ptr(ws), ws.numel(),
           L.stream_of(f))
    return out, rho


def drift_pair(f: torch.Tensor, tx: DriftTable, ty: DriftTable, xfirst: bool, out: torch.Tensor | None = None,
               rows: tuple[int, int] | None = None, scale: float | None = None, rho: torch.Tensor | None = None):
    """Both position drifts of f[Nx][Ny][Nvx][Nvy] in one pass (x then y or
    y then x; vp_drift_pair). rows = (first, count) restricts the output rows
    (default all); with xfirst and `scale` the density of those rows goes into
    rho[Nx, Ny] (float64, allocated if None). Returns (out, rho or None).
    Raises VlasovError (VP_ERR_UNSUPPORTED) when the layout does not fit."""
    L.require_cuda(f)
    out = torch.empty_like(f) if out is None else out
    Nx, Ny, Nvx, Nvy = f.shape
    x0, nrows = rows if rows is not None else (0, Nx)
    ws = None
    if scale is not None:
        if not xfirst:
            raise ValueError("the density comes with the x-then-y order")
        if rho is None:
            rho = torch.empty((Nx, Ny), dtype=torch.float64, device=f.device)
        nb = L.query("vp_drift_pair_workspace_bytes", Nx, Ny, Nvx, Nvy)
        ws = workspace(f.device, nb, "drift_pair")
    L.call("vp_drift_pair", L.ptr(f), L.ptr(out), L.dtype_code(f.dtype), Nx, Ny, Nvx, Nvy, 1 if xfirst else 0,
           int(x0), int(nrows), L.ptr(tx.shift), L.ptr(tx.W), L.ptr(ty.shift), L.ptr(ty.W),
           float(scale) if scale is not None else 1.0, L.ptr(rho) if scale is not None else None,
           L.ptr(ws), ws.numel() if ws is not None else 0, L.stream_of(f))
    return out, (rho if scale is not None else None)


def kick(f: torch.Tensor, E: torch.Tensor, dt: float, dv: float, axis: int, window: int = -1,
         out: torch.Tensor | None = None):
    """Dirichlet kick along `axis` with a field E over the leading dims
    (E.numel() must divide the product of the dims before `axis`)."""
    L.require_cuda(f, E)
    out = torch.empty_like(f) if out is None else out
    n_outer, n_line, n_inner = _olc(f.shape, axis)
    if E.dtype not in (torch.float32, torch.float64):
        E = E.to(torch.float64)
    E = E.contiguous()
    if E.numel() == 0 or n_outer % E.numel():
        raise ValueError(f"field of {E.numel()} values does not tile {n_outer} rows")
    e_div = n_outer // E.numel()
    L.call("vp_kick", L.ptr(f), L.ptr(out), L.dtype_code(f.dtype), n_outer, n_line, n_inner, L.ptr(E),
           L.VP_F64 if E.dtype == torch.float64 else L.VP_F32, e_div, float(dt), float(dv), int(window),
           L.stream_of(f))
    return out


def kick2d(f: torch.Tensor, Ex: torch.Tensor, Ey: torch.Tensor, dt: float, dvx: float, dvy: float,
           window: int = -1, out: torch.Tensor | None = None, vx=None, vy=None, moments=None):
    """Both kicks of a 2D2V step in one pass (Ex, Ey float64 (Nx, Ny))."""
    L.require_cuda(f, Ex, Ey)
    out = torch.empty_like(f) if out is None else out
    Nx, Ny, Nvx, Nvy = f.shape
    L.call("vp_kick2d", L.ptr(f), L.ptr(out), L.dtype_code(f.dtype), Nx * Ny, Nvx, Nvy,
           L.ptr(Ex.to(torch.float64).contiguous()), L.ptr(Ey.to(torch.float64).contiguous()), float(dt), float(dvx),
           float(dvy), int(window), L.ptr(vx), L.ptr(vy), L.ptr(moments), L.stream_of(f))
    return out


def advect_gather(f: torch.Tensor, vel: torch.Tensor, axis: int, dt: float, dx: float, periodic: bool,
                  out: torch.Tensor | None = None, vel_strides=None):
    """Per-element departure sweep. vel is broadcast to the batch shape (every
    dim but `axis`) unless explicit (outer, line, inner) strides are given."""
    L.require_cuda(f, vel)
    out = torch.empty_like(f) if out is None else out
    n_outer, n_line, n_inner = _olc(f.shape, axis)
    cdt = L.compute_dtype(f.dtype)
    if vel_strides is None:
        batch = tuple(f.shape[:axis]) + tuple(f.shape[axis + 1:])
        vel = vel.to(cdt).expand(batch).contiguous()
        vel_strides = (n_inner, 0, 1)
    else:
        vel = vel.to(cdt).contiguous()
    L.call("vp_advect_gather", L.ptr(f), L.ptr(out), L.dtype_code(f.dtype), n_outer, n_line, n_inner, L.ptr(vel),
           int(vel_strides[0]), int(vel_strides[1]), int(vel_strides[2]), float(dt), float(dx),
           1 if periodic else 0, L.stream_of(f))
    return out


def init_product(space: torch.Tensor, vel: torch.Tensor, dtype: torch.dtype) -> torch.Tensor:
    """f = space (x) vel: shape space.shape + vel.shape, each element the FP64
    product space[p] * vel[v] rounded once to dtype (the drivers' initial
    conditions, vlasov2D2V.py:1319-1355; the same bits as
    (space[..., None] * vel).to(dtype))."""
    L.require_cuda(space)
    s = space.to(torch.float64).contiguous()
    v = vel.to(device=space.device, dtype=torch.float64).contiguous()
    f = torch.empty(tuple(space.shape) + tuple(vel.shape), dtype=dtype, device=space.device)
    L.call("vp_init_product", L.ptr(s), L.ptr(v), L.ptr(f), L.dtype_code(dtype), s.numel(), v.numel(),
           L.stream_of(f))
    return f


def velocity_moment(f: torch.Tensor, dvx: float, dvy: float, n_v_dims: int, out_dtype=torch.float64):
    """sum over the trailing n_v_dims dims, times dvx*dvy (FP64 accumulation)."""
    L.require_cuda(f)
    lead = tuple(f.shape[: f.dim() - n_v_dims])
    n_v = int(np.prod(f.shape[f.dim() - n_v_dims:], dtype=np.int64))
    n_points = int(np.prod(lead, dtype=np.int64))
    if out_dtype not in (torch.float32, torch.float64):
        out_dtype = torch.float32
    rho = torch.empty(lead, dtype=out_dtype, device=f.device)
    L.call("vp_rho", L.ptr(f), L.dtype_code(f.dtype), n_points, n_v, float(dvx), float(dvy), L.ptr(rho),
           L.VP_F64 if out_dtype == torch.float64 else L.VP_F32, L.stream_of(f))
    return rho


# ---------------------------------------------------------------------------
# field solves (FP64)
# ---------------------------------------------------------------------------
def spectral_2d(Nx: int, Ny: int, Lx: float, Ly: float, device):
    """kx (Nx,), ky (Ny//2+1,), inv_ksq (Nx, Ny//2+1) in float64, as Grid.create
    builds them (vlasov2D2V.py:158-162)."""
    dx, dy = Lx / Nx, Ly / Ny
    kx = 2 * math.pi * torch.fft.fftfreq(Nx, d=dx, dtype=torch.float64)
    ky = 2 * math.pi * torch.fft.rfftfreq(Ny, d=dy, dtype=torch.float64)
    ksq = kx[:, None] ** 2 + ky[None, :] ** 2
    inv = torch.where(ksq == 0, torch.tensor(0.0, dtype=torch.float64), 1.0 / ksq)
    return kx.to(device), ky.to(device), inv.contiguous().to(device)


def poisson2d(rho: torch.Tensor, kx: torch.Tensor, ky: torch.Tensor, inv_ksq: torch.Tensor, dx: float = 1.0,
              dy: float = 1.0, want_energy: bool = False):
    """(Ex, Ey, delta_rho, phi[, energy]) in float64 from rho (float64 (Nx, Ny))."""
    L.require_cuda(rho)
    rho = rho.to(torch.float64).contiguous()
    Nx, Ny = rho.shape
    kx = kx.reshape(-1).to(device=rho.device, dtype=torch.float64).contiguous()
    ky = ky.reshape(-1).to(device=rho.device, dtype=torch.float64).contiguous()
    inv_ksq = inv_ksq.to(device=rho.device, dtype=torch.float64).contiguous()
    if kx.numel() != Nx or ky.numel() != Ny // 2 + 1 or tuple(inv_ksq.shape) != (Nx, Ny // 2 + 1):
        raise ValueError("spectral arrays do not match rho's shape")
    ex = torch.empty_like(rho)
    ey = torch.empty_like(rho)
    drho = torch.empty_like(rho)
    phi = torch.empty_like(rho)
    energy = torch.empty(2, dtype=torch.float64, device=rho.device) if want_energy else None
    nb = L.query("vp_poisson2d_workspace_bytes", Nx, Ny)
    ws = workspace(rho.device, nb, "poisson")
    L.call("vp_poisson2d", L.ptr(rho), Nx, Ny, L.ptr(kx), L.ptr(ky), L.ptr(inv_ksq), float(dx), float(dy),
           L.ptr(ex), L.ptr(ey), L.ptr(drho), L.ptr(phi), L.ptr(energy), L.ptr(ws), ws.numel(), L.stream_of(rho))
    return (ex, ey, drho, phi, energy) if want_energy else (ex, ey, drho, phi)


def spectral_1d(Nx: int, Lx: float, device):
    dx = Lx / Nx
    kx = 2 * math.pi * torch.fft.rfftfreq(Nx, d=dx, dtype=torch.float64)
    inv = torch.where(kx == 0, torch.tensor(0.0, dtype=torch.float64), 1.0 / kx)
    return inv.to(device), (inv * inv).to(device)


def poisson1d(n: torch.Tensor, inv_kx: torch.Tensor, inv_kx_sq: torch.Tensor, dx: float = 1.0,
              want_energy: bool = False):
    """(E, rho, phi[, energy]) in float64 from the density n = sum(f, 1) * dv."""
    L.require_cuda(n)
    n = n.to(torch.float64).contiguous()
    Nx = n.numel()
    inv_kx = inv_kx.to(device=n.device, dtype=torch.float64).contiguous()
    inv_kx_sq = inv_kx_sq.to(device=n.device, dtype=torch.float64).contiguous()
    e = torch.empty_like(n)
    rho = torch.empty_like(n)
    phi = torch.empty_like(n)
    energy = torch.empty(2, dtype=torch.float64, device=n.device) if want_energy else None
    nb = L.query("vp_poisson1d_workspace_bytes", Nx)
    ws = workspace(n.device, nb, "poisson1d")
    L.call("vp_poisson1d", L.ptr(n), Nx, L.ptr(inv_kx), L.ptr(inv_kx_sq), float(dx), L.ptr(e), L.ptr(rho),
           L.ptr(phi), L.ptr(energy), L.ptr(ws), ws.numel(), L.stream_of(n))
    return (e, rho, phi, energy) if want_energy else (e, rho, phi)
