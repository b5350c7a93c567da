"""x-slab decomposition of one 2D2V run over several GPUs (one process each).

The reference runs one device; this module splits a single large run along
x, the only axis whose drift crosses a slab boundary (the y drift and both
kicks act inside each (x, y) plane or x row).

Rank r of R owns the rows [x0, x1) of f[Nx][Ny][Nvx][Nvy] and keeps them in
an extended buffer with hl rows before and hr rows after, all of them
periodic on the buffer's own length. The library's periodic sweeps then run
on that buffer unchanged: an output row whose stencil window stays inside
the buffer gets exactly the inputs the whole domain would give it, so it is
bit-identical to the one-GPU step. One x half-drift reads the rows
x - s - 3 .. x - s + 2 (s = the drift table's shift); a step has two of them
with only row-local work in between, so the halo is twice one drift's reach
on each side, refreshed once per step from the two ring neighbours. Halo
rows come out of a step wrong and are overwritten by the next exchange.

The field: every rank sums rho on its own rows (the fused y-drift epilogue),
the slabs' rho are all-gathered (Nx*Ny float64, 128 KiB at 128^2) and every
rank solves the small Poisson problem for the whole domain, so the kick of
every local row (halo rows included) uses the global field.

Where the layout allows (FP32, 16 <= Ny <= 128, Nvy a multiple of 32) each
pair of position drifts runs as one fused pass over the extended buffer
(vp_drift_pair), as the one-GPU step does. The halo exchange then overlaps the
first pass: the rows whose x windows stay inside the rank's own rows are
computed while the halo rows are in flight, the rows next to the halo after
they have arrived.

`SlabPlan` is pure host logic; `exchange_halos` / `gather_rho` take a
torch.distributed process group (NCCL for CUDA tensors, gloo for CPU ones);
`SlabStepper2D` runs the two halves of a step around the field solve on the
library's kernels, so a driver can also emulate ranks in one process.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch
import torch.distributed as dist

from . import _lib as L
from . import ops


def drift_reach(shift: np.ndarray) -> tuple[int, int]:
    """Rows one periodic drift reads before and after an output row, for the
    shifts of its table (window rows x - s - 3 .. x - s + 2)."""
    s = np.asarray(shift, dtype=np.int64)
    return max(0, int(s.max()) + 3), max(0, 2 - int(s.min()))


@dataclass(frozen=True)
class SlabPlan:
    """Rows of every rank, with the halo widths of a whole step."""
    nx: int
    ranks: int
    hl: int  # halo rows before the slab
    hr: int  # halo rows after the slab
    starts: tuple  # first global row of each rank, and nx at the end

    @classmethod
    def build(cls, nx: int, ranks: int, shift_x: np.ndarray) -> "SlabPlan":
        if ranks < 1 or nx < ranks:
            raise ValueError(f"cannot split {nx} x rows over {ranks} ranks")
        lo, hi = drift_reach(shift_x)
        hl, hr = 2 * lo, 2 * hi  # two x half-drifts per step
        starts = tuple(nx * r // ranks for r in range(ranks + 1))
        smallest = min(starts[r + 1] - starts[r] for r in range(ranks))
        if ranks > 1 and smallest < max(hl, hr):
            raise ValueError(f"slabs of {smallest} rows are thinner than the halo ({hl}, {hr}): use fewer ranks")
        return cls(nx, ranks, hl, hr, starts)

    def rows(self, r: int) -> tuple[int, int]:
        return self.starts[r], self.starts[r + 1]

    def local(self, r: int) -> int:
        return self.starts[r + 1] - self.starts[r]

    def extended(self, r: int) -> int:
        return self.local(r) + self.hl + self.hr

    def global_rows(self, r: int) -> np.ndarray:
        """Global row of every row of rank r's extended buffer."""
        x0, _ = self.rows(r)
        return (x0 - self.hl + np.arange(self.extended(r))) % self.nx

    def halo_sources(self, r: int) -> list[tuple[int, int, int, int]]:
        """(source rank, its first slab row, row count, first extended row of
        rank r to fill) for the halo of rank r, in the order before, after."""
        left, right = (r - 1) % self.ranks, (r + 1) % self.ranks
        out = []
        if self.hl:
            out.append((left, self.local(left) - self.hl, self.hl, 0))
        if self.hr:
            out.append((right, 0, self.hr, self.hl + self.local(r)))
        return out


def _slab(f_ext: torch.Tensor, plan: SlabPlan, r: int) -> torch.Tensor:
    return f_ext[plan.hl:plan.hl + plan.local(r)]


def start_halo_exchange(f_ext: torch.Tensor, plan: SlabPlan, rank: int, group=None) -> list:
    """Start filling the halo rows of this rank's extended buffer from its ring
    neighbours' slab rows (point-to-point over the process group; a single
    rank copies its own rows at once). Returns the requests to wait on; until
    then the halo rows must not be read nor the slab rows written. With NCCL
    the transfers run on the library's own stream, so kernels launched on the
    current stream meanwhile overlap them."""
    slab = _slab(f_ext, plan, rank)
    if plan.ranks == 1:
        # the halo may be wider than the line itself: gather by global row
        n, ext = plan.local(0), plan.extended(0)
        halo = torch.cat([torch.arange(0, plan.hl), torch.arange(plan.hl + n, ext)]).to(f_ext.device)
        rows = torch.as_tensor(plan.global_rows(0), device=f_ext.device)
        f_ext[halo] = slab[rows[halo]]
        return []
    left, right = (rank - 1) % plan.ranks, (rank + 1) % plan.ranks
    ops_ = []
    # my last hl rows are the right neighbour's "before" halo, my first hr
    # rows the left neighbour's "after" halo
    if plan.hl:
        ops_.append(dist.P2POp(dist.isend, slab[plan.local(rank) - plan.hl:].contiguous(), right, group))
        ops_.append(dist.P2POp(dist.irecv, f_ext[0:plan.hl], left, group))
    if plan.hr:
        ops_.append(dist.P2POp(dist.isend, slab[:plan.hr].contiguous(), left, group))
        ops_.append(dist.P2POp(dist.irecv, f_ext[plan.hl + plan.local(rank):], right, group))
    return list(dist.batch_isend_irecv(ops_))


def finish_halo_exchange(reqs: list) -> None:
    """Wait for the requests of start_halo_exchange (with NCCL: the current
    stream waits for the transfers)."""
    for req in reqs:
        req.wait()


def exchange_halos(f_ext: torch.Tensor, plan: SlabPlan, rank: int, group=None) -> None:
    """Fill the halo rows of this rank's extended buffer (start and wait)."""
    finish_halo_exchange(start_halo_exchange(f_ext, plan, rank, group))


def gather_rho(rho_slab: torch.Tensor, plan: SlabPlan, group=None) -> torch.Tensor:
    """All ranks' rho rows in global order, (Nx, Ny) float64."""
    if plan.ranks == 1:
        return rho_slab
    pad = max(plan.local(r) for r in range(plan.ranks))
    buf = torch.zeros((pad,) + tuple(rho_slab.shape[1:]), dtype=rho_slab.dtype, device=rho_slab.device)
    buf[:rho_slab.shape[0]].copy_(rho_slab)
    parts = [torch.empty_like(buf) for _ in range(plan.ranks)]
    dist.all_gather(parts, buf, group=group)
    return torch.cat([parts[r][:plan.local(r)] for r in range(plan.ranks)])


class SlabStepper2D:
    """One rank's share of a 2D2V Strang step (the schedule of vp_step2d: x,
    y + rho, field, fused kick, y, x; each drift pair as one fused pass where
    the layout allows, else one sweep per axis), on the extended buffer of
    `SlabPlan`. The same arguments as engine.Stepper2D, for the whole domain;
    fuse_drifts=False keeps one sweep per axis."""

    def __init__(self, plan: SlabPlan, rank: int, Nx, Ny, Nvx, Nvy, Lx, Ly, Vx_max, Vy_max, dt,
                 dtype=torch.float32, device="cuda", window=-1, fuse_drifts=True):
        if Nx != plan.nx:
            raise ValueError("the plan is for another Nx")
        self.plan, self.rank = plan, rank
        self.shape = (plan.extended(rank), int(Ny), int(Nvx), int(Nvy))
        self.dtype, self.device = dtype, torch.device(device)
        self.dt, self.window = float(dt), int(window)
        self.dx, self.dy = float(Lx) / Nx, float(Ly) / Ny
        self.dvx, self.dvy = 2 * Vx_max / (Nvx - 1), 2 * Vy_max / (Nvy - 1)
        grid_dt = torch.float64 if dtype == torch.float64 else torch.float32
        vx = torch.linspace(-Vx_max, Vx_max, Nvx, dtype=grid_dt)
        vy = torch.linspace(-Vy_max, Vy_max, Nvy, dtype=grid_dt)
        self.tx = ops.DriftTable.from_velocity(vx, self.dt / 2.0, self.dx, dtype, self.device)
        self.ty = ops.DriftTable.from_velocity(vy, self.dt / 2.0, self.dy, dtype, self.device)
        self.kx, self.ky, self.inv_ksq = ops.spectral_2d(Nx, Ny, float(Lx), float(Ly), self.device)
        self.rows = torch.as_tensor(plan.global_rows(rank), device=self.device)
        # the fused drift pairs (vp_drift_pair's layout conditions)
        self.fused = bool(fuse_drifts) and dtype == torch.float32 and 16 <= Ny <= 128 and Nvy % 32 == 0
        # first-pass rows whose x windows stay inside the rank's own rows
        lo, hi = drift_reach(self.tx.shift.cpu().numpy())
        a, b = plan.hl + lo, plan.hl + plan.local(rank) - hi
        self.interior = (a, b - a) if b > a else None

    @staticmethod
    def plan_for(Nx, ranks, Lx, Vx_max, Nvx, dt, dtype=torch.float32) -> SlabPlan:
        """The plan of a run (its x drift table decides the halo)."""
        grid_dt = torch.float64 if dtype == torch.float64 else torch.float32
        vx = torch.linspace(-Vx_max, Vx_max, Nvx, dtype=grid_dt)
        shift, _ = ops.drift_table_np(vx, float(dt) / 2.0, float(Lx) / Nx, dtype)
        return SlabPlan.build(Nx, ranks, shift)

    def empty(self) -> torch.Tensor:
        return torch.empty(self.shape, dtype=self.dtype, device=self.device)

    def first_half(self, f_ext: torch.Tensor):
        """x and y drifts of the extended buffer (its halo filled): the
        drifted buffer and this rank's rho rows."""
        if self.fused:
            b, rho = ops.drift_pair(f_ext, self.tx, self.ty, True, scale=self.dvx * self.dvy)
            return b, _slab(rho, self.plan, self.rank)
        a = ops.drift(f_ext, self.tx, 0, 2)
        b, rho = ops.drift_rho(a, self.ty, 1, 3, self.dvx * self.dvy)
        return b, _slab(rho, self.plan, self.rank)

    def first_half_overlapped(self, f_ext: torch.Tensor, reqs: list):
        """first_half while the halo exchange `reqs` is in flight: the interior
        rows first, then (after the exchange) the rows next to the halo. The
        same results as first_half after the exchange."""
        if not self.fused or self.interior is None:
            finish_halo_exchange(reqs)
            return self.first_half(f_ext)
        ext = self.shape[0]
        i0, n = self.interior
        scale = self.dvx * self.dvy
        b, rho = ops.drift_pair(f_ext, self.tx, self.ty, True, rows=(i0, n), scale=scale)
        finish_halo_exchange(reqs)
        if i0 > 0:
            ops.drift_pair(f_ext, self.tx, self.ty, True, out=b, rows=(0, i0), scale=scale, rho=rho)
        if i0 + n < ext:
            ops.drift_pair(f_ext, self.tx, self.ty, True, out=b, rows=(i0 + n, ext - i0 - n), scale=scale, rho=rho)
        return b, _slab(rho, self.plan, self.rank)

    def field(self, rho_global: torch.Tensor):
        """The global field from the gathered rho: (Ex, Ey, drho, phi)."""
        return ops.poisson2d(rho_global, self.kx, self.ky, self.inv_ksq)

    def second_half(self, b: torch.Tensor, Ex: torch.Tensor, Ey: torch.Tensor, out: torch.Tensor | None = None):
        """Kicks with the global field on every local row, then y and x."""
        c = ops.kick2d(b, Ex[self.rows], Ey[self.rows], self.dt, self.dvx, self.dvy, self.window)
        if self.fused:
            return ops.drift_pair(c, self.tx, self.ty, False, out=out)[0]
        d = ops.drift(c, self.ty, 1, 3)
        return ops.drift(d, self.tx, 0, 2, out=out)

    def step(self, f_ext: torch.Tensor, group=None, out: torch.Tensor | None = None):
        """One step over the process group: halo exchange (overlapped with the
        interior of the first pass where the drifts are fused), first half, rho
        all-gather, field, second half. Returns (f_ext', drho, phi)."""
        L.require_cuda(f_ext)
        reqs = start_halo_exchange(f_ext, self.plan, self.rank, group)
        b, rho = self.first_half_overlapped(f_ext, reqs)
        Ex, Ey, drho, phi = self.field(gather_rho(rho, self.plan, group))
        return self.second_half(b, Ex, Ey, out), drho, phi


    def run(self, f_ext: torch.Tensor, nsteps: int, group=None) -> torch.Tensor:
        """nsteps steps over the process group; returns the extended buffer
        (its slab rows are this rank's share of f)."""
        out = self.empty()
        for _ in range(nsteps):
            res, _, _ = self.step(f_ext, group, out)
            f_ext, out = res, f_ext
        return f_ext


def scatter(f: torch.Tensor, plan: SlabPlan, r: int) -> torch.Tensor:
    """Rank r's extended buffer cut from a whole-domain f (halo included)."""
    return f[torch.as_tensor(plan.global_rows(r), device=f.device)].contiguous()


def slab_rows(f_ext: torch.Tensor, plan: SlabPlan, r: int) -> torch.Tensor:
    """The rows rank r owns, from its extended buffer."""
    return _slab(f_ext, plan, r)


__all__ = ["SlabPlan", "SlabStepper2D", "drift_reach", "exchange_halos", "finish_halo_exchange", "gather_rho",
           "scatter", "slab_rows", "start_halo_exchange"]
