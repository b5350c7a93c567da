"""Learned correction of the interpolation weights (BF16 tensor-core
network, vp_mlp_kick / vp_mlp_drift and their training passes), its training
on pairs the method generates itself, and a coarse-grid stepper that uses it.

The network (see include/vlasov_b200.h): per cell, x = [f_k / max|f|,
alpha - 1/2, 1] -> 64 -> 64 -> 6 with ReLU, output dw (zero mean) added to
the 6 Lagrange weights of a sweep. On coarse grids the velocity kicks carry
almost all of the interpolation error (the periodic x / y drifts of the
smooth spatial profile are accurate to round-off), so the stepper corrects
the kicks; drift correction is available too. Plain Lagrange interpolation
stays the fallback: with W3 = 0 the correction vanishes.

Training data: a run on the 2x-refined grid (Nx, Ny doubled; Nv -> 2 Nv - 1
so that every coarse velocity is a fine one) is restricted to the coarse grid
(every second point); the pair (restricted state before a fine sweep,
restricted state after it) teaches the coarse sweep what the refined one
does. The forward and backward passes run in the project's own tcgen05
kernels; the optimizer (Adam) is a few elementwise torch operations on the
7,000 FP32 master weights.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib as L
from . import ops

HID, K1, K2, NO = 64, 16, 80, 16
NET_ELEMS = HID * K1 + HID * K2 + NO * K2 + HID * NO + HID * HID
GRAD_ELEMS = HID * K1 + HID * K2 + NO * K2


def alpha_table(v, dt: float, dx: float) -> np.ndarray:
    """Fractional drift shift d - floor(d), d = (v dt)/dx, in float32 (the
    arithmetic of precompute_x_drift, vlasov2D2V.py:670-714)."""
    vn = (v.detach().cpu().numpy() if torch.is_tensor(v) else np.asarray(v)).astype(np.float32)
    d = (vn * np.float32(dt)) / np.float32(dx)
    return (d - np.floor(d)).astype(np.float32)


class Corrector:
    """FP32 master weights, their packed BF16 copy, gradient and Adam state.

    The output layer is stored as W3 / w3_scale: the corrections the network
    must learn are small (the plain weights are already close), and the fixed
    scale keeps Adam's steps on W3 proportionate. out_scale: standard
    deviation of the initial (effective) W3 entries; 0 starts from the plain
    method."""

    def __init__(self, device="cuda", seed: int = 0, out_scale: float = 0.0, w3_scale: float = 1e-2):
        self.device = torch.device(device)
        self.w3_scale = float(w3_scale)
        g = torch.Generator().manual_seed(seed)
        W1 = torch.zeros(HID, K1)
        W1[:, :7] = torch.randn(HID, 7, generator=g) * math.sqrt(2.0 / 7.0)
        W2 = torch.zeros(HID, K2)
        W2[:, :HID] = torch.randn(HID, HID, generator=g) * math.sqrt(2.0 / HID)
        W3 = torch.zeros(NO, K2)
        W3[:6, :HID] = torch.randn(6, HID, generator=g) * (out_scale / self.w3_scale)
        self.params = torch.cat([W1.reshape(-1), W2.reshape(-1), W3.reshape(-1)]).to(self.device)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.t = 0
        self.net = torch.empty(NET_ELEMS, dtype=torch.bfloat16, device=self.device)
        self.grad = torch.zeros(GRAD_ELEMS, dtype=torch.float32, device=self.device)
        self.loss = torch.zeros(1, dtype=torch.float64, device=self.device)
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.pack()

    # views of the master weights
    @property
    def W1(self):
        return self.params[:HID * K1].view(HID, K1)

    @property
    def W2(self):
        return self.params[HID * K1: HID * K1 + HID * K2].view(HID, K2)

    @property
    def W3(self):
        """The effective output layer (w3_scale times the stored one)."""
        return self.params[HID * K1 + HID * K2:].view(NO, K2) * self.w3_scale

    def pack(self):
        """Refresh the BF16 network (W1, W2, W3 and the transposed copies)."""
        W3T = self.W3[:, :HID].t().contiguous()
        W2T = self.W2[:, :HID].t().contiguous()
        flat = torch.cat([self.W1.reshape(-1), self.W2.reshape(-1), self.W3.reshape(-1), W3T.reshape(-1),
                          W2T.reshape(-1)])
        self.net.copy_(flat.to(torch.bfloat16))

    def state_dict(self):
        return {"params": self.params.detach().cpu().clone(), "w3_scale": self.w3_scale}

    def load_state_dict(self, sd):
        self.params.copy_(sd["params"].to(self.device))
        self.w3_scale = float(sd.get("w3_scale", self.w3_scale))
        self.pack()

    def check(self):
        if int(self.status.item()):
            raise L.VlasovError("a tensor-core completion wait timed out in the corrector kernel")

    # ---- kernels ---------------------------------------------------------------
    def drift(self, f, table, alpha, axis: int, vel_axis: int, out=None):
        """Corrected periodic drift of f (float32) along axis."""
        L.require_cuda(f)
        if f.dtype != torch.float32:
            raise ValueError("the learned drift runs on float32 storage")
        out = torch.empty_like(f) if out is None else out
        n_outer, n_line, n_inner = ops._olc(f.shape, axis)
        sel_div = int(np.prod(f.shape[vel_axis + 1:], dtype=np.int64))
        sel_mod = int(f.shape[vel_axis])
        L.call("vp_mlp_drift", L.ptr(f), L.ptr(out), n_outer, n_line, n_inner, sel_div, sel_mod,
               L.ptr(table.shift), L.ptr(table.W), L.ptr(alpha), L.ptr(self.net), L.ptr(self.status),
               L.stream_of(f))
        return out

    def accumulate(self, f, target, table, alpha, axis: int, vel_axis: int, inv_scale: float):
        """Add the gradient of sum((drift(f) - target)^2 * inv_scale^2) to self.grad."""
        L.require_cuda(f, target)
        n_outer, n_line, n_inner = ops._olc(f.shape, axis)
        sel_div = int(np.prod(f.shape[vel_axis + 1:], dtype=np.int64))
        sel_mod = int(f.shape[vel_axis])
        L.call("vp_mlp_train", L.ptr(f), L.ptr(target), n_outer, n_line, n_inner, sel_div, sel_mod,
               L.ptr(table.shift), L.ptr(table.W), L.ptr(alpha), L.ptr(self.net), float(inv_scale),
               L.ptr(self.grad), L.ptr(self.loss), L.ptr(self.status), L.stream_of(f))

    def kick(self, f, E, axis: int, dt: float, dv: float, out=None):
        """Corrected exact kick of f (float32) along velocity axis `axis` with
        the field E over the dims before it (E.numel() divides their product)."""
        L.require_cuda(f, E)
        if f.dtype != torch.float32:
            raise ValueError("the learned kick runs on float32 storage")
        out = torch.empty_like(f) if out is None else out
        n_outer, n_line, n_inner = ops._olc(f.shape, axis)
        E = E.to(torch.float64).contiguous()
        L.call("vp_mlp_kick", L.ptr(f), L.ptr(out), n_outer, n_line, n_inner, L.ptr(E), n_outer // E.numel(),
               float(dt), float(dv), L.ptr(self.net), L.ptr(self.status), L.stream_of(f))
        return out

    def accumulate_kick(self, f, target, E, axis: int, dt: float, dv: float, inv_scale: float):
        """Add the gradient of sum((kick(f) - target)^2 * inv_scale^2) to self.grad."""
        L.require_cuda(f, target, E)
        n_outer, n_line, n_inner = ops._olc(f.shape, axis)
        E = E.to(torch.float64).contiguous()
        L.call("vp_mlp_train_kick", L.ptr(f), L.ptr(target), n_outer, n_line, n_inner, L.ptr(E),
               n_outer // E.numel(), float(dt), float(dv), L.ptr(self.net), float(inv_scale), L.ptr(self.grad),
               L.ptr(self.loss), L.ptr(self.status), L.stream_of(f))

    def zero_grad(self):
        self.grad.zero_()
        self.loss.zero_()

    def adam(self, n_cells: int, lr: float = 1e-3, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
        """One Adam step on the mean loss over n_cells, then repack."""
        self.t += 1
        g = self.grad / float(n_cells)
        g[HID * K1 + HID * K2:] *= self.w3_scale  # gradient of the stored (unscaled) W3
        self.m.mul_(b1).add_(g, alpha=1 - b1)
        self.v.mul_(b2).addcmul_(g, g, value=1 - b2)
        mh = self.m / (1 - b1 ** self.t)
        vh = self.v / (1 - b2 ** self.t)
        self.params.addcdiv_(mh, vh.sqrt().add_(eps), value=-lr)
        self.pack()


class PairSource:
    """Coarse / 2x-refined pairs of one configuration. The fine run uses
    (2 Nx, 2 Ny, 2 Nvx - 1, 2 Nvy - 1) so that the coarse grid is every second
    fine point; restriction is f_fine[::2, ::2, ::2, ::2]."""

    def __init__(self, Nx, Ny, Nvx, Nvy, Lx, Ly, Vx_max, Vy_max, dt, device="cuda"):
        from .engine import Stepper2D

        self.coarse_shape = (Nx, Ny, Nvx, Nvy)
        self.fine = Stepper2D(2 * Nx, 2 * Ny, 2 * Nvx - 1, 2 * Nvy - 1, Lx, Ly, Vx_max, Vy_max, dt,
                              dtype=torch.float32, device=device, window=-1, diagnostics=0, precise_tables=True)
        self.coarse = Stepper2D(Nx, Ny, Nvx, Nvy, Lx, Ly, Vx_max, Vy_max, dt, dtype=torch.float32, device=device,
                                window=-1, diagnostics=0, precise_tables=True)
        c = self.coarse
        vx = torch.linspace(-Vx_max, Vx_max, Nvx, dtype=torch.float64)
        vy = torch.linspace(-Vy_max, Vy_max, Nvy, dtype=torch.float64)
        self.alpha_x = torch.from_numpy(alpha_table(vx, dt / 2.0, c.dx)).to(c.device)
        self.alpha_y = torch.from_numpy(alpha_table(vy, dt / 2.0, c.dy)).to(c.device)

    @staticmethod
    def restrict(f):
        return f[::2, ::2, ::2, ::2].contiguous()

    def pairs(self, f_fine):
        """The x and y drift pairs at this fine state: ((f_c, g_c) for x,
        (g_c, h_c) for y), with g = fine x drift of f, h = fine y drift of g."""
        F = self.fine
        g = ops.drift(f_fine, F.tx, axis=0, vel_axis=2)
        h = ops.drift(g, F.ty, axis=1, vel_axis=3)
        r = self.restrict
        return (r(f_fine), r(g)), (r(g), r(h))

    def kick_pairs(self, f_fine):
        """The vx and vy kick pairs of the fine step from this state, in the
        step's order: h = y drift(x drift(f)), field E from h, k1 = vx kick(h),
        k2 = vy kick(k1). Returns ((h_c, k1_c, Ex_c), (k1_c, k2_c, Ey_c)) with
        the fine field at the coarse points."""
        F = self.fine
        h = ops.drift(ops.drift(f_fine, F.tx, axis=0, vel_axis=2), F.ty, axis=1, vel_axis=3)
        rho = ops.velocity_moment(h, F.dvx, F.dvy, 2)
        ex, ey, _, _ = ops.poisson2d(rho, F.kx, F.ky, F.inv_ksq)
        k1 = ops.kick(h, ex, F.dt, F.dvx, axis=2)
        k2 = ops.kick(k1, ey, F.dt, F.dvy, axis=3)
        r = self.restrict
        exc = ex[::2, ::2].contiguous()
        eyc = ey[::2, ::2].contiguous()
        return (r(h), r(k1), exc), (r(k1), r(k2), eyc)


class LearnedStepper2D:
    """Coarse FP32 2D2V Strang step with learned corrections:
    x(dt/2), y(dt/2), rho, Poisson, vx(dt), vy(dt), y(dt/2), x(dt/2).
    kick_net corrects the two kicks, drift_net (optional) the four drifts;
    a sweep without a network is the plain one."""

    def __init__(self, kick_net: Corrector | None, Nx, Ny, Nvx, Nvy, Lx, Ly, Vx_max, Vy_max, dt, device="cuda",
                 precise_tables=True, drift_net: Corrector | None = None):
        from .engine import Stepper2D

        self.kick_net = kick_net
        self.drift_net = drift_net
        self.base = Stepper2D(Nx, Ny, Nvx, Nvy, Lx, Ly, Vx_max, Vy_max, dt, dtype=torch.float32, device=device,
                              window=-1, diagnostics=1, precise_tables=precise_tables)
        b = self.base
        gdt = torch.float64 if precise_tables else torch.float32
        vx = torch.linspace(-Vx_max, Vx_max, Nvx, dtype=gdt)
        vy = torch.linspace(-Vy_max, Vy_max, Nvy, dtype=gdt)
        self.alpha_x = torch.from_numpy(alpha_table(vx, dt / 2.0, b.dx)).to(b.device)
        self.alpha_y = torch.from_numpy(alpha_table(vy, dt / 2.0, b.dy)).to(b.device)
        self.shape = b.shape
        self.t1 = b.empty_f()
        self.t2 = b.empty_f()
        self.rho = torch.empty((Nx, Ny), dtype=torch.float64, device=b.device)
        self.energy = torch.zeros(2, dtype=torch.float64, device=b.device)
        nb = L.query("vp_poisson2d_workspace_bytes", Nx, Ny)
        self.ws = torch.empty(nb, dtype=torch.uint8, device=b.device)
        self._graphs = {}
        # the fused drift pairs take the layout (vp_drift_pair's conditions)
        self._pairs = b.passes(b.empty_f(), b.empty_f())[1]

    def _drift(self, f, axis, out):
        b = self.base
        table = b.tx if axis == 0 else b.ty
        if self.drift_net is not None:
            return self.drift_net.drift(f, table, self.alpha_x if axis == 0 else self.alpha_y, axis, axis + 2,
                                        out=out)
        return ops.drift(f, table, axis, axis + 2, out=out)

    def _kick(self, f, E, axis, out):
        b = self.base
        dv = b.dvx if axis == 2 else b.dvy
        if self.kick_net is not None:
            return self.kick_net.kick(f, E, axis, b.dt, dv, out=out)
        return ops.kick(f, E, b.dt, dv, axis, window=-1, out=out)

    def step(self, f_in, f_out, energy=None):
        """One step f_in -> f_out (distinct buffers); energy: optional float64
        [2] = {field energy, mass} of the mid-step field. Without a drift
        network the position drifts go in pairs through the fused passes
        (the first one forms the density) where the layout allows."""
        b = self.base
        st = L.stream_of(f_in)
        Nx, Ny, Nvx, Nvy = self.shape
        fused = self.drift_net is None and self._pairs
        if fused:
            ops.drift_pair(f_in, b.tx, b.ty, True, out=self.t2, scale=b.dvx * b.dvy, rho=self.rho)
        else:
            self._drift(f_in, 0, self.t1)
            self._drift(self.t1, 1, self.t2)
            L.call("vp_rho", L.ptr(self.t2), L.VP_F32, Nx * Ny, Nvx * Nvy, float(b.dvx), float(b.dvy),
                   L.ptr(self.rho), L.VP_F64, st)
        e = self.energy if energy is None else energy
        L.call("vp_poisson2d", L.ptr(self.rho), Nx, Ny, L.ptr(b.kx), L.ptr(b.ky), L.ptr(b.inv_ksq), float(b.dx),
               float(b.dy), L.ptr(b.ex), L.ptr(b.ey), L.ptr(b.drho), L.ptr(b.phi), L.ptr(e), L.ptr(self.ws),
               self.ws.numel(), st)
        self._kick(self.t2, b.ex, 2, self.t1)
        self._kick(self.t1, b.ey, 3, self.t2)
        if fused:
            ops.drift_pair(self.t2, b.tx, b.ty, False, out=f_out)
        else:
            self._drift(self.t2, 1, self.t1)
            self._drift(self.t1, 0, f_out)
        return f_out

    def run(self, f, nsteps: int, history=None, graph: bool = True, chunk: int = 10):
        """Advance f (float32) by nsteps, the result back in f; history:
        optional float64 [nsteps, 2] of {field energy, mass}. With graph=True,
        chunks of `chunk` (even) steps are captured once per state buffer and
        replayed."""
        done = 0
        key = (f.data_ptr(), chunk)
        entry = self._graphs.get(key)
        bb = entry[2] if entry is not None else torch.empty_like(f)
        a = f
        if graph and chunk % 2 == 0 and (entry is not None or nsteps >= chunk + 2):
            if entry is None:
                stage = torch.zeros((chunk, 2), dtype=torch.float64, device=f.device)
                s = torch.cuda.Stream(f.device)
                s.wait_stream(torch.cuda.current_stream(f.device))
                with torch.cuda.stream(s):  # first launches outside the capture
                    self.step(a, bb, stage[0])
                    self.step(bb, a, stage[1])
                torch.cuda.current_stream(f.device).wait_stream(s)
                if history is not None:
                    history[0:2].copy_(stage[:2])
                done = 2
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g):
                    x, y = a, bb
                    for i in range(chunk):
                        self.step(x, y, stage[i])
                        x, y = y, x
                entry = (g, stage, bb)
                self._graphs[key] = entry
            g, stage, _ = entry
            while nsteps - done >= chunk:
                g.replay()
                if history is not None:
                    history[done: done + chunk].copy_(stage)
                done += chunk
        while done < nsteps:
            e = history[done] if history is not None else None
            self.step(a, bb, e)
            a, bb = bb, a
            done += 1
        if a.data_ptr() != f.data_ptr():
            f.copy_(a)
        return f


# ---------------------------------------------------------------------------
# seeded training and evaluation (the learned-corrector configuration)
# ---------------------------------------------------------------------------
def draw_ic(rng: np.random.Generator, L: float) -> dict:
    """One initial condition on a box of side L: Landau (Maxwellian shifted by
    v0 ~ U[0, 1.5]) or two-stream (beams at +-v0, v0 ~ U[1.5, 3]), amplitude
    eps ~ U[0.001, 0.1], wave number k = m 2 pi / L with m in {1, 2}."""
    kind = "landau" if rng.integers(0, 2) == 0 else "two_stream"
    eps = float(rng.uniform(0.001, 0.1))
    k = float(rng.integers(1, 3)) * 2.0 * math.pi / L
    v0 = float(rng.uniform(0.0, 1.5) if kind == "landau" else rng.uniform(1.5, 3.0))
    return dict(kind=kind, eps=eps, k=k, v0=v0)


def initial(ic: dict, shape, L: float, V: float, device="cuda"):
    from . import workloads

    Nx, Ny, Nvx, Nvy = shape
    return workloads.initial_2d(ic["kind"], Nx, Ny, Nvx, Nvy, L, L, V, V, ic["eps"], ic["k"], ic["v0"],
                                dtype=torch.float32, device=device)


def collect_kick_pairs(src: PairSource, ics, snapshot_steps, L: float, V: float):
    """Kick pairs (input, target, field, axis, 1/max|input|) of the fine runs
    of `ics`, restricted to the coarse grid, at the given step numbers."""
    pairs = []
    last = max(snapshot_steps)
    for ic in ics:
        f = initial(ic, src.fine.shape, L, V, src.fine.device)
        for it in range(last + 1):
            if it in snapshot_steps:
                (a, b, ex), (c, d, ey) = src.kick_pairs(f)
                pairs.append((a, b, ex, 2, 1.0 / max(a.abs().max().item(), 1e-30)))
                pairs.append((c, d, ey, 3, 1.0 / max(c.abs().max().item(), 1e-30)))
            if it < last:
                f = src.fine.step(f)
    return pairs


def train_kicks(net: Corrector, pairs, coarse, iters: int, batch: int, lr: float = 1e-3, seed: int = 0,
                log=None, auto_scale: float = 250.0):
    """Adam on random minibatches of kick pairs; returns the mean loss per
    cell of every iteration (computed by the training pass itself).

    auto_scale: when the network starts from the plain method (W3 = 0), its
    output scale is set to auto_scale * sqrt(plain loss per cell) from the
    first minibatch, so that Adam's steps on W3 match the size of the
    corrections the pairs ask for (0 keeps the scale given to the net)."""
    rng = np.random.default_rng(seed)
    fresh = auto_scale > 0 and net.t == 0 and not bool(net.W3.abs().max().item() > 0)
    losses = []
    for it in range(iters):
        net.zero_grad()
        cells = 0
        for i in rng.choice(len(pairs), size=min(batch, len(pairs)), replace=False):
            fi, tg, E, axis, inv = pairs[i]
            dv = coarse.dvx if axis == 2 else coarse.dvy
            net.accumulate_kick(fi, tg, E, axis, coarse.dt, dv, inv)
            cells += fi.numel()
        losses.append(net.loss.item() / cells)
        if fresh and it == 0:
            net.w3_scale = auto_scale * math.sqrt(max(losses[0], 1e-30))
        net.adam(cells, lr=lr)
        if log and (it % 50 == 0 or it == iters - 1):
            log(f"iter {it}: loss {losses[-1]:.4g}")
    net.check()
    return losses
