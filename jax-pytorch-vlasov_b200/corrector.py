"""Learned correction of the drift interpolation weights (BF16 tensor-core
network, vp_mlp_drift / vp_mlp_train), its training on pairs the method
generates itself, and a coarse-grid stepper that uses it.

The network (see include/vlasov_b200.h): per cell, x = [f_k / max|f|,
alpha - 1/2, 1] -> 64 -> 64 -> 6 with ReLU, output dw (zero mean) added to
the 6 Lagrange weights of the periodic x / y drifts. Plain Lagrange
interpolation stays the fallback: with W3 = 0 the correction vanishes.

Training data: a run on the 2x-refined grid (Nx, Ny doubled; Nv -> 2 Nv - 1
so that every coarse velocity is a fine one) is restricted to the coarse grid
(every second point); the pair (restricted state before a drift, restricted
state after the fine drift) teaches the coarse drift what the refined one
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
    """FP32 master weights, their packed BF16 copy, gradient and Adam state."""

    def __init__(self, device="cuda", seed: int = 0, out_scale: float = 1e-3):
        self.device = torch.device(device)
        g = torch.Generator().manual_seed(seed)
        W1 = torch.zeros(HID, K1)
        W1[:, :7] = torch.randn(HID, 7, generator=g) * math.sqrt(2.0 / 7.0)
        W2 = torch.zeros(HID, K2)
        W2[:, :HID] = torch.randn(HID, HID, generator=g) * math.sqrt(2.0 / HID)
        W3 = torch.zeros(NO, K2)
        W3[:6, :HID] = torch.randn(6, HID, generator=g) * out_scale
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
        return self.params[HID * K1 + HID * K2:].view(NO, K2)

    def pack(self):
        """Refresh the BF16 network (W1, W2, W3 and the transposed copies)."""
        W3T = self.W3[:, :HID].t().contiguous()
        W2T = self.W2[:, :HID].t().contiguous()
        flat = torch.cat([self.W1.reshape(-1), self.W2.reshape(-1), self.W3.reshape(-1), W3T.reshape(-1),
                          W2T.reshape(-1)])
        self.net.copy_(flat.to(torch.bfloat16))

    def state_dict(self):
        return {"params": self.params.detach().cpu().clone()}

    def load_state_dict(self, sd):
        self.params.copy_(sd["params"].to(self.device))
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

    def zero_grad(self):
        self.grad.zero_()
        self.loss.zero_()

    def adam(self, n_cells: int, lr: float = 1e-3, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
        """One Adam step on the mean loss over n_cells, then repack."""
        self.t += 1
        g = self.grad / float(n_cells)
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


class LearnedStepper2D:
    """Coarse FP32 2D2V Strang step with corrected x / y drifts:
    x(dt/2), y(dt/2), rho, Poisson, vx + vy kick, y(dt/2), x(dt/2)."""

    def __init__(self, corrector: Corrector, Nx, Ny, Nvx, Nvy, Lx, Ly, Vx_max, Vy_max, dt, device="cuda",
                 precise_tables=True):
        from .engine import Stepper2D

        self.net = corrector
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

    def step(self, f_in, f_out, energy=None):
        """One step f_in -> f_out (distinct buffers); energy: optional float64
        [2] = {field energy, mass} of the mid-step field."""
        b, n = self.base, self.net
        st = L.stream_of(f_in)
        n.drift(f_in, b.tx, self.alpha_x, 0, 2, out=self.t1)
        n.drift(self.t1, b.ty, self.alpha_y, 1, 3, out=self.t2)
        Nx, Ny, Nvx, Nvy = self.shape
        L.call("vp_rho", L.ptr(self.t2), L.VP_F32, Nx * Ny, Nvx * Nvy, float(b.dvx), float(b.dvy), L.ptr(self.rho),
               L.VP_F64, st)
        e = self.energy if energy is None else energy
        L.call("vp_poisson2d", L.ptr(self.rho), Nx, Ny, L.ptr(b.kx), L.ptr(b.ky), L.ptr(b.inv_ksq), float(b.dx),
               float(b.dy), L.ptr(b.ex), L.ptr(b.ey), L.ptr(b.drho), L.ptr(b.phi), L.ptr(e), L.ptr(self.ws),
               self.ws.numel(), st)
        L.call("vp_kick2d", L.ptr(self.t2), L.ptr(self.t1), L.VP_F32, Nx * Ny, Nvx, Nvy, L.ptr(b.ex), L.ptr(b.ey),
               float(b.dt), float(b.dvx), float(b.dvy), -1, None, None, None, st)
        n.drift(self.t1, b.ty, self.alpha_y, 1, 3, out=self.t2)
        n.drift(self.t2, b.tx, self.alpha_x, 0, 2, out=f_out)
        return f_out

    def run(self, f, nsteps: int, history=None, graph: bool = True, chunk: int = 10):
        """Advance f (float32) by nsteps, the result back in f; history:
        optional float64 [nsteps, 2] of {field energy, mass}. With graph=True,
        chunks of `chunk` (even) steps are captured once and replayed."""
        a, bb = f, torch.empty_like(f)
        done = 0
        if graph and nsteps >= chunk + 2 and chunk % 2 == 0:
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
