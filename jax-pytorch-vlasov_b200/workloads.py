"""Seeded synthetic workloads of the 2D2V step: initial conditions on the
device and the parameter draws of the batched uneven-runs configuration.

Initial conditions follow Vlasov.initialize (vlasov2D2V.py:1319-1355) with
the perturbation (1 + eps (cos kx + cos ky)) and a velocity profile:
  landau      M(vx - v0) M(vy)                       (shifted Maxwellian)
  two_stream  1/2 [M(vx - v0) + M(vx + v0)] M(vy)
with M the unit 1D Maxwellian. Grids are those of Grid.create
(vlasov2D2V.py:146-156): x = linspace(0, L, N + 1)[:-1], v = linspace(-V, V, N).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import ops

# draws of the batched configuration (64 runs of uneven size)
BATCH_SEED = 20261203
BATCH_NX = (16, 24, 32, 48, 64)
BATCH_NV = (32, 48, 64)


def maxwellian(v: torch.Tensor) -> torch.Tensor:
    return torch.exp(-0.5 * v * v) / math.sqrt(2.0 * math.pi)


def velocity_factors(kind: str, vx: torch.Tensor, vy: torch.Tensor, v0: float = 0.0):
    """(A(vx), B(vy)) of the separable velocity profile, float64."""
    vx = vx.to(torch.float64)
    vy = vy.to(torch.float64)
    if kind == "landau":
        return maxwellian(vx - v0), maxwellian(vy)
    if kind == "two_stream":
        return 0.5 * (maxwellian(vx - v0) + maxwellian(vx + v0)), maxwellian(vy)
    raise ValueError(f"unknown initial condition {kind!r}")


def initial_2d(kind: str, Nx: int, Ny: int, Nvx: int, Nvy: int, Lx: float, Ly: float, Vx_max: float,
               Vy_max: float, eps: float, k: float, v0: float = 0.0, dtype=torch.float32,
               device="cuda") -> torch.Tensor:
    """f0 on the device: evaluated in float64, rounded once to dtype."""
    x = torch.linspace(0.0, Lx, Nx + 1, dtype=torch.float64, device=device)[:-1]
    y = torch.linspace(0.0, Ly, Ny + 1, dtype=torch.float64, device=device)[:-1]
    vx = torch.linspace(-Vx_max, Vx_max, Nvx, dtype=torch.float64, device=device)
    vy = torch.linspace(-Vy_max, Vy_max, Nvy, dtype=torch.float64, device=device)
    sp = 1.0 + eps * (torch.cos(k * x)[:, None] + torch.cos(k * y)[None, :])
    A, B = velocity_factors(kind, vx, vy, v0)
    # the product sp (x) (A B) in FP64, rounded once, in one write of f
    return ops.init_product(sp, A[:, None] * B[None, :], dtype)


def batch_runs(n: int = 64, seed: int = BATCH_SEED, dt: float = 0.05) -> list[dict]:
    """Parameters of n independent runs drawn with numpy's default_rng(seed):
    Nx = Ny from BATCH_NX, Nvx = Nvy from BATCH_NV, eps ~ U[0.001, 0.05],
    k ~ U[0.3, 1.0] (L = 2 pi / k), v0 ~ U[0, 3], kind Landau or two-stream,
    v in [-6 - v0, 6 + v0]."""
    rng = np.random.default_rng(seed)
    runs = []
    for _ in range(n):
        nx = int(rng.choice(BATCH_NX))
        nv = int(rng.choice(BATCH_NV))
        eps = float(rng.uniform(0.001, 0.05))
        k = float(rng.uniform(0.3, 1.0))
        v0 = float(rng.uniform(0.0, 3.0))
        kind = "landau" if rng.integers(0, 2) == 0 else "two_stream"
        L = 2.0 * math.pi / k
        V = 6.0 + v0
        runs.append(dict(Nx=nx, Ny=nx, Nvx=nv, Nvy=nv, Lx=L, Ly=L, Vx_max=V, Vy_max=V, dt=dt, eps=eps, k=k,
                         v0=v0, kind=kind))
    return runs


def cells(runs) -> int:
    return int(sum(r["Nx"] * r["Ny"] * r["Nvx"] * r["Nvy"] for r in runs))
