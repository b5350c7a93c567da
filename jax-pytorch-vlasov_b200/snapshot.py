"""Snapshot writers for the drivers' diagnostics output.

The reference writes field_{step:06d}.nc with xarray (vlasov2D2V.py:1357-1390,
vlasov1D1V.py:913-941): variables f, f0, rho, phi, coordinates x, y, vx, vy
(or x, v), attributes step, dt, Lx, Ly, Vx_max, Vy_max, physics_mode. netCDF
is not available here, so the same variables, coordinates and attributes
are written to a numpy .npz archive, and write_raw() writes the raw
row-major binaries that the reference's C++ twin produces
(kokkos/src/vlasov_poisson.hpp:928-955: one file per array).
"""
from __future__ import annotations

import pathlib

import numpy as np
import torch


def _np(t):
    if t is None:
        return None
    if torch.is_tensor(t):
        t = t.detach()
        if t.dtype == torch.bfloat16:
            t = t.float()
        return t.cpu().numpy()
    return np.asarray(t)


def write_snapshot_2d(path, state, solver) -> None:
    g = solver.grid
    np.savez(
        path,
        f=_np(state.variables.fn)[None], f0=_np(state.variables.f0)[None],
        rho=_np(state.field.rho)[None], phi=_np(state.field.phi)[None],
        time=np.array([float(state.t)]), x=_np(g.x), y=_np(g.y), vx=_np(g.vx), vy=_np(g.vy),
        step=np.array(int(state.step)), dt=np.array(solver.dt), Lx=np.array(g.Lx), Ly=np.array(g.Ly),
        Vx_max=np.array(g.Vx_max), Vy_max=np.array(g.Vy_max), physics_mode=np.array(int(solver.physics_mode)),
    )


def write_snapshot_1d(path, state, solver) -> None:
    g = solver.grid
    np.savez(
        path,
        f=_np(state.variables.fn)[None], f0=_np(state.variables.f0)[None],
        rho=_np(state.field.rho)[None], phi=_np(state.field.phi)[None],
        time=np.array([float(state.t)]), x=_np(g.x), v=_np(g.v),
        step=np.array(int(state.step)), dt=np.array(solver.dt), physics_mode=np.array(int(solver.physics_mode)),
    )


def write_raw(directory, step: int, **arrays) -> None:
    """{name}_{step:06d}.bin, row-major, native dtype, one per array."""
    d = pathlib.Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    for name, a in arrays.items():
        _np(a).tofile(d / f"{name}_{int(step):06d}.bin")


def read_raw(path, shape, dtype) -> np.ndarray:
    return np.fromfile(path, dtype=dtype).reshape(shape)
