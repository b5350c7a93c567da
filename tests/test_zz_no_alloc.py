"""The allocation-free field solve, vp_poisson2d_static.

Some callers cannot allocate device memory where they call the library: a
foreign runtime that owns all device memory and only hands over its own input
and output buffers, or an embedded solver whose device footprint is fixed at
start-up. For them vp_poisson2d_static
takes no workspace: its scratch is a device array inside the library. This
test calls it through the C ABI, twice in a row on different grids (the
second call reuses the scratch the first one left behind), and checks every
output against vp_poisson2d with a caller-provided workspace. It also checks
that a grid beyond the static limit is rejected.

The file name sorts last so that a run stopping at its first failure has
already run every other test.
"""
import ctypes
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-13  # the Poisson tolerance of the other GPU tests (relative to max |value|)


def _inputs(vp, nx, ny, seed):
    dev = torch.device("cuda", torch.cuda.current_device())
    rho = torch.from_numpy(1.0 + 0.01 * np.random.default_rng(seed).standard_normal((nx, ny))).to(dev)
    Lx, Ly = 4.0 * math.pi, 3.3
    kx, ky, inv = vp.ops.spectral_2d(nx, ny, Lx, Ly, dev)
    return rho.contiguous(), kx, ky, inv, Lx / nx, Ly / ny


def _outputs(rho):
    return [torch.full_like(rho, float("nan")) for _ in range(4)], torch.full((2,), float("nan"), dtype=torch.float64,
                                                                           device=rho.device)


def _call_static(lib, rho, kx, ky, inv, dx, dy, outs, energy):
    nx, ny = rho.shape
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ex, ey, drho, phi = outs
    return lib.vp_poisson2d_static(rho.data_ptr(), nx, ny, kx.data_ptr(), ky.data_ptr(), inv.data_ptr(), dx, dy,
                                   ex.data_ptr(), ey.data_ptr(), drho.data_ptr(), phi.data_ptr(), energy.data_ptr(),
                                   stream)


def _call_workspace(vp, lib, rho, kx, ky, inv, dx, dy, outs, energy):
    nx, ny = rho.shape
    ws = torch.empty(lib.vp_poisson2d_workspace_bytes(nx, ny), dtype=torch.uint8, device=rho.device)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ex, ey, drho, phi = outs
    return lib.vp_poisson2d(rho.data_ptr(), nx, ny, kx.data_ptr(), ky.data_ptr(), inv.data_ptr(), dx, dy,
                            ex.data_ptr(), ey.data_ptr(), drho.data_ptr(), phi.data_ptr(), energy.data_ptr(),
                            ws.data_ptr(), ws.numel(), stream), ws


def test_poisson2d_static_matches_workspace_version(vp):
    lib = vp.load()
    for nx, ny, seed in ((128, 128, 1), (48, 40, 2)):  # two calls in a row, different grids
        rho, kx, ky, inv, dx, dy = _inputs(vp, nx, ny, seed)
        got, got_e = _outputs(rho)
        want, want_e = _outputs(rho)
        assert _call_static(lib, rho, kx, ky, inv, dx, dy, got, got_e) == 0, lib.vp_last_error()
        rc, ws = _call_workspace(vp, lib, rho, kx, ky, inv, dx, dy, want, want_e)
        assert rc == 0, lib.vp_last_error()
        torch.cuda.synchronize()
        for g, w in zip(got + [got_e], want + [want_e]):
            g, w = g.cpu().numpy(), w.cpu().numpy()
            assert np.isfinite(g).all()
            assert np.abs(g - w).max() <= TOL * max(np.abs(w).max(), 1e-300)


def test_poisson2d_static_rejects_oversize_grid(vp):
    lib = vp.load()
    n = 257  # VP_POISSON2D_STATIC_MAX_N + 1
    p = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.vp_poisson2d_static(p, n, 8, p, p, p, 1.0, 1.0, p, p, p, p, None, None)
    assert rc == 5 and b"VP_POISSON2D_STATIC_MAX_N" in lib.vp_last_error()
