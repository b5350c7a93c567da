"""x-slab decomposition of one run on the GPU: the ranks are emulated one
after another on one device (each rank's kernels finish before the next
rank's start; none waits on another), each stepping its extended slab with
the library's kernels; halo rows are copied from the neighbours' slab rows
and rho is concatenated as the process-group calls would. The slabs equal
the one-GPU step (single-axis sweeps) bit for bit."""
import importlib
import math

import numpy as np
import pytest
import torch

from conftest import PACKAGE

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("world", [1, 2, 3])
def test_emulated_slabs_equal_one_gpu(vp, world, dtype):
    slab = importlib.import_module(PACKAGE + ".slab")
    Nx, Ny, Nvx, Nvy = 48, 16, 16, 32
    Lx = Ly = 4 * math.pi
    args = (Nx, Ny, Nvx, Nvy, Lx, Ly, 6.0, 5.0, 0.2)
    plan = slab.SlabStepper2D.plan_for(Nx, world, Lx, 6.0, Nvx, 0.2, dtype)
    ranks = [slab.SlabStepper2D(plan, r, *args, dtype=dtype) for r in range(world)]
    one = vp.Stepper2D(*args, dtype=dtype, fuse_drifts=False)
    g = np.random.default_rng(2)
    x = torch.linspace(0, Lx, Nx + 1, dtype=torch.float64)[:-1]
    f = ((1.0 + 0.2 * torch.cos(0.5 * x))[:, None, None, None]
         * torch.from_numpy(1.0 + 0.1 * g.random((1, Ny, Nvx, Nvy)))).to(dtype).cuda()
    fe = [slab.scatter(f, plan, r) for r in range(world)]
    ref = f
    for _ in range(3):
        if world == 1:
            slab.exchange_halos(fe[0], plan, 0)
        else:
            for r in range(world):
                for s, first, n, dst in plan.halo_sources(r):
                    fe[r][dst:dst + n].copy_(slab.slab_rows(fe[s], plan, s)[first:first + n])
        halves = [ranks[r].first_half(fe[r]) for r in range(world)]
        Ex, Ey, drho, phi = ranks[0].field(torch.cat([h[1] for h in halves]))
        fe = [ranks[r].second_half(halves[r][0], Ex, Ey) for r in range(world)]
        ref = one.step(ref)
        got = torch.cat([slab.slab_rows(fe[r], plan, r) for r in range(world)])
        assert torch.equal(got, ref)
        assert torch.equal(drho, one.drho) and torch.equal(phi, one.phi)
