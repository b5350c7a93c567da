"""x-slab decomposition of one run on the GPU: the ranks are emulated one
after another on one device (each rank's kernels finish before the next
rank's start; none waits on another), each stepping its extended slab with
the library's kernels; halo rows are copied from the neighbours' slab rows
and rho is concatenated as the process-group calls would. The slabs equal
the one-GPU step bit for bit: with one sweep per axis, and (FP32) with the
fused drift pairs, whole or split into the interior rows and the rows next to
the halo as the overlapped step runs them."""
import importlib
import math

import numpy as np
import pytest
import torch

from conftest import PACKAGE

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,fused,overlapped", [(torch.float32, False, False), (torch.float64, False, False),
                                                    (torch.float32, True, False), (torch.float32, True, True)])
@pytest.mark.parametrize("world", [1, 2, 3])
def test_emulated_slabs_equal_one_gpu(vp, world, dtype, fused, overlapped):
    slab = importlib.import_module(PACKAGE + ".slab")
    Nx, Ny, Nvx, Nvy = 48, 16, 16, 32
    Lx = Ly = 4 * math.pi
    args = (Nx, Ny, Nvx, Nvy, Lx, Ly, 6.0, 5.0, 0.2)
    plan = slab.SlabStepper2D.plan_for(Nx, world, Lx, 6.0, Nvx, 0.2, dtype)
    ranks = [slab.SlabStepper2D(plan, r, *args, dtype=dtype, fuse_drifts=fused) for r in range(world)]
    assert all(st.fused == fused for st in ranks)
    one = vp.Stepper2D(*args, dtype=dtype, fuse_drifts=fused)
    assert one.passes(one.empty_f(), one.empty_f())[1] == fused
    g = np.random.default_rng(2)
    x = torch.linspace(0, Lx, Nx + 1, dtype=torch.float64)[:-1]
    f = ((1.0 + 0.2 * torch.cos(0.5 * x))[:, None, None, None]
         * torch.from_numpy(1.0 + 0.1 * g.random((1, Ny, Nvx, Nvy)))).to(dtype).cuda()
    fe = [slab.scatter(f, plan, r) for r in range(world)]
    ref = f
    for _ in range(3):
        if world == 1:
            reqs = slab.start_halo_exchange(fe[0], plan, 0)
            assert reqs == []
        else:
            for r in range(world):
                for s, first, n, dst in plan.halo_sources(r):
                    fe[r][dst:dst + n].copy_(slab.slab_rows(fe[s], plan, s)[first:first + n])
        if overlapped:
            halves = [ranks[r].first_half_overlapped(fe[r], []) for r in range(world)]
        else:
            halves = [ranks[r].first_half(fe[r]) for r in range(world)]
        Ex, Ey, drho, phi = ranks[0].field(torch.cat([h[1] for h in halves]))
        fe = [ranks[r].second_half(halves[r][0], Ex, Ey) for r in range(world)]
        ref = one.step(ref)
        got = torch.cat([slab.slab_rows(fe[r], plan, r) for r in range(world)])
        assert torch.equal(got, ref)
        assert torch.equal(drho, one.drho) and torch.equal(phi, one.phi)


def test_drift_pair_rows_and_fallback(vp):
    """vp_drift_pair: split into row ranges it gives the whole pass's f and
    density; a layout it cannot fuse is refused (the caller runs sweeps)."""
    Nx, Ny, Nvx, Nvy = 20, 24, 4, 64
    st = vp.Stepper2D(Nx, Ny, Nvx, Nvy, 4 * math.pi, 3.0, 6.0, 5.0, 0.6, dtype=torch.float32)
    f = torch.from_numpy(1.0 + 0.25 * np.random.default_rng(4).standard_normal((Nx, Ny, Nvx, Nvy))).float().cuda()
    for xfirst in (True, False):
        scale = 0.5 if xfirst else None
        whole, rho = vp.ops.drift_pair(f, st.tx, st.ty, xfirst, scale=scale)
        parts = torch.full_like(f, float("nan"))
        rho2 = torch.full((Nx, Ny), float("nan"), dtype=torch.float64, device="cuda") if xfirst else None
        for r0, n in ((7, 9), (0, 7), (16, 4)):
            vp.ops.drift_pair(f, st.tx, st.ty, xfirst, out=parts, rows=(r0, n), scale=scale, rho=rho2)
        assert torch.equal(parts, whole)
        if xfirst:
            assert torch.equal(rho2, rho)
    # the pair equals the two sweeps bit for bit
    a = vp.ops.drift(f, st.tx, 0, 2)
    assert torch.equal(vp.ops.drift_pair(f, st.tx, st.ty, True)[0], vp.ops.drift(a, st.ty, 1, 3))
    wide = torch.zeros((4, 8, 2, 32), dtype=torch.float32, device="cuda")  # ny < 16
    t8 = vp.Stepper2D(4, 8, 2, 32, 4 * math.pi, 3.0, 6.0, 5.0, 0.6, dtype=torch.float32)
    with pytest.raises(vp._lib.VlasovError, match="needs FP32"):
        vp.ops.drift_pair(wide, t8.tx, t8.ty, True)
