"""The steps' device status word: a bounded device wait that runs out, and a
non-finite field energy or mass, are reported to the host (no GPU fault is
involved: the test hook makes one TMA completion wait per CTA run out after
its 1 s bound, and a NaN in f makes the diagnostics non-finite)."""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def seeded(shape, seed):
    g = np.random.default_rng(seed)
    return torch.from_numpy(1.0 + 0.25 * g.standard_normal(shape)).float().cuda()


# 128 rows: the register-window x-first kernel; 64 rows: the plane-exchange kernels
@pytest.mark.parametrize("shape", [(8, 128, 2, 32), (8, 64, 2, 32)])
def test_wait_timeout_is_reported_and_the_context_survives(vp, shape):
    st = vp.Stepper2D(*shape, 4 * math.pi, 4 * math.pi, 6.0, 6.0, 0.1, dtype=torch.float32)
    assert st.passes(st.empty_f(), st.empty_f()) == (3, True)
    f = seeded(shape, 5)
    st.test_stall = 1
    out = st.step(f)
    torch.cuda.synchronize()
    assert int(st.status.item()) & vp._lib.STATUS_WAIT_TIMEOUT
    assert torch.isnan(out).any()
    with pytest.raises(vp._lib.VlasovError, match="device wait ran out"):
        st.check()
    assert int(st.status.item()) == 0
    # the context is usable: the next step equals a fresh stepper's
    st.test_stall = 0
    got = st.step(f)
    fresh = vp.Stepper2D(*shape, 4 * math.pi, 4 * math.pi, 6.0, 6.0, 0.1, dtype=torch.float32)
    want = fresh.step(f)
    st.check()
    assert torch.equal(got, want)


@pytest.mark.parametrize("kind,shape", [("2d", (16, 16, 8, 32)), ("2d", (8, 8, 16, 12)), ("1d", (64, 32)),
                                        ("1d", (24, 20))])
def test_nonfinite_diagnostics_are_reported(vp, kind, shape):
    if kind == "2d":
        st = vp.Stepper2D(*shape, 4 * math.pi, 4 * math.pi, 6.0, 6.0, 0.1, dtype=torch.float32)
    else:
        st = vp.Stepper1D(*shape, 4 * math.pi, 6.0, 0.1, dtype=torch.float32)
    f = seeded(shape, 6)
    st.step(f)
    st.check()  # finite: nothing reported
    f.view(-1)[7] = float("nan")
    st.step(f)
    assert int(st.status.item()) & vp._lib.STATUS_NONFINITE
    with pytest.raises(vp._lib.VlasovError, match="non-finite"):
        st.check()


def test_batch_wait_timeout_is_reported_per_run(vp):
    """The batched fused passes: the test hook on run 0 makes the first wait
    of the CTAs that start on it run out; run 0 reports it and reads NaN, the
    other runs step normally, and after the hook is cleared the batch steps
    as a fresh one."""
    base = dict(Nx=8, Ny=32, Nvx=2, Nvy=32, Lx=4 * math.pi, Ly=4 * math.pi, Vx_max=6.0, Vy_max=6.0, dt=0.1)
    runs = [dict(base), dict(base), dict(base, Ny=16)]
    b = vp.BatchStepper2D(runs, dtype=torch.float32, window=-1, diagnostics=1)
    assert b.fused == [True, True, False]
    f0 = [seeded((p["Nx"], p["Ny"], p["Nvx"], p["Nvy"]), 7 + r) for r, p in enumerate(runs)]
    for r in range(3):
        b.set_state(r, f0[r])
    b.set_test_stall(0)
    b.step(0)
    torch.cuda.synchronize()
    bits = b.status.cpu().tolist()
    assert bits[0] & vp._lib.STATUS_WAIT_TIMEOUT and not bits[1] & vp._lib.STATUS_WAIT_TIMEOUT and bits[2] == 0
    assert torch.isnan(b.f[0]).any() and torch.isfinite(b.f[1]).all() and torch.isfinite(b.f[2]).all()
    with pytest.raises(vp._lib.VlasovError, match=r"device wait ran out on runs \[0\]"):
        b.check()
    assert int(b.status.abs().sum()) == 0
    b.set_test_stall(0, False)
    fresh = vp.BatchStepper2D(runs, dtype=torch.float32, window=-1, diagnostics=1)
    for r in range(3):
        b.set_state(r, f0[r])
        fresh.set_state(r, f0[r])
    b.step(0)
    fresh.step(0)
    b.check()
    for r in range(3):
        assert torch.equal(b.f[r], fresh.f[r]), r
