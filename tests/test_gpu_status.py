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
