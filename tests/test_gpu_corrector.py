"""Learned drift correction on tensor cores (vp_mlp_drift / vp_mlp_train)
against the CPU oracle of the same network (oracle/corrector.py): the
forward pass, the loss and the weight gradients; training lowers the loss on
coarse / refined pairs; with a zero output layer the corrected drift is the
plain drift."""
import math

import numpy as np
import pytest
import torch

from oracle import corrector as OC

pytestmark = pytest.mark.gpu

SHAPE = (12, 16, 24, 20)  # (Nx, Ny, Nvx, Nvy): 92,160 cells, a partial last tile


def _setup(vp, seed=0, out_scale=0.05):
    C = vp.corrector
    net = C.Corrector("cuda", seed=seed, out_scale=out_scale)
    Nx, Ny, Nvx, Nvy = SHAPE
    st = vp.Stepper2D(Nx, Ny, Nvx, Nvy, 4 * math.pi, 3 * math.pi, 6.0, 5.0, 0.4, dtype=torch.float32,
                      precise_tables=True)
    f = vp.workloads.initial_2d("two_stream", Nx, Ny, Nvx, Nvy, 4 * math.pi, 3 * math.pi, 6.0, 5.0, 0.2, 0.5, 1.5)
    g = torch.Generator().manual_seed(seed)
    f = f * (1.0 + 0.05 * torch.rand(f.shape, generator=g)).cuda()
    return C, net, st, f.contiguous()


def _alpha(C, st, axis):
    vel_axis = axis + 2
    vmax = 6.0 if axis == 0 else 5.0
    v = torch.linspace(-vmax, vmax, SHAPE[vel_axis], dtype=torch.float64)
    return torch.from_numpy(C.alpha_table(v, 0.2, st.dx if axis == 0 else st.dy)).cuda()


def _oracle_args(net):
    return (net.W1.cpu().numpy(), net.W2.cpu().numpy(), net.W3.cpu().numpy())


@pytest.mark.parametrize("axis", [0, 1])
def test_forward_matches_oracle(vp, axis):
    C, net, st, f = _setup(vp)
    vel_axis = axis + 2
    table = st.tx if axis == 0 else st.ty
    alpha = _alpha(C, st, axis)
    y = net.drift(f, table, alpha, axis, vel_axis)
    torch.cuda.synchronize()
    net.check()
    plain = vp.ops.drift(f, table, axis, vel_axis)
    yo, _ = OC.forward(f.cpu().numpy(), table.shift.cpu().numpy(), table.W.cpu().numpy(), alpha.cpu().numpy(),
                       axis, vel_axis, *_oracle_args(net))
    corr_gpu = (y - plain).cpu().numpy()
    corr_or = yo - plain.cpu().numpy()
    assert np.abs(corr_or).max() > 1e-3 * f.abs().max().item()  # the correction is not negligible
    err = np.linalg.norm(corr_gpu - corr_or) / np.linalg.norm(corr_or)
    assert err < 1e-2, err


def test_zero_output_layer_is_plain_drift(vp):
    C, net, st, f = _setup(vp, out_scale=0.0)
    y = net.drift(f, st.tx, _alpha(C, st, 0), 0, 2)
    plain = vp.ops.drift(f, st.tx, 0, 2)
    torch.cuda.synchronize()
    net.check()
    assert (y - plain).abs().max().item() <= 2e-6 * f.abs().max().item()


@pytest.mark.parametrize("axis", [0, 1])
def test_gradients_match_oracle(vp, axis):
    C, net, st, f = _setup(vp, seed=1)
    vel_axis = axis + 2
    table = st.tx if axis == 0 else st.ty
    alpha = _alpha(C, st, axis)
    target = vp.ops.drift(f, table, axis, vel_axis) * 1.01  # a target the plain drift misses
    inv_scale = 1.0 / f.abs().max().item()
    net.zero_grad()
    net.accumulate(f, target, table, alpha, axis, vel_axis, inv_scale)
    torch.cuda.synchronize()
    net.check()
    loss, dW1, dW2, dW3 = OC.train_grad(f.cpu().numpy(), target.cpu().numpy(), table.shift.cpu().numpy(),
                                        table.W.cpu().numpy(), alpha.cpu().numpy(), axis, vel_axis,
                                        *_oracle_args(net), inv_scale)
    assert abs(net.loss.item() - loss) <= 1e-3 * loss
    g = net.grad.cpu().numpy()
    n1, n2 = C.HID * C.K1, C.HID * C.K2
    for got, ref in ((g[:n1].reshape(C.HID, C.K1), dW1), (g[n1:n1 + n2].reshape(C.HID, C.K2), dW2),
                     (g[n1 + n2:].reshape(C.NO, C.K2), dW3)):
        err = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-30)
        assert err < 2e-2, err


def test_training_lowers_loss(vp):
    """Forty Adam steps on coarse / 2x-refined pairs lower the pair loss."""
    C = vp.corrector
    Nx = Nv = 16
    L_ = 4 * math.pi
    src = C.PairSource(Nx, Nx, Nv, Nv, L_, L_, 6.0, 6.0, 0.2)
    net = C.Corrector("cuda", seed=3)
    f = vp.workloads.initial_2d("landau", 2 * Nx, 2 * Nx, 2 * Nv - 1, 2 * Nv - 1, L_, L_, 6.0, 6.0, 0.1, 0.5)
    for _ in range(5):
        f = src.fine.step(f)
    (fx, gx), (fy, gy) = src.pairs(f)
    inv = 1.0 / fx.abs().max().item()
    cells = fx.numel()
    losses = []
    for _ in range(40):
        net.zero_grad()
        net.accumulate(fx, gx, src.coarse.tx, src.alpha_x, 0, 2, inv)
        net.accumulate(fy, gy, src.coarse.ty, src.alpha_y, 1, 3, inv)
        losses.append(net.loss.item() / (2 * cells))
        net.adam(2 * cells, lr=3e-3)
    net.check()
    assert losses[-1] < 0.7 * losses[0], (losses[0], losses[-1])


def test_learned_step_runs(vp):
    C = vp.corrector
    net = C.Corrector("cuda", seed=0)
    n = 16
    ls = C.LearnedStepper2D(net, n, n, n, n, 4 * math.pi, 4 * math.pi, 6.0, 6.0, 0.1)
    f = vp.workloads.initial_2d("landau", n, n, n, n, 4 * math.pi, 4 * math.pi, 6.0, 6.0, 0.05, 0.5)
    h = torch.zeros((12, 2), dtype=torch.float64, device="cuda")
    ls.run(f, 12, history=h, graph=True, chunk=4)
    torch.cuda.synchronize()
    net.check()
    hh = h.cpu().numpy()
    assert np.isfinite(hh).all() and (hh[:, 0] > 0).all()
    assert abs(hh[-1, 1] / hh[0, 1] - 1) < 1e-3
