"""Learned interpolation correction on tensor cores (vp_mlp_drift /
vp_mlp_kick and their training passes) against the CPU oracle of the same
network (oracle/corrector.py): the forward pass, the loss and the weight
gradients, for drifts and kicks, with and without the line projection (power-
of-two lines: every line keeps the plain sweep's sum); with a zero output
layer the corrected sweep is the plain one; training lowers the loss on
coarse / refined pairs."""
import math

import numpy as np
import pytest
import torch

from oracle import corrector as OC

pytestmark = pytest.mark.gpu

SHAPE = (12, 16, 24, 20)  # (Nx, Ny, Nvx, Nvy): 92,160 cells, a partial last tile, no projection
# power-of-two shapes (projected sweeps); lines (n, n_inner) by axis:
#   (4, 4, 32, 16):  x (4, 2048), y (4, 512): one lane in each of 4 tiles;
#                    vx (32, 16): 8 lanes in each of 4 tiles; vy (16, 1): 8 lines per tile
#   (2, 2, 16, 256): vx (16, 256): 2 column blocks; vy (256, 1): 128 lanes in each of 2 tiles
POW2 = [(4, 4, 32, 16), (2, 2, 16, 256)]


def _setup(vp, seed=0, out_scale=0.05, shape=SHAPE):
    C = vp.corrector
    net = C.Corrector("cuda", seed=seed, out_scale=out_scale)
    Nx, Ny, Nvx, Nvy = shape
    st = vp.Stepper2D(Nx, Ny, Nvx, Nvy, 4 * math.pi, 3 * math.pi, 6.0, 5.0, 0.4, dtype=torch.float32,
                      precise_tables=True)
    f = vp.workloads.initial_2d("two_stream", Nx, Ny, Nvx, Nvy, 4 * math.pi, 3 * math.pi, 6.0, 5.0, 0.2, 0.5, 1.5)
    g = torch.Generator().manual_seed(seed)
    f = f * (1.0 + 0.05 * torch.rand(f.shape, generator=g)).cuda()
    return C, net, st, f.contiguous()


def _alpha(C, st, axis, shape=SHAPE):
    vel_axis = axis + 2
    vmax = 6.0 if axis == 0 else 5.0
    v = torch.linspace(-vmax, vmax, shape[vel_axis], dtype=torch.float64)
    return torch.from_numpy(C.alpha_table(v, 0.2, st.dx if axis == 0 else st.dy)).cuda()


def _line_sums(y, axis):
    return y.double().sum(dim=axis)


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


@pytest.mark.parametrize("axis", [2, 3])
def test_kick_forward_matches_oracle(vp, axis):
    C, net, st, f = _setup(vp, seed=2)
    g = torch.Generator().manual_seed(7)
    E = (torch.randn(SHAPE[:2], generator=g, dtype=torch.float64) * 3.0).cuda()
    dv = st.dvx if axis == 2 else st.dvy
    y = net.kick(f, E, axis, 0.4, dv)
    torch.cuda.synchronize()
    net.check()
    plain = vp.ops.kick(f, E, 0.4, dv, axis, window=-1)
    F, w, al = OC.kick_cells(f.cpu().numpy(), E.cpu().numpy(), 0.4, dv, axis)
    yo, _ = OC.forward_cells(F, w, al, *_oracle_args(net))
    corr_gpu = (y - plain).cpu().numpy().reshape(-1)
    corr_or = yo - plain.cpu().numpy().reshape(-1)
    assert np.abs(corr_or).max() > 1e-3 * f.abs().max().item()
    err = np.linalg.norm(corr_gpu - corr_or) / np.linalg.norm(corr_or)
    assert err < 1e-2, err


@pytest.mark.parametrize("shape", POW2)
@pytest.mark.parametrize("axis", [2, 3])
def test_projected_kick_matches_oracle(vp, shape, axis):
    """Power-of-two lines: the projected correction against the oracle, and
    every line's sum equal to the plain kick's (the zero-output network's)."""
    C, net, st, f = _setup(vp, seed=5, shape=shape)
    lines = OC.lines_of(shape, axis)
    assert lines is not None
    g = torch.Generator().manual_seed(9)
    E = (torch.randn(shape[:2], generator=g, dtype=torch.float64) * 3.0).cuda()
    dv = st.dvx if axis == 2 else st.dvy
    y = net.kick(f, E, axis, 0.4, dv)
    plain32 = C.Corrector("cuda", out_scale=0.0).kick(f, E, axis, 0.4, dv)  # FP32 weights, no correction
    torch.cuda.synchronize()
    net.check()
    F, w, al = OC.kick_cells(f.cpu().numpy(), E.cpu().numpy(), 0.4, dv, axis)
    yo, _ = OC.forward_cells(F, w, al, *_oracle_args(net), lines=lines)
    corr_gpu = (y - plain32).cpu().numpy().reshape(-1)
    corr_or = yo - plain32.cpu().numpy().reshape(-1)
    assert np.abs(corr_or).max() > 1e-3 * f.abs().max().item()
    err = np.linalg.norm(corr_gpu - corr_or) / np.linalg.norm(corr_or)
    assert err < 1e-2, err
    # conservation: each velocity line keeps the plain kick's sum
    scale = _line_sums(f.abs(), axis).max().item()
    assert (_line_sums(y, axis) - _line_sums(plain32, axis)).abs().max().item() <= 2e-6 * scale
    # the unprojected correction would not
    yu, _ = OC.forward_cells(F, w, al, *_oracle_args(net))
    dn = np.abs((yu - yo).reshape(-1)).max()
    assert dn > 1e-4 * f.abs().max().item()


@pytest.mark.parametrize("shape", POW2)
@pytest.mark.parametrize("axis", [2, 3])
def test_projected_kick_gradients_match_oracle(vp, shape, axis):
    C, net, st, f = _setup(vp, seed=6, shape=shape)
    g = torch.Generator().manual_seed(10)
    E = (torch.randn(shape[:2], generator=g, dtype=torch.float64) * 2.0).cuda()
    dv = st.dvx if axis == 2 else st.dvy
    target = vp.ops.kick(f, E, 0.4, dv, axis, window=-1) * 0.99 + 0.01 * f.mean()
    inv_scale = 1.0 / f.abs().max().item()
    net.zero_grad()
    net.accumulate_kick(f, target, E, axis, 0.4, dv, inv_scale)
    torch.cuda.synchronize()
    net.check()
    F, w, al = OC.kick_cells(f.cpu().numpy(), E.cpu().numpy(), 0.4, dv, axis)
    loss, dW1, dW2, dW3 = OC.train_cells(F, w, al, target.cpu().numpy(), *_oracle_args(net), inv_scale,
                                         lines=OC.lines_of(shape, axis))
    assert abs(net.loss.item() - loss) <= 1e-3 * loss
    gr = net.grad.cpu().numpy()
    n1, n2 = C.HID * C.K1, C.HID * C.K2
    for got, ref in ((gr[:n1].reshape(C.HID, C.K1), dW1), (gr[n1:n1 + n2].reshape(C.HID, C.K2), dW2),
                     (gr[n1 + n2:].reshape(C.NO, C.K2), dW3)):
        err = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-30)
        assert err < 2e-2, err


@pytest.mark.parametrize("axis", [0, 1])
def test_projected_drift_matches_oracle(vp, axis):
    """Power-of-two drift lines: forward, loss and gradients against the
    oracle; every line keeps its sum (the periodic drift conserves it)."""
    shape = POW2[0]
    C, net, st, f = _setup(vp, seed=7, shape=shape)
    vel_axis = axis + 2
    table = st.tx if axis == 0 else st.ty
    alpha = _alpha(C, st, axis, shape)
    y = net.drift(f, table, alpha, axis, vel_axis)
    plain = vp.ops.drift(f, table, axis, vel_axis)
    torch.cuda.synchronize()
    net.check()
    args = (table.shift.cpu().numpy(), table.W.cpu().numpy(), alpha.cpu().numpy(), axis, vel_axis)
    yo, _ = OC.forward(f.cpu().numpy(), *args, *_oracle_args(net))
    corr_gpu = (y - plain).cpu().numpy()
    corr_or = yo - plain.cpu().numpy()
    err = np.linalg.norm(corr_gpu - corr_or) / np.linalg.norm(corr_or)
    assert err < 1e-2, err
    scale = _line_sums(f.abs(), axis).max().item()
    assert (_line_sums(y, axis) - _line_sums(f, axis)).abs().max().item() <= 2e-6 * scale
    target = plain * 1.01
    inv_scale = 1.0 / f.abs().max().item()
    net.zero_grad()
    net.accumulate(f, target, table, alpha, axis, vel_axis, inv_scale)
    torch.cuda.synchronize()
    net.check()
    loss, dW1, dW2, dW3 = OC.train_grad(f.cpu().numpy(), target.cpu().numpy(), *args, *_oracle_args(net),
                                        inv_scale)
    assert abs(net.loss.item() - loss) <= 1e-3 * loss
    gr = net.grad.cpu().numpy()
    n1, n2 = C.HID * C.K1, C.HID * C.K2
    for got, ref in ((gr[:n1].reshape(C.HID, C.K1), dW1), (gr[n1:n1 + n2].reshape(C.HID, C.K2), dW2),
                     (gr[n1 + n2:].reshape(C.NO, C.K2), dW3)):
        err = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-30)
        assert err < 2e-2, err


def test_kick_zero_output_layer_is_plain_kick(vp):
    C, net, st, f = _setup(vp, out_scale=0.0)
    E = torch.linspace(-4, 4, SHAPE[0] * SHAPE[1], dtype=torch.float64).reshape(SHAPE[:2]).cuda()
    for axis, dv in ((2, st.dvx), (3, st.dvy)):
        y = net.kick(f, E, axis, 0.4, dv)
        plain = vp.ops.kick(f, E, 0.4, dv, axis, window=-1)
        torch.cuda.synchronize()
        assert (y - plain).abs().max().item() <= 2e-6 * f.abs().max().item()
    net.check()


@pytest.mark.parametrize("axis", [2, 3])
def test_kick_gradients_match_oracle(vp, axis):
    C, net, st, f = _setup(vp, seed=4)
    g = torch.Generator().manual_seed(8)
    E = (torch.randn(SHAPE[:2], generator=g, dtype=torch.float64) * 2.0).cuda()
    dv = st.dvx if axis == 2 else st.dvy
    target = vp.ops.kick(f, E, 0.4, dv, axis, window=-1) * 0.99
    inv_scale = 1.0 / f.abs().max().item()
    net.zero_grad()
    net.accumulate_kick(f, target, E, axis, 0.4, dv, inv_scale)
    torch.cuda.synchronize()
    net.check()
    F, w, al = OC.kick_cells(f.cpu().numpy(), E.cpu().numpy(), 0.4, dv, axis)
    loss, dW1, dW2, dW3 = OC.train_cells(F, w, al, target.cpu().numpy(), *_oracle_args(net), inv_scale)
    assert abs(net.loss.item() - loss) <= 1e-3 * loss
    gr = net.grad.cpu().numpy()
    n1, n2 = C.HID * C.K1, C.HID * C.K2
    for got, ref in ((gr[:n1].reshape(C.HID, C.K1), dW1), (gr[n1:n1 + n2].reshape(C.HID, C.K2), dW2),
                     (gr[n1 + n2:].reshape(C.NO, C.K2), dW3)):
        err = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-30)
        assert err < 2e-2, err


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
    """Sixty Adam steps on the kick pairs of a 2x-refined run restricted to a
    16^4 grid lower the pair loss."""
    C = vp.corrector
    Nx = Nv = 16
    L_ = 4 * math.pi
    src = C.PairSource(Nx, Nx, Nv, Nv, L_, L_, 6.0, 6.0, 0.1)
    net = C.Corrector("cuda", seed=3)
    ic = dict(kind="landau", eps=0.1, k=0.5, v0=0.0)
    pairs = C.collect_kick_pairs(src, [ic], (20, 40, 60), L_, 6.0)
    assert len(pairs) == 6
    losses = C.train_kicks(net, pairs, src.coarse, iters=60, batch=6, lr=1e-3)
    assert losses[-1] < 0.8 * losses[0], (losses[0], losses[-1])


@pytest.mark.parametrize("with_drift_net", [True, False])
def test_learned_step_with_zero_nets_is_plain_step(vp, with_drift_net):
    """With zero output layers the learned stepper is the plain step (up to
    FP32 summation order: separate kicks instead of the fused one). Without a
    drift network its position drifts are the fused pairs."""
    C = vp.corrector
    n = 32  # the fused pairs take 32^4 (nvy a multiple of 32)
    L_ = 4 * math.pi
    ls = C.LearnedStepper2D(C.Corrector("cuda"), n, n, n, n, L_, L_, 6.0, 6.0, 0.1,
                            drift_net=C.Corrector("cuda") if with_drift_net else None)
    assert ls._pairs
    st = vp.Stepper2D(n, n, n, n, L_, L_, 6.0, 6.0, 0.1, dtype=torch.float32, window=-1, precise_tables=True)
    f = vp.workloads.initial_2d("landau", n, n, n, n, L_, L_, 6.0, 6.0, 0.05, 0.5)
    h = torch.zeros((12, 2), dtype=torch.float64, device="cuda")
    ls.run(f.clone(), 12, history=h, graph=True, chunk=4)
    hp = torch.zeros((12, 8), dtype=torch.float64, device="cuda")
    st.run(f.clone(), 12, history=hp, graph=False)
    torch.cuda.synchronize()
    np.testing.assert_allclose(h[:, :2].cpu().numpy(), hp[:, :2].cpu().numpy(), rtol=1e-5)


def test_learned_step_runs(vp):
    """An untrained network: the step runs (graph-captured), stays finite and
    keeps the mass (16^4: the corrected kicks are projected line by line)."""
    C = vp.corrector
    net = C.Corrector("cuda", seed=0, out_scale=1e-4)
    n = 16
    ls = C.LearnedStepper2D(net, n, n, n, n, 4 * math.pi, 4 * math.pi, 6.0, 6.0, 0.1)
    f = vp.workloads.initial_2d("landau", n, n, n, n, 4 * math.pi, 4 * math.pi, 6.0, 6.0, 0.05, 0.5)
    h = torch.zeros((12, 2), dtype=torch.float64, device="cuda")
    ls.run(f, 12, history=h, graph=True, chunk=4)
    torch.cuda.synchronize()
    net.check()
    hh = h.cpu().numpy()
    assert np.isfinite(hh).all() and (hh[:, 0] > 0).all()
    assert abs(hh[-1, 1] / hh[0, 1] - 1) < 1e-5
