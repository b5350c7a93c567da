"""CPU restatement of the learned drift correction (test infrastructure: the
checker of the tensor-core kernels vp_mlp_drift / vp_mlp_train, never part
of the product path).

The network and its use follow the kernel's specification (no reference
counterpart: the reference interpolates with plain Lagrange weights,
vlasov2D2V.py:210-285, and this corrects those weights):
  x  = [bf16(f_k * (1/s)) for k < 6, bf16(alpha - 1/2), 1, 0 x 8],  s = max|f_k|
  z1 = W1 x,            h1 = bf16(relu(z1))
  z2 = W2 [h1, 1, 0],   h2 = bf16(relu(z2))
  o  = W3 [h2, 1, 0]
  y  = sum_k (w_k + o_k - mean(o_0..5)) f_k
and, when the line length n and the stride n_inner of the swept lines are
powers of two, the line projection
  y_l -= mean_l (y_l - p_l),  p_l = sum_k w_k f_k  (the plain sweep)
that keeps each line's sum equal to the plain sweep's.
BF16 values are rounded to nearest even exactly as the device does; the
matrix products are summed in float64 here (FP32 on the device), so the two
agree to accumulation round-off, not bit for bit.
"""
from __future__ import annotations

import numpy as np

HID, K1, K2, NO = 64, 16, 80, 16


def bf16(x) -> np.ndarray:
    """Round float32 values to the nearest bfloat16 (ties to even), as float32."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def bf16_bits(x) -> np.ndarray:
    """bfloat16 bit patterns (uint16) of float32 values, ties to even."""
    return (bf16(x).view(np.uint32) >> 16).astype(np.uint16)


def pack_net(W1: np.ndarray, W2: np.ndarray, W3: np.ndarray) -> np.ndarray:
    """The packed bf16 network of vp_mlp_*: W1, W2, W3, W3T, W2T (uint16 bits)."""
    W1 = np.asarray(W1, np.float32).reshape(HID, K1)
    W2 = np.asarray(W2, np.float32).reshape(HID, K2)
    W3 = np.asarray(W3, np.float32).reshape(NO, K2)
    W3T = np.ascontiguousarray(W3[:, :HID].T)  # [64][16]
    W2T = np.ascontiguousarray(W2[:, :HID].T)  # [64][64]
    return np.concatenate([bf16_bits(m).reshape(-1) for m in (W1, W2, W3, W3T, W2T)])


def stencil(f: np.ndarray, shift: np.ndarray, axis: int, vel_axis: int):
    """f_k (k = 0..5) of every cell of a periodic drift along axis, with the
    table column j of each cell given by its index along vel_axis:
    f_k = f[..., (l - s_j - (k - 2)) mod n, ...]. Returns (F [6, ...], j index array)."""
    n = f.shape[axis]
    idx = np.arange(n)
    shp = [1] * f.ndim
    shp[vel_axis] = f.shape[vel_axis]
    s = np.asarray(shift).reshape(shp)
    F = []
    for k in range(6):
        src = (idx.reshape([-1 if d == axis else 1 for d in range(f.ndim)]) - s - (k - 2)) % n
        F.append(np.take_along_axis(f, np.broadcast_to(src, f.shape), axis=axis))
    jj = np.broadcast_to(np.arange(f.shape[vel_axis]).reshape(shp), f.shape)
    return np.stack(F), jj


def kick_cells(f: np.ndarray, E: np.ndarray, dt: float, dv: float, axis: int):
    """Per-cell stencil F [cells][6], plain weights w [cells][6] (float32) and
    fraction alpha [cells] of the exact kick along axis (vp_kick, window < 0):
    row o of the [outer][line][inner] view moves by d = (E_o dt)/dv (float32),
    s = floor(d), f_k = f[o, l - s - (k - 2), c] (zero outside the line)."""
    f = np.asarray(f, np.float32)
    shape = f.shape
    n_outer = int(np.prod(shape[:axis]))
    n, n_inner = shape[axis], int(np.prod(shape[axis + 1:]))
    Eo = np.repeat(np.asarray(E, np.float64).reshape(-1).astype(np.float32), n_outer // np.asarray(E).size)
    d = (Eo * np.float32(dt)) / np.float32(dv)  # float32, as the corrected kick evaluates it
    s = np.floor(d)
    al = (d - s).astype(np.float32)
    from oracle.core import lagrange5_weights

    w6 = np.asarray(lagrange5_weights(al)).astype(np.float32)  # [6][outer]
    g = f.reshape(n_outer, n, n_inner)
    F = np.zeros((6, n_outer, n, n_inner), np.float32)
    for k in range(6):
        src = np.arange(n)[None, :] - s.astype(np.int64)[:, None] + 2 - k  # [outer][line]
        ok = (src >= 0) & (src < n)
        F[k] = np.where(ok[:, :, None], np.take_along_axis(g, np.clip(src, 0, n - 1)[:, :, None], axis=1), 0)
    cells = n_outer * n * n_inner
    w = np.broadcast_to(w6.T[:, None, None, :], (n_outer, n, n_inner, 6)).reshape(cells, 6)
    alc = np.broadcast_to(al.astype(np.float32)[:, None, None], (n_outer, n, n_inner)).reshape(cells)
    return F.reshape(6, cells).T, w, alc


def drift_cells(f: np.ndarray, shift, W, alpha, axis: int, vel_axis: int):
    """Per-cell stencil, table weights and fraction of the periodic drift."""
    f = np.asarray(f, np.float32)
    F, jj = stencil(f, shift, axis, vel_axis)
    j = jj.reshape(-1)
    return F.reshape(6, -1).T, np.asarray(W, np.float32)[:, j].T, np.asarray(alpha, np.float32)[j]


def lines_of(shape, axis: int):
    """(n_outer, n, n_inner) of the lines swept along axis when the corrected
    sweep projects them (n and n_inner powers of two), else None."""
    n_outer = int(np.prod(shape[:axis]))
    n, n_inner = int(shape[axis]), int(np.prod(shape[axis + 1:]))

    def pow2(v):
        return v > 0 and (v & (v - 1)) == 0

    return (n_outer, n, n_inner) if pow2(n) and pow2(n_inner) else None


def line_mean(v, lines) -> np.ndarray:
    """Per cell (memory order), the float32 mean of v over the cell's line."""
    n_outer, n, n_inner = lines
    m = (np.asarray(v, np.float64).reshape(n_outer, n, n_inner).sum(axis=1) / n).astype(np.float32)
    return np.broadcast_to(m[:, None, :], (n_outer, n, n_inner)).reshape(-1)


def plain_cells(F, w) -> np.ndarray:
    """The plain sweep sum_k w_k f_k (fused multiply-adds in k order)."""
    y = np.zeros(F.shape[0], np.float32)
    for k in range(6):
        y = (w[:, k].astype(np.float64) * F[:, k].astype(np.float64) + y.astype(np.float64)).astype(np.float32)
    return y


def forward_cells(F, w, al, W1, W2, W3, lines=None):
    """The corrected sweep of cells with stencils F, weights w, fractions al;
    lines (from lines_of) turns on the line projection."""
    s = np.abs(F).max(axis=1)
    inv = np.where(s > 0, np.float32(1.0) / np.where(s > 0, s, 1).astype(np.float32), np.float32(0.0))
    inv = inv.astype(np.float32)
    N = F.shape[0]
    x = np.zeros((N, K1), np.float32)
    x[:, :6] = bf16(F * inv[:, None])
    x[:, 6] = bf16(al - np.float32(0.5))
    x[:, 7] = 1.0
    W1b, W2b, W3b = bf16(W1).reshape(HID, K1), bf16(W2).reshape(HID, K2), bf16(W3).reshape(NO, K2)
    z1 = x.astype(np.float64) @ W1b.T.astype(np.float64)
    h1 = np.zeros((N, K2), np.float32)
    h1[:, :HID] = bf16(np.maximum(z1, 0).astype(np.float32))
    h1[:, HID] = 1.0
    z2 = h1.astype(np.float64) @ W2b.T.astype(np.float64)
    h2 = np.zeros((N, K2), np.float32)
    h2[:, :HID] = bf16(np.maximum(z2, 0).astype(np.float32))
    h2[:, HID] = 1.0
    o = (h2.astype(np.float64) @ W3b.T.astype(np.float64)).astype(np.float32)
    mean = o[:, :6].sum(axis=1, dtype=np.float32) * np.float32(1.0 / 6.0)
    y = np.zeros(N, np.float32)
    for k in range(6):  # fused multiply-add: exact product, one rounding
        a = (w[:, k] + (o[:, k] - mean)).astype(np.float32)
        y = (a.astype(np.float64) * F[:, k].astype(np.float64) + y.astype(np.float64)).astype(np.float32)
    if lines is not None:
        y = (y - line_mean(y - plain_cells(F, w), lines)).astype(np.float32)
    cache = dict(F=F, x=x, z1=z1, h1=h1, z2=z2, h2=h2, o=o, W1b=W1b, W2b=W2b, W3b=W3b)
    return y, cache


def train_cells(F, w, al, target, W1, W2, W3, inv_scale, lines=None):
    """(sum r^2, dW1, dW2, dW3) of r = (y - target) * inv_scale; with the
    line projection dL/dy loses its line mean (the projection's transpose)."""
    y, c = forward_cells(F, w, al, W1, W2, W3, lines)
    r = ((y - np.asarray(target, np.float32).reshape(-1)) * np.float32(inv_scale)).astype(np.float32)
    loss = float(np.sum(r.astype(np.float64) ** 2))
    gy = (np.float32(2.0) * r * np.float32(inv_scale)).astype(np.float32)
    if lines is not None:
        gy = (gy - line_mean(gy, lines)).astype(np.float32)
    g = gy[:, None] * c["F"]
    gm = g.sum(axis=1, dtype=np.float32) * np.float32(1.0 / 6.0)
    N = g.shape[0]
    do = np.zeros((N, NO), np.float32)
    do[:, :6] = bf16(g - gm[:, None])
    dh2 = do.astype(np.float64) @ c["W3b"][:, :HID].astype(np.float64)
    dz2 = bf16(np.where(c["z2"] > 0, dh2, 0).astype(np.float32))
    dh1 = dz2.astype(np.float64) @ c["W2b"][:, :HID].astype(np.float64)
    dz1 = bf16(np.where(c["z1"] > 0, dh1, 0).astype(np.float32))
    dW1 = dz1.T.astype(np.float64) @ c["x"].astype(np.float64)
    dW2 = dz2.T.astype(np.float64) @ c["h1"].astype(np.float64)
    dW3 = do.T.astype(np.float64) @ c["h2"].astype(np.float64)
    return loss, dW1, dW2, dW3


def forward(f, shift, W, alpha, axis, vel_axis, W1, W2, W3):
    """Corrected drift of f (float32) and the intermediates of every cell."""
    y, cache = forward_cells(*drift_cells(f, shift, W, alpha, axis, vel_axis), W1, W2, W3,
                             lines_of(np.shape(f), axis))
    return y.reshape(np.shape(f)), cache


def train_grad(f, target, shift, W, alpha, axis, vel_axis, W1, W2, W3, inv_scale):
    """(sum r^2, dW1, dW2, dW3) of the corrected drift against target."""
    return train_cells(*drift_cells(f, shift, W, alpha, axis, vel_axis), target, W1, W2, W3, inv_scale,
                       lines_of(np.shape(f), axis))
