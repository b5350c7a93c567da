"""Damping and growth rates from a field-energy history.

The reference checks Landau damping by eye: its post-processing script plots
the potential against exp(-0.153 t) (simulations/vlasov2d_2v/postscript/
postscript.py:29-44). These functions turn that into numbers from the
per-step field energy W_E = 1/2 sum |E|^2 dx dy that the steps report
(diagnostic 0), so a run can pass or fail on its rate.

For a damped mode |E| ~ exp(-gamma t) |cos(omega t + phase)|, so
W_E ~ exp(-2 gamma t) cos^2(...): gamma is minus the slope of 1/2 log W_E
through the peaks of W_E. For a growing mode (two-stream) it is the slope of
1/2 log W_E over the exponential phase. Host-side numpy only.
"""
from __future__ import annotations

import numpy as np

# linear Landau damping rate of a Maxwellian plasma at k = 0.5 (in plasma
# units), the value the reference's plot is drawn against
LANDAU_RATE_K05 = 0.1533


def _window(t, y, t_min, t_max):
    t = np.asarray(t, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    if t.shape != y.shape or t.ndim != 1:
        raise ValueError("t and the field energy must be 1D arrays of the same length")
    keep = np.ones(t.shape, dtype=bool)
    if t_min is not None:
        keep &= t >= t_min
    if t_max is not None:
        keep &= t <= t_max
    return t, y, keep


def energy_peaks(t, we, t_min=None, t_max=None):
    """Local maxima of the field energy inside [t_min, t_max] (both optional),
    each refined by the parabola through the three samples around it in
    1/2 log W_E (uniform sampling is assumed around each peak). Returns
    (times, values of 1/2 log W_E at the refined peaks)."""
    t, we, keep = _window(t, we, t_min, t_max)
    if np.any(we <= 0) or not np.all(np.isfinite(we)):
        raise ValueError("the field energy must be finite and positive")
    h = 0.5 * np.log(we)
    tp, hp = [], []
    for i in range(1, len(h) - 1):
        if not keep[i] or not (h[i - 1] < h[i] >= h[i + 1]):
            continue
        a, b, c = h[i - 1], h[i], h[i + 1]
        den = a - 2.0 * b + c
        off = 0.5 * (a - c) / den if den != 0.0 else 0.0  # in samples, |off| <= 1/2
        tp.append(t[i] + off * 0.5 * (t[i + 1] - t[i - 1]))
        hp.append(b - 0.25 * (a - c) * off)
    return np.asarray(tp), np.asarray(hp)


def damping_rate(t, we, t_min=None, t_max=None):
    """gamma > 0 of a damped field, |E| ~ exp(-gamma t): minus the
    least-squares slope of 1/2 log W_E through its refined peaks in
    [t_min, t_max]. Needs at least two peaks."""
    tp, hp = energy_peaks(t, we, t_min, t_max)
    if len(tp) < 2:
        raise ValueError(f"{len(tp)} peak(s) of the field energy in the window; two or more are needed")
    return -float(np.polyfit(tp, hp, 1)[0])


def growth_rate(t, we, t_min=None, t_max=None):
    """gamma of a growing field, |E| ~ exp(gamma t): the least-squares slope
    of 1/2 log W_E over the samples in [t_min, t_max] (choose the window
    inside the exponential phase)."""
    t, we, keep = _window(t, we, t_min, t_max)
    if keep.sum() < 2:
        raise ValueError("fewer than two samples in the window")
    if np.any(we[keep] <= 0) or not np.all(np.isfinite(we[keep])):
        raise ValueError("the field energy must be finite and positive")
    return float(np.polyfit(t[keep], 0.5 * np.log(we[keep]), 1)[0])
