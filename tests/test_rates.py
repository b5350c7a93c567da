"""Damping and growth rates from field-energy histories: synthetic signals
with known rates, and the reference's own C1 (Landau) and C2 (two-stream)
runs stored as golden histories."""
import importlib

import numpy as np
import pytest

R = importlib.import_module("jax-pytorch-vlasov_b200.rates")


@pytest.mark.parametrize("gamma,omega,dt", [(0.1533, 1.4156, 0.1), (0.05, 2.0, 0.05), (0.3, 1.0, 0.02)])
def test_damping_rate_of_a_damped_oscillation(gamma, omega, dt):
    t = dt * np.arange(1, 401)
    we = np.exp(-2 * gamma * t) * (np.cos(omega * t + 0.3) ** 2 + 1e-4)
    assert abs(R.damping_rate(t, we) - gamma) <= 2e-3 * gamma


def test_growth_rate_of_an_exponential_phase():
    t = 0.05 * np.arange(1, 401)
    we = 1e-8 * np.exp(2 * 0.2 * t) * (1.0 + 0.01 * np.sin(3 * t))
    assert abs(R.growth_rate(t, we, 2.0, 12.0) - 0.2) <= 1e-3 * 0.2


def test_peak_refinement_finds_the_true_maximum():
    # a single peak of a parabola in 1/2 log W_E between samples
    t = np.arange(10.0)
    h = -((t - 4.3) ** 2)
    tp, hp = R.energy_peaks(t, np.exp(2 * h))
    assert len(tp) == 1 and abs(tp[0] - 4.3) < 1e-12 and abs(hp[0]) < 1e-12


def test_errors():
    t = np.arange(10.0)
    with pytest.raises(ValueError, match="peak"):
        R.damping_rate(t, np.exp(-t))  # monotone: no peak
    with pytest.raises(ValueError, match="positive"):
        R.damping_rate(t, np.zeros(10))
    with pytest.raises(ValueError, match="samples"):
        R.growth_rate(t, np.exp(t), 3.0, 3.5)


def test_reference_c1_landau_rate(golden):
    """The reference's C1 run (Landau, k = 0.5, 32^4, 100 steps of 0.1): its
    field energy damps at the linear Landau rate 0.1533 (to 2 %), the value
    the reference's post-processing plot is drawn against."""
    H = golden("history_c1")
    t = 0.1 * np.arange(1, len(H["W_E"]) + 1)
    assert abs(R.damping_rate(t, H["W_E"]) - R.LANDAU_RATE_K05) <= 0.02 * R.LANDAU_RATE_K05


def test_reference_c2_two_stream_growth(golden):
    """The reference's C2 run (two-stream, 400 steps of 0.05): after an
    oscillating start its field energy grows, and the rate over the second
    half of the run is positive and of the order of 0.2."""
    H = golden("history_c2")
    t = 0.05 * np.arange(1, len(H["W_E"]) + 1)
    g = R.growth_rate(t, H["W_E"], 10.0, 20.0)
    assert 0.1 < g < 0.4, g
