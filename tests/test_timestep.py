"""The LSRK4 coefficient table (CPU): on y' = lambda y one step's
amplification agrees with exp(lambda dt) to fourth order, and each stage
time c_s equals the time the stage's state has reached (the sum of the
B-weighted residual increments), as for the reference's table
(hedge/timestep/runge_kutta.py:43-66)."""
import numpy as np
import pytest

from hedge_b200.timestep import RK4A, RK4B, RK4C, GraphedLSRK4


def _step(lam, dt):
    y, res = 1.0 + 0j, 0j
    for a, b in zip(RK4A, RK4B):
        res = a * res + dt * lam * y
        y = y + b * res
    return y


def test_fourth_order_amplification():
    lam = -1.0 + 0.7j
    errs = [abs(_step(lam, dt) - np.exp(lam * dt)) for dt in (0.1, 0.05)]
    # local error O(dt^5): halving dt divides it by ~32
    assert 25 < errs[0] / errs[1] < 40, errs
    assert errs[1] < 1e-8


def test_stage_times():
    """With y' = 1 the state after stage s is t + c_{s+1} dt."""
    dt, y, res = 1.0, 0.0, 0.0
    for s, (a, b) in enumerate(zip(RK4A, RK4B)):
        res = a * res + dt * 1.0
        y = y + b * res
        c_next = RK4C[s + 1] if s + 1 < 5 else 1.0
        assert abs(y - c_next) < 1e-14


def test_graphed_stepper_needs_a_bound_operator():
    with pytest.raises(TypeError):
        GraphedLSRK4(lambda t, w: w, None, 0.1)
