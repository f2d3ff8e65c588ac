"""The reference's CPU-runnable configuration, end to end on the GPU:
2D advection on [-1,1]^2 with 41 x 41 grid points (K = 3200 jittered
triangles, seed 0, periodic), N = 4, FP64, Gaussian pulse of width 0.2,
v = (1, 0.5), upwind flux, dt from the CFL estimate, 100 LSRK4 steps.  The
GPU right-hand side and the fused stepper are compared with the CPU oracle
after one RHS (rel-L2 <= 1e-12) and after the 100 steps (<= 1e-11)."""
import numpy as np
import pytest

import hedge_b200 as hb
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def test_advection_2d_reference_configuration(cuda_device):
    from oracle import OracleRHS
    h = 2.0 / 40
    mesh = hb.make_regular_rect_mesh((-1, -1), (1, 1), (41, 41), periodicity=(True, True),
                                     jitter=0.1 * h, seed=0)
    d = hb.Discretization(mesh, order=4)
    assert d.K == 3200
    op = hb.StrongAdvectionOperator(np.array([1.0, 0.5]), flux_type="upwind")
    u0 = np.exp(-(d.nodes ** 2).sum(1) / 0.2 ** 2)
    rhs = op.bind(d)
    orc = OracleRHS(d, op.descriptor())
    got = rhs(0.0, u0).cpu().numpy()
    assert rel_l2(got, orc(u0[None])[0]) <= 1e-12

    dt = op.estimate_timestep(d)
    stepper = hb.LSRK4TimeStepper()
    y = d.to_device(u0).reshape(1, -1)
    yo, res = u0[None].copy(), np.zeros((1, len(d)))
    t = 0.0
    for _ in range(100):
        y = stepper(y, t, dt, rhs)
        yo, res = orc.lsrk4_step(yo, t, dt, res)
        t += dt
    err = rel_l2(y.reshape(1, -1).cpu().numpy(), yo)
    assert err <= 1e-11, err
    # the pulse is transported, not lost: its L2 norm stays within 1 %
    assert abs(d.norm(y) / d.norm(d.to_device(u0)) - 1) < 1e-2
