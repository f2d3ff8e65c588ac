"""BF16x3 split-precision tensor-core path (tcgen05) against the FP64 oracle:
relative L2 error of one RHS and of LSRK4 steps."""
import numpy as np
import pytest

import hedge_b200 as hb
from conftest import rel_l2
from test_gpu_parity import _fields, rect, box

pytestmark = pytest.mark.gpu

# Tolerance of one BF16x3 RHS against the FP64 oracle (relative L2).
SPLIT_TOL = 1e-4


def _split_err(discr, op, seed=0, bc_in=None, c_field=None):
    from oracle import OracleRHS
    ot = op.op_template()
    comp = discr.compile(ot, precision="bf16x3")
    if c_field is not None:
        comp.set_coefficient(c_field)
    q = _fields(discr, ot.n_fields, seed)
    ref = OracleRHS(discr, ot, c_field=c_field)(q, bc_in=bc_in)
    got = comp(w=q, bc_in=bc_in)
    comp.check()
    return rel_l2(got.cpu().numpy().reshape(ref.shape), ref)


@pytest.mark.parametrize("n,order", [(2, 4), (3, 4), (2, 3)])
def test_split_maxwell(cuda_device, n, order):
    d = hb.Discretization(box(n, 0.05, 5), order=order)
    err = _split_err(d, hb.MaxwellOperator(1.0, 1.0, flux_type=1))
    print("bf16x3 maxwell n=%d N=%d rel-L2 %.3e" % (n, order, err))
    assert err <= SPLIT_TOL


def test_split_advection_2d(cuda_device):
    d = hb.Discretization(rect(9, True, 0.02, 0), order=4)
    err = _split_err(d, hb.StrongAdvectionOperator(np.array([1.0, 0.5]), flux_type="upwind"))
    print("bf16x3 advection rel-L2 %.3e" % err)
    assert err <= SPLIT_TOL


def test_split_wave_3d(cuda_device):
    d = hb.Discretization(box(2, 0.05, 3), order=4)
    err = _split_err(d, hb.StrongWaveOperator(1.0, 3, flux_type="upwind"))
    print("bf16x3 wave3d rel-L2 %.3e" % err)
    assert err <= SPLIT_TOL


def test_split_varwave_2d(cuda_device):
    d = hb.Discretization(rect(8, False, 0.02, 4), order=5)
    c = np.repeat(np.random.default_rng(4).uniform(0.8, 1.2, d.K), d.Np)
    op = hb.VariableVelocityStrongWaveOperator(c, 2, flux_type="upwind")
    err = _split_err(d, op, c_field=c)
    print("bf16x3 varwave2d rel-L2 %.3e" % err)
    assert err <= SPLIT_TOL


def test_split_lsrk_steps(cuda_device):
    """Fused BF16x3 RHS + FP64 stage update over 5 steps vs the FP64 oracle."""
    import torch
    from oracle import OracleRHS
    d = hb.Discretization(box(2, 0.05, 1), order=4, precision="bf16x3")
    op = hb.MaxwellOperator(1.0, 1.0, flux_type=1)
    rhs = op.bind(d)
    x = d.nodes
    q = np.stack([np.sin(np.pi * x[:, (f + 1) % 3] / 2) * np.cos(0.5 * x[:, f % 3])
                  for f in range(6)])
    dt = op.estimate_timestep(d)
    y = d.to_device(q).reshape(6, -1)
    orc = OracleRHS(d, op.op_template())
    yo, res = q.copy(), np.zeros_like(q)
    st = hb.LSRK4TimeStepper()
    for s in range(5):
        y = st(y, s * dt, dt, rhs)
        yo, res = orc.lsrk4_step(yo, s * dt, dt, res)
    rhs.compiled.check()
    err = rel_l2(y.cpu().numpy().reshape(yo.shape), yo)
    print("bf16x3 5 LSRK4 steps rel-L2 %.3e" % err)
    assert err <= SPLIT_TOL
