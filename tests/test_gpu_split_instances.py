"""Every compiled split-precision kernel instance (resident operators for
3D orders <= 4 / 2D <= 6, streamed operators for 3D orders 5-7; the resident
3D order-5 kernel serves partitioned operators, tests/test_gpu_partition.py) on a small
mesh against the FP64 oracle, in both split precisions: relative L2 of one
RHS on rough fields (smooth modes + 10 % noise) <= 1e-6 for FP16x3 and
<= 1e-5 for BF16x3."""
import numpy as np
import pytest

import hedge_b200 as hb
from conftest import rel_l2
from test_gpu_parity import _fields, rect, box

pytestmark = pytest.mark.gpu

RESIDENT = [("advection", 2, o) for o in (3, 4, 5, 6)] + [("advection", 3, o) for o in (3, 4)] \
    + [("wave", 2, o) for o in (3, 4, 5, 6)] + [("wave", 3, o) for o in (3, 4)] \
    + [("varwave", 2, o) for o in (3, 4, 5, 6)] + [("varwave", 3, o) for o in (3, 4)] \
    + [("maxwell", 3, o) for o in (3, 4)]
STREAMED = [("wave", 3, 5), ("wave", 3, 6), ("wave", 3, 7), ("maxwell", 3, 5), ("maxwell", 3, 6)]


def _case(model, dim, order):
    d = hb.Discretization(rect(5, False, 0.03, 1) if dim == 2 else box(2, 0.04, 2),
                          order=order)
    bc = c = None
    if model == "advection":
        op = hb.StrongAdvectionOperator(np.array([0.8, -0.5, 0.3][:dim]), flux_type="upwind",
                                        inflow_tag=hb.TAG_ALL)
        bc = np.sin(2 * d.get_boundary(hb.TAG_ALL).nodes[:, 0])
    elif model == "wave":
        op = hb.StrongWaveOperator(1.1, dim, flux_type="upwind")
    elif model == "varwave":
        c = np.repeat(np.random.default_rng(3).uniform(0.8, 1.2, d.K), d.Np)
        op = hb.VariableVelocityStrongWaveOperator(c, dim, flux_type="upwind")
    else:
        op = hb.MaxwellOperator(1.0, 1.0, flux_type=1)
    return d, op, bc, c


@pytest.mark.parametrize("precision", ["fp16x3", "bf16x3"])
@pytest.mark.parametrize("model,dim,order", RESIDENT + STREAMED)
def test_split_instance(cuda_device, model, dim, order, precision):
    from oracle import OracleRHS
    d, op, bc, c = _case(model, dim, order)
    comp = d.compile(op.op_template(), precision=precision)
    if c is not None:
        comp.set_coefficient(c)
    q = _fields(d, op.descriptor().n_fields, 7)
    ref = OracleRHS(d, op.descriptor(), c_field=c)(q, bc_in=bc)
    got = comp(w=q, bc_in=bc)
    comp.check()
    err = rel_l2(got.cpu().numpy().reshape(ref.shape), ref)
    print("%s %s %dD N=%d rel-L2 %.3e" % (precision, model, dim, order, err))
    assert err <= (1e-6 if precision == "fp16x3" else 1e-5)


@pytest.mark.parametrize("precision", ["fp16x3", "bf16x3"])
@pytest.mark.parametrize("model,dim,order", RESIDENT + STREAMED)
def test_split_instance_stage(cuda_device, model, dim, order, precision):
    """One fused LSRK stage of every instance against the oracle's RHS:
    res1 = a res0 + dt RHS(q0) and q1 = q0 + b res1, with a residual of the
    size of dt RHS (the FP64 update reads it from shared memory or HBM,
    depending on the instance)."""
    import torch
    from oracle import OracleRHS
    d, op, bc, c = _case(model, dim, order)
    comp = d.compile(op.op_template(), precision=precision)
    F = op.descriptor().n_fields
    q0 = _fields(d, F, 8)
    rhs = OracleRHS(d, op.descriptor(), c_field=c)(q0, bc_in=bc).reshape(F, -1)
    a, b, dt = -0.4, 0.6, 0.01
    res0 = dt * np.abs(rhs).max() * np.random.default_rng(9).uniform(-1, 1, rhs.shape)
    ref_res = a * res0 + dt * rhs
    ref_q = q0 + b * ref_res
    dev = d.device
    q_in = torch.tensor(q0, device=dev)
    q_out = torch.empty_like(q_in)
    res = torch.tensor(res0, device=dev)
    cf = torch.tensor(c, device=dev) if c is not None else None
    bt = torch.tensor(bc, device=dev) if bc is not None else None
    comp.lsrk_stage(a, b, dt, q_in, q_out, res, bc_in=bt, coeff=cf)
    comp.check()
    r1 = res.cpu().numpy()
    e_res = rel_l2(r1, ref_res)
    # the FP64 update itself: q1 = q0 + b res1 with the kernel's own res1
    e_q = rel_l2(q_out.cpu().numpy(), q0 + b * r1)
    print("%s %s %dD N=%d stage: res rel-L2 %.3e, q rel-L2 %.3e (vs oracle %.3e)"
          % (precision, model, dim, order, e_res, e_q, rel_l2(q_out.cpu().numpy(), ref_q)))
    assert e_res <= (2e-6 if precision == "fp16x3" else 2e-5)
    assert e_q <= 1e-14
