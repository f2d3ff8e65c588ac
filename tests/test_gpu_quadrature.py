"""Quadrature kernel (variable-coefficient advection, rhs_quad.cu) on the
GPU against the template executor, which integrates the template tree with
the reference's quadrature rules on the CPU
(test/test_cuda.py:57-119 is the reference's CPU-vs-GPU quadrature test).

* RHS parity for every flux type, with and without inflow data, 2D and 3D,
  FP64 (rel-L2 <= 1e-12) and FP32 (<= 1e-5 on FP32-rounded inputs);
* the nodal fallback (no degree for the tag) against the executor run on
  the template without up-samplers;
* the fused LSRK stage against RHS + the stage combination on the host;
* 20 LSRK4 steps of the bound model (the reference's var-velocity example:
  rotating velocity, inflow data on the right half) against the executor's
  LSRK4, and a time-dependent velocity;
* a CUDA-graph replay of the stages equals the eager stepper bitwise;
* bad calls raise.
"""
import numpy as np
import pytest

import hedge_b200 as hb
from hedge_b200.timestep import RK4A, RK4B, RK4C

from conftest import rel_l2
from test_optemplate import box, rect
from test_quadrature import state, velocity

pytestmark = pytest.mark.gpu


def _exec(d, tpl, env):
    from optemplate_exec import TemplateExecutor
    return TemplateExecutor(d)(tpl, **env)[0]


def _setup(dim, order=None, degree=True, precision="fp64"):
    N = order or (4 if dim == 2 else 3)
    m = rect(8, False, 0.03, 21) if dim == 2 else box(2, 0.03, 22)
    kw = {"quad_min_degrees": {"quad": 3 * N}} if degree else {}
    return hb.Discretization(m, order=N, precision=precision, **kw)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("with_bc", [False, True])
@pytest.mark.parametrize("flux_type", ["central", "upwind", "lf"])
@pytest.mark.parametrize("dim", [2, 3])
def test_rhs_parity(cuda_device, dim, flux_type, with_bc, precision):
    d = _setup(dim, precision=precision)
    op = hb.VariableCoefficientAdvectionOperator(
        dim, None, bc_u_f=1 if with_bc else "None", flux_type=flux_type)
    tpl = op.op_template()
    u, v = state(d, 3), velocity(d)
    if precision == "fp32":
        u = u.astype(np.float32).astype(np.float64)
    env = {"u": u, "v": v}
    if with_bc:
        env["bc_u"] = np.sin(3 * d.get_boundary(hb.TAG_ALL).nodes[:, 0])
    ref = _exec(d, tpl, env)
    comp = d.compile(tpl)
    got = comp(**env).double().cpu().numpy()
    comp.check()
    assert rel_l2(got, ref) <= (1e-12 if precision == "fp64" else 1e-5)


def test_nodal_fallback(cuda_device):
    from hedge_b200.lowering import _strip_samplers
    d = _setup(2, degree=False)
    op = hb.VariableCoefficientAdvectionOperator(2, None, bc_u_f=1, flux_type="upwind")
    tpl = op.op_template()
    u, v = state(d, 4), velocity(d)
    bc = np.cos(2 * d.get_boundary(hb.TAG_ALL).nodes[:, 1])
    ref = _exec(d, _strip_samplers(tpl), {"u": u, "v": v, "bc_u": bc})
    with pytest.warns(UserWarning, match="nodal evaluation"):
        comp = d.compile(tpl)
    got = comp(u=u, v=v, bc_u=bc).cpu().numpy()
    comp.check()
    assert rel_l2(got, ref) <= 1e-12


@pytest.mark.parametrize("dim", [2, 3])
def test_fused_stage(cuda_device, dim):
    import torch
    d = _setup(dim)
    op = hb.VariableCoefficientAdvectionOperator(dim, None, flux_type="lf")
    comp = d.compile(op.op_template())
    u, v = state(d, 5), velocity(d)
    vt = d.to_device(v, torch.float64).reshape(-1).contiguous()
    q = d.to_device(u).reshape(1, -1)
    res0 = d.to_device(0.1 * np.cos(d.nodes[:, 0])).reshape(1, -1)
    res, out, rhs = res0.clone(), torch.empty_like(q), torch.empty_like(q)
    comp.lsrk_stage(RK4A[2], RK4B[2], 1e-3, q, out, res, coeff=vt)
    comp.rhs_into(q, rhs, coeff=vt)
    comp.check()
    r = RK4A[2] * res0 + 1e-3 * rhs
    assert torch.allclose(res, r, rtol=1e-14, atol=1e-16)
    assert torch.allclose(out, q + RK4B[2] * r, rtol=1e-14, atol=1e-16)


def _executor_lsrk4(d, tpl, u, env_at, t, dt, steps):
    res = np.zeros_like(u)
    for _ in range(steps):
        for a, b, c in zip(RK4A, RK4B, RK4C):
            r = _exec(d, tpl, dict(env_at(t + c * dt), u=u))
            res = a * res + dt * r
            u = u + b * res
        t += dt
    return u


def test_bound_model_steps_reference_example(cuda_device):
    """advection/var-velocity.py: rotating velocity (-y, x), inflow u = 1
    where x > 0, upwind flux, quadrature degree 3N; 20 LSRK4 steps."""
    d = _setup(2)
    vf = hb.TimeConstantGivenFunction(lambda x: np.stack([-x[:, 1], x[:, 0]]))
    bf = hb.TimeConstantGivenFunction(lambda x: (x[:, 0] > 0).astype(np.float64))
    op = hb.VariableCoefficientAdvectionOperator(2, vf, bc_u_f=bf, flux_type="upwind")
    rhs = op.bind(d)
    x = d.nodes
    u0 = np.exp(-64 * np.sum((x - np.array([0.3, 0.5])) ** 2, axis=1))
    dt = 0.5 * op.estimate_timestep(d, t=0.0)
    st = hb.LSRK4TimeStepper()
    y = d.to_device(u0).reshape(1, -1)
    for k in range(20):
        y = st(y, k * dt, dt, rhs)
    rhs.compiled.check()
    v = vf.f(x)
    bc = bf.boundary_interpolant(0.0, d, hb.TAG_ALL)
    ref = _executor_lsrk4(d, op.op_template(), u0, lambda t: {"v": v, "bc_u": bc},
                          0.0, dt, 20)
    assert rel_l2(y[0].cpu().numpy(), ref) <= 1e-11


def test_time_dependent_velocity(cuda_device):
    """A velocity given as f(x, t): the bound RHS evaluates it at t."""
    d = _setup(2)
    vf = hb.TimeDependentGivenFunction(
        lambda x, t: np.stack([-x[:, 1], x[:, 0]]) * np.cos(np.pi * t))
    op = hb.VariableCoefficientAdvectionOperator(2, vf, flux_type="central")
    rhs = op.bind(d)
    u = state(d, 6)
    for t in (0.0, 0.3):
        got = rhs(t, u).cpu().numpy()
        ref = _exec(d, op.op_template(), {"u": u, "v": vf.f(d.nodes, t)})
        assert rel_l2(got, ref) <= 1e-12
    rhs.compiled.check()


def test_graph_replay_equals_eager(cuda_device):
    import torch
    d = _setup(2)
    vf = hb.TimeConstantGivenFunction(lambda x: np.stack([0.5 - x[:, 1], x[:, 0]]))
    op = hb.VariableCoefficientAdvectionOperator(2, vf, flux_type="lf")
    rhs = op.bind(d)
    rhs.compiled.set_coefficient(vf.f(d.nodes))
    u0 = d.to_device(state(d, 7)).reshape(1, -1)
    dt = 0.5 * op.estimate_timestep(d, t=0.0)
    g = hb.GraphedLSRK4(rhs, u0, dt)
    st = hb.LSRK4TimeStepper()
    y = u0
    for k in range(5):
        g.step()
        y = st(y, k * dt, dt, rhs)
    g.check()
    assert torch.equal(g.state, y)


def test_bad_calls(cuda_device):
    d = _setup(2)
    op = hb.VariableCoefficientAdvectionOperator(2, None, flux_type="central")
    comp = d.compile(op.op_template())
    with pytest.raises(ValueError, match="velocity"):
        comp(u=state(d))
    with pytest.raises(ValueError):
        comp(u=state(d), v=velocity(d)[:1])
    with pytest.raises(NotImplementedError):
        hb.Discretization(d.mesh, order=d.order, precision="fp16x3",
                          quad_min_degrees={"quad": 12}).compile(op.op_template())
