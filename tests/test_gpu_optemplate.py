"""Compiled operator templates on the GPU: hand-written templates lowered
onto the kernels and called with their own field names agree with the CPU
template executor (FP64, rel-L2 <= 1e-12); a model's template and its
descriptor compile to the same kernels (bit-identical RHS)."""
import numpy as np
import pytest

import hedge_b200 as hb
from conftest import rel_l2
from test_optemplate import (_fields, _tagger_lr, advection_by_hand, box,
                             maxwell_by_hand, rect, varwave_by_hand, wave_by_hand)

pytestmark = pytest.mark.gpu


def _exec(d, tpl, env):
    from optemplate_exec import TemplateExecutor
    return TemplateExecutor(d)(tpl, **env)


def test_compiled_advection_template(cuda_device):
    d = hb.Discretization(rect(6, tagger=lambda *a: ["in"]), order=4)
    tpl = advection_by_hand(np.array([0.7, -0.4]), "in")
    q = _fields(d, 1, 5)
    g = np.cos(2 * d.get_boundary("in").nodes[:, 1])
    comp = d.compile(tpl, precision="fp64")
    got = comp(phi=q[0], g=g).cpu().numpy()
    comp.check()
    assert rel_l2(got, _exec(d, tpl, {"phi": q[0], "g": g})[0]) <= 1e-12


def test_compiled_wave_template_named_fields(cuda_device):
    d = hb.Discretization(rect(6, tagger=_tagger_lr(["neu", "dir", "dir"])), order=4)
    tpl = wave_by_hand(1.2, ("dir", "neu"))
    q = _fields(d, 3, 6)
    comp = d.compile(tpl, precision="fp64")
    got = comp(p=q[0], vx=q[1], vy=q[2]).cpu().numpy()
    comp.check()
    assert rel_l2(got, _exec(d, tpl, {"p": q[0], "vx": q[1], "vy": q[2]})) <= 1e-12


def test_compiled_varwave_template_coefficient_and_source(cuda_device):
    d = hb.Discretization(rect(6), order=4)
    tpl = varwave_by_hand()
    rng = np.random.default_rng(2)
    c = np.repeat(rng.uniform(0.8, 1.2, d.K), d.Np)
    f = np.sin(d.nodes[:, 0])
    q = _fields(d, 3, 7)
    comp = d.compile(tpl, precision="fp64")
    with pytest.raises(ValueError):
        comp(q=q)                     # the coefficient field is required
    got = comp(q=q, speed=c, f=f).cpu().numpy()
    comp.check()
    assert rel_l2(got, _exec(d, tpl, {"q": q, "speed": c, "f": f})) <= 1e-12


@pytest.mark.parametrize("alpha", [1.0, 0.25])
def test_compiled_maxwell_template(cuda_device, alpha):
    d = hb.Discretization(box(3), order=3)
    tpl = maxwell_by_hand(alpha)
    q = _fields(d, 6, 8)
    comp = d.compile(tpl, precision="fp64")
    got = comp(em=q).cpu().numpy()
    comp.check()
    assert rel_l2(got, _exec(d, tpl, {"em": q})) <= 1e-12


@pytest.mark.parametrize("precision", ["fp64", "fp16x3"])
def test_template_and_descriptor_compile_alike(cuda_device, precision):
    d = hb.Discretization(box(3, 0.05, 2), order=4)
    op = hb.MaxwellOperator(1.0, 1.0, flux_type=1)
    q = _fields(d, 6, 9)
    a = d.compile(op.op_template(), precision=precision)(w=q)
    b = d.compile(op.descriptor(), precision=precision)(w=q)
    assert bool((a == b).all())


def test_bound_model_through_its_template(cuda_device):
    """model.bind compiles the template; the model's c array and source
    vector are bound from the model."""
    d = hb.Discretization(rect(6), order=3)
    rng = np.random.default_rng(3)
    c = np.repeat(rng.uniform(0.8, 1.2, d.K), d.Np)
    src = np.exp(-3 * (d.nodes ** 2).sum(1))
    op = hb.VariableVelocityStrongWaveOperator(c, 2, source=src)
    q = _fields(d, 3, 10)
    got = op.bind(d)(0.0, q).cpu().numpy()
    ref = _exec(d, op.op_template(), {"w": q, "c": c, "source": src})
    assert rel_l2(got, ref) <= 1e-12


@pytest.mark.parametrize("quadrature", [False, True])
def test_compiled_weak_advection(cuda_device, quadrature):
    """The weak form (nodal or over-integrated) compiled onto the strong
    advection kernel equals the executor run on the weak tree."""
    from test_optemplate import _in_out_tagger, weak_quadrature_advection
    v = np.array([0.7, -0.4])
    d = hb.Discretization(rect(6, tagger=_in_out_tagger(v)), order=4)
    tpl = weak_quadrature_advection(v, "upwind") if quadrature else \
        hb.WeakAdvectionOperator(v, inflow_tag="in", outflow_tag="out",
                                 flux_type="upwind").op_template()
    q = _fields(d, 1, 11)
    bc = np.cos(2 * d.get_boundary("in").nodes[:, 1])
    comp = d.compile(tpl, precision="fp64")
    got = comp(u=q[0], bc_in=bc).cpu().numpy()
    comp.check()
    assert rel_l2(got, _exec(d, tpl, {"u": q[0], "bc_in": bc})[0]) <= 1e-12
