"""Maxwell with spatially variable material on the GPU (the CUDA-core
kernels): the bound model's RHS against the CPU template executor on the
model's own template (FP64 <= 1e-12, FP32 <= 1e-5 on FP32-rounded inputs),
for smooth eps(x), mu(x) in 3D, TM and TE with PEC, PMC and absorbing walls
and every flux type; with a source current (given with the model and by
name per call); constant fields against the fixed-material kernel; 20
fused LSRK4 steps against the executor's; the material passed by name to a
compiled template; the split precisions and the adjoint refused."""
import numpy as np
import pytest

import hedge_b200 as hb
from conftest import rel_l2
from test_maxwell_material import FLUXES, _discr

pytestmark = pytest.mark.gpu


def _material(d):
    x = d.nodes
    eps = 1.0 + 0.4 * np.sin(1.7 * x[:, 0] + 0.3) * np.cos(0.9 * x[:, 1])
    mu = 1.2 + 0.3 * np.cos(1.1 * x[:, 1] - 0.2 * x[:, 0])
    return eps, mu


def _fields(d, F, seed):
    rng = np.random.default_rng(seed)
    x = d.nodes
    base = np.stack([np.sin(1.1 * (f + 1) * x[:, 0] + 0.5 * f) * np.cos(0.8 * x[:, -1] - 0.2 * f)
                     for f in range(F)])
    return base + 0.1 * rng.uniform(-1, 1, base.shape)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("ft,bft", FLUXES)
@pytest.mark.parametrize("kind", ["3d", "tm", "te"])
def test_variable_material_rhs(cuda_device, kind, ft, bft, precision):
    from optemplate_exec import TemplateExecutor
    d, cls, F = _discr(kind)
    eps, mu = _material(d)
    op = cls(eps, mu, flux_type=ft, bdry_flux_type=bft, pec_tag="pec", pmc_tag="pmc",
             absorb_tag="abs")
    q = _fields(d, F, 3)
    if precision == "fp32":
        q = q.astype(np.float32).astype(np.float64)
    ref = np.asarray(TemplateExecutor(d)(op.op_template(), w=q, epsilon=eps, mu=mu),
                     dtype=np.float64)
    dp = hb.Discretization(d.mesh, order=d.order, precision=precision)
    rhs = dp.compile(op.op_template()).bind_model(op)
    got = rhs(0.0, q).double().cpu().numpy()
    rhs.compiled.check()
    assert rel_l2(got, ref) <= (1e-12 if precision == "fp64" else 1e-5)


@pytest.mark.parametrize("kind", ["3d", "tm", "te"])
def test_constant_material_equals_fixed_kernel(cuda_device, kind):
    d, cls, F = _discr(kind)
    kw = dict(flux_type=0.7, bdry_flux_type=1, pec_tag="pec", pmc_tag="pmc", absorb_tag="abs")
    q = _fields(d, F, 4)
    fixed = d.compile(cls(1.4, 0.6, **kw).op_template())(w=q).cpu().numpy()
    var_op = cls(np.full(len(d), 1.4), np.full(len(d), 0.6), **kw)
    var = d.compile(var_op.op_template()).bind_model(var_op)(0.0, q).cpu().numpy()
    assert rel_l2(var, fixed) <= 1e-13


def test_variable_material_lsrk_steps(cuda_device):
    """20 LSRK4 steps of a 3D PEC cavity with variable material (fused
    stages, hb_lsrk_stage) against the executor's RHS in the same LSRK4
    loop on the CPU."""
    from optemplate_exec import TemplateExecutor
    from hedge_b200.timestep import RK4A, RK4B
    d = hb.Discretization(hb.make_box_tet_mesh(n=(2, 2, 2), jitter=0.03, seed=6), order=3)
    eps, mu = _material(d)
    op = hb.MaxwellOperator(eps, mu, flux_type=1)
    rhs = op.bind(d)
    dt = 0.5 * op.estimate_timestep(d)
    q = _fields(d, 6, 5)
    y = hb.LSRK4TimeStepper()
    yd = d.to_device(q).reshape(6, -1)
    ex = TemplateExecutor(d)
    tpl = op.op_template()
    yo, res, t = q.copy(), np.zeros_like(q), 0.0
    for _ in range(20):
        yd = y(yd, t, dt, rhs)
        for s in range(5):
            r = np.asarray(ex(tpl, w=yo, epsilon=eps, mu=mu), dtype=np.float64)
            res = RK4A[s] * res + dt * r
            yo = yo + RK4B[s] * res
        t += dt
    rhs.compiled.check()
    assert rel_l2(yd.cpu().numpy(), yo) <= 1e-11


def test_material_by_name_and_refusals(cuda_device):
    import torch
    from optemplate_exec import TemplateExecutor
    d, cls, F = _discr("3d")
    eps, mu = _material(d)
    from hedge_b200 import optemplate as ot
    op = hb.MaxwellOperator(ot.Field("epsilon"), ot.Field("mu"), flux_type=0.5,
                            pec_tag="pec", pmc_tag="pmc", absorb_tag="abs")
    tpl = op.op_template()
    comp = d.compile(tpl)
    q = _fields(d, F, 7)
    with pytest.raises(ValueError):
        comp(w=q)
    got = comp(w=q, epsilon=eps, mu=mu).cpu().numpy()
    ref = np.asarray(TemplateExecutor(d)(tpl, w=q, epsilon=eps, mu=mu), dtype=np.float64)
    assert rel_l2(got, ref) <= 1e-12
    for precision in ("fp16x3", "bf16x3"):
        with pytest.raises(NotImplementedError):
            d.compile(tpl, precision=precision)
    var = hb.MaxwellOperator(eps, mu, flux_type=1)
    c2 = var.bind(d).compiled
    lam = torch.ones((6, len(d)), dtype=torch.float64, device=d.device)
    with pytest.raises(Exception):
        c2.adjoint(lam)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("kind", ["3d", "tm", "te"])
def test_variable_material_current(cuda_device, kind, precision):
    """(curl H - J + lift) / eps(x) on the E rows: the current given with
    the model (bound RHS) and by name per call (compiled template), against
    the template executor."""
    from optemplate_exec import TemplateExecutor
    d, cls, F = _discr(kind)
    eps, mu = _material(d)
    ne = {"3d": 3, "tm": 1, "te": 2}[kind]
    x = d.nodes
    J = np.stack([np.cos((k + 1) * x[:, 0] - 0.3 * x[:, 1]) for k in range(ne)])
    op = cls(eps, mu, flux_type=0.5, bdry_flux_type="lf", pec_tag="pec", pmc_tag="pmc",
             absorb_tag="abs", current=J)
    q = _fields(d, F, 11)
    if precision == "fp32":
        q = q.astype(np.float32).astype(np.float64)
    tol = 1e-12 if precision == "fp64" else 1e-5
    ex = TemplateExecutor(d)
    tpl = op.op_template()
    ref = np.asarray(ex(tpl, w=q, epsilon=eps, mu=mu, current=J), dtype=np.float64)
    dp = hb.Discretization(d.mesh, order=d.order, precision=precision)
    rhs = dp.compile(tpl).bind_model(op)
    got = rhs(0.0, q).double().cpu().numpy()
    rhs.compiled.check()
    assert rel_l2(got, ref) <= tol
    ref2 = np.asarray(ex(tpl, w=q, epsilon=eps, mu=mu, current=-2 * J), dtype=np.float64)
    comp = dp.compile(tpl)
    got2 = comp(w=q, epsilon=eps, mu=mu, current=-2 * J).double().cpu().numpy()
    comp.check()
    assert rel_l2(got2, ref2) <= tol
