"""Maxwell's incident-field boundary with the reference's default (zero)
incident data (em.py:289-307) on the GPU: every kernel path against the
CPU oracle -- CUDA cores in FP64 and FP32, the FP32 and FP16x3 / BF16x3
tensor-core kernels (resident at 3D N = 3, 4; streamed at N = 5, 6) -- for
3D, TM and TE with PEC, PMC and incident walls and non-upwind fluxes (with
the upwind flux a zero exterior and the absorbing state give the same
flux); variable material against the template executor; the adjoint
against the oracle's Jacobian transpose; and 10 fused LSRK4 steps."""
import numpy as np
import pytest

import hedge_b200 as hb
from conftest import rel_l2
from test_gpu_parity import TOL, _fields
from test_maxwell_material import _discr

pytestmark = pytest.mark.gpu

TOLS = dict(TOL, fp16x3=1e-6, bf16x3=1e-5)


def _op(cls, ft, bft, eps=1.3, mu=0.7):
    return cls(eps, mu, flux_type=ft, bdry_flux_type=bft, pec_tag="pec", pmc_tag="pmc",
               incident_tag="abs")


def _check(d, op, precision, seed=0):
    from oracle import OracleRHS
    from hedge_b200.models import BC_INCIDENT
    tpl = op.op_template()
    comp = d.compile(tpl, precision=precision)
    assert dict(comp.ot.bcs)["abs"] == BC_INCIDENT
    q = _fields(d, op.n_fields, seed)
    if precision in ("fp32", "fp32-simt"):
        q = q.astype(np.float32).astype(np.float64)
    ref = OracleRHS(d, tpl)(q)
    got = comp(w=q).double().cpu().numpy().reshape(ref.shape)
    comp.check()
    err = rel_l2(got, ref)
    assert err <= TOLS[precision], (precision, err)


@pytest.mark.parametrize("ft,bft", [(0.5, 0.5), ("lf", 0.3), (1, 0.0)])
@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32-simt", "fp16x3", "bf16x3"])
@pytest.mark.parametrize("kind", ["3d", "tm", "te"])
def test_incident_rhs(cuda_device, kind, precision, ft, bft):
    d, cls, F = _discr(kind)
    if kind != "3d" and precision in ("fp16x3", "bf16x3"):
        pytest.skip("2D Maxwell has no split-precision kernel")
    _check(d, _op(cls, ft, bft), precision)


@pytest.mark.parametrize("order", [4, 5, 6])
def test_incident_split_orders(cuda_device, order):
    """FP16x3 at N = 4 (resident kernel) and N = 5, 6 (streamed kernel)."""
    from test_maxwell_material import _tagger
    m = hb.make_box_tet_mesh(n=(2, 2, 2), jitter=0.03, seed=5, boundary_tagger=_tagger)
    d = hb.Discretization(m, order=order)
    _check(d, _op(hb.MaxwellOperator, 0.5, "lf"), "fp16x3", seed=order)


@pytest.mark.parametrize("kind", ["3d", "tm", "te"])
def test_incident_variable_material(cuda_device, kind):
    from optemplate_exec import TemplateExecutor
    d, cls, F = _discr(kind)
    x = d.nodes
    eps = 1.0 + 0.4 * np.sin(1.7 * x[:, 0] + 0.3) * np.cos(0.9 * x[:, 1])
    mu = 1.2 + 0.3 * np.cos(1.1 * x[:, 1] - 0.2 * x[:, 0])
    op = _op(cls, 0.5, "lf", eps=eps, mu=mu)
    q = _fields(d, F, 3)
    ref = np.asarray(TemplateExecutor(d)(op.op_template(), w=q, epsilon=eps, mu=mu),
                     dtype=np.float64)
    rhs = d.compile(op.op_template()).bind_model(op)
    got = rhs(0.0, q).double().cpu().numpy()
    rhs.compiled.check()
    assert rel_l2(got, ref) <= 1e-12


@pytest.mark.parametrize("kind", ["3d", "tm"])
def test_incident_adjoint(cuda_device, kind):
    from test_gpu_adjoint import _check_adjoint
    from test_maxwell_material import _tagger
    if kind == "3d":
        m = hb.make_box_tet_mesh(n=(1, 1, 1), jitter=0.0, boundary_tagger=_tagger)
        d, cls = hb.Discretization(m, order=2), hb.MaxwellOperator
    else:
        d, cls, F = _discr(kind)
    _check_adjoint(d, _op(cls, 0.5, 0.5))


def test_incident_lsrk_steps(cuda_device):
    """10 LSRK4 steps through the fused stage against the oracle's loop."""
    from oracle import OracleRHS
    d, cls, F = _discr("3d")
    op = _op(cls, 0.5, "lf")
    rhs = d.compile(op.op_template()).bind_model(op)
    q = _fields(d, F, 9)
    dt = 0.5 * op.estimate_timestep(d)
    orc = OracleRHS(d, op.op_template())
    y = hb.LSRK4TimeStepper()
    yd = d.to_device(q).reshape(F, -1)
    yo, res, t = q.copy(), np.zeros_like(q), 0.0
    for _ in range(10):
        yd = y(yd, t, dt, rhs)
        yo, res = orc.lsrk4_step(yo, t, dt, res)
        t += dt
    rhs.compiled.check()
    assert rel_l2(yd.cpu().numpy(), yo) <= 1e-11


# -- incident data given per call --------------------------------------------

def _inc_op(cls, F, ft=0.5, bft="lf", eps=1.3, mu=0.7):
    from hedge_b200 import optemplate as ot
    return cls(eps, mu, flux_type=ft, bdry_flux_type=bft, pec_tag="pec", pmc_tag="pmc",
               incident_tag="abs", incident_bc=lambda o, e, h: ot.make_sym_vector("inc", F))


def _inc_data(d, F, seed=5):
    x = d.get_boundary("abs").nodes
    rng = np.random.default_rng(seed)
    return np.stack([np.sin((f + 1) * x[:, 1] + 0.4 * f) + 0.1 * rng.standard_normal(len(x))
                     for f in range(F)])


@pytest.mark.parametrize("ft,bft", [(1, 1), (0.5, "lf")])
@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32-simt"])
@pytest.mark.parametrize("kind", ["3d", "tm", "te"])
def test_incident_data_rhs(cuda_device, kind, precision, ft, bft):
    """The exterior state -data on the incident faces: the compiled template
    with the data by name, the bound model with it as extra context, and the
    data's components named one by one, against the oracle."""
    from oracle import OracleRHS
    d, cls, F = _discr(kind)
    op = _inc_op(cls, F, ft, bft)
    g = _inc_data(d, F)
    q = _fields(d, F, 4)
    if precision != "fp64":
        q = q.astype(np.float32).astype(np.float64)
        g = g.astype(np.float32).astype(np.float64)
    ref = OracleRHS(d, op.op_template())(q, bc_in=g)
    comp = d.compile(op.op_template(), precision=precision)
    got = comp(w=q, inc=g).double().cpu().numpy()
    comp.check()
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert rel_l2(got, ref) <= tol
    rhs = comp.bind_model(op)
    got2 = rhs(0.0, q, inc=[g[f] for f in range(F)]).double().cpu().numpy()
    assert rel_l2(got2, ref) <= tol
    with pytest.raises(ValueError):
        comp(w=q, inc=g[:, :-1])


def test_incident_data_variable_material(cuda_device):
    from optemplate_exec import TemplateExecutor
    d, cls, F = _discr("3d")
    x = d.nodes
    eps = 1.0 + 0.4 * np.sin(1.7 * x[:, 0] + 0.3)
    mu = 1.2 + 0.3 * np.cos(1.1 * x[:, 1])
    op = _inc_op(cls, F, 0.5, 0.5, eps=eps, mu=mu)
    g, q = _inc_data(d, F, 8), _fields(d, F, 8)
    ref = np.asarray(TemplateExecutor(d)(op.op_template(), w=q, inc=g, epsilon=eps, mu=mu),
                     dtype=np.float64)
    rhs = d.compile(op.op_template()).bind_model(op)
    got = rhs(0.0, q, inc=g).double().cpu().numpy()
    rhs.compiled.check()
    assert rel_l2(got, ref) <= 1e-12


def test_incident_data_lsrk_steps(cuda_device):
    """5 LSRK4 steps with the data as the stepper's extra context, against
    the oracle's loop."""
    from oracle import OracleRHS
    import torch
    d, cls, F = _discr("te")
    op = _inc_op(cls, F, 0.5, "lf")
    comp = d.compile(op.op_template())
    g = _inc_data(d, F, 9)
    gd = torch.as_tensor(g, device=d.device)
    q = _fields(d, F, 9)
    dt = 0.5 * op.estimate_timestep(d)
    orc = OracleRHS(d, op.op_template())
    yd = d.to_device(q).reshape(F, -1).contiguous()
    res = torch.zeros_like(yd)
    tmp = torch.empty_like(yd)
    from hedge_b200.timestep import RK4A, RK4B
    yo, reso, t = q.copy(), np.zeros_like(q), 0.0
    for _ in range(5):
        for a, b in zip(RK4A, RK4B):
            comp.lsrk_stage(a, b, dt, yd, tmp, res, bc_in=gd)
            yd, tmp = tmp, yd
        yo, reso = orc.lsrk4_step(yo, t, dt, reso, bc_fn=lambda s: g)
        t += dt
    comp.check()
    assert rel_l2(yd.cpu().numpy(), yo) <= 1e-11


def test_incident_data_refused_on_split_kernels(cuda_device):
    import torch
    from hedge_b200 import _native
    d, cls, F = _discr("3d")
    with pytest.raises(NotImplementedError):
        d.compile(_inc_op(cls, F).op_template(), precision="fp16x3")
    # the C ABI: incident data handed to a tensor-core Maxwell operator is
    # refused before any launch
    comp = d.compile(_op(cls, 0.5, "lf").op_template(), precision="fp16x3")
    q = comp.as_state(_fields(d, F, 1))
    out = torch.empty_like(q)
    data = torch.zeros(F * 64, dtype=torch.float64, device=d.device)
    st = comp._lib.hb_rhs(comp._handle, q.data_ptr(), out.data_ptr(), None, data.data_ptr(),
                          None, torch.cuda.current_stream().cuda_stream)
    assert st == _native.HB_ERR_UNSUPPORTED
