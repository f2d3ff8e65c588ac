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
