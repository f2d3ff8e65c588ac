"""Diagnostics on the GPU: the DG gradient / divergence (evaluated with the
wave kernel) against the CPU executor of their reference templates, and the
electromagnetic log quantities against host computations."""
import numpy as np
import pytest

import hedge_b200 as hb
from hedge_b200 import log as hlog
from hedge_b200.mesh import TAG_ALL
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _exec(d, tpl, **env):
    from optemplate_exec import TemplateExecutor
    return TemplateExecutor(d)(tpl, **env)


@pytest.mark.parametrize("dim", [2, 3])
def test_gradient_divergence_match_templates(cuda_device, dim):
    m = hb.make_regular_rect_mesh((-1, -1), (1, 1), (6, 6), jitter=0.03, seed=0) if dim == 2 \
        else hb.make_box_tet_mesh(n=(3, 3, 3), jitter=0.03, seed=1)
    d = hb.Discretization(m, order=4)
    b = d.get_boundary(TAG_ALL).vol_indices
    x = d.nodes
    u = np.sin(x[:, 0]) * np.cos(1.3 * x[:, 1]) + x[:, -1] ** 2
    g = hb.GradientOperator(dim).bind(d)(u).cpu().numpy()
    assert rel_l2(g, _exec(d, hb.GradientOperator(dim).op_template(), u=u, bc=u[b])) <= 1e-12
    v = np.stack([np.cos(x[:, k] + 0.3 * k) * x[:, (k + 1) % dim] for k in range(dim)])
    dv = hb.DivergenceOperator(dim).bind(d)(v).cpu().numpy()
    ref = _exec(d, hb.DivergenceOperator(dim).op_template(), v=v, bc=v[:, b])[0]
    assert rel_l2(dv, ref) <= 1e-12


def test_em_quantities(cuda_device):
    d = hb.Discretization(hb.make_box_tet_mesh(n=(3, 3, 3), jitter=0.03, seed=2), order=3)
    op = hb.MaxwellOperator(2.0, 0.5, flux_type=1)
    x = d.nodes
    rng = np.random.default_rng(3)
    w = np.stack([np.sin((k + 1) * x[:, k % 3]) + 0.1 * rng.standard_normal(len(d))
                  for k in range(6)])
    fields = hlog.EMFieldGetter(d, op, lambda: w)
    mgr = hlog.LogManager()
    hlog.add_em_quantities(mgr, op, fields)
    mgr.tick()
    M = d.ldis.mass_matrix
    J = np.abs(d.mesh.jacobians)

    def integral(f):
        return float(np.einsum("j,kj,k->", M.sum(0), f.reshape(d.K, d.Np), J))

    e, h = w[:3], w[3:]
    assert np.isclose(mgr.get_series("W_el")[0], integral(0.5 * 2.0 * (e * e).sum(0)), rtol=1e-12)
    assert np.isclose(mgr.get_series("W_mag")[0], integral(0.5 * 0.5 * (h * h).sum(0)), rtol=1e-12)
    s = np.cross(e.T, h.T).T
    for i, a in enumerate("xyz"):
        assert np.isclose(mgr.get_series("p%s_field" % a)[0], integral(s[i] / op.c ** 2),
                          rtol=1e-11, atol=1e-13)
    b = d.get_boundary(TAG_ALL).vol_indices
    div = hb.DivergenceOperator(3).op_template()
    dd = _exec(d, div, v=2.0 * e, bc=(2.0 * e)[:, b])[0]
    db = _exec(d, div, v=0.5 * h, bc=(0.5 * h)[:, b])[0]
    assert np.isclose(mgr.get_series("divD")[0], integral(dd), rtol=1e-9, atol=1e-12)
    assert np.isclose(mgr.get_series("divB")[0], integral(db), rtol=1e-9, atol=1e-12)
    assert np.isclose(mgr.get_series("err_divB_l1")[0], integral(np.abs(db)), rtol=1e-11)
