"""Maxwell with spatially variable material (em.py:38-100, 118-190, 309-371),
host side: the template with epsilon and mu as volume fields, evaluated by
the CPU template executor, equals the fixed-material template wherever the
fields are constant (3D, TM and TE; every flux type; PEC, PMC and absorbing
walls), the lowering recognises it as the Maxwell kernel with variable
material, and the constructor refuses what the path does not carry."""
import numpy as np
import pytest

import hedge_b200 as hb
from hedge_b200.lowering import lower
from hedge_b200.models import BC_ABSORB, BC_PEC, BC_PMC

from conftest import rel_l2
from test_optemplate import box, rect


def _tagger(fvi, el, fn, allv):
    c = allv[list(fvi)].mean(0)
    return ["abs"] if c[0] > 0.99 else (["pmc"] if c[0] < -0.99 else ["pec"])


def _discr(kind):
    if kind == "3d":
        m = hb.make_box_tet_mesh(n=(2, 2, 2), jitter=0.03, seed=3, boundary_tagger=_tagger)
        return hb.Discretization(m, order=3), hb.MaxwellOperator, 6
    m = hb.make_regular_rect_mesh((-1, -1), (1, 1), (5, 5), jitter=0.03, seed=4,
                                  boundary_tagger=_tagger)
    cls = hb.TMMaxwellOperator if kind == "tm" else hb.TEMaxwellOperator
    return hb.Discretization(m, order=3), cls, 3


FLUXES = [(1, 1), (0.5, "lf"), ("lf", 0.3), (0.0, 0.0)]


@pytest.mark.parametrize("ft,bft", FLUXES)
@pytest.mark.parametrize("kind", ["3d", "tm", "te"])
def test_constant_fields_equal_fixed_material(kind, ft, bft):
    from optemplate_exec import TemplateExecutor
    d, cls, F = _discr(kind)
    kw = dict(flux_type=ft, bdry_flux_type=bft, pec_tag="pec", pmc_tag="pmc", absorb_tag="abs")
    fixed = cls(1.3, 0.7, **kw)
    var = cls(np.full(len(d), 1.3), np.full(len(d), 0.7), **kw)
    w = np.random.default_rng(1).standard_normal((F, len(d)))
    ex = TemplateExecutor(d)
    rf = np.asarray(ex(fixed.op_template(), w=w), dtype=np.float64)
    rv = np.asarray(ex(var.op_template(), w=w, epsilon=np.full(len(d), 1.3),
                       mu=np.full(len(d), 0.7)), dtype=np.float64)
    assert rel_l2(rv, rf) <= 1e-13


@pytest.mark.parametrize("ft,bft", FLUXES)
@pytest.mark.parametrize("kind", ["3d", "tm", "te"])
def test_lowering_recognises_variable_material(kind, ft, bft):
    d, cls, F = _discr(kind)
    op = cls(np.linspace(1.0, 2.0, len(d)), 0.8, flux_type=ft, bdry_flux_type=bft,
             pec_tag="pec", pmc_tag="pmc", absorb_tag="abs")
    desc = lower(op.op_template(), d.dimensions, d.mesh)
    want = op.descriptor()
    assert desc.model == want.model
    assert desc.params.get("variable_material") is True
    assert desc.flux_type == want.flux_type
    assert abs(desc.params["alpha"] - want.params["alpha"]) <= 1e-9
    if bft == 0.0:
        # on a boundary both sides have the same impedance, so the numeric
        # flux with alpha = 0 is the "lf" flux: either lowering is exact
        assert desc.params["bdry_flux_type"] == 1 or abs(desc.params["bdry_alpha"]) <= 1e-9
    else:
        for k in ("bdry_flux_type", "bdry_alpha"):
            assert abs(desc.params[k] - want.params[k]) <= 1e-9, k
    assert dict(desc.bcs) == {"pec": BC_PEC, "pmc": BC_PMC, "abs": BC_ABSORB}
    assert desc.fields["coeffs"] == [("epsilon", None), ("mu", None)]


def test_material_arguments():
    d, cls, F = _discr("3d")
    x = d.nodes
    eps = hb.TimeConstantGivenFunction(lambda p: 1.0 + 0.5 * p[..., 0] ** 2)
    op = hb.MaxwellOperator(eps, lambda p: 2.0 + 0.0 * p[..., 0], flux_type=1)
    e, m = op.material_values(d)
    assert np.allclose(e, 1.0 + 0.5 * x[:, 0] ** 2) and np.allclose(m, 2.0)
    assert not op.fixed_material
    lam = op.max_eigenvalue(discr=d)
    assert abs(lam - np.max(1 / np.sqrt(e * m))) <= 1e-15
    assert op.estimate_timestep(d) > 0
    with pytest.raises(ValueError):
        op.max_eigenvalue()
    with pytest.raises(RuntimeError):
        op.c
    # a source current with variable material (em.py:192-214, 339-371)
    hb.MaxwellOperator(np.ones(len(d)), 1.0, flux_type=1, current=1.0)
    fixed = hb.MaxwellOperator(2.0, 0.5, flux_type=1)
    assert fixed.fixed_material and abs(fixed.c - 1.0) <= 1e-15


@pytest.mark.parametrize("kind", ["3d", "tm", "te"])
def test_variable_material_with_current(kind):
    """A source current with variable material: the template's E rows read
    (curl H - J + lift) / eps; with constant fields it equals the fixed
    material's template with the same current, and the lowering names the
    current as the E rows' source field."""
    from optemplate_exec import TemplateExecutor
    d, cls, F = _discr(kind)
    ne = {"3d": 3, "tm": 1, "te": 2}[kind]
    rng = np.random.default_rng(7)
    J = rng.standard_normal((ne, len(d)))
    kw = dict(flux_type=0.5, pec_tag="pec", pmc_tag="pmc", absorb_tag="abs", current=J)
    w = rng.standard_normal((F, len(d)))
    ex = TemplateExecutor(d)
    fixed = np.asarray(ex(cls(1.3, 0.7, **kw).op_template(), w=w, current=J), dtype=np.float64)
    var = cls(np.full(len(d), 1.3), np.full(len(d), 0.7), **kw)
    got = np.asarray(ex(var.op_template(), w=w, current=J, epsilon=np.full(len(d), 1.3),
                        mu=np.full(len(d), 0.7)), dtype=np.float64)
    assert rel_l2(got, fixed) <= 1e-13
    desc = lower(var.op_template(), d.dimensions, d.mesh)
    assert desc.params.get("variable_material") is True
    src = desc.fields["sources"]
    assert [o for o, _, _, _ in src] == list(range(ne))
    assert all(f == ("current", o) and abs(c + 1.0) <= 1e-9 and k == 0.0
               for o, k, f, c in src)


@pytest.mark.parametrize("ft,bft", FLUXES)
@pytest.mark.parametrize("kind", ["3d", "tm", "te"])
def test_oracle_variable_material_equals_executor(kind, ft, bft):
    """The jit-loop oracle with variable material (flux argument
    (epsilon, mu, w), impedances from each side, the local absorbing
    impedance, the per-node divisor) against the template executor, with
    PEC, PMC and absorbing walls, and with incident walls and a current."""
    from oracle import OracleRHS
    from optemplate_exec import TemplateExecutor
    d, cls, F = _discr(kind)
    x = d.nodes
    eps = 1.0 + 0.4 * np.sin(1.7 * x[:, 0] + 0.3) * np.cos(0.9 * x[:, 1])
    mu = 1.2 + 0.3 * np.cos(1.1 * x[:, 1] - 0.2 * x[:, 0])
    w = np.random.default_rng(8).standard_normal((F, len(d)))
    ex = TemplateExecutor(d)
    op = cls(eps, mu, flux_type=ft, bdry_flux_type=bft, pec_tag="pec", pmc_tag="pmc",
             absorb_tag="abs")
    ref = np.asarray(ex(op.op_template(), w=w, epsilon=eps, mu=mu), dtype=np.float64)
    assert rel_l2(OracleRHS(d, op.op_template())(w), ref) <= 1e-12
    ne = {"3d": 3, "tm": 1, "te": 2}[kind]
    J = np.cos(x[:, :1].T * np.arange(1, ne + 1)[:, None])
    op2 = cls(eps, mu, flux_type=ft, bdry_flux_type=bft, pec_tag="pec", pmc_tag="pmc",
              incident_tag="abs", current=J)
    ref2 = np.asarray(ex(op2.op_template(), w=w, epsilon=eps, mu=mu, current=J),
                      dtype=np.float64)
    assert rel_l2(OracleRHS(d, op2.op_template())(w), ref2) <= 1e-12
