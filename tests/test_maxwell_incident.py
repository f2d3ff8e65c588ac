"""Maxwell's incident-field boundary (em.py:289-307), host side: with the
reference's default incident data (zero) the exterior state is zero on the
incident faces, with incident data given per call as boundary vectors it
is minus the data; the jit-loop oracle and the template executor agree on
both (3D, TM, TE; fixed and variable material; every flux type); the
lowering names the incident kind and the data; bind checks that the tag is
covered; and data of the wrong shape is refused."""
import numpy as np
import pytest

import hedge_b200 as hb
from hedge_b200.lowering import lower
from hedge_b200.mesh import MeshError
from hedge_b200.models import BC_ABSORB, BC_INCIDENT, BC_PEC, BC_PMC

from conftest import rel_l2
from test_maxwell_material import FLUXES, _discr


def _op(cls, ft, bft, eps=1.3, mu=0.7):
    return cls(eps, mu, flux_type=ft, bdry_flux_type=bft, pec_tag="pec", pmc_tag="pmc",
               incident_tag="abs")


@pytest.mark.parametrize("ft,bft", FLUXES)
@pytest.mark.parametrize("kind", ["3d", "tm", "te"])
def test_oracle_equals_executor(kind, ft, bft):
    from oracle import OracleRHS
    from optemplate_exec import TemplateExecutor
    d, cls, F = _discr(kind)
    op = _op(cls, ft, bft)
    w = np.random.default_rng(2).standard_normal((F, len(d)))
    ref = np.asarray(TemplateExecutor(d)(op.op_template(), w=w), dtype=np.float64)
    got = OracleRHS(d, op.descriptor())(w)
    assert rel_l2(got, ref) <= 1e-12


@pytest.mark.parametrize("kind", ["3d", "tm", "te"])
def test_incident_differs_from_the_walls(kind):
    """The incident faces' RHS is none of the PEC, PMC, absorbing or
    flux-free faces' on the same tag (with a flux that is not the upwind
    one: with upwind fluxes the first-order absorbing state and a zero
    exterior give the same flux)."""
    from optemplate_exec import TemplateExecutor
    d, cls, F = _discr(kind)
    w = np.random.default_rng(3).standard_normal((F, len(d)))
    ex = TemplateExecutor(d)
    inc = np.asarray(ex(_op(cls, 0.5, 0.5).op_template(), w=w), dtype=np.float64)
    for kw in ({"absorb_tag": "abs"}, {"pmc_tag": "abs"}, {"pec_tag": "abs"}, {}):
        tags = dict({"pec_tag": "pec", "pmc_tag": "pmc"}, **kw)
        other = np.asarray(ex(cls(1.3, 0.7, flux_type=0.5, **tags).op_template(), w=w),
                           dtype=np.float64)
        assert rel_l2(other, inc) > 1e-3, kw
    up_inc = np.asarray(ex(_op(cls, 1, 1).op_template(), w=w), dtype=np.float64)
    up_abs = np.asarray(ex(cls(1.3, 0.7, flux_type=1, pec_tag="pec", pmc_tag="pmc",
                               absorb_tag="abs").op_template(), w=w), dtype=np.float64)
    assert rel_l2(up_abs, up_inc) <= 1e-13


@pytest.mark.parametrize("ft,bft", FLUXES)
@pytest.mark.parametrize("kind", ["3d", "tm", "te"])
def test_lowering_names_incident(kind, ft, bft):
    d, cls, F = _discr(kind)
    for eps in (1.3, np.linspace(1.0, 2.0, len(d))):
        op = _op(cls, ft, bft, eps=eps)
        desc = lower(op.op_template(), d.dimensions, d.mesh)
        bcs = dict(desc.bcs)
        # upwind boundary fluxes: the absorbing state and a zero exterior
        # give the same flux, and the lowering may name either
        want = (BC_INCIDENT, BC_ABSORB) if bft == 1 else (BC_INCIDENT,)
        assert bcs.pop("abs") in want
        assert bcs == {"pec": BC_PEC, "pmc": BC_PMC}
        assert desc.model == op.descriptor().model
        assert dict(op.descriptor().bcs)["abs"] == BC_INCIDENT


def test_variable_material_with_constant_fields_equals_fixed():
    """Variable material with constant fields and an incident wall equals the
    fixed-material template (the boundary vector carries B(eps), B(mu))."""
    from optemplate_exec import TemplateExecutor
    d, cls, F = _discr("3d")
    w = np.random.default_rng(4).standard_normal((F, len(d)))
    ex = TemplateExecutor(d)
    fixed = np.asarray(ex(_op(cls, 0.5, "lf").op_template(), w=w), dtype=np.float64)
    var = _op(cls, 0.5, "lf", eps=np.full(len(d), 1.3), mu=np.full(len(d), 0.7))
    got = np.asarray(ex(var.op_template(), w=w, epsilon=np.full(len(d), 1.3),
                        mu=np.full(len(d), 0.7)), dtype=np.float64)
    assert rel_l2(got, fixed) <= 1e-13


def _tag_pec_inc(fvi, el, fn, allv):
    return ["inc"] if allv[list(fvi)].mean(0)[0] > 0.99 else ["pec"]


def test_bind_checks_incident_coverage_and_refuses_data():
    from hedge_b200 import optemplate as ot
    from hedge_b200.discretization import build_face_table
    m = hb.make_box_tet_mesh(n=(2, 2, 2), jitter=0.03, seed=3, boundary_tagger=_tag_pec_inc)
    d = hb.Discretization(m, order=2)
    # the incident tag is part of bind's coverage check (em.py:373-377)
    from hedge_b200.mesh import check_bc_coverage
    op = hb.MaxwellOperator(1.0, 1.0, flux_type=0.5, pec_tag="pec", incident_tag="inc")
    check_bc_coverage(d.mesh, op.bc_tags())
    with pytest.raises(MeshError):
        hb.MaxwellOperator(1.0, 1.0, flux_type=0.5, pec_tag="pec").bind(d)
    conn = build_face_table(d, op.op_template())[0]
    n_inc = np.count_nonzero((conn[..., 0] < 0) & (conn[..., 1] == BC_INCIDENT))
    assert n_inc == len(d.mesh.boundary_faces("inc")) > 0
    with pytest.raises(ValueError):
        hb.MaxwellOperator(1.0, 1.0, flux_type=1, incident_tag="inc",
                           incident_bc=lambda o, e, h: ot.make_sym_vector("inc", 5))
    # zero data written out as a vector is the default
    hb.MaxwellOperator(1.0, 1.0, flux_type=1, incident_tag="inc",
                       incident_bc=lambda o, e, h: np.zeros(6, dtype=object))


def _inc_op(cls, F, ft=0.5, bft="lf", eps=1.3, mu=0.7):
    from hedge_b200 import optemplate as ot
    return cls(eps, mu, flux_type=ft, bdry_flux_type=bft, pec_tag="pec", pmc_tag="pmc",
               incident_tag="abs", incident_bc=lambda o, e, h: ot.make_sym_vector("inc", F))


def _inc_data(d, F, seed=5):
    x = d.get_boundary("abs").nodes
    rng = np.random.default_rng(seed)
    return np.stack([np.sin((f + 1) * x[:, 1] + 0.4 * f) + 0.1 * rng.standard_normal(len(x))
                     for f in range(F)])


@pytest.mark.parametrize("ft,bft", [(1, 1), (0.5, "lf"), ("lf", 0.3)])
@pytest.mark.parametrize("kind", ["3d", "tm", "te"])
def test_incident_data_oracle_equals_executor(kind, ft, bft):
    from oracle import OracleRHS
    from optemplate_exec import TemplateExecutor
    d, cls, F = _discr(kind)
    op = _inc_op(cls, F, ft, bft)
    w = np.random.default_rng(6).standard_normal((F, len(d)))
    g = _inc_data(d, F)
    ref = np.asarray(TemplateExecutor(d)(op.op_template(), w=w, inc=g), dtype=np.float64)
    got = OracleRHS(d, op.descriptor())(w, bc_in=g)
    assert rel_l2(got, ref) <= 1e-12
    # zero data is the default incident boundary
    zero = np.asarray(TemplateExecutor(d)(op.op_template(), w=w, inc=0 * g), dtype=np.float64)
    base = np.asarray(TemplateExecutor(d)(_op(cls, ft, bft).op_template(), w=w),
                      dtype=np.float64)
    assert rel_l2(zero, base) <= 1e-13


@pytest.mark.parametrize("kind", ["3d", "tm", "te"])
def test_lowering_names_incident_data(kind):
    from hedge_b200.discretization import build_face_table
    d, cls, F = _discr(kind)
    for eps in (1.3, np.linspace(1.0, 2.0, len(d))):
        op = _inc_op(cls, F, 1, 1, eps=eps)
        desc = lower(op.op_template(), d.dimensions, d.mesh)
        assert dict(desc.bcs) == {"pec": BC_PEC, "pmc": BC_PMC, "abs": BC_INCIDENT}
        assert desc.params.get("incident_data") is True
        assert desc.fields["given"] == "inc"
        assert op.descriptor().params.get("incident_data") is True
        conn, n_given, tag = build_face_table(d, op.op_template())
        assert tag == "abs" and n_given == len(d.mesh.boundary_faces("abs")) * d.Nfp
        b = -1 - conn[..., 0][conn[..., 1] == BC_INCIDENT]
        assert sorted(b.tolist()) == list(range(len(d.mesh.boundary_faces("abs"))))


def test_incident_data_components_named_one_by_one():
    from hedge_b200 import optemplate as ot
    d, cls, F = _discr("tm")
    data = np.array([ot.Field("ez_inc"), ot.Field("b_hx"), ot.Field("a_hy")], dtype=object)
    op = cls(1.0, 1.0, flux_type=0.5, pec_tag="pec", pmc_tag="pmc", incident_tag="abs",
             incident_bc=lambda o, e, h: data)
    desc = lower(op.op_template(), d.dimensions, d.mesh)
    assert desc.params.get("incident_data") is True
    assert [n for n, _ in desc.fields["given_keys"]] == ["ez_inc", "b_hx", "a_hy"]


def test_incident_data_of_the_state_is_refused():
    """Incident data that is an expression of the state (not a given
    boundary field) matches no kernel boundary condition."""
    from hedge_b200 import optemplate as ot
    d, cls, F = _discr("3d")
    op = cls(1.0, 1.0, flux_type=0.5, pec_tag="pec", pmc_tag="pmc", incident_tag="abs",
             incident_bc=lambda o, e, h: np.array(
                 [ot.BoundarizeOperator("abs")(x) for x in list(e) + list(h)], dtype=object))
    with pytest.raises(NotImplementedError):
        lower(op.op_template(), d.dimensions, d.mesh)
