"""Operator templates (CPU): the models' symbolic templates, their lowering
onto the kernel models, and hand-written templates.

* every model template lowers to the model's own descriptor;
* the CPU template executor (oracle/optemplate_exec.py), which evaluates a
  tree node by node like the reference's jit executor, agrees with the C
  oracle on the model templates (rel-L2 <= 1e-12) -- this pins the
  templates to the reference formulas the oracle restates;
* hand-written templates (other field names, rearranged algebra, per-tag
  boundary conditions) lower to the right kernel model, and the oracle run
  on the lowered descriptor agrees with the executor run on the tree -- this
  pins the lowering;
* templates outside the path raise NotImplementedError.
"""
import numpy as np
import pytest

import hedge_b200 as hb
from hedge_b200 import flux as fl
from hedge_b200 import optemplate as ot
from hedge_b200.lowering import lower
from hedge_b200.mesh import TAG_ALL, TAG_NONE
from hedge_b200.models import (BC_ABSORB, BC_DIRICHLET, BC_GIVEN, BC_NEUMANN, BC_PEC,
                               BC_PMC, BC_RADIATION, MODEL_ADVECTION, MODEL_MAXWELL,
                               MODEL_VARWAVE, MODEL_WAVE)

from conftest import rel_l2


def rect(n=6, periodic=False, jitter=0.02, seed=0, tagger=None):
    kw = {"boundary_tagger": tagger} if tagger else {}
    return hb.make_regular_rect_mesh((-1, -1), (1, 1), (n, n),
                                     periodicity=(periodic, periodic) if periodic else None,
                                     jitter=jitter, seed=seed, **kw)


def box(n=2, jitter=0.03, seed=1, tagger=None):
    kw = {"boundary_tagger": tagger} if tagger else {}
    return hb.make_box_tet_mesh(n=(n, n, n), jitter=jitter, seed=seed, **kw)


def _fields(d, F, seed):
    rng = np.random.default_rng(seed)
    x = d.nodes
    return np.stack([np.sin(1.1 * (f + 1) * x[:, 0] + 0.4 * f) * np.cos(0.8 * x[:, -1])
                     + 0.1 * rng.uniform(-1, 1, len(d)) for f in range(F)])


def _same_descriptor(a, b):
    assert a.model == b.model and a.n_fields == b.n_fields and a.flux_type == b.flux_type
    for k, v in b.params.items():
        if k == "source":
            continue
        assert np.allclose(a.params[k], v, rtol=1e-12, atol=1e-12), (k, a.params[k], v)
    keep = {(t, k) for t, k in b.bcs if t is not TAG_NONE and k != 0}
    assert set(a.bcs) <= {(t, k) for t, k in b.bcs}
    # every tag the model gives a flux-carrying condition appears
    assert {t for t, k in keep} <= {t for t, _ in a.bcs} | {
        t for t, k in keep if k == BC_GIVEN and t is TAG_NONE}


def _tagger_lr(names):
    def tagger(fvi, el, fn, allv):
        x = allv[list(fvi)].mean(0)
        if x[0] < -0.99:
            return [names[0]]
        if x[0] > 0.99:
            return [names[1]]
        return [names[2]]
    return tagger


MODELS = [
    lambda: hb.StrongAdvectionOperator(np.array([1.0, 0.5]), flux_type="upwind"),
    lambda: hb.StrongAdvectionOperator(np.array([0.6, -0.8]), flux_type="central",
                                       inflow_tag=TAG_ALL),
    lambda: hb.StrongAdvectionOperator(np.array([0.3, 0.2, -0.4]), flux_type="lf"),
    lambda: hb.StrongWaveOperator(-0.7, 2, flux_type="upwind"),
    lambda: hb.StrongWaveOperator(1.0, 2, flux_type="central", dirichlet_tag="dir",
                                  neumann_tag="neu", radiation_tag="rad", source_f=0.25),
    lambda: hb.StrongWaveOperator(1.3, 3),
    lambda: hb.StrongWaveOperator(0.9, 2, dirichlet_tag="dir", dirichlet_bc_f=1,
                                  neumann_tag="neu"),
    lambda: hb.VariableVelocityStrongWaveOperator(np.ones(3), 2, time_sign=-1,
                                                  radiation_tag="rad", dirichlet_tag="dir"),
    lambda: hb.MaxwellOperator(1.0, 1.0, flux_type=1),
    lambda: hb.MaxwellOperator(2.0, 0.5, flux_type=0.5, bdry_flux_type="lf",
                               pec_tag="pec", pmc_tag="pmc", absorb_tag="abs"),
    lambda: hb.TMMaxwellOperator(1.0, 1.0, flux_type=1),
    lambda: hb.TEMaxwellOperator(1.5, 0.5, flux_type=0.25, bdry_flux_type="lf",
                                 pec_tag="pec", absorb_tag="abs"),
]


@pytest.mark.parametrize("make", MODELS)
def test_model_templates_lower_to_their_descriptors(make):
    m = make()
    _same_descriptor(lower(m.op_template(), m.dimensions), m.descriptor())


def _executor_vs_oracle(d, template, desc, env, q, bc_in=None, c_field=None, source=None):
    from oracle import OracleRHS
    from optemplate_exec import TemplateExecutor
    got = TemplateExecutor(d)(template, **env)
    ref = OracleRHS(d, desc, c_field=c_field, source=source)(q, bc_in=bc_in)
    assert got.shape == ref.shape
    return rel_l2(got, ref)


CASES = ["adv_periodic", "adv_inflow", "wave_mixed", "wave_dirichlet_data", "wave3d",
         "varwave", "maxwell_pec", "maxwell_mixed"]


@pytest.mark.parametrize("case", CASES)
def test_model_templates_match_oracle(case):
    """The model templates, executed as trees, equal the C oracle's RHS."""
    bc = c = src = None
    if case == "adv_periodic":
        d = hb.Discretization(rect(6, True, 0.0), order=3)
        op = hb.StrongAdvectionOperator(np.array([1.0, 0.5]), flux_type="upwind")
    elif case == "adv_inflow":
        d = hb.Discretization(rect(5, tagger=lambda *a: ["inflow"]), order=3)
        op = hb.StrongAdvectionOperator(np.array([0.6, -0.8]), flux_type="lf",
                                        inflow_tag="inflow")
        bc = np.sin(3 * d.get_boundary("inflow").nodes[:, 0])
    elif case == "wave_mixed":
        d = hb.Discretization(rect(5, tagger=_tagger_lr(["neu", "rad", "dir"])), order=3)
        op = hb.StrongWaveOperator(-0.8, 2, dirichlet_tag="dir", neumann_tag="neu",
                                   radiation_tag="rad", source_f=0.3)
    elif case == "wave_dirichlet_data":
        d = hb.Discretization(rect(5, tagger=_tagger_lr(["neu", "dir", "dir"])), order=3)
        op = hb.StrongWaveOperator(0.9, 2, dirichlet_tag="dir", dirichlet_bc_f=1,
                                   neumann_tag="neu")
        bc = np.cos(2 * d.get_boundary("dir").nodes[:, 1])
    elif case == "wave3d":
        d = hb.Discretization(box(2), order=2)
        op = hb.StrongWaveOperator(1.0, 3, flux_type="central")
    elif case == "varwave":
        d = hb.Discretization(rect(5, tagger=_tagger_lr(["dir", "rad", "dir"])), order=3)
        rng = np.random.default_rng(4)
        c = np.repeat(rng.uniform(0.8, 1.2, d.K), d.Np)
        src = np.exp(-4 * (d.nodes ** 2).sum(1))
        op = hb.VariableVelocityStrongWaveOperator(c, 2, source=src, dirichlet_tag="dir",
                                                   radiation_tag="rad", time_sign=-1)
    elif case == "maxwell_pec":
        d = hb.Discretization(box(2), order=2)
        op = hb.MaxwellOperator(1.0, 1.0, flux_type=1)
    else:
        def tagger(fvi, el, fn, allv):
            x = allv[list(fvi)].mean(0)
            return ["abs"] if x[2] > 0.99 else (["pmc"] if x[2] < -0.99 else ["pec"])
        d = hb.Discretization(box(2, tagger=tagger), order=2)
        op = hb.MaxwellOperator(2.0, 0.5, flux_type=0.5, bdry_flux_type="lf",
                                pec_tag="pec", pmc_tag="pmc", absorb_tag="abs")
    desc = op.descriptor()
    q = _fields(d, desc.n_fields, 3)
    if desc.model == MODEL_ADVECTION:
        env = {"u": q[0], "bc_in": bc if bc is not None else 0.0}
    else:
        env = {"w": q}
        if bc is not None:
            env["dir_bc_u"] = bc
    if c is not None:
        env["c"] = c
    if src is not None:
        env["source"] = src
    err = _executor_vs_oracle(d, op.op_template(), desc, env, q, bc_in=bc, c_field=c,
                              source=src)
    assert err <= 1e-12, err


# --------------------------------------------------------------------------
# hand-written templates

def advection_by_hand(v, tag):
    """Upwind advection written out: field 'phi', inflow data 'g'."""
    phi, g = ot.Field("phi"), ot.Field("g")
    u = fl.FluxScalarPlaceholder(0)
    n = fl.make_normal(len(v))
    nv = n[0] * v[0] + n[1] * v[1]
    flux = nv * (u.int - fl.IfPositive(nv, u.int, u.ext))
    F = ot.FluxOperator(flux)
    grad = [ot.DifferentiationOperator(i)(phi) for i in range(2)]
    return -(v[0] * grad[0] + v[1] * grad[1]) + ot.InverseMassOperator()(
        F(phi) + F(ot.BoundaryPair(phi, g, tag)))


def wave_by_hand(c, tags):
    """2D wave with separately named fields (p, vx, vy), central flux,
    Dirichlet on tags[0] and Neumann on tags[1]."""
    p, vx, vy = ot.Field("p"), ot.Field("vx"), ot.Field("vy")
    w = ot.join_fields(p, vx, vy)
    W = fl.FluxVectorPlaceholder(3)
    n = fl.make_normal(2)
    # c * (jump terms) of the central strong-form flux, written per component
    fu = -c * 0.5 * ((W[1].int - W[1].ext) * n[0] + (W[2].int - W[2].ext) * n[1])
    fv = [-c * 0.5 * (W[0].int - W[0].ext) * n[i] for i in range(2)]
    Fop = ot.get_flux_operator(ot.join_fields(fu, fv[0], fv[1]))
    B0, B1 = ot.BoundarizeOperator(tags[0]), ot.BoundarizeOperator(tags[1])
    dir_bc = ot.join_fields(-B0(p), B0(vx), B0(vy))
    neu_bc = ot.join_fields(B1(p), -B1(vx), -B1(vy))
    D = ot.make_nabla(2)
    vol = ot.join_fields(c * (D[0](vx) + D[1](vy)), c * D[0](p), c * D[1](p))
    return vol + ot.InverseMassOperator()(
        Fop(w) + Fop(ot.BoundaryPair(w, dir_bc, tags[0]))
        + Fop(ot.BoundaryPair(w, neu_bc, tags[1])))


def varwave_by_hand():
    """Variable-speed wave with coefficient 'speed' and source 2*f."""
    w = ot.make_sym_vector("q", 3)
    speed = ot.Field("speed")
    m = hb.VariableVelocityStrongWaveOperator(speed, 2, flux_type="upwind",
                                              source=2 * ot.Field("f"))
    return m.op_template(w=w)


def maxwell_by_hand(alpha):
    """Maxwell with eps = mu = 1 written with explicit curls, PEC walls."""
    w = ot.make_sym_vector("em", 6)
    e, h = w[:3], w[3:]
    D = ot.make_nabla(3)
    curl = ot.cross
    W = fl.FluxVectorPlaceholder(6)
    n = fl.make_normal(3)
    de = W[0:3].int - W[0:3].ext
    dh = W[3:6].int - W[3:6].ext
    fe = -0.5 * curl(n, dh - alpha * curl(n, de))
    fh = 0.5 * curl(n, de + alpha * curl(n, dh))
    Fop = ot.get_flux_operator(ot.join_fields(fe, fh))
    B = ot.BoundarizeOperator(TAG_ALL)
    pec = ot.join_fields(-B(e), B(h))
    return ot.join_fields(curl(D, h), -curl(D, e)) + ot.InverseMassOperator()(
        Fop(w) + Fop(ot.BoundaryPair(w, pec, TAG_ALL)))


def test_hand_written_advection():
    d = hb.Discretization(rect(5, tagger=lambda *a: ["in"]), order=3)
    tpl = advection_by_hand(np.array([0.7, -0.4]), "in")
    desc = lower(tpl, 2)
    assert desc.model == MODEL_ADVECTION and desc.flux_type == 1
    assert np.allclose(desc.params["v"], [0.7, -0.4]) and desc.bcs == [("in", BC_GIVEN)]
    assert desc.fields["state"] == "phi" and desc.fields["given"] == "g"
    q = _fields(d, 1, 5)
    bc = np.cos(2 * d.get_boundary("in").nodes[:, 1])
    err = _executor_vs_oracle(d, tpl, desc, {"phi": q[0], "g": bc}, q, bc_in=bc)
    assert err <= 1e-12, err


def test_hand_written_wave_named_fields():
    d = hb.Discretization(rect(5, tagger=_tagger_lr(["neu", "dir", "dir"])), order=3)
    tpl = wave_by_hand(1.2, ("dir", "neu"))
    desc = lower(tpl, 2)
    assert desc.model == MODEL_WAVE and desc.flux_type == 0
    assert np.isclose(desc.params["c"], 1.2)
    assert set(desc.bcs) == {("dir", BC_DIRICHLET), ("neu", BC_NEUMANN)}
    assert desc.fields["state_keys"] == [("p", None), ("vx", None), ("vy", None)]
    q = _fields(d, 3, 6)
    err = _executor_vs_oracle(d, tpl, desc, {"p": q[0], "vx": q[1], "vy": q[2]}, q)
    assert err <= 1e-12, err


def test_hand_written_varwave_source():
    d = hb.Discretization(rect(5), order=3)
    desc = lower(varwave_by_hand(), 2)
    assert desc.model == MODEL_VARWAVE and desc.fields["coeff"] == "speed"
    # the template's output 0 carries -2 f (the model subtracts its source)
    assert desc.fields["source"] == ("f", None) and desc.fields["source_coef"] == -2.0
    rng = np.random.default_rng(2)
    c = np.repeat(rng.uniform(0.8, 1.2, d.K), d.Np)
    f = np.sin(d.nodes[:, 0])
    q = _fields(d, 3, 7)
    err = _executor_vs_oracle(d, varwave_by_hand(), desc,
                              {"q": q, "speed": c, "f": f}, q, c_field=c, source=2 * f)
    assert err <= 1e-12, err


@pytest.mark.parametrize("alpha", [1.0, 0.25])
def test_hand_written_maxwell(alpha):
    d = hb.Discretization(box(2), order=2)
    tpl = maxwell_by_hand(alpha)
    desc = lower(tpl, 3)
    assert desc.model == MODEL_MAXWELL and desc.flux_type == 0
    assert np.isclose(desc.params["alpha"], alpha) and np.isclose(desc.params["bdry_alpha"], alpha)
    assert desc.bcs == [(TAG_ALL, BC_PEC)]
    q = _fields(d, 6, 8)
    err = _executor_vs_oracle(d, tpl, desc, {"em": q}, q)
    assert err <= 1e-12, err


def test_per_tag_conditions_beyond_one_tag_per_kind():
    """Two Dirichlet tags and a radiation tag (the model class has one tag
    per kind; the lowered table has any number)."""
    w = ot.make_sym_vector("w", 3)
    parts = []
    for tag in ("a", "b"):
        m = hb.StrongWaveOperator(1.0, 2, dirichlet_tag=tag)
        parts.append(m.op_template(w=w))
    m = hb.StrongWaveOperator(1.0, 2, dirichlet_tag=TAG_NONE, radiation_tag="r")
    bare = hb.StrongWaveOperator(1.0, 2, dirichlet_tag=TAG_NONE).op_template(w=w)
    # interior and volume terms once, boundary terms of the three templates
    tpl = m.op_template(w=w) + (parts[0] - bare) + (parts[1] - bare)
    desc = lower(tpl, 2)
    assert set(desc.bcs) == {("a", BC_DIRICHLET), ("b", BC_DIRICHLET), ("r", BC_RADIATION)}


def test_nonmodel_templates_raise():
    u = ot.Field("u")
    U = fl.FluxScalarPlaceholder(0)
    n = fl.make_normal(2)
    D = ot.make_nabla(2)
    central = ot.FluxOperator(0.5 * (U.int - U.ext) * n[0])
    M = ot.InverseMassOperator()
    bad = {
        "mass operator": -D[0](u) + ot.MassOperator()(u),
        "flux outside the inverse mass": -D[0](u) + central(u),
        "derivative of a product": -D[0](2 * u * u) + M(central(u)),
        "nonlinear flux": -D[0](u) + M(ot.FluxOperator(U.int * U.ext * n[0])(u)),
        "penalty term": -D[0](u) + M(ot.FluxOperator(fl.PenaltyTerm() * (U.int - U.ext))(u)),
        "volume term under the inverse mass": M(D[0](u) + central(u)),
        "nonlinear volume term": -D[0](u) * u + M(central(u)),
        "boundary data a multiple of the interior": -D[0](u) + M(central(u) + central(
            ot.BoundaryPair(u, 3 * ot.BoundarizeOperator("out")(u), "out"))),
        "weak derivative outside the inverse mass": ot.StiffnessTOperator(0)(u)
        + M(central(u)),
        "weak derivative of a product": M(ot.StiffnessTOperator(0)(ot.Field("c") * u)
                                          + central(u)),
    }
    for what, tpl in bad.items():
        with pytest.raises(NotImplementedError):
            lower(tpl, 2)
            pytest.fail(what)


def test_zero_boundary_flux_lowers_to_no_condition():
    """Extrapolated boundary data (ext = int) gives a zero central flux."""
    u = ot.Field("u")
    U = fl.FluxScalarPlaceholder(0)
    n = fl.make_normal(2)
    central = ot.FluxOperator(0.5 * (U.int - U.ext) * n[0])
    tpl = -ot.DifferentiationOperator(0)(u) + ot.InverseMassOperator()(
        central(u) + central(ot.BoundaryPair(u, ot.BoundarizeOperator("out")(u), "out")))
    desc = lower(tpl, 2)
    assert desc.model == MODEL_ADVECTION and desc.bcs == [("out", 0)]


def test_wrong_wave_boundary_raises():
    w = ot.make_sym_vector("w", 3)
    m = hb.StrongWaveOperator(1.0, 2, dirichlet_tag=TAG_NONE)
    tpl = m.op_template(w=w)
    Fop = ot.get_flux_operator(m.flux())
    B = ot.BoundarizeOperator("x")
    tpl = tpl + ot.InverseMassOperator()(Fop(ot.BoundaryPair(w, 2.0 * B(w), "x")))
    with pytest.raises(NotImplementedError, match="boundary"):
        lower(tpl, 2)


def test_template_arithmetic_prunes_zeros():
    u = ot.Field("u")
    assert ot.is_zero(0 * u) and (0 + u) is u and (u * 1) is u
    D = ot.make_nabla(2)
    e = np.dot(np.array([0.0, 2.0]), D * u)
    assert isinstance(e, ot.OperatorBinding) or isinstance(e, ot.Product)
    assert "d/dx0" not in str(e)


@pytest.mark.parametrize("dim", [2, 3])
def test_nd_calculus_templates_equal_wave_pieces(dim):
    """The DG gradient (divergence) template equals the v-part (u-part) of
    the central-flux wave template with c = 1 and Neumann (Dirichlet) walls,
    which is how nd_calculus evaluates them."""
    from optemplate_exec import TemplateExecutor
    d = hb.Discretization(rect(5) if dim == 2 else box(2), order=3)
    ex = TemplateExecutor(d)
    b = d.get_boundary(TAG_ALL).vol_indices
    x = d.nodes
    u = np.sin(x[:, 0]) * np.cos(x[:, 1]) + x[:, -1] ** 3
    w = np.zeros((dim + 1, len(d)))
    w[0] = u
    g = ex(hb.GradientOperator(dim).op_template(), u=u, bc=u[b])
    wave_n = hb.StrongWaveOperator(1.0, dim, flux_type="central", dirichlet_tag=TAG_NONE,
                                   neumann_tag=TAG_ALL)
    assert rel_l2(g, ex(wave_n.op_template(), w=w)[1:]) <= 1e-14
    v = np.stack([np.cos(x[:, k]) * x[:, (k + 1) % dim] for k in range(dim)])
    w = np.zeros((dim + 1, len(d)))
    w[1:] = v
    dv = ex(hb.DivergenceOperator(dim).op_template(), v=v, bc=v[:, b])
    wave_d = hb.StrongWaveOperator(1.0, dim, flux_type="central", dirichlet_tag=TAG_ALL)
    assert rel_l2(dv[0], ex(wave_d.op_template(), w=w)[0]) <= 1e-13
    # linear fields are differentiated exactly
    gx = ex(hb.GradientOperator(dim).op_template(), u=x[:, 0], bc=x[b, 0])
    assert np.abs(gx[0] - 1).max() < 1e-12 and np.abs(gx[1:]).max() < 1e-12


# --------------------------------------------------------------------------
# weak form and over-integration

def _in_out_tagger(v):
    """Boundary faces with v.n < 0 'in', the others 'out' (unit square)."""
    def tagger(fvi, el, fn, allv):
        x = allv[list(fvi)].mean(0)
        n = np.array([-1.0, 0.0]) if x[0] < -0.99 else np.array([1.0, 0.0]) if x[0] > 0.99 \
            else np.array([0.0, -1.0]) if x[1] < -0.99 else np.array([0.0, 1.0])
        return ["in"] if np.dot(n, v) < 0 else ["out"]
    return tagger


def weak_quadrature_advection(v, flux_type):
    """The weak-form advection written with over-integration: the
    stiffness acts on up-sampled u, the fluxes on face-quadrature traces."""
    u, bc = ot.Field("u"), ot.Field("bc_in")
    to_quad = ot.QuadratureGridUpsampler("quad")
    to_if = ot.QuadratureInteriorFacesGridUpsampler("quad")
    m = hb.WeakAdvectionOperator(v, inflow_tag="in", outflow_tag="out", flux_type=flux_type)
    flux_op = ot.get_flux_operator(m.flux())
    st = ot.make_stiffness_t(2)
    bc_out = to_quad(ot.BoundarizeOperator("out")(u))
    return ot.InverseMassOperator()(
        np.dot(v, st * to_quad(u))
        - (flux_op(to_if(u)) + flux_op(ot.BoundaryPair(to_if(u), to_quad(bc), "in"))
           + flux_op(ot.BoundaryPair(to_if(u), bc_out, "out"))))


@pytest.mark.parametrize("flux_type", ["upwind", "central", "lf"])
@pytest.mark.parametrize("quadrature", [False, True])
def test_weak_advection_equals_strong_kernel_model(flux_type, quadrature):
    """The weak form (nodal or over-integrated), evaluated as a tree, equals
    the oracle's strong-form advection it is lowered to."""
    v = np.array([0.7, -0.4])
    d = hb.Discretization(rect(5, tagger=_in_out_tagger(v)), order=3)
    tpl = weak_quadrature_advection(v, flux_type) if quadrature else \
        hb.WeakAdvectionOperator(v, inflow_tag="in", outflow_tag="out",
                                 flux_type=flux_type).op_template()
    desc = lower(tpl, 2, d.mesh)
    assert desc.model == MODEL_ADVECTION and np.allclose(desc.params["v"], v)
    assert desc.flux_type == ["central", "upwind", "lf"].index(flux_type)
    assert set(desc.bcs) == {("in", BC_GIVEN), ("out", 0)}
    q = _fields(d, 1, 4)
    bc = np.cos(2 * d.get_boundary("in").nodes[:, 1])
    err = _executor_vs_oracle(d, tpl, desc, {"u": q[0], "bc_in": bc}, q, bc_in=bc)
    assert err <= 1e-12, err


def test_weak_form_needs_every_boundary_face_tagged():
    """Without the mesh (or with untagged boundary faces) the weak form's
    face term on the remaining boundary faces has no kernel condition."""
    v = np.array([0.7, -0.4])
    tpl = hb.WeakAdvectionOperator(v, inflow_tag="in", outflow_tag="out").op_template()
    with pytest.raises(NotImplementedError, match="boundary"):
        lower(tpl, 2)


def test_other_quadrature_templates_are_refused():
    """A coefficient field under the quadrature stiffness goes to the
    quadrature kernel, which implements the variable-coefficient advection
    operator (advection.py:282-368) only: this template (no velocity in the
    flux, no boundary pair) is refused."""
    u, vx = ot.Field("u"), ot.Field("vx")
    to_quad = ot.QuadratureGridUpsampler("quad")
    U = fl.FluxScalarPlaceholder(0)
    flux = ot.FluxOperator(0.5 * (U.int - U.ext) * fl.make_normal(2)[0])
    tpl = ot.InverseMassOperator()(ot.StiffnessTOperator(0)(to_quad(vx) * to_quad(u))
                                   - flux(u))
    with pytest.raises(NotImplementedError):
        lower(tpl, 2)


def test_wave_dirichlet_data_lowers_to_given_condition():
    """Inhomogeneous Dirichlet data (wave.py:133-142) lowers onto the wave
    kernel with a given-data condition on the Dirichlet tag, and the bound
    RHS takes the data as dir_bc_u (the reference's field name)."""
    op = hb.StrongWaveOperator(1.0, 2, dirichlet_tag="dir", dirichlet_bc_f=1,
                               neumann_tag="neu")
    desc = lower(op.op_template(), 2)
    assert desc.model == MODEL_WAVE
    assert ("dir", BC_GIVEN) in desc.bcs and ("neu", BC_NEUMANN) in desc.bcs
    assert desc.fields["given"] == "dir_bc_u"
    # homogeneous data: the plain Dirichlet condition
    op0 = hb.StrongWaveOperator(1.0, 2, dirichlet_tag="dir", neumann_tag="neu")
    assert ("dir", BC_DIRICHLET) in lower(op0.op_template(), 2).bcs


@pytest.mark.parametrize("kind", ["field", "numbers"])
def test_maxwell_current_lowers_and_matches_oracle(kind):
    """Maxwell with a source current J (em.py:192-214: eps dE/dt = curl H - J
    + flux): the template lowers onto the Maxwell kernel with per-E-component
    sources -J/eps, and the executed template equals the oracle."""
    from oracle import OracleRHS
    from optemplate_exec import TemplateExecutor
    d = hb.Discretization(box(2), order=2)
    rng = np.random.default_rng(11)
    J = rng.standard_normal((3, len(d))) if kind == "field" else [0.5, 0.0, -1.0]
    op = hb.MaxwellOperator(2.0, 0.5, flux_type=1, current=J)
    desc = lower(op.op_template(), 3)
    assert desc.model == MODEL_MAXWELL
    outs = sorted(o for o, *_ in desc.fields["sources"])
    assert outs == ([0, 1, 2] if kind == "field" else [0, 2])
    q = _fields(d, 6, 4)
    env = {"w": q}
    if kind == "field":
        env["current"] = J
    got = TemplateExecutor(d)(op.op_template(), **env)
    ref = OracleRHS(d, op.op_template())(q)
    assert rel_l2(got, ref) <= 1e-12


@pytest.mark.parametrize("kind", ["tm", "te"])
def test_maxwell_2d_templates_lower_and_match_oracle(kind):
    """TM / TE Maxwell templates (em.py:485-515, subset cross products) lower
    onto their kernel models, not onto each other, and the executed templates
    equal the oracle with mixed walls and a source current."""
    from hedge_b200.models import MODEL_MAXWELL_TE, MODEL_MAXWELL_TM
    from oracle import OracleRHS
    from optemplate_exec import TemplateExecutor
    d = hb.Discretization(rect(5, tagger=_tagger_lr(["pmc", "abs", "pec"])), order=3)
    cls = hb.TMMaxwellOperator if kind == "tm" else hb.TEMaxwellOperator
    ne = 1 if kind == "tm" else 2
    J = np.sin(d.nodes.T[:ne])
    op = cls(0.8, 1.7, flux_type=0.6, bdry_flux_type=1, pec_tag="pec", pmc_tag="pmc",
             absorb_tag="abs", current=J)
    desc = lower(op.op_template(), 2)
    assert desc.model == (MODEL_MAXWELL_TM if kind == "tm" else MODEL_MAXWELL_TE)
    assert abs(desc.params["eps"] - 0.8) < 1e-12 and abs(desc.params["mu"] - 1.7) < 1e-12
    q = _fields(d, 3, 5)
    got = TemplateExecutor(d)(op.op_template(), w=q, current=J)
    ref = OracleRHS(d, op.op_template())(q)
    assert rel_l2(got, ref) <= 1e-12


def test_maxwell_two_tags_of_one_kind():
    """A hand-written Maxwell template with PEC walls on two tags and an
    absorbing one on a third (a combination no model constructor makes)
    lowers with each tag's kind, and the oracle on the lowered descriptor
    agrees with the executor on the tree."""
    from oracle import OracleRHS
    from optemplate_exec import TemplateExecutor

    def tagger(fvi, el, fn, allv):
        c = allv[list(fvi)].mean(0)
        return ["a"] if c[0] > 0.99 else (["b"] if c[0] < -0.99 else ["c"])
    d = hb.Discretization(box(2, tagger=tagger), order=2)
    w = ot.make_sym_vector("w", 6)
    B = ot.BoundarizeOperator
    op = hb.MaxwellOperator(1.0, 1.0, flux_type=0.5, pec_tag="a", absorb_tag="b")
    pec_c = ot.join_fields(*[-1 * (B("c") * w[k]) for k in range(3)],
                           *[B("c") * w[k] for k in range(3, 6)])
    tpl = op.op_template(w) + ot.InverseMassOperator()(
        ot.get_flux_operator(op.flux(0.5))(ot.BoundaryPair(w, pec_c, "c")))
    desc = lower(tpl, 3, d.mesh)
    assert dict(desc.bcs) == {"a": BC_PEC, "b": BC_ABSORB, "c": BC_PEC}
    q = np.random.default_rng(1).standard_normal((6, len(d)))
    ref = np.asarray(TemplateExecutor(d)(tpl, w=q), dtype=np.float64)
    assert rel_l2(OracleRHS(d, desc)(q), ref) <= 1e-12
