"""Quadrature (over-integration), CPU: the rules, their known answers, the
element quadrature matrices and the variable-coefficient advection
template.

* the rules restate hedge/quadrature.py (Gauss-Legendre by Golub-Welsch,
  Grundmann-Moeller on simplices): exact to their degree on monomials,
  weights summing to the simplex volume, the package's and the oracle's
  independent restatements equal point for point;
* the reference's known answer (test/test_jit_discretization.py:90-131):
  the quadrature mass of f^2, f = x^2 y, on a square is 4/15 to 1e-14 while
  the nodal mass misses by more than 1e-8;
* the quadrature matrices the kernel applies, run through a host restatement
  of the kernel's algorithm, equal the template executor (which integrates
  the tree with the reference's rules) for every flux type, with and
  without inflow data, in 2D and 3D, and with the nodal fallback when the
  discretization has no degree for the tag;
* the variable-coefficient advection template lowers onto the quadrature
  kernel; altered templates do not.
"""
import itertools
from math import factorial

import numpy as np
import pytest

import hedge_b200 as hb
from hedge_b200 import optemplate as ot
from hedge_b200.discretization import build_face_table
from hedge_b200.lowering import lower
from hedge_b200.models import BC_DIRICHLET, BC_GIVEN, MODEL_VARADV
from hedge_b200.quadrature import (collapsed_gauss, get_simplex_cubature,
                                   grundmann_moeller, legendre_gauss)

from conftest import rel_l2
from test_optemplate import box, rect


def _monomial_error(x, w, deg):
    """Largest relative error on prod (1 + x_i)^a_i, |a| <= deg, over the
    biunit simplex: exact integral 2^(|a|+n) prod a_i! / (|a|+n)!."""
    n = x.shape[1]
    worst = 0.0
    for a in itertools.product(range(deg + 1), repeat=n):
        if sum(a) > deg:
            continue
        exact = 2 ** (sum(a) + n) * np.prod([factorial(k) for k in a]) / factorial(sum(a) + n)
        num = float(np.sum(w * np.prod((1 + x) ** np.array(a), axis=1)))
        worst = max(worst, abs(num - exact) / exact)
    return worst


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("degree", [1, 4, 9, 12, 15])
def test_reference_rule_is_exact_to_its_degree(dim, degree):
    x, w = get_simplex_cubature(degree, dim)
    assert abs(w.sum() - 2 ** dim / factorial(dim)) <= 1e-13
    assert _monomial_error(x, w, degree) <= 1e-12
    s = int(np.ceil((degree - 1) / 2))
    if dim == 1:
        assert len(w) == s + 1
    elif s >= 1:
        assert (w < 0).any()      # Grundmann-Moeller has negative weights


def test_gauss_legendre_matches_numpy():
    for n in range(0, 12):
        x, w = legendre_gauss(n)
        xr, wr = np.polynomial.legendre.leggauss(n + 1)
        assert np.abs(x - xr).max() <= 1e-14 and np.abs(w - wr).max() <= 1e-14


@pytest.mark.parametrize("dim", [2, 3])
def test_collapsed_rule_is_exact(dim):
    for n in (2, 5, 7):
        x, w = collapsed_gauss(dim, n)
        assert _monomial_error(x, w, 2 * n - 1) <= 1e-12


def test_grundmann_moeller_point_counts():
    """Distinct points: 79 at s = 6 in 2D (84 generated, the centroid
    and other coincident points merged), 209 at s = 6 in 3D."""
    assert len(grundmann_moeller(6, 2)[1]) == 79
    assert len(grundmann_moeller(6, 3)[1]) == 209
    assert len(grundmann_moeller(0, 2)[1]) == 1


def test_oracle_and_package_rules_agree():
    from optemplate_exec import reference_cubature
    for dim in (1, 2, 3):
        for deg in range(1, 16):
            a, b = reference_cubature(deg, dim), get_simplex_cubature(deg, dim)
            ia, ib = np.lexsort(a[0].T[::-1]), np.lexsort(b[0].T[::-1])
            assert a[0].shape == b[0].shape
            assert np.abs(a[0][ia] - b[0][ib]).max() <= 1e-13
            assert np.abs(a[1][ia] - b[1][ib]).max() <= 1e-12


def test_quadrature_mass_of_monomial_square_kat():
    """test_jit_discretization.py:90-131: on a square of a few triangles at
    order 4 and quad degree 12, the quadrature mass of (x^2 y)^2 integrates
    to 4/15 (error < 1e-14); the nodal mass does not (error > 1e-8)."""
    mesh = hb.make_regular_rect_mesh((-1, -1), (1, 1), (2, 2))
    d = hb.Discretization(mesh, order=4, quad_min_degrees={"quad": 12})
    q = d.get_quadrature_info("quad")
    f = d.nodes[:, 0] ** 2 * d.nodes[:, 1]
    F = f.reshape(d.K, d.Np)
    absj = np.abs(mesh.jacobians)
    quad = float(np.sum(absj[:, None] * q.volume_weights[None, :] * (F @ q.vol_interp.T) ** 2))
    nodal = float(np.sum(absj[:, None] * ((F * F) @ d.ldis.mass_matrix.T)))
    exact = 4 / 15
    assert abs(quad - exact) < 1e-14
    assert abs(nodal - exact) > 1e-8


# ---------------------------------------------------------------------------
# the kernel's algorithm on the host, from the matrices the product ships

def emulate_kernel(d, desc, u, v, bc=None):
    """rhs of the quadrature kernel (hedge_b200/csrc/rhs_quad.cu) restated
    with numpy: the same matrices, face table and gather."""
    from hedge_b200.discretization import quadrature_descriptor
    _, (vi, vp, fi, fl) = quadrature_descriptor(d, desc)
    conn, n_given, _ = build_face_table(d, desc)
    K, Np, Nfp, Nf, dim = d.K, d.Np, d.Nfp, d.Nfaces, d.dimensions
    geo = d.geometry
    imd = geo[:, :dim * dim].reshape(K, dim, dim)
    U = u.reshape(K, Np)
    V = v.reshape(dim, K, Np)
    uq, vq = U @ vi.T, V @ vi.T
    g = uq[None] * np.einsum("krx,xkq->rkq", imd, vq)
    rhs = np.einsum("riq,rkq->ki", vp, g)
    cmax = np.max(np.sum(V ** 2, axis=0), axis=1)
    fmask, sh = d.fmask, d.ldis.face_shuffle_table
    nqf = fi.shape[1]
    for e in range(K):
        for f in range(Nf):
            nbr, code = conn[e, f]
            own = np.concatenate([U[e][None], V[:, e]])[:, fmask[f]]      # [1+d, Nfp]
            if nbr >= 0:
                nn = fmask[code & 3][sh[code >> 2]]
                oth = np.concatenate([U[nbr][None], V[:, nbr]])[:, nn]
                cp = cmax[nbr]
            else:
                if code == 0:
                    continue
                oth = own.copy()
                oth[0] = bc[(-1 - nbr) * Nfp:(-nbr) * Nfp] if code == BC_GIVEN else 0.0
                cp = cmax[e]
            wm, wp = own @ fi[f].T, oth @ fi[f].T                          # [1+d, Qf]
            n = geo[e, dim * dim + f * (dim + 1): dim * dim + f * (dim + 1) + dim]
            fs = geo[e, dim * dim + f * (dim + 1) + dim]
            nvm, nvp = n @ wm[1:], n @ wp[1:]
            if desc.flux_type == 0:
                flux = 0.5 * (wm[0] * nvm + wp[0] * nvp)
            elif desc.flux_type == 2:
                flux = 0.5 * (nvm * wm[0] + nvp * wp[0]) - 0.5 * (wp[0] - wm[0]) * max(cmax[e], cp)
            else:
                navg = n @ (0.5 * (wm[1:] + wp[1:]))
                flux = np.where(navg > 0, nvm * wm[0], nvp * wp[0])
            rhs[e] -= fl[:, f * nqf:(f + 1) * nqf] @ (fs * flux)
    return rhs.reshape(-1)


def velocity(d, kind="vortex"):
    x = d.nodes
    if d.dimensions == 2:
        return np.stack([-x[:, 1] + 0.3, x[:, 0] + 0.2 * np.sin(2 * x[:, 1])])
    return np.stack([-x[:, 1] + 0.2, x[:, 0] + 0.1 * x[:, 2], 0.3 + 0.2 * np.cos(x[:, 0])])


def state(d, seed=0):
    rng = np.random.default_rng(seed)
    x = d.nodes
    return np.exp(-4 * np.sum((x - 0.2) ** 2, axis=1)) + 0.05 * rng.uniform(-1, 1, len(d))


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("flux_type", ["central", "upwind", "lf"])
@pytest.mark.parametrize("with_bc", [False, True])
def test_kernel_algorithm_equals_executor(dim, flux_type, with_bc):
    from optemplate_exec import TemplateExecutor
    N = 3 if dim == 2 else 2
    mesh = rect(4) if dim == 2 else box(2)
    d = hb.Discretization(mesh, order=N, quad_min_degrees={"quad": 3 * N})
    op = hb.VariableCoefficientAdvectionOperator(
        dim, None, bc_u_f=1 if with_bc else "None", flux_type=flux_type)
    tpl = op.op_template()
    desc = lower(tpl, dim)
    assert desc.model == MODEL_VARADV
    u, v = state(d), velocity(d)
    env = {"u": u, "v": v}
    bc = None
    if with_bc:
        bc = np.sin(3 * d.get_boundary(hb.TAG_ALL).nodes[:, 0])
        env["bc_u"] = bc
    ref = TemplateExecutor(d)(tpl, **env)[0]
    got = emulate_kernel(d, desc, u, v, bc)
    assert rel_l2(got, ref) <= 1e-12


def test_nodal_fallback_equals_executor_without_samplers():
    """No degree for the tag: the reference evaluates the template with the
    up-samplers removed (mappers/__init__.py:937-958); so do the kernel's
    matrices."""
    from optemplate_exec import TemplateExecutor
    from hedge_b200.lowering import _strip_samplers
    d = hb.Discretization(rect(4), order=3)
    op = hb.VariableCoefficientAdvectionOperator(2, None, bc_u_f=1, flux_type="lf")
    tpl = op.op_template()
    desc = lower(tpl, 2)
    u, v = state(d), velocity(d)
    bc = np.cos(2 * d.get_boundary(hb.TAG_ALL).nodes[:, 1])
    ref = TemplateExecutor(d)(_strip_samplers(tpl), u=u, v=v, bc_u=bc)[0]
    with pytest.warns(UserWarning, match="nodal evaluation"):
        got = emulate_kernel(d, desc, u, v, bc)
    assert rel_l2(got, ref) <= 1e-12


def test_exact_volume_rule_is_used_only_when_exact():
    """The volume matrices come from the collapsed rule (fewer points) only
    when the requested degree integrates v u d(phi)/dx exactly."""
    d = hb.Discretization(rect(2), order=4, quad_min_degrees={"quad": 12})
    vi = d.quadrature_matrices("quad", 11)[0]
    assert vi.shape[0] == 36          # collapsed, 6 x 6, instead of 79
    d2 = hb.Discretization(rect(2), order=4, quad_min_degrees={"quad": 8})
    vi2 = d2.quadrature_matrices("quad", 11)[0]
    assert vi2.shape[0] == len(get_simplex_cubature(8, 2)[1])


# ---------------------------------------------------------------------------
# lowering

@pytest.mark.parametrize("dim", [2, 3])
def test_var_advection_lowers_to_quadrature_kernel(dim):
    for ft in ("central", "upwind", "lf"):
        for bc in ("None", 1):
            m = hb.VariableCoefficientAdvectionOperator(dim, None, bc_u_f=bc, flux_type=ft)
            desc = lower(m.op_template(), dim)
            assert desc.model == MODEL_VARADV and desc.n_fields == 1
            assert desc.flux_type == ["central", "upwind", "lf"].index(ft)
            assert desc.bcs == [(hb.TAG_ALL, BC_GIVEN if bc == 1 else BC_DIRICHLET)]
            assert desc.fields == {"state": "u", "coeff": "v",
                                   "given": "bc_u" if bc == 1 else None}


def test_var_advection_with_other_names_and_tag():
    """Other field names and another quadrature tag lower too, with the
    names and the tag recorded."""
    m = hb.VariableCoefficientAdvectionOperator(2, None, bc_u_f=1, flux_type="upwind")
    tpl = m.op_template(u=ot.Field("phi"), v=ot.make_sym_vector("vel", 2),
                        bc_u=ot.Field("inflow"))
    from hedge_b200.lowering import _retag
    from hedge_b200.lowering import _rebuild
    tpl = _rebuild(tpl, lambda n: _retag(n, "fine"))
    desc = lower(tpl, 2)
    assert desc.fields == {"state": "phi", "coeff": "vel", "given": "inflow"}
    assert desc.params["quad_tag"] == "fine"


def _altered(kind):
    """The 2D central template with one part changed."""
    from hedge_b200 import flux as fl
    d = 2
    u, v = ot.Field("u"), ot.make_sym_vector("v", d)
    to_quad = ot.QuadratureGridUpsampler("quad")
    to_if = ot.QuadratureInteriorFacesGridUpsampler("quad")
    c = ot.ElementwiseMaxOperator()(ot.ptwise_dot(1, 1, v, v))
    if kind == "no_elmax":
        c = ot.ptwise_dot(1, 1, v, v)
    w = ot.join_fields(u, v, c)
    qw = to_if(w)
    bc_w = ot.join_fields(0, to_quad(ot.BoundarizeOperator(hb.TAG_ALL)(v)),
                          to_quad(ot.BoundarizeOperator(hb.TAG_ALL)(c)))
    W = fl.FluxVectorPlaceholder(d + 2)
    n = fl.make_normal(d)
    scale = 0.6 if kind == "flux_scale" else 0.5
    flux = (W[0].int * np.dot(W[1:3].int, n) + W[0].ext * np.dot(W[1:3].ext, n)) * scale
    if kind == "lf_with_norm":
        flux = 0.5 * (np.dot(n, W[1:3].int) * W[0].int + np.dot(n, W[1:3].ext) * W[0].ext) \
            - 0.5 * (W[0].ext - W[0].int) * fl.flux_max(W[3].int, W[3].ext) * 2
    fo = ot.get_flux_operator(flux)
    vol_v = to_quad(v) * to_quad(u)
    if kind == "vol_sign":
        vol_v = -1 * vol_v
    st = ot.make_stiffness_t(d)
    return ot.InverseMassOperator()(np.dot(st, vol_v) - (fo(qw) + fo(ot.BoundaryPair(
        qw, bc_w, hb.TAG_ALL))))


def test_central_template_by_hand_lowers():
    desc = lower(_altered("none"), 2)
    assert desc.model == MODEL_VARADV and desc.flux_type == 0


@pytest.mark.parametrize("kind", ["flux_scale", "vol_sign", "lf_with_norm"])
def test_altered_templates_are_refused(kind):
    with pytest.raises(NotImplementedError):
        lower(_altered(kind), 2)


def test_central_without_element_max_still_lowers():
    """c does not enter the central flux, so a template that builds c
    without the element maximum is the same operator."""
    assert lower(_altered("no_elmax"), 2).model == MODEL_VARADV


def test_diffusion_is_refused():
    with pytest.raises(NotImplementedError):
        hb.VariableCoefficientAdvectionOperator(2, None, diffusion_coeff=0.1)
