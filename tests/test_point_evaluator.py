"""Discretization.get_point_evaluator (hedge/discretization/__init__.py:1217-1249)
pinned directly: the nodal interpolant of a polynomial of total degree <= N
is that polynomial, so evaluating it at any point inside an element must give
the polynomial's value there to rounding.  Points are drawn inside random
elements from random barycentric coordinates (kept away from the faces, so
the containing element is unique); 2D triangles and 3D tetrahedra, orders
1-6, jittered meshes."""
import itertools

import numpy as np
import pytest

import hedge_b200 as hb

TOL = 1e-12


def _poly(dim, order, rng):
    """A random polynomial of total degree <= order: (exponents, coefficients)."""
    exps = [e for e in itertools.product(range(order + 1), repeat=dim) if sum(e) <= order]
    return np.array(exps), rng.uniform(-1, 1, len(exps))


def _eval(exps, coef, x):
    x = np.atleast_2d(x)
    return (coef[None, :] * np.prod(x[:, None, :] ** exps[None, :, :], axis=2)).sum(1)


def _points(mesh, dim, n, rng):
    """n points inside random elements (barycentric coordinates >= 0.05)."""
    els = rng.integers(0, len(mesh.elements), n)
    pts = []
    for el in els:
        lam = rng.uniform(0.05, 1.0, dim + 1)
        lam /= lam.sum()
        lam = 0.05 + (1 - 0.05 * (dim + 1)) * lam
        verts = mesh.points[mesh.elements[el]]
        pts.append(lam @ verts)
    return els, np.array(pts)


@pytest.mark.parametrize("order", [1, 2, 4, 6])
def test_point_evaluator_exact_on_polynomials_2d(order):
    rng = np.random.default_rng(10 + order)
    mesh = hb.make_regular_rect_mesh((-1, -1), (1, 1), (7, 7), jitter=0.03, seed=2)
    d = hb.Discretization(mesh, order=order)
    exps, coef = _poly(2, order, rng)
    u = _eval(exps, coef, d.nodes)
    els, pts = _points(mesh, 2, 16, rng)
    for el, p in zip(els, pts):
        ev = d.get_point_evaluator(p)
        assert ev.el == el
        want = _eval(exps, coef, p)[0]
        assert abs(ev(u) - want) <= TOL * max(1.0, np.abs(u).max())


@pytest.mark.parametrize("order", [1, 3, 5])
def test_point_evaluator_exact_on_polynomials_3d(order):
    rng = np.random.default_rng(20 + order)
    mesh = hb.make_box_tet_mesh(n=(3, 3, 3), jitter=0.03, seed=3)
    d = hb.Discretization(mesh, order=order)
    exps, coef = _poly(3, order, rng)
    u = _eval(exps, coef, d.nodes)
    els, pts = _points(mesh, 3, 16, rng)
    for el, p in zip(els, pts):
        ev = d.get_point_evaluator(p)
        assert ev.el == el
        want = _eval(exps, coef, p)[0]
        assert abs(ev(u) - want) <= TOL * max(1.0, np.abs(u).max())


def test_point_evaluator_at_nodes_and_on_several_fields():
    """At a node the evaluator returns the nodal value itself; a [F, K*Np]
    field array gives F values (torch tensors likewise)."""
    import torch
    rng = np.random.default_rng(3)
    d = hb.Discretization(hb.make_regular_rect_mesh((-1, -1), (1, 1), (5, 5), jitter=0.02,
                                                    seed=4), order=3)
    w = rng.standard_normal((3, len(d)))
    el = 7
    # an interior node of element 7 (order 3 triangle: node 4 is the centroid node)
    ld = d.ldis
    interior = [i for i in range(d.Np) if np.all(ld.unit_nodes[i] > -1 + 1e-9)
                and ld.unit_nodes[i].sum() < -(d.dimensions - 2) - 1e-9]
    i = interior[0]
    ev = d.get_point_evaluator(d.nodes[el * d.Np + i])
    assert ev.el == el
    got = ev(w)
    assert got.shape == (3,)
    assert np.abs(got - w[:, el * d.Np + i]).max() <= 1e-13
    gt = ev(torch.as_tensor(w))
    assert torch.allclose(gt, torch.as_tensor(got), rtol=0, atol=1e-15)


def test_point_evaluator_outside_mesh_raises():
    d = hb.Discretization(hb.make_regular_rect_mesh((-1, -1), (1, 1), (4, 4)), order=2)
    with pytest.raises(RuntimeError):
        d.get_point_evaluator(np.array([3.0, 0.0]))
