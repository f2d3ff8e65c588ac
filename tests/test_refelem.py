"""Reference-element known-answer tests, restated from the reference's
test/test_basics.py and test/test_jit_discretization.py."""
import math

import numpy as np
import pytest

from hedge_b200.refelem import (TriangleElement, TetrahedronElement, WarpFactor,
                                tuples_summing_to_at_most, triangle_basis, tet_basis)
from hedge_b200.mesh import Mesh


def monomial(exps, x, factor=1.0):
    y = (x + 1) / 2
    return factor * np.prod([y[:, i] ** a for i, a in enumerate(exps)], axis=0)


def simplex_integral(exps):
    return (2 ** len(exps) * np.prod([math.factorial(a) for a in exps])
            / math.factorial(len(exps) + sum(exps)))


@pytest.mark.parametrize("el", [TriangleElement(3), TetrahedronElement(5)])
def test_simp_mass_and_diff_matrices_by_monomial(el):
    """test_jit_discretization.py:239-277, threshold 1e-13."""
    un = el.unit_nodes
    for comb in tuples_summing_to_at_most(el.order, el.dimensions):
        f = monomial(comb, un)
        assert abs(np.ones(len(un)) @ el.mass_matrix @ f - simplex_integral(comb)) < 1e-13
        for i in range(el.dimensions):
            e = list(comb)
            if e[i] == 0:
                df = np.zeros(len(un))
            else:
                fac = e[i]
                e[i] -= 1
                df = monomial(e, un, fac)
            assert np.abs(df / 2 - el.differentiation_matrices[i] @ f).max() < 1e-13


def test_tri_nodes_against_known_values():
    """test_basics.py:564-628: warped triangle nodes at N=8 vs the explicit
    (older) construction, 3e-15; node tuple set."""
    tri = TriangleElement(8)
    alpha = tri.alpha_opt[7]
    warp = WarpFactor(8)
    e1 = np.array([1.0, 0.0])
    e2 = np.array([math.cos(2 * math.pi / 3), math.sin(2 * math.pi / 3)])
    e3 = np.array([math.cos(4 * math.pi / 3), math.sin(4 * math.pi / 3)])
    for n1, (l1, l2, l3) in zip(tri.equilateral_nodes(), tri.equidistant_barycentric_nodes()):
        p = tri.barycentric_to_equilateral((l1, l2, l3))
        w1 = 4 * l1 * l2 * warp(l2 - l1) * (1 + (alpha * l3) ** 2)
        w2 = 4 * l3 * l2 * warp(l3 - l2) * (1 + (alpha * l1) ** 2)
        w3 = 4 * l3 * l1 * warp(l1 - l3) * (1 + (alpha * l2) ** 2)
        assert np.linalg.norm(n1 - (p + w1 * e1 + w2 * e2 + w3 * e3)) < 3e-15
    assert set(tri.node_tuples) == {(m, n) for n in range(9) for m in range(9 - n)}


@pytest.mark.parametrize("el", [TriangleElement(1), TriangleElement(2), TriangleElement(3),
                                TetrahedronElement(1), TetrahedronElement(2),
                                TetrahedronElement(3)])
def test_simp_orthogonality(el):
    """test_basics.py:30-60: basis orthonormality.  The reference integrates
    with Grundmann-Moeller cubature; here a collapsed Gauss-Jacobi rule of
    the same exactness is used."""
    from numpy.polynomial.legendre import leggauss
    q = el.order * 2 + 2
    x, w = leggauss(q)
    if el.dimensions == 2:
        a, b = np.meshgrid(x, x, indexing="ij")
        wa, wb = np.meshgrid(w, w, indexing="ij")
        r = (1 + a) * (1 - b) / 2 - 1
        s = b
        pts = np.stack([r.ravel(), s.ravel()], 1)
        wt = (wa * wb * (1 - b) / 2).ravel()
        basis = [triangle_basis(i, j, pts) for i, j in el.mode_ids()]
    else:
        a, b, c = np.meshgrid(x, x, x, indexing="ij")
        wa, wb, wc = np.meshgrid(w, w, w, indexing="ij")
        r = (1 + a) * (1 - b) * (1 - c) / 4 - 1
        s = (1 + b) * (1 - c) / 2 - 1
        t = c
        pts = np.stack([r.ravel(), s.ravel(), t.ravel()], 1)
        wt = (wa * wb * wc * (1 - b) * (1 - c) ** 2 / 8).ravel()
        basis = [tet_basis(i, j, k, pts) for i, j, k in el.mode_ids()]
    B = np.stack(basis)
    G = (B * wt) @ B.T
    assert np.abs(G - np.eye(len(basis))).max() < 1e-13


@pytest.mark.parametrize("dim,order", [(2, 4), (3, 1), (3, 4)])
def test_simp_face_normals_and_jacobians(dim, order):
    """test_basics.py:704-779: unit normals orthogonal to the face, pointing
    away from the opposite vertex, face Jacobians against the face area."""
    rng = np.random.default_rng(3)
    el = TriangleElement(order) if dim == 2 else TetrahedronElement(order)
    for _ in range(50):
        verts = rng.standard_normal((dim + 1, dim))
        m = Mesh(verts, np.arange(dim + 1)[None])
        nodes = (m.map_a[0] @ el.unit_nodes.T).T + m.map_b[0]
        fv = [(0, 1), (1, 2), (0, 2)] if dim == 2 else \
            [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)]
        for f, fvi in enumerate(fv):
            normal, jac = m.face_normals[0, f], m.face_jacobians[0, f]
            corners = verts[list(fvi)]
            close = sum(np.linalg.norm(nodes[i] - c) < 1e-13
                        for i in el.face_indices[f] for c in corners)
            assert close == len(corners)
            if dim == 2:
                true_jac = np.linalg.norm(corners[1] - corners[0]) / 2
            else:
                true_jac = np.linalg.norm(np.cross(corners[1] - corners[0],
                                                   corners[2] - corners[0])) / 4
            assert abs(true_jac - jac) / true_jac < 1e-13
            assert abs(np.linalg.norm(normal) - 1) < 1e-13
            for c in corners[1:]:
                assert abs(normal @ (c - corners[0])) < 1e-13
            opp = verts[list(set(range(dim + 1)) - set(fvi))[0]]
            for c in corners:
                assert (opp - c) @ normal < 0


def test_tri_map_jacobian_and_mass_matrix():
    """test_basics.py:806-827."""
    for i in range(1, 10):
        el = TriangleElement(i)
        ones = np.ones(el.node_count())
        assert abs(ones @ el.mass_matrix @ ones - 2) < 1e-14
    rng = np.random.default_rng(1)
    for _ in range(10):
        v = rng.standard_normal((3, 2))
        m = Mesh(v, np.array([[0, 1, 2]]))
        area = abs(np.linalg.det(np.stack([v[1] - v[0], v[2] - v[0]], 1)) / 2)
        assert abs(area - abs(2 * m.jacobians[0])) / area < 5e-15


def test_face_vertex_order_and_counts():
    """Face index lists / vertex conventions (local.py:300-323, 838-953)."""
    tri = TriangleElement(4)
    assert tri.node_count() == 15 and tri.face_node_count() == 5
    tet = TetrahedronElement(4)
    assert tet.node_count() == 35 and tet.face_node_count() == 15
    tet7 = TetrahedronElement(7)
    assert tet7.node_count() == 120 and tet7.face_node_count() == 36
    # face f of a triangle: AB, BC, AC
    un = tri.unit_nodes
    assert np.allclose(un[list(tri.face_indices[0])][:, 1], -1)
    assert np.allclose(un[list(tri.face_indices[2])][:, 0], -1)
    assert np.allclose(un[list(tri.face_indices[1])].sum(1), 0)


def test_lift_is_minv_times_face_mass():
    for el in (TriangleElement(4), TetrahedronElement(4)):
        L = el.lifting_matrix
        assert np.allclose(el.mass_matrix @ L, el.multi_face_mass_matrix, atol=1e-12)
