"""Mesh construction (CPU): rejected inputs, and the geometry of single
elements in both vertex orientations (outward unit normals, closed surface,
volume from the Jacobian)."""
import numpy as np
import pytest

import hedge_b200 as hb
from hedge_b200.mesh import MeshError

TRI = np.array([[0.1, -0.2], [1.3, 0.1], [0.2, 0.9]])
TET = np.array([[0.0, 0.1, -0.1], [1.2, 0.0, 0.1], [0.1, 0.9, 0.0], [0.2, 0.1, 1.1]])


@pytest.mark.parametrize("points,elements", [
    (np.zeros((0, 2)), np.zeros((0, 3), dtype=int)),          # no elements
    (TRI, np.array([[0, 1]])),                                # too few vertices
    (np.zeros((3, 4)), np.array([[0, 1, 2]])),                # 4D points
    (np.array([[0., 0], [1, 1], [2, 2]]), np.array([[0, 1, 2]])),   # zero area
])
def test_invalid_mesh_rejected(points, elements):
    with pytest.raises(MeshError):
        hb.Mesh(points, elements)


@pytest.mark.parametrize("flip", [False, True])
@pytest.mark.parametrize("dim", [2, 3])
def test_single_element_geometry(dim, flip):
    pts = TRI if dim == 2 else TET
    el = np.arange(dim + 1)
    if flip:
        el = el[[0, 2, 1] + ([3] if dim == 3 else [])]
    m = hb.Mesh(pts, el[None, :])
    assert len(m.interfaces) == 0
    n = m.face_normals[0]
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-14)
    # closed surface: the area-weighted outward normals cancel
    area = 2.0 * m.face_jacobians[0]     # the reference faces have measure 2
    assert np.allclose((area[:, None] * n).sum(0), 0.0, atol=1e-13)
    # each normal points away from the centroid
    c = pts.mean(0)
    fv = m.element_faces()[0]
    for f in range(dim + 1):
        assert np.dot(pts[fv[f]].mean(0) - c, n[f]) > 0
    vol = abs(np.linalg.det(np.stack([pts[i] - pts[0] for i in range(1, dim + 1)])))
    vol /= 2.0 if dim == 2 else 6.0
    ref_vol = 2.0 if dim == 2 else 4.0 / 3.0     # the reference simplex
    assert np.isclose(abs(m.jacobians[0]) * ref_vol, vol, rtol=1e-13)


def test_bind_checks_coverage_compile_does_not():
    """The models' bind checks boundary coverage (Maxwell: the PEC,
    absorbing and incident tags only, em.py:373-377; hedge/mesh/__init__.py
    check_bc_coverage); Discretization.compile does not, so a PMC-walled
    mesh compiles directly (its face table is built without a check)."""
    from hedge_b200.discretization import build_face_table
    def tagger(fvi, el, fn, allv):
        return ["pmc"] if allv[list(fvi)].mean(0)[0] < -0.99 else ["pec"]
    m = hb.make_regular_rect_mesh((-1, -1), (1, 1), (4, 4), boundary_tagger=tagger)
    d = hb.Discretization(m, order=2)
    op = hb.TMMaxwellOperator(1.0, 1.0, flux_type=1, pec_tag="pec", pmc_tag="pmc")
    with pytest.raises(MeshError):
        op.bind(d)
    conn = build_face_table(d, op.op_template())[0]
    assert conn.shape == (d.K, d.dimensions + 1, 2)
