"""Conformal simplicial meshes: geometry, connectivity, boundary tags.

Host-side FP64 set-up, vectorised with numpy.  Restates:

* the simplex unit-to-global affine map A r + b with
  A[:, i] = (v_{i+1} - v_0)/2, b = sum_{i>=1} v_i / 2 - (d-2) v_0 / 2
  (hedge src/wrapper/wrap_base.cpp:61-76);
* triangle face normals / face Jacobians (hedge/mesh/element.py:167-187) and
  tetrahedron ones (src/wrapper/wrap_mesh.cpp:40-82, face signs -1,1,-1,1);
* conformal face matching, boundary tagging and periodic pairing
  (hedge/mesh/__init__.py:186-405);
* the 2D regular rectangle generator with its (a,b,c),(d,c,b) split
  (hedge/mesh/generator.py:132-205).

The 3D structured box generator (6 tetrahedra per cube) is new: the
reference's box generator needs the tetgen mesher, which is not part of the
hot path.  Seeded vertex jitter moves interior vertices only.
"""

from __future__ import annotations

import numpy as np


class TAG_NONE:
    """Boundary tag of an empty boundary."""


class TAG_ALL:
    """Boundary tag of the entire (non-periodic) boundary."""


class MeshError(ValueError):
    pass


TRI_FACES = np.array([[0, 1], [1, 2], [0, 2]], dtype=np.int64)
TET_FACES = np.array([[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]], dtype=np.int64)
TET_FACE_SIGNS = np.array([-1.0, 1.0, -1.0, 1.0])


def face_vertex_table(dim):
    return TRI_FACES if dim == 2 else TET_FACES


class Mesh:
    """A conformal simplicial mesh.

    Attributes
    ----------
    points : [Nv, d] float64
    elements : [K, d+1] int64 vertex indices (reference vertex order A,B,C(,D))
    map_a, map_b : unit-to-global affine map per element
    inv_map_a : [K, d, d] inverse map matrix (rows: r,s,t; cols: x,y,z)
    jacobians : [K] signed det(A)
    face_normals : [K, Nf, d], face_jacobians : [K, Nf]
    interfaces : [n_if, 4] int64 rows (el_l, face_l, el_n, face_n)
    tag_to_boundary : dict tag -> [n, 2] int64 rows (el, face)
    periodic_opposite_faces : dict face-vertex tuple -> (opposite tuple, axis)
    """

    def __init__(self, points, elements, boundary_tagger=None,
                 periodicity=None):
        points = np.ascontiguousarray(points, dtype=np.float64)
        elements = np.ascontiguousarray(elements, dtype=np.int64)
        if points.ndim != 2 or points.shape[1] not in (2, 3):
            raise MeshError("points must be [Nv, 2] or [Nv, 3]")
        d = points.shape[1]
        if elements.ndim != 2 or elements.shape[1] != d + 1:
            raise MeshError("elements must be [K, d+1]")
        if len(elements) == 0:
            raise MeshError("mesh contains no elements")
        self.points = points
        self.elements = elements
        self.dimensions = d
        self._build_geometry()
        self._build_connectivity(boundary_tagger, periodicity)

    # geometry ---------------------------------------------------------------
    def _build_geometry(self):
        d = self.dimensions
        v = self.points[self.elements]                     # [K, d+1, d]
        a = 0.5 * (v[:, 1:, :] - v[:, :1, :]).transpose(0, 2, 1)   # [K, d, d]
        b = 0.5 * v[:, 1:, :].sum(axis=1) - 0.5 * (d - 2) * v[:, 0, :]
        self.map_a = np.ascontiguousarray(a)
        self.map_b = np.ascontiguousarray(b)
        self.jacobians = np.linalg.det(a)
        if np.any(self.jacobians == 0):
            raise MeshError("degenerate element")
        self.inv_map_a = np.linalg.inv(a)
        orient = np.sign(self.jacobians)
        if d == 2:
            m = a
            face1 = m[:, :, 1] - m[:, :, 0]
            raw = np.stack([
                np.stack([m[:, 1, 0], -m[:, 0, 0]], axis=-1),
                np.stack([face1[:, 1], -face1[:, 0]], axis=-1),
                np.stack([-m[:, 1, 1], m[:, 0, 1]], axis=-1)], axis=1)
            raw = raw * orient[:, None, None]
            lens = np.linalg.norm(raw, axis=-1)
            self.face_normals = raw / lens[..., None]
            self.face_jacobians = lens
        else:
            fv = v[:, TET_FACES, :]                          # [K, 4, 3, 3]
            n = np.cross(fv[:, :, 1] - fv[:, :, 0], fv[:, :, 2] - fv[:, :, 0])
            nlen = np.linalg.norm(n, axis=-1)
            scale = orient[:, None] * TET_FACE_SIGNS[None, :] / nlen
            self.face_normals = n * scale[..., None]
            self.face_jacobians = nlen / 4

    @property
    def face_count(self):
        return self.dimensions + 1

    def element_faces(self):
        """[K, Nf, d] face vertex tuples in each element's face order."""
        return self.elements[:, face_vertex_table(self.dimensions)]

    # connectivity ----------------------------------------------------------
    def _build_connectivity(self, boundary_tagger, periodicity):
        d = self.dimensions
        K = len(self.elements)
        nf = d + 1
        faces = self.element_faces().reshape(K * nf, d)
        keys = np.sort(faces, axis=1)
        order = np.lexsort(keys.T[::-1])
        sk = keys[order]
        same_next = np.all(sk[1:] == sk[:-1], axis=1)
        if np.any(same_next[1:] & same_next[:-1]):
            raise MeshError("face can at most border two elements")
        first = np.nonzero(same_next)[0]
        pair_a, pair_b = order[first], order[first + 1]
        paired = np.zeros(K * nf, dtype=bool)
        paired[pair_a] = True
        paired[pair_b] = True
        interfaces = [np.stack([pair_a // nf, pair_a % nf,
                                pair_b // nf, pair_b % nf], axis=1)]
        bdry = np.nonzero(~paired)[0]
        bdry_ef = np.stack([bdry // nf, bdry % nf], axis=1)

        tag_to_boundary: dict = {TAG_NONE: [], TAG_ALL: []}
        bdry_tags = []
        for el, fn in bdry_ef:
            fvi = tuple(int(x) for x in faces[el * nf + fn])
            tags = list(boundary_tagger(fvi, int(el), int(fn), self.points)) \
                if boundary_tagger is not None else []
            bdry_tags.append(tags)
            for t in tags:
                tag_to_boundary.setdefault(t, []).append((int(el), int(fn)))
            tag_to_boundary[TAG_ALL].append((int(el), int(fn)))

        self.periodicity = list(periodicity) if periodicity else [None] * d
        if len(self.periodicity) != d:
            raise MeshError("periodicity needs one entry per axis")
        self.periodic_opposite_faces = {}
        key_to_ef = {tuple(k): (int(i) // nf, int(i) % nf)
                     for k, i in zip(keys[bdry], bdry)}
        for axis, per in enumerate(self.periodicity):
            if per is None:
                continue
            minus_tag, plus_tag = per
            minus_faces = tag_to_boundary.get(minus_tag, [])
            plus_faces = tag_to_boundary.get(plus_tag, [])
            mv = sorted({int(x) for el, fn in minus_faces
                         for x in faces[el * nf + fn]})
            pv = sorted({int(x) for el, fn in plus_faces
                         for x in faces[el * nf + fn]})
            mp, pp = self.points[mv].copy(), self.points[pv].copy()
            mp[:, axis] = 0
            pp[:, axis] = 0
            dist = np.linalg.norm(mp[:, None, :] - pp[None, :, :], axis=-1)
            j = np.argmin(dist, axis=1)
            ok = dist[np.arange(len(mv)), j] < 1e-12
            minus_to_plus = {mv[i]: pv[j[i]] for i in range(len(mv)) if ok[i]}
            plus_to_minus = {b: a for a, b in minus_to_plus.items()}
            new_if = []
            for el, fn in minus_faces:
                m_fvi = tuple(int(x) for x in faces[el * nf + fn])
                mapped = tuple(minus_to_plus[i] for i in m_fvi)
                pel, pfn = key_to_ef[tuple(sorted(mapped))]
                new_if.append((el, fn, pel, pfn))
                p_fvi = tuple(int(x) for x in faces[pel * nf + pfn])
                self.periodic_opposite_faces[m_fvi] = (mapped, axis)
                self.periodic_opposite_faces[p_fvi] = (
                    tuple(plus_to_minus[i] for i in p_fvi), axis)
                for t in (TAG_ALL,):
                    tag_to_boundary[t].remove((el, fn))
                    tag_to_boundary[t].remove((pel, pfn))
            if new_if:
                interfaces.append(np.array(new_if, dtype=np.int64))
        self.interfaces = np.concatenate(interfaces, axis=0) \
            if interfaces else np.zeros((0, 4), dtype=np.int64)
        self.tag_to_boundary = {
            t: np.array(v, dtype=np.int64).reshape(-1, 2)
            for t, v in tag_to_boundary.items()}

    def boundary_faces(self, tag):
        return self.tag_to_boundary.get(tag, np.zeros((0, 2), dtype=np.int64))

    def is_boundary_tag_nonempty(self, tag):
        return len(self.boundary_faces(tag)) > 0

    def face_vertex_tuple(self, el, fn):
        return tuple(int(x) for x in
                     self.elements[el, face_vertex_table(self.dimensions)[fn]])


def check_bc_coverage(mesh: Mesh, bc_tags):
    """Every TAG_ALL boundary face must carry one of `bc_tags`
    (hedge/mesh/__init__.py check_bc_coverage)."""
    covered = set()
    for t in bc_tags:
        if t is TAG_ALL:
            return
        for el, fn in mesh.boundary_faces(t):
            covered.add((int(el), int(fn)))
    for el, fn in mesh.boundary_faces(TAG_ALL):
        if (int(el), int(fn)) not in covered:
            raise MeshError("boundary face (%d, %d) not covered by any BC"
                            % (el, fn))


def _jitter(points, interior, amount, seed):
    if amount and seed is not None:
        rng = np.random.default_rng(seed)
        delta = rng.uniform(-amount, amount, size=points.shape)
        points = points + delta * interior[:, None]
    return points


def make_regular_rect_mesh(a=(0, 0), b=(1, 1), n=(5, 5), periodicity=None,
                           boundary_tagger=None, jitter=0.0, seed=None):
    """Rectangle of n[0] x n[1] grid points, each square split into
    (a,b,c), (d,c,b) triangles (hedge/mesh/generator.py:132-205).

    Boundary faces carry "minus_x", "plus_x", "minus_y", "plus_y";
    `periodicity` is a pair of bools.  `jitter` (absolute, uniform) moves
    interior grid vertices only, from `seed`.
    """
    nx, ny = n
    if min(n) < 2:
        raise MeshError("need at least two points in each direction")
    xs = np.linspace(a[0], b[0], nx)
    ys = np.linspace(a[1], b[1], ny)
    jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    points = np.stack([xs[ii.ravel()], ys[jj.ravel()]], axis=1)
    node = lambda i, j: j * nx + i   # noqa: E731  (points ordered j-major)
    i, j = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), indexing="ij")
    i, j = i.ravel(), j.ravel()
    pa, pb, pc, pd = node(i, j), node(i + 1, j), node(i, j + 1), node(i + 1, j + 1)
    elements = np.empty((2 * len(i), 3), dtype=np.int64)
    elements[0::2] = np.stack([pa, pb, pc], axis=1)
    elements[1::2] = np.stack([pd, pc, pb], axis=1)

    interior = np.ones(len(points), dtype=bool)
    interior[(ii.ravel() == 0) | (ii.ravel() == nx - 1)
             | (jj.ravel() == 0) | (jj.ravel() == ny - 1)] = False
    points = _jitter(points, interior, jitter, seed)

    periodicity = periodicity or (False, False)
    mesh_per, per_tags = [], set()
    for ax, name in enumerate("xy"):
        if periodicity[ax]:
            mesh_per.append(("minus_" + name, "plus_" + name))
            per_tags |= {"minus_" + name, "plus_" + name}
        else:
            mesh_per.append(None)

    gi = np.empty(len(points), dtype=np.int64)
    gj = np.empty(len(points), dtype=np.int64)
    gi[:] = ii.ravel()
    gj[:] = jj.ravel()

    def tagger(fvi, el, fn, allv):
        fi, fj = gi[list(fvi)], gj[list(fvi)]
        if np.all(fi == 0):
            t = "minus_x"
        elif np.all(fi == nx - 1):
            t = "plus_x"
        elif np.all(fj == 0):
            t = "minus_y"
        else:
            t = "plus_y"
        if t in per_tags:
            return [t]
        extra = boundary_tagger(fvi, el, fn, allv) if boundary_tagger else []
        return [t] + list(extra)

    return Mesh(points, elements, tagger, mesh_per)


def make_box_tet_mesh(a=(-1, -1, -1), b=(1, 1, 1), n=(20, 20, 20),
                      jitter=0.0, seed=None, boundary_tagger=None):
    """Box of n[0]*n[1]*n[2] cubes, each split into 6 tetrahedra sharing the
    cube's main diagonal (conforming across cubes).  K = 6*n0*n1*n2.

    Elements are positively oriented.  `jitter` (absolute, uniform) moves
    interior vertices only, from `seed`.  Boundary faces carry "minus_x",
    "plus_x", ... tags, plus whatever `boundary_tagger` adds.
    """
    nx, ny, nz = n
    xs = [np.linspace(a[k], b[k], n[k] + 1) for k in range(3)]
    kk, jj, ii = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1),
                             np.arange(nx + 1), indexing="ij")
    gi, gj, gk = ii.ravel(), jj.ravel(), kk.ravel()
    points = np.stack([xs[0][gi], xs[1][gj], xs[2][gk]], axis=1)

    def node(i, j, k):
        return (k * (ny + 1) + j) * (nx + 1) + i

    ci, cj, ck = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz),
                             indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()
    # order cubes z-slowest so that element numbers follow a raster order
    o = np.lexsort((ci, cj, ck))
    ci, cj, ck = ci[o], cj[o], ck[o]
    unit = np.eye(3, dtype=np.int64)
    perms = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]
    tets = []
    for p in perms:
        c0 = np.zeros(3, dtype=np.int64)
        c1 = c0 + unit[p[0]]
        c2 = c1 + unit[p[1]]
        c3 = np.ones(3, dtype=np.int64)
        tets.append([c0, c1, c2, c3])
    elements = np.empty((len(ci), 6, 4), dtype=np.int64)
    for t, corners in enumerate(tets):
        for v, c in enumerate(corners):
            elements[:, t, v] = node(ci + c[0], cj + c[1], ck + c[2])
    elements = elements.reshape(-1, 4)

    interior = ((gi > 0) & (gi < nx) & (gj > 0) & (gj < ny)
                & (gk > 0) & (gk < nz))
    points = _jitter(points, interior, jitter, seed)

    # positive orientation: swap vertices 1 and 2 where det < 0
    v = points[elements]
    det = np.linalg.det((v[:, 1:, :] - v[:, :1, :]))
    neg = det < 0
    elements[neg, 1], elements[neg, 2] = elements[neg, 2].copy(), elements[neg, 1].copy()

    lo = np.array([0, 0, 0])
    hi = np.array([nx, ny, nz])
    gidx = np.stack([gi, gj, gk], axis=1)

    def tagger(fvi, el, fn, allv):
        g = gidx[list(fvi)]
        tags = []
        for ax, name in enumerate("xyz"):
            if np.all(g[:, ax] == lo[ax]):
                tags.append("minus_" + name)
            elif np.all(g[:, ax] == hi[ax]):
                tags.append("plus_" + name)
        if boundary_tagger:
            tags += list(boundary_tagger(fvi, el, fn, allv))
        return tags

    return Mesh(points, elements, tagger, None)
