"""Face connectivity: the reference's face-pair groups and the compact
per-element-face table the CUDA kernels read.

Reference semantics (hedge/discretization/__init__.py:565-774,
hedge/discretization/data.py:199-248, hedge/tools/indexing.py:106-148):

* an interior face pair (el_l, f_l | el_n, f_n) gathers the int side through
  ``face_indices[f_l]`` and the ext side through
  ``face_indices[f_n]`` shuffled by the face-index shuffle that matches
  el_n's face vertices to el_l's (periodic faces first map el_n's vertices
  through ``periodic_opposite_faces``);
* ``ext_native_write_map`` equals the shuffle's index map;
* face-pair outputs ("fluxes on faces") sit at
  ``Nfp * (local_el_number * Nf + face)``, local element numbers from the
  sorted (el_base_index, element_id) set;
* index lists are deduplicated in first-seen order.

The compact table replaces the per-pair records on the GPU: for every
(element, face) one int32 pair (neighbour, code).  Interior:
neighbour >= 0, code = nbr_face | perm_id << 2, and the neighbour volume node
of local face node i is ``fmask[nbr_face][shuffle[perm_id][i]]``.  Boundary:
neighbour = -1 - (face's number in its boundary vector), code = BC kind.
"""

from __future__ import annotations

import numpy as np

from .mesh import Mesh, TAG_ALL, face_vertex_table
from .refelem import SimplexElement


def _face_tuples(mesh: Mesh, els, fns):
    return mesh.elements[els[:, None], face_vertex_table(mesh.dimensions)[fns]]


def interior_shuffle_ids(mesh: Mesh, ldis: SimplexElement, el_l, f_l, el_n, f_n):
    """Shuffle id (index into ldis.face_shuffle_perms) matching el_n's face
    to el_l's face, for arrays of face pairs."""
    d = mesh.dimensions
    vl = _face_tuples(mesh, el_l, f_l)      # [n, d]
    vn = _face_tuples(mesh, el_n, f_n).copy()
    # periodic faces: map the neighbour's vertices to the local side
    if mesh.periodic_opposite_faces:
        hit = (vn[:, :, None] == vl[:, None, :]).any(axis=2).all(axis=1)
        for r in np.nonzero(~hit)[0]:
            vn[r] = mesh.periodic_opposite_faces[tuple(int(x) for x in vn[r])][0]
    pos = np.full(vn.shape, -1, dtype=np.int64)
    for k in range(d):
        for m in range(d):
            pos[:, k] = np.where(vn[:, k] == vl[:, m], m, pos[:, k])
    if np.any(pos < 0):
        raise ValueError("face vertices do not match")
    perm_lut = {p: i for i, p in enumerate(ldis.face_shuffle_perms)}
    codes = pos @ (d ** np.arange(d - 1, -1, -1))
    code_lut = np.full(d ** d, -1, dtype=np.int64)
    for p, i in perm_lut.items():
        code_lut[int(np.dot(p, d ** np.arange(d - 1, -1, -1)))] = i
    ids = code_lut[codes]
    if np.any(ids < 0):
        raise ValueError("invalid face vertex permutation")
    return ids


class IndexListRegistry:
    """Deduplicating index-list numbering (hedge/tools/indexing.py:106-148)."""

    def __init__(self):
        self.index_lists = []
        self._by_id = {}
        self._by_list = {}

    def register(self, identifier, generator):
        try:
            return self._by_id[identifier]
        except KeyError:
            il = tuple(int(x) for x in generator())
            nbr = self._by_list.get(il)
            if nbr is None:
                nbr = len(self.index_lists)
                self.index_lists.append(il)
                self._by_list[il] = nbr
            self._by_id[identifier] = nbr
            return nbr


class FaceGroup:
    """Reference-format face group (StraightFaceGroup after commit), as
    structure-of-arrays."""

    def __init__(self, **kw):
        self.__dict__.update(kw)


def build_interior_face_group(mesh: Mesh, ldis: SimplexElement) -> FaceGroup:
    """Interior face group (discretization/__init__.py:596-689)."""
    np_ = ldis.node_count()
    nfp = ldis.face_node_count()
    nf = ldis.face_count()
    ifs = mesh.interfaces
    el_l, f_l, el_n, f_n = ifs[:, 0], ifs[:, 1], ifs[:, 2], ifs[:, 3]
    ids = interior_shuffle_ids(mesh, ldis, el_l, f_l, el_n, f_n)
    reg = IndexListRegistry()
    fi = ldis.face_indices
    table = ldis.face_shuffle_table
    int_il = np.empty(len(ifs), dtype=np.int32)
    ext_il = np.empty(len(ifs), dtype=np.int32)
    ewm = np.empty(len(ifs), dtype=np.int32)
    for p in range(len(ifs)):
        a, b, s = int(f_l[p]), int(f_n[p]), int(ids[p])
        int_il[p] = reg.register(a, lambda: fi[a])
        ext_il[p] = reg.register((b, s), lambda: [fi[b][k] for k in table[s]])
        ewm[p] = reg.register((b, s, "wtm"), lambda: table[s])
    used = np.unique(np.concatenate([el_l, el_n]))
    local = np.full(len(mesh.elements), -1, dtype=np.int64)
    local[used] = np.arange(len(used))
    return FaceGroup(
        n_pairs=len(ifs), face_length=nfp, face_count=nf,
        n_local_els=len(used), double_sided=True,
        int_element=el_l, int_face=f_l, ext_element=el_n, ext_face=f_n,
        shuffle_id=ids,
        int_el_base=(el_l * np_).astype(np.int64),
        ext_el_base=(el_n * np_).astype(np.int64),
        int_ilist=int_il, ext_ilist=ext_il, ext_write_map=ewm,
        int_fof_base=(nfp * (local[el_l] * nf + f_l)).astype(np.int64),
        ext_fof_base=(nfp * (local[el_n] * nf + f_n)).astype(np.int64),
        normal=np.ascontiguousarray(mesh.face_normals[el_l, f_l]),
        face_jacobian=np.ascontiguousarray(mesh.face_jacobians[el_l, f_l]),
        index_lists=np.array(reg.index_lists, dtype=np.uint32).reshape(-1, nfp),
        local_el_write_base=(used * np_).astype(np.int64),
        local_el_inverse_jacobians=1.0 / np.abs(mesh.jacobians[used]),
    )


class Boundary:
    """Boundary of one tag (discretization/__init__.py:697-774): node
    coordinates, the volume indices they come from, and the one-sided face
    group whose ext side indexes the boundary vector."""

    def __init__(self, mesh: Mesh, ldis: SimplexElement, nodes, tag):
        np_ = ldis.node_count()
        nfp = ldis.face_node_count()
        nf = ldis.face_count()
        ef = mesh.boundary_faces(tag)
        self.tag = tag
        self.element_faces = ef
        fmask = ldis.fmask
        if len(ef):
            vol = ef[:, 0:1] * np_ + fmask[ef[:, 1]]
        else:
            vol = np.zeros((0, nfp), dtype=np.int64)
        self.vol_indices = vol.reshape(-1).astype(np.int64)
        self.nodes = nodes[self.vol_indices]
        if len(ef) == 0:
            self.face_group = None
            return
        reg = IndexListRegistry()
        fi = ldis.face_indices
        int_il = np.array([reg.register(int(f), lambda f=f: fi[int(f)])
                           for f in ef[:, 1]], dtype=np.int32)
        ext_id = reg.register((), lambda: range(nfp))
        used = np.unique(ef[:, 0])
        local = np.full(len(mesh.elements), -1, dtype=np.int64)
        local[used] = np.arange(len(used))
        self.face_group = FaceGroup(
            n_pairs=len(ef), face_length=nfp, face_count=nf,
            n_local_els=len(used), double_sided=False,
            int_element=ef[:, 0], int_face=ef[:, 1],
            int_el_base=(ef[:, 0] * np_).astype(np.int64),
            ext_el_base=(np.arange(len(ef)) * nfp).astype(np.int64),
            int_ilist=int_il, ext_ilist=np.full(len(ef), ext_id, dtype=np.int32),
            ext_write_map=np.zeros(len(ef), dtype=np.int32),
            int_fof_base=(nfp * (local[ef[:, 0]] * nf + ef[:, 1])).astype(np.int64),
            ext_fof_base=np.zeros(len(ef), dtype=np.int64),
            normal=np.ascontiguousarray(mesh.face_normals[ef[:, 0], ef[:, 1]]),
            face_jacobian=np.ascontiguousarray(mesh.face_jacobians[ef[:, 0], ef[:, 1]]),
            index_lists=np.array(reg.index_lists, dtype=np.uint32).reshape(-1, nfp),
            local_el_write_base=(used * np_).astype(np.int64),
            local_el_inverse_jacobians=1.0 / np.abs(mesh.jacobians[used]),
        )

    def is_empty(self):
        return len(self.vol_indices) == 0


def build_compact_connectivity(mesh: Mesh, ldis: SimplexElement):
    """[K, Nf] neighbour element and neighbour-face/shuffle code for every
    element face, from that element's own perspective.  Boundary faces get
    neighbour -1 (resolved per operator by `resolve_boundary`)."""
    K, nf = len(mesh.elements), mesh.face_count
    nbr = np.full((K, nf), -1, dtype=np.int64)
    code = np.zeros((K, nf), dtype=np.int64)
    ifs = mesh.interfaces
    for (a, fa, b, fb) in ((0, 1, 2, 3), (2, 3, 0, 1)):
        el_l, f_l, el_n, f_n = ifs[:, a], ifs[:, fa], ifs[:, b], ifs[:, fb]
        ids = interior_shuffle_ids(mesh, ldis, el_l, f_l, el_n, f_n)
        nbr[el_l, f_l] = el_n
        code[el_l, f_l] = f_n | (ids << 2)
    return nbr, code


def gather_index_pairs_from_face_group(fg: FaceGroup, np_):
    """Canonical form of an interior face group's gather maps: the sorted
    (int volume index, ext volume index) pairs over all face nodes."""
    il = fg.index_lists.astype(np.int64)
    ii = fg.int_el_base[:, None] + il[fg.int_ilist]
    ee = fg.ext_el_base[:, None] + il[fg.ext_ilist]
    pairs = np.stack([ii.ravel(), ee.ravel()], axis=1)
    both = np.concatenate([pairs, pairs[:, ::-1]], axis=0)
    o = np.lexsort((both[:, 1], both[:, 0]))
    return both[o]


__all__ = ["FaceGroup", "Boundary", "build_interior_face_group",
           "build_compact_connectivity", "interior_shuffle_ids",
           "gather_index_pairs_from_face_group", "TAG_ALL"]
