"""Reference simplex elements (triangle, tetrahedron): nodes, bases, operators.

FP64 host set-up, evaluated once per (dimension, order).  Restates the
reference's local discretization:

* orthonormal Jacobi recurrence and its derivative
  (hedge/include/hedge/special_function.hpp:39-130);
* Koornwinder/Dubiner bases and gradients
  (special_function.hpp:135-345);
* Legendre-Gauss-Lobatto points by Golub-Welsch (hedge/quadrature.py:35-158);
* Warburton warp-and-blend nodes (hedge/discretization/local.py:38-109,
  978-1001, 1243-1306);
* node tuple order, face index lists, vertex indices
  (local.py:277-323, 897-953, 1120-1211);
* Vandermonde, D_r = V_r V^-1, M^-1 = V V^T, face mass, multi-face mass,
  LIFT (local.py:135-260, 342-357);
* face-node shuffles matching neighbour face orientation (local.py:401-481);
* time-step factors (local.py:531-540, 1052-1056, 1378-1386).
"""

from __future__ import annotations

import itertools
from functools import cached_property
from math import sqrt, gamma

import numpy as np


# ---------------------------------------------------------------------------
# enumeration helpers (same orders as the reference's pytools helpers)
# ---------------------------------------------------------------------------

def tuples_summing_to_at_most(n: int, length: int):
    """All non-negative integer tuples of `length` with sum <= n, first entry
    varying fastest, last entry slowest (the reference's node/mode order)."""
    if length == 0:
        yield ()
        return
    for i in range(n + 1):
        for rest in tuples_summing_to_at_most(n - i, length - 1):
            yield rest + (i,)


def wandering_element(length: int, wanderer=1, landscape=0):
    for i in range(length):
        yield i * (landscape,) + (wanderer,) + (length - 1 - i) * (landscape,)


# ---------------------------------------------------------------------------
# orthonormal Jacobi polynomials (special_function.hpp:39-130)
# ---------------------------------------------------------------------------

class JacobiPolynomial:
    """Orthonormal Jacobi polynomial P_n^(alpha,beta) on [-1, 1]."""

    def __init__(self, alpha: float, beta: float, n: int):
        self.alpha, self.beta, self.n = float(alpha), float(beta), int(n)
        a_, b_ = self.alpha, self.beta
        self.gamma0 = (2.0 ** (a_ + b_ + 1) / (a_ + b_ + 1)
                       * gamma(a_ + 1) * gamma(b_ + 1) / gamma(a_ + b_ + 1))
        self.gamma1 = (a_ + 1) * (b_ + 1) / (a_ + b_ + 3) * self.gamma0
        self.a = [2 / (2 + a_ + b_) * sqrt((a_ + 1) * (b_ + 1) / (a_ + b_ + 3))]
        self.b = [0.0]
        for i in range(1, self.n):
            h1 = 2 * i + a_ + b_
            self.a.append(2.0 / (h1 + 2) * sqrt(
                (i + 1) * (i + 1 + a_ + b_) * (i + 1 + a_) * (i + 1 + b_)
                / (h1 + 1) / (h1 + 3)))
            self.b.append(-(a_ * a_ - b_ * b_) / h1 / (h1 + 2))

    def __call__(self, x):
        x = np.asarray(x, dtype=np.float64)
        llast = np.full_like(x, 1 / sqrt(self.gamma0))
        if self.n == 0:
            return llast
        last = ((self.alpha + self.beta + 2) / 2 * x
                + (self.alpha - self.beta) / 2) / sqrt(self.gamma1)
        if self.n == 1:
            return last
        i = 1
        for i in range(1, self.n - 1):
            cur = 1 / self.a[i] * (-self.a[i - 1] * llast + (x - self.b[i]) * last)
            llast, last = last, cur
        if self.n == 2:
            i = 1
        else:
            i = self.n - 1
        return 1 / self.a[i] * (-self.a[i - 1] * llast + (x - self.b[i]) * last)


class DiffJacobiPolynomial:
    def __init__(self, alpha, beta, n):
        if n == 0:
            self.jf = None
            self.factor = 0.0
        else:
            self.jf = JacobiPolynomial(alpha + 1, beta + 1, n - 1)
            self.factor = sqrt(n * (n + alpha + beta + 1))

    def __call__(self, x):
        x = np.asarray(x, dtype=np.float64)
        if self.jf is None:
            return np.zeros_like(x)
        return self.factor * self.jf(x)


# ---------------------------------------------------------------------------
# simplex bases (special_function.hpp:135-345); vectorised over points
# ---------------------------------------------------------------------------

def triangle_basis(i, j, pts):
    r, s = pts[:, 0], pts[:, 1]
    with np.errstate(divide="ignore", invalid="ignore"):
        a = np.where(1 - s != 0, 2 * (1 + r) / (1 - s) - 1, 1.0)
    f, g = JacobiPolynomial(0, 0, i), JacobiPolynomial(2 * i + 1, 0, j)
    return sqrt(2) * f(a) * g(s) * (1 - s) ** i


def grad_triangle_basis(i, j, pts):
    r, s = pts[:, 0].copy(), pts[:, 1].copy()
    s = np.where(s >= 1, 1 - np.finfo(np.float64).eps, s)
    with np.errstate(divide="ignore", invalid="ignore"):
        a = np.where(1 - s != 0, 2 * (1 + r) / (1 - s) - 1, 1.0)
    f, df = JacobiPolynomial(0, 0, i), DiffJacobiPolynomial(0, 0, i)
    g, dg = JacobiPolynomial(2 * i + 1, 0, j), DiffJacobiPolynomial(2 * i + 1, 0, j)
    fa, gs, dfa, dgs = f(a), g(s), df(a), dg(s)
    one_s = 1 - s
    with np.errstate(divide="ignore", invalid="ignore"):
        dr = 2 * sqrt(2) * gs * one_s ** (i - 1.0) * dfa
        ds = sqrt(2) * (fa * one_s ** i * dgs
                        + (2 * r + 2) * gs * one_s ** (i - 2.0) * dfa
                        - i * fa * gs * one_s ** (i - 1.0))
    return np.stack([dr, ds])


def _tet_collapsed(pts):
    r, s, t = pts[:, 0], pts[:, 1], pts[:, 2]
    with np.errstate(divide="ignore", invalid="ignore"):
        a = np.where(s + t != 0, -2 * (1 + r) / (s + t) - 1, -1.0)
        b = np.where(1 - t != 0, 2 * (1 + s) / (1 - t) - 1, -1.0)
    return a, b, t


def tet_basis(i, j, k, pts):
    a, b, c = _tet_collapsed(pts)
    f = JacobiPolynomial(0, 0, i)
    g = JacobiPolynomial(2 * i + 1, 0, j)
    h = JacobiPolynomial(2 * i + 2 * j + 2, 0, k)
    return sqrt(8) * f(a) * g(b) * (1 - b) ** i * h(c) * (1 - c) ** (i + j)


def grad_tet_basis(i, j, k, pts):
    a, b, c = _tet_collapsed(pts)
    fa = JacobiPolynomial(0, 0, i)(a)
    gb = JacobiPolynomial(2 * i + 1, 0, j)(b)
    hc = JacobiPolynomial(2 * i + 2 * j + 2, 0, k)(c)
    dfa = DiffJacobiPolynomial(0, 0, i)(a)
    dgb = DiffJacobiPolynomial(2 * i + 1, 0, j)(b)
    dhc = DiffJacobiPolynomial(2 * i + 2 * j + 2, 0, k)(c)
    one_b, one_c = 1 - b, 1 - c
    vr = dfa * (gb * hc)
    if i > 0:
        vr = vr * (0.5 * one_b) ** (i - 1)
    if i + j > 0:
        vr = vr * (0.5 * one_c) ** (i + j - 1)
    vs = 0.5 * (1 + a) * vr
    tmp = dgb * (0.5 * one_b) ** i
    if i > 0:
        tmp = tmp + (-0.5 * i) * (gb * (0.5 * one_b) ** (i - 1))
    if i + j > 0:
        tmp = tmp * (0.5 * one_c) ** (i + j - 1)
    tmp = fa * (tmp * hc)
    vs = vs + tmp
    vt = 0.5 * (1 + a) * vr + 0.5 * (1 + b) * tmp
    tmp = dhc * (0.5 * one_c) ** (i + j)
    if i + j > 0:
        tmp = tmp - 0.5 * (i + j) * (hc * (0.5 * one_c) ** (i + j - 1))
    tmp = fa * (gb * tmp)
    tmp = tmp * (0.5 * one_b) ** i
    vt = vt + tmp
    scale = 2.0 ** (2 * i + j + 1.5)
    return np.stack([vr * scale, vs * scale, vt * scale])


# ---------------------------------------------------------------------------
# 1D helpers: LGL points (quadrature.py:35-158), warp factor (local.py:38-62)
# ---------------------------------------------------------------------------

def jacobi_gauss_points(alpha, beta, n):
    """Golub-Welsch: eigenvalues of the Jacobi matrix (ascending)."""
    apb = alpha + beta

    def a(m):
        return (2 / (2 * m + apb) * sqrt(
            (m * (m + apb) * (m + alpha) * (m + beta))
            / ((2 * m + apb - 1) * (2 * m + apb + 1))))

    def b(m):
        if m == 0:
            return -(alpha - beta) / (apb + 2)
        return -(alpha ** 2 - beta ** 2) / ((2 * m + apb) * (2 * m + apb + 2))

    T = np.zeros((n + 1, n + 1))
    for m in range(n + 1):
        T[m, m] = b(m)
        if m < n:
            T[m, m + 1] = T[m + 1, m] = a(m + 1)
    return np.linalg.eigh(T)[0]


def legendre_gauss_lobatto_points(n):
    x = np.zeros(n + 1)
    x[0], x[-1] = -1.0, 1.0
    if n == 1:
        return x
    x[1:-1] = jacobi_gauss_points(1.0, 1.0, n - 2)
    return x


class WarpFactor:
    """Warburton's 1D warp: Newton interpolant of (r_lgl - r_eq) / (1 - x^2)."""

    def __init__(self, n):
        r_lgl = legendre_gauss_lobatto_points(n)
        r_eq = np.linspace(-1, 1, n + 1)
        y = r_lgl - r_eq
        # divided differences (hedge/interpolation.py:30-47)
        coeffs = [y[0]]
        last = list(y)
        for step in range(1, len(r_eq)):
            nxt = [(last[i + 1] - last[i]) / (r_eq[i + step] - r_eq[i])
                   for i in range(len(r_eq) - step)]
            coeffs.append(nxt[0])
            last = nxt
        self.x = r_eq
        self.coeffs = coeffs

    def poly(self, x):
        result, prod = 0.0, 1.0
        for c, xm in zip(self.coeffs, self.x):
            result = result + c * prod
            prod = prod * (x - xm)
        return result

    def __call__(self, x):
        if abs(x) > 1 - 1e-10:
            return 0.0
        return self.poly(x) / (1 - x ** 2)


class FaceVertexMismatch(Exception):
    pass


def _normalize(v):
    return v / np.linalg.norm(v)


def identify_affine_map(from_points, to_points):
    """Affine (A, b) with A from_i + b = to_i (hedge/tools/affine.py:69-104)."""
    x = np.array(from_points, dtype=np.float64).T
    y = np.array(to_points, dtype=np.float64).T
    dim = x.shape[0]
    xd = (x - np.roll(x, -1, axis=1))[:, :dim]
    yd = (y - np.roll(y, -1, axis=1))[:, :dim]
    a = np.linalg.solve(xd.T, yd.T).T
    b = y[:, 0] - a @ x[:, 0]
    return a, b


def find_index_map_from_node_sets(old_nodes, new_nodes, threshold=1e-12):
    """imap with new_nodes[imap[k]] == old_nodes[k] (tools/indexing.py:151-172)."""
    imap = []
    for on in old_nodes:
        for j, nn in enumerate(new_nodes):
            if np.linalg.norm(on - nn) < threshold:
                imap.append(j)
                break
        else:
            raise ValueError("a corresponding node for %s was not found" % on)
    return tuple(imap)


# ---------------------------------------------------------------------------
# simplex reference element
# ---------------------------------------------------------------------------

class SimplexElement:
    """Order-N nodal simplex element in unit coordinates on [-1,1]^d."""

    dimensions: int

    def __init__(self, order: int):
        if order < 1:
            raise ValueError("order must be >= 1")
        self.order = int(order)

    # numbering ------------------------------------------------------------
    @cached_property
    def node_tuples(self):
        return list(tuples_summing_to_at_most(self.order, self.dimensions))

    def node_count(self):
        d, o = self.dimensions, self.order
        num = 1
        for i in range(d):
            num *= (o + 1 + i)
        return num // (1 if d == 1 else (2 if d == 2 else 6))

    def face_count(self):
        return self.dimensions + 1

    def face_node_count(self):
        return len(self.face_indices[0])

    @cached_property
    def vertex_indices(self):
        lut = {t: i for i, t in enumerate(self.node_tuples)}
        vts = [self.dimensions * (0,)] + list(
            wandering_element(self.dimensions, wanderer=self.order))
        return [lut[v] for v in vts]

    @cached_property
    def face_indices(self):
        lut = {t: i for i, t in enumerate(self.node_tuples)}
        faces = [[] for _ in range(self.dimensions + 1)]
        for t in tuples_summing_to_at_most(self.order, self.dimensions):
            for fi in self.faces_for_node_tuple(t):
                faces[fi].append(lut[t])
        return [tuple(f) for f in faces]

    @property
    def fmask(self):
        """[Nf, Nfp] local node numbers per face (int32)."""
        return np.array(self.face_indices, dtype=np.int32)

    # nodes ----------------------------------------------------------------
    def equidistant_barycentric_nodes(self):
        for idx in self.node_tuples:
            div = tuple(i / self.order for i in idx)
            yield (1 - sum(div),) + div

    @cached_property
    def unit_nodes(self):
        eq = np.array(self.equilateral_nodes(), dtype=np.float64)
        a, b = self.equilateral_to_unit
        return eq @ a.T + b

    def mode_ids(self):
        return list(tuples_summing_to_at_most(self.order, self.dimensions))

    # matrices -------------------------------------------------------------
    @cached_property
    def vandermonde(self):
        pts = self.unit_nodes
        return np.stack([self.basis(m, pts) for m in self.mode_ids()], axis=1)

    @cached_property
    def grad_vandermonde(self):
        pts = self.unit_nodes
        g = [self.grad_basis(m, pts) for m in self.mode_ids()]
        return [np.stack([gm[r] for gm in g], axis=1)
                for r in range(self.dimensions)]

    @cached_property
    def inverse_mass_matrix(self):
        v = self.vandermonde
        return v @ v.T

    @cached_property
    def mass_matrix(self):
        return np.ascontiguousarray(np.linalg.inv(self.inverse_mass_matrix))

    @cached_property
    def differentiation_matrices(self):
        v = self.vandermonde
        # leftsolve(V, Vr) = solve(V^T, Vr^T)^T
        return [np.ascontiguousarray(np.linalg.solve(v.T, vr.T).T)
                for vr in self.grad_vandermonde]

    @cached_property
    def unit_face_nodes(self):
        un = self.unit_nodes
        return np.array([un[i][:self.dimensions - 1]
                         for i in self.face_indices[0]])

    @cached_property
    def face_vandermonde(self):
        pts = self.unit_face_nodes
        return np.stack([f(pts) for f in self.face_basis()], axis=1)

    @cached_property
    def face_mass_matrix(self):
        fv = self.face_vandermonde
        return np.ascontiguousarray(np.linalg.inv(fv @ fv.T))

    @cached_property
    def multi_face_mass_matrix(self):
        fmm = self.face_mass_matrix
        nfp = fmm.shape[1]
        out = np.zeros((self.node_count(), self.face_count() * nfp))
        for f, fi in enumerate(self.face_indices):
            out[np.array(fi), f * nfp:(f + 1) * nfp] = fmm
        return out

    @cached_property
    def lifting_matrix(self):
        return self.inverse_mass_matrix @ self.multi_face_mass_matrix

    # face matching (local.py:401-481) --------------------------------------
    @cached_property
    def face_shuffle_lookup(self):
        """vertex permutation tuple -> face-node index map (imap)."""
        d = self.dimensions
        un = self.unit_nodes
        first_face_vertex_nodes = self.face_vertices(self.vertex_indices)[0]
        for i in first_face_vertex_nodes:
            assert abs(un[i][-1] + 1) < 1e-13
        fuv = [un[i][:-1] for i in first_face_vertex_nodes]
        face_nodes = self.unit_face_nodes
        result = {}
        for perm in sorted(set(itertools.permutations(range(d)))):
            a, b = identify_affine_map(fuv, [fuv[i] for i in perm])
            new_nodes = face_nodes @ a.T + b
            result[perm] = find_index_map_from_node_sets(face_nodes, new_nodes)
        return result

    @cached_property
    def face_shuffle_perms(self):
        """Ordered list of vertex permutations; a face pair stores its index."""
        return sorted(self.face_shuffle_lookup.keys())

    @cached_property
    def face_shuffle_table(self):
        """[n_perms, Nfp] int32: imap for each permutation id."""
        return np.array([self.face_shuffle_lookup[p]
                         for p in self.face_shuffle_perms], dtype=np.int32)

    def face_shuffle_id(self, face_1_vertices, face_2_vertices):
        lut = {v: i for i, v in enumerate(face_1_vertices)}
        try:
            norm = tuple(lut[v] for v in face_2_vertices)
        except KeyError:
            raise FaceVertexMismatch("face vertices do not match")
        return self.face_shuffle_perms.index(norm)

    # time step (local.py:531-540) -----------------------------------------
    def dt_non_geometric_factor(self):
        un = self.unit_nodes
        vi = self.vertex_indices
        return 2 / 3 * min(
            min(min(np.linalg.norm(un[fn] - un[v]) for v in vi if v != fn)
                for fn in face)
            for face in self.face_indices)


class TriangleElement(SimplexElement):
    """Faces AB, BC, AC (local.py:838-1058)."""

    dimensions = 2
    equilateral_to_unit = (np.array([[1, -1 / sqrt(3)], [0, 2 / sqrt(3)]]),
                           np.array([-1 / 3, -1 / 3]))
    alpha_opt = [0.0000, 0.0000, 1.4152, 0.1001, 0.2751, 0.9800, 1.0999,
                 1.2832, 1.3648, 1.4773, 1.4959, 1.5743, 1.5770, 1.6223, 1.6258]

    @staticmethod
    def face_vertices(v):
        return [(v[0], v[1]), (v[1], v[2]), (v[0], v[2])]

    def faces_for_node_tuple(self, t):
        m, n = t
        res = []
        if n == 0:
            res.append(0)
        if n + m == self.order:
            res.append(1)
        if m == 0:
            res.append(2)
        return res

    @staticmethod
    def barycentric_to_equilateral(bp):
        l1, l2, l3 = bp
        return np.array([(-l1 + l2), (-l1 - l2 + 2 * l3) / sqrt(3.0)])

    def _warper(self, alpha):
        warp = WarpFactor(self.order)
        verts = [self.barycentric_to_equilateral(b)
                 for b in wandering_element(3)]
        fvi = self.face_vertices([0, 1, 2])
        fverts = self.face_vertices(verts)
        edgedirs = [_normalize(v2 - v1) for v1, v2 in fverts]
        opp = [(set(range(3)) - set(f)).pop() for f in fvi]
        info = list(zip(fvi, edgedirs, opp))

        def apply(bp):
            shift = np.zeros(2)
            for f, ed, o in info:
                blend = 4 * bp[f[0]] * bp[f[1]]
                amt = blend * warp(bp[f[1]] - bp[f[0]]) * (1 + (alpha * bp[o]) ** 2)
                shift = shift + amt * ed
            return shift
        return apply

    def equilateral_nodes(self):
        try:
            alpha = self.alpha_opt[self.order - 1]
        except IndexError:
            alpha = 5 / 3
        warp = self._warper(alpha)
        return [self.barycentric_to_equilateral(bp) + warp(bp)
                for bp in self.equidistant_barycentric_nodes()]

    def basis(self, mode, pts):
        return triangle_basis(mode[0], mode[1], pts)

    def grad_basis(self, mode, pts):
        return grad_triangle_basis(mode[0], mode[1], pts)

    def face_basis(self):
        return [(lambda p, i=i: JacobiPolynomial(0, 0, i)(p[:, 0]))
                for i in range(self.order + 1)]

    @staticmethod
    def dt_geometric_factor(vertices, jacobian):
        area = abs(2 * jacobian)
        semiperim = sum(np.linalg.norm(vertices[a] - vertices[b])
                        for a, b in [(0, 1), (1, 2), (2, 0)]) / 2
        return area / semiperim


class TetrahedronElement(SimplexElement):
    """Faces ABC, ABD, ACD, BCD (local.py:1062-1386)."""

    dimensions = 3
    equilateral_to_unit = (np.array([[1, -1 / sqrt(3), -1 / sqrt(6)],
                                     [0, 2 / sqrt(3), -1 / sqrt(6)],
                                     [0, 0, sqrt(6) / 2]]),
                           np.array([-1 / 2, -1 / 2, -1 / 2]))
    alpha_opt = [0, 0, 0, 0.1002, 1.1332, 1.5608, 1.3413, 1.2577, 1.1603,
                 1.10153, 0.6080, 0.4523, 0.8856, 0.8717, 0.9655]

    @staticmethod
    def face_vertices(v):
        return [(v[0], v[1], v[2]), (v[0], v[1], v[3]),
                (v[0], v[2], v[3]), (v[1], v[2], v[3])]

    def faces_for_node_tuple(self, t):
        m, n, o = t
        res = []
        if o == 0:
            res.append(0)
        if n == 0:
            res.append(1)
        if m == 0:
            res.append(2)
        if n + m + o == self.order:
            res.append(3)
        return res

    @staticmethod
    def barycentric_to_equilateral(bp):
        l1, l2, l3, l4 = bp
        return np.array([(-l1 + l2), (-l1 - l2 + 2 * l3) / sqrt(3.0),
                         (-l1 - l2 - l3 + 3 * l4) / sqrt(6.0)])

    def equilateral_nodes(self):
        if self.order - 1 < len(self.alpha_opt):
            alpha = self.alpha_opt[self.order - 1]
        else:
            alpha = 1
        verts = [self.barycentric_to_equilateral(b)
                 for b in wandering_element(4)]
        fvi_all = self.face_vertices([0, 1, 2, 3])
        fverts = self.face_vertices(verts)
        bary = list(self.equidistant_barycentric_nodes())
        equi = [self.barycentric_to_equilateral(bp) for bp in bary]
        tri_warp = TriangleElement(self.order)._warper(alpha)
        for fvi, (v1, v2, v3) in zip(fvi_all, fverts):
            dirs = [_normalize(v2 - v1), _normalize(v3 - (v1 + v2) / 2)]
            opp = (set(range(4)) - set(fvi)).pop()
            shifted = []
            for bp, ep in zip(bary, equi):
                face_bp = [bp[i] for i in fvi]
                blend = face_bp[0] * face_bp[1] * face_bp[2] \
                    * (1 + alpha * bp[opp]) ** 2
                for i in fvi:
                    denom = bp[i] + 0.5 * bp[opp]
                    if abs(denom) > 1e-12:
                        blend /= denom
                    else:
                        blend = 0.5
                        break
                tw = tri_warp(face_bp)
                shifted.append(ep + blend * (tw[0] * dirs[0] + tw[1] * dirs[1]))
            equi = shifted
        return equi

    def basis(self, mode, pts):
        return tet_basis(mode[0], mode[1], mode[2], pts)

    def grad_basis(self, mode, pts):
        return grad_tet_basis(mode[0], mode[1], mode[2], pts)

    def face_basis(self):
        return [(lambda p, m=m: triangle_basis(m[0], m[1], p))
                for m in tuples_summing_to_at_most(self.order, 2)]

    def dt_geometric_factor_from(self, jacobian, face_jacobians):
        res = abs(jacobian) / max(abs(fj) for fj in face_jacobians)
        if self.order in (1, 2):
            res /= 2
        return res


def make_element(dimensions: int, order: int) -> SimplexElement:
    if dimensions == 2:
        return TriangleElement(order)
    if dimensions == 3:
        return TetrahedronElement(order)
    raise ValueError("only triangles (2D) and tetrahedra (3D) are supported")
