"""Quadrature rules and the per-element quadrature matrices of the
over-integrated (quadrature-grid) operators.

Rules (hedge/quadrature.py):

* Gauss-Jacobi points and weights by Golub-Welsch (quadrature.py:79-168):
  eigenvalues of the symmetric Jacobi matrix are the points, the squared
  first eigenvector components times the weight function's integral the
  weights;
* Grundmann-Moeller cubature on the biunit n-simplex (quadrature.py:241-327;
  A. Grundmann, H. M. Moeller, SIAM J. Numer. Anal. 15 (1978) 282-290),
  exact to degree 2s+1, with both signs of weights; points that coincide
  exactly (as fractions) are merged as the reference merges them;
* ``get_simplex_cubature(exact_to_degree, dim)`` chooses s =
  ceil((degree - 1) / 2): Gauss-Legendre with s + 1 points in 1D,
  Grundmann-Moeller otherwise (quadrature.py:379-400).

Element quadrature (hedge/discretization/local.py:545-690, QuadratureInfo):
the volume rule and the face rule of ``exact_to_degree``; the face rule is
mapped onto each face through the face's vertices.  The rules are invariant
under permutations of the simplex vertices, so the physical face points do
not depend on which side of a face maps them.

``element_quadrature`` turns a rule into the four matrices the quadrature
kernel applies (hedge/optemplate/operators.py:149-168, 262-314, 593-631):
nodal values to volume points, the inverse mass times the weighted
reference-gradient transpose (the quadrature stiffness transpose with M^-1
folded in), face-node values to face points, and the inverse mass times the
weighted face basis (the quadrature face mass with M^-1 folded in).

When the requested degree is at least the degree of the integrand a model
integrates (3N - 1 for the variable-coefficient advection volume term v u
d(phi)/dx), every rule exact to that degree gives the same integral, and the
volume matrices may come from the collapsed Gauss-Jacobi rule (Duffy
transform) exact to the integrand's degree, which needs fewer points than
Grundmann-Moeller in 2D (``volume_rule="exact"``).  The face rule is always the reference's: the
upwind flux switches sign inside a face, so its face integral depends on the
points.
"""

from __future__ import annotations

from fractions import Fraction
from math import ceil, exp, factorial, lgamma

import numpy as np

from .refelem import make_element


def jacobi_gauss(alpha, beta, n):
    """(points, weights) of the n+1-point Gauss-Jacobi rule on (-1, 1) for
    the weight (1-x)^alpha (1+x)^beta, by Golub-Welsch."""
    apb = alpha + beta
    T = np.zeros((n + 1, n + 1))
    for m in range(n + 1):
        if m == 0:
            T[0, 0] = -(alpha - beta) / (apb + 2)
        else:
            T[m, m] = -(alpha ** 2 - beta ** 2) / ((2 * m + apb) * (2 * m + apb + 2))
        if m < n:
            k = m + 1
            T[m, k] = T[k, m] = 2 / (2 * k + apb) * np.sqrt(
                (k * (k + apb) * (k + alpha) * (k + beta))
                / ((2 * k + apb - 1) * (2 * k + apb + 1)))
    x, vec = np.linalg.eigh(T)
    mu0 = 2 ** (apb + 1) * exp(lgamma(alpha + 1) + lgamma(beta + 1) - lgamma(apb + 2))
    return x, mu0 * vec[0, :] ** 2


def legendre_gauss(n):
    """n+1-point Gauss-Legendre rule (quadrature.py:162-168)."""
    return jacobi_gauss(0.0, 0.0, n)


def _compositions(total, parts):
    """All tuples of ``parts`` non-negative integers summing to ``total``."""
    if parts == 1:
        yield (total,)
        return
    for first in range(total, -1, -1):
        for rest in _compositions(total - first, parts - 1):
            yield (first,) + rest


def grundmann_moeller(s, n):
    """(points [P, n], weights [P]) of the Grundmann-Moeller rule of index s
    (exact to degree 2s + 1) on the biunit n-simplex {x_i >= -1,
    sum x_i <= 2 - n}, vertices (-1, ..., -1) and -1 + 2 e_k; the weights
    sum to its volume 2^n / n!.  Points sorted lexicographically."""
    d = 2 * s + 1
    acc = {}
    for i in range(s + 1):
        w = Fraction((-1) ** i * (d + n - 2 * i) ** d,
                     2 ** (2 * s) * factorial(i) * factorial(d + n - i))
        den = d + n - 2 * i
        for beta in _compositions(s - i, n + 1):
            key = tuple(Fraction(2 * b + 1, den) for b in beta)
            acc[key] = acc.get(key, 0) + w
    pts, wts = [], []
    scale = 2 ** n
    for lam, w in acc.items():
        # barycentric lam_0 .. lam_n over vertices v_0 = -1, v_k = -1 + 2 e_k
        x = np.array([-1.0 + 2.0 * float(lam[k + 1]) for k in range(n)])
        pts.append(x)
        wts.append(float(scale * w))
    order = np.lexsort(np.array(pts).T[::-1])
    return np.array(pts)[order], np.array(wts)[order]


def collapsed_gauss(dim, n):
    """Collapsed Gauss-Jacobi rule (Duffy transform) with n points per
    direction on the biunit simplex, exact to degree 2n - 1."""
    a, wa = legendre_gauss(n - 1)
    if dim == 1:
        return a[:, None], wa
    b, wb = jacobi_gauss(1.0, 0.0, n - 1)
    if dim == 2:
        A, B = np.meshgrid(a, b, indexing="ij")
        r = (1 + A) * (1 - B) / 2 - 1
        return (np.stack([r.ravel(), B.ravel()], 1),
                (wa[:, None] * wb[None, :]).ravel() / 2)
    c, wc = jacobi_gauss(2.0, 0.0, n - 1)
    A, B, Cc = np.meshgrid(a, b, c, indexing="ij")
    r = (1 + A) * (1 - B) * (1 - Cc) / 4 - 1
    s_ = (1 + B) * (1 - Cc) / 2 - 1
    w = (wa[:, None, None] * wb[None, :, None] * wc[None, None, :]).ravel() / 8
    return np.stack([r.ravel(), s_.ravel(), Cc.ravel()], 1), w


def get_simplex_cubature(exact_to_degree, dim):
    """The reference's rule for ``exact_to_degree`` in ``dim`` dimensions
    (quadrature.py:379-400): (points [P, dim], weights [P])."""
    s = int(ceil((exact_to_degree - 1) / 2))
    if dim == 1:
        x, w = legendre_gauss(s)
        return x[:, None], w
    return grundmann_moeller(s, dim)


def _nodal_basis(el, pts):
    """Nodal basis values [P, Np] and reference gradients [d, P, Np] at
    reference points ``pts`` [P, d]."""
    vinv = np.linalg.inv(el.vandermonde)
    modes = el.mode_ids()
    P = np.stack([el.basis(m, pts) for m in modes], 1)
    G = [el.grad_basis(m, pts) for m in modes]
    dP = np.stack([np.stack([g[r] for g in G], 1) for r in range(el.dimensions)])
    return P @ vinv, dP @ vinv


def face_points(el, rule_points):
    """[Nf, Pf, d] element-reference coordinates of the face rule's points on
    every face (through the face's vertices, local.py face_affine_maps)."""
    d = el.dimensions
    verts = el.unit_nodes[el.vertex_indices]
    out = []
    for fv in el.face_vertices(list(range(d + 1))):
        V = verts[list(fv)]                                   # [d, d]
        lam = (rule_points + 1) / 2                           # [Pf, d-1]
        bary = np.concatenate([1 - lam.sum(1, keepdims=True), lam], 1)
        out.append(bary @ V)
    return np.stack(out)


class ElementQuadrature:
    """Quadrature matrices of one reference element for one degree.

    ``vol_interp`` [Q, Np]: nodal -> volume points; ``vol_project``
    [d, Np, Q]: M^-1 (d phi / d r_r at the points)^T W; ``face_interp``
    [Nf, Qf, Nfp]: a face's nodes (fmask order) -> its face points;
    ``face_lift`` [Np, Nf*Qf]: M^-1 phi(face points)^T W_face.  Weights are
    reference weights: the geometric factors (d r / d x and face Jacobian
    over element Jacobian) are applied per element by the kernel."""

    def __init__(self, el, exact_to_degree, volume_rule="reference"):
        d = el.dimensions
        self.exact_to_degree = int(exact_to_degree)
        if volume_rule == "exact":
            # the fewest collapsed points exact to the degree: 2n - 1 >= degree
            vp, vw = collapsed_gauss(d, max(1, int(ceil((exact_to_degree + 1) / 2))))
        elif volume_rule == "reference":
            vp, vw = get_simplex_cubature(exact_to_degree, d)
        else:
            raise ValueError("volume_rule: 'reference' or 'exact'")
        fp, fw = get_simplex_cubature(exact_to_degree, d - 1)
        minv = el.inverse_mass_matrix
        phi, dphi = _nodal_basis(el, vp)
        self.volume_points, self.volume_weights = vp, vw
        self.face_rule_points, self.face_weights = fp, fw
        self.vol_interp = np.ascontiguousarray(phi)
        self.vol_project = np.ascontiguousarray(
            np.stack([minv @ (dphi[r].T * vw[None, :]) for r in range(d)]))
        fx = face_points(el, fp)                               # [Nf, Qf, d]
        nf, qf = fx.shape[0], fx.shape[1]
        fmask = el.fmask
        fi, fl = [], []
        for f in range(nf):
            ph, _ = _nodal_basis(el, fx[f])                    # [Qf, Np]
            fi.append(ph[:, fmask[f]])
            fl.append(minv @ (ph.T * fw[None, :]))             # [Np, Qf]
        self.face_points = fx
        self.face_interp = np.ascontiguousarray(np.stack(fi))
        self.face_lift = np.ascontiguousarray(np.concatenate(fl, 1))
        self.nq, self.nqf = len(vw), qf


def element_quadrature(dimensions, order, exact_to_degree, volume_rule="reference"):
    return ElementQuadrature(make_element(dimensions, order), exact_to_degree, volume_rule)


__all__ = ["jacobi_gauss", "legendre_gauss", "grundmann_moeller", "collapsed_gauss",
           "get_simplex_cubature", "ElementQuadrature", "element_quadrature",
           "face_points"]
