"""CPU executor of operator templates (numpy) -- test infrastructure only.

It evaluates a template built with ``hedge_b200.optemplate`` /
``hedge_b200.flux`` directly, node by node, the way the reference's jit
executor runs a compiled template (hedge/backends/jit/__init__.py:39-358),
without the lowering onto kernel models that ``Discretization.compile``
does.  Comparing it with the C oracle (``OracleRHS``) pins the models'
templates, and comparing it with compiled templates on the GPU pins the
lowering.

* derivatives: D_r per element then the chain rule with the per-element
  inverse metric (jit/diff.py:137-175; mappers/__init__.py:556-591);
* flux operators: per face node, Fjac * flux(n, int, ext) on the interior
  face pairs, both sides (the ext side with the normal negated and int/ext
  swapped, hedge/flux FluxFlipper), written through the ext write map
  (jit/flux.py:239-360); on a boundary pair's faces one-sided with the ext
  values from the boundary vector (jit/flux.py:365-480); then the face-mass
  lift E (face_operators.hpp:154-263);
* inverse mass: M^-1 (1/J u) per element (jit/__init__.py:249-258);
* BoundarizeOperator: the volume vector at the boundary's nodes
  (discretization/__init__.py:1055-1093); boundary normals per boundary node;
* weak derivative S_x^T u: per element (M D_r)^T u times dr/dx |J|
  (operators.py:141-143 with the reference element's matrices);
* over-integration (operators.py:149-168, 262-314, 593-631): where a
  stiffness-transpose or a flux operator acts on up-sampled fields, the
  integrals are taken by quadrature on the elements and on every face, with
  the interior / exterior traces evaluated from each element's own
  polynomial at the physical quadrature points and boundary data
  interpolated from the face nodes.  The rule: when the discretization has a
  minimum degree for the up-samplers' tag (``quad_min_degrees``), the
  reference's own (hedge/quadrature.py:379-400: Gauss-Legendre with s + 1
  points on 1D faces, Grundmann-Moeller of index s otherwise,
  s = ceil((degree - 1) / 2)), restated here in ``reference_cubature``;
  else collapsed Gauss-Jacobi rules (Duffy transform, Gauss-Legendre x
  Gauss-Jacobi(1,0) [x Gauss-Jacobi(2,0)] points, exact to degree
  2(N+2)-1 per direction), an independent evaluation of the integrals the
  nodal operators compute in closed form;
* ElementwiseMaxOperator: each element's nodes set to its largest nodal
  value (volume_operators.hpp:356-369).
"""

from __future__ import annotations

import numbers

import numpy as np

from hedge_b200 import flux as fl
from hedge_b200 import optemplate as ot
from hedge_b200.mesh import TAG_ALL, TAG_NONE, face_vertex_table
from hedge_b200.refelem import make_element

_QUAD = (ot.QuadratureGridUpsampler, ot.QuadratureInteriorFacesGridUpsampler,
         ot.QuadratureBoundaryGridUpsampler)


def _has_quad(x):
    return any(isinstance(n, ot.OperatorBinding) and isinstance(n.op, _QUAD)
               for n in ot.walk(x))


def _gauss_jacobi(n, alpha):
    from scipy.special import roots_jacobi
    return roots_jacobi(n, alpha, 0.0)


def simplex_rule(dim, n):
    """Collapsed Gauss-Jacobi rule on the reference simplex (vertices -1 /
    unit vectors scaled to [-1, 1]); weights sum to its volume."""
    a, wa = np.polynomial.legendre.leggauss(n)
    if dim == 1:
        return a[:, None], wa
    b, wb = _gauss_jacobi(n, 1.0)
    if dim == 2:
        A, B = np.meshgrid(a, b, indexing="ij")
        r = (1 + A) * (1 - B) / 2 - 1
        return np.stack([r.ravel(), B.ravel()], 1), (wa[:, None] * wb[None, :]).ravel() / 2
    c, wc = _gauss_jacobi(n, 2.0)
    A, B, Cc = np.meshgrid(a, b, c, indexing="ij")
    r = (1 + A) * (1 - B) * (1 - Cc) / 4 - 1
    s_ = (1 + B) * (1 - Cc) / 2 - 1
    w = (wa[:, None, None] * wb[None, :, None] * wc[None, None, :]).ravel() / 8
    return np.stack([r.ravel(), s_.ravel(), Cc.ravel()], 1), w


def reference_cubature(exact_to_degree, dim):
    """The reference's simplex rule for ``exact_to_degree``
    (hedge/quadrature.py:241-327, 379-400): points on the biunit simplex
    and weights.  1D: the s+1-point Gauss-Legendre rule; dim >= 2: the
    Grundmann-Moeller rule of index s (Grundmann, Moeller, SIAM J. Numer.
    Anal. 15 (1978) 282-290): weight (-1)^i 2^(-2s) (d+n-2i)^d / (i! (d+n-i)!)
    at the barycentric points ((2 b_k + 1) / (d+n-2i))_k for every
    composition b of s - i into n + 1 parts, i = 0..s, d = 2s + 1; equal
    points merged; times 2^n for the biunit simplex."""
    from fractions import Fraction
    from itertools import product
    from math import ceil, factorial
    s = int(ceil((exact_to_degree - 1) / 2))
    if dim == 1:
        x, w = np.polynomial.legendre.leggauss(s + 1)
        return x[:, None], w
    n, d = dim, 2 * s + 1
    acc = {}
    for i in range(s + 1):
        den = d + n - 2 * i
        wt = Fraction((-1) ** i * den ** d, 4 ** s * factorial(i) * factorial(d + n - i))
        for b in product(range(s - i + 1), repeat=n):
            if sum(b) > s - i:
                continue
            bb = (s - i - sum(b),) + b
            key = tuple(Fraction(2 * k + 1, den) for k in bb)
            acc[key] = acc.get(key, Fraction(0)) + wt
    pts = np.array([[2 * float(lam[k]) - 1 for k in range(1, n + 1)] for lam in acc])
    wts = np.array([float(w * 2 ** n) for w in acc.values()])
    return pts, wts


def _num(x):
    return isinstance(x, numbers.Number) and not isinstance(x, bool)


def _quad_tag(x):
    for n in ot.walk(x):
        if isinstance(n, ot.OperatorBinding) and isinstance(
                n.op, _QUAD + (ot.QuadratureStiffnessTOperator,)):
            return n.op.quadrature_tag
    return None


class TemplateExecutor:
    def __init__(self, discr):
        self.d = discr
        ld = discr.ldis
        self.K, self.Np, self.dim = discr.K, discr.Np, discr.dimensions
        self.N = self.K * self.Np
        self.dmats = np.stack(ld.differentiation_matrices)          # [r, Np, Np]
        self.emat = np.asarray(ld.multi_face_mass_matrix)           # [Np, Nf*Nfp]
        self.minv = np.asarray(ld.inverse_mass_matrix)
        self.imd = discr.mesh.inv_map_a                             # [K, r, x]
        self.absj = np.abs(discr.mesh.jacobians)
        self._groups = {}
        self._quad = {}

    # -- nodal basis at arbitrary points ----------------------------------------------
    def _phi(self, r):
        """Nodal basis values [P, Np] (and reference gradients [d, P, Np]) at
        reference points r [P, d]."""
        ld = self.d.ldis
        modes = ld.mode_ids()
        vinv = np.linalg.inv(ld.vandermonde)
        P = np.stack([ld.basis(m, r) for m in modes], 1)
        G = [ld.grad_basis(m, r) for m in modes]
        dP = np.stack([np.stack([g[k] for g in G], 1) for k in range(self.dim)])
        return P @ vinv, dP @ vinv

    def _to_ref(self, k, x):
        m = self.d.mesh
        return (x - m.map_b[k]) @ m.inv_map_a[k].T

    def _setup_quadrature(self, tag=None):
        """Volume and face quadrature of ``tag``: the reference's rule of the
        discretization's minimum degree for the tag, else collapsed rules of
        degree 2 (N + 2) - 1 per direction."""
        if tag in self._quad:
            return self._quad[tag]
        d, N, m = self.dim, self.d.order, self.d.mesh
        degree = getattr(self.d, "quad_min_degrees", {}).get(tag)
        if degree is not None:
            rq, wq = reference_cubature(degree, d)
            fr, fw = reference_cubature(degree, d - 1)
        else:
            rq, wq = simplex_rule(d, N + 2)
            fr, fw = simplex_rule(d - 1, N + 2)
        phi_q, dphi_q = self._phi(rq)
        # faces: physical points, weights, normals, int / ext basis values
        nf = d + 1
        ftab = face_vertex_table(d)
        K = self.K
        nbr = {}
        for el_l, f_l, el_n, f_n in m.interfaces:
            nbr[(int(el_l), int(f_l))] = int(el_n)
            nbr[(int(el_n), int(f_n))] = int(el_l)
        faces = []
        for k in range(K):
            verts = m.points[m.elements[k]]
            for f in range(nf):
                P = verts[list(ftab[f])]
                if d == 2:
                    x = P[0] + (fr[:, :1] + 1) / 2 * (P[1] - P[0])
                    dA = fw * np.linalg.norm(P[1] - P[0]) / 2
                else:
                    x = P[0] + (fr[:, :1] + 1) / 2 * (P[1] - P[0]) + \
                        (fr[:, 1:2] + 1) / 2 * (P[2] - P[0])
                    dA = fw * np.linalg.norm(np.cross(P[1] - P[0], P[2] - P[0])) / 4
                phi_i, _ = self._phi(self._to_ref(k, x))
                e = nbr.get((k, f))
                phi_e = self._phi(self._to_ref(e, x))[0] if e is not None else None
                faces.append(dict(k=k, f=f, x=x, dA=dA, n=m.face_normals[k, f],
                                  phi_i=phi_i, ext=e, phi_e=phi_e, P=P))
        self._quad[tag] = dict(wq=wq, phi_q=phi_q, dphi_q=dphi_q, faces=faces)
        return self._quad[tag]

    # -- element-local operators ---------------------------------------------------
    def grad(self, u, axis):
        ue = u.reshape(self.K, self.Np)
        dr = np.einsum("rij,kj->kri", self.dmats, ue)                # [K, r, Np]
        return np.einsum("kr,kri->ki", self.imd[:, :, axis], dr).reshape(-1)

    def stiffness_t(self, f, axis):
        """Nodal S_x^T f per element: dr/dx |J| (M D_r)^T f."""
        M = self.d.ldis.mass_matrix
        fe = f.reshape(self.K, self.Np)
        out = np.zeros_like(fe)
        for r in range(self.dim):
            S = M @ self.dmats[r]
            out += (self.imd[:, r, axis] * self.absj)[:, None] * (fe @ S)
        return out.reshape(-1)

    def _qvol(self, x, env, tag=None):
        """An up-sampled expression at the volume quadrature points [K, Q]."""
        q = self._setup_quadrature(tag)
        if _num(x):
            return np.full((self.K, len(q["wq"])), float(x))
        if isinstance(x, ot.Field):
            return self.vol(x, env).reshape(self.K, self.Np) @ q["phi_q"].T
        if isinstance(x, ot.Sum):
            return sum(self._qvol(c, env, tag) for c in x.children)
        if isinstance(x, ot.Product):
            r = 1.0
            for c in x.children:
                r = r * self._qvol(c, env, tag)
            return r
        if isinstance(x, ot.OperatorBinding) and isinstance(x.op, ot.QuadratureGridUpsampler):
            return self._qvol(x.field, env, tag)
        raise NotImplementedError("quadrature-grid node %r" % (x,))

    def quad_stiffness_t(self, x, axis, env, tag=None):
        tag = _quad_tag(x) if tag is None else tag
        q = self._setup_quadrature(tag)
        fq = self._qvol(x, env, tag)                                # [K, Q]
        dphi = np.einsum("kr,rqi->kqi", self.imd[:, :, axis], q["dphi_q"])
        return (np.einsum("q,kq,kqi->ki", q["wq"], fq, dphi) * self.absj[:, None]).reshape(-1)

    def _strip(self, x):
        """Template with the up-samplers removed (their operands' values at
        a point are the same polynomial's)."""
        if isinstance(x, np.ndarray):
            return np.array([self._strip(c) for c in x.reshape(-1)], dtype=object)
        if isinstance(x, ot.OperatorBinding) and isinstance(x.op, _QUAD):
            return self._strip(x.field)
        if isinstance(x, ot.Sum):
            r = 0
            for c in x.children:
                r = ot.add(r, self._strip(c))
            return r
        if isinstance(x, ot.Product):
            r = 1
            for c in x.children:
                r = ot.mul(r, self._strip(c))
            return r
        if isinstance(x, ot.OperatorBinding):
            return ot.OperatorBinding(x.op, self._strip(x.field))
        return x

    def _face_interp(self, face, vals_at_nodes):
        """Boundary data given at a face's nodes -> its quadrature points
        (polynomial of degree N in the face's own coordinates)."""
        d, N = self.dim, self.d.order
        k, f = face["k"], face["f"]
        xn = self.d.nodes[k * self.Np + self.d.ldis.fmask[f]]
        P = face["P"]

        def coords(x):
            A = (P[1:] - P[0]).T                                   # [d, d-1]
            ab = np.linalg.lstsq(A, (x - P[0]).T, rcond=None)[0].T
            return 2 * ab - 1
        if d == 2:
            vn = np.polynomial.legendre.legvander(coords(xn)[:, 0], N)
            vq = np.polynomial.legendre.legvander(coords(face["x"])[:, 0], N)
        else:
            tri = make_element(2, N)
            modes = tri.mode_ids()
            vn = np.stack([tri.basis(m, coords(xn)) for m in modes], 1)
            vq = np.stack([tri.basis(m, coords(face["x"])) for m in modes], 1)
        return vq @ np.linalg.solve(vn, vals_at_nodes)

    def _bq(self, x, env, face, bpos):
        """Boundary data at a face's quadrature points."""
        if _num(x):
            return np.full(len(face["dA"]), float(x))
        if isinstance(x, ot.Field):
            v = env[x.name]
            v = v[x.index] if x.index is not None else v
            v = np.broadcast_to(np.asarray(v, dtype=np.float64), (bpos[1],))
            return self._face_interp(face, v[bpos[0]:bpos[0] + self.d.Nfp])
        if isinstance(x, ot.Sum):
            return sum(self._bq(c, env, face, bpos) for c in x.children)
        if isinstance(x, ot.Product):
            r = 1.0
            for c in x.children:
                r = r * self._bq(c, env, face, bpos)
            return r
        if isinstance(x, ot.BoundaryNormalComponent):
            return np.full(len(face["dA"]), face["n"][x.axis])
        if isinstance(x, ot.OperatorBinding):
            if isinstance(x.op, _QUAD):
                return self._bq(x.field, env, face, bpos)
            if isinstance(x.op, ot.BoundarizeOperator):
                return face["phi_i"] @ self.vol(self._strip(x.field), env).reshape(
                    self.K, self.Np)[face["k"]]
        raise NotImplementedError("boundary quadrature node %r" % (x,))

    def quad_flux(self, flux, arg, env):
        """Face integrals of the flux against the test functions, by face
        quadrature, on interior faces (arg a volume vector) or on a
        boundary pair's faces."""
        q = self._setup_quadrature(_quad_tag(arg.field if isinstance(arg, ot.BoundaryPair)
                                             else arg))
        out = np.zeros((self.K, self.Np))
        pair = arg if isinstance(arg, ot.BoundaryPair) else None
        field = self._strip(pair.field if pair is not None else arg)
        vals = [self.vol(c, env).reshape(self.K, self.Np) for c in _comps(field)]
        bfaces = None
        if pair is not None:
            if pair.tag is TAG_NONE:
                return out.reshape(-1)
            ef = self.d.mesh.boundary_faces(pair.tag)
            nb = len(ef) * self.d.Nfp
            bfaces = {(int(a), int(b)): i * self.d.Nfp for i, (a, b) in enumerate(ef)}
        for face in q["faces"]:
            k, f = face["k"], face["f"]
            iv = [face["phi_i"] @ v[k] for v in vals]
            if pair is None:
                if face["ext"] is None:
                    continue
                ev = [face["phi_e"] @ v[face["ext"]] for v in vals]
            else:
                if (k, f) not in bfaces:
                    continue
                ev = [self._bq(c, env, face, (bfaces[(k, f)], nb)) for c in _comps(pair.bfield)]
            nvec = np.broadcast_to(face["n"], (len(face["dA"]), self.dim))
            fv = self._flux_vals(flux, iv, ev, nvec)
            out[k] += (face["dA"] * fv) @ face["phi_i"]
        return out.reshape(-1)

    def inverse_mass(self, v):
        ve = v.reshape(self.K, self.Np) / self.absj[:, None]
        return (ve @ self.minv.T).reshape(-1)

    def _lift(self, fg, fof):
        out = np.zeros(self.N)
        nf, nfp = fg.face_count, fg.face_length
        loc = fof.reshape(fg.n_local_els, nf * nfp) @ self.emat.T   # [n_local, Np]
        idx = fg.local_el_write_base[:, None] + np.arange(self.Np)
        np.add.at(out, idx.reshape(-1), loc.reshape(-1))
        return out

    # -- fluxes --------------------------------------------------------------------
    def _flux_vals(self, f, iv, ev, n):
        if _num(f):
            return np.full(n.shape[:-1], float(f))
        if isinstance(f, fl.FieldComponent):
            return (iv if f.is_interior else ev)[f.index]
        if isinstance(f, fl.Normal):
            return n[..., f.axis]
        if isinstance(f, ot.Sum):
            return sum(self._flux_vals(c, iv, ev, n) for c in f.children)
        if isinstance(f, ot.Product):
            r = 1.0
            for c in f.children:
                r = r * self._flux_vals(c, iv, ev, n)
            return r
        if isinstance(f, ot.Quotient):
            return self._flux_vals(f.num, iv, ev, n) / self._flux_vals(f.den, iv, ev, n)
        if isinstance(f, ot.Power):
            return self._flux_vals(f.base, iv, ev, n) ** self._flux_vals(f.exponent, iv, ev, n)
        if isinstance(f, fl.IfPositive):
            return np.where(self._flux_vals(f.criterion, iv, ev, n) > 0,
                            self._flux_vals(f.then, iv, ev, n),
                            self._flux_vals(f.else_, iv, ev, n))
        if isinstance(f, fl.FunctionCall):
            a = [self._flux_vals(x, iv, ev, n) for x in f.args]
            return {"abs": np.abs, "max": np.maximum, "min": np.minimum}[f.name](*a)
        raise NotImplementedError("flux term %s" % f)

    def _interior_flux(self, flux, arg, env):
        fg = self.d.interior_face_group
        vals = [self.vol(c, env) for c in _comps(arg)]
        il = fg.index_lists.astype(np.int64)
        ii = fg.int_el_base[:, None] + il[fg.int_ilist]
        ee = fg.ext_el_base[:, None] + il[fg.ext_ilist]
        n = np.broadcast_to(fg.normal[:, None, :], ii.shape + (self.dim,))
        fj = fg.face_jacobian[:, None]
        iv = [v[ii] for v in vals]
        ev = [v[ee] for v in vals]
        fof = np.zeros(fg.n_local_els * fg.face_count * fg.face_length)
        k = np.arange(fg.face_length)
        fof[fg.int_fof_base[:, None] + k] = fj * self._flux_vals(flux, iv, ev, n)
        wm = il[fg.ext_write_map]
        fof[fg.ext_fof_base[:, None] + wm] = fj * self._flux_vals(flux, ev, iv, -n)
        return self._lift(fg, fof)

    def _boundary_flux(self, flux, pair, env):
        b = self.d.get_boundary(pair.tag)
        if b.is_empty():
            return np.zeros(self.N)
        fg = b.face_group
        vals = [self.vol(c, env) for c in _comps(pair.field)]
        bvals = [self.bdry(c, env, b) for c in _comps(pair.bfield)]
        il = fg.index_lists.astype(np.int64)
        ii = fg.int_el_base[:, None] + il[fg.int_ilist]
        ee = fg.ext_el_base[:, None] + il[fg.ext_ilist]
        n = np.broadcast_to(fg.normal[:, None, :], ii.shape + (self.dim,))
        iv = [v[ii] for v in vals]
        ev = [np.broadcast_to(v, (len(b.vol_indices),))[ee] for v in bvals]
        fof = np.zeros(fg.n_local_els * fg.face_count * fg.face_length)
        k = np.arange(fg.face_length)
        fof[fg.int_fof_base[:, None] + k] = fg.face_jacobian[:, None] * \
            self._flux_vals(flux, iv, ev, n)
        return self._lift(fg, fof)

    # -- evaluation ----------------------------------------------------------------
    def vol(self, x, env):
        if _num(x):
            return np.full(self.N, float(x))
        if isinstance(x, ot.Field):
            v = env[x.name]
            v = v[x.index] if x.index is not None else v
            return np.broadcast_to(np.asarray(v, dtype=np.float64), (self.N,))
        if isinstance(x, ot.Sum):
            return sum(self.vol(c, env) for c in x.children)
        if isinstance(x, ot.Product):
            r = 1.0
            for c in x.children:
                r = r * self.vol(c, env)
            return r
        if isinstance(x, ot.Quotient):
            return self.vol(x.num, env) / self.vol(x.den, env)
        if isinstance(x, ot.Power):
            return self.vol(x.base, env) ** self.vol(x.exponent, env)
        if isinstance(x, ot.OperatorBinding):
            op = x.op
            if isinstance(op, ot.DifferentiationOperator):
                return self.grad(self.vol(x.field, env), op.xyz_axis)
            if isinstance(op, ot.InverseMassOperator):
                return self.inverse_mass(self.vol(x.field, env))
            if isinstance(op, ot.QuadratureStiffnessTOperator):
                return self.quad_stiffness_t(x.field, op.xyz_axis, env, op.quadrature_tag)
            if isinstance(op, ot.ElementwiseMaxOperator):
                v = np.asarray(self.vol(x.field, env)).reshape(self.K, self.Np)
                return np.repeat(v.max(axis=1), self.Np)
            if isinstance(op, ot.StiffnessTOperator):
                if _has_quad(x.field):
                    return self.quad_stiffness_t(x.field, op.xyz_axis, env)
                return self.stiffness_t(self.vol(x.field, env), op.xyz_axis)
            if isinstance(op, ot.FluxOperator) and _has_quad(
                    x.field.field if isinstance(x.field, ot.BoundaryPair) else x.field):
                return self.quad_flux(op.flux, x.field, env)
            if isinstance(op, ot.FluxOperator):
                arg = x.field
                if isinstance(arg, ot.BoundaryPair):
                    if arg.tag is TAG_NONE:
                        return np.zeros(self.N)
                    return self._boundary_flux(op.flux, arg, env)
                return self._interior_flux(op.flux, arg, env)
        raise NotImplementedError("volume node %r" % (x,))

    def bdry(self, x, env, b):
        nb = len(b.vol_indices)
        if _num(x):
            return np.full(nb, float(x))
        if isinstance(x, ot.Field):
            v = env[x.name]
            v = v[x.index] if x.index is not None else v
            return np.broadcast_to(np.asarray(v, dtype=np.float64), (nb,))
        if isinstance(x, ot.Sum):
            return sum(self.bdry(c, env, b) for c in x.children)
        if isinstance(x, ot.Product):
            r = 1.0
            for c in x.children:
                r = r * self.bdry(c, env, b)
            return r
        if isinstance(x, ot.Quotient):
            return self.bdry(x.num, env, b) / self.bdry(x.den, env, b)
        if isinstance(x, ot.Power):
            return self.bdry(x.base, env, b) ** self.bdry(x.exponent, env, b)
        if isinstance(x, ot.BoundaryNormalComponent):
            return self.d.boundary_normals(x.boundary_tag)[:, x.axis]
        if isinstance(x, ot.OperatorBinding) and isinstance(x.op, ot.BoundarizeOperator):
            return self.vol(x.field, env)[b.vol_indices]
        raise NotImplementedError("boundary node %r" % (x,))

    def __call__(self, template, **env):
        """Outputs of ``template`` for the named fields: [n_outputs, K*Np]."""
        return np.stack([np.array(self.vol(x, env)) for x in _comps(template)])


def _comps(x):
    if isinstance(x, np.ndarray):
        return list(x.reshape(-1))
    return [x]


__all__ = ["TemplateExecutor"]
