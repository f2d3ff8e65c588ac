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
  (discretization/__init__.py:1055-1093); boundary normals per boundary node.
"""

from __future__ import annotations

import numbers

import numpy as np

from hedge_b200 import flux as fl
from hedge_b200 import optemplate as ot
from hedge_b200.mesh import TAG_NONE


def _num(x):
    return isinstance(x, numbers.Number) and not isinstance(x, bool)


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

    # -- element-local operators ---------------------------------------------------
    def grad(self, u, axis):
        ue = u.reshape(self.K, self.Np)
        dr = np.einsum("rij,kj->kri", self.dmats, ue)                # [K, r, Np]
        return np.einsum("kr,kri->ki", self.imd[:, :, axis], dr).reshape(-1)

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
