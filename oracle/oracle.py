"""CPU ORACLE -- test infrastructure only (the checker, never the product).

Evaluates a model's DG right-hand side the way hedge's jit CPU backend does:
the loops of liboracle.so (hedge_oracle.cpp, a restatement of the jit
backend's generated diff / flux-gather / lift code) composed with numpy
vector expressions exactly as the reference's compiled op template orders
them (hedge/backends/jit/__init__.py:39-258):

  1. DiffBatchAssign: d_r u for every operand            (jit/diff.py:137-175)
  2. chain rule  du/dx_k = sum_r (dr/dx_k) d_r u
                                  (optemplate/mappers/__init__.py:556-591)
  3. FluxBatchAssign per face group: gather + multi-face mass lift, no
     scaling (is_lift False, jit/__init__.py:155-168)
  4. InverseMass(1/J * flux sum): ReferenceInverseMass elementwise
     (mappers/__init__.py:579-581; jit/__init__.py:501-519)
  5. the model's vector combination (models/*.py op templates)
  6. LSRK4 (timestep/runge_kutta.py:104-131) with numpy linear combination.

Parity is pinned against the reference's own known-answer tests (restated
in tests/test_oracle_kat.py); the reference itself cannot run here.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

OR_ADVECTION, OR_WAVE, OR_VARWAVE, OR_MAXWELL, OR_NORMAL_DOT = 1, 2, 3, 4, 9
OR_MAXWELL_TM, OR_MAXWELL_TE = 5, 6        # 2D (Ez, Hx, Hy) and (Ex, Ey, Hz)
_MAXWELLS = (OR_MAXWELL, OR_MAXWELL_TM, OR_MAXWELL_TE)
# positions of a Maxwell system's fields in (Ex Ey Ez Hx Hy Hz), E count
_SLOTS = {OR_MAXWELL: ([0, 1, 2, 3, 4, 5], 3), OR_MAXWELL_TM: ([2, 3, 4], 1),
          OR_MAXWELL_TE: ([0, 1, 5], 2)}
(BC_NONE, BC_GIVEN, BC_DIRICHLET, BC_NEUMANN, BC_RADIATION, BC_PEC, BC_PMC, BC_ABSORB,
 BC_INCIDENT) = range(9)


class or_flux_params(C.Structure):
    _fields_ = [("model", C.c_int), ("dim", C.c_int), ("flux_type", C.c_int),
                ("n_args", C.c_int), ("v", C.c_double * 3), ("c", C.c_double),
                ("eps", C.c_double), ("mu", C.c_double), ("alpha", C.c_double),
                ("time_sign", C.c_double)]


class or_face_group(C.Structure):
    _fields_ = [("n_pairs", C.c_int64), ("face_length", C.c_int),
                ("face_count", C.c_int), ("n_local_els", C.c_int64),
                ("double_sided", C.c_int),
                ("int_el_base", C.c_void_p), ("int_ilist", C.c_void_p),
                ("int_fof_base", C.c_void_p), ("ext_el_base", C.c_void_p),
                ("ext_ilist", C.c_void_p), ("ext_fof_base", C.c_void_p),
                ("ext_write_map", C.c_void_p), ("normal", C.c_void_p),
                ("face_jacobian", C.c_void_p), ("index_lists", C.c_void_p),
                ("local_el_write_base", C.c_void_p),
                ("local_el_inverse_jacobians", C.c_void_p)]


_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB) or (os.path.getmtime(LIB) <
                                       os.path.getmtime(os.path.join(HERE, "hedge_oracle.cpp"))):
            build()
        lib = C.CDLL(LIB)
        vp = C.c_void_p
        lib.or_diff.argtypes = [C.c_int64, C.c_int, C.c_int, vp, vp, vp]
        lib.or_elwise.argtypes = [C.c_int64, C.c_int, C.c_int, vp, vp, vp, vp]
        lib.or_gather_interior.argtypes = [vp, vp, C.c_int64, vp, vp]
        lib.or_gather_boundary.argtypes = [vp, vp, C.c_int64, vp, C.c_int64, vp, vp]
        lib.or_lift.argtypes = [vp, C.c_int, vp, vp, vp, vp]
        lib.or_lincomb.argtypes = [C.c_int64, C.c_double, vp, C.c_double, vp, vp]
        lib.or_max_threads.argtypes = [C.c_int]
        lib.or_max_threads.restype = C.c_int
        _lib = lib
    return _lib


def set_threads(n):
    return load().or_max_threads(int(n))


def _p(a):
    return a.ctypes.data


class _FG:
    """ctypes view of a reference-format face group (keeps arrays alive)."""

    def __init__(self, fg):
        self.keep = [np.ascontiguousarray(getattr(fg, k)) for k in (
            "int_el_base", "int_ilist", "int_fof_base", "ext_el_base", "ext_ilist",
            "ext_fof_base", "ext_write_map", "normal", "face_jacobian",
            "index_lists", "local_el_write_base", "local_el_inverse_jacobians")]
        self.c = or_face_group(fg.n_pairs, fg.face_length, fg.face_count,
                               fg.n_local_els, int(fg.double_sided),
                               *[_p(a) for a in self.keep])
        self.fg = fg


class OracleRHS:
    """Model RHS on the CPU, following the reference jit backend.

    discr: a hedge_b200 Discretization (only its host-side set-up arrays are
    read: reference matrices, geometry, face groups, boundaries)."""

    def __init__(self, discr, optemplate, c_field=None, source=None, material=None):
        """material: (epsilon, mu) volume vectors of a Maxwell operator with
        variable material (default: the model's own values)."""
        from hedge_b200.lowering import as_descriptor
        self.discr = discr
        self.ot = ot = as_descriptor(optemplate, discr.dimensions, discr.mesh)
        ld = discr.ldis
        self.dim = discr.dimensions
        self.K, self.Np = discr.K, discr.Np
        self.N = self.K * self.Np
        self.dmats = np.ascontiguousarray(np.stack(ld.differentiation_matrices))
        self.emat = np.ascontiguousarray(ld.multi_face_mass_matrix)
        self.minv = np.ascontiguousarray(ld.inverse_mass_matrix)
        m = discr.mesh
        # per-node metric d r_r / d x_k (discretization/__init__.py:488-532)
        self.imd = np.repeat(m.inv_map_a, self.Np, axis=0)       # [N, r, x]
        self.inv_jac = np.repeat(1.0 / np.abs(m.jacobians), self.Np)
        self.fg_int = _FG(discr.interior_face_group) if len(m.interfaces) else None
        p = ot.params
        self.c_field = None if c_field is None else np.asarray(c_field, dtype=np.float64)
        if ot.model == OR_VARWAVE and self.c_field is None:
            c = ot.operator.c
            self.c_field = np.full(self.N, float(c)) if np.isscalar(c) else \
                np.asarray(c, dtype=np.float64)
        self.source = source
        if self.source is None and ot.model == OR_WAVE and p.get("source", 0) != 0:
            self.source = p["source"]
        if self.source is None and ot.model == OR_VARWAVE:
            s = getattr(ot.operator, "source", 0)
            if not (np.isscalar(s) and s == 0):
                self.source = s
        if self.source is None and ot.model in _MAXWELLS and \
                hasattr(ot.operator, "current_value"):
            # Maxwell: the source is the current J (em.py:192-214)
            j = ot.operator.current_value()
            if not (np.isscalar(j) and j == 0):
                self.source = j
        self.material = None
        if ot.model in _MAXWELLS and p.get("variable_material"):
            if material is None and hasattr(ot.operator, "material_values"):
                material = ot.operator.material_values(discr)
            if material is None or any(x is None for x in material):
                raise ValueError("variable material: pass material=(epsilon, mu)")
            self.material = np.ascontiguousarray(
                np.stack([np.asarray(x, dtype=np.float64).reshape(-1) for x in material]))
        self.params = self._params(bdry=False)
        self.bparams = self._params(bdry=True)
        self.bdry = []
        for tag, kind in ot.bcs:
            b = discr.get_boundary(tag)
            if b.is_empty():
                continue
            self.bdry.append((tag, kind, b, _FG(b.face_group),
                              discr.boundary_normals(tag)))

    def _params(self, bdry):
        ot, p = self.ot, self.ot.params
        v = np.zeros(3)
        if "v" in p:
            v[:len(p["v"])] = p["v"]
        ft = ot.flux_type
        alpha = p.get("alpha", 1.0)
        if ot.model in _MAXWELLS and bdry:
            ft, alpha = p["bdry_flux_type"], p["bdry_alpha"]
        return or_flux_params(ot.model, self.dim, ft, ot.n_flux_args,
                              (C.c_double * 3)(*v), p.get("c", 0.0), p.get("eps", 1.0),
                              p.get("mu", 1.0), alpha, p.get("time_sign", 1.0))

    # -- pieces -----------------------------------------------------------------
    def ref_diff(self, u):
        out = np.empty((self.dim, self.N))
        load().or_diff(self.K, self.Np, self.dim, _p(self.dmats),
                       _p(np.ascontiguousarray(u)), _p(out))
        return out

    def grad(self, u):
        """Physical gradient [d, N] of a volume vector."""
        dr = self.ref_diff(u)
        return np.einsum("nrx,rn->xn", self.imd, dr)

    def _lift_e(self, fgw, fof):
        out = np.zeros((fof.shape[0], self.N))
        lib = load()
        for c in range(fof.shape[0]):
            lib.or_lift(C.byref(fgw.c), self.Np, _p(self.emat), None,
                        _p(np.ascontiguousarray(fof[c])), _p(out[c]))
        return out

    def flux_args(self, fields):
        if self.ot.model == OR_VARWAVE:
            return np.ascontiguousarray(np.vstack([self.c_field[None], fields]))
        if self.material is not None:
            # em.py:309-371: flux_w = (epsilon, mu, w)
            return np.ascontiguousarray(np.vstack([self.material, fields]))
        return np.ascontiguousarray(fields)

    def bc_values(self, kind, args, b, normals, bc_in):
        """Ext-state vectors on a boundary (BoundarizeOperator + BC formula)."""
        ab = args[:, b.vol_indices]
        m = self.ot.model
        if kind == BC_GIVEN and m == OR_WAVE:
            # inhomogeneous Dirichlet data g (wave.py:133-142): (2 g - u, v)
            out = ab.copy()
            out[0] = 2.0 * np.asarray(bc_in, dtype=np.float64).reshape(-1) - ab[0]
            return out
        if kind == BC_GIVEN:
            return np.asarray(bc_in, dtype=np.float64).reshape(1, -1)
        if m in (OR_WAVE, OR_VARWAVE):
            C0 = 1 if m == OR_VARWAVE else 0
            sgn = (1.0 if self.ot.params.get("c", 1.0) > 0 else -1.0) if m == OR_WAVE \
                else self.ot.params["time_sign"]
            out = ab.copy()
            u, v = ab[C0], ab[C0 + 1:]
            if kind == BC_DIRICHLET:
                out[C0] = -u
            elif kind == BC_NEUMANN:
                out[C0 + 1:] = -v
            elif kind == BC_RADIATION:
                nv = np.einsum("nx,xn->n", normals, v)
                out[C0] = 0.5 * (u - sgn * nv)
                out[C0 + 1:] = 0.5 * normals.T * (nv - sgn * u)
            return out
        if m in _MAXWELLS:
            # em.py:226-307 on the six components (2D systems embedded, n_z =
            # 0); variable material: the boundary vector is (B(eps), B(mu),
            # bc) and the absorbing impedance is the local one
            slots, _ = _SLOTS[m]
            mat = ab[:2] if self.material is not None else None
            if mat is not None:
                ab = ab[2:]
            full = np.zeros((6, ab.shape[1]))
            full[slots] = ab
            e, h = full[:3], full[3:]
            nrm = np.zeros((ab.shape[1], 3))
            nrm[:, :normals.shape[1]] = normals
            if kind == BC_PEC:
                out = np.vstack([-e, h])
            elif kind == BC_PMC:
                out = np.vstack([e, -h])
            elif kind == BC_ABSORB:
                p = self.ot.params
                Z = np.sqrt(p["mu"] / p["eps"]) if mat is None else np.sqrt(mat[1] / mat[0])
                ne, nh = np.cross(nrm, e.T).T, np.cross(nrm, h.T).T
                nne, nnh = np.cross(nrm, ne.T).T, np.cross(nrm, nh.T).T
                out = np.vstack([e + 0.5 * (nne - Z * nh), h + 0.5 * (nnh + ne / Z)])
            elif kind == BC_INCIDENT:
                # -(incident data) (em.py:289-307): the given [F][n] values,
                # or the default zero data
                if bc_in is not None:
                    out = np.zeros_like(full)
                    out[slots] = -np.asarray(bc_in, dtype=np.float64).reshape(len(slots), -1)
                else:
                    out = np.zeros_like(full)
            else:
                raise ValueError("unsupported boundary kind %d" % kind)
            return out[slots] if mat is None else np.vstack([mat, out[slots]])
        raise ValueError("unsupported boundary kind %d" % kind)

    def flux_volume(self, fields, bc_in=None):
        """Sum over face groups of E * (Fjac * flux), one row per component."""
        lib = load()
        args = self.flux_args(fields)
        ncomp = self.ot.n_fields
        total = np.zeros((ncomp, self.N))
        if self.fg_int is not None:
            fg = self.fg_int.fg
            fof = np.zeros((ncomp, fg.n_local_els * fg.face_count * fg.face_length))
            lib.or_gather_interior(C.byref(self.fg_int.c), C.byref(self.params),
                                   self.N, _p(args), _p(fof))
            total += self._lift_e(self.fg_int, fof)
        for tag, kind, b, fgw, normals in self.bdry:
            if kind == BC_NONE:
                continue
            bargs = np.ascontiguousarray(self.bc_values(kind, args, b, normals, bc_in))
            fg = fgw.fg
            fof = np.zeros((ncomp, fg.n_local_els * fg.face_count * fg.face_length))
            lib.or_gather_boundary(C.byref(fgw.c), C.byref(self.bparams), self.N,
                                   _p(args), bargs.shape[1], _p(bargs), _p(fof))
            total += self._lift_e(fgw, fof)
        return total

    def inverse_mass(self, v):
        """ReferenceInverseMass(1/J * v) elementwise."""
        out = np.empty_like(v)
        lib = load()
        for c in range(v.shape[0]):
            scaled = np.ascontiguousarray(self.inv_jac * v[c])
            lib.or_elwise(self.K, self.Np, self.Np, _p(self.minv), None,
                          _p(scaled), _p(out[c]))
        return out

    # -- full RHS -----------------------------------------------------------------
    def __call__(self, fields, t=0.0, bc_in=None):
        fields = np.atleast_2d(np.asarray(fields, dtype=np.float64))
        m, p, d = self.ot.model, self.ot.params, self.dim
        lifted = self.inverse_mass(self.flux_volume(fields, bc_in))
        if m == OR_ADVECTION:
            g = self.grad(fields[0])
            vol = -np.einsum("x,xn->n", p["v"][:d], g)[None]
            return vol + lifted
        if m in (OR_WAVE, OR_VARWAVE):
            u, v = fields[0], fields[1:]
            gu = self.grad(u)
            div = sum(self.grad(v[k])[k] for k in range(d))
            c = p["c"] if m == OR_WAVE else p["time_sign"] * self.c_field
            out = np.vstack([(c * div)[None], c * gu]) + lifted
            if self.source is not None:
                src = np.full(self.N, self.source) if np.isscalar(self.source) \
                    else np.asarray(self.source)
                out[0] += src if m == OR_WAVE else -src
            return out
        if m in _MAXWELLS:
            # the six components' gradients (2D systems: fields not carried
            # and z derivatives zero)
            slots, ne = _SLOTS[m]
            g = np.zeros((6, 3, self.N))
            for k, slot in enumerate(slots):
                g[slot, :d] = self.grad(fields[k])

            def curl(a):
                return np.stack([g[a + 2, 1] - g[a + 1, 2], g[a, 2] - g[a + 2, 0],
                                 g[a + 1, 0] - g[a, 1]])
            vol = np.vstack([curl(3), -curl(0)])[slots]
            if self.source is not None:
                # eps dE/dt = curl H - J + lifted flux
                j = np.asarray(self.source, dtype=np.float64)
                vol[:ne] -= j.reshape(ne, -1) if j.size >= ne * self.N else \
                    np.broadcast_to(j.reshape(-1, 1), (ne, self.N))
            if self.material is not None:
                div = np.vstack([self.material[0]] * ne + [self.material[1]] * (len(slots) - ne))
            else:
                div = np.array([p["eps"]] * ne + [p["mu"]] * (len(slots) - ne))[:, None]
            return (vol + lifted) / div
        raise ValueError("unknown model")

    def lsrk4_step(self, y, t, dt, residual, bc_fn=None):
        """One LSRK4 step (runge_kutta.py:104-131); returns (y, residual)."""
        from hedge_b200.timestep import RK4A, RK4B, RK4C
        for a, b, c in zip(RK4A, RK4B, RK4C):
            bc = bc_fn(t + c * dt) if bc_fn else None
            r = self(y, t + c * dt, bc_in=bc)
            residual = a * residual + dt * r
            y = y + b * residual
        return y, residual
