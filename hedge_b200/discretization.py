"""The B200 discretization backend: set-up on the host, RHS on the device.

Mirrors the reference's discretization plug-in surface
(hedge/discretization/__init__.py:217-1302): ``Discretization(mesh, order=)``,
``.nodes``, ``.volume_zeros``, ``.interpolate_volume_function``,
``.get_boundary``, ``.norm``, ``.integral``, ``.get_point_evaluator``,
``.dt_*_factor`` and ``.compile(op_template)``.  Volume vectors are torch
CUDA tensors in the reference layout ([K*Np], element-major; F fields are
stacked as [F, K*Np]).  ``compile`` uploads the operator once and returns a
callable that evaluates the right-hand side through the C ABI
(libhedge_b200.so); there is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
from functools import cached_property

import numpy as np

from . import _native
from .facegroups import Boundary, build_compact_connectivity, build_interior_face_group
from .mesh import Mesh, TAG_ALL, TAG_NONE
from .lowering import as_descriptor
from .optemplate import Expr
from .models import (BC_GIVEN, BC_INCIDENT, BC_NONE, MODEL_MAXWELL, MODEL_MAXWELL_TE,
                     MODEL_MAXWELL_TM, MODEL_VARADV, MODEL_VARWAVE, MODEL_WAVE,
                     MODEL_ADVECTION, OpTemplate)
from .quadrature import ElementQuadrature
from .refelem import make_element

PRECISIONS = {"plain": None, "fp64": _native.PREC_FP64, "fp32": _native.PREC_FP32,
              "fp32-simt": _native.PREC_FP32_SIMT,
              "bf16x3": _native.PREC_BF16X3, "fp16x3": _native.PREC_FP16X3}
# precisions whose state (and residual) is FP32
FP32_STATE = ("fp32", "fp32-simt")


def _torch():
    import torch
    return torch


class Discretization:
    """Nodal DG discretization of a conformal simplicial mesh.

    precision: "plain" (the state dtype is ``default_scalar_type``, FP64 or
    FP32, and so is the arithmetic), "fp32", "fp64", "bf16x3" (FP64 state,
    differentiation and lift as split-BF16 tensor-core products with FP32
    accumulation) or "fp16x3" (the same with FP16 planes of power-of-two
    scaled rows: same cost, ~8x smaller error).  "fp32" runs the two
    contractions as FP16x3 tensor-core products where a resident tensor-core
    kernel is built for the (model, dimension, order) and on CUDA cores
    otherwise; "fp32-simt" keeps them on CUDA cores.
    """

    def __init__(self, mesh: Mesh, order=None, local_discretization=None,
                 default_scalar_type=np.float64, precision="plain", debug=(),
                 device=None, quad_min_degrees=None):
        if not isinstance(mesh, Mesh):
            raise TypeError("mesh must be of type hedge_b200.mesh.Mesh")
        if (order is None) == (local_discretization is None):
            raise ValueError("must supply exactly one of local_discretization and order")
        self.quad_min_degrees = dict(quad_min_degrees or {})
        self.mesh = mesh
        self.ldis = local_discretization or make_element(mesh.dimensions, order)
        self.dimensions = mesh.dimensions
        self.order = self.ldis.order
        self.debug = set(debug)
        self.default_scalar_type = np.dtype(default_scalar_type).type
        if precision not in PRECISIONS:
            raise ValueError("unknown precision %r" % precision)
        if precision == "plain":
            precision = "fp64" if self.default_scalar_type == np.float64 else "fp32"
        if self.default_scalar_type not in (np.float64, np.float32):
            raise ValueError("default_scalar_type must be float64 or float32")
        self.precision = precision
        self._device = device
        self._handle = None

        ld = self.ldis
        self.K = len(mesh.elements)
        self.Np = ld.node_count()
        self.Nfp = ld.face_node_count()
        self.Nfaces = ld.face_count()
        un = ld.unit_nodes
        # nodes[el*Np + i] = A_el r_i + b_el  (wrap_base.cpp:82-90)
        self.nodes = np.ascontiguousarray(
            (np.einsum("kxr,nr->knx", mesh.map_a, un) + mesh.map_b[:, None, :])
            .reshape(-1, self.dimensions))
        self.fmask = ld.fmask
        self.nbr, self.nbr_code = build_compact_connectivity(mesh, ld)
        d, nf = self.dimensions, self.Nfaces
        geo = np.empty((self.K, d * d + nf * (d + 1)))
        geo[:, :d * d] = mesh.inv_map_a.reshape(self.K, d * d)
        fs = mesh.face_jacobians / np.abs(mesh.jacobians)[:, None]
        per_face = np.concatenate([mesh.face_normals, fs[..., None]], axis=-1)
        geo[:, d * d:] = per_face.reshape(self.K, nf * (d + 1))
        self.geometry = np.ascontiguousarray(geo)
        self._boundaries = {}
        if "node_permutation" in self.debug:
            self.check_node_permutation()

    # -- sizes / vectors ------------------------------------------------------
    def __len__(self):
        return self.K * self.Np

    @property
    def state_dtype(self):
        torch = _torch()
        return torch.float32 if self.precision in FP32_STATE else torch.float64

    @property
    def device(self):
        torch = _torch()
        if self._device is None:
            self._device = torch.device("cuda", torch.cuda.current_device())
        return torch.device(self._device)

    def volume_zeros(self, shape=(), dtype=None, kind="gpu"):
        torch = _torch()
        dt = self.state_dtype if dtype is None else dtype
        if kind == "numpy":
            return np.zeros(tuple(shape) + (len(self),), dtype=self.default_scalar_type)
        return torch.zeros(tuple(shape) + (len(self),), dtype=dt, device=self.device)

    def volume_empty(self, shape=(), dtype=None):
        torch = _torch()
        dt = self.state_dtype if dtype is None else dtype
        return torch.empty(tuple(shape) + (len(self),), dtype=dt, device=self.device)

    def interpolate_volume_function(self, f, dtype=None, kind="gpu"):
        """f(x) evaluated at all nodes; f takes an [N, d] array and returns
        [N] (or [F, N])."""
        vals = np.asarray(f(self.nodes), dtype=np.float64)
        if kind == "numpy":
            return vals
        return self.to_device(vals, dtype)

    def to_device(self, arr, dtype=None):
        torch = _torch()
        dt = self.state_dtype if dtype is None else dtype
        if isinstance(arr, torch.Tensor):
            return arr.to(device=self.device, dtype=dt).contiguous()
        return torch.as_tensor(np.ascontiguousarray(arr)).to(
            device=self.device, dtype=dt).contiguous()

    # -- set-up data ------------------------------------------------------------
    @cached_property
    def interior_face_group(self):
        """Reference-format interior face group (face pairs, index lists)."""
        return build_interior_face_group(self.mesh, self.ldis)

    def get_boundary(self, tag) -> Boundary:
        try:
            return self._boundaries[tag]
        except KeyError:
            b = self._boundaries[tag] = Boundary(self.mesh, self.ldis, self.nodes, tag)
            return b

    def is_boundary_tag_nonempty(self, tag):
        return self.mesh.is_boundary_tag_nonempty(tag)

    def len_boundary(self, tag):
        return len(self.get_boundary(tag).vol_indices)

    def interpolate_boundary_function(self, f, tag, kind="numpy"):
        b = self.get_boundary(tag)
        if b.is_empty():
            return np.zeros(0)
        return np.asarray(f(b.nodes), dtype=np.float64)

    def boundary_normals(self, tag):
        """[n_bdry_nodes, d] int-side normals of a boundary's nodes."""
        b = self.get_boundary(tag)
        if b.is_empty():
            return np.zeros((0, self.dimensions))
        n = self.mesh.face_normals[b.element_faces[:, 0], b.element_faces[:, 1]]
        return np.repeat(n, self.Nfp, axis=0)

    def check_node_permutation(self):
        """The reference's "node_permutation" debug check
        (discretization/__init__.py:667-678): matched face nodes coincide."""
        fg = self.interior_face_group
        il = fg.index_lists.astype(np.int64)
        ii = (fg.int_el_base[:, None] + il[fg.int_ilist]).ravel()
        ee = (fg.ext_el_base[:, None] + il[fg.ext_ilist]).ravel()
        dist = self.nodes[ii] - self.nodes[ee]
        lo, hi = self.mesh.points.min(0), self.mesh.points.max(0)
        for ax, per in enumerate(self.mesh.periodicity):
            if per is not None:
                ext = hi[ax] - lo[ax]
                dist[:, ax] = np.where(np.abs(np.abs(dist[:, ax]) - ext) < 1e-9, 0,
                                       dist[:, ax])
        err = np.abs(dist).max() if len(dist) else 0.0
        if err >= 1e-13:
            raise AssertionError("face node mismatch %g" % err)
        return err

    # -- quadrature grids (discretization/__init__.py:779-889) -------------------
    def get_quadrature_info(self, quad_tag, volume_rule="reference"):
        """The element quadrature of ``quad_tag``'s minimum degree
        (:class:`hedge_b200.quadrature.ElementQuadrature`); RuntimeError when
        the discretization has no degree for the tag, as the reference."""
        try:
            degree = self.quad_min_degrees[quad_tag]
        except KeyError:
            raise RuntimeError("minimum degree for quadrature tag '%s' is undefined"
                               % quad_tag)
        cache = self.__dict__.setdefault("_quad_cache", {})
        key = (quad_tag, volume_rule)
        if key not in cache:
            cache[key] = ElementQuadrature(self.ldis, degree, volume_rule)
        return cache[key]

    def quadrature_matrices(self, quad_tag, integrand_degree):
        """(vol_interp, vol_project, face_interp, face_lift) of the
        quadrature kernel for an integrand of ``integrand_degree`` in the
        volume: the reference's rules, except that the volume rule is the
        collapsed Gauss-Jacobi one when both are exact for the integrand and
        it has fewer points.  Without a degree for the tag, the nodal
        operators (the reference's fallback to nodal evaluation,
        mappers/__init__.py:937-958): identity interpolation,
        M^-1 D_r^T M, the face nodes and LIFT."""
        ld = self.ldis
        if self.quad_min_degrees.get(quad_tag) is None:
            import warnings
            warnings.warn("No minimum degree for quadrature tag '%s' specified--"
                          "falling back to nodal evaluation" % quad_tag)
            np_, nfp, nf = self.Np, self.Nfp, self.Nfaces
            M, Minv = ld.mass_matrix, ld.inverse_mass_matrix
            proj = np.stack([Minv @ D.T @ M for D in ld.differentiation_matrices])
            fint = np.broadcast_to(np.eye(nfp), (nf, nfp, nfp))
            return (np.eye(np_), proj, np.ascontiguousarray(fint),
                    np.ascontiguousarray(ld.lifting_matrix))
        q = vol = self.get_quadrature_info(quad_tag)
        if q.exact_to_degree >= integrand_degree:
            cache = self.__dict__.setdefault("_quad_cache", {})
            key = ("exact-volume", integrand_degree)
            if key not in cache:
                cache[key] = ElementQuadrature(self.ldis, integrand_degree, "exact")
            if cache[key].nq < q.nq:
                vol = cache[key]
        return vol.vol_interp, vol.vol_project, q.face_interp, q.face_lift

    # -- time step factors (local.py:531-540, 1052-1056, 1378-1386) -----------
    def dt_non_geometric_factor(self):
        return self.ldis.dt_non_geometric_factor()

    def dt_geometric_factor(self):
        m = self.mesh
        if self.dimensions == 2:
            v = m.points[m.elements]
            area = np.abs(2 * m.jacobians)
            semi = (np.linalg.norm(v[:, 0] - v[:, 1], axis=1)
                    + np.linalg.norm(v[:, 1] - v[:, 2], axis=1)
                    + np.linalg.norm(v[:, 2] - v[:, 0], axis=1)) / 2
            return float(np.min(area / semi))
        res = np.abs(m.jacobians) / np.max(np.abs(m.face_jacobians), axis=1)
        if self.order in (1, 2):
            res = res / 2
        return float(np.min(res))

    # -- reductions -----------------------------------------------------------
    @cached_property
    def _mass_dev(self):
        torch = _torch()
        return (torch.as_tensor(self.ldis.mass_matrix, device=self.device),
                torch.as_tensor(np.abs(self.mesh.jacobians), device=self.device))

    def integral(self, u):
        """Sum over elements of |J| 1^T M u (FP64)."""
        torch = _torch()
        M, J = self._mass_dev
        u = self.to_device(u, torch.float64)
        uu = u.reshape(*u.shape[:-1], self.K, self.Np)
        return torch.einsum("i,...ki,k->...", M.sum(0), uu, J)

    def norm(self, u, p=2):
        """L2 (energy) norm sqrt(sum_k |J_k| u_k^T M u_k), summed over leading
        field axes; FP64 accumulation on the device (hb_norm)."""
        if p != 2:
            raise NotImplementedError("only the L2 norm")
        torch = _torch()
        uu = u if isinstance(u, torch.Tensor) and u.is_cuda else self.to_device(u)
        if uu.dtype not in (torch.float64, torch.float32):
            uu = uu.double()
        uu = uu.reshape(-1, len(self)).contiguous()
        out = torch.empty(1, dtype=torch.float64, device=self.device)
        lib = _native.load()
        _native.check(lib.hb_norm(self._native_handle(), uu.shape[0],
                                  0 if uu.dtype == torch.float64 else 1, uu.data_ptr(),
                                  out.data_ptr(),
                                  torch.cuda.current_stream(self.device).cuda_stream))
        return float(out.item())

    def get_point_evaluator(self, point, thresh=0.0):
        """(discretization/__init__.py:1217-1249)"""
        m = self.mesh
        x = np.asarray(point, dtype=np.float64)
        r = np.einsum("kij,kj->ki", m.inv_map_a, x[None, :] - m.map_b)
        inside = np.all(r >= -1 - thresh, axis=1) & \
            (r.sum(axis=1) <= -(self.dimensions - 2) + thresh)
        hits = np.nonzero(inside)[0]
        if len(hits) == 0:
            raise RuntimeError("point %s not found" % (point,))
        el = int(hits[0])
        ld = self.ldis
        phi = np.array([ld.basis(mid, r[el][None, :])[0] for mid in ld.mode_ids()])
        coeff = np.linalg.solve(ld.vandermonde.T, phi)
        return PointEvaluator(self, el, coeff)

    # -- device handle ----------------------------------------------------------
    def _native_handle(self):
        if self._handle is None:
            lib = _native.load()
            ld = self.ldis
            self._keep = dict(
                dmats=np.ascontiguousarray(np.stack(ld.differentiation_matrices)),
                lift=np.ascontiguousarray(ld.lifting_matrix),
                geo=self.geometry,
                fmask=np.ascontiguousarray(ld.fmask, dtype=np.int32),
                shuffle=np.ascontiguousarray(ld.face_shuffle_table, dtype=np.int32),
                unit_nodes=np.ascontiguousarray(ld.unit_nodes, dtype=np.float64),
                mass=np.ascontiguousarray(ld.mass_matrix, dtype=np.float64),
                absjac=np.ascontiguousarray(np.abs(self.mesh.jacobians), dtype=np.float64))
            k = self._keep
            desc = _native.hb_discr_desc(
                self.dimensions, self.order, self.Np, self.Nfp, self.Nfaces,
                len(ld.face_shuffle_perms), self.K,
                k["dmats"].ctypes.data, k["lift"].ctypes.data, k["geo"].ctypes.data,
                k["fmask"].ctypes.data, k["shuffle"].ctypes.data,
                int(self.device.index or 0), k["unit_nodes"].ctypes.data,
                k["mass"].ctypes.data, k["absjac"].ctypes.data)
            h = C.c_void_p()
            _native.check(lib.hb_discr_create(C.byref(desc), C.byref(h)))
            self._handle = h
        return self._handle

    def close(self):
        if self._handle is not None:
            _native.load().hb_discr_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def compile(self, optemplate, precision=None):
        """Compile an operator template (``hedge_b200.optemplate``; lowered
        by ``hedge_b200.lowering.lower``) or an already lowered
        :class:`OpTemplate` (discretization/__init__.py:1288-1302)."""
        return CompiledOperator(self, as_descriptor(optemplate, self.dimensions, self.mesh),
                                precision or self.precision)


class PointEvaluator:
    def __init__(self, discr, el, coeff):
        self.discr, self.el, self.coeff = discr, el, coeff

    def __call__(self, field):
        torch = _torch()
        s = slice(self.el * self.discr.Np, (self.el + 1) * self.discr.Np)
        if isinstance(field, torch.Tensor):
            c = torch.as_tensor(self.coeff, dtype=field.dtype, device=field.device)
            return field[..., s] @ c
        return np.asarray(field)[..., s] @ self.coeff


def build_face_table(discr, ot):
    """Host face table of an operator: [K][Nf][2] int32, interior faces
    (neighbour, nbr_face | perm << 2), boundary faces (-1 - b, BC kind) with
    b numbering the BC_GIVEN faces (or the Maxwell incident faces with
    incident data); and the number of given boundary nodes and the given
    tag."""
    ot = as_descriptor(ot, discr.dimensions, discr.mesh)
    mesh = discr.mesh
    # BC coverage is checked where the reference checks it: in the models'
    # bind (em.py:373-377, wave.py:182-186, advection.py:86-90), not here
    nbr = discr.nbr.astype(np.int64).copy()
    code = discr.nbr_code.astype(np.int64).copy()
    bdry_faces = nbr < 0
    # boundary faces without a BC of this operator contribute no flux
    code[bdry_faces] = BC_NONE
    given_tag = None
    n_given = 0
    for tag, kind in ot.bcs:
        if tag is TAG_NONE:
            continue
        ef = mesh.boundary_faces(tag)
        if len(ef) == 0:
            continue
        code[ef[:, 0], ef[:, 1]] = kind
        if kind == BC_GIVEN or (kind == BC_INCIDENT and ot.params.get("incident_data")):
            nbr[ef[:, 0], ef[:, 1]] = -1 - np.arange(len(ef))
            given_tag = tag
            n_given = len(ef) * discr.Nfp
    conn = np.ascontiguousarray(np.stack([nbr, code], axis=-1).astype(np.int32))
    return conn, n_given, given_tag


def op_descriptor(ot, prec, conn, n_given, num_halo_faces=0, quadrature=None):
    """hb_op_desc of a model operator over a face table (``quadrature``: an
    hb_quad_desc for the quadrature models)."""
    p = ot.params
    v = np.zeros(3)
    if "v" in p:
        v[:len(p["v"])] = p["v"]
    return _native.hb_op_desc(
        ot.model, ot.n_fields, prec, ot.flux_type, p.get("bdry_flux_type", ot.flux_type),
        (C.c_double * 3)(*v), p.get("c", 0.0), p.get("eps", 1.0), p.get("mu", 1.0),
        p.get("alpha", 1.0), p.get("bdry_alpha", p.get("alpha", 1.0)),
        p.get("time_sign", 1.0), conn.ctypes.data, n_given, int(num_halo_faces),
        C.pointer(quadrature) if quadrature is not None else None)


def quadrature_descriptor(discr, ot):
    """(hb_quad_desc, host arrays it points to) of a quadrature operator:
    the integrand of the variable-coefficient advection volume term,
    v u d(phi)/dx, has degree 3N - 1."""
    mats = discr.quadrature_matrices(ot.params.get("quad_tag", "quad"), 3 * discr.order - 1)
    keep = [np.ascontiguousarray(m, dtype=np.float64) for m in mats]
    q = _native.hb_quad_desc(keep[0].shape[0], keep[2].shape[1], keep[0].ctypes.data,
                             keep[1].ctypes.data, keep[2].ctypes.data, keep[3].ctypes.data)
    return q, keep


class CompiledOperator:
    """A model right-hand side compiled for the device.

    ``op(w=..., t=..., bc_in=...)`` returns the RHS as a tensor [F, K*Np]
    ([K*Np] for a single field), like the reference's compiled op template
    (hedge/backends/jit/__init__.py:521-523).
    """

    def __init__(self, discr: Discretization, ot: OpTemplate, precision: str):
        self.discr = discr
        self.ot = ot
        self.precision = precision
        self.F = ot.n_fields
        self.conn, self.n_given, self.given_tag = build_face_table(discr, ot)
        prec = PRECISIONS[precision] if precision != "plain" else (
            _native.PREC_FP64 if discr.default_scalar_type == np.float64
            else _native.PREC_FP32)
        # Maxwell with variable material or incident data: the CUDA-core kernels
        self.var_material = bool(ot.params.get("variable_material"))
        self.incident_data = bool(ot.params.get("incident_data"))
        self.given_rows = ot.n_fields if self.incident_data else 1
        if self.var_material or self.incident_data:
            if prec in (_native.PREC_BF16X3, _native.PREC_FP16X3):
                raise NotImplementedError(
                    "Maxwell with %s: fp64 or fp32 (CUDA-core kernels)"
                    % ("variable material" if self.var_material else "incident data"))
            if prec == _native.PREC_FP32:
                prec = _native.PREC_FP32_SIMT
        self.prec_code = prec
        model = ot.operator
        p = ot.params
        quad = None
        if ot.model == MODEL_VARADV:
            if precision not in ("fp64", "fp32", "fp32-simt"):
                raise NotImplementedError("the quadrature operator runs in fp64 or fp32")
            quad, self._quad_keep = quadrature_descriptor(discr, ot)
        desc = op_descriptor(ot, prec, self.conn, self.n_given, quadrature=quad)
        lib = _native.load()
        h = C.c_void_p()
        _native.check(lib.hb_op_create(discr._native_handle(), C.byref(desc), C.byref(h)))
        self._handle = h
        self._lib = lib
        self._coeff = None
        self._source = None
        names = ot.fields or {}
        self._msrc_spec = None
        # Maxwell systems: number of carried E components (their source rows)
        self._n_e = {MODEL_MAXWELL: 3, MODEL_MAXWELL_TM: 1, MODEL_MAXWELL_TE: 2}.get(ot.model, 0)
        if self._n_e:
            self._init_maxwell_source(names, model)
        if ot.model == MODEL_VARWAVE:
            c = model.c if model is not None else (None if names.get("coeff") else 1.0)
            if c is not None and not isinstance(c, Expr):
                self.set_coefficient(c)
        if self.var_material and model is not None and hasattr(model, "material_values"):
            e, m = model.material_values(discr)
            if e is not None and m is not None:
                self.set_coefficient((e, m))
        if names and not self._n_e:
            # lowered from a template: source = sign * (const + coef * field)
            self._src_spec = (-1.0 if ot.model == MODEL_VARWAVE else 1.0,
                              float(names.get("source_const", 0.0)), names.get("source"),
                              float(names.get("source_coef", 0.0)))
            val = None
            if self._src_spec[2] is not None and model is not None:
                val = model.source if ot.model == MODEL_VARWAVE else \
                    getattr(model, "source_f", None)
                if isinstance(val, Expr):
                    val = None
            src = self._source_from(val)
            if src is not None:
                self._source = src
        elif not self._n_e:
            src = p.get("source", 0) if ot.model == MODEL_WAVE else (
                getattr(model, "source", 0) if ot.model == MODEL_VARWAVE else 0)
            if not (np.isscalar(src) and src == 0):
                self.set_source(src)

    # -- Maxwell current ----------------------------------------------------------
    def _init_maxwell_source(self, names, model):
        """Maxwell's source rows: E_c's rhs gains s_c = -J_c / eps
        (em.py:192-214).  From a lowered template: per E component
        const + coef * field (``names["sources"]``); from a descriptor: the
        model's current."""
        if names:
            self._msrc_spec = names.get("sources") or []
        elif model is not None and hasattr(model, "current_template"):
            eps = float(self.ot.params["eps"])
            cur = model.current_template()
            spec = []
            if not (np.isscalar(cur) and cur == 0):
                for o in range(self._n_e):
                    x = cur[o]
                    if isinstance(x, Expr):
                        spec.append((o, 0.0, (x.name, x.index), -1.0 / eps))
                    elif x != 0:
                        spec.append((o, -float(x) / eps, None, 0.0))
            self._msrc_spec = spec
        else:
            self._msrc_spec = []
        if not self._msrc_spec:
            return
        value = model.current_value() if model is not None and \
            hasattr(model, "current_value") else None
        src = self._maxwell_source_from(value)
        if src is not None:
            self._source = src

    def _maxwell_source_from(self, value):
        """Device [n_E, K*Np] source rows for the current field's value
        ([n_E, N] or numbers; None: not known yet and needed)."""
        torch = _torch()
        d = self.discr
        out = torch.zeros((self._n_e, len(d)), dtype=torch.float64, device=d.device)
        for o, const, fld, coef in self._msrc_spec:
            row = torch.full((len(d),), float(const), dtype=torch.float64, device=d.device)
            if fld is not None:
                if value is None:
                    return None
                v = value[fld[1]] if fld[1] is not None else value
                v = torch.full((len(d),), float(v), dtype=torch.float64, device=d.device) \
                    if np.isscalar(v) else d.to_device(v, torch.float64).reshape(-1)
                row = row + coef * v
            out[o] = row
        return out.contiguous()

    @property
    def state_dtype(self):
        torch = _torch()
        return torch.float32 if self.prec_code in (_native.PREC_FP32, _native.PREC_FP32_SIMT) \
            else torch.float64

    def set_coefficient(self, c):
        """Variable-velocity wave speed: a number or a volume vector; for the
        quadrature advection the velocity [d, K*Np]; for Maxwell with
        variable material the pair (epsilon, mu) of numbers or volume
        vectors.  Kept for calls (and recorded stages) that pass none."""
        torch = _torch()
        d = self.discr
        if self.var_material:
            eps, mu = c
            t = torch.cat([d.to_device(np.full(len(d), float(x)) if np.isscalar(x) else x,
                                       torch.float64).reshape(-1) for x in (eps, mu)])
            if t.numel() != 2 * len(d):
                raise ValueError("epsilon and mu must be volume vectors of length %d" % len(d))
            if bool((t <= 0).any()):
                raise ValueError("epsilon and mu must be positive")
            self._coeff = t.contiguous()
            return
        if self.ot.model == MODEL_VARADV:
            t = d.to_device(np.asarray(c) if not isinstance(c, torch.Tensor) else c,
                            torch.float64).reshape(-1).contiguous()
            if t.numel() != d.dimensions * len(d):
                raise ValueError("the velocity must be [%d, %d]" % (d.dimensions, len(d)))
            self._coeff = t
            return
        if np.isscalar(c):
            t = torch.full((len(d),), float(c), dtype=torch.float64, device=d.device)
        else:
            t = d.to_device(c, torch.float64)
        if t.shape != (len(d),):
            raise ValueError("c must be a volume vector of length %d" % len(d))
        self._coeff = t

    def _source_from(self, value):
        """Device source vector of a lowered template for the value of its
        source field (None: the field's value is not known yet)."""
        sign, const, name, coef = self._src_spec
        if name is None:
            if const == 0:
                return None
            value, coef = 0.0, 0.0
        elif value is None:
            return None
        torch = _torch()
        d = self.discr
        v = torch.full((len(d),), float(value), dtype=torch.float64, device=d.device) \
            if np.isscalar(value) else d.to_device(value, torch.float64).reshape(-1)
        return (sign * (const + coef * v)).contiguous()

    def set_source(self, s):
        torch = _torch()
        d = self.discr
        t = torch.full((len(d),), float(s), dtype=torch.float64, device=d.device) \
            if np.isscalar(s) else d.to_device(s, torch.float64)
        self._source = t

    def __del__(self):
        try:
            if getattr(self, "_handle", None) is not None:
                self._lib.hb_op_destroy(self._handle)
                self._handle = None
        except Exception:
            pass

    # -- argument marshalling ---------------------------------------------------
    def as_state(self, w):
        """[F, K*Np] contiguous device tensor of the state dtype (copies only
        when the input is not already that)."""
        torch = _torch()
        d = self.discr
        if isinstance(w, (list, tuple)) or (isinstance(w, np.ndarray) and w.dtype == object):
            w = torch.stack([d.to_device(x, self.state_dtype) for x in w])
        elif not isinstance(w, torch.Tensor):
            w = torch.as_tensor(np.asarray(w))
        w = w.to(device=d.device, dtype=self.state_dtype)
        w = w.reshape(self.F, len(d))
        return w.contiguous()

    def _bdry_ptr(self, bc_in):
        if self.n_given == 0:
            return None, None
        torch = _torch()
        if bc_in is None:
            raise ValueError("this operator needs boundary values (bc_in)")
        if isinstance(bc_in, (list, tuple)) or (isinstance(bc_in, np.ndarray)
                                                 and bc_in.dtype == object):
            bc_in = torch.stack([self.discr.to_device(x, torch.float64).reshape(-1)
                                 for x in bc_in])
        t = self.discr.to_device(bc_in, torch.float64).contiguous()
        if t.numel() != self.given_rows * self.n_given:
            raise ValueError("bc_in must have %s%d entries" % (
                "%d x " % self.given_rows if self.given_rows > 1 else "", self.n_given))
        return t, t.data_ptr()

    def _stream(self):
        torch = _torch()
        return torch.cuda.current_stream(self.discr.device).cuda_stream

    # -- evaluation -------------------------------------------------------------
    def _field_ptrs(self, coeff, source):
        """Device pointers of the c field (the velocity [d * K*Np] of the
        quadrature advection) and the source: the per-call tensors when given
        (FP64 on the device), else the operator's."""
        c = self._coeff if coeff is None else coeff
        s = self._source if source is None else source
        crows = self.discr.dimensions if self.ot.model == MODEL_VARADV else (
            2 if self.var_material else 1)
        for t, rows in ((coeff, crows), (source, self._n_e or 1)):
            if t is not None:
                if t.dtype != _torch().float64 or not t.is_contiguous() or \
                        t.numel() != rows * len(self.discr) or t.device != self.discr.device:
                    raise ValueError("c / source: contiguous FP64 [%d * K*Np] on the device"
                                     % rows)
        if self.var_material and s is not None and c is not None:
            # the source rows hold -J (the template's source with the
            # material at 1); the kernel adds them after dividing by
            # epsilon, so they go in as -J / epsilon (em.py:192-214, 339-371)
            n = len(self.discr)
            s = (s.reshape(self._n_e, n) / c[:n]).contiguous()
            self._src_over_eps = s       # alive until the launch is queued
        return (c.data_ptr() if c is not None else None,
                s.data_ptr() if s is not None else None)

    def rhs_into(self, q, out, bc_in=None, coeff=None, source=None):
        """out <- RHS(q); q, out: [F, K*Np] device tensors of the state dtype."""
        keep, bptr = self._bdry_ptr(bc_in)
        cptr, sptr = self._field_ptrs(coeff, source)
        _native.check(self._lib.hb_rhs(self._handle, q.data_ptr(), out.data_ptr(), cptr,
                                       bptr, sptr, self._stream()))
        return out

    def lsrk_stage(self, a, b, dt, q_in, q_out, res, bc_in=None, coeff=None, source=None):
        keep, bptr = self._bdry_ptr(bc_in)
        cptr, sptr = self._field_ptrs(coeff, source)
        _native.check(self._lib.hb_lsrk_stage(
            self._handle, float(a), float(b), float(dt), q_in.data_ptr(),
            q_out.data_ptr(), res.data_ptr(), cptr, bptr, sptr, self._stream()))

    def adjoint(self, lam, q=None, coeff=None, want_c=False):
        """Adjoint of the RHS (hb_rhs_adjoint), FP64: returns
        (q_bar, c_bar) = ((dR/dq)^T lam, (dR/dc)^T lam at the state q).
        lam, q: [F, K*Np]; c_bar ([K*Np], per node of the c field) only for
        the variable-velocity wave with ``want_c`` (else None)."""
        torch = _torch()
        d = self.discr
        lam = lam.to(device=d.device, dtype=torch.float64).reshape(self.F, len(d)).contiguous()
        if q is not None:
            q = q.to(device=d.device, dtype=torch.float64).reshape(self.F, len(d)).contiguous()
        if want_c and (self.ot.model != MODEL_VARWAVE or q is None):
            raise ValueError("c gradient: variable-velocity wave, with the state q")
        q_bar = torch.empty_like(lam)
        c_bar = torch.empty(len(d), dtype=torch.float64, device=d.device) if want_c else None
        nbytes = C.c_int64()
        _native.check(self._lib.hb_rhs_adjoint_work_size(self._handle, C.byref(nbytes)))
        work = getattr(self, "_adj_work", None)
        if work is None or work.numel() * 8 < nbytes.value:
            work = torch.empty((nbytes.value + 7) // 8, dtype=torch.float64, device=d.device)
            self._adj_work = work
        c = self._coeff if coeff is None else coeff
        _native.check(self._lib.hb_rhs_adjoint(
            self._handle, q.data_ptr() if q is not None else None, lam.data_ptr(),
            q_bar.data_ptr(), c_bar.data_ptr() if c_bar is not None else None,
            c.data_ptr() if c is not None else None, work.data_ptr(), self._stream()))
        return q_bar, c_bar

    def check(self):
        """Synchronise and raise if a kernel flagged bad input."""
        _native.check(self._lib.hb_op_check(self._handle, self._stream()))

    def launch_info(self):
        """{grid, threads, smem, elems_per_batch, ops_in_smem, blocks_per_sm}."""
        info = (C.c_int64 * 6)()
        _native.check(self._lib.hb_op_launch_info(self._handle, info, 6))
        return dict(zip(["grid", "threads", "smem", "elems_per_batch", "ops_in_smem",
                         "blocks_per_sm"], list(info)))

    def gather_map(self):
        """Device-expanded (int, ext) gather indices, [K*Nf*Nfp] each."""
        torch = _torch()
        d = self.discr
        n = d.K * d.Nfaces * d.Nfp
        ii = torch.empty(n, dtype=torch.int64, device=d.device)
        ee = torch.empty(n, dtype=torch.int64, device=d.device)
        _native.check(self._lib.hb_gather_map(self._handle, ii.data_ptr(),
                                              ee.data_ptr(), self._stream()))
        return ii, ee

    def __call__(self, w=None, t=0.0, bc_in=None, u=None, coeff=None, **kwargs):
        """Evaluate the RHS.  A compiled template takes its fields by the
        names it uses (state, given boundary data, coefficient, source),
        like the reference's compiled templates (``op(w=..., c=...)``);
        ``coeff`` gives the coefficient as the device tensor the kernels
        read (FP64, contiguous)."""
        names = self.ot.fields or {}
        source = None
        if names.get("state") in kwargs:
            w = kwargs.pop(names["state"])
        elif names.get("state_keys") and names["state_keys"][0][0] in kwargs:
            # state components named one by one
            w = [kwargs[n] if i is None else kwargs[n][i] for n, i in names["state_keys"]]
        if names.get("given") in kwargs:
            bc_in = kwargs.pop(names["given"])
        elif names.get("given_keys") and all(n in kwargs for n, _ in names["given_keys"]):
            # incident data components named one by one
            bc_in = [kwargs[n] if i is None else kwargs[n][i] for n, i in names["given_keys"]]
            for n, _ in names["given_keys"]:
                kwargs.pop(n, None)
        if names.get("coeffs") and all(n in kwargs for n, _ in names["coeffs"]):
            # variable material: epsilon, mu by their template names
            vals = [kwargs.pop(n) if i is None else kwargs.pop(n)[i] for n, i in names["coeffs"]]
            cval = _torch().cat([self.discr.to_device(x, _torch().float64).reshape(-1)
                                 for x in vals])
            coeff = cval.contiguous()
        elif names.get("coeff") in kwargs:
            cval = kwargs.pop(names["coeff"])
            if isinstance(cval, (list, tuple)) or (isinstance(cval, np.ndarray)
                                                   and cval.dtype == object):
                cval = _torch().stack([self.discr.to_device(x, _torch().float64)
                                       for x in cval])
            coeff = self.discr.to_device(cval, _torch().float64)
            coeff = coeff.reshape(-1).contiguous()
        if self._msrc_spec:
            fnames = {fld[0] for _, _, fld, _ in self._msrc_spec if fld is not None}
            for nm in fnames:
                if nm in kwargs:
                    source = self._maxwell_source_from(kwargs.pop(nm))
            if fnames and source is None and self._source is None:
                raise ValueError("this template needs its current field %r" % sorted(fnames))
        src_name = names.get("source")
        if src_name is not None and src_name[0] in kwargs:
            val = kwargs.pop(src_name[0])
            if src_name[1] is not None:
                val = val[src_name[1]]
            source = self._source_from(val)
        if w is None:
            w = u
        if self.ot.model == MODEL_VARWAVE and coeff is None and self._coeff is None:
            raise ValueError("this template needs its coefficient field %r"
                             % names.get("coeff", "c"))
        if self.ot.model == MODEL_VARADV and coeff is None and self._coeff is None:
            raise ValueError("this template needs its velocity field %r"
                             % names.get("coeff", "v"))
        if self.var_material and coeff is None and self._coeff is None:
            raise ValueError("this template needs its material fields %r"
                             % [n for n, _ in names.get("coeffs", [("epsilon", None),
                                                                   ("mu", None)])])
        if src_name is not None and source is None and self._source is None:
            raise ValueError("this template needs its source field %r" % src_name[0])
        q = self.as_state(w)
        out = self.discr.volume_empty((self.F,), self.state_dtype)
        self.rhs_into(q, out, bc_in=bc_in, coeff=coeff, source=source)
        return out[0] if self.F == 1 and self.ot.model in (MODEL_ADVECTION, MODEL_VARADV) \
            else out

    def bind_model(self, model):
        return BoundRHS(self, model)


class BoundRHS:
    """``rhs(t, w)`` of a bound model (the reference's closure from
    ``op.bind(discr)``)."""

    def __init__(self, compiled: CompiledOperator, model):
        self.compiled = compiled
        self.model = model
        self.discr = compiled.discr

    def context(self, t):
        """Given boundary data at time t that the model can evaluate itself
        (advection inflow, wave Dirichlet values given as functions)."""
        if self.compiled.n_given or self.compiled.ot.model == MODEL_VARADV:
            m = self.model
            if hasattr(m, "context"):
                return m.context(self.discr, t)
        return {}

    def __call__(self, t, w, **extra_context):
        kw = self.context(t)
        kw.update(extra_context)
        return self.compiled(w=w, t=t, **kw)


__all__ = ["Discretization", "CompiledOperator", "BoundRHS", "PointEvaluator",
           "TAG_ALL", "TAG_NONE", "MODEL_ADVECTION", "MODEL_MAXWELL"]
