"""Hyperbolic DG operators: advection, wave, variable-velocity wave, Maxwell.

Constructor signatures, ``op_template()`` and ``bind(discr) -> rhs(t, w)``
mirror the reference's models.  ``op_template()`` builds the reference's
symbolic template in this package's template language
(``hedge_b200.optemplate`` / ``hedge_b200.flux``); ``Discretization.compile``
lowers any such template onto the fused kernels.  ``descriptor()`` gives the
lowered form (:class:`OpTemplate`) directly:

* StrongAdvectionOperator  hedge/models/advection.py:124-149
  rhs = -v.grad u + M^-1 (flux(u) + flux(BoundaryPair(u, bc_in, inflow)))
* StrongWaveOperator       hedge/models/wave.py:37-197
  rhs = (c div v, c grad u) + M^-1 (fluxes) [+ source on u]
* VariableVelocityStrongWaveOperator  hedge/models/wave.py:204-418
  rhs = (ts c div v - source, ts c grad u) + M^-1 (fluxes of (c, u, v))
* MaxwellOperator          hedge/models/em.py:38-387 (fixed material)
  rhs = ((curl H - J) , -curl E) + M^-1 (fluxes)) / (eps | mu)
* TMMaxwellOperator, TEMaxwellOperator  hedge/models/em.py:485-515 (2D
  subsets (Ez, Hx, Hy) and (Ex, Ey, Hz) of the same system)
* VariableCoefficientAdvectionOperator  hedge/models/advection.py:190-391
  rhs = M^-1 (S^T_quad (v u) - fluxes of (u, v, elmax |v|^2) on the face
  quadrature grid), the velocity a volume field given per call
"""

from __future__ import annotations

import weakref
from dataclasses import dataclass, field
from math import sqrt

import numpy as np

from . import flux as fl
from . import optemplate as ot
from .mesh import TAG_ALL, TAG_NONE, check_bc_coverage

# model ids shared with the C-ABI (include/hedge_b200.h)
MODEL_ADVECTION = 1
MODEL_WAVE = 2
MODEL_VARWAVE = 3
MODEL_MAXWELL = 4
MODEL_MAXWELL_TM = 5
MODEL_MAXWELL_TE = 6
MODEL_VARADV = 7

# boundary-condition kinds shared with the C-ABI
BC_NONE = 0        # face contributes no boundary flux
BC_GIVEN = 1       # ext state = caller-supplied boundary vector
BC_DIRICHLET = 2   # wave: (-u, v); var-c wave: (c, -u, v)
BC_NEUMANN = 3     # wave: (u, -v)
BC_RADIATION = 4   # wave: characteristic
BC_PEC = 5         # Maxwell: (-E, H)
BC_PMC = 6         # Maxwell: (E, -H)
BC_ABSORB = 7      # Maxwell: first-order absorbing
BC_INCIDENT = 8    # Maxwell: incident field, zero data (0, 0)


@dataclass
class OpTemplate:
    """Lowered right-hand side: the kernel model, its parameters and the
    boundary kind of each tag.  ``fields`` names the template's volume
    fields when it was lowered from a symbolic template (state, given
    boundary data, coefficient, source)."""

    model: int
    dimensions: int
    n_fields: int
    flux_type: int            # model-specific numeric code
    params: dict
    bcs: list                 # [(tag, bc_kind)], disjoint tags
    operator: object = field(repr=False, default=None)
    fields: dict = field(default_factory=dict)

    @property
    def n_flux_args(self):
        """Fields of the flux argument: the state, plus c (variable-velocity
        wave) or epsilon and mu (Maxwell with variable material)."""
        if self.params.get("variable_material"):
            return self.n_fields + 2
        return self.n_fields + (1 if self.model == MODEL_VARWAVE else 0)


# templates made by a model's op_template(): id -> (weak reference, model),
# so that compiling one binds the model's data (variable c, source vectors)
_ORIGIN = {}


def _remember(model, tree):
    key = id(tree)
    ref = weakref.ref(tree, lambda r, k=key: _ORIGIN.pop(k, None))
    _ORIGIN[key] = (ref, model)
    return tree


def template_model(tree):
    """The model whose op_template() made ``tree`` (None for a template
    built by hand)."""
    e = _ORIGIN.get(id(tree))
    return e[1] if e is not None and e[0]() is tree else None


class HyperbolicOperator:
    """Base class: time-step estimate (hedge/models/__init__.py:53-67)."""

    def estimate_timestep(self, discr, stepper=None, stepper_class=None,
                          stepper_args=None, t=None, fields=None):
        # LSRK4's relative imaginary stability region is 1
        # (hedge/timestep/stability.py:33-58)
        return (1 / self.max_eigenvalue(t, fields, discr)
                * discr.dt_non_geometric_factor()
                * discr.dt_geometric_factor())

    def bind(self, discr):
        """hedge/models/*.py bind(): coverage check, then the compiled
        template with this model's data (boundary values, c, sources)."""
        check_bc_coverage(discr.mesh, self.bc_tags())
        return discr.compile(self.op_template()).bind_model(self)


class TimeConstantGivenFunction:
    """Boundary/volume data given as f(x) (hedge/data.py)."""

    def __init__(self, f):
        self.f = f

    def boundary_interpolant(self, t, discr, tag):
        return discr.interpolate_boundary_function(self.f, tag)

    def volume_interpolant(self, t, discr):
        return discr.interpolate_volume_function(self.f, kind="numpy")


class TimeDependentGivenFunction:
    """Boundary/volume data given as f(x, t) with x an [N, d] array
    (hedge/data.py TimeDependentGivenFunction)."""

    def __init__(self, f):
        self.f = f

    def boundary_interpolant(self, t, discr, tag):
        return discr.interpolate_boundary_function(lambda x: self.f(x, t), tag)

    def volume_interpolant(self, t, discr):
        return discr.interpolate_volume_function(lambda x: self.f(x, t), kind="numpy")


def make_tdep_constant(value):
    return TimeConstantGivenFunction(lambda x, el=None: value)


# --------------------------------------------------------------------------
class StrongAdvectionOperator(HyperbolicOperator):
    flux_types = ["central", "upwind", "lf"]

    def __init__(self, v, inflow_tag="inflow", inflow_u=None,
                 outflow_tag="outflow", flux_type="central"):
        self.dimensions = len(v)
        self.v = np.asarray(v, dtype=np.float64)
        self.inflow_tag = inflow_tag
        self.inflow_u = inflow_u if inflow_u is not None else make_tdep_constant(0.0)
        self.outflow_tag = outflow_tag
        if flux_type not in self.flux_types:
            raise ValueError("invalid flux type")
        self.flux_type = flux_type

    def max_eigenvalue(self, t=None, fields=None, discr=None):
        return float(np.linalg.norm(self.v))

    def weak_flux(self):
        """advection.py:58-80"""
        u = fl.FluxScalarPlaceholder(0)
        normal = fl.make_normal(self.dimensions)
        nv = np.dot(normal, self.v)
        if self.flux_type == "central":
            return u.avg * nv
        if self.flux_type == "lf":
            return u.avg * nv + 0.5 * float(np.linalg.norm(self.v)) * (u.int - u.ext)
        return nv * fl.IfPositive(nv, u.int, u.ext)

    def flux(self):
        """advection.py:125-131"""
        u = fl.FluxScalarPlaceholder(0)
        normal = fl.make_normal(self.dimensions)
        return u.int * np.dot(normal, self.v) - self.weak_flux()

    def op_template(self, u=None, bc_in=None):
        """advection.py:133-149"""
        u = ot.Field("u") if u is None else u
        bc_in = ot.Field("bc_in") if bc_in is None else bc_in
        nabla = ot.make_nabla(self.dimensions)
        m_inv = ot.InverseMassOperator()
        flux_op = ot.get_flux_operator(self.flux())
        return _remember(self, -np.dot(self.v, nabla * u)
                         + m_inv(flux_op(u) + flux_op(ot.BoundaryPair(u, bc_in,
                                                                      self.inflow_tag))))

    def descriptor(self):
        return OpTemplate(MODEL_ADVECTION, self.dimensions, 1,
                          self.flux_types.index(self.flux_type),
                          {"v": self.v.copy()},
                          [(self.inflow_tag, BC_GIVEN),
                           (self.outflow_tag, BC_NONE)], self)

    def bc_tags(self):
        return [self.inflow_tag, self.outflow_tag]

    def context(self, discr, t, fields=None):
        return {"bc_in": self.inflow_u.boundary_interpolant(t, discr, self.inflow_tag)}


class WeakAdvectionOperator(StrongAdvectionOperator):
    """advection.py:153-187: M^-1 (v . S^T u - fluxes), the weak form with
    the weak flux and outflow data taken from the interior.  Lowered onto
    the strong-form advection kernel (summation by parts; see
    hedge_b200.lowering), hence the same descriptor."""

    def flux(self):
        return self.weak_flux()

    def op_template(self, u=None, bc_in=None):
        u = ot.Field("u") if u is None else u
        bc_in = ot.Field("bc_in") if bc_in is None else bc_in
        bc_out = ot.BoundarizeOperator(self.outflow_tag) * u
        stiff_t = ot.make_stiffness_t(self.dimensions)
        flux_op = ot.get_flux_operator(self.flux())
        return _remember(self, ot.InverseMassOperator()(
            np.dot(self.v, stiff_t * u)
            - (flux_op(u) + flux_op(ot.BoundaryPair(u, bc_in, self.inflow_tag))
               + flux_op(ot.BoundaryPair(u, bc_out, self.outflow_tag)))))


class StrongWaveOperator(HyperbolicOperator):
    def __init__(self, c, dimensions, source_f=0, flux_type="upwind",
                 dirichlet_tag=TAG_ALL, dirichlet_bc_f=0,
                 neumann_tag=TAG_NONE, radiation_tag=TAG_NONE):
        """``dirichlet_bc_f``: 0 (homogeneous Dirichlet walls), or the Dirichlet
        value g of u on ``dirichlet_tag`` (ext state (2g - u, v), wave.py:133-142):
        a TimeConstantGivenFunction / TimeDependentGivenFunction, which the
        bound RHS and the steppers evaluate on the boundary, or any other true
        value, in which case the caller passes the boundary vector as
        ``rhs(t, w, dir_bc_u=...)`` (the reference's field name)."""
        assert isinstance(dimensions, int)
        if flux_type not in ("central", "upwind"):
            raise ValueError("invalid flux type '%s'" % flux_type)
        self.dirichlet_bc_f = dirichlet_bc_f
        self.c = float(c)
        self.dimensions = dimensions
        self.source_f = source_f
        self.sign = 1 if self.c > 0 else -1
        self.dirichlet_tag = dirichlet_tag
        self.neumann_tag = neumann_tag
        self.radiation_tag = radiation_tag
        self.flux_type = flux_type

    def max_eigenvalue(self, t=None, fields=None, discr=None):
        return abs(self.c)

    def flux(self):
        """wave.py:80-108"""
        dim = self.dimensions
        w = fl.FluxVectorPlaceholder(1 + dim)
        u, v = w[0], w[1:]
        normal = fl.make_normal(dim)
        flux_weak = ot.join_fields(np.dot(v.avg, normal), u.avg * normal)
        if self.flux_type == "upwind":
            flux_weak = flux_weak - self.sign * ot.join_fields(
                0.5 * (u.int - u.ext), 0.5 * (normal * np.dot(normal, v.int - v.ext)))
        flux_strong = ot.join_fields(np.dot(v.int, normal), u.int * normal) - flux_weak
        return -self.c * flux_strong

    def op_template(self, w=None, dir_bc_u=None):
        """wave.py:110-180"""
        d = self.dimensions
        w = ot.make_sym_vector("w", d + 1) if w is None else w
        u, v = w[0], w[1:]
        B = ot.BoundarizeOperator
        if self.dirichlet_bc_f:
            g = ot.Field("dir_bc_u") if dir_bc_u is None else dir_bc_u
            dir_bc = ot.join_fields(2 * g - B(self.dirichlet_tag) * u, B(self.dirichlet_tag) * v)
        else:
            dir_bc = ot.join_fields(-(B(self.dirichlet_tag) * u), B(self.dirichlet_tag) * v)
        neu_bc = ot.join_fields(B(self.neumann_tag) * u, -(B(self.neumann_tag) * v))
        rn = ot.normal(self.radiation_tag, d)
        rad_u, rad_v = B(self.radiation_tag) * u, B(self.radiation_tag) * v
        rad_bc = ot.join_fields(0.5 * (rad_u - self.sign * np.dot(rn, rad_v)),
                                0.5 * rn * (np.dot(rn, rad_v) - self.sign * rad_u))
        nabla = ot.make_nabla(d)
        flux_op = ot.get_flux_operator(self.flux())
        result = (-ot.join_fields(-self.c * np.dot(nabla, v), -self.c * (nabla * u))
                  + ot.InverseMassOperator() * (
                      flux_op(w)
                      + flux_op(ot.BoundaryPair(w, dir_bc, self.dirichlet_tag))
                      + flux_op(ot.BoundaryPair(w, neu_bc, self.neumann_tag))
                      + flux_op(ot.BoundaryPair(w, rad_bc, self.radiation_tag))))
        result[0] = result[0] + _template_value(self.source_f, "source")
        return _remember(self, result)

    def descriptor(self):
        return OpTemplate(MODEL_WAVE, self.dimensions, self.dimensions + 1,
                          1 if self.flux_type == "upwind" else 0,
                          {"c": self.c, "source": self.source_f},
                          [(self.dirichlet_tag, BC_GIVEN if self.dirichlet_bc_f else BC_DIRICHLET),
                           (self.neumann_tag, BC_NEUMANN),
                           (self.radiation_tag, BC_RADIATION)], self)

    def bc_tags(self):
        return [self.dirichlet_tag, self.neumann_tag, self.radiation_tag]

    def context(self, discr, t, fields=None):
        """Boundary data of the bound RHS at time t (Dirichlet values given
        as a function); empty when the caller supplies dir_bc_u."""
        f = self.dirichlet_bc_f
        if f and hasattr(f, "boundary_interpolant"):
            return {"bc_in": f.boundary_interpolant(t, discr, self.dirichlet_tag)}
        return {}


class VariableVelocityStrongWaveOperator(HyperbolicOperator):
    """``c`` is a volume field (array of length len(discr)) or a number;
    ``source`` a volume field or 0."""

    def __init__(self, c, dimensions, source=0, flux_type="upwind",
                 dirichlet_tag=TAG_ALL, neumann_tag=TAG_NONE,
                 radiation_tag=TAG_NONE, time_sign=1, diffusion_coeff=None):
        assert isinstance(dimensions, int)
        if flux_type not in ("central", "upwind"):
            raise ValueError("invalid flux type '%s'" % flux_type)
        if diffusion_coeff:
            raise NotImplementedError("artificial diffusion is not on this path")
        self.c = c
        self.dimensions = dimensions
        self.source = source
        self.time_sign = time_sign
        self.dirichlet_tag = dirichlet_tag
        self.neumann_tag = neumann_tag
        self.radiation_tag = radiation_tag
        self.flux_type = flux_type

    def max_eigenvalue(self, t=None, fields=None, discr=None):
        return float(np.max(np.abs(np.asarray(_to_numpy(self.c)))))

    def flux(self):
        """wave.py:246-273"""
        dim = self.dimensions
        w = fl.FluxVectorPlaceholder(2 + dim)
        c, u, v = w[0], w[1], w[2:]
        normal = fl.make_normal(dim)
        flux = self.time_sign * 0.5 * ot.join_fields(
            c.ext * np.dot(v.ext, normal) - c.int * np.dot(v.int, normal),
            normal * (c.ext * u.ext - c.int * u.int))
        if self.flux_type == "upwind":
            flux = flux + ot.join_fields(
                c.ext * u.ext - c.int * u.int,
                c.ext * normal * np.dot(normal, v.ext) - c.int * normal * np.dot(normal, v.int))
        return flux

    def op_template(self, w=None):
        """wave.py:287-395 without artificial diffusion; a numeric or array
        ``c`` (``source``) enters as the field "c" ("source")."""
        d = self.dimensions
        w = ot.make_sym_vector("w", d + 1) if w is None else w
        u, v = w[0], w[1:]
        c = _template_value(self.c, "c")
        flux_w = ot.join_fields(c, w)
        B = ot.BoundarizeOperator
        dt_, nt_, rt_ = self.dirichlet_tag, self.neumann_tag, self.radiation_tag
        dir_bc = ot.join_fields(B(dt_) * c, -(B(dt_) * u), B(dt_) * v)
        neu_bc = ot.join_fields(B(nt_) * c, B(nt_) * u, -(B(nt_) * v))
        rn = ot.normal(rt_, d)
        rad_u, rad_v = B(rt_) * u, B(rt_) * v
        rad_bc = ot.join_fields(B(rt_) * c,
                                0.5 * (rad_u - self.time_sign * np.dot(rn, rad_v)),
                                0.5 * rn * (np.dot(rn, rad_v) - self.time_sign * rad_u))
        nabla = ot.make_nabla(d)
        flux_op = ot.get_flux_operator(self.flux())
        src = _template_value(self.source, "source")
        return _remember(self, -ot.join_fields(-self.time_sign * c * np.dot(nabla, v) + src,
                                               -self.time_sign * c * (nabla * u))
                         + ot.InverseMassOperator() * (
                             flux_op(flux_w)
                             + flux_op(ot.BoundaryPair(flux_w, dir_bc, dt_))
                             + flux_op(ot.BoundaryPair(flux_w, neu_bc, nt_))
                             + flux_op(ot.BoundaryPair(flux_w, rad_bc, rt_))))

    def descriptor(self):
        return OpTemplate(MODEL_VARWAVE, self.dimensions, self.dimensions + 1,
                          1 if self.flux_type == "upwind" else 0,
                          {"time_sign": float(self.time_sign)},
                          [(self.dirichlet_tag, BC_DIRICHLET),
                           (self.neumann_tag, BC_NEUMANN),
                           (self.radiation_tag, BC_RADIATION)], self)

    def bc_tags(self):
        return [self.dirichlet_tag, self.neumann_tag, self.radiation_tag]


class MaxwellOperator(HyperbolicOperator):
    """Maxwell's equations, isotropic non-dispersive material (em.py:38-387):
    the full 3D system, field order [Ex Ey Ez Hx Hy Hz]; the subclasses carry
    a subset of the components (get_eh_subset) in 2D, the fields not carried
    and all z derivatives (and normal z components) being zero.

    ``epsilon`` and ``mu`` are numbers (fixed material) or, for spatially
    variable material, volume fields: given functions
    (TimeConstantGivenFunction, ``volume_interpolant(t, discr)``), callables
    f(x) of the node coordinates, volume vectors [K*Np], or template fields.
    Variable material runs on the CUDA-core kernels (fp64, fp32)."""

    _default_dimensions = 3
    model_id = MODEL_MAXWELL

    def __init__(self, epsilon, mu, flux_type, bdry_flux_type=None,
                 pec_tag=TAG_ALL, pmc_tag=TAG_NONE, absorb_tag=TAG_NONE,
                 incident_tag=TAG_NONE, incident_bc=lambda maxwell_op, e, h: 0,
                 current=0, dimensions=None):
        """``current``: the source current J of em.py:192-214 (the E equations
        read eps dE/dt = curl H - J) over the carried E components: 0,
        numbers, a volume field [n_E, K*Np] (array, tensor or vectors), or a
        template vector.

        ``incident_tag`` / ``incident_bc``: the incident-field boundary of
        em.py:289-307, whose exterior state is -incident_bc(op, e, h).  The
        reference's default incident_bc (zero) gives a zero exterior state
        (every kernel); incident data given per call as boundary vectors
        (template fields outside any BoundarizeOperator, one per carried
        component, e.g. ``make_sym_vector("inc", n_fields)``) runs on the
        CUDA-core kernels."""
        self.dimensions = dimensions or self._default_dimensions
        if self.dimensions != self._default_dimensions:
            raise NotImplementedError("%s is a %dD system" % (type(self).__name__,
                                                             self._default_dimensions))
        self.fixed_material = bool(np.isscalar(epsilon) and np.isscalar(mu))
        self.current = current
        self.incident_bc_data = incident_bc
        self.incident_data = None     # [n_fields] template terms, or None (zero)
        if incident_tag is not TAG_NONE:
            e, h = self.split_eh(ot.make_sym_vector("w", self.n_fields))
            data = incident_bc(self, e, h)
            if not ot.is_zero(data):
                arr = np.asarray(data, dtype=object).reshape(-1)
                if len(arr) != self.n_fields:
                    raise ValueError("incident data: %d components, one per carried field"
                                     % self.n_fields)
                if not all(ot.is_zero(x) for x in arr):
                    self.incident_data = arr
        if self.fixed_material:
            self.epsilon, self.mu = float(epsilon), float(mu)
        else:
            self.epsilon, self.mu = epsilon, mu
        self.flux_type = flux_type
        self.bdry_flux_type = flux_type if bdry_flux_type is None else bdry_flux_type
        for ft in (self.flux_type, self.bdry_flux_type):
            if not (ft == "lf" or isinstance(ft, (int, float))):
                raise ValueError("maxwell: invalid flux_type (%s)" % ft)
        self.pec_tag, self.pmc_tag = pec_tag, pmc_tag
        self.absorb_tag, self.incident_tag = absorb_tag, incident_tag

    @property
    def c(self):
        if not self.fixed_material:
            raise RuntimeError("Cannot compute speed of light for non-constant material")
        return 1 / sqrt(self.mu * self.epsilon)

    def material_templates(self):
        """(epsilon, mu) as they enter the template: numbers (fixed
        material) or template fields ("epsilon", "mu" unless given as
        fields)."""
        if self.fixed_material:
            return self.epsilon, self.mu
        e = self.epsilon if isinstance(self.epsilon, ot.Expr) else ot.Field("epsilon")
        m = self.mu if isinstance(self.mu, ot.Expr) else ot.Field("mu")
        return e, m

    def material_values(self, discr):
        """(epsilon, mu) at the nodes of ``discr``, two numpy vectors [K*Np]
        (None for a material given as a template field)."""
        def vals(x):
            if isinstance(x, ot.Expr):
                return None
            if np.isscalar(x):
                return np.full(len(discr), float(x))
            if hasattr(x, "volume_interpolant"):
                return np.asarray(_to_numpy(x.volume_interpolant(0.0, discr)),
                                  dtype=np.float64).reshape(-1)
            if callable(x):
                return np.asarray(discr.interpolate_volume_function(x, kind="numpy"),
                                  dtype=np.float64).reshape(-1)
            return np.asarray(_to_numpy(x), dtype=np.float64).reshape(-1)
        return vals(self.epsilon), vals(self.mu)

    def get_eh_subset(self):
        """em.py: which of (Ex, Ey, Ez, Hx, Hy, Hz) the operator carries."""
        return (True,) * 6

    @property
    def _slots(self):
        return [i for i, on in enumerate(self.get_eh_subset()) if on]

    @property
    def n_e(self):
        """Number of carried E components (they come first)."""
        return sum(self.get_eh_subset()[:3])

    @property
    def n_fields(self):
        return len(self._slots)

    def split_eh(self, w):
        """(E, H) of a field vector [n_fields, ...] (carried components)."""
        return w[0:self.n_e], w[self.n_e:self.n_fields]

    def assemble_eh(self, e, h):
        import torch
        ne, nh = self.n_e, self.n_fields - self.n_e
        if isinstance(e, torch.Tensor):
            return torch.cat([e.reshape(ne, -1), h.reshape(nh, -1)])
        return np.concatenate([np.asarray(e).reshape(ne, -1), np.asarray(h).reshape(nh, -1)])

    def _embed(self, w):
        """The 6 components (Ex .. Hz) of a carried-field vector, zeros elsewhere."""
        full = np.array([0] * 6, dtype=object)
        for k, slot in enumerate(self._slots):
            full[slot] = w[k]
        return full

    def _pick(self, full):
        return np.array([full[slot] for slot in self._slots], dtype=object)

    @staticmethod
    def _pad3(x):
        return np.array(list(x) + [0] * (3 - len(x)), dtype=object)

    def max_eigenvalue(self, t=None, fields=None, discr=None):
        """1/sqrt(eps mu) (em.py:466-482).  Variable material: the reference
        raises here (use max_eigenvalue_expr); with ``discr`` this evaluates
        that expression, the nodal maximum of 1/sqrt(eps mu), instead."""
        if self.fixed_material:
            return 1 / sqrt(self.epsilon * self.mu)
        if discr is None:
            raise ValueError("max_eigenvalue of variable material needs the discretization")
        e, m = self.material_values(discr)
        if e is None or m is None:
            raise ValueError("material given as template fields: no values to evaluate")
        return float(np.max(1.0 / np.sqrt(e * m)))

    def estimate_timestep(self, discr, stepper=None, stepper_class=None,
                          stepper_args=None, t=None, fields=None):
        return (1 / self.max_eigenvalue(t, fields, discr)
                * discr.dt_non_geometric_factor() * discr.dt_geometric_factor())

    def flux(self, flux_type):
        """em.py:118-190: fixed material (constants), or variable material
        (the flux argument carries epsilon and mu first)."""
        normal = self._pad3(fl.make_normal(self.dimensions))
        if self.fixed_material:
            w = fl.FluxVectorPlaceholder(self.n_fields)
            epsilon = fl.FluxConstantPlaceholder(self.epsilon)
            mu = fl.FluxConstantPlaceholder(self.mu)
            fw = [w[k] for k in range(self.n_fields)]
        else:
            w = fl.FluxVectorPlaceholder(2 + self.n_fields)
            epsilon, mu = w[0], w[1]
            fw = [w[2 + k] for k in range(self.n_fields)]
        wi = self._embed([x.int for x in fw])
        we = self._embed([x.ext for x in fw])
        Z_int = (mu.int / epsilon.int) ** 0.5
        Y_int = 1 / Z_int
        Z_ext = (mu.ext / epsilon.ext) ** 0.5
        Y_ext = 1 / Z_ext
        de, dh = wi[0:3] - we[0:3], wi[3:6] - we[3:6]
        if flux_type == "lf":
            full = ot.join_fields(0.5 * -ot.cross(normal, dh), 0.5 * ot.cross(normal, de))
        else:
            full = ot.join_fields(
                -1 / (Z_int + Z_ext) * ot.cross(normal, Z_ext * dh - flux_type * ot.cross(normal, de)),
                1 / (Y_int + Y_ext) * ot.cross(normal, Y_ext * de + flux_type * ot.cross(normal, dh)))
        return self._pick(full)

    def current_template(self):
        """The current over the carried E components as template terms: 0,
        numbers, or the components of the volume field ``current``."""
        ne = self.n_e
        j = self.current
        if isinstance(j, np.ndarray) and j.dtype == object:
            return j
        if np.isscalar(j):
            return 0 if j == 0 else np.array([float(j)] * ne, dtype=object)
        a = _to_numpy(j)
        if isinstance(a, (list, tuple)) and len(a) == ne and all(np.isscalar(x) for x in a):
            return np.array([float(x) if x != 0 else 0 for x in a], dtype=object)
        return ot.make_sym_vector("current", ne)

    def current_value(self):
        """The current's volume values [n_E, K*Np] (or numbers) for binding."""
        j = self.current
        if isinstance(j, (list, tuple)) and not all(np.isscalar(x) for x in j):
            return np.stack([np.asarray(_to_numpy(x), dtype=np.float64).reshape(-1) for x in j])
        return _to_numpy(j)

    def local_derivatives(self, w):
        """em.py:192-214: (current - curl H, curl E), over the carried components"""
        full = self._embed(w)
        e, h = full[0:3], full[3:6]
        nabla = self._pad3(ot.make_nabla(self.dimensions))
        cur = self.current_template()
        j = np.array([0] * 3, dtype=object)
        if not (np.isscalar(cur) and cur == 0):
            for k, slot in enumerate(self._slots[:self.n_e]):
                j[slot] = cur[k]
        return self._pick(ot.join_fields(j - ot.cross(nabla, h), ot.cross(nabla, e)))

    def op_template(self, w=None):
        """em.py:226-371: (-local derivatives + M^-1 (fluxes)) / material
        divisor; with variable material the flux argument is
        (epsilon, mu, w) and every boundary vector (B(eps), B(mu), bc)."""
        F = self.n_fields
        w = ot.make_sym_vector("w", F) if w is None else w
        B = ot.BoundarizeOperator
        eps, mu = self.material_templates()

        def bfull(tag):
            return self._embed([B(tag) * w[k] for k in range(F)])
        pe = bfull(self.pec_tag)
        pec = self._pick(ot.join_fields(-pe[0:3], pe[3:6]))
        pm = bfull(self.pmc_tag)
        pmc = self._pick(ot.join_fields(pm[0:3], -pm[3:6]))
        an = self._pad3(ot.normal(self.absorb_tag, self.dimensions))
        if self.fixed_material:
            Z = (self.mu / self.epsilon) ** 0.5
        else:
            Z = (B(self.absorb_tag) * mu / (B(self.absorb_tag) * eps)) ** 0.5
        ab = bfull(self.absorb_tag)
        ae, ah = ab[0:3], ab[3:6]
        absorb = self._pick(ot.join_fields(
            ae + 0.5 * (ot.cross(an, ot.cross(an, ae)) - Z * ot.cross(an, ah)),
            ah + 0.5 * (ot.cross(an, ot.cross(an, ah)) + (1 / Z) * ot.cross(an, ae))))
        flux_op = ot.get_flux_operator(self.flux(self.flux_type))
        bdry_flux_op = ot.get_flux_operator(self.flux(self.bdry_flux_type))
        divisor = np.array([eps] * self.n_e + [mu] * (F - self.n_e), dtype=object)
        if self.fixed_material:
            flux_w = w

            def bvec(tag, bc):
                return bc
        else:
            flux_w = ot.join_fields(eps, mu, w)

            def bvec(tag, bc):
                return ot.join_fields(B(tag) * eps, B(tag) * mu, bc)
        # incident boundary: the exterior state is -(incident data)
        # (em.py:289-307)
        incident = np.array([0] * F, dtype=object) if self.incident_data is None else \
            np.array([-x for x in self.incident_data], dtype=object)
        bdry = sum(bdry_flux_op(ot.BoundaryPair(flux_w, bvec(tag, bc), tag)) for tag, bc in
                   [(self.pec_tag, pec), (self.pmc_tag, pmc), (self.absorb_tag, absorb),
                    (self.incident_tag, incident)])
        return _remember(self, (-self.local_derivatives(w)
                                + ot.InverseMassOperator()(flux_op(flux_w) + bdry)) / divisor)

    def descriptor(self):
        def code(ft):
            return (1, 0.0) if ft == "lf" else (0, float(ft))
        ft, alpha = code(self.flux_type)
        bft, balpha = code(self.bdry_flux_type)
        eps, mu = (self.epsilon, self.mu) if self.fixed_material else (1.0, 1.0)
        params = {"eps": eps, "mu": mu, "alpha": alpha,
                  "bdry_flux_type": bft, "bdry_alpha": balpha}
        if not self.fixed_material:
            params["variable_material"] = True
        if self.incident_data is not None and self.incident_tag is not TAG_NONE:
            params["incident_data"] = True
        return OpTemplate(self.model_id, self.dimensions, self.n_fields, ft, params,
                          [(self.pec_tag, BC_PEC), (self.pmc_tag, BC_PMC),
                           (self.absorb_tag, BC_ABSORB),
                           (self.incident_tag, BC_INCIDENT)], self)

    def bc_tags(self):
        return [self.pec_tag, self.absorb_tag, self.incident_tag]


class TMMaxwellOperator(MaxwellOperator):
    """2D TM Maxwell (em.py:485-498), field order [Ez Hx Hy]."""

    _default_dimensions = 2
    model_id = MODEL_MAXWELL_TM

    def get_eh_subset(self):
        return (False, False, True) + (True, True, False)


class TEMaxwellOperator(MaxwellOperator):
    """2D TE Maxwell (em.py:501-515), field order [Ex Ey Hz]."""

    _default_dimensions = 2
    model_id = MODEL_MAXWELL_TE

    def get_eh_subset(self):
        return (True, True, False) + (False, False, True)


class VariableCoefficientAdvectionOperator(HyperbolicOperator):
    """Space- and time-dependent advection in weak form with over-integration
    (advection.py:190-391): the velocity ``advec_v`` is a given function
    (``volume_interpolant(t, discr)`` -> [d, K*Np]), ``bc_u_f`` the inflow
    data on every boundary face (``"None"``: zero).  The volume and face
    integrals are taken on the quadrature grid "quad" of the
    discretization's ``quad_min_degrees`` (nodal evaluation when it has no
    degree for "quad", as the reference falls back to).  Diffusion
    (second-order terms) is not on this path."""

    flux_types = ["central", "upwind", "lf"]

    def __init__(self, dimensions, advec_v, bc_u_f="None", flux_type="central",
                 diffusion_coeff=None, diffusion_scheme=None):
        if flux_type not in self.flux_types:
            raise ValueError("invalid flux type")
        if diffusion_coeff is not None and diffusion_coeff != 0:
            raise NotImplementedError("diffusion (second-order terms) is not on this path")
        self.dimensions = int(dimensions)
        self.advec_v = advec_v
        self.bc_u_f = bc_u_f
        self.flux_type = flux_type
        self.diffusion_coeff = diffusion_coeff

    def _has_bc(self):
        return not (isinstance(self.bc_u_f, str) and self.bc_u_f == "None")

    def flux(self):
        """advection.py:224-266, w = (u, v, c)."""
        d = self.dimensions
        w = fl.FluxVectorPlaceholder(1 + d + 1)
        u, v, c = w[0], w[1:d + 1], w[1 + d]
        normal = fl.make_normal(d)
        if self.flux_type == "central":
            return (u.int * np.dot(v.int, normal) + u.ext * np.dot(v.ext, normal)) * 0.5
        if self.flux_type == "lf":
            n_vint = np.dot(normal, v.int)
            n_vext = np.dot(normal, v.ext)
            return 0.5 * (n_vint * u.int + n_vext * u.ext) \
                - 0.5 * (u.ext - u.int) * fl.flux_max(c.int, c.ext)
        return fl.IfPositive(np.dot(normal, v.avg),
                             np.dot(normal, v.int) * u.int,
                             np.dot(normal, v.ext) * u.ext)

    def op_template(self, u=None, v=None, bc_u=None, with_sensor=False):
        """advection.py:282-368 without the diffusion part."""
        if with_sensor:
            raise NotImplementedError("diffusion (second-order terms) is not on this path")
        d = self.dimensions
        u = ot.Field("u") if u is None else u
        v = ot.make_sym_vector("v", d) if v is None else v
        c = ot.ElementwiseMaxOperator()(ot.ptwise_dot(1, 1, v, v))
        to_quad = ot.QuadratureGridUpsampler("quad")
        to_if_quad = ot.QuadratureInteriorFacesGridUpsampler("quad")
        quad_u = to_quad(u)
        quad_v = to_quad(v)
        w = ot.join_fields(u, v, c)
        quad_face_w = to_if_quad(w)
        bc_c = to_quad(ot.BoundarizeOperator(TAG_ALL)(c))
        bc_v = to_quad(ot.BoundarizeOperator(TAG_ALL)(v))
        if self._has_bc():
            bc_w = ot.join_fields(to_quad(ot.Field("bc_u") if bc_u is None else bc_u),
                                  bc_v, bc_c)
        else:
            bc_w = ot.join_fields(0, bc_v, bc_c)
        minv_st = ot.make_stiffness_t(d)
        m_inv = ot.InverseMassOperator()
        flux_op = ot.get_flux_operator(self.flux())
        return _remember(self, m_inv(
            np.dot(minv_st, quad_v * quad_u)
            - (flux_op(quad_face_w) + flux_op(ot.BoundaryPair(quad_face_w, bc_w, TAG_ALL)))))

    def descriptor(self):
        return OpTemplate(MODEL_VARADV, self.dimensions, 1,
                          self.flux_types.index(self.flux_type), {"quad_tag": "quad"},
                          [(TAG_ALL, BC_GIVEN if self._has_bc() else BC_DIRICHLET)], self,
                          {"state": "u", "coeff": "v", "given": "bc_u" if self._has_bc()
                           else None})

    def bc_tags(self):
        return [TAG_ALL]

    def context(self, discr, t, fields=None):
        """The velocity at time t as the device coefficient [d * K*Np] (FP64;
        computed once for a time-constant velocity) and the inflow data."""
        if isinstance(self.advec_v, TimeConstantGivenFunction):
            cache = self.__dict__.setdefault("_v_dev", {})
            if id(discr) not in cache:
                cache.clear()
                cache[id(discr)] = self._velocity(discr, t)
            v = cache[id(discr)]
        else:
            v = self._velocity(discr, t)
        ctx = {"coeff": v}
        if self._has_bc():
            ctx["bc_in"] = self.bc_u_f.boundary_interpolant(t, discr, TAG_ALL)
        return ctx

    def _velocity(self, discr, t):
        import torch
        v = self.advec_v.volume_interpolant(t, discr)
        return discr.to_device(v, torch.float64).reshape(-1).contiguous()

    def max_eigenvalue(self, t=None, fields=None, discr=None):
        """advection.py:381-391: the largest nodal |v|."""
        v = np.asarray(_to_numpy(self.advec_v.volume_interpolant(t, discr)), dtype=np.float64)
        return float(np.sqrt(np.max(np.sum(v.reshape(self.dimensions, -1) ** 2, axis=0))))


def _template_value(x, name):
    """A model datum as a template term: expressions and numbers as they
    are, volume vectors as the field ``name`` (bound when the model binds)."""
    if isinstance(x, ot.Expr):
        return x
    if np.isscalar(x):
        return float(x) if x != 0 else 0
    return ot.Field(name)


def _to_numpy(x):
    try:
        import torch
        if isinstance(x, torch.Tensor):
            return x.detach().cpu().numpy()
    except ImportError:   # pragma: no cover
        pass
    return x


__all__ = ["template_model", "StrongAdvectionOperator", "WeakAdvectionOperator", "StrongWaveOperator",
           "VariableVelocityStrongWaveOperator", "MaxwellOperator", "TMMaxwellOperator",
           "TEMaxwellOperator", "VariableCoefficientAdvectionOperator",
           "OpTemplate", "make_tdep_constant", "TimeConstantGivenFunction",
           "TimeDependentGivenFunction",
           "check_bc_coverage"]
