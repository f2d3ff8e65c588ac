"""Hyperbolic DG operators: advection, wave, variable-velocity wave, Maxwell.

Constructor signatures and ``bind(discr) -> rhs(t, w)`` mirror the
reference's models.  pymbolic (the reference's op-template language) is not
available, so ``op_template()`` returns an :class:`OpTemplate` descriptor of
the same right-hand side instead of a symbolic tree:

* StrongAdvectionOperator  hedge/models/advection.py:124-149
  rhs = -v.grad u + M^-1 (flux(u) + flux(BoundaryPair(u, bc_in, inflow)))
* StrongWaveOperator       hedge/models/wave.py:37-197
  rhs = (c div v, c grad u) + M^-1 (fluxes) [+ source on u]
* VariableVelocityStrongWaveOperator  hedge/models/wave.py:204-418
  rhs = (ts c div v - source, ts c grad u) + M^-1 (fluxes of (c, u, v))
* MaxwellOperator          hedge/models/em.py:38-387 (fixed material)
  rhs = ((curl H - J) , -curl E) + M^-1 (fluxes)) / (eps | mu)
"""

from __future__ import annotations

from dataclasses import dataclass, field
from math import sqrt

import numpy as np

from .mesh import TAG_ALL, TAG_NONE, check_bc_coverage

# model ids shared with the C-ABI (include/hedge_b200.h)
MODEL_ADVECTION = 1
MODEL_WAVE = 2
MODEL_VARWAVE = 3
MODEL_MAXWELL = 4

# boundary-condition kinds shared with the C-ABI
BC_NONE = 0        # face contributes no boundary flux
BC_GIVEN = 1       # ext state = caller-supplied boundary vector
BC_DIRICHLET = 2   # wave: (-u, v); var-c wave: (c, -u, v)
BC_NEUMANN = 3     # wave: (u, -v)
BC_RADIATION = 4   # wave: characteristic
BC_PEC = 5         # Maxwell: (-E, H)
BC_PMC = 6         # Maxwell: (E, -H)
BC_ABSORB = 7      # Maxwell: first-order absorbing


@dataclass
class OpTemplate:
    """Typed description of a model's right-hand side."""

    model: int
    dimensions: int
    n_fields: int
    flux_type: int            # model-specific numeric code
    params: dict
    bcs: list                 # [(tag, bc_kind)], disjoint tags
    operator: object = field(repr=False, default=None)

    @property
    def n_flux_args(self):
        return self.n_fields + (1 if self.model == MODEL_VARWAVE else 0)


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
        return discr.compile(self.op_template()).bind_model(self)


class TimeConstantGivenFunction:
    """Boundary/volume data given as f(x) (hedge/data.py)."""

    def __init__(self, f):
        self.f = f

    def boundary_interpolant(self, t, discr, tag):
        return discr.interpolate_boundary_function(self.f, tag)


class TimeDependentGivenFunction:
    """Boundary/volume data given as f(x, t) with x an [N, d] array
    (hedge/data.py TimeDependentGivenFunction)."""

    def __init__(self, f):
        self.f = f

    def boundary_interpolant(self, t, discr, tag):
        return discr.interpolate_boundary_function(lambda x: self.f(x, t), tag)

    def volume_interpolant(self, t, discr):
        return discr.interpolate_volume_function(lambda x: self.f(x, t))


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

    def op_template(self):
        return OpTemplate(MODEL_ADVECTION, self.dimensions, 1,
                          self.flux_types.index(self.flux_type),
                          {"v": self.v.copy()},
                          [(self.inflow_tag, BC_GIVEN),
                           (self.outflow_tag, BC_NONE)], self)

    def bc_tags(self):
        return [self.inflow_tag, self.outflow_tag]

    def context(self, discr, t, fields):
        return {"bc_in": self.inflow_u.boundary_interpolant(t, discr, self.inflow_tag)}


class StrongWaveOperator(HyperbolicOperator):
    def __init__(self, c, dimensions, source_f=0, flux_type="upwind",
                 dirichlet_tag=TAG_ALL, dirichlet_bc_f=0,
                 neumann_tag=TAG_NONE, radiation_tag=TAG_NONE):
        assert isinstance(dimensions, int)
        if flux_type not in ("central", "upwind"):
            raise ValueError("invalid flux type '%s'" % flux_type)
        if dirichlet_bc_f:
            raise NotImplementedError("inhomogeneous Dirichlet data")
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

    def op_template(self):
        return OpTemplate(MODEL_WAVE, self.dimensions, self.dimensions + 1,
                          1 if self.flux_type == "upwind" else 0,
                          {"c": self.c, "source": self.source_f},
                          [(self.dirichlet_tag, BC_DIRICHLET),
                           (self.neumann_tag, BC_NEUMANN),
                           (self.radiation_tag, BC_RADIATION)], self)

    def bc_tags(self):
        return [self.dirichlet_tag, self.neumann_tag, self.radiation_tag]


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

    def op_template(self):
        return OpTemplate(MODEL_VARWAVE, self.dimensions, self.dimensions + 1,
                          1 if self.flux_type == "upwind" else 0,
                          {"time_sign": float(self.time_sign)},
                          [(self.dirichlet_tag, BC_DIRICHLET),
                           (self.neumann_tag, BC_NEUMANN),
                           (self.radiation_tag, BC_RADIATION)], self)

    def bc_tags(self):
        return [self.dirichlet_tag, self.neumann_tag, self.radiation_tag]


class MaxwellOperator(HyperbolicOperator):
    """3D Maxwell, fixed isotropic material, field order [Ex Ey Ez Hx Hy Hz]."""

    def __init__(self, epsilon, mu, flux_type, bdry_flux_type=None,
                 pec_tag=TAG_ALL, pmc_tag=TAG_NONE, absorb_tag=TAG_NONE,
                 incident_tag=TAG_NONE, current=0, dimensions=None):
        self.dimensions = dimensions or 3
        if self.dimensions != 3:
            raise NotImplementedError("only the full 3D Maxwell system")
        if not (np.isscalar(epsilon) and np.isscalar(mu)):
            raise NotImplementedError("only fixed material")
        if current != 0:
            raise NotImplementedError("source currents are not on this path")
        self.epsilon, self.mu = float(epsilon), float(mu)
        self.flux_type = flux_type
        self.bdry_flux_type = flux_type if bdry_flux_type is None else bdry_flux_type
        for ft in (self.flux_type, self.bdry_flux_type):
            if not (ft == "lf" or isinstance(ft, (int, float))):
                raise ValueError("maxwell: invalid flux_type (%s)" % ft)
        self.pec_tag, self.pmc_tag = pec_tag, pmc_tag
        self.absorb_tag, self.incident_tag = absorb_tag, incident_tag

    @property
    def c(self):
        return 1 / sqrt(self.mu * self.epsilon)

    def max_eigenvalue(self, t=None, fields=None, discr=None):
        return 1 / sqrt(self.epsilon * self.mu)

    def op_template(self):
        def code(ft):
            return (1, 0.0) if ft == "lf" else (0, float(ft))
        ft, alpha = code(self.flux_type)
        bft, balpha = code(self.bdry_flux_type)
        return OpTemplate(MODEL_MAXWELL, 3, 6, ft,
                          {"eps": self.epsilon, "mu": self.mu, "alpha": alpha,
                           "bdry_flux_type": bft, "bdry_alpha": balpha},
                          [(self.pec_tag, BC_PEC), (self.pmc_tag, BC_PMC),
                           (self.absorb_tag, BC_ABSORB),
                           (self.incident_tag, BC_NONE)], self)

    def bc_tags(self):
        return [self.pec_tag, self.absorb_tag, self.incident_tag]


def _to_numpy(x):
    try:
        import torch
        if isinstance(x, torch.Tensor):
            return x.detach().cpu().numpy()
    except ImportError:   # pragma: no cover
        pass
    return x


__all__ = ["StrongAdvectionOperator", "StrongWaveOperator",
           "VariableVelocityStrongWaveOperator", "MaxwellOperator",
           "OpTemplate", "make_tdep_constant", "TimeConstantGivenFunction",
           "TimeDependentGivenFunction",
           "check_bc_coverage"]
