"""Lowering of symbolic operator templates onto the fused kernels.

The reference compiles an op template into instructions (diff batches, flux
batches, vector expressions; hedge/optemplate/tools.py:255-326 and
hedge/compiler.py:547-1103) and runs them one by one.  Here the kernels are
fused per model, so compiling a template means recognising which kernel
model, with which parameters and which boundary condition on each tag, it
is equal to.  ``lower(template)`` does that in four steps:

1. structure: flux operators appear only inside one inverse mass, the
   inverse mass holds nothing but fluxes, derivatives act on fields only,
   and every operator is one the path supports (else ``NotImplementedError``);
2. roles: the interior flux argument names the state fields (differentiated)
   and at most one coefficient field (not differentiated, first); fields in
   boundary data outside ``BoundarizeOperator`` are given boundary data;
   remaining fields outside the fluxes are sources;
3. parameters: the template is evaluated pointwise on probe values, with each
   derivative, interior / exterior value and face normal an independent
   random number (the inverse mass and the lift act on every flux term
   alike, so they drop out).  Unit derivative probes give the volume
   coefficients, from which the model's parameters follow (advection
   velocity, wave speed, time sign, permittivity and permeability);
4. verification: the model's own template with those parameters (and each
   candidate flux type / boundary kind) is evaluated on the same probes, in
   the volume, on interior faces and on each boundary tag's faces.  The first
   candidate that agrees everywhere to rounding gives the lowered
   :class:`~hedge_b200.models.OpTemplate`.

Two rewrites come first.  Weak-form derivatives: inside the inverse mass,
``S_x^T f`` (the weak derivative, int f d(phi)/dx) becomes
``-M D_x f + int_faces n_x f.int phi``, so that ``M^-1 S_x^T f`` is
``-D_x f + M^-1 (flux n_x f.int on every face)``.  That is summation by
parts, which the nodal mass, stiffness and face-mass matrices satisfy
exactly on affine simplices, so weak-form templates (the reference's
WeakAdvectionOperator) run on the strong-form kernels.  Over-integration:
the quadrature up-samplers and the quadrature stiffness operator are
dropped when every integrand they feed is a polynomial of degree <= 2N
(state fields with constant coefficients, flux coefficients constant per
face), which the nodal operators integrate exactly; a template with a
coefficient field under a quadrature operator is refused.

Templates that integrate a product of fields by quadrature (a coefficient
field under an up-sampler or a quadrature stiffness operator, or an element
maximum) go to the quadrature kernel instead: they must equal the
variable-coefficient advection template (advection.py:282-368) built from
the same fields, for one of its flux types and with or without given inflow
data.  The comparison evaluates both templates on the same probes, with the
up-samplers as identities (their operands' values at a point are the same
polynomial's), each weak derivative S_x^T a random factor per axis times its
integrand, and the element maximum a fixed non-linear function of its
operand.

A template that no kernel model reproduces raises ``NotImplementedError``
naming the part that differs.
"""

from __future__ import annotations

import numbers
import zlib

import numpy as np

from . import flux as fl
from . import optemplate as ot
from .mesh import TAG_ALL, TAG_NONE
from .models import (BC_ABSORB, BC_DIRICHLET, BC_GIVEN, BC_INCIDENT, BC_NEUMANN, BC_NONE,
                     BC_PEC, BC_PMC, BC_RADIATION, MODEL_ADVECTION, MODEL_MAXWELL, MODEL_MAXWELL_TE,
                     MODEL_MAXWELL_TM, MODEL_VARADV, MODEL_VARWAVE, MODEL_WAVE,
                     MaxwellOperator, TEMaxwellOperator, TMMaxwellOperator, OpTemplate,
                     StrongAdvectionOperator, StrongWaveOperator,
                     VariableCoefficientAdvectionOperator, VariableVelocityStrongWaveOperator)

PROBES = 16
TOL = 1e-10


def _is_num(x):
    return isinstance(x, numbers.Number) and not isinstance(x, bool)


def _comps(x):
    if isinstance(x, np.ndarray):
        return list(x.reshape(-1))
    if isinstance(x, (list, tuple)):
        return list(x)
    return [x]


# --------------------------------------------------------------------------
# structure and roles

class _Scan:
    """One pass over a template: checks the structure and records the
    interior flux arguments, boundary pairs and field roles."""

    def __init__(self):
        self.interior_args = []
        self.pairs = []
        self.diff_keys = []
        self.outside_fields = {}    # fields outside any flux argument
        self.given_fields = {}      # fields in boundary data, not boundarized
        self.flux_fields = {}

    def run(self, outs):
        for x in outs:
            self._visit(x, in_minv=False, in_flux=False, in_bnd=False)

    def _visit(self, x, in_minv, in_flux, in_bnd, in_bfield=False):
        if _is_num(x):
            return
        if isinstance(x, np.ndarray):
            for c in x.reshape(-1):
                self._visit(c, in_minv, in_flux, in_bnd, in_bfield)
            return
        if isinstance(x, ot.Field):
            if in_minv and not in_flux:
                raise NotImplementedError(
                    "inverse mass of a volume term (%s): only fluxes are lifted" % x)
            if in_flux:
                self.flux_fields[x.key] = x
                if in_bfield and not in_bnd:
                    self.given_fields[x.key] = x
            else:
                self.outside_fields[x.key] = x
            return
        if isinstance(x, (ot.Sum, ot.Product)):
            for c in x.children:
                self._visit(c, in_minv, in_flux, in_bnd, in_bfield)
            return
        if isinstance(x, ot.Quotient):
            self._visit(x.num, in_minv, in_flux, in_bnd, in_bfield)
            self._visit(x.den, in_minv, in_flux, in_bnd, in_bfield)
            return
        if isinstance(x, ot.Power):
            self._visit(x.base, in_minv, in_flux, in_bnd, in_bfield)
            self._visit(x.exponent, in_minv, in_flux, in_bnd, in_bfield)
            return
        if isinstance(x, ot.BoundaryNormalComponent):
            if not in_bfield:
                raise NotImplementedError("boundary normal outside boundary data")
            return
        if isinstance(x, ot.OperatorBinding):
            op = x.op
            if isinstance(op, ot.DifferentiationOperator):
                if in_flux or in_minv:
                    raise NotImplementedError("derivative inside a flux or an inverse mass")
                if not isinstance(x.field, ot.Field):
                    raise NotImplementedError(
                        "derivative of an expression (%s): only fields are "
                        "differentiated on this path" % x.field)
                self.diff_keys.append(x.field.key)
                return
            if isinstance(op, ot.InverseMassOperator):
                if in_minv or in_flux:
                    raise NotImplementedError("nested inverse mass")
                self._visit(x.field, True, False, False)
                return
            if isinstance(op, ot.BoundarizeOperator):
                if not in_bfield:
                    raise NotImplementedError("boundary restriction outside boundary data")
                self._visit(x.field, in_minv, in_flux, True, in_bfield)
                return
            if isinstance(op, ot.FluxOperator):
                if not in_minv or in_flux:
                    raise NotImplementedError(
                        "flux outside an inverse mass: only the strong-form lift "
                        "M^-1 (flux) is on this path")
                arg = x.field
                if isinstance(arg, ot.BoundaryPair):
                    if arg.tag is TAG_NONE:
                        return
                    self.pairs.append((op, arg))
                    self._visit(arg.field, in_minv, True, False, False)
                    self._visit(arg.bfield, in_minv, True, False, True)
                else:
                    self.interior_args.append(_comps(arg))
                    self._visit(arg, in_minv, True, False, False)
                return
            raise NotImplementedError("operator %s is not on this path" % op)
        raise NotImplementedError("template node %r is not on this path" % (x,))


# --------------------------------------------------------------------------
# rewrites: over-integration and weak-form derivatives

_QUAD_SAMPLERS = (ot.QuadratureGridUpsampler, ot.QuadratureInteriorFacesGridUpsampler,
                  ot.QuadratureBoundaryGridUpsampler)


def _rebuild(x, f):
    """Copy of a template with ``f`` applied bottom-up to every node."""
    if isinstance(x, np.ndarray):
        out = np.empty(x.shape, dtype=object)
        for i in np.ndindex(x.shape):
            out[i] = _rebuild(x[i], f)
        return out
    if isinstance(x, ot.Sum):
        r = 0
        for c in x.children:
            r = ot.add(r, _rebuild(c, f))
        return f(r)
    if isinstance(x, ot.Product):
        r = 1
        for c in x.children:
            r = ot.mul(r, _rebuild(c, f))
        return f(r)
    if isinstance(x, ot.Quotient):
        return f(ot.div(_rebuild(x.num, f), _rebuild(x.den, f)))
    if isinstance(x, ot.Power):
        return f(ot.power(_rebuild(x.base, f), _rebuild(x.exponent, f)))
    if isinstance(x, ot.BoundaryPair):
        return ot.BoundaryPair(_rebuild(x.field, f), _rebuild(x.bfield, f), x.tag)
    if isinstance(x, ot.OperatorBinding):
        return f(ot.OperatorBinding(x.op, _rebuild(x.field, f)))
    return f(x)


def _linear_terms(x):
    """x as [(number, node)] with x = sum number * node, nodes free of
    top-level sums and numeric factors; None if x is not of that form."""
    if _is_num(x):
        return None if x != 0 else []
    if isinstance(x, ot.Sum):
        out = []
        for c in x.children:
            t = _linear_terms(c)
            if t is None:
                return None
            out.extend(t)
        return out
    if isinstance(x, ot.Product):
        coef, rest = 1.0, []
        for c in x.children:
            if _is_num(c):
                coef *= c
            else:
                rest.append(c)
        if len(rest) != 1:
            return None
        t = _linear_terms(rest[0])
        return None if t is None else [(coef * c, n) for c, n in t]
    if isinstance(x, ot.Quotient) and _is_num(x.den):
        t = _linear_terms(x.num)
        return None if t is None else [(c / x.den, n) for c, n in t]
    return [(1.0, x)]


def _linear_in_fields(x):
    """Linear combination of fields (possibly restricted to a boundary)
    with numeric coefficients."""
    if isinstance(x, np.ndarray):
        return all(_linear_in_fields(c) for c in x.reshape(-1))
    t = _linear_terms(x)
    if t is None:
        return False
    for _, n in t:
        if isinstance(n, ot.Field):
            continue
        if isinstance(n, ot.OperatorBinding) and isinstance(
                n.op, (ot.BoundarizeOperator,) + _QUAD_SAMPLERS) and _linear_in_fields(n.field):
            continue
        return False
    return True


class _Rewrites:
    def __init__(self):
        self.quadrature = False
        self.weak = False

    def run(self, outs):
        outs = [_rebuild(x, self._strip_quadrature) for x in outs]
        return [_rebuild(x, self._weak_to_strong) for x in outs]

    def _strip_quadrature(self, node):
        if not isinstance(node, ot.OperatorBinding):
            return node
        op = node.op
        if isinstance(op, _QUAD_SAMPLERS):
            if not _linear_in_fields(node.field):
                raise NotImplementedError(
                    "over-integration of %s: only fields with constant coefficients are "
                    "integrated exactly without quadrature on this path" % (node.field,))
            self.quadrature = True
            return node.field
        if isinstance(op, ot.QuadratureStiffnessTOperator):
            if not _linear_in_fields(node.field):
                raise NotImplementedError("quadrature stiffness of a non-linear integrand")
            self.quadrature = True
            return ot.OperatorBinding(ot.StiffnessTOperator(op.xyz_axis), node.field)
        return node

    def _weak_to_strong(self, node):
        if not (isinstance(node, ot.OperatorBinding)
                and isinstance(node.op, ot.InverseMassOperator)):
            return node
        terms = _linear_terms(node.field) if not isinstance(node.field, np.ndarray) else None
        if terms is None or not any(
                isinstance(n, ot.OperatorBinding) and isinstance(n.op, ot.StiffnessTOperator)
                for _, n in terms):
            return node
        self.weak = True
        vol, rest = 0, 0
        U = fl.FluxScalarPlaceholder(0)
        for c, n in terms:
            if not (isinstance(n, ot.OperatorBinding)
                    and isinstance(n.op, ot.StiffnessTOperator)):
                rest = ot.add(rest, ot.mul(c, n))
                continue
            x = n.op.xyz_axis
            inner = _linear_terms(n.field)
            if inner is None or not all(isinstance(g, ot.Field) for _, g in inner):
                raise NotImplementedError("weak derivative of %s: only of fields" % (n.field,))
            face = ot.FluxOperator(fl.Normal(x) * U.int)
            for cf, g in inner:
                vol = ot.add(vol, ot.mul(-c * cf, ot.DifferentiationOperator(x)(g)))
                both = ot.add(face(g), face(ot.BoundaryPair(
                    g, ot.BoundarizeOperator(TAG_ALL)(g), TAG_ALL)))
                rest = ot.add(rest, ot.mul(c * cf, both))
        return ot.add(vol, ot.InverseMassOperator()(rest))


# --------------------------------------------------------------------------
# pointwise evaluation

def _rand(key, lo, hi, n):
    seed = zlib.crc32(repr(key).encode())
    return np.random.default_rng(seed).uniform(lo, hi, n)


class _Ctx:
    """Probe values: fields (interior / exterior), derivatives, normals and
    the face kind evaluated (None: volume terms only; "interior"; or a
    boundary tag).  ``fixed`` overrides values by key."""

    def __init__(self, dims, face=None, coeff_keys=(), zero_state=False, fixed=None,
                 deriv=None, P=PROBES, salt=0):
        self.dims, self.face, self.P, self.salt = dims, face, P, salt
        self.coeff_keys = set(coeff_keys)
        self.fixed = fixed or {}
        self.deriv = deriv
        self.zero_state = zero_state
        n = _rand(("normal", salt), -1, 1, dims * P).reshape(dims, P)
        self.n = n / np.linalg.norm(n, axis=0)

    def val(self, key, interior):
        if (key, interior) in self.fixed:
            return self.fixed[(key, interior)]
        if key in self.fixed:
            return self.fixed[key]
        if key in self.coeff_keys:
            return _rand((key, interior, self.salt), 0.5, 1.5, self.P)
        if self.zero_state:
            return np.zeros(self.P)
        return _rand((key, interior, self.salt), -1, 1, self.P)

    def der(self, key, axis):
        if self.deriv is not None:
            return self.deriv(key, axis)
        return _rand(("d", key, axis, self.salt), -1, 1, self.P)

    def weak(self, axis):
        """Stand-in for the test-function derivative of S_axis^T."""
        return _rand(("w", axis, self.salt), -1, 1, self.P)


def _ev(x, ctx, interior=True):
    if _is_num(x):
        return float(x)
    if isinstance(x, ot.Field):
        return ctx.val(x.key, interior)
    if isinstance(x, ot.Sum):
        r = 0.0
        for c in x.children:
            r = r + _ev(c, ctx, interior)
        return r
    if isinstance(x, ot.Product):
        r = 1.0
        for c in x.children:
            r = r * _ev(c, ctx, interior)
        return r
    if isinstance(x, ot.Quotient):
        return _ev(x.num, ctx, interior) / _ev(x.den, ctx, interior)
    if isinstance(x, ot.Power):
        return _ev(x.base, ctx, interior) ** _ev(x.exponent, ctx, interior)
    if isinstance(x, ot.BoundaryNormalComponent):
        return ctx.n[x.axis]
    if isinstance(x, ot.OperatorBinding):
        op = x.op
        if isinstance(op, ot.DifferentiationOperator):
            return ctx.der(x.field.key, op.xyz_axis)
        if isinstance(op, (ot.InverseMassOperator, ot.BoundarizeOperator) + _QUAD_SAMPLERS):
            return _ev(x.field, ctx, interior)
        if isinstance(op, ot.FluxOperator):
            return _ev_binding(op, x.field, ctx)
        if isinstance(op, (ot.StiffnessTOperator, ot.QuadratureStiffnessTOperator)):
            return ctx.weak(op.xyz_axis) * _ev(x.field, ctx, interior)
        if isinstance(op, ot.ElementwiseMaxOperator):
            y = _ev(x.field, ctx, interior)
            return 1.7 * y + np.sin(y)
    raise NotImplementedError("cannot evaluate %r" % (x,))


def _ev_binding(op, arg, ctx):
    if isinstance(arg, ot.BoundaryPair):
        if ctx.face is None or ctx.face == "interior" or arg.tag is TAG_NONE:
            return 0.0
        if not (arg.tag is TAG_ALL or arg.tag == ctx.face):
            return 0.0
        iv = [_ev(c, ctx, True) for c in _comps(arg.field)]
        ev = [_ev(c, ctx, True) for c in _comps(arg.bfield)]
        if len(iv) != len(ev):
            raise ValueError("boundary pair: %d volume vs %d boundary components"
                             % (len(iv), len(ev)))
    else:
        if ctx.face != "interior":
            return 0.0
        iv = [_ev(c, ctx, True) for c in _comps(arg)]
        ev = [_ev(c, ctx, False) for c in _comps(arg)]
    return _ev_flux(op.flux, iv, ev, ctx.n)


def _ev_flux(x, iv, ev, n):
    if _is_num(x):
        return float(x)
    if isinstance(x, fl.FieldComponent):
        vals = iv if x.is_interior else ev
        if not 0 <= x.index < len(vals):
            raise ValueError("flux refers to component %d of a %d-vector"
                             % (x.index, len(vals)))
        v = vals[x.index]
        return v if not _is_num(v) else np.full(n.shape[1], float(v))
    if isinstance(x, fl.Normal):
        return n[x.axis]
    if isinstance(x, ot.Sum):
        r = 0.0
        for c in x.children:
            r = r + _ev_flux(c, iv, ev, n)
        return r
    if isinstance(x, ot.Product):
        r = 1.0
        for c in x.children:
            r = r * _ev_flux(c, iv, ev, n)
        return r
    if isinstance(x, ot.Quotient):
        return _ev_flux(x.num, iv, ev, n) / _ev_flux(x.den, iv, ev, n)
    if isinstance(x, ot.Power):
        return _ev_flux(x.base, iv, ev, n) ** _ev_flux(x.exponent, iv, ev, n)
    if isinstance(x, fl.IfPositive):
        c = np.broadcast_to(_ev_flux(x.criterion, iv, ev, n), (n.shape[1],))
        return np.where(c > 0, _ev_flux(x.then, iv, ev, n), _ev_flux(x.else_, iv, ev, n))
    if isinstance(x, fl.FunctionCall):
        a = [_ev_flux(y, iv, ev, n) for y in x.args]
        return {"abs": lambda: np.abs(a[0]), "max": lambda: np.maximum(a[0], a[1]),
                "min": lambda: np.minimum(a[0], a[1])}[x.name]()
    raise NotImplementedError("flux term %s is not on this path" % (x,))


def evaluate(outs, ctx):
    """Outputs of a template at the probes of ``ctx``: [n_outputs, P]."""
    return np.stack([np.broadcast_to(np.asarray(_ev(x, ctx), dtype=np.float64), (ctx.P,))
                     for x in outs])


def _close(a, b):
    return np.max(np.abs(a - b)) <= TOL * (1.0 + np.max(np.abs(a)))


# --------------------------------------------------------------------------
# kernel models

class _Roles:
    def __init__(self, state, coeff, given, source, coeffs=(), givens=()):
        self.state = state          # object array of the state Fields
        self.coeff = coeff          # Field or None (one coefficient field)
        self.coeffs = list(coeffs)  # every coefficient field (Maxwell material: eps, mu)
        self.given = given          # Field or None (one given boundary field)
        self.givens = list(givens)  # every given boundary field (Maxwell incident data)
        self.source = source        # expression of the user's source (or 0)

    def names(self):
        st = self.state
        names = {st[0].name} if all(f.name == st[0].name for f in st) else None
        d = {"state": st[0].name if names else None,
             "state_keys": [f.key for f in st]}
        if self.coeff is not None:
            d["coeff"] = self.coeff.name
        elif len(self.coeffs) > 1:
            d["coeffs"] = [(f.name, f.index) for f in self.coeffs]
        if self.given is not None:
            d["given"] = self.given.name
        elif len(self.givens) > 1:
            g = self.givens
            if all(f.name == g[0].name for f in g):
                d["given"] = g[0].name
            d["given_keys"] = [f.key for f in g]
        return d


class _Family:
    model = None
    kinds = ()
    source_outputs = ()      # outputs the kernel model can add a source to

    def applies(self, dims, F, ncoeff):
        return False

    def volume_params(self, V):
        return None

    def flux_choices(self, user, roles, params, dims):
        return []

    def bdry_choices(self, user, roles, params, dims, tag, kind):
        return [None]

    def build(self, roles, params, bc):
        raise NotImplementedError


class _Advection(_Family):
    model = MODEL_ADVECTION
    kinds = (BC_GIVEN,)

    def applies(self, dims, F, ncoeff):
        return F == 1 and ncoeff == 0

    def volume_params(self, V):
        return {"v": -V[0, 0, :]}

    def flux_choices(self, user, roles, params, dims):
        return [dict(params, flux_type=t) for t in ("central", "upwind", "lf")]

    def build(self, roles, p, bc):
        tag = bc[0] if bc is not None else TAG_NONE
        m = StrongAdvectionOperator(p["v"], inflow_tag=tag, flux_type=p["flux_type"])
        if bc is not None and roles.given is None:
            return None
        return m, _comps(m.op_template(u=roles.state[0],
                                       bc_in=roles.given if roles.given is not None
                                       else ot.Field("bc_in")))


class _Wave(_Family):
    model = MODEL_WAVE
    kinds = (BC_DIRICHLET, BC_NEUMANN, BC_RADIATION, BC_GIVEN)
    source_outputs = (0,)

    def applies(self, dims, F, ncoeff):
        return F == dims + 1 and ncoeff == 0

    def volume_params(self, V):
        c = V[0, 1, 0]
        return {"c": c} if c != 0 else None

    def flux_choices(self, user, roles, params, dims):
        return [dict(params, flux_type=t) for t in ("upwind", "central")]

    def _tags(self, bc):
        t = {BC_DIRICHLET: TAG_NONE, BC_NEUMANN: TAG_NONE, BC_RADIATION: TAG_NONE}
        if bc is not None:
            # given data on a tag: inhomogeneous Dirichlet there
            t[BC_DIRICHLET if bc[1] == BC_GIVEN else bc[1]] = bc[0]
        return dict(dirichlet_tag=t[BC_DIRICHLET], neumann_tag=t[BC_NEUMANN],
                    radiation_tag=t[BC_RADIATION])

    def build(self, roles, p, bc):
        dims = len(roles.state) - 1
        given = bc is not None and bc[1] == BC_GIVEN
        if given and roles.given is None:
            return None
        m = StrongWaveOperator(p["c"], dims, source_f=0, flux_type=p["flux_type"],
                               dirichlet_bc_f=1 if given else 0, **self._tags(bc))
        m.source_f = roles.source
        return m, _comps(m.op_template(w=roles.state,
                                       dir_bc_u=roles.given if given else None))


class _VarWave(_Wave):
    model = MODEL_VARWAVE
    kinds = (BC_DIRICHLET, BC_NEUMANN, BC_RADIATION)

    def applies(self, dims, F, ncoeff):
        return F == dims + 1 and ncoeff == 1

    def volume_params(self, V):
        ts = V[0, 1, 0]      # time_sign * c with the coefficient probed at 1
        return {"time_sign": ts} if ts != 0 else None

    def build(self, roles, p, bc):
        dims = len(roles.state) - 1
        m = VariableVelocityStrongWaveOperator(
            roles.coeff, dims, source=0, flux_type=p["flux_type"],
            time_sign=p["time_sign"], **self._tags(bc))
        m.source = -1 * roles.source if not ot.is_zero(roles.source) else 0
        return m, _comps(m.op_template(w=roles.state))


class _Maxwell(_Family):
    model = MODEL_MAXWELL
    kinds = (BC_PEC, BC_PMC, BC_ABSORB, BC_INCIDENT)
    source_outputs = (0, 1, 2)
    cls = MaxwellOperator

    def applies(self, dims, F, ncoeff):
        return dims == 3 and F == 6 and ncoeff == 0

    def volume_params(self, V):
        # d/dy Hz -> Ex is 1/eps, d/dy Ez -> Hx is -1/mu
        a, b = V[0, 5, 1], V[3, 2, 1]
        if a <= 0 or b >= 0:
            return None
        return {"eps": 1.0 / a, "mu": -1.0 / b}

    def _fit(self, user, roles, p, ctx, key, bc):
        """Numeric flux types enter affinely: fit from the templates at 0, 1."""
        ys = []
        for alpha in (0.0, 1.0):
            q = dict(p, **{key: alpha})
            ys.append(evaluate(self.build(roles, q, bc)[1], ctx))
        y = evaluate(user, ctx)
        dy = ys[1] - ys[0]
        den = float(np.sum(dy * dy))
        return float(np.sum((y - ys[0]) * dy) / den) if den > 0 else 0.0

    def flux_choices(self, user, roles, params, dims):
        ctx = _Ctx(dims, face="interior", coeff_keys=[f.key for f in roles.coeffs])
        alpha = self._fit(user, roles, dict(params, bdry_flux_type=0.0), ctx, "flux_type",
                          None)
        return [dict(params, flux_type="lf", bdry_flux_type="lf"),
                dict(params, flux_type=alpha, bdry_flux_type=alpha)]

    def bdry_choices(self, user, roles, params, dims, tag, kind):
        ctx = _Ctx(dims, face=tag, coeff_keys=[f.key for f in roles.coeffs])
        return ["lf", self._fit(user, roles, params, ctx, "bdry_flux_type", (tag, kind))]

    @staticmethod
    def _incident(roles, bc):
        """incident_bc of the kernel model: the given boundary fields (one per
        component, the data whose negative is the exterior state), or zero."""
        if bc is not None and bc[1] == BC_INCIDENT and len(roles.givens) > 1:
            data = np.array(roles.givens, dtype=object)
            return lambda op, e, h: data
        return lambda op, e, h: 0

    def build(self, roles, p, bc):
        t = {BC_PEC: TAG_NONE, BC_PMC: TAG_NONE, BC_ABSORB: TAG_NONE, BC_INCIDENT: TAG_NONE}
        if bc is not None:
            t[bc[1]] = bc[0]
        m = self.cls(p["eps"], p["mu"], p["flux_type"],
                     bdry_flux_type=p.get("bdry_flux_type", p["flux_type"]),
                     pec_tag=t[BC_PEC], pmc_tag=t[BC_PMC], absorb_tag=t[BC_ABSORB],
                     incident_tag=t[BC_INCIDENT], incident_bc=self._incident(roles, bc))
        # E_c's rhs source s_c = -J_c / eps: the current is -eps s
        ne = m.n_e
        srcs = getattr(roles, "sources", None)
        if srcs is not None and any(not ot.is_zero(x) for x in srcs[:ne]):
            m.current = np.array([-p["eps"] * x if not ot.is_zero(x) else 0
                                  for x in srcs[:ne]], dtype=object)
        if srcs is not None and any(not ot.is_zero(x) for x in srcs[ne:]):
            return None
        return m, _comps(m.op_template(w=roles.state))


class _MaxwellVar(_Maxwell):
    """Maxwell with variable material: the flux argument's first two fields
    are epsilon and mu (em.py:309-371).  A source current J enters the E
    rows as (curl H - J) / eps; with the material probed at 1 the source
    probe reads -J."""
    source_outputs = (0, 1, 2)

    def applies(self, dims, F, ncoeff):
        return dims == 3 and F == 6 and ncoeff == 2

    def volume_params(self, V):
        # with the material probed at 1: d/dy Hz -> Ex is 1/eps = 1, d/dy Ez
        # -> Hx is -1/mu = -1
        return {} if _close(np.array([V[0, 5, 1], V[3, 2, 1]]), np.array([1.0, -1.0])) \
            else None

    def build(self, roles, p, bc):
        t = {BC_PEC: TAG_NONE, BC_PMC: TAG_NONE, BC_ABSORB: TAG_NONE, BC_INCIDENT: TAG_NONE}
        if bc is not None:
            t[bc[1]] = bc[0]
        m = self.cls(roles.coeffs[0], roles.coeffs[1], p["flux_type"],
                     bdry_flux_type=p.get("bdry_flux_type", p["flux_type"]),
                     pec_tag=t[BC_PEC], pmc_tag=t[BC_PMC], absorb_tag=t[BC_ABSORB],
                     incident_tag=t[BC_INCIDENT], incident_bc=self._incident(roles, bc))
        ne = m.n_e
        srcs = getattr(roles, "sources", None)
        if srcs is not None and any(not ot.is_zero(x) for x in srcs[:ne]):
            m.current = np.array([-1 * x if not ot.is_zero(x) else 0 for x in srcs[:ne]],
                                 dtype=object)
        if srcs is not None and any(not ot.is_zero(x) for x in srcs[ne:]):
            return None
        return m, _comps(m.op_template(w=roles.state))


class _MaxwellTMVar(_MaxwellVar):
    model = MODEL_MAXWELL_TM
    cls = TMMaxwellOperator
    source_outputs = (0,)

    def applies(self, dims, F, ncoeff):
        return dims == 2 and F == 3 and ncoeff == 2

    def volume_params(self, V):
        return {} if _close(np.array([V[0, 2, 0], V[1, 0, 1]]), np.array([1.0, -1.0])) \
            else None


class _MaxwellTEVar(_MaxwellVar):
    model = MODEL_MAXWELL_TE
    cls = TEMaxwellOperator
    source_outputs = (0, 1)

    def applies(self, dims, F, ncoeff):
        return dims == 2 and F == 3 and ncoeff == 2

    def volume_params(self, V):
        return {} if _close(np.array([V[0, 2, 1], V[2, 1, 0]]), np.array([1.0, -1.0])) \
            else None


class _MaxwellTM(_Maxwell):
    model = MODEL_MAXWELL_TM
    source_outputs = (0,)
    cls = TMMaxwellOperator

    def applies(self, dims, F, ncoeff):
        return dims == 2 and F == 3 and ncoeff == 0

    def volume_params(self, V):
        # (Ez, Hx, Hy): d/dx Hy -> Ez is 1/eps, d/dy Ez -> Hx is -1/mu
        a, b = V[0, 2, 0], V[1, 0, 1]
        if a <= 0 or b >= 0:
            return None
        return {"eps": 1.0 / a, "mu": -1.0 / b}


class _MaxwellTE(_Maxwell):
    model = MODEL_MAXWELL_TE
    source_outputs = (0, 1)
    cls = TEMaxwellOperator

    def applies(self, dims, F, ncoeff):
        return dims == 2 and F == 3 and ncoeff == 0

    def volume_params(self, V):
        # (Ex, Ey, Hz): d/dy Hz -> Ex is 1/eps, d/dx Ey -> Hz is -1/mu
        a, b = V[0, 2, 1], V[2, 1, 0]
        if a <= 0 or b >= 0:
            return None
        return {"eps": 1.0 / a, "mu": -1.0 / b}


_FAMILIES = (_Advection(), _Wave(), _VarWave(), _Maxwell(), _MaxwellTM(), _MaxwellTE(),
             _MaxwellVar(), _MaxwellTMVar(), _MaxwellTEVar())


# --------------------------------------------------------------------------

def _source(user, roles_keys, src_fields, dims, coeff_keys=()):
    """The template's sources: output values with the state, derivatives and
    fluxes at zero (coefficient fields at one), per output as
    const + sum coef_k * field_k.  Returns (expressions, constants, terms)
    with one entry per output."""
    zero = {k: np.zeros(PROBES) for k in roles_keys}
    zero.update({k: np.ones(PROBES) for k in coeff_keys})

    def at(fixed):
        ctx = _Ctx(dims, face=None, fixed={**zero, **fixed},
                   deriv=lambda k, a: np.zeros(PROBES))
        return evaluate(user, ctx)

    allzero = {k: np.zeros(PROBES) for k in src_fields}
    base = at(allzero)
    if np.any(base != base[:, :1]):
        raise NotImplementedError("sources that vary with the state")
    consts = base[:, 0]
    exprs = [float(c) if c != 0 else 0 for c in consts]
    terms = [[] for _ in consts]
    for k, f in src_fields.items():
        one = at({**allzero, k: np.ones(PROBES)})
        for o in range(len(consts)):
            coef = one[o, 0] - consts[o]
            if coef != 0:
                exprs[o] = exprs[o] + coef * f
                terms[o].append((f.name, f.index, coef))
    return exprs, consts, terms


def lower(template, dimensions, mesh=None):
    """The :class:`~hedge_b200.models.OpTemplate` a symbolic template equals
    (see the module docstring); raises ``NotImplementedError`` when no
    kernel model reproduces it.  With ``mesh``, boundary faces that carry
    none of the template's specific tags are known to exist or not (else a
    TAG_ALL-only boundary condition must match too)."""
    if _needs_quadrature_kernel(_comps(template)):
        return _lower_quadrature(_comps(template), dimensions)
    rw = _Rewrites()
    outs = rw.run(_comps(template))
    F = len(outs)
    scan = _Scan()
    scan.run(outs)
    if not scan.interior_args:
        raise NotImplementedError("template has no interior flux")
    arg = scan.interior_args[0]
    for a in scan.interior_args[1:]:
        if [getattr(x, "key", x) for x in a] != [getattr(x, "key", x) for x in arg]:
            raise NotImplementedError("interior fluxes of different arguments")
    if not all(isinstance(x, ot.Field) for x in arg):
        raise NotImplementedError("flux argument components must be fields")
    diff = set(scan.diff_keys)
    state = [x for x in arg if x.key in diff]
    coeff = [x for x in arg if x.key not in diff]
    if len(coeff) > 2 or any(arg[k] is not coeff[k] for k in range(len(coeff))):
        raise NotImplementedError("at most two coefficient fields, first in the flux argument")
    if len(state) != F:
        raise NotImplementedError("%d outputs but %d differentiated state fields in the "
                                  "flux argument" % (F, len(state)))
    st_keys = {x.key for x in state}
    co_keys = {x.key for x in coeff}
    given = [f for k, f in scan.given_fields.items() if k not in st_keys | co_keys]
    if len(given) > 1 and len(given) != F:
        raise NotImplementedError("%d given boundary fields: one, or one per output "
                                  "(Maxwell incident data)" % len(given))
    # several given fields: a Maxwell system's incident data, one per
    # component, in the order the boundary data names them (a vector's
    # components in index order)
    if len(given) > 1 and all(f.name == given[0].name and f.index is not None
                              for f in given):
        given.sort(key=lambda f: f.index)
    src_fields = {k: f for k, f in scan.outside_fields.items()
                  if k not in st_keys | co_keys and k not in diff}
    roles_keys = st_keys | co_keys | {f.key for f in given}
    src_exprs, src_consts, src_terms = _source(outs, roles_keys, src_fields, dimensions,
                                               co_keys)
    if any(len(t) > 1 for t in src_terms):
        raise NotImplementedError("more than one source field on an output")
    src_outputs = [o for o in range(F) if src_terms[o] or src_consts[o] != 0]
    state_arr = ot.join_fields(state)
    roles = _Roles(state_arr, coeff[0] if len(coeff) == 1 else None,
                   given[0] if len(given) == 1 else None, src_exprs[0], coeffs=coeff,
                   givens=given)
    roles.sources = src_exprs

    # volume coefficients V[f, g, x]: unit derivative probes less the
    # zero-derivative value (the constant source), coefficient fields = 1
    keys = [x.key for x in state]
    fixed = {k: np.zeros(PROBES) for k in st_keys}
    fixed.update({k: np.ones(PROBES) for k in co_keys})
    fixed.update({k: np.zeros(PROBES) for k in src_fields})
    V0 = evaluate(outs, _Ctx(dimensions, face=None, fixed=fixed,
                             deriv=lambda k, a: np.zeros(PROBES)))[:, 0]
    V = np.zeros((F, F, dimensions))
    for g, kg in enumerate(keys):
        for x in range(dimensions):
            def der(k, a, kg=kg, x=x):
                return np.full(PROBES, 1.0 if (k == kg and a == x) else 0.0)
            ctx = _Ctx(dimensions, face=None, fixed=fixed, deriv=der)
            V[:, g, x] = evaluate(outs, ctx)[:, 0] - V0

    if rw.quadrature and coeff:
        raise NotImplementedError("over-integration with a coefficient field")
    tags = []
    for _, pair in scan.pairs:
        if not any(pair.tag is t or pair.tag == t for t in tags):
            tags.append(pair.tag)
    specific = [t for t in tags if t is not TAG_ALL]
    if specific and any(t is TAG_ALL for t in tags):
        # TAG_ALL pairs act on every boundary face: in each specific tag's
        # context together with that tag's pairs, and alone on the faces
        # no specific tag covers (if the mesh has any)
        tags = specific[:]
        if mesh is None or _uncovered(mesh, specific):
            tags.insert(0, TAG_ALL)

    # the reason reported is the one from the furthest stage reached
    why = [0, "no kernel model has %d fields in %dD" % (F, dimensions)]

    def fail(stage, msg):
        if stage >= why[0]:
            why[:] = [stage, msg]
    for fam in _FAMILIES:
        if not fam.applies(dimensions, F, len(coeff)):
            continue
        if any(o not in fam.source_outputs for o in src_outputs):
            fail(1, "sources on outputs the %s kernel has none for" % type(fam).__name__[1:])
            continue
        params = fam.volume_params(V)
        if params is None:
            fail(1, "volume terms match no kernel model")
            continue
        vol_ctx = _Ctx(dimensions, face=None, coeff_keys=co_keys)
        int_ctx = _Ctx(dimensions, face="interior", coeff_keys=co_keys)
        y_vol, y_int = evaluate(outs, vol_ctx), evaluate(outs, int_ctx)
        for choice in fam.flux_choices(outs, roles, params, dimensions):
            built = fam.build(roles, choice, None)
            if built is None:
                continue
            canon = built[1]
            if not _close(y_vol, evaluate(canon, vol_ctx)):
                fail(1, "volume terms differ from the %s kernel's" % type(fam).__name__[1:])
                break
            if not _close(y_int, evaluate(canon, int_ctx)):
                fail(2, "interior flux matches no flux type of the %s kernel"
                     % type(fam).__name__[1:])
                continue
            bcs, bft = [], None
            ok = True
            for tag in tags:
                b_ctx = _Ctx(dimensions, face=tag, coeff_keys=co_keys)
                y_b = evaluate(outs, b_ctx)
                hit = None
                if _close(y_b, evaluate(canon, b_ctx)):
                    hit = (BC_NONE, None)     # no boundary flux on these faces
                for kind in ([] if hit else fam.kinds):
                    for bchoice in fam.bdry_choices(outs, roles, choice, dimensions, tag, kind):
                        q = dict(choice) if bchoice is None else dict(choice, bdry_flux_type=bchoice)
                        b = fam.build(roles, q, (tag, kind))
                        if b is not None and _close(y_b, evaluate(b[1], b_ctx)):
                            hit = (kind, bchoice)
                            break
                    if hit:
                        break
                if hit is None:
                    fail(3, "boundary %s: no boundary condition of the %s kernel matches" % (
                        getattr(tag, "__name__", tag), type(fam).__name__[1:]))
                    ok = False
                    break
                if hit[1] is not None:
                    if bft is not None and not _same_ft(bft, hit[1]):
                        fail(3, "boundary fluxes of different flux types")
                        ok = False
                        break
                    bft = hit[1]
                bcs.append((tag, hit[0]))
            if not ok:
                continue
            final = dict(choice)
            if bft is not None:
                final["bdry_flux_type"] = bft
            model = fam.build(roles, final, None)[0]
            desc = model.descriptor()
            bcs = [(t, k) for t, k in bcs if not (k == BC_NONE and t is TAG_ALL)]
            names = roles.names()
            if len(roles.givens) > 1:
                inc = [t for t, k in bcs if k == BC_INCIDENT]
                if len(inc) != 1:
                    fail(3, "given boundary fields outside one incident boundary")
                    continue
                desc.params["incident_data"] = True
            if desc.model in (MODEL_MAXWELL, MODEL_MAXWELL_TM, MODEL_MAXWELL_TE):
                # per E component: the value added to its rhs, const + coef * field
                names["sources"] = [(o, float(src_consts[o]),
                                     src_terms[o][0][:2] if src_terms[o] else None,
                                     src_terms[o][0][2] if src_terms[o] else 0.0)
                                    for o in src_outputs]
            else:
                if src_terms[0]:
                    names["source"] = src_terms[0][0][:2]
                    names["source_coef"] = src_terms[0][0][2]
                names["source_const"] = float(src_consts[0])
            return OpTemplate(desc.model, desc.dimensions, desc.n_fields, desc.flux_type,
                              _lowered_params(desc, float(src_consts[0])), bcs, None, names)
    raise NotImplementedError("op template is not one the B200 kernels implement: " + why[1])


def _needs_quadrature_kernel(outs):
    """Whether the template integrates a product of fields by quadrature
    (or takes an element maximum): the work of the quadrature kernel."""
    for x in outs:
        for n in ot.walk(x):
            if not isinstance(n, ot.OperatorBinding):
                continue
            if isinstance(n.op, ot.ElementwiseMaxOperator):
                return True
            if isinstance(n.op, _QUAD_SAMPLERS + (ot.QuadratureStiffnessTOperator,)) and \
                    not _linear_in_fields(n.field):
                return True
            if isinstance(n.op, ot.StiffnessTOperator) and any(
                    isinstance(m, ot.OperatorBinding) and isinstance(m.op, _QUAD_SAMPLERS)
                    for m in ot.walk(n.field)) and not _linear_in_fields(n.field):
                return True
    return False


def _strip_samplers(x):
    return _rebuild(x, lambda n: n.field if isinstance(n, ot.OperatorBinding)
                    and isinstance(n.op, _QUAD_SAMPLERS) else n)


def _lower_quadrature(outs, dims):
    """The variable-coefficient advection operator a quadrature template
    equals (see the module docstring)."""
    if len(outs) != 1:
        raise NotImplementedError("quadrature templates: one output (the advected field)")
    tags = {n.op.quadrature_tag for x in outs for n in ot.walk(x)
            if isinstance(n, ot.OperatorBinding)
            and isinstance(n.op, _QUAD_SAMPLERS + (ot.QuadratureStiffnessTOperator,))}
    if len(tags) > 1:
        raise NotImplementedError("more than one quadrature tag")
    qtag = tags.pop() if tags else "quad"
    interior, pairs = [], []
    for n in ot.walk(outs[0]):
        if isinstance(n, ot.OperatorBinding) and isinstance(n.op, ot.FluxOperator):
            (pairs if isinstance(n.field, ot.BoundaryPair) else interior).append(n.field)
    if not interior:
        raise NotImplementedError("quadrature template without an interior flux")
    arg = [_strip_samplers(c) for c in _comps(interior[0])]
    if len(arg) != dims + 2 or not all(isinstance(c, ot.Field) for c in arg[:dims + 1]):
        raise NotImplementedError(
            "quadrature template: the flux argument must be (u, v_0 .. v_%d, c) with "
            "u and v fields" % (dims - 1))
    u, v = arg[0], arg[1:dims + 1]
    if not all(f.name == v[0].name and f.index == i for i, f in enumerate(v)):
        raise NotImplementedError("the velocity components must be one vector field "
                                  "(make_sym_vector)")
    given = None
    for p in pairs:
        b0 = _strip_samplers(_comps(p.bfield)[0])
        if isinstance(b0, ot.Field):
            given = b0
    v_arr = ot.join_fields(v)
    why = "no flux type of the variable-coefficient advection kernel matches"
    for has_bc in ((True, False) if given is not None else (False,)):
        for ft in VariableCoefficientAdvectionOperator.flux_types:
            m = VariableCoefficientAdvectionOperator(dims, None, bc_u_f=1 if has_bc else "None",
                                                     flux_type=ft)
            canon = _comps(m.op_template(u=u, v=v_arr, bc_u=given if has_bc else None))
            canon = [_rebuild(c, lambda n: _retag(n, qtag)) for c in canon]
            ok = True
            for face in (None, "interior", TAG_ALL):
                ctx = _Ctx(dims, face=face)
                if not _close(evaluate(outs, ctx), evaluate(canon, ctx)):
                    if face is None:
                        why = "volume terms differ from the variable-coefficient advection kernel's"
                    ok = False
                    break
            if ok:
                names = {"state": u.name, "coeff": v[0].name,
                         "given": given.name if has_bc else None}
                return OpTemplate(MODEL_VARADV, dims, 1,
                                  VariableCoefficientAdvectionOperator.flux_types.index(ft),
                                  {"quad_tag": qtag},
                                  [(TAG_ALL, BC_GIVEN if has_bc else BC_DIRICHLET)], None, names)
    raise NotImplementedError("op template is not one the B200 kernels implement: " + why)


def _retag(n, tag):
    """The model template's up-samplers with the user template's tag."""
    if isinstance(n, ot.OperatorBinding):
        if isinstance(n.op, ot.QuadratureGridUpsampler):
            return ot.OperatorBinding(ot.QuadratureGridUpsampler(tag), n.field)
        if isinstance(n.op, ot.QuadratureInteriorFacesGridUpsampler):
            return ot.OperatorBinding(ot.QuadratureInteriorFacesGridUpsampler(tag), n.field)
    return n


def _uncovered(mesh, tags):
    """Whether some boundary face carries none of ``tags``."""
    covered = set()
    for t in tags:
        covered.update(map(tuple, mesh.boundary_faces(t).tolist()))
    return any(tuple(f) not in covered for f in mesh.boundary_faces(TAG_ALL).tolist())


def as_descriptor(template, dimensions, mesh=None):
    """A lowered :class:`OpTemplate` for a template or an OpTemplate (the
    model that made the template, if any, attached as its operator)."""
    if isinstance(template, OpTemplate):
        return template
    from .models import template_model
    desc = lower(template, dimensions, mesh)
    desc.operator = template_model(template)
    return desc


def _same_ft(a, b):
    if isinstance(a, str) or isinstance(b, str):
        return a == b
    return abs(a - b) <= 1e-9


def _lowered_params(desc, src_const):
    p = dict(desc.params)
    if "source" in p:
        p["source"] = src_const
    return p


__all__ = ["lower", "as_descriptor", "evaluate", "PROBES"]
