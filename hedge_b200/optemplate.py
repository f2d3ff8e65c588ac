"""Operator templates: symbolic right-hand sides, as in hedge.optemplate.

A template is an expression, or a numpy object array of expressions (one per
output field), built from fields, the element-local operators
(differentiation, inverse mass, restriction to a boundary), flux operators
applied to a volume vector or to a :class:`BoundaryPair`, and arithmetic.
The construction API follows the reference's:

=============================  ==============================================
here                           reference
=============================  ==============================================
Field, make_sym_vector         hedge/optemplate/primitives.py:52-57
                               (pymbolic Variable / make_sym_vector)
OperatorBinding                primitives.py:91-110
BoundaryPair                   primitives.py:132-162
BoundaryNormalComponent,       primitives.py:193-209
normal / make_normal
Operator (call / ``op * f``)   operators.py:36-74
DifferentiationOperator        operators.py:107-139
MassOperator,                  operators.py:389-415
InverseMassOperator
StiffnessOperator,             operators.py:133-143 (S_x = M D_x and the
StiffnessTOperator,            weak derivative S_x^T)
make_stiffness(_t)
Quadrature*Upsampler,          operators.py:149-168, 262-314
QuadratureStiffnessTOperator   (over-integration)
BoundarizeOperator             operators.py:488-495
FluxOperator,                  operators.py:529-657
VectorFluxOperator
get_flux_operator, make_nabla  tools.py:40-60
join_fields                    pytools.obj_array.join_fields
cse                            pymbolic CommonSubexpression (identity here:
                               the lowering evaluates trees, it does not
                               generate code)
=============================  ==============================================

Arithmetic folds numbers and drops zero terms the way the reference's
``is_zero`` pruning does, so ``numpy.dot`` over object arrays of
expressions gives compact trees.  ``Discretization.compile`` lowers a
template onto the fused kernels (``hedge_b200.lowering``).
"""

from __future__ import annotations

import numbers

import numpy as np


def is_zero(x):
    return isinstance(x, numbers.Number) and not isinstance(x, bool) and x == 0


def _is_one(x):
    return isinstance(x, numbers.Number) and not isinstance(x, bool) and x == 1


def _map_array(f, a):
    out = np.empty(a.shape, dtype=object)
    for i in np.ndindex(a.shape):
        out[i] = f(a[i])
    return out


def _binary(fn, a, b):
    if isinstance(a, np.ndarray) or isinstance(b, np.ndarray):
        aa = np.asarray(a, dtype=object)
        bb = np.asarray(b, dtype=object)
        aa, bb = np.broadcast_arrays(aa, bb)
        out = np.empty(aa.shape, dtype=object)
        for i in np.ndindex(aa.shape):
            out[i] = fn(aa[i], bb[i])
        return out
    return fn(a, b)


def _number(x):
    return isinstance(x, numbers.Number) and not isinstance(x, bool)


def add(a, b):
    if is_zero(a):
        return b
    if is_zero(b):
        return a
    if _number(a) and _number(b):
        return a + b
    terms = []
    for x in (a, b):
        terms.extend(x.children if isinstance(x, Sum) else (x,))
    return Sum(tuple(terms))


def mul(a, b):
    if is_zero(a) or is_zero(b):
        return 0
    if _is_one(a):
        return b
    if _is_one(b):
        return a
    if _number(a) and _number(b):
        return a * b
    factors = []
    for x in (a, b):
        factors.extend(x.children if isinstance(x, Product) else (x,))
    return Product(tuple(factors))


def div(a, b):
    if is_zero(b):
        raise ZeroDivisionError("division by a zero expression")
    if is_zero(a):
        return 0
    if _is_one(b):
        return a
    if _number(a) and _number(b):
        return a / b
    return Quotient(a, b)


def power(a, b):
    if _number(a) and _number(b):
        return a ** b
    if _is_one(b):
        return a
    return Power(a, b)


class Expr:
    """Base of every expression node (volume and flux languages)."""

    # numpy defers binary operators with an Expr operand to the Expr
    __array_ufunc__ = None

    def __add__(self, o):
        return _binary(add, self, o)

    def __radd__(self, o):
        return _binary(add, o, self)

    def __sub__(self, o):
        return _binary(lambda x, y: add(x, mul(-1, y)), self, o)

    def __rsub__(self, o):
        return _binary(lambda x, y: add(x, mul(-1, y)), o, self)

    def __mul__(self, o):
        return _binary(mul, self, o)

    def __rmul__(self, o):
        return _binary(lambda x, y: x * y if isinstance(x, (Operator, VectorFluxOperator))
                       else mul(x, y), o, self)

    def __truediv__(self, o):
        return _binary(div, self, o)

    def __rtruediv__(self, o):
        return _binary(div, o, self)

    def __neg__(self):
        return mul(-1, self)

    def __pos__(self):
        return self

    def __pow__(self, o):
        return _binary(power, self, o)

    def __rpow__(self, o):
        return _binary(power, o, self)

    def __repr__(self):
        return self.__str__()


class Sum(Expr):
    def __init__(self, children):
        self.children = children

    def __str__(self):
        return "(" + " + ".join(str(c) for c in self.children) + ")"


class Product(Expr):
    def __init__(self, children):
        self.children = children

    def __str__(self):
        return "*".join(_paren(c) for c in self.children)


class Quotient(Expr):
    def __init__(self, num, den):
        self.num, self.den = num, den

    def __str__(self):
        return "%s/%s" % (_paren(self.num), _paren(self.den))


class Power(Expr):
    def __init__(self, base, exponent):
        self.base, self.exponent = base, exponent

    def __str__(self):
        return "%s**%s" % (_paren(self.base), _paren(self.exponent))


def _paren(x):
    return "(%s)" % x if isinstance(x, (Sum, Quotient)) else str(x)


# --------------------------------------------------------------------------
# leaves of the volume language

class Field(Expr):
    """A named volume vector; ``index`` selects a component of a vector
    field made by :func:`make_sym_vector`."""

    def __init__(self, name, index=None):
        self.name = name
        self.index = index

    @property
    def key(self):
        return (self.name, self.index)

    def __eq__(self, other):
        return isinstance(other, Field) and other.key == self.key

    def __hash__(self):
        return hash(("Field",) + self.key)

    def __str__(self):
        return self.name if self.index is None else "%s[%d]" % (self.name, self.index)


def make_field(name):
    return Field(name)


def make_sym_vector(name, components):
    return np.array([Field(name, i) for i in range(components)], dtype=object)


make_vector_field = make_sym_vector


class BoundaryNormalComponent(Expr):
    """Component ``axis`` of the outward unit normal on boundary ``tag``."""

    def __init__(self, boundary_tag, axis):
        self.boundary_tag = boundary_tag
        self.axis = axis

    def __str__(self):
        return "normal(%s)[%d]" % (self.boundary_tag, self.axis)


def normal(tag, dimensions):
    return np.array([BoundaryNormalComponent(tag, i) for i in range(dimensions)],
                    dtype=object)


make_normal = normal


class BoundaryPair:
    """A volume vector paired with its boundary (ext-side) values on ``tag``;
    the argument of a boundary flux."""

    def __init__(self, field, bfield, tag):
        self.field = field
        self.bfield = bfield
        self.tag = tag

    def __str__(self):
        return "BPair(%s, %s, %s)" % (self.field, self.bfield, self.tag)


class OperatorBinding(Expr):
    def __init__(self, op, field):
        self.op = op
        self.field = field

    def __str__(self):
        return "%s(%s)" % (self.op, self.field)


# --------------------------------------------------------------------------
# operators

class Operator:
    """Applied with a call or by multiplication (``op * field``); applies
    itself to each entry of an object array and leaves zeros alone."""

    def __call__(self, expr):
        if isinstance(expr, np.ndarray):
            return _map_array(self.__call__, expr)
        if is_zero(expr):
            return expr
        return OperatorBinding(self, expr)

    def __mul__(self, expr):
        return self(expr)

    def _args(self):
        return ()

    def __eq__(self, other):
        return type(other) is type(self) and other._args() == self._args()

    def __hash__(self):
        return hash((type(self).__name__,) + self._args())

    def __str__(self):
        a = self._args()
        return type(self).__name__ + ("[%s]" % ",".join(str(x) for x in a) if a else "")


class DifferentiationOperator(Operator):
    """Strong-form derivative d/dx_axis (operators.py:137-139)."""

    def __init__(self, xyz_axis):
        self.xyz_axis = xyz_axis

    def _args(self):
        return (self.xyz_axis,)

    def __str__(self):
        return "d/dx%d" % self.xyz_axis


class MassOperator(Operator):
    pass


class StiffnessOperator(Operator):
    """S_x = M D_x (operators.py:133-135)."""

    def __init__(self, xyz_axis):
        self.xyz_axis = xyz_axis

    def _args(self):
        return (self.xyz_axis,)


class StiffnessTOperator(Operator):
    """Weak derivative S_x^T: (S_x^T u)_i = int u d(phi_i)/dx
    (operators.py:141-143)."""

    def __init__(self, xyz_axis):
        self.xyz_axis = xyz_axis

    def _args(self):
        return (self.xyz_axis,)

    def __str__(self):
        return "ST%d" % self.xyz_axis


class QuadratureGridUpsampler(Operator):
    """A volume (or, applied to boundary data, boundary) field sampled at
    the quadrature nodes of ``quadrature_tag`` (operators.py:262-276)."""

    def __init__(self, quadrature_tag):
        self.quadrature_tag = quadrature_tag

    def _args(self):
        return (self.quadrature_tag,)


class QuadratureInteriorFacesGridUpsampler(Operator):
    """Face traces sampled at the face quadrature nodes
    (operators.py:278-292)."""

    def __init__(self, quadrature_tag):
        self.quadrature_tag = quadrature_tag

    def _args(self):
        return (self.quadrature_tag,)


class QuadratureBoundaryGridUpsampler(Operator):
    def __init__(self, quadrature_tag, boundary_tag):
        self.quadrature_tag = quadrature_tag
        self.boundary_tag = boundary_tag

    def _args(self):
        return (self.quadrature_tag, self.boundary_tag)


class QuadratureStiffnessTOperator(Operator):
    """S_x^T with the integral taken by quadrature (operators.py:149-168)."""

    def __init__(self, xyz_axis, quadrature_tag):
        self.xyz_axis = xyz_axis
        self.quadrature_tag = quadrature_tag

    def _args(self):
        return (self.xyz_axis, self.quadrature_tag)


class InverseMassOperator(Operator):
    def __str__(self):
        return "MInv"


class ElementwiseMaxOperator(Operator):
    """Each element's nodes set to the largest of its nodal values
    (operators.py:256-257; volume_operators.hpp:356-369)."""

    def __str__(self):
        return "ElMax"


class BoundarizeOperator(Operator):
    """Restriction of a volume vector to the nodes of boundary ``tag``."""

    def __init__(self, tag):
        self.tag = tag

    def _args(self):
        return (self.tag,)


class FluxOperator(Operator):
    """Numerical flux ``flux`` (an expression of the flux language) on the
    faces, applied to a whole volume vector (interior faces) or to a
    :class:`BoundaryPair` (the boundary's faces)."""

    def __init__(self, flux, is_lift=False):
        self.flux = flux
        self.is_lift = is_lift

    def __call__(self, arg):
        if is_zero(arg):
            return 0
        return OperatorBinding(self, arg)

    def _args(self):
        return (id(self.flux), self.is_lift)

    def __str__(self):
        return "Flux{%s}" % (self.flux,)


class VectorFluxOperator:
    """Applied to an argument, gives one flux-operator binding per component
    of the flux vector (operators.py:634-657)."""

    def __init__(self, fluxes):
        self.fluxes = fluxes

    def __call__(self, arg):
        if is_zero(arg):
            return 0
        return np.array([OperatorBinding(FluxOperator(f), arg) for f in self.fluxes],
                        dtype=object)

    def __mul__(self, arg):
        return self(arg)


def get_flux_operator(flux):
    if isinstance(flux, np.ndarray):
        return VectorFluxOperator(flux)
    return FluxOperator(flux)


def make_nabla(dim):
    return np.array([DifferentiationOperator(i) for i in range(dim)], dtype=object)


def make_stiffness(dim):
    return np.array([StiffnessOperator(i) for i in range(dim)], dtype=object)


def make_stiffness_t(dim):
    return np.array([StiffnessTOperator(i) for i in range(dim)], dtype=object)


def join_fields(*args):
    out = []
    for a in args:
        if isinstance(a, np.ndarray):
            out.extend(a.reshape(-1))
        elif isinstance(a, (list, tuple)):
            out.extend(a)
        else:
            out.append(a)
    arr = np.empty(len(out), dtype=object)
    for i, x in enumerate(out):
        arr[i] = x
    return arr


def make_obj_array(items):
    return join_fields(list(items))


def cse(expr, prefix=None):
    return expr


def ptwise_dot(logdims1, logdims2, a1, a2):
    """Pointwise dot product of two object vectors (optemplate/tools.py:228-248
    for vectors: sum_k a1[k] * a2[k])."""
    if logdims1 != 1 or logdims2 != 1:
        raise NotImplementedError("ptwise_dot of vectors only")
    r = 0
    for x, y in zip(a1, a2):
        r = add(r, mul(x, y))
    return r


def cross(a, b):
    """3-vector cross product of object arrays (hedge.tools cross products
    with full subsets)."""
    return join_fields(a[1] * b[2] - a[2] * b[1],
                       a[2] * b[0] - a[0] * b[2],
                       a[0] * b[1] - a[1] * b[0])


def walk(expr):
    """Every node of a template (depth first), descending into object
    arrays, operator bindings and boundary pairs."""
    stack = [expr]
    while stack:
        x = stack.pop()
        if isinstance(x, np.ndarray):
            stack.extend(x.reshape(-1))
            continue
        yield x
        if isinstance(x, (Sum, Product)):
            stack.extend(x.children)
        elif isinstance(x, Quotient):
            stack.extend((x.num, x.den))
        elif isinstance(x, Power):
            stack.extend((x.base, x.exponent))
        elif isinstance(x, OperatorBinding):
            stack.append(x.field)
        elif isinstance(x, BoundaryPair):
            stack.extend((x.field, x.bfield))


def pretty(template):
    if isinstance(template, np.ndarray):
        return "\n".join("[%d] %s" % (i, x) for i, x in enumerate(template.reshape(-1)))
    return str(template)


__all__ = ["Field", "make_field", "make_sym_vector", "make_vector_field",
           "BoundaryPair", "BoundaryNormalComponent", "normal", "make_normal",
           "OperatorBinding", "Operator", "DifferentiationOperator", "MassOperator",
           "StiffnessOperator", "StiffnessTOperator", "QuadratureGridUpsampler",
           "QuadratureInteriorFacesGridUpsampler", "QuadratureBoundaryGridUpsampler",
           "QuadratureStiffnessTOperator", "make_stiffness", "make_stiffness_t",
           "InverseMassOperator", "ElementwiseMaxOperator", "BoundarizeOperator", "FluxOperator",
           "VectorFluxOperator", "get_flux_operator", "make_nabla", "join_fields",
           "make_obj_array", "cse", "cross", "ptwise_dot", "is_zero", "pretty", "walk"]
