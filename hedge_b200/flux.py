"""The flux language: numerical fluxes as expressions of the interior and
exterior face values of the flux argument and of the face normal.

Follows hedge/flux/__init__.py:38-263: ``FieldComponent(i, is_interior)``
leaves reached through ``FluxScalarPlaceholder(i).int / .ext / .avg`` and
``FluxVectorPlaceholder(n)``, ``Normal(axis)`` leaves from ``make_normal``,
``FluxConstantPlaceholder``, ``IfPositive`` (pymbolic.primitives.IfPositive)
and the function symbols ``Abs``, ``Max``, ``Min``.  The penalty-term leaves
(face / element Jacobian, element order, local mesh size) exist so that
templates using them build; the lowering rejects them, since no flux on
this path uses them.
"""

from __future__ import annotations

import numpy as np

from .optemplate import Expr


class FieldComponent(Expr):
    def __init__(self, index, is_interior):
        self.index = index
        self.is_interior = is_interior

    def __str__(self):
        return "%s%d" % ("int" if self.is_interior else "ext", self.index)


class Normal(Expr):
    def __init__(self, axis):
        self.axis = axis

    def __str__(self):
        return "n%d" % self.axis


class IfPositive(Expr):
    """``then`` where ``criterion > 0``, else ``else_``."""

    def __init__(self, criterion, then, else_):
        self.criterion, self.then, self.else_ = criterion, then, else_

    def __str__(self):
        return "if_pos(%s, %s, %s)" % (self.criterion, self.then, self.else_)


class FunctionCall(Expr):
    def __init__(self, name, args):
        self.name, self.args = name, tuple(args)

    def __str__(self):
        return "%s(%s)" % (self.name, ", ".join(str(a) for a in self.args))


class _FluxFunction:
    name = None
    arg_count = 1

    def __call__(self, *args):
        if len(args) != self.arg_count:
            raise TypeError("%s takes %d arguments" % (self.name, self.arg_count))
        return FunctionCall(self.name, args)


class Abs(_FluxFunction):
    name, arg_count = "abs", 1


class Max(_FluxFunction):
    name, arg_count = "max", 2


class Min(_FluxFunction):
    name, arg_count = "min", 2


flux_abs = Abs()
flux_max = Max()
flux_min = Min()


class _PenaltyLeaf(Expr):
    def __init__(self, is_interior=True):
        self.is_interior = is_interior

    def __str__(self):
        return type(self).__name__


class FaceJacobian(_PenaltyLeaf):
    pass


class ElementJacobian(_PenaltyLeaf):
    pass


class ElementOrder(_PenaltyLeaf):
    pass


class LocalMeshSize(_PenaltyLeaf):
    pass


def make_penalty_term(power=1):
    return (ElementOrder() ** 2 / LocalMeshSize()) ** power


PenaltyTerm = make_penalty_term


def norm(v):
    return np.dot(v, v) ** 0.5


def make_normal(dimensions):
    return np.array([Normal(i) for i in range(dimensions)], dtype=object)


class FluxConstantPlaceholder:
    def __init__(self, constant):
        self.constant = constant

    @property
    def int(self):
        return self.constant

    @property
    def ext(self):
        return self.constant

    @property
    def avg(self):
        return self.constant


class FluxZeroPlaceholder(FluxConstantPlaceholder):
    def __init__(self):
        super().__init__(0)


class FluxScalarPlaceholder:
    def __init__(self, component=0):
        self.component = component

    @property
    def int(self):
        return FieldComponent(self.component, True)

    @property
    def ext(self):
        return FieldComponent(self.component, False)

    @property
    def avg(self):
        return 0.5 * (self.int + self.ext)


class FluxVectorPlaceholder:
    def __init__(self, components=None, scalars=None):
        if (components is None) == (scalars is None):
            raise ValueError("exactly one of components and scalars must be given")
        if components is not None:
            self.scalars = [FluxScalarPlaceholder(i) for i in range(components)]
        else:
            self.scalars = list(scalars)

    def __len__(self):
        return len(self.scalars)

    def __getitem__(self, idx):
        if isinstance(idx, (int, np.integer)):
            return self.scalars[idx]
        return FluxVectorPlaceholder(scalars=self.scalars[idx])

    def _arr(self, attr):
        out = np.empty(len(self.scalars), dtype=object)
        for i, s in enumerate(self.scalars):
            out[i] = getattr(s, attr)
        return out

    @property
    def int(self):
        return self._arr("int")

    @property
    def ext(self):
        return self._arr("ext")

    @property
    def avg(self):
        return self._arr("avg")


__all__ = ["FieldComponent", "Normal", "IfPositive", "FunctionCall", "Abs", "Max",
           "Min", "flux_abs", "flux_max", "flux_min", "FaceJacobian", "ElementJacobian",
           "ElementOrder", "LocalMeshSize", "make_penalty_term", "PenaltyTerm", "norm",
           "make_normal", "FluxConstantPlaceholder", "FluxZeroPlaceholder",
           "FluxScalarPlaceholder", "FluxVectorPlaceholder"]
