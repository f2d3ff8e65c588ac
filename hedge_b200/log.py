"""Log quantities of device fields (hedge/log.py:43-286).

pytools.log is not available, so this module carries a minimal
``LogQuantity`` / ``MultiLogQuantity`` base and an in-memory ``LogManager``
(``add_quantity``, ``tick``, ``get_series``, ``save``), enough to record
the reference's quantities step by step:

* ``Integral(getter, discr)`` -- volume integral (sum of integrals of |v_i|
  for a vector), ``LpNorm(getter, discr, p)``;
* ``EMFieldGetter(discr, maxwell_op, fgetter)`` and the electromagnetic
  quantities ``ElectricFieldEnergy`` (1/2 int E.eps E), ``MagneticFieldEnergy``
  (1/2 int H.mu H), ``EMFieldMomentum`` (int E x H / c0^2),
  ``EMFieldDivergenceD`` (int div eps E) and ``EMFieldDivergenceB``
  (int div mu H, int |div mu H|), with ``add_em_energies`` /
  ``add_em_quantities``.

Pointwise products stay on the device (torch); integrals are the
discretization's mass-weighted sums (``Discretization.integral``) and
divergences the DG divergence (``hedge_b200.nd_calculus``).
"""

from __future__ import annotations

import json

import numpy as np


def _torch():
    import torch
    return torch


def axis_name(axis):
    return "xyz"[axis] if 0 <= axis < 3 else _raise(axis)


def _raise(axis):
    raise RuntimeError("invalid axis index %r" % (axis,))


class LogQuantity:
    """A named scalar sampled once per tick."""

    sort_weight = 0

    def __init__(self, name, unit=None, description=None):
        self.name, self.unit, self.description = name, unit, description

    @property
    def default_aggregator(self):
        return None

    def __call__(self):
        raise NotImplementedError


class MultiLogQuantity:
    """Several named scalars sampled together."""

    def __init__(self, names, units=None, descriptions=None):
        self.names = list(names)
        self.units = units or [None] * len(self.names)
        self.descriptions = descriptions or [None] * len(self.names)

    def __call__(self):
        raise NotImplementedError


class LogManager:
    """In-memory log: each ``tick()`` samples every quantity once."""

    def __init__(self):
        self.quantities = []
        self.series = {}
        self.tick_count = 0
        self.constants = {}

    def add_quantity(self, q):
        self.quantities.append(q)
        for n in (q.names if isinstance(q, MultiLogQuantity) else [q.name]):
            self.series.setdefault(n, [])

    def set_constant(self, name, value):
        self.constants[name] = value

    def tick(self):
        for q in self.quantities:
            v = q()
            if isinstance(q, MultiLogQuantity):
                for n, x in zip(q.names, v):
                    self.series[n].append((self.tick_count, _scalar(x)))
            else:
                self.series[q.name].append((self.tick_count, _scalar(v)))
        self.tick_count += 1

    def get_series(self, name):
        return [v for _, v in self.series[name]]

    def save(self, path):
        with open(path, "w") as f:
            json.dump({"constants": self.constants, "series": self.series}, f)

    def close(self):
        pass


def _scalar(x):
    if hasattr(x, "item"):
        return float(x.item()) if getattr(x, "numel", lambda: 1)() == 1 else \
            np.asarray(x.detach().cpu() if hasattr(x, "detach") else x).tolist()
    if isinstance(x, (list, tuple, np.ndarray)):
        return [float(y) for y in np.asarray(x).reshape(-1)]
    return float(x)


def _rows(var):
    """A field as a list of volume vectors (1 for a scalar field)."""
    torch = _torch()
    if isinstance(var, (list, tuple)) or (isinstance(var, np.ndarray) and var.dtype == object):
        return list(var)
    if isinstance(var, torch.Tensor) and var.dim() == 2:
        return [var[i] for i in range(var.shape[0])]
    if isinstance(var, np.ndarray) and var.ndim == 2:
        return list(var)
    return None


class Integral(LogQuantity):
    def __init__(self, getter, discr, name=None, unit="1", description=None):
        self.getter = getter
        if name is None:
            try:
                name = "int_%s" % self.getter.name()
            except AttributeError:
                raise ValueError("must specify a name")
        super().__init__(name, unit, description)
        self.discr = discr

    @property
    def default_aggregator(self):
        return sum

    def __call__(self):
        var = self.getter()
        rows = _rows(var)
        if rows is not None:
            return sum(self.discr.integral(_abs(v)) for v in rows)
        return self.discr.integral(var)


class LpNorm(LogQuantity):
    def __init__(self, getter, discr, p=2, name=None, unit="1", description=None):
        self.getter, self.discr, self.p = getter, discr, p
        if name is None:
            try:
                name = "l%d_%s" % (int(p), self.getter.name())
            except AttributeError:
                raise ValueError("must specify a name")
        super().__init__(name, unit, description)

    def __call__(self):
        return self.discr.norm(self.getter(), self.p)


def _abs(v):
    torch = _torch()
    return torch.abs(v) if isinstance(v, torch.Tensor) else np.abs(v)


# -- electromagnetic quantities ----------------------------------------------------

class EMFieldGetter:
    """E and H of the current fields (``fgetter()``), split by the operator."""

    def __init__(self, discr, maxwell_op, fgetter):
        self.discr, self.maxwell_op, self.fgetter = discr, maxwell_op, fgetter

    def _dev(self):
        f = self.fgetter()
        torch = _torch()
        if not isinstance(f, torch.Tensor):
            f = self.discr.to_device(f, torch.float64)
        return f.reshape(6, len(self.discr))

    @property
    def e(self):
        return self.maxwell_op.split_eh(self._dev())[0]

    @property
    def h(self):
        return self.maxwell_op.split_eh(self._dev())[1]


class ElectricFieldEnergy(LogQuantity):
    def __init__(self, fields, name="W_el"):
        super().__init__(name, "J", "Energy of the electric field")
        self.fields = fields

    def __call__(self):
        op = self.fields.maxwell_op
        e = self.fields.e
        return self.fields.discr.integral(0.5 * op.epsilon * (e * e).sum(0))


class MagneticFieldEnergy(LogQuantity):
    def __init__(self, fields, name="W_mag"):
        super().__init__(name, "J", "Energy of the magnetic field")
        self.fields = fields

    def __call__(self):
        op = self.fields.maxwell_op
        h = self.fields.h
        return self.fields.discr.integral(0.5 * op.mu * (h * h).sum(0))


class EMFieldMomentum(MultiLogQuantity):
    def __init__(self, fields, c0, names=None):
        names = names or ["p%s_field" % axis_name(i) for i in range(3)]
        super().__init__(names, units=["N*s"] * 3, descriptions=["Field Momentum"] * 3)
        self.fields, self.c0 = fields, c0

    def __call__(self):
        torch = _torch()
        e, h = self.fields.e, self.fields.h
        s = torch.linalg.cross(e, h, dim=0)
        return [self.fields.discr.integral(s[i] / self.c0 ** 2) for i in range(3)]


class EMFieldDivergenceD(LogQuantity):
    def __init__(self, maxwell_op, fields, name="divD"):
        super().__init__(name, "C", "Integral over div D")
        from .nd_calculus import DivergenceOperator
        self.fields = fields
        self.div = DivergenceOperator(maxwell_op.dimensions).bind(fields.discr,
                                                                  precision="fp64")

    def __call__(self):
        op = self.fields.maxwell_op
        return self.fields.discr.integral(self.div(op.epsilon * self.fields.e))


class EMFieldDivergenceB(MultiLogQuantity):
    def __init__(self, maxwell_op, fields, names=None):
        from .nd_calculus import DivergenceOperator
        self.fields = fields
        self.div = DivergenceOperator(maxwell_op.dimensions).bind(fields.discr,
                                                                  precision="fp64")
        super().__init__(names or ["divB", "err_divB_l1"], units=["T/m", "T/m"],
                         descriptions=["Integral over div B", "Integral over |div B|"])

    def __call__(self):
        op = self.fields.maxwell_op
        div_b = self.div(op.mu * self.fields.h)
        d = self.fields.discr
        return [d.integral(div_b), d.integral(_abs(div_b))]


def add_em_energies(mgr, maxwell_op, fields):
    mgr.add_quantity(ElectricFieldEnergy(fields))
    mgr.add_quantity(MagneticFieldEnergy(fields))


def add_em_quantities(mgr, maxwell_op, fields):
    add_em_energies(mgr, maxwell_op, fields)
    mgr.add_quantity(EMFieldMomentum(fields, maxwell_op.c))
    mgr.add_quantity(EMFieldDivergenceD(maxwell_op, fields))
    mgr.add_quantity(EMFieldDivergenceB(maxwell_op, fields))


__all__ = ["LogQuantity", "MultiLogQuantity", "LogManager", "Integral", "LpNorm",
           "EMFieldGetter", "ElectricFieldEnergy", "MagneticFieldEnergy",
           "EMFieldMomentum", "EMFieldDivergenceD", "EMFieldDivergenceB",
           "add_em_energies", "add_em_quantities", "axis_name"]
