"""DG gradient and divergence (hedge/models/nd_calculus.py:35-137).

``GradientOperator(d)`` computes grad u - M^-1 (flux(u) + boundary flux)
with the flux (u.int - u.avg) n and the boundary value u itself, and
``DivergenceOperator(d)`` the same for div v with (v.int - v.avg).n.
``op_template()`` builds the reference's templates.

Both equal pieces of the central-flux wave right-hand side with c = 1
(wave.py:80-108): the wave RHS is (div v, grad u) + M^-1 (flux), and its
central flux is -(v.int - v.avg).n for u and -(u.int - u.avg) n for v.  With
Neumann walls the wave's ext u on the boundary is u itself; with Dirichlet
walls its ext v is v itself.  So ``bind`` evaluates them with the wave
kernel: the gradient is the v-part of the wave RHS of (u, 0) with Neumann
walls, the divergence the u-part of the wave RHS of (0, v) with Dirichlet
walls.  The tests check the identity on the CPU (template executor) and the
compiled result on the GPU.
"""

from __future__ import annotations

import numpy as np

from . import flux as fl
from . import optemplate as ot
from .mesh import TAG_ALL, TAG_NONE


class GradientOperator:
    def __init__(self, dimensions):
        self.dimensions = dimensions

    def flux(self):
        u = fl.FluxScalarPlaceholder()
        normal = fl.make_normal(self.dimensions)
        return u.int * normal - u.avg * normal

    def op_template(self):
        u, bc = ot.Field("u"), ot.Field("bc")
        nabla = ot.make_nabla(self.dimensions)
        flux_op = ot.get_flux_operator(self.flux())
        return nabla * u - ot.InverseMassOperator()(
            flux_op(u) + flux_op(ot.BoundaryPair(u, bc, TAG_ALL)))

    def bind(self, discr, precision=None):
        from .models import StrongWaveOperator
        d = self.dimensions
        comp = discr.compile(StrongWaveOperator(1.0, d, flux_type="central",
                                                dirichlet_tag=TAG_NONE,
                                                neumann_tag=TAG_ALL).descriptor(),
                             precision=precision)

        def op(u):
            torch = _torch()
            u = discr.to_device(u, comp.state_dtype).reshape(-1)
            w = torch.zeros((d + 1, len(discr)), dtype=comp.state_dtype, device=u.device)
            w[0] = u
            return comp(w=w)[1:]

        return op


class DivergenceOperator:
    def __init__(self, dimensions, subset=None):
        self.dimensions = dimensions
        self.subset = [True] * dimensions if subset is None else list(subset)[:dimensions]
        if not all(self.subset):
            raise NotImplementedError("divergence of a component subset")
        self.arg_count = dimensions

    def flux(self):
        v = fl.FluxVectorPlaceholder(self.arg_count)
        normal = fl.make_normal(self.dimensions)
        d = v.int - v.avg
        return sum(d[i] * normal[i] for i in range(self.dimensions))

    def op_template(self):
        nabla = ot.make_nabla(self.dimensions)
        v = ot.make_sym_vector("v", self.arg_count)
        bc = ot.make_sym_vector("bc", self.arg_count)
        local = sum(nabla[i] * v[i] for i in range(self.dimensions))
        flux_op = ot.get_flux_operator(self.flux())
        return local - ot.InverseMassOperator()(
            flux_op(v) + flux_op(ot.BoundaryPair(v, bc, TAG_ALL)))

    def bind(self, discr, precision=None):
        from .models import StrongWaveOperator
        d = self.dimensions
        comp = discr.compile(StrongWaveOperator(1.0, d, flux_type="central",
                                                dirichlet_tag=TAG_ALL).descriptor(),
                             precision=precision)

        def op(v):
            torch = _torch()
            if isinstance(v, (list, tuple)) or (isinstance(v, np.ndarray) and v.dtype == object):
                v = torch.stack([discr.to_device(x, comp.state_dtype).reshape(-1) for x in v])
            v = discr.to_device(v, comp.state_dtype).reshape(d, -1)
            w = torch.zeros((d + 1, len(discr)), dtype=comp.state_dtype, device=v.device)
            w[1:] = v
            return comp(w=w)[0]

        return op


def _torch():
    import torch
    return torch


__all__ = ["GradientOperator", "DivergenceOperator"]
