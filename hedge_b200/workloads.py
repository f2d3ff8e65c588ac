"""The benchmark workloads as constructors, shared by ``bench.py`` and the
full-size parity tests so that both see the same meshes and fields.

* 3D Maxwell cavity: [-1,1]^3 in n^3 cubes of 6 tetrahedra (n = 20 gives
  K = 48000), interior vertices jittered +-0.05h (seed 1), order 4, eps = mu
  = 1, upwind flux, PEC walls; the (1,1,1) mode of the cavity plus 1e-3
  uniform noise (seed 2).
* 3D acoustic wave pulse: the same mesh at order 7, c = 1, upwind flux,
  reflecting (Dirichlet) walls; a Gaussian pressure pulse of width 0.15 at
  rest.
* 2D variable-coefficient advection (the reference's var-velocity example,
  examples/advection/var-velocity.py): [-1,1]^2 in n x n squares of two
  triangles, order 5, quadrature degree 3N = 15, rotating velocity (-y, x),
  inflow u = 1 where x > 0, upwind flux; a Gaussian pulse of width 1/8 at
  (0.3, 0.5).
"""

from __future__ import annotations

import numpy as np

CAVITY_MODE = (1, 1, 1)


def box_mesh(n=20, stretch=1, seed=1):
    """[-1, -1 + 2 stretch] x [-1,1]^2 in (stretch n) x n x n cubes of 6
    tetrahedra, interior vertices jittered +-0.05 h."""
    from .mesh import make_box_tet_mesh
    h = 2.0 / n
    if stretch == 1:
        return make_box_tet_mesh(n=(n, n, n), jitter=0.05 * h, seed=seed)
    return make_box_tet_mesh(a=(-1, -1, -1), b=(-1 + 2 * stretch, 1, 1),
                             n=(n * stretch, n, n), jitter=0.05 * h, seed=seed)


def operator(workload):
    from . import models
    if workload == "wave7":
        return models.StrongWaveOperator(1.0, 3, flux_type="upwind")
    return models.MaxwellOperator(1.0, 1.0, flux_type=1)


def cavity_ic(discr):
    """(1,1,1) mode of the cavity [-1,1]^3 (reference
    examples/maxwell/analytic_solutions.py:240-300, dimensions (2,2,2),
    coordinates shifted by +1), real part at t=0, plus 1e-3 uniform noise."""
    x, y, z = (discr.nodes + 1.0).T
    f, g, h = [np.pi * m / 2.0 for m in CAVITY_MODE]
    k2 = f * f + g * g
    # zdep_add = 2 cos(hz), zdep_sub = 2i sin(hz), C = i/(f^2+g^2)
    ex = -(1.0 / k2) * f * h * np.cos(f * x) * np.sin(g * y) * 2 * np.sin(h * z)
    ey = -(1.0 / k2) * g * h * np.sin(f * x) * np.cos(g * y) * 2 * np.sin(h * z)
    ez = np.sin(f * x) * np.sin(g * y) * 2 * np.cos(h * z)
    w = np.stack([ex, ey, ez, np.zeros_like(x), np.zeros_like(x), np.zeros_like(x)])
    rng = np.random.default_rng(2)
    return w + 1e-3 * rng.uniform(-1, 1, w.shape)


def pulse_ic(discr):
    """Gaussian pressure pulse of width 0.15 at the origin, velocity 0."""
    x = discr.nodes
    w = np.zeros((4, len(discr)))
    w[0] = np.exp(-(x ** 2).sum(1) / 0.15 ** 2)
    return w


def initial_state(discr, workload="maxwell"):
    return pulse_ic(discr) if workload == "wave7" else cavity_ic(discr)


def varadv_problem(n=400, order=5, device=None, precision="fp64"):
    """(discretization, operator, initial u) of the 2D variable-coefficient
    advection workload."""
    from . import models
    from .discretization import Discretization
    from .mesh import make_regular_rect_mesh
    mesh = make_regular_rect_mesh((-1, -1), (1, 1), (n, n))
    d = Discretization(mesh, order=order, precision=precision, device=device,
                       quad_min_degrees={"quad": 3 * order})
    vf = models.TimeConstantGivenFunction(lambda x: np.stack([-x[:, 1], x[:, 0]]))
    bf = models.TimeConstantGivenFunction(lambda x: (x[:, 0] > 0).astype(np.float64))
    op = models.VariableCoefficientAdvectionOperator(2, vf, bc_u_f=bf, flux_type="upwind")
    x = d.nodes
    u0 = np.exp(-64 * np.sum((x - np.array([0.3, 0.5])) ** 2, axis=1))
    return d, op, u0
