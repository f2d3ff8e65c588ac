"""The reference's integration known-answer tests run through the CUDA path
(test/test_jit_discretization.py:726-912)."""
import math

import numpy as np
import pytest

import hedge_b200 as hb
from test_oracle_kat import symmetry_mesh, mirror_permutation

pytestmark = pytest.mark.gpu


def l2(discr, e):
    M = discr.ldis.mass_matrix
    e = e.reshape(discr.K, discr.Np)
    return math.sqrt(np.einsum("ki,ij,kj,k->", e, M, e, np.abs(discr.mesh.jacobians)))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_symmetry_preservation_2d_gpu(cuda_device, precision):
    """Mirror symmetry at every step: FP64 within the reference's 4e-15,
    FP32 within 4e-6."""
    mesh, v = symmetry_mesh()
    discr = hb.Discretization(mesh, order=4, precision=precision)
    perm = mirror_permutation(discr)

    def u_an(x, t):
        s = -(x @ v) + t
        return np.where(s < 0.5, 0.0, s - 0.5)
    tol = 4e-15 if precision == "fp64" else 4e-6
    for flux_type in hb.StrongAdvectionOperator.flux_types:
        op = hb.StrongAdvectionOperator(
            v, flux_type=flux_type, inflow_u=hb.TimeDependentGivenFunction(u_an))
        rhs = op.bind(discr)
        stepper = hb.LSRK4TimeStepper()
        dt = op.estimate_timestep(discr)
        u = discr.interpolate_volume_function(lambda x: u_an(x, 0.0)).reshape(1, -1)
        for step in range(int(1 / dt)):
            u = stepper(u, step * dt, dt, rhs)
            un = u[0].double().cpu().numpy()
            assert l2(discr, un - un[perm]) < tol


def test_convergence_advec_2d_gpu(cuda_device):
    v = np.array([0.27, 0.0])
    na = np.linalg.norm(v)

    def u_an(x, t):
        return np.sin(-(x @ v) / na + t * na)

    mesh = hb.make_regular_rect_mesh((0, 0), (2 * math.pi, 1), (8, 4),
                                     periodicity=(True, False),
                                     boundary_tagger=lambda *a: ["outflow"])
    for flux_type in hb.StrongAdvectionOperator.flux_types:
        errs, orders = [], [1, 2, 3, 4, 5, 6]
        for order in orders:
            discr = hb.Discretization(mesh, order=order)
            op = hb.StrongAdvectionOperator(v, flux_type=flux_type)
            rhs = op.bind(discr)
            stepper = hb.LSRK4TimeStepper()
            dt = op.estimate_timestep(discr)
            n = int(1 / dt)
            u = discr.interpolate_volume_function(lambda x: u_an(x, 0)).reshape(1, -1)
            for step in range(n):
                u = stepper(u, step * dt, dt, rhs)
            errs.append(l2(discr, u[0].cpu().numpy() - u_an(discr.nodes, n * dt)))
        lo, le = np.log10(orders), np.log10(errs)
        assert -np.polyfit(lo, le, 1)[0] > 4
        assert -np.polyfit(lo[-2:], le[-2:], 1)[0] > 10
