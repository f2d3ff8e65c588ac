"""The full-size benchmark configurations against the CPU oracle.

C2: 3D Maxwell, [-1,1]^3 in 20^3 cubes x 6 tetrahedra (K = 48000), jitter
+-0.05h (seed 1), N = 4, upwind flux, PEC walls, the (1,1,1) cavity mode +
1e-3 noise (seed 2).  C3: the same mesh at N = 7, acoustic wave c = 1,
upwind, reflecting walls, Gaussian pressure pulse of width 0.15.  Both are
built by hedge_b200.workloads, exactly as bench.py builds them.

Per configuration the oracle runs one trajectory of 20 LSRK4 steps at half
the CFL estimate (its first RHS, at t = 0, is the one-RHS check), and every
GPU path is compared with it: one RHS (FP64 <= 1e-12, FP32 <= 1e-5,
FP16x3 <= 1e-6 relative L2) and the state after the 20 steps (FP64 <= 1e-11,
FP32 <= 1e-5, FP16x3 <= 1e-6).  The reference's CPU-vs-GPU pattern is
test/test_cuda.py:57-119."""
import os

import numpy as np
import pytest

import hedge_b200 as hb
from hedge_b200 import workloads as W
from conftest import rel_l2

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

NSTEPS = 20
RHS_TOL = {"fp64": 1e-12, "fp32": 1e-5, "fp16x3": 1e-6}
STEP_TOL = {"fp64": 1e-11, "fp32": 1e-5, "fp16x3": 1e-6}

_cache = {}


def _oracle_run(workload, order):
    """(mesh, w0, dt, oracle rhs at t=0, oracle state after NSTEPS), once."""
    key = (workload, order)
    if key not in _cache:
        from oracle import OracleRHS, set_threads
        set_threads(os.cpu_count() or 1)
        mesh = W.box_mesh(20)
        d = hb.Discretization(mesh, order=order)
        assert d.K == 48000
        op = W.operator(workload)
        w0 = W.initial_state(d, workload)
        dt = 0.5 * op.estimate_timestep(d)
        orc = OracleRHS(d, op.op_template())
        r0 = orc(w0)
        y, res, t = w0.copy(), np.zeros_like(w0), 0.0
        for _ in range(NSTEPS):
            y, res = orc.lsrk4_step(y, t, dt, res)
            t += dt
        _cache[key] = (mesh, op, w0, dt, r0, y)
    return _cache[key]


def _gpu_run(workload, order, precision):
    import torch
    mesh, op, w0, dt, r0, y_ref = _oracle_run(workload, order)
    d = hb.Discretization(mesh, order=order, precision=precision)
    rhs = op.bind(d)
    F = w0.shape[0]
    r = rhs(0.0, w0).double().cpu().numpy()
    rhs.compiled.check()
    st = hb.LSRK4TimeStepper()
    y = d.to_device(w0).reshape(F, -1)
    t = 0.0
    for _ in range(NSTEPS):
        y = st(y, t, dt, rhs)
        t += dt
    rhs.compiled.check()
    assert torch.isfinite(y).all()
    return rel_l2(r, r0), rel_l2(y.double().cpu().numpy(), y_ref)


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp16x3"])
def test_c2_maxwell_K48000_N4(cuda_device, precision):
    e_rhs, e_steps = _gpu_run("maxwell", 4, precision)
    print("C2 %s: rel-L2 1 RHS %.2e, %d steps %.2e" % (precision, e_rhs, NSTEPS, e_steps))
    assert e_rhs <= RHS_TOL[precision]
    assert e_steps <= STEP_TOL[precision]


@pytest.mark.parametrize("precision", ["fp64", "fp16x3"])
def test_c3_wave_K48000_N7(cuda_device, precision):
    e_rhs, e_steps = _gpu_run("wave7", 7, precision)
    print("C3 %s: rel-L2 1 RHS %.2e, %d steps %.2e" % (precision, e_rhs, NSTEPS, e_steps))
    assert e_rhs <= RHS_TOL[precision]
    assert e_steps <= STEP_TOL[precision]
