"""LSRK4 steps replayed from a CUDA graph (GraphedLSRK4) against the eager
fused stepper: the same kernels in the same order, so the states agree
bitwise; operators that need host data per stage are refused."""
import time

import numpy as np
import pytest

import hedge_b200 as hb
from test_gpu_parity import _fields, box, rect

pytestmark = pytest.mark.gpu


def _compare(d, op, nsteps, seed):
    import torch
    rhs = op.bind(d)
    F = op.descriptor().n_fields
    q = _fields(d, F, seed)
    dt = 0.5 * op.estimate_timestep(d)
    st = hb.LSRK4TimeStepper()
    y = d.to_device(q).reshape(F, -1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for n in range(nsteps):
        y = st(y, n * dt, dt, rhs)
    torch.cuda.synchronize()
    t_eager = time.perf_counter() - t0
    g = hb.GraphedLSRK4(rhs, d.to_device(q).reshape(F, -1), dt)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(nsteps):
        yg = g.step()
    torch.cuda.synchronize()
    t_graph = time.perf_counter() - t0
    rhs.compiled.check()
    return bool(torch.equal(y, yg)), t_eager, t_graph


def test_graphed_wave_2d_fp64(cuda_device):
    d = hb.Discretization(rect(9, False, 0.02, 1), order=4)
    same, te, tg = _compare(d, hb.StrongWaveOperator(1.0, 2, flux_type="upwind"), 20, 1)
    print("wave 2D FP64, 20 steps: eager %.2f ms, graph %.2f ms" % (te * 1e3, tg * 1e3))
    assert same


def test_graphed_maxwell_fp16x3(cuda_device):
    d = hb.Discretization(box(2, 0.05, 1), order=4, precision="fp16x3")
    same, te, tg = _compare(d, hb.MaxwellOperator(1.0, 1.0, flux_type=1), 10, 2)
    print("maxwell FP16x3, 10 steps: eager %.2f ms, graph %.2f ms" % (te * 1e3, tg * 1e3))
    assert same


def test_graphed_periodic_advection_small_mesh(cuda_device):
    """The reference's CPU-sized configuration: 2D periodic advection, N = 4,
    K = 3200; prints the time per step eager and replayed."""
    m = hb.make_regular_rect_mesh((-1, -1), (1, 1), (41, 41), periodicity=(True, True),
                                  jitter=0.1 * 2 / 40, seed=0)
    d = hb.Discretization(m, order=4)
    op = hb.StrongAdvectionOperator(np.array([1.0, 0.5]), flux_type="upwind")
    same, te, tg = _compare(d, op, 100, 3)
    print("advection 2D K=%d FP64, 100 steps: eager %.2f ms, graph %.2f ms"
          % (d.K, te * 1e3, tg * 1e3))
    assert same


def test_graphed_refuses_time_dependent_inflow(cuda_device):
    from test_optemplate import _in_out_tagger
    from test_optemplate import rect as tagged_rect
    v = np.array([0.7, -0.4])
    d = hb.Discretization(tagged_rect(6, tagger=_in_out_tagger(v)), order=3)
    op = hb.StrongAdvectionOperator(v, inflow_tag="in", outflow_tag="out", flux_type="upwind")
    rhs = op.bind(d)
    with pytest.raises(ValueError):
        hb.GraphedLSRK4(rhs, d.to_device(np.zeros((1, len(d)))).reshape(1, -1), 1e-3)


def test_graphed_variable_coefficient_kept_and_guarded(cuda_device):
    """The recorded stages read the c field and the source at their addresses
    at construction: the stepper keeps those tensors alive (replays after the
    caller dropped its own references stay bitwise equal to the eager
    stepper), and a coefficient set after construction makes step() raise
    instead of replaying against freed memory."""
    import gc
    import torch
    d = hb.Discretization(rect(7, False, 0.02, 4), order=3)
    rng = np.random.default_rng(5)
    c = rng.uniform(0.8, 1.2, len(d))
    src = 0.1 * rng.uniform(-1, 1, len(d))
    op = hb.VariableVelocityStrongWaveOperator(c, 2, flux_type="upwind", source=src)
    rhs = op.bind(d)
    q = _fields(d, 3, 6)
    dt = 0.5 * op.estimate_timestep(d)
    g = hb.GraphedLSRK4(rhs, d.to_device(q).reshape(3, -1), dt)
    st = hb.LSRK4TimeStepper()
    y = d.to_device(q).reshape(3, -1)
    for n in range(5):
        y = st(y, n * dt, dt, rhs)
    # churn the caching allocator: freed blocks of the c/source size get reused
    junk = [torch.full((len(d),), 7.0, dtype=torch.float64, device=d.device)
            for _ in range(8)]
    del junk
    gc.collect()
    for _ in range(5):
        yg = g.step()
    g.check()
    assert torch.equal(y, yg)
    rhs.compiled.set_coefficient(np.ones(len(d)))
    with pytest.raises(RuntimeError):
        g.step()
