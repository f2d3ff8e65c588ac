"""Batched ensemble (hb_batch_*): one launch per LSRK stage over members of
mixed order, size and model.

* one step of every member against the CPU oracle (FP64 RHS, the same LSRK4
  recurrences) from the same FP32 initial state: the step's increment agrees
  to rel-L2 <= 1e-5 (FP32 right-hand side);
* a member advanced inside the batch equals the same member advanced alone,
  bit for bit, and CUDA-graph replay equals eager launches bit for bit;
* the autotuner returns a tile size among its candidates;
* members the batch kernel does not cover are refused with a status.
"""
import ctypes as C

import numpy as np
import pytest

import hedge_b200 as hb
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _members(seed=3):
    from hedge_b200.ensemble import _rect_member
    rng = np.random.default_rng(seed)
    spec = [(120, 3, "advection"), (300, 4, "wave"), (60, 5, "advection"),
            (200, 6, "wave"), (90, 6, "advection"), (150, 3, "wave")]
    return [_rect_member(k, o, m, rng) for k, o, m in spec]


def test_ensemble_step_matches_oracle(cuda_device):
    from oracle import OracleRHS
    from hedge_b200.ensemble import Ensemble
    from hedge_b200.timestep import RK4A, RK4B
    ms = _members()
    ens = Ensemble(ms)
    ens.step(1)
    ens.check()
    for k, m in enumerate(ms):
        q = m.q0.astype(np.float32).astype(np.float64)
        orc = OracleRHS(m.discr, m.model.op_template())
        res = np.zeros_like(q)
        y = q.copy()
        for s in range(5):
            res = RK4A[s] * res + m.dt * orc(y)
            y = y + RK4B[s] * res
        got = ens.state(k).double().cpu().numpy()
        err = rel_l2(got - q, y - q)
        assert err <= 1e-5, (k, err)


def test_ensemble_member_independent_and_graph_equals_eager(cuda_device):
    import torch
    from hedge_b200.ensemble import Ensemble
    ms = _members(5)
    a = Ensemble(ms)
    a.step(3)
    alone = Ensemble([ms[3]])
    alone.step(3)
    assert torch.equal(a.state(3), alone.state(0))
    b = Ensemble(ms)
    b.capture()
    b.step(3)
    b.check()
    for k in range(len(ms)):
        assert torch.equal(a.state(k), b.state(k)), k


def test_ensemble_tile_sizes_do_not_change_results(cuda_device):
    import torch
    from hedge_b200.ensemble import Ensemble
    ms = _members(7)[:3]
    r1 = Ensemble(ms, tiles={m.key: 1 for m in ms})
    r2 = Ensemble(ms, tiles={m.key: 37 for m in ms})
    r1.step(2)
    r2.step(2)
    for k in range(3):
        assert torch.equal(r1.state(k), r2.state(k)), k


def test_autotune_small(cuda_device):
    from hedge_b200.ensemble import autotune
    ms = _members(9)[:3]
    table, res = autotune(ms, budgets=(64, 256), steps=1, table={})
    assert set(table) == {m.key for m in ms}
    for k, E in table.items():
        assert E in res[k]


def test_ensemble_refuses_unsupported_member(cuda_device):
    import torch
    from hedge_b200 import _native
    d = hb.Discretization(hb.make_regular_rect_mesh((-1, -1), (1, 1), (4, 4)), order=2)
    c = np.ones(len(d))
    comp = d.compile(hb.VariableVelocityStrongWaveOperator(c, 2).op_template(),
                     precision="fp32")
    q = torch.zeros((3, len(d)), dtype=torch.float32, device=d.device)
    r = torch.zeros((3, len(d)), dtype=torch.float64, device=d.device)
    arr = (_native.hb_batch_member * 1)()
    arr[0] = _native.hb_batch_member(comp._handle, q.data_ptr(), q.data_ptr(), r.data_ptr(),
                                     0.01, 0)
    h = C.c_void_p()
    st = _native.load().hb_batch_create(C.cast(arr, C.c_void_p), 1, C.byref(h))
    assert st == _native.HB_ERR_UNSUPPORTED
