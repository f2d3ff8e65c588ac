"""Failure detection on the GPU without a GPU fault: a bounded device wait is
made to run out (an mbarrier that nothing arrives on, hb_op_wait_selftest),
the kernel raises the operator's device error flag and returns, hb_op_check
reports HB_ERR_DEVICE_FLAG once, and the same operator's next tensor-core
launch runs normally and matches the oracle.  The tensor-core kernels use the
same bounded wait (tc::mbar_wait) on every MMA and data hand-off."""
import time

import numpy as np
import pytest

import hedge_b200 as hb
from hedge_b200 import _native
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _maxwell(precision):
    d = hb.Discretization(hb.make_box_tet_mesh(n=(2, 2, 2), jitter=0.03, seed=8), order=4,
                          precision=precision)
    op = hb.MaxwellOperator(1.0, 1.0, flux_type=1)
    rng = np.random.default_rng(1)
    w = np.sin(d.nodes.T[[0, 1, 2, 2, 0, 1]]) + 0.05 * rng.uniform(-1, 1, (6, len(d)))
    return d, op, w


def test_bounded_wait_runs_out_and_operator_recovers(cuda_device):
    import torch
    from oracle import OracleRHS
    d, op, w = _maxwell("fp16x3")
    rhs = op.bind(d)
    comp = rhs.compiled
    ref = OracleRHS(d, op.op_template())(w)
    assert rel_l2(rhs(0.0, w).cpu().numpy(), ref) <= 1e-6
    comp.check()
    lib = _native.load()
    stream = torch.cuda.current_stream(d.device).cuda_stream
    limit_ns = 20_000_000          # 20 ms
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _native.check(lib.hb_op_wait_selftest(comp._handle, limit_ns, stream))
    torch.cuda.synchronize()
    waited = time.perf_counter() - t0
    # the wait ended by its limit, not by anything arriving
    assert waited >= 0.9 * limit_ns * 1e-9
    assert waited < 2.0
    st = lib.hb_op_check(comp._handle, stream)
    assert st == _native.HB_ERR_DEVICE_FLAG
    assert b"bounded wait ran out" in lib.hb_last_error_string()
    # reported once, then cleared; the context and the operator still work
    assert lib.hb_op_check(comp._handle, stream) == _native.HB_OK
    got = rhs(0.0, w).cpu().numpy()
    comp.check()
    assert rel_l2(got, ref) <= 1e-6
    y = hb.LSRK4TimeStepper()(d.to_device(w).reshape(6, -1), 0.0,
                              0.5 * op.estimate_timestep(d), rhs)
    comp.check()
    assert torch.isfinite(y).all()


def test_wait_selftest_rejects_bad_limits(cuda_device):
    d, op, w = _maxwell("fp64")
    comp = op.bind(d).compiled
    lib = _native.load()
    assert lib.hb_op_wait_selftest(comp._handle, 10, None) == _native.HB_ERR_INVALID_ARGUMENT
    assert lib.hb_op_wait_selftest(comp._handle, 3_000_000_000, None) == \
        _native.HB_ERR_INVALID_ARGUMENT
    assert lib.hb_op_wait_selftest(None, 1_000_000, None) == _native.HB_ERR_INVALID_ARGUMENT
