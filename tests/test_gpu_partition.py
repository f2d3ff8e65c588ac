"""Element-partitioned operators on one GPU: each part's RHS / LSRK stage,
with its cut faces read from the halo buffer that hb_pack + the exchange
filled, equals the unpartitioned operator's on the same elements (FP64:
bitwise; FP32: <= 1e-6 relative)."""
import numpy as np
import pytest

import hedge_b200 as hb
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _setup(kind, nparts, precision):
    from hedge_b200.partition import LocalExchange, PartitionPlan, PartitionedOperator
    if kind == "maxwell":
        d = hb.Discretization(hb.make_box_tet_mesh(n=(3, 3, 3), jitter=0.03, seed=5), order=3)
        model = hb.MaxwellOperator(1.0, 1.0, flux_type=1)
    elif kind == "maxwell_incident":
        def tagger(fvi, el, fn, allv):
            return ["inc"] if allv[list(fvi)].mean(0)[0] > 0.99 else ["pec"]
        m = hb.make_box_tet_mesh(n=(3, 3, 3), jitter=0.03, seed=5, boundary_tagger=tagger)
        d = hb.Discretization(m, order=3)
        model = hb.MaxwellOperator(1.0, 1.0, flux_type=0.5, pec_tag="pec", incident_tag="inc")
    else:
        m = hb.make_regular_rect_mesh((-1, -1), (1, 1), (9, 9), jitter=0.02, seed=4)
        d = hb.Discretization(m, order=4)
        c = np.repeat(np.random.default_rng(4).uniform(0.8, 1.2, d.K), d.Np)
        model = hb.VariableVelocityStrongWaveOperator(c, 2, flux_type="upwind")
    plan = PartitionPlan(d, model.op_template(), nparts)
    parts = [PartitionedOperator(d, model, plan, r, precision=precision) for r in range(nparts)]
    return d, model, plan, parts, LocalExchange(plan, parts)


@pytest.mark.parametrize("by_ranges", [False, True])
@pytest.mark.parametrize("kind", ["maxwell", "maxwell_incident", "varwave"])
@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32-simt", "fp16x3", "bf16x3"])
def test_partitioned_rhs_equals_global(cuda_device, kind, precision, by_ranges):
    import torch
    d, model, plan, parts, ex = _setup(kind, 3, precision)
    F = model.descriptor().n_fields
    q = np.random.default_rng(1).standard_normal((F, len(d)))
    comp = d.compile(model.op_template(), precision=precision)
    if kind == "varwave":
        comp.set_coefficient(model.c)
    ref = comp(w=q).double().cpu().numpy().reshape(F, -1)
    ql = [p.scatter(q) for p in parts]
    for p, x in zip(parts, ql):
        p.pack(x)
    ex.exchange_all()
    for p, x in zip(parts, ql):
        got = p.rhs(x, exchanged=True, by_ranges=by_ranges)
        p.check()
        want = ref[:, p.local_nodes()]
        g = got.double().cpu().numpy()
        if precision in ("fp32", "fp32-simt"):
            assert rel_l2(g, want) <= 1e-6
        else:
            # per-row arithmetic does not depend on the batch an element lands in
            assert rel_l2(g, want) <= 1e-13, rel_l2(g, want)


@pytest.mark.parametrize("by_ranges", [False, True])
def test_partitioned_lsrk_step(cuda_device, by_ranges):
    """Five fused stages per part, as one launch or as the two element
    ranges of the overlapped stage (hb_lsrk_stage_elements), bitwise equal
    to the unpartitioned LSRK4 step."""
    import torch
    from hedge_b200.timestep import RK4A, RK4B
    d, model, plan, parts, ex = _setup("maxwell", 4, "fp64")
    q = np.random.default_rng(2).standard_normal((6, len(d)))
    dt = model.estimate_timestep(d)
    rhs = model.bind(d)
    y = hb.LSRK4TimeStepper()(d.to_device(q), 0.0, dt, rhs).cpu().numpy()
    cur = [p.scatter(q) for p in parts]
    res = [torch.zeros_like(x) for x in cur]
    for s in range(5):
        for p, x in zip(parts, cur):
            p.pack(x)
        ex.exchange_all()
        nxt = []
        for p, x, r in zip(parts, cur, res):
            o = torch.empty_like(x)
            p.lsrk_stage(RK4A[s], RK4B[s], dt, x, o, r, exchanged=True, by_ranges=by_ranges)
            nxt.append(o)
        cur = nxt
    for p, x in zip(parts, cur):
        assert np.array_equal(x.cpu().numpy(), y[:, p.local_nodes()])


def test_halo_op_refusals(cuda_device):
    import ctypes as C
    import torch
    from hedge_b200 import _native
    from hedge_b200.discretization import op_descriptor
    from hedge_b200.partition import PartitionPlan, PartitionedOperator
    lib = _native.load()
    d = hb.Discretization(hb.make_regular_rect_mesh((-1, -1), (1, 1), (5, 5)), order=2)
    model = hb.StrongWaveOperator(1.0, 2)
    plan = PartitionPlan(d, model.op_template(), 2)
    p = PartitionedOperator(d, model, plan, 0)
    part = plan.parts[0]
    # an operator with halo faces refuses to run before it has a halo buffer
    od = op_descriptor(model.descriptor(), _native.PREC_FP64, part.conn, 0, part.n_halo_faces)
    h = C.c_void_p()
    assert lib.hb_op_create(p._dh, C.byref(od), C.byref(h)) == _native.HB_OK
    q = torch.zeros((3, p.K * p.Np), dtype=torch.float64, device=p.device)
    out = torch.empty_like(q)
    st = lib.hb_rhs(h, q.data_ptr(), out.data_ptr(), None, None, None, None)
    assert st == _native.HB_ERR_INVALID_ARGUMENT
    lib.hb_op_destroy(h)
    # halo slots beyond num_halo_faces are refused at creation
    od = op_descriptor(model.descriptor(), _native.PREC_FP64, part.conn, 0,
                       max(part.n_halo_faces - 1, 0))
    assert lib.hb_op_create(p._dh, C.byref(od), C.byref(h)) == _native.HB_ERR_INVALID_ARGUMENT


def test_partitioned_norm_equals_global(cuda_device):
    """Per-part squared energy norms summed (as the all-reduce does across
    ranks) equal the norm of the whole field."""
    from hedge_b200.partition import partitioned_norm, sum_over_ranks
    d, model, plan, parts, ex = _setup("maxwell", 3, "fp64")
    q = np.random.default_rng(5).standard_normal((6, len(d)))
    want = d.norm(d.to_device(q))
    got = partitioned_norm(parts, [p.scatter(q) for p in parts])
    assert abs(got - want) <= 1e-13 * want
    # without a process group, a part's norm is its own
    x = parts[0].scatter(q)
    assert sum_over_ranks(parts[0].norm_sq(x)) == parts[0].norm_sq(x)
    assert abs(parts[0].norm(x) - parts[0].norm_sq(x) ** 0.5) <= 1e-15 * parts[0].norm(x)


@pytest.mark.parametrize("kind,order", [("maxwell", 5), ("wave", 7)])
@pytest.mark.parametrize("precision", ["fp64", "fp16x3", "bf16x3"])
def test_partitioned_high_order(cuda_device, precision, kind, order):
    """3D N = 5 Maxwell and N = 7 wave: the parts, with halo faces, run on the
    streamed-operator split kernel (256 threads per CTA) on the split
    precisions; each part's RHS against the oracle on its elements."""
    import ctypes as C
    from oracle import OracleRHS
    from hedge_b200.partition import LocalExchange, PartitionPlan, PartitionedOperator
    from test_gpu_parity import _fields
    d = hb.Discretization(hb.make_box_tet_mesh(n=(2, 2, 2), jitter=0.03, seed=5), order=order)
    model = hb.MaxwellOperator(1.0, 1.0, flux_type=1) if kind == "maxwell" else \
        hb.StrongWaveOperator(1.0, 3, flux_type="upwind")
    F = 6 if kind == "maxwell" else 4
    plan = PartitionPlan(d, model.op_template(), 3)
    parts = [PartitionedOperator(d, model, plan, r, precision=precision) for r in range(3)]
    ex = LocalExchange(plan, parts)
    q = _fields(d, F, 12)
    ref = OracleRHS(d, model.op_template())(q).reshape(F, -1)
    tol = {"fp64": 1e-12, "fp16x3": 1e-6, "bf16x3": 1e-5}[precision]
    ql = [p.scatter(q) for p in parts]
    for p, x in zip(parts, ql):
        p.pack(x)
    ex.exchange_all()
    for p, x in zip(parts, ql):
        assert p.part.n_halo_faces > 0
        if precision != "fp64":
            info = (C.c_int64 * 6)()
            p.lib.hb_op_launch_info(p._h, info, 6)
            assert info[1] == 256, list(info)
        for by_ranges in (False, True):
            got = p.rhs(x, exchanged=True, by_ranges=by_ranges)
            p.check()
            err = rel_l2(got.double().cpu().numpy(), ref[:, p.local_nodes()])
            print("%s %s N=%d part rel-L2 %.3e" % (precision, kind, order, err))
            assert err <= tol


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp16x3", "bf16x3"])
def test_stage_over_element_ranges(cuda_device, precision):
    """hb_lsrk_stage_elements over [0, k) then [k, K), k not a multiple of
    any batch size, equals one hb_lsrk_stage (bitwise); ranges outside
    [0, K] are refused."""
    import torch
    from hedge_b200 import _native
    d = hb.Discretization(hb.make_box_tet_mesh(n=(4, 4, 4), jitter=0.03, seed=7), order=4,
                          precision=precision)
    model = hb.MaxwellOperator(1.0, 1.0, flux_type=1)
    comp = model.bind(d).compiled
    lib, h = comp._lib, comp._handle
    dt = torch.float32 if precision == "fp32" else torch.float64
    rng = np.random.default_rng(3)
    q = torch.as_tensor(rng.standard_normal((6, len(d))), dtype=dt, device=d.device)
    r0 = torch.as_tensor(rng.standard_normal((6, len(d))), dtype=dt, device=d.device)
    a, b, step = -0.41, 0.37, 1e-3
    st = comp._stream()
    want_q, want_r = torch.empty_like(q), r0.clone()
    _native.check(lib.hb_lsrk_stage(h, a, b, step, q.data_ptr(), want_q.data_ptr(),
                                    want_r.data_ptr(), None, None, None, st))
    got_q, got_r = torch.empty_like(q), r0.clone()
    k = 137
    for e0, e1 in ((0, k), (k, d.K)):
        _native.check(lib.hb_lsrk_stage_elements(h, e0, e1, a, b, step, q.data_ptr(),
                                                 got_q.data_ptr(), got_r.data_ptr(), None,
                                                 None, None, st))
    comp.check()
    assert torch.equal(got_q, want_q) and torch.equal(got_r, want_r)
    for e0, e1 in ((-1, 5), (5, 4), (0, d.K + 1)):
        assert lib.hb_lsrk_stage_elements(h, e0, e1, a, b, step, q.data_ptr(),
                                          got_q.data_ptr(), got_r.data_ptr(), None, None,
                                          None, st) == _native.HB_ERR_INVALID_ARGUMENT
