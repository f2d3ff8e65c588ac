"""Edge cases of the mesh and the batching on every kernel path, against the
CPU oracle: a single element (every face a boundary face, both vertex
orientations), and meshes whose element count is one short of, exactly, and
one past a full batch of the split kernels (20 elements for Maxwell, 32 for
the 3D wave), so the last batch is full, ragged or a single element."""
import numpy as np
import pytest

import hedge_b200 as hb
from conftest import rel_l2
from test_gpu_parity import _fields

pytestmark = pytest.mark.gpu

# FP64 / FP32 as in the plain parity tests; the split paths as on rough fields
TOL = {"fp64": 1e-12, "fp32": 1e-5, "fp32-simt": 1e-5, "bf16x3": 1e-5, "fp16x3": 1e-6}
PRECS = ["fp64", "fp32", "fp32-simt", "bf16x3", "fp16x3"]

TRI = np.array([[0.1, -0.2], [1.3, 0.1], [0.2, 0.9]])
TET = np.array([[0.0, 0.1, -0.1], [1.2, 0.0, 0.1], [0.1, 0.9, 0.0], [0.2, 0.1, 1.1]])


def _err(d, op, precision, seed):
    from oracle import OracleRHS
    ot = op.op_template()
    q = _fields(d, op.descriptor().n_fields, seed)
    if precision in ("fp32", "fp32-simt"):
        q = q.astype(np.float32).astype(np.float64)
    ref = OracleRHS(d, ot)(q)
    comp = d.compile(ot, precision=precision)
    got = comp(w=q)
    comp.check()
    return rel_l2(got.double().cpu().numpy().reshape(ref.shape), ref)


def _one(dim, flip):
    pts = TRI if dim == 2 else TET
    el = np.arange(dim + 1)[None, :]
    if flip:
        el = el[:, [0, 2, 1] + ([3] if dim == 3 else [])]
    return hb.Mesh(pts, el)


@pytest.mark.parametrize("precision", PRECS)
@pytest.mark.parametrize("flip", [False, True])
@pytest.mark.parametrize("dim", [2, 3])
def test_single_element_wave(cuda_device, dim, flip, precision):
    d = hb.Discretization(_one(dim, flip), order=4)
    assert d.K == 1
    err = _err(d, hb.StrongWaveOperator(1.0, dim, flux_type="upwind"), precision, 1)
    print("one element wave %dD flip=%s %s rel-L2 %.3e" % (dim, flip, precision, err))
    assert err <= TOL[precision]


@pytest.mark.parametrize("precision", PRECS)
def test_single_element_maxwell(cuda_device, precision):
    d = hb.Discretization(_one(3, False), order=4)
    err = _err(d, hb.MaxwellOperator(1.0, 1.0, flux_type=1), precision, 2)
    print("one element maxwell %s rel-L2 %.3e" % (precision, err))
    assert err <= TOL[precision]


@pytest.mark.parametrize("precision", ["bf16x3", "fp16x3"])
def test_single_element_streamed(cuda_device, precision):
    """N = 6 in 3D runs the operator-streaming split kernel."""
    d = hb.Discretization(_one(3, True), order=6)
    err = _err(d, hb.StrongWaveOperator(1.0, 3, flux_type="upwind"), precision, 3)
    print("one element wave N=6 %s rel-L2 %.3e" % (precision, err))
    assert err <= TOL[precision]


def _first_elements(k):
    """The first k tetrahedra of a jittered 3x3x3 box (162 elements)."""
    m = hb.make_box_tet_mesh(n=(3, 3, 3), jitter=0.05, seed=4)
    return hb.Mesh(m.points, m.elements[:k])


@pytest.mark.parametrize("precision", ["fp64", "fp16x3"])
@pytest.mark.parametrize("k", [19, 20, 21, 40, 41])
def test_batch_boundaries_maxwell(cuda_device, k, precision):
    d = hb.Discretization(_first_elements(k), order=4)
    err = _err(d, hb.MaxwellOperator(1.0, 1.0, flux_type=1), precision, 4)
    print("maxwell K=%d %s rel-L2 %.3e" % (k, precision, err))
    assert err <= TOL[precision]


@pytest.mark.parametrize("precision", ["fp64", "fp16x3"])
@pytest.mark.parametrize("k,order", [(31, 4), (32, 4), (33, 4), (33, 7)])
def test_batch_boundaries_wave(cuda_device, k, order, precision):
    d = hb.Discretization(_first_elements(k), order=order)
    err = _err(d, hb.StrongWaveOperator(1.0, 3, flux_type="upwind"), precision, 5)
    print("wave K=%d N=%d %s rel-L2 %.3e" % (k, order, precision, err))
    assert err <= TOL[precision]
