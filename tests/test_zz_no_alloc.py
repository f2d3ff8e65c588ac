"""hb_norm_noalloc through the C ABI against hb_norm on the same inputs.

Two calls in a row (a larger mesh, then a smaller one, so the second call
reads a scratch array the first one left full), each within 1e-13 of hb_norm
and, since both run the same kernels in the same reduction order, equal to it
bit for bit; a call captured into a CUDA graph (which an allocation or a
synchronisation would break) and replayed; plus the size limit and operands
that are not memory of the current device, both rejected before any
launch."""
import numpy as np
import pytest

import hedge_b200 as hb
from hedge_b200 import _native

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _case(n, order, nfields, seed):
    import torch
    d = hb.Discretization(hb.make_box_tet_mesh(n=(n, n, n), jitter=0.05, seed=1),
                          order=order)
    rng = np.random.default_rng(seed)
    u = torch.as_tensor(rng.standard_normal((nfields, len(d))), device=d.device)
    mass = torch.as_tensor(np.ascontiguousarray(d.ldis.mass_matrix), device=d.device)
    absjac = torch.as_tensor(np.abs(d.mesh.jacobians), device=d.device)
    return d, u, mass, absjac


def _noalloc(d, u, mass, absjac):
    import torch
    out = torch.full((1,), -1.0, dtype=torch.float64, device=d.device)
    lib = _native.load()
    _native.check(lib.hb_norm_noalloc(
        d.K, d.Np, u.shape[0], 0, mass.data_ptr(), absjac.data_ptr(), u.data_ptr(),
        out.data_ptr(), torch.cuda.current_stream(d.device).cuda_stream))
    return float(out.item())


def test_noalloc_norm_matches_hb_norm_twice(cuda_device):
    big = _case(6, 4, 6, 3)       # K = 1296, 186 partial blocks
    small = _case(2, 3, 3, 4)     # K = 48, 4 partial blocks
    for d, u, mass, absjac in (big, small):
        want = d.norm(u)
        got = _noalloc(d, u, mass, absjac)
        assert abs(got - want) <= TOL * want, (got, want)
        assert got == want, (got, want)
    d, u, mass, absjac = big
    got = _noalloc(d, u, mass, absjac)
    assert abs(got - d.norm(u)) <= TOL * d.norm(u)
    assert got == d.norm(u)


def test_noalloc_norm_captures_in_a_cuda_graph(cuda_device):
    """After its first call on the device, a call captures into a CUDA
    graph (stream capture fails on an allocation or a synchronisation) and
    the replay gives hb_norm's value bit for bit, also after the field
    changed in place."""
    import torch
    d, u, mass, absjac = _case(4, 4, 6, 8)
    _noalloc(d, u, mass, absjac)          # first call: the scratch address lookup
    lib = _native.load()
    out = torch.full((1,), -1.0, dtype=torch.float64, device=d.device)
    graph = torch.cuda.CUDAGraph()
    status = []
    with torch.cuda.graph(graph):
        status.append(lib.hb_norm_noalloc(
            d.K, d.Np, u.shape[0], 0, mass.data_ptr(), absjac.data_ptr(), u.data_ptr(),
            out.data_ptr(), torch.cuda.current_stream(d.device).cuda_stream))
    assert status == [_native.HB_OK]
    for scale in (1.0, 0.5):
        u.mul_(scale)
        out.fill_(-1.0)
        graph.replay()
        torch.cuda.synchronize(d.device)
        assert float(out.item()) == d.norm(u)


def test_noalloc_norm_rejects_oversized_mesh(cuda_device):
    import torch
    d, u, mass, absjac = _case(2, 4, 1, 5)
    lib = _native.load()
    epb = max(1, 256 // d.Np)
    too_many = 8192 * epb + 1
    out = torch.zeros(1, dtype=torch.float64, device=d.device)
    st = lib.hb_norm_noalloc(too_many, d.Np, 1, 0, mass.data_ptr(), absjac.data_ptr(),
                             u.data_ptr(), out.data_ptr(), None)
    assert st == _native.HB_ERR_INVALID_ARGUMENT
    assert b"scratch limit" in lib.hb_last_error_string()


def test_noalloc_norm_rejects_host_memory(cuda_device):
    """The scratch address is the current device's: a field in host memory
    is refused instead of being read by the kernels."""
    import torch
    d, u, mass, absjac = _case(2, 3, 1, 6)
    host_u = np.ascontiguousarray(u.cpu().numpy())
    out = torch.zeros(1, dtype=torch.float64, device=d.device)
    lib = _native.load()
    st = lib.hb_norm_noalloc(d.K, d.Np, 1, 0, mass.data_ptr(), absjac.data_ptr(),
                             host_u.ctypes.data, out.data_ptr(), None)
    assert st == _native.HB_ERR_INVALID_ARGUMENT
    assert b"not device memory" in lib.hb_last_error_string()


def test_noalloc_norm_rejects_other_device(cuda_device):
    """u on another GPU than the current one is refused (needs two GPUs)."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("one GPU")
    d, u, mass, absjac = _case(2, 3, 1, 7)
    u1 = u.to("cuda:1")
    out = torch.zeros(1, dtype=torch.float64, device=d.device)
    lib = _native.load()
    st = lib.hb_norm_noalloc(d.K, d.Np, 1, 0, mass.data_ptr(), absjac.data_ptr(),
                             u1.data_ptr(), out.data_ptr(), None)
    assert st == _native.HB_ERR_INVALID_ARGUMENT
