"""VTK output and the in-memory log manager (CPU)."""
import os
import re
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import hedge_b200 as hb
from hedge_b200.log import LogManager, LogQuantity, MultiLogQuantity
from hedge_b200.visualization import (LegacyVtkVisualizer, VtkVisualizer,
                                      submesh_indices)


def _discr(dim, order):
    m = hb.make_regular_rect_mesh((-1, -1), (1, 1), (4, 4), jitter=0.05, seed=0) if dim == 2 \
        else hb.make_box_tet_mesh(n=(2, 2, 2), jitter=0.05, seed=1)
    return hb.Discretization(m, order=order)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("order", [1, 2, 4, 7])
def test_submesh_tiles_each_element(dim, order):
    """N^d positively oriented sub-simplices per element whose volumes add up
    to the element's (the nodes on the element's faces lie on the faces)."""
    d = _discr(dim, order)
    smi = np.array(submesh_indices(d.ldis))
    assert len(smi) == order ** dim
    assert set(smi.reshape(-1)) == set(range(d.Np))
    x = d.nodes.reshape(d.K, d.Np, dim)
    v = x[:, smi]                                    # [K, cells, d+1, d]
    vol = np.linalg.det(v[:, :, 1:] - v[:, :, :1])   # d! * signed volume
    assert (vol > 0).all()
    ref = np.abs(d.mesh.jacobians) * (2.0 if dim == 2 else 4.0 / 3.0)
    fact = 2.0 if dim == 2 else 6.0
    assert np.allclose(vol.sum(1) / fact, ref, rtol=1e-12)


def _read_vtu(path):
    raw = open(path, "rb").read()
    head, _, tail = raw.partition(b'<AppendedData encoding="raw">\n_')
    xml = head.decode() + ("</VTKFile>" if tail else "")
    root = ET.fromstring(xml if tail else raw.decode())
    arrays = {}
    types = {"Float64": np.float64, "Int64": np.int64, "UInt8": np.uint8}
    for da in root.iter("DataArray"):
        t = types[da.get("type")]
        if da.get("format") == "appended":
            off = int(da.get("offset"))
            n = int(np.frombuffer(tail[off:off + 8], dtype="<u8")[0])
            arrays[da.get("Name")] = np.frombuffer(tail[off + 8:off + 8 + n], dtype=t)
        else:
            arrays[da.get("Name")] = np.array(da.text.split(), dtype=t)
    piece = root.find(".//Piece")
    return arrays, int(piece.get("NumberOfPoints")), int(piece.get("NumberOfCells"))


@pytest.mark.parametrize("binary", [True, False])
def test_vtu_roundtrip(tmp_path, binary):
    d = _discr(3, 3)
    u = np.sin(d.nodes[:, 0])
    e = np.stack([d.nodes[:, k] ** 2 for k in range(3)])
    vis = VtkVisualizer(d, basename=str(tmp_path / "run"), binary=binary)
    for step, t in enumerate([0.0, 0.5]):
        f = vis.make_file(str(tmp_path / ("fld-%04d" % step)))
        vis.add_data(f, [("u", u * (1 + t)), ("e", list(e))], time=t, step=step)
        f.close()
    vis.close()
    arrays, npts, ncells = _read_vtu(str(tmp_path / "fld-0001.vtu"))
    assert npts == len(d) and ncells == d.K * 27
    assert np.allclose(arrays["points"].reshape(-1, 3), d.nodes)
    conn = arrays["connectivity"].reshape(-1, 4)
    assert conn.min() == 0 and conn.max() == len(d) - 1
    assert (arrays["offsets"] == 4 * np.arange(1, ncells + 1)).all()
    assert (arrays["types"] == 10).all()
    assert np.array_equal(arrays["u"], u * 1.5)
    assert np.array_equal(arrays["e"].reshape(-1, 3), e.T)
    pvd = ET.parse(str(tmp_path / "run.pvd")).getroot()
    files = [(float(ds.get("timestep")), ds.get("file")) for ds in pvd.iter("DataSet")]
    assert files == [(0.0, "fld-0000.vtu"), (0.5, "fld-0001.vtu")]


def test_legacy_vtk(tmp_path):
    d = _discr(2, 4)
    vis = LegacyVtkVisualizer(d)
    f = vis.make_file(str(tmp_path / "a"))
    vis.add_data(f, [("u", d.nodes[:, 1]), ("v", [d.nodes[:, 0], d.nodes[:, 1]])])
    f.close()
    txt = open(str(tmp_path / "a.vtk")).read()
    assert "POINTS %d double" % len(d) in txt
    n = d.K * 16
    assert re.search(r"CELLS %d %d" % (n, 4 * n), txt)
    assert "SCALARS u double" in txt and "VECTORS v double" in txt


def test_wrong_length_field_rejected(tmp_path):
    d = _discr(2, 2)
    vis = VtkVisualizer(d)
    f = vis.make_file(str(tmp_path / "x"))
    with pytest.raises(ValueError):
        vis.add_data(f, [("u", np.zeros(len(d) - 1))])


def test_log_manager_records_ticks(tmp_path):
    class Count(LogQuantity):
        def __init__(self):
            super().__init__("count", "1", "ticks so far")
            self.n = 0

        def __call__(self):
            self.n += 1
            return self.n

    class Pair(MultiLogQuantity):
        def __call__(self):
            return [1.0, 2.0]

    mgr = LogManager()
    mgr.add_quantity(Count())
    mgr.add_quantity(Pair(["a", "b"]))
    for _ in range(3):
        mgr.tick()
    assert mgr.get_series("count") == [1.0, 2.0, 3.0]
    assert mgr.get_series("b") == [2.0] * 3
    mgr.save(str(tmp_path / "log.json"))
    assert os.path.getsize(str(tmp_path / "log.json")) > 0
