"""VTK output of (device) volume fields (hedge/visualization.py:62-332).

``VtkVisualizer(discr, basename=...)`` writes one XML UnstructuredGrid file
(``.vtu``) per ``make_file`` / ``add_data`` / ``close`` and, on ``close()``,
a ParaView collection (``.pvd``) indexing the files by time.
``LegacyVtkVisualizer`` writes legacy ASCII ``.vtk`` files.  The grid's
points are the discretization's nodes; every element is cut into linear
sub-simplices through its node lattice (``submesh_indices``), so a field is
shown with its nodal values.  Fields may be torch tensors on the device
(copied to the host once per file), numpy arrays, or lists of components.

Arrays are written raw in the file's appended-data block (little endian,
UInt64 byte-count headers), or as ASCII with ``binary=False``.
"""

from __future__ import annotations

import os

import numpy as np

VTK_TRIANGLE = 5
VTK_TETRA = 10


def submesh_indices(ldis):
    """Sub-simplices of the reference element through its node lattice
    (node tuples (i, j[, k]) with i + j [+ k] <= N), as node-index tuples,
    positively oriented.

    Triangle: per lattice point an upward triangle, and a downward one where
    it fits (N^2 in all).  Tetrahedron: per lattice point an upward corner
    tet, an octahedron cut into 4 tets along one diagonal, and a downward
    tet, where they fit (N^3 in all)."""
    tuples = [tuple(t) for t in ldis.node_tuples]
    idx = {t: i for i, t in enumerate(tuples)}
    N = ldis.order
    d = len(tuples[0])

    def add(p, *ds):
        return tuple(p[a] + sum(dd[a] for dd in ds) for a in range(d))

    e = [tuple(1 if a == b else 0 for a in range(d)) for b in range(d)]
    out = []
    if d == 2:
        for p in tuples:
            s = sum(p)
            if s <= N - 1:
                out.append((p, add(p, e[0]), add(p, e[1])))
            if s <= N - 2:
                out.append((add(p, e[0]), add(p, e[0], e[1]), add(p, e[1])))
    elif d == 3:
        for p in tuples:
            s = sum(p)
            if s <= N - 1:
                out.append((p, add(p, e[0]), add(p, e[1]), add(p, e[2])))
            if s <= N - 2:
                a, b, c = add(p, e[0]), add(p, e[1]), add(p, e[2])
                ab, ac, bc = add(p, e[0], e[1]), add(p, e[0], e[2]), add(p, e[1], e[2])
                # diagonal a - bc; the other four vertices in cyclic order
                ring = (b, c, ac, ab)
                for q in range(4):
                    out.append((a, bc, ring[q], ring[(q + 1) % 4]))
            if s <= N - 3:
                out.append((add(p, e[0], e[1]), add(p, e[0], e[2]), add(p, e[1], e[2]),
                            add(p, e[0], e[1], e[2])))
    else:
        raise NotImplementedError("%dD elements" % d)
    cells = []
    for simplex in out:
        x = np.array(simplex, dtype=np.float64)
        if np.linalg.det(x[1:] - x[0]) < 0:
            simplex = (simplex[1], simplex[0]) + simplex[2:]
        cells.append(tuple(idx[t] for t in simplex))
    return cells


def _host(field):
    try:
        import torch
        if isinstance(field, torch.Tensor):
            return field.detach().to("cpu", torch.float64).numpy()
    except ImportError:      # pragma: no cover
        pass
    if isinstance(field, (list, tuple)) or (isinstance(field, np.ndarray) and field.dtype == object):
        return np.stack([_host(f) for f in field])
    return np.asarray(field, dtype=np.float64)


class _Grid:
    def __init__(self, discr):
        smi = np.array(submesh_indices(discr.ldis), dtype=np.int64)
        K, Np = discr.K, discr.Np
        self.cells = (np.arange(K, dtype=np.int64)[:, None, None] * Np + smi[None]).reshape(
            -1, smi.shape[1])
        self.cell_type = VTK_TRIANGLE if smi.shape[1] == 3 else VTK_TETRA
        pts = np.asarray(discr.nodes, dtype=np.float64)
        self.points = np.zeros((len(pts), 3))
        self.points[:, :pts.shape[1]] = pts
        self.n_points = len(pts)


def _as_point_data(grid, name, field, scale):
    a = _host(field) * scale
    if a.ndim == 1:
        if a.shape[0] != grid.n_points:
            raise ValueError("%s: %d values for %d nodes" % (name, a.shape[0], grid.n_points))
        return a, 1
    a = a.reshape(a.shape[0], -1)
    if a.shape[1] != grid.n_points:
        raise ValueError("%s: %d values for %d nodes" % (name, a.shape[1], grid.n_points))
    nc = 3 if a.shape[0] <= 3 else a.shape[0]
    out = np.zeros((grid.n_points, nc))
    out[:, :a.shape[0]] = a.T
    return out, nc


class VtkFile:
    """One ``.vtu`` file; written by ``close()``."""

    def __init__(self, pathname, grid, binary=True):
        self.pathname = pathname
        self.grid = grid
        self.binary = binary
        self.point_data = []
        self._closed = False

    def get_head_pathname(self):
        return self.pathname

    def add_pointdata(self, name, array, ncomp):
        self.point_data.append((name, array, ncomp))

    def close(self):
        if self._closed:
            return
        self._closed = True
        g = self.grid
        nv = g.cells.shape[1]
        arrays = [("Points", "points", g.points, 3),
                  ("Cells", "connectivity", g.cells.reshape(-1), 1),
                  ("Cells", "offsets", np.arange(1, len(g.cells) + 1, dtype=np.int64) * nv, 1),
                  ("Cells", "types", np.full(len(g.cells), g.cell_type, dtype=np.uint8), 1)]
        arrays += [("PointData", n, a, c) for n, a, c in self.point_data]
        types = {np.dtype(np.float64): "Float64", np.dtype(np.int64): "Int64",
                 np.dtype(np.uint8): "UInt8"}
        blobs, offset = [], 0
        sections = {"Points": [], "Cells": [], "PointData": []}
        for sec, name, a, nc in arrays:
            a = np.ascontiguousarray(a)
            t = types[a.dtype]
            if self.binary:
                raw = a.astype(a.dtype.newbyteorder("<"), copy=False).tobytes()
                blobs.append(np.uint64(len(raw)).tobytes() + raw)
                sections[sec].append('<DataArray type="%s" Name="%s" NumberOfComponents="%d" '
                                     'format="appended" offset="%d"/>' % (t, name, nc, offset))
                offset += 8 + len(raw)
            else:
                fmt = "%d" if a.dtype != np.float64 else "%.17g"
                body = " ".join(fmt % x for x in a.reshape(-1))
                sections[sec].append('<DataArray type="%s" Name="%s" NumberOfComponents="%d" '
                                     'format="ascii">%s</DataArray>' % (t, name, nc, body))
        head = ['<?xml version="1.0"?>',
                '<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" '
                'header_type="UInt64">',
                '<UnstructuredGrid>',
                '<Piece NumberOfPoints="%d" NumberOfCells="%d">' % (g.n_points, len(g.cells)),
                '<Points>'] + sections["Points"] + ['</Points>', '<Cells>'] + \
            sections["Cells"] + ['</Cells>', '<PointData>'] + sections["PointData"] + \
            ['</PointData>', '</Piece>', '</UnstructuredGrid>']
        with open(self.pathname, "wb") as f:
            f.write("\n".join(head).encode())
            if self.binary:
                f.write(b'\n<AppendedData encoding="raw">\n_')
                for b in blobs:
                    f.write(b)
                f.write(b"\n</AppendedData>")
            f.write(b"\n</VTKFile>\n")


class VtkVisualizer:
    def __init__(self, discr, pcontext=None, basename=None, compressor=None, binary=True):
        if compressor is not None:
            raise NotImplementedError("compressed VTK output")
        self.discr = discr
        self.grid = _Grid(discr)
        self.binary = binary
        self.pvd_name = basename + ".pvd" if basename is not None else None
        if self.pvd_name is not None and os.path.exists(self.pvd_name):
            raise RuntimeError("%s exists already" % self.pvd_name)
        self.timestep_to_pathnames = {}

    def make_file(self, pathname):
        """A file ``pathname + '.vtu'`` (the extension is appended)."""
        return VtkFile(pathname + ".vtu", self.grid, self.binary)

    def add_data(self, visf, variables=(), scalars=(), vectors=(), time=None, step=None,
                 scale_factor=1):
        for name, field in list(variables) + list(scalars) + list(vectors):
            arr, nc = _as_point_data(self.grid, name, field, scale_factor)
            visf.add_pointdata(name, arr, nc)
        if time is not None:
            self.timestep_to_pathnames.setdefault(time, []).append(visf.get_head_pathname())

    def update_pvd(self):
        if not self.pvd_name or not self.timestep_to_pathnames:
            return
        start = os.path.dirname(self.pvd_name)
        lines = ['<?xml version="1.0"?>',
                 '<VTKFile type="Collection" version="0.1" byte_order="LittleEndian">',
                 '<Collection>']
        for t in sorted(self.timestep_to_pathnames):
            for part, p in enumerate(self.timestep_to_pathnames[t]):
                lines.append('<DataSet timestep="%.17g" part="%d" file="%s"/>'
                             % (t, part, os.path.relpath(p, start or ".")))
        lines += ['</Collection>', '</VTKFile>']
        with open(self.pvd_name, "w") as f:
            f.write("\n".join(lines) + "\n")

    def close(self):
        self.update_pvd()


class LegacyVtkFile:
    def __init__(self, pathname, grid, description="hedge_b200 output"):
        self.pathname, self.grid, self.description = pathname, grid, description
        self.point_data = []

    def add_pointdata(self, name, array, ncomp):
        self.point_data.append((name, array, ncomp))

    def get_head_pathname(self):
        return self.pathname

    def close(self):
        g = self.grid
        nv = g.cells.shape[1]
        with open(self.pathname, "w") as f:
            f.write("# vtk DataFile Version 2.0\n%s\nASCII\nDATASET UNSTRUCTURED_GRID\n"
                    % self.description)
            f.write("POINTS %d double\n" % g.n_points)
            np.savetxt(f, g.points, fmt="%.17g")
            f.write("CELLS %d %d\n" % (len(g.cells), len(g.cells) * (nv + 1)))
            np.savetxt(f, np.hstack([np.full((len(g.cells), 1), nv), g.cells]), fmt="%d")
            f.write("CELL_TYPES %d\n" % len(g.cells))
            np.savetxt(f, np.full(len(g.cells), g.cell_type), fmt="%d")
            if self.point_data:
                f.write("POINT_DATA %d\n" % g.n_points)
            for name, a, nc in self.point_data:
                if nc == 1:
                    f.write("SCALARS %s double 1\nLOOKUP_TABLE default\n" % name)
                    np.savetxt(f, a, fmt="%.17g")
                elif nc == 3:
                    f.write("VECTORS %s double\n" % name)
                    np.savetxt(f, a, fmt="%.17g")
                else:
                    f.write("FIELD FieldData 1\n%s %d %d double\n" % (name, nc, g.n_points))
                    np.savetxt(f, a, fmt="%.17g")


class LegacyVtkVisualizer:
    def __init__(self, discr, pcontext=None):
        self.discr = discr
        self.grid = _Grid(discr)

    def make_file(self, pathname):
        return LegacyVtkFile(pathname + ".vtk", self.grid)

    def add_data(self, visf, variables=(), scalars=(), vectors=(), time=None, step=None,
                 scale_factor=1):
        for name, field in list(variables) + list(scalars) + list(vectors):
            arr, nc = _as_point_data(self.grid, name, field, scale_factor)
            visf.add_pointdata(name, arr, nc)

    def close(self):
        pass


__all__ = ["VtkVisualizer", "LegacyVtkVisualizer", "VtkFile", "LegacyVtkFile",
           "submesh_indices"]
