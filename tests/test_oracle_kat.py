"""The CPU oracle pinned against the reference's own known-answer tests
(test/test_jit_discretization.py), restated on structured meshes where the
reference used meshpy-generated ones."""
import ctypes as C
import math

import numpy as np
import pytest

import hedge_b200 as hb
import oracle as orc
from hedge_b200.models import OpTemplate


def normal_dot_template(dim, alpha, bcs=()):
    return OpTemplate(orc.OR_NORMAL_DOT, dim, 1, 0, {"alpha": alpha}, list(bcs))


def flux_sum(discr, args, alpha, boundary):
    """E (Fjac * flux) summed with ones: the surface integral of the flux."""
    ot = normal_dot_template(discr.dimensions, alpha)
    o = orc.OracleRHS.__new__(orc.OracleRHS)
    o.discr, o.ot = discr, ot
    o.dim, o.K, o.Np = discr.dimensions, discr.K, discr.Np
    o.N = o.K * o.Np
    o.emat = np.ascontiguousarray(discr.ldis.multi_face_mass_matrix)
    args = np.ascontiguousarray(args, dtype=np.float64)
    o.params = o._params(False)
    o.params.n_args = args.shape[0]
    lib = orc.load()
    total = np.zeros((1, o.N))
    if boundary:
        b = discr.get_boundary(hb.TAG_ALL)
        fgw = orc._FG(b.face_group)
        bargs = np.zeros((args.shape[0], len(b.vol_indices)))
        fg = b.face_group
        fof = np.zeros((1, fg.n_local_els * fg.face_count * fg.face_length))
        lib.or_gather_boundary(C.byref(fgw.c), C.byref(o.params), o.N, orc._p(args),
                               bargs.shape[1], orc._p(bargs), orc._p(fof))
    else:
        fgw = orc._FG(discr.interior_face_group)
        fg = fgw.fg
        fof = np.zeros((1, fg.n_local_els * fg.face_count * fg.face_length))
        lib.or_gather_interior(C.byref(fgw.c), C.byref(o.params), o.N, orc._p(args),
                               orc._p(fof))
    total += o._lift_e(fgw, fof)
    return total[0].sum()


def volume_integral(discr, u):
    M = discr.ldis.mass_matrix
    J = np.abs(discr.mesh.jacobians)
    return float(np.einsum("i,ki,k->", M.sum(0), u.reshape(discr.K, discr.Np), J))


def test_2d_gauss_theorem():
    """test_jit_discretization.py:164-236 (disk mesh -> jittered rectangle)."""
    mesh = hb.make_regular_rect_mesh((-1, -1), (1, 1), (9, 7), jitter=0.03, seed=11)
    discr = hb.Discretization(mesh, order=2)
    x = discr.nodes
    f1 = np.sin(3 * x[:, 0]) + np.cos(3 * x[:, 1])
    f2 = np.sin(2 * x[:, 0]) + np.cos(x[:, 1])
    o = orc.OracleRHS(discr, hb.StrongAdvectionOperator(np.array([1.0, 0])).op_template())
    div = o.grad(f1)[0] + o.grad(f2)[1]
    int_div = volume_integral(discr, div)
    bdry = flux_sum(discr, np.stack([f1, f2]), 0.0, boundary=True)
    assert abs(bdry - int_div) < 5e-14


@pytest.mark.parametrize("dim", [2, 3])
def test_simp_gauss_theorem(dim):
    """test_jit_discretization.py:280-431: one simplex with far-off vertices."""
    rng = np.random.default_rng(7)
    for trial in range(5):
        verts = rng.uniform(-8, 8, (dim + 1, dim))
        mesh = hb.Mesh(verts, np.arange(dim + 1)[None])
        discr = hb.Discretization(mesh, order=4 if dim == 2 else 3)
        x = discr.nodes
        if dim == 2:
            fs = [np.sin(3 * x[:, 0]) + np.cos(3 * x[:, 1]),
                  np.sin(2 * x[:, 0]) + np.cos(x[:, 1])]
        else:
            fs = [np.sin(3 * x[:, 0]) + np.cos(3 * x[:, 1]) + np.sin(1.9 * x[:, 2]),
                  np.sin(1.2 * x[:, 0]) + np.cos(2.1 * x[:, 1]) - np.cos(1.5 * x[:, 2]),
                  5 * np.sin(-0.2 * x[:, 0]) - 3 * np.cos(x[:, 1]) + np.cos(x[:, 2])]
        o = orc.OracleRHS(discr, hb.StrongAdvectionOperator(np.ones(dim)).op_template())
        div = sum(o.grad(f)[k] for k, f in enumerate(fs))
        lhs = volume_integral(discr, div)
        rhs = flux_sum(discr, np.stack(fs), 0.0, boundary=True)
        scale = max(abs(lhs), 1.0)
        assert abs(lhs - rhs) / scale < 1e-12


def test_interior_fluxes_tri():
    """test_jit_discretization.py:528-618: sum of (u- - u+) n_y over interior
    faces of a two-region mesh, u = 2 cos(x - y) above y = 0; known value 0."""
    mesh = hb.make_regular_rect_mesh((-math.pi, -1), (math.pi, 1), (17, 9))
    discr = hb.Discretization(mesh, order=4)
    cen = mesh.points[mesh.elements].mean(1)
    upper = np.repeat(cen[:, 1] > 0, discr.Np)
    x = discr.nodes
    u = np.where(upper, 2 * np.cos(x[:, 0] - x[:, 1]), 0.0)
    val = flux_sum(discr, np.stack([np.zeros_like(u), u]), 1.0, boundary=False)
    assert abs(val) < 5e-14


def symmetry_mesh():
    """The 8-triangle mesh of test_jit_discretization.py:730-773."""
    pts = np.array([[-0.5, -0.5], [-0.5, 0.5], [0.5, 0.5], [0.5, -0.5], [0.0, 0.0],
                    [-0.5, 0.0], [0.0, -0.5], [0.5, 0.0], [0.0, 0.5]])
    els = np.array([[8, 7, 4], [8, 7, 2], [6, 7, 3], [7, 4, 6], [5, 6, 0], [5, 6, 4],
                    [5, 8, 4], [1, 5, 8]])
    v = np.array([-1.0, 0.0])
    probe = hb.Mesh(pts, els)

    def tagger(fvi, el, fn, allv):
        return ["inflow"] if probe.face_normals[el, fn] @ v < 0 else ["outflow"]
    return hb.Mesh(pts, els, tagger), v


def mirror_permutation(discr, el_map={0: 3, 2: 1, 5: 6, 7: 4}):
    """Node permutation of the reflection y -> -y, element by element
    (the reference's SymmetryMap with its element map)."""
    full = dict(el_map)
    full.update({b: a for a, b in el_map.items()})
    x = discr.nodes.reshape(discr.K, discr.Np, -1)
    perm = np.empty(discr.K * discr.Np, dtype=np.int64)
    for e in range(discr.K):
        t = full.get(e, e)
        m = x[e] * np.array([1.0, -1.0])
        d = np.linalg.norm(m[:, None, :] - x[t][None, :, :], axis=-1)
        j = np.argmin(d, axis=1)
        assert np.all(d[np.arange(discr.Np), j] < 1e-13)
        perm[e * discr.Np:(e + 1) * discr.Np] = t * discr.Np + j
    return perm


def test_symmetry_preservation_2d():
    """test_jit_discretization.py:726-838: mirror-symmetric advection stays
    symmetric to 4e-15 at every RK step, for every flux type."""
    mesh, v = symmetry_mesh()
    discr = hb.Discretization(mesh, order=4, debug={"node_permutation"})
    perm = mirror_permutation(discr)

    def f(s):
        return np.where(s < 0.5, 0.0, s - 0.5)

    def u_an(x, t):
        return f(-(x @ v) + t)
    for flux_type in hb.StrongAdvectionOperator.flux_types:
        op = hb.StrongAdvectionOperator(v, flux_type=flux_type)
        o = orc.OracleRHS(discr, op.op_template())
        bnodes = discr.get_boundary("inflow").nodes
        dt = op.estimate_timestep(discr)
        u = u_an(discr.nodes, 0.0)[None]
        res = np.zeros_like(u)
        for step in range(int(1 / dt)):
            u, res = o.lsrk4_step(u, step * dt, dt, res,
                                  bc_fn=lambda t: u_an(bnodes, t))
            err = u[0] - u[0][perm]
            M = discr.ldis.mass_matrix
            l2 = math.sqrt(np.einsum("ki,ij,kj,k->", err.reshape(discr.K, -1), M,
                                     err.reshape(discr.K, -1), np.abs(mesh.jacobians)))
            assert l2 < 4e-15


@pytest.mark.slow
def test_convergence_advec_2d():
    """test_jit_discretization.py:842-912 (periodic rectangle part): EOC in
    the order N > 4 over all orders and > 10 for the last pair."""
    v = np.array([0.27, 0.0])
    na = np.linalg.norm(v)

    def u_an(x, t):
        return np.sin(-(x @ v) / na + t * na)

    def tagger(fvi, el, fn, allv):
        return ["outflow"]
    mesh = hb.make_regular_rect_mesh((0, 0), (2 * math.pi, 1), (8, 4),
                                     periodicity=(True, False), boundary_tagger=tagger)
    for flux_type in hb.StrongAdvectionOperator.flux_types:
        errs = []
        orders = [1, 2, 3, 4, 5, 6]
        for order in orders:
            discr = hb.Discretization(mesh, order=order)
            op = hb.StrongAdvectionOperator(v, flux_type=flux_type)
            o = orc.OracleRHS(discr, op.op_template())
            dt = op.estimate_timestep(discr)
            n = int(1 / dt)
            u = u_an(discr.nodes, 0)[None]
            res = np.zeros_like(u)
            for step in range(n):
                u, res = o.lsrk4_step(u, step * dt, dt, res)
            e = u[0] - u_an(discr.nodes, n * dt)
            M = discr.ldis.mass_matrix
            errs.append(math.sqrt(np.einsum("ki,ij,kj,k->", e.reshape(discr.K, -1), M,
                                            e.reshape(discr.K, -1),
                                            np.abs(mesh.jacobians))))
        lo, le = np.log10(orders), np.log10(errs)
        assert -np.polyfit(lo, le, 1)[0] > 4
        assert -np.polyfit(lo[-2:], le[-2:], 1)[0] > 10
