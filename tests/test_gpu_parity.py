"""GPU parity: the CUDA right-hand side through the C ABI against the CPU
oracle (a restatement of the reference jit backend), on the same seeded
inputs.  FP64: relative L2 <= 1e-12 per RHS; FP32: <= 1e-5; gather maps
bit-exact in canonical form."""
import numpy as np
import pytest

import hedge_b200 as hb
from conftest import rel_l2

pytestmark = pytest.mark.gpu

# "fp32" runs the contractions on the tensor cores (FP16x3) where that
# instance is built, "fp32-simt" always on CUDA cores
TOL = {"fp64": 1e-12, "fp32": 1e-5, "fp32-simt": 1e-5}


def _fields(discr, F, seed):
    rng = np.random.default_rng(seed)
    x = discr.nodes
    base = np.stack([np.sin(1.3 * (f + 1) * x[:, 0] + 0.7 * f) *
                     np.cos(0.9 * x[:, -1] - 0.3 * f) for f in range(F)])
    return base + 0.1 * rng.uniform(-1, 1, base.shape)


def _check(discr, op, precision, seed=0, bc_in=None, c_field=None, source=None):
    from oracle import OracleRHS
    ot = op.op_template()
    comp = discr.compile(ot, precision=precision)
    if c_field is not None:
        comp.set_coefficient(c_field)
    if source is not None:
        comp.set_source(source)
    q = _fields(discr, op.descriptor().n_fields, seed)
    orc = OracleRHS(discr, ot, c_field=c_field, source=source)
    ref = orc(q, bc_in=bc_in)
    fp32 = precision in ("fp32", "fp32-simt")
    qs = q.astype(np.float32).astype(np.float64) if fp32 else q
    if fp32:
        ref = orc(qs, bc_in=bc_in)
    out = comp(w=qs, bc_in=bc_in)
    comp.check()
    got = out.double().cpu().numpy().reshape(ref.shape)
    err = rel_l2(got, ref)
    assert err <= TOL[precision], (precision, err)
    return err


def rect(n=9, periodic=True, jitter=0.0, seed=None):
    return hb.make_regular_rect_mesh((-1, -1), (1, 1), (n, n),
                                     periodicity=(periodic, periodic) if periodic else None,
                                     jitter=jitter, seed=seed)


def box(n=3, jitter=0.0, seed=None):
    return hb.make_box_tet_mesh(n=(n, n, n), jitter=jitter, seed=seed)


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32-simt"])
@pytest.mark.parametrize("flux", ["upwind", "central", "lf"])
def test_advection_2d_periodic(cuda_device, precision, flux):
    d = hb.Discretization(rect(9, True, 0.2 / 8, 0), order=4)
    _check(d, hb.StrongAdvectionOperator(np.array([1.0, 0.5]), flux_type=flux), precision)


@pytest.mark.parametrize("order", [1, 3, 6])
def test_advection_2d_inflow(cuda_device, order):
    m = rect(7, periodic=False, jitter=0.02, seed=1)
    d = hb.Discretization(m, order=order)

    def tagger(fvi, el, fn, allv):
        return ["inflow"]
    m2 = hb.make_regular_rect_mesh((-1, -1), (1, 1), (7, 7), boundary_tagger=tagger,
                                   jitter=0.02, seed=1)
    d = hb.Discretization(m2, order=order)
    op = hb.StrongAdvectionOperator(np.array([0.6, -0.8]), flux_type="upwind",
                                    inflow_tag="inflow")
    bc = np.sin(3 * d.get_boundary("inflow").nodes[:, 0])
    _check(d, op, "fp64", bc_in=bc)


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32-simt"])
@pytest.mark.parametrize("flux", ["upwind", "central"])
def test_wave_2d_dirichlet(cuda_device, precision, flux):
    d = hb.Discretization(rect(8, False, 0.02, 2), order=5)
    _check(d, hb.StrongWaveOperator(-0.7, 2, flux_type=flux), precision)


def test_wave_2d_mixed_bcs(cuda_device):
    def tagger(fvi, el, fn, allv):
        x = allv[list(fvi)].mean(0)
        if x[0] < -0.99:
            return ["neu"]
        if x[0] > 0.99:
            return ["rad"]
        return ["dir"]
    m = hb.make_regular_rect_mesh((-1, -1), (1, 1), (8, 8), boundary_tagger=tagger)
    d = hb.Discretization(m, order=3)
    op = hb.StrongWaveOperator(1.0, 2, dirichlet_tag="dir", neumann_tag="neu",
                               radiation_tag="rad", source_f=0)
    _check(d, op, "fp64")


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32-simt"])
def test_wave_3d(cuda_device, precision):
    d = hb.Discretization(box(3, 0.05, 3), order=4)
    _check(d, hb.StrongWaveOperator(1.0, 3, flux_type="upwind"), precision)


def _lr_tagger(names):
    def tagger(fvi, el, fn, allv):
        x = allv[list(fvi)].mean(0)
        if x[0] < -0.99:
            return [names[0]]
        if x[0] > 0.99:
            return [names[1]]
        return [names[2]]
    return tagger


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32-simt", "fp16x3", "bf16x3"])
@pytest.mark.parametrize("dim", [2, 3])
def test_wave_dirichlet_data(cuda_device, precision, dim):
    """Inhomogeneous Dirichlet data g on a tag (ext state (2g - u, v),
    wave.py:133-142), given as the boundary vector dir_bc_u."""
    from oracle import OracleRHS
    tagger = _lr_tagger(["neu", "dir", "dir"])
    m = hb.make_regular_rect_mesh((-1, -1), (1, 1), (8, 8), boundary_tagger=tagger,
                                  jitter=0.02, seed=5) if dim == 2 else \
        hb.make_box_tet_mesh(n=(3, 3, 3), jitter=0.03, seed=5, boundary_tagger=tagger)
    d = hb.Discretization(m, order=4)
    op = hb.StrongWaveOperator(1.2, dim, dirichlet_tag="dir", dirichlet_bc_f=1,
                               neumann_tag="neu")
    g = np.cos(2 * d.get_boundary("dir").nodes[:, 1]) + 0.3
    q = _fields(d, dim + 1, 7)
    fp32 = precision in ("fp32", "fp32-simt")
    qs = q.astype(np.float32).astype(np.float64) if fp32 else q
    ref = OracleRHS(d, op.op_template())(qs, bc_in=g)
    comp = d.compile(op.op_template(), precision=precision)
    got = comp(w=qs, dir_bc_u=g).double().cpu().numpy()
    comp.check()
    tol = {"fp64": 1e-12, "fp32": 1e-5, "fp32-simt": 1e-5, "fp16x3": 1e-6, "bf16x3": 1e-5}
    assert rel_l2(got, ref) <= tol[precision]


def test_wave_dirichlet_data_time_dependent_steps(cuda_device):
    """Time-dependent Dirichlet data given as a function: the bound RHS and
    the fused LSRK4 stages evaluate it at every stage time; 20 steps against
    the oracle's LSRK4 with the same data."""
    from oracle import OracleRHS
    m = hb.make_regular_rect_mesh((-1, -1), (1, 1), (9, 9), jitter=0.02, seed=6,
                                  boundary_tagger=_lr_tagger(["dir", "rad", "dir"]))
    d = hb.Discretization(m, order=4)
    gf = hb.TimeDependentGivenFunction(lambda x, t: np.sin(3 * t) * np.cos(x[:, 1]))
    op = hb.StrongWaveOperator(1.0, 2, dirichlet_tag="dir", dirichlet_bc_f=gf,
                               radiation_tag="rad")
    rhs = op.bind(d)
    q = _fields(d, 3, 8)
    dt = 0.5 * op.estimate_timestep(d)
    orc = OracleRHS(d, op.op_template())
    y = d.to_device(q).reshape(3, -1)
    yo, res, t = q.copy(), np.zeros_like(q), 0.0
    st = hb.LSRK4TimeStepper()
    for _ in range(20):
        y = st(y, t, dt, rhs)
        yo, res = orc.lsrk4_step(yo, t, dt, res,
                                 bc_fn=lambda tt: gf.boundary_interpolant(tt, d, "dir"))
        t += dt
    rhs.compiled.check()
    assert rel_l2(y.cpu().numpy(), yo) <= 1e-11


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32-simt", "fp16x3", "bf16x3"])
def test_maxwell_current(cuda_device, precision):
    """Maxwell with a source current J [3, K*Np] (em.py:192-214), given with
    the model and as the template's field ``current`` per call."""
    from oracle import OracleRHS
    d = hb.Discretization(box(3, 0.04, 9), order=4)
    rng = np.random.default_rng(9)
    J = np.sin(d.nodes.T) + 0.1 * rng.uniform(-1, 1, (3, len(d)))
    op = hb.MaxwellOperator(1.5, 0.8, flux_type=1, current=J)
    q = _fields(d, 6, 10)
    fp32 = precision in ("fp32", "fp32-simt")
    qs = q.astype(np.float32).astype(np.float64) if fp32 else q
    ref = OracleRHS(d, op.op_template())(qs)
    tol = {"fp64": 1e-12, "fp32": 1e-5, "fp32-simt": 1e-5, "fp16x3": 1e-6, "bf16x3": 1e-5}
    rhs = op.bind(d.__class__(d.mesh, order=4, precision=precision))
    got = rhs(0.0, qs).double().cpu().numpy()
    rhs.compiled.check()
    assert rel_l2(got, ref) <= tol[precision]
    # the same template with the current passed per call
    comp = d.__class__(d.mesh, order=4, precision=precision).compile(op.op_template())
    J2 = 2 * J
    ref2 = OracleRHS(d, hb.MaxwellOperator(1.5, 0.8, flux_type=1, current=J2).op_template())(qs)
    got2 = comp(w=qs, current=J2).double().cpu().numpy()
    comp.check()
    assert rel_l2(got2, ref2) <= tol[precision]


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32-simt"])
@pytest.mark.parametrize("kind", ["tm", "te"])
def test_maxwell_2d(cuda_device, kind, precision):
    """2D TM (Ez, Hx, Hy) and TE (Ex, Ey, Hz) Maxwell (em.py:485-515): PEC, PMC
    and absorbing walls, a numeric interior and an "lf" boundary flux, and a
    source current, against the oracle."""
    from oracle import OracleRHS
    m = hb.make_regular_rect_mesh((-1, -1), (1, 1), (9, 9), jitter=0.03, seed=11,
                                  boundary_tagger=_lr_tagger(["pmc", "abs", "pec"]))
    d = hb.Discretization(m, order=5, precision=precision)
    cls = hb.TMMaxwellOperator if kind == "tm" else hb.TEMaxwellOperator
    ne = 1 if kind == "tm" else 2
    J = np.cos(d.nodes.T[:ne] * 2.0)
    op = cls(1.2, 0.9, flux_type=0.7, bdry_flux_type="lf", pec_tag="pec", pmc_tag="pmc",
             absorb_tag="abs", current=J)
    q = _fields(d, 3, 12)
    fp32 = precision != "fp64"
    qs = q.astype(np.float32).astype(np.float64) if fp32 else q
    ref = OracleRHS(d, op.op_template())(qs)
    # the reference's bind checks only the PEC, absorbing and incident tags
    # (em.py:373-377), so a mesh with PMC walls is compiled directly
    rhs = d.compile(op.op_template()).bind_model(op)
    got = rhs(0.0, qs).double().cpu().numpy()
    rhs.compiled.check()
    assert rel_l2(got, ref) <= (1e-12 if precision == "fp64" else 1e-5)


@pytest.mark.parametrize("kind", ["tm", "te"])
def test_maxwell_2d_lsrk_steps(cuda_device, kind):
    """20 fused LSRK4 steps of a PEC cavity mode against the oracle's."""
    from oracle import OracleRHS
    d = hb.Discretization(rect(8, False, 0.02, 13), order=4)
    cls = hb.TMMaxwellOperator if kind == "tm" else hb.TEMaxwellOperator
    op = cls(1.0, 1.0, flux_type=1)
    x, y = d.nodes.T
    q = np.stack([np.sin(np.pi * (x + 1) / 2) * np.sin(np.pi * (y + 1) / 2),
                  0 * x, 0 * x]) if kind == "tm" else _fields(d, 3, 14)
    rhs = op.bind(d)
    dt = 0.5 * op.estimate_timestep(d)
    orc = OracleRHS(d, op.op_template())
    yd = d.to_device(q).reshape(3, -1)
    yo, res, t = q.copy(), np.zeros_like(q), 0.0
    st = hb.LSRK4TimeStepper()
    for _ in range(20):
        yd = st(yd, t, dt, rhs)
        yo, res = orc.lsrk4_step(yo, t, dt, res)
        t += dt
    rhs.compiled.check()
    assert rel_l2(yd.cpu().numpy(), yo) <= 1e-11


@pytest.mark.parametrize("dim", [2, 3])
def test_varwave(cuda_device, dim):
    m = rect(8, False, 0.02, 4) if dim == 2 else box(2, 0.03, 4)
    d = hb.Discretization(m, order=5 if dim == 2 else 3)
    rng = np.random.default_rng(4)
    ck = rng.uniform(0.8, 1.2, d.K)
    c = np.repeat(ck, d.Np)
    src = np.exp(-10 * (d.nodes ** 2).sum(1))
    op = hb.VariableVelocityStrongWaveOperator(c, dim, flux_type="upwind", source=src)
    _check(d, op, "fp64", c_field=c, source=src)


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32-simt"])
@pytest.mark.parametrize("flux", [1, 0.5, 0, "lf"])
def test_maxwell_pec(cuda_device, precision, flux):
    d = hb.Discretization(box(3, 0.05, 5), order=4)
    _check(d, hb.MaxwellOperator(1.0, 1.0, flux_type=flux), precision)


def test_maxwell_material_absorbing(cuda_device):
    def tagger(fvi, el, fn, allv):
        x = allv[list(fvi)].mean(0)
        return ["abs"] if x[2] > 0.99 else ["pec"]
    m = hb.make_box_tet_mesh(n=(3, 3, 3), jitter=0.04, seed=6, boundary_tagger=tagger)
    d = hb.Discretization(m, order=3)
    op = hb.MaxwellOperator(2.0, 0.5, flux_type=1, pec_tag="pec", absorb_tag="abs")
    _check(d, op, "fp64")


@pytest.mark.parametrize("order", [1, 2, 7])
def test_maxwell_orders(cuda_device, order):
    d = hb.Discretization(box(2, 0.05, 7), order=order)
    _check(d, hb.MaxwellOperator(1.0, 1.0, flux_type=1), "fp64")


def test_gather_map_bit_exact(cuda_device):
    """Device-expanded gather indices == the reference face group's index
    lists, in canonical (sorted pair) form."""
    from hedge_b200.facegroups import gather_index_pairs_from_face_group
    for m, order in ((rect(9, True, 0.02, 0), 4), (box(3, 0.05, 1), 4), (box(2), 7)):
        d = hb.Discretization(m, order=order)
        op = hb.StrongWaveOperator(1.0, m.dimensions) if m.dimensions == 3 else \
            hb.StrongAdvectionOperator(np.array([1.0, 0.0]))
        comp = d.compile(op.op_template())
        ii, ee = comp.gather_map()
        comp.check()
        ii, ee = ii.cpu().numpy(), ee.cpu().numpy()
        ok = ee >= 0
        pairs = np.stack([ii[ok], ee[ok]], 1)
        pairs = pairs[np.lexsort((pairs[:, 1], pairs[:, 0]))]
        ref = gather_index_pairs_from_face_group(d.interior_face_group, d.Np)
        assert np.array_equal(pairs, ref)
        # boundary face nodes: (element, face, node) -> volume index
        for tag in (hb.TAG_ALL,):
            b = d.get_boundary(tag)
            if b.is_empty():
                continue
            e, f = b.element_faces[:, 0], b.element_faces[:, 1]
            slots = ((e * d.Nfaces + f)[:, None] * d.Nfp + np.arange(d.Nfp)).ravel()
            assert np.array_equal(ii[slots], b.vol_indices)
            assert np.all(ee[slots] < 0)


@pytest.mark.parametrize("model", ["advection", "maxwell"])
def test_fused_lsrk_matches_oracle(cuda_device, model):
    import torch
    from oracle import OracleRHS
    if model == "advection":
        d = hb.Discretization(rect(9, True, 0.02, 0), order=4)
        op = hb.StrongAdvectionOperator(np.array([1.0, 0.5]), flux_type="upwind")
    else:
        d = hb.Discretization(box(2, 0.05, 1), order=4)
        op = hb.MaxwellOperator(1.0, 1.0, flux_type=1)
    ot = op.op_template()
    rhs = op.bind(d)
    q = _fields(d, op.descriptor().n_fields, 9)
    dt = op.estimate_timestep(d) * 0.5
    stepper = hb.LSRK4TimeStepper()
    y = d.to_device(q).reshape(op.descriptor().n_fields, -1)
    orc = OracleRHS(d, ot)
    yo, res = q.copy(), np.zeros_like(q)
    t = 0.0
    for _ in range(3):
        y = stepper(y, t, dt, rhs)
        yo, res = orc.lsrk4_step(yo, t, dt, res)
        t += dt
    torch.cuda.synchronize()
    assert rel_l2(y.cpu().numpy().reshape(yo.shape), yo) <= 1e-12


def test_generic_stepper_path(cuda_device):
    """A plain callable rhs goes through hb_lincomb (the linear combiner)."""
    import torch
    d = hb.Discretization(rect(7, True), order=3)
    op = hb.StrongAdvectionOperator(np.array([1.0, 0.0]), flux_type="upwind")
    comp = d.compile(op.op_template())
    q = _fields(d, 1, 2)
    y0 = d.to_device(q).reshape(1, -1)
    fused = hb.LSRK4TimeStepper()(y0, 0.0, 1e-3, op.bind(d))
    generic = hb.LSRK4TimeStepper()(y0, 0.0, 1e-3,
                                    lambda t, w: comp(w=w).reshape(1, -1))
    assert rel_l2(generic.cpu().numpy(), fused.cpu().numpy()) <= 1e-13


def test_invalid_connectivity_rejected(cuda_device):
    from hedge_b200 import _native
    d = hb.Discretization(rect(5, True), order=2)
    comp = d.compile(hb.StrongAdvectionOperator(np.array([1.0, 0.0])).op_template())
    bad = comp.conn.copy()
    bad[0, 0, 0] = d.K + 5
    import ctypes as C
    desc = _native.hb_op_desc(1, 1, 0, 1, 1, (C.c_double * 3)(1, 0, 0), 0, 1, 1, 1, 1, 1,
                              bad.ctypes.data, 0)
    h = C.c_void_p()
    st = _native.load().hb_op_create(d._native_handle(), C.byref(desc), C.byref(h))
    assert st == _native.HB_ERR_INVALID_ARGUMENT
    assert b"out of range" in _native.load().hb_last_error_string()


def test_energy_norm_matches_oracle(cuda_device):
    """hb_norm (FP64, deterministic) vs sqrt(sum |J| u^T M u) in numpy."""
    for m, order in ((rect(9, True, 0.02, 0), 4), (box(3, 0.05, 1), 4)):
        d = hb.Discretization(m, order=order)
        u = _fields(d, 3, 5)
        M = d.ldis.mass_matrix
        J = np.abs(m.jacobians)
        uu = u.reshape(3, d.K, d.Np)
        ref = np.sqrt(np.einsum("fki,ij,fkj,k->", uu, M, uu, J))
        got = d.norm(u)
        assert abs(got - ref) <= 1e-13 * ref
        assert d.norm(u) == got   # bitwise reproducible
        d32 = hb.Discretization(m, order=order, default_scalar_type=np.float32)
        u32 = u.astype(np.float32)
        uu32 = u32.astype(np.float64).reshape(3, d.K, d.Np)
        ref32 = np.sqrt(np.einsum("fki,ij,fkj,k->", uu32, M, uu32, J))
        assert abs(d32.norm(u32) - ref32) <= 1e-12 * ref32
