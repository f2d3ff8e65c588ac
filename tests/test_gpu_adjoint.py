"""The hand-written adjoint of the RHS (hb_rhs_adjoint) and the gradients of
the checkpointed LSRK4 time loop built on it.

* RHS level: q_bar = J^T lam against the transpose of the oracle's Jacobian,
  assembled column by column from oracle RHS evaluations (R is affine in
  q), for every model and boundary kind; rel-L2 <= 1e-12.
* c gradient of the variable-velocity wave against oracle differences in
  each nodal c (R is linear in c); rel-L2 <= 1e-12.
* Time loop (receiver traces over LSRK4 steps, checkpointed): gradients in
  the initial field and the per-element c_k against central finite
  differences (h = 1e-6) on random directions (rel <= 1e-6) and against an
  FP64 reference gradient computed on the CPU from the oracle (<= 1e-10).
"""
import numpy as np
import pytest

import hedge_b200 as hb
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def rect(n, periodic=False, jitter=0.0, seed=None, tagger=None):
    return hb.make_regular_rect_mesh((-1, -1), (1, 1), (n, n),
                                     periodicity=(periodic, periodic) if periodic else None,
                                     jitter=jitter, seed=seed, boundary_tagger=tagger)


def _oracle_jacobian(orc, n_state, **kw):
    """Dense Jacobian of the oracle RHS (affine in the state)."""
    r0 = orc(np.zeros((orc.F, n_state // orc.F)), **kw).reshape(-1)
    J = np.empty((r0.size, n_state))
    e = np.zeros(n_state)
    for j in range(n_state):
        e[j] = 1.0
        J[:, j] = orc(e.reshape(orc.F, -1), **kw).reshape(-1) - r0
        e[j] = 0.0
    return J


def _check_adjoint(d, op, bc_in=None, c_field=None, source=None, seed=0):
    import torch
    from oracle import OracleRHS
    ot = op.op_template()
    comp = d.compile(ot, precision="fp64")
    if c_field is not None:
        comp.set_coefficient(c_field)
    F = op.descriptor().n_fields
    orc = OracleRHS(d, ot, c_field=c_field, source=source)
    orc.F = F
    n = F * len(d)
    kw = {"bc_in": bc_in} if bc_in is not None else {}
    J = _oracle_jacobian(orc, n, **kw)
    lam = np.random.default_rng(seed).standard_normal(n)
    ref = J.T @ lam
    q_bar, _ = comp.adjoint(torch.as_tensor(lam.reshape(F, -1), device=d.device))
    got = q_bar.cpu().numpy().reshape(-1)
    err = rel_l2(got, ref)
    assert err <= 1e-12, err
    return err


def test_adjoint_advection_periodic(cuda_device):
    d = hb.Discretization(rect(4, True, 0.05, 1), order=3)
    _check_adjoint(d, hb.StrongAdvectionOperator(np.array([1.0, 0.5]), flux_type="upwind"))


def test_adjoint_advection_central_inflow(cuda_device):
    m = rect(4, False, 0.05, 2, tagger=lambda fvi, el, fn, allv: ["inflow"])
    d = hb.Discretization(m, order=2)
    op = hb.StrongAdvectionOperator(np.array([0.6, -0.8]), flux_type="central",
                                    inflow_tag="inflow")
    bc = np.sin(3 * d.get_boundary("inflow").nodes[:, 0])
    _check_adjoint(d, op, bc_in=bc)


def test_adjoint_wave_mixed_bcs(cuda_device):
    def tagger(fvi, el, fn, allv):
        x = allv[list(fvi)].mean(0)
        if x[0] < -0.99:
            return ["neu"]
        if x[0] > 0.99:
            return ["rad"]
        return ["dir"]
    d = hb.Discretization(rect(4, tagger=tagger, jitter=0.03, seed=3), order=3)
    op = hb.StrongWaveOperator(-0.7, 2, dirichlet_tag="dir", neumann_tag="neu",
                               radiation_tag="rad", flux_type="upwind")
    _check_adjoint(d, op)


def test_adjoint_varwave_with_source(cuda_device):
    d = hb.Discretization(rect(4, jitter=0.05, seed=4), order=3)
    rng = np.random.default_rng(4)
    c = np.repeat(rng.uniform(0.8, 1.2, d.K), d.Np)
    src = np.exp(-4 * (d.nodes ** 2).sum(1))
    op = hb.VariableVelocityStrongWaveOperator(c, 2, flux_type="upwind", source=src)
    _check_adjoint(d, op, c_field=c, source=src)


@pytest.mark.parametrize("flux", [1, 0.5])
def test_adjoint_maxwell(cuda_device, flux):
    def tagger(fvi, el, fn, allv):
        x = allv[list(fvi)].mean(0)
        return ["abs"] if x[2] > 0.99 else ["pec"]
    m = hb.make_box_tet_mesh(n=(1, 1, 1), jitter=0.0, boundary_tagger=tagger)
    d = hb.Discretization(m, order=2)
    op = hb.MaxwellOperator(2.0, 0.5, flux_type=flux, pec_tag="pec", absorb_tag="abs")
    _check_adjoint(d, op)


@pytest.mark.parametrize("kind", ["tm", "te"])
def test_adjoint_maxwell_2d(cuda_device, kind):
    """2D TM / TE Maxwell (em.py:485-515) with PEC, PMC and absorbing walls."""
    def tagger(fvi, el, fn, allv):
        x = allv[list(fvi)].mean(0)
        return ["abs"] if x[0] > 0.99 else (["pmc"] if x[0] < -0.99 else ["pec"])
    m = hb.make_regular_rect_mesh((-1, -1), (1, 1), (4, 4), boundary_tagger=tagger,
                                  jitter=0.05, seed=3)
    d = hb.Discretization(m, order=3)
    cls = hb.TMMaxwellOperator if kind == "tm" else hb.TEMaxwellOperator
    op = cls(1.4, 0.6, flux_type=0.5, bdry_flux_type=1, pec_tag="pec", pmc_tag="pmc",
             absorb_tag="abs")
    _check_adjoint(d, op)


def test_adjoint_c_gradient(cuda_device):
    import torch
    from oracle import OracleRHS
    d = hb.Discretization(rect(4, jitter=0.05, seed=5), order=3)
    rng = np.random.default_rng(5)
    c = np.repeat(rng.uniform(0.8, 1.2, d.K), d.Np)
    op = hb.VariableVelocityStrongWaveOperator(c, 2, flux_type="upwind")
    ot = op.op_template()
    comp = d.compile(ot, precision="fp64")
    comp.set_coefficient(c)
    q = rng.standard_normal((3, len(d)))
    lam = rng.standard_normal((3, len(d)))
    orc = OracleRHS(d, ot, c_field=c)
    base = orc(q)
    ref = np.empty(len(d))
    for j in range(len(d)):
        orc.c_field = c.copy()
        orc.c_field[j] += 1.0
        ref[j] = np.sum(lam * (orc(q) - base))
    _, c_bar = comp.adjoint(torch.as_tensor(lam, device=d.device),
                            q=torch.as_tensor(q, device=d.device), want_c=True)
    err = rel_l2(c_bar.cpu().numpy(), ref)
    assert err <= 1e-12, err


def test_rhs_function_autograd(cuda_device):
    """torch.autograd through RHSFunction: <lam, dR> = <grad, d(q, c)>."""
    import torch
    from hedge_b200.adjoint import RHSFunction
    d = hb.Discretization(rect(6, jitter=0.05, seed=6), order=4)
    rng = np.random.default_rng(6)
    c0 = np.repeat(rng.uniform(0.8, 1.2, d.K), d.Np)
    comp = hb.VariableVelocityStrongWaveOperator(c0, 2).bind(d).compiled
    dev = d.device
    q = torch.tensor(rng.standard_normal((3, len(d))), device=dev, requires_grad=True)
    ck = torch.tensor(rng.uniform(0.8, 1.2, d.K), device=dev, requires_grad=True)
    lam = torch.as_tensor(rng.standard_normal((3, len(d))), device=dev)
    out = RHSFunction.apply(q, ck.repeat_interleave(d.Np), comp)
    (out * lam).sum().backward()
    dq = torch.as_tensor(rng.standard_normal((3, len(d))), device=dev)
    dc = torch.as_tensor(rng.standard_normal(d.K), device=dev)
    h = 1e-6
    with torch.no_grad():
        fp = RHSFunction.apply(q + h * dq, (ck + h * dc).repeat_interleave(d.Np), comp)
        fm = RHSFunction.apply(q - h * dq, (ck - h * dc).repeat_interleave(d.Np), comp)
    fd = float(((fp - fm) * lam).sum()) / (2 * h)
    an = float((q.grad * dq).sum() + (ck.grad * dc).sum())
    assert abs(fd - an) <= 1e-8 * abs(an), (fd, an)


def _small_problem(n=7, order=3, nrec=4):
    from hedge_b200.adjoint import make_wave_inversion_problem
    return make_wave_inversion_problem(n=n, order=order, n_receivers=nrec, f0=3.0)


def _loss(P, q0, ck, nsteps, every):
    from hedge_b200.adjoint import ReceiverTraces, trace_loss
    d = P["discr"]
    tr = ReceiverTraces.apply(q0, ck.repeat_interleave(d.Np), P["comp"], P["receivers"],
                              P["dt"], nsteps, P["source"], every)
    return trace_loss(tr)


def test_time_loop_gradient_vs_finite_differences(cuda_device):
    import torch
    P = _small_problem()
    d = P["discr"]
    rng = np.random.default_rng(11)
    x = d.nodes
    q0 = torch.as_tensor(np.stack([np.exp(-8 * ((x - 0.2) ** 2).sum(1)),
                                   0 * x[:, 0], 0 * x[:, 0]]), device=d.device)
    ck = P["c_k"].clone()
    q0.requires_grad_(True)
    ck.requires_grad_(True)
    nsteps, every = 24, 7
    L = _loss(P, q0, ck, nsteps, every)
    L.backward()
    gq, gc = q0.grad.clone(), ck.grad.clone()
    h = 1e-6
    worst = 0.0
    for k in range(6):
        dq = torch.as_tensor(rng.standard_normal(q0.shape), device=d.device) if k < 3 \
            else torch.zeros_like(q0)
        dc = torch.as_tensor(rng.standard_normal(ck.shape), device=d.device) if k >= 3 \
            else torch.zeros_like(ck)
        with torch.no_grad():
            lp = float(_loss(P, q0 + h * dq, ck + h * dc, nsteps, every))
            lm = float(_loss(P, q0 - h * dq, ck - h * dc, nsteps, every))
        fd = (lp - lm) / (2 * h)
        an = float((gq * dq).sum() + (gc * dc).sum())
        worst = max(worst, abs(fd - an) / abs(an))
    assert worst <= 1e-6, worst


def test_time_loop_gradient_vs_cpu_reference(cuda_device):
    """FP64 reference gradient on the CPU: oracle forward, transpose of the
    oracle's Jacobian and oracle c-derivatives, same LSRK4 recurrences."""
    import torch
    from oracle import OracleRHS
    from hedge_b200.timestep import RK4A, RK4B, RK4C
    P = _small_problem(n=4, order=2, nrec=2)
    d, comp, rec = P["discr"], P["comp"], P["receivers"]
    vec, amp = P["source"]
    vec_h = vec.cpu().numpy()
    K, Np, F = d.K, d.Np, 3
    n = F * len(d)
    nsteps, every, dt = 8, 3, P["dt"]
    rng = np.random.default_rng(12)
    q0 = rng.standard_normal((F, len(d))) * 0.1
    ck = P["c_k"].cpu().numpy()
    c_nodes = np.repeat(ck, Np)
    ot = P["op"].op_template()
    orc = OracleRHS(d, ot, c_field=c_nodes)
    orc.F = F
    J = _oracle_jacobian(orc, n)

    def R(q, t, c=None):
        orc.c_field = c_nodes if c is None else c
        r = orc(q)
        r[0] -= amp(t) * vec_h
        return r
    # receiver operator on the host
    Pm = np.zeros((len(rec.coeff), n))
    idx = rec.idx.cpu().numpy()
    co = rec.coeff.cpu().numpy()
    for r in range(len(co)):
        Pm[r, idx[r]] = co[r]
    # forward with stage inputs
    q, t, states, stages = q0.copy(), 0.0, [q0.copy()], []
    for _ in range(nsteps):
        res = np.zeros_like(q)
        keep = []
        for s in range(5):
            keep.append(q.copy())
            res = RK4A[s] * res + dt * R(q, t + RK4C[s] * dt)
            q = q + RK4B[s] * res
        stages.append(keep)
        states.append(q.copy())
        t += dt
    traces = np.array([Pm @ s.reshape(-1) for s in states])
    # reverse
    lq = Pm.T @ (2 * traces[nsteps])
    gc = np.zeros(K)
    for step in range(nsteps - 1, -1, -1):
        lres = np.zeros(n)
        for s in range(4, -1, -1):
            lres = lres + RK4B[s] * lq
            lq = lq + dt * (J.T @ lres)
            qs = stages[step][s]
            for k in range(K):
                ind = np.zeros(len(d))
                ind[k * Np:(k + 1) * Np] = 1.0
                orc.c_field = ind
                lk = orc(qs).reshape(-1)
                orc.c_field = np.zeros(len(d))
                l0 = orc(qs).reshape(-1)
                gc[k] += dt * lres @ (lk - l0)
            lres = RK4A[s] * lres
        lq = lq + Pm.T @ (2 * traces[step])
    # GPU
    q0t = torch.tensor(q0, device=d.device, requires_grad=True)
    ckt = torch.tensor(ck, device=d.device, requires_grad=True)
    L = _loss(P, q0t, ckt, nsteps, every)
    assert abs(float(L.detach()) - float((traces ** 2).sum())) <= 1e-11 * float((traces ** 2).sum())
    L.backward()
    eq = rel_l2(q0t.grad.cpu().numpy().reshape(-1), lq)
    ec = rel_l2(ckt.grad.cpu().numpy(), gc)
    assert eq <= 1e-10 and ec <= 1e-10, (eq, ec)
