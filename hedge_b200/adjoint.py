"""Gradients through the DG right-hand side and through LSRK4 time loops.

* ``RHSFunction``: ``torch.autograd.Function`` around one RHS evaluation
  (hb_rhs forward, hb_rhs_adjoint backward): gradients with respect to the
  state and, for the variable-velocity wave, the nodal wave speed.
* ``ReceiverTraces``: ``torch.autograd.Function`` around a whole LSRK4 time
  loop (hedge/timestep/runge_kutta.py:104-131) that records point receivers
  (hedge/discretization/__init__.py:1217-1249) after every step.  Forward
  keeps only a checkpoint of the state every ``checkpoint_every`` steps;
  backward recomputes each segment's stage states from its checkpoint and
  runs the discrete adjoint of the LSRK4 recurrences through it:

      res_s = a_s res_{s-1} + dt R(q_{s-1}, t_s),   q_s = q_{s-1} + b_s res_s

  reversed as   lres += b_s lq;  lq += dt R_q^T lres;  c_bar += dt R_c^T lres;
  lres *= a_s   (a_1 = 0 cuts the residual between steps).

The reference has no adjoint; the forward it differentiates is the
reference's RHS and LSRK4 stepper, unchanged.
"""

from __future__ import annotations

import numpy as np

from .timestep import RK4A, RK4B, RK4C


def _torch():
    import torch
    return torch


class RHSFunction:
    """``RHSFunction.apply(q, c, comp)`` -> R(q; c) as [F, K*Np] FP64.

    ``q``: [F, K*Np] state; ``c``: nodal c field [K*Np] (variable-velocity
    wave) or None; ``comp``: a CompiledOperator with FP64 state.
    """

    _fn = None

    @classmethod
    def apply(cls, q, c, comp):
        if cls._fn is None:
            torch = _torch()

            class _F(torch.autograd.Function):
                @staticmethod
                def forward(ctx, q, c, comp):
                    qq = comp.as_state(q)
                    cc = c.detach().contiguous() if c is not None else None
                    out = comp.discr.volume_empty((comp.F,), torch.float64)
                    comp.rhs_into(qq, out, coeff=cc)
                    ctx.comp = comp
                    ctx.save_for_backward(qq, cc if cc is not None else torch.empty(0))
                    ctx.has_c = cc is not None
                    return out

                @staticmethod
                def backward(ctx, g):
                    qq, cc = ctx.saved_tensors
                    cc = cc if ctx.has_c else None
                    want_c = ctx.has_c and ctx.needs_input_grad[1]
                    q_bar, c_bar = ctx.comp.adjoint(g.contiguous(), q=qq, coeff=cc,
                                                    want_c=want_c)
                    return q_bar.reshape(qq.shape), c_bar, None

            cls._fn = _F
        return cls._fn.apply(q, c, comp)


class Receivers:
    """Point receivers on field ``field`` (default 0): trace value at receiver
    r = sum_i coeff[r, i] * q[field, el[r]*Np + i] (the reference's point
    evaluator, hedge/discretization/__init__.py:1217-1249)."""

    def __init__(self, discr, points, field=0):
        torch = _torch()
        evs = [discr.get_point_evaluator(p) for p in points]
        Np = discr.Np
        self.field = field
        self.idx = torch.as_tensor(
            np.array([[ev.el * Np + i for i in range(Np)] for ev in evs]), device=discr.device)
        self.coeff = torch.as_tensor(np.array([ev.coeff for ev in evs]), dtype=torch.float64,
                                     device=discr.device)

    def __call__(self, q):
        return (q[self.field][self.idx] * self.coeff).sum(dim=1)

    def transpose(self, g, like):
        """P^T g as a state-shaped tensor (g: one trace row [n_receivers])."""
        out = _torch().zeros_like(like)
        out[self.field].index_add_(0, self.idx.reshape(-1),
                                   (self.coeff * g[:, None]).reshape(-1))
        return out


def projected_point_source(discr, point):
    """Nodal vector whose element-local L2 projection reproduces a point
    delta: on the element containing ``point``, M^-1 l(x_s) / |J| (l = the
    nodal basis at the point), zero elsewhere."""
    ev = discr.get_point_evaluator(point)
    ld = discr.ldis
    vec = np.zeros(len(discr))
    jac = abs(discr.mesh.jacobians[ev.el])
    vec[ev.el * discr.Np:(ev.el + 1) * discr.Np] = ld.inverse_mass_matrix @ ev.coeff / jac
    return vec


def ricker(t, f0, t0=None):
    """Ricker wavelet of peak frequency f0 centred at t0 (default 1/f0)."""
    t0 = 1.0 / f0 if t0 is None else t0
    a = (np.pi * f0 * (t - t0)) ** 2
    return (1.0 - 2.0 * a) * np.exp(-a)


class ReceiverTraces:
    """``ReceiverTraces.apply(q0, c, comp, receivers, dt, nsteps, source,
    checkpoint_every)`` -> traces [nsteps + 1, n_receivers] (after every step,
    step 0 = the initial state).  ``source``: None or (vector [K*Np] FP64
    tensor, amplitude function of t); the RHS gets amplitude(t) * vector at
    every stage time.  Differentiable in q0 and c (nodal, variable-velocity
    wave)."""

    _fn = None

    @staticmethod
    def _stage_source(source, t):
        if source is None:
            return None
        vec, amp = source
        return vec * float(amp(t))

    @classmethod
    def _step(cls, comp, q, res, c, dt, t, source, keep=None):
        torch = _torch()
        cur = q
        for s in range(5):
            a, b, cs = RK4A[s], RK4B[s], RK4C[s]
            if keep is not None:
                keep.append(cur)
            nxt = torch.empty_like(cur)
            comp.lsrk_stage(a, b, dt, cur, nxt, res, coeff=c,
                            source=cls._stage_source(source, t + cs * dt))
            cur = nxt
        return cur

    @classmethod
    def apply(cls, q0, c, comp, receivers, dt, nsteps, source=None, checkpoint_every=20):
        if cls._fn is None:
            torch = _torch()

            class _F(torch.autograd.Function):
                @staticmethod
                def forward(ctx, q0, c, comp, receivers, dt, nsteps, source, every):
                    q = comp.as_state(q0).clone()
                    cc = c.detach().contiguous() if c is not None else None
                    res = torch.zeros_like(q)
                    traces = [receivers(q)]
                    checkpoints = {0: q}
                    t = 0.0
                    for n in range(nsteps):
                        q = cls._step(comp, q, res, cc, dt, t, source)
                        t += dt
                        traces.append(receivers(q))
                        if (n + 1) % every == 0 and n + 1 < nsteps:
                            checkpoints[n + 1] = q
                    ctx.comp, ctx.receivers, ctx.dt, ctx.nsteps = comp, receivers, dt, nsteps
                    ctx.source, ctx.every, ctx.checkpoints = source, every, checkpoints
                    ctx.has_c = cc is not None
                    ctx.save_for_backward(cc if cc is not None else torch.empty(0))
                    return torch.stack(traces)

                @staticmethod
                def backward(ctx, g):
                    (cc,) = ctx.saved_tensors
                    cc = cc if ctx.has_c else None
                    comp, rec, dt = ctx.comp, ctx.receivers, ctx.dt
                    want_c = ctx.has_c and ctx.needs_input_grad[1]
                    q_last = ctx.checkpoints[0]
                    lq = rec.transpose(g[ctx.nsteps], q_last)
                    c_bar = torch.zeros_like(cc) if want_c else None
                    starts = sorted(ctx.checkpoints)
                    ends = starts[1:] + [ctx.nsteps]
                    for s0, s1 in reversed(list(zip(starts, ends))):
                        # recompute the segment's stage inputs
                        q = ctx.checkpoints[s0]
                        res = torch.zeros_like(q)
                        stages = []
                        t = s0 * dt
                        for n in range(s0, s1):
                            keep = []
                            q = cls._step(comp, q, res, cc, dt, t, ctx.source, keep)
                            stages.append(keep)
                            t += dt
                        # reverse through the segment
                        for n in range(s1 - 1, s0 - 1, -1):
                            keep = stages[n - s0]
                            lres = torch.zeros_like(lq)
                            for s in range(4, -1, -1):
                                lres = lres + RK4B[s] * lq
                                q_bar, cb = comp.adjoint(lres, q=keep[s], coeff=cc,
                                                         want_c=want_c)
                                lq = lq + dt * q_bar
                                if want_c:
                                    c_bar = c_bar + dt * cb
                                lres = RK4A[s] * lres
                            lq = lq + rec.transpose(g[n], lq)
                    q0_bar = lq.reshape(ctx.checkpoints[0].shape)
                    return q0_bar, c_bar, None, None, None, None, None, None

            cls._fn = _F
        return cls._fn.apply(q0, c, comp, receivers, dt, nsteps, source, checkpoint_every)


def make_wave_inversion_problem(n=61, order=5, jitter=0.1, mesh_seed=3, c_seed=4,
                                n_receivers=16, receiver_seed=8, f0=4.0, device=None):
    """The adjoint workload: 2D variable-velocity acoustic wave on [-1,1]^2
    ((n-1)^2 x 2 jittered triangles; n = 61 gives K = 7200), order 5, per-
    element c_k ~ U[0.8, 1.2], reflecting (Dirichlet) walls, a Ricker point
    source at the origin and seeded receivers.  Returns a dict with the
    discretization, compiled operator, receivers, source, c_k and dt."""
    import hedge_b200 as hb
    torch = _torch()
    h = 2.0 / (n - 1)
    mesh = hb.make_regular_rect_mesh((-1, -1), (1, 1), (n, n), jitter=jitter * h,
                                     seed=mesh_seed)
    discr = hb.Discretization(mesh, order=order, device=device)
    K, Np = discr.K, discr.Np
    rng = np.random.default_rng(c_seed)
    c_k = rng.uniform(0.8, 1.2, K)
    c_nodes = np.repeat(c_k, Np)
    op = hb.VariableVelocityStrongWaveOperator(c_nodes, 2, flux_type="upwind")
    comp = op.bind(discr).compiled
    rr = np.random.default_rng(receiver_seed)
    pts = rr.uniform(-0.8, 0.8, (n_receivers, 2))
    receivers = Receivers(discr, pts)
    src_vec = torch.as_tensor(projected_point_source(discr, (0.013, -0.007)),
                              dtype=torch.float64, device=discr.device)
    # the var-c wave subtracts its source from du/dt
    source = (src_vec, lambda t: -ricker(t, f0))
    # The variable-velocity upwind flux (hedge/models/wave.py:246-273) carries
    # twice the jump penalty of the constant-c one, which puts its spectrum
    # outside the LSRK4 region at the reference's CFL estimate (the solution
    # grows without bound there); half of the estimate is stable.
    dt = 0.5 * op.estimate_timestep(discr)
    return {"discr": discr, "op": op, "comp": comp, "receivers": receivers,
            "source": source, "c_k": torch.as_tensor(c_k, device=discr.device),
            "dt": dt}


def trace_loss(traces):
    """Squared L2 of the receiver traces over all steps."""
    return (traces * traces).sum()


def check_gradients(P, nsteps=400, every=20, ndirs=32, h=1e-6, seed=5, q0=None):
    """Gradient of the trace loss in (q0, c_k) by the adjoint, against central
    finite differences on ``ndirs`` random joint directions.  Returns a dict
    with the loss, the worst and median relative disagreement and timings
    (forward, forward + backward) in seconds."""
    import time
    torch = _torch()
    d = P["discr"]
    rng = np.random.default_rng(seed)
    if q0 is None:
        q0 = torch.zeros((3, len(d)), dtype=torch.float64, device=d.device)
    q0 = q0.clone().requires_grad_(True)
    ck = P["c_k"].clone().requires_grad_(True)

    def loss(q, c):
        tr = ReceiverTraces.apply(q, c.repeat_interleave(d.Np), P["comp"], P["receivers"],
                                  P["dt"], nsteps, P["source"], every)
        return trace_loss(tr)

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with torch.no_grad():
        L0 = float(loss(q0.detach(), ck.detach()))
    torch.cuda.synchronize()
    t_fwd = time.perf_counter() - t0
    t0 = time.perf_counter()
    L = loss(q0, ck)
    L.backward()
    torch.cuda.synchronize()
    t_fb = time.perf_counter() - t0
    gq, gc = q0.grad.detach(), ck.grad.detach()
    errs = {"q0": [], "c": []}
    with torch.no_grad():
        for k in range(ndirs):
            # half of the directions move the initial field, half the c_k
            if k % 2 == 0:
                dq = torch.as_tensor(rng.standard_normal(q0.shape), device=d.device)
                dc = torch.zeros_like(ck)
            else:
                dq = torch.zeros_like(q0)
                dc = torch.as_tensor(rng.standard_normal(ck.shape), device=d.device)
            lp = float(loss(q0 + h * dq, ck + h * dc))
            lm = float(loss(q0 - h * dq, ck - h * dc))
            fd = (lp - lm) / (2 * h)
            an = float((gq * dq).sum() + (gc * dc).sum())
            errs["q0" if k % 2 == 0 else "c"].append(abs(fd - an) / max(abs(an), 1e-300))
    allerr = errs["q0"] + errs["c"]
    worst = lambda v: max(v) if v else None  # noqa: E731  (fewer than two directions)
    return {"loss": L0, "fd_rel_err_max": worst(allerr),
            "fd_rel_err_median": float(np.median(allerr)) if allerr else None,
            "fd_rel_err_max_q0": worst(errs["q0"]), "fd_rel_err_max_c": worst(errs["c"]),
            "directions": ndirs, "h": h, "t_forward_s": t_fwd, "t_forward_backward_s": t_fb,
            "grad_c_norm": float(gc.norm()), "grad_q0_norm": float(gq.norm())}


def main(argv=None):
    """Adjoint workload: K = 7200 triangles, order 5, var-c wave, 400 LSRK4
    steps, checkpoints every 20, 32 central-difference directions (h = 1e-6).
    Prints one JSON line."""
    import argparse
    import json
    p = argparse.ArgumentParser()
    p.add_argument("--n", type=int, default=61)
    p.add_argument("--order", type=int, default=5)
    p.add_argument("--steps", type=int, default=400)
    p.add_argument("--every", type=int, default=20)
    p.add_argument("--dirs", type=int, default=32)
    a = p.parse_args(argv)
    P = make_wave_inversion_problem(n=a.n, order=a.order)
    torch = _torch()
    x = P["discr"].nodes
    # initial pressure pulse (width 0.2) beside the source
    q0 = np.stack([np.exp(-((x - 0.3) ** 2).sum(1) / 0.2 ** 2), 0 * x[:, 0], 0 * x[:, 0]])
    q0 = torch.as_tensor(q0, device=P["discr"].device)
    r = check_gradients(P, nsteps=a.steps, every=a.every, ndirs=a.dirs, q0=q0)
    d = P["discr"]
    r.update({"workload": "varwave2d_K%d_N%d_steps%d" % (d.K, a.order, a.steps),
              "K": d.K, "order": a.order, "checkpoint_every": a.every, "dtype": "f64",
              "dof_updates_forward_per_s": d.K * d.Np * 3 * 5 * a.steps / r["t_forward_s"]})
    print(json.dumps(r), flush=True)


if __name__ == "__main__":
    main()
