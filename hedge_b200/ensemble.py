"""Batched ensembles: many independent discretizations advanced together.

``Ensemble`` owns, per member, two FP32 state buffers and an FP64 residual
and advances every member by one LSRK4 step (hedge/timestep/
runge_kutta.py:104-131) with five launches of the batched kernel
(hb_batch_stage), one per stage.  ``capture()`` records a step as a CUDA
graph; since a step's five stages flip the state buffers an odd number of
times, two graphs are kept (the step starting from buffer 0 or buffer 1).

``autotune`` picks the tile size (elements per tile) for each (order, field
count) by timing the candidates on the ensemble itself; ``make_c5_members``
builds the ensemble workload (256 2D advection / wave members of K
log-uniform in [500, 20000], orders 3..6).
"""

from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _native
from .timestep import RK4A, RK4B


def _torch():
    import torch
    return torch


class Member:
    """One ensemble member: discretization, FP32 compiled operator, initial
    state (numpy [F, K*Np]) and time step."""

    def __init__(self, discr, model, q0, dt=None):
        self.discr = discr
        self.model = model
        self.comp = discr.compile(model.op_template(), precision="fp32")
        self.F = self.comp.F
        self.q0 = np.asarray(q0, dtype=np.float64).reshape(self.F, len(discr))
        self.dt = float(model.estimate_timestep(discr) if dt is None else dt)

    @property
    def key(self):
        return (self.discr.order, self.F, self.discr.dimensions)


# (order, F, dim) -> elements per tile, filled by autotune()
TILE_TABLE: dict = {}


class Ensemble:
    def __init__(self, members, tiles=None):
        torch = _torch()
        self.members = members
        self.lib = _native.load()
        tiles = TILE_TABLE if tiles is None else tiles
        self.q = []
        self.res = []
        arr = (_native.hb_batch_member * len(members))()
        for k, m in enumerate(members):
            dev = m.discr.device
            q0 = torch.as_tensor(m.q0, dtype=torch.float32, device=dev).contiguous()
            q1 = torch.empty_like(q0)
            r = torch.zeros(q0.shape, dtype=torch.float64, device=dev)
            self.q.append([q0, q1])
            self.res.append(r)
            arr[k] = _native.hb_batch_member(m.comp._handle, q0.data_ptr(), q1.data_ptr(),
                                             r.data_ptr(), m.dt, int(tiles.get(m.key, 0)))
        self._members_c = arr
        h = C.c_void_p()
        _native.check(self.lib.hb_batch_create(C.cast(arr, C.c_void_p), len(members),
                                               C.byref(h)))
        self._h = h
        self.parity = 0          # buffer that holds the current state
        self.graphs = None
        self.device = members[0].discr.device

    def __del__(self):
        try:
            if getattr(self, "_h", None) is not None:
                self.graphs = None
                self.lib.hb_batch_destroy(self._h)
                self._h = None
        except Exception:
            pass

    def info(self):
        v = (C.c_int64 * 5)()
        _native.check(self.lib.hb_batch_info(self._h, v, 5))
        return dict(zip(["tiles", "grid", "threads", "smem", "dofs"], list(v)))

    def _stream(self):
        return _torch().cuda.current_stream(self.device).cuda_stream

    def _step_from(self, parity):
        p = parity
        for s in range(5):
            _native.check(self.lib.hb_batch_stage(self._h, float(RK4A[s]), float(RK4B[s]),
                                                  p, self._stream()))
            p ^= 1

    def step(self, nsteps=1):
        """Advance every member by nsteps LSRK4 steps (eager launches, or the
        captured graphs after capture())."""
        for _ in range(nsteps):
            if self.graphs is not None:
                self.graphs[self.parity].replay()
            else:
                self._step_from(self.parity)
            self.parity ^= 1

    def capture(self):
        """Record one step from each buffer parity as a CUDA graph."""
        torch = _torch()
        torch.cuda.synchronize(self.device)
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        graphs = []
        with torch.cuda.stream(s):
            for p in (0, 1):
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=s):
                    self._step_from(p)
                graphs.append(g)
        torch.cuda.current_stream(self.device).wait_stream(s)
        self.graphs = graphs

    def check(self):
        _native.check(self.lib.hb_batch_check(self._h, self._stream()))

    def state(self, k):
        """Member k's current state [F, K*Np] (FP32)."""
        return self.q[k][self.parity]

    def dof_updates_per_step(self):
        return 5 * sum(m.discr.K * m.discr.Np * m.F for m in self.members)

    def algorithmic_bytes_per_step(self):
        """Per stage and DOF: FP32 state read + write (8 B), FP64 residual
        read + write (16 B); per element: FP32 geometry and the face table."""
        tot = 0
        for m in self.members:
            d = m.discr
            dim, nf = d.dimensions, d.Nfaces
            g_el = 4 * (dim * dim + nf * (dim + 1)) + 8 * nf
            tot += d.K * d.Np * m.F * 24 + d.K * g_el
        return 5 * tot


def _rect_member(K, order, model_kind, rng, device=None):
    """A 2D member of about K jittered triangles on [-1,1]^2."""
    import hedge_b200 as hb
    n = max(2, int(round(np.sqrt(K / 2.0)))) + 1
    h = 2.0 / (n - 1)
    seed = int(rng.integers(1 << 30))
    if model_kind == "advection":
        mesh = hb.make_regular_rect_mesh((-1, -1), (1, 1), (n, n), periodicity=(True, True),
                                         jitter=0.1 * h, seed=seed)
        ang = rng.uniform(0, 2 * np.pi)
        v = rng.uniform(0.5, 1.5) * np.array([np.cos(ang), np.sin(ang)])
        model = hb.StrongAdvectionOperator(v, flux_type="upwind")
    else:
        mesh = hb.make_regular_rect_mesh((-1, -1), (1, 1), (n, n), jitter=0.1 * h, seed=seed)
        model = hb.StrongWaveOperator(rng.uniform(0.5, 1.5), 2, flux_type="upwind")
    discr = hb.Discretization(mesh, order=order, device=device)
    x = discr.nodes
    c = rng.uniform(-0.5, 0.5, 2)
    w = rng.uniform(0.1, 0.3)
    g = np.exp(-((x - c) ** 2).sum(1) / w ** 2)
    F = 1 if model_kind == "advection" else 3
    q0 = np.zeros((F, len(discr)))
    q0[0] = g
    return Member(discr, model, q0)


def make_c5_members(n=256, seed=6, ic_seed=7, kmin=500, kmax=20000, orders=(3, 4, 5, 6),
                    device=None):
    """The ensemble workload: n 2D members, K log-uniform in [kmin, kmax],
    order uniform in `orders`, advection (periodic, random velocity) or wave
    (reflecting walls, random speed), random Gaussian initial pulses."""
    rng = np.random.default_rng(seed)
    ks = np.exp(rng.uniform(np.log(kmin), np.log(kmax), n))
    ords = rng.choice(orders, n)
    kinds = rng.choice(["advection", "wave"], n)
    ic = np.random.default_rng(ic_seed)
    return [_rect_member(int(k), int(o), str(m), ic, device) for k, o, m in zip(ks, ords, kinds)]


def autotune(members, budgets=(128, 256, 512, 1024), steps=5, passes=1, table=None):
    """Tile size (elements per tile) per (order, F, dim) for this ensemble:
    coordinate descent over the keys present, each candidate (budget // Np
    elements, budget = nodes per tile) timed by `steps` LSRK4 steps of the
    whole ensemble with CUDA events, the other keys held at their current
    best.  Fills and returns `table` (default: the module's TILE_TABLE) and
    the timings {key: {elements: ms per step}}."""
    torch = _torch()
    table = TILE_TABLE if table is None else table
    keys = sorted({m.key for m in members})
    np_of = {m.key: m.discr.Np for m in members}
    cur = {k: table.get(k, max(1, 256 // np_of[k])) for k in keys}
    timings = {}

    def measure(tiles):
        ens = Ensemble(members, tiles=tiles)
        ens.step(1)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ens.step(steps)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    for _ in range(passes):
        for k in keys:
            res = {}
            for b in budgets:
                E = max(1, b // np_of[k])
                if E in res:
                    continue
                trial = dict(cur)
                trial[k] = E
                res[E] = measure(trial)
            cur[k] = min(res, key=res.get)
            timings[k] = res
    table.update(cur)
    return table, timings


def main(argv=None):
    """Ensemble workload: 256 members, 100 steps captured as CUDA graphs.
    Prints one JSON line (DOF-updates/s, achieved HBM GB/s against the
    measured peak, eager vs graph)."""
    import argparse
    import json
    import os
    torch = _torch()
    p = argparse.ArgumentParser()
    p.add_argument("--members", type=int, default=256)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--no-autotune", action="store_true")
    a = p.parse_args(argv)
    members = make_c5_members(a.members)
    t0 = time.perf_counter()
    tuned = None
    if not a.no_autotune:
        _, tuned = autotune(members)
    t_tune = time.perf_counter() - t0
    ens = Ensemble(members)
    info = ens.info()
    ens.step(3)
    ens.check()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record()
    ens.step(10)
    ev1.record()
    torch.cuda.synchronize()
    eager_ms = ev0.elapsed_time(ev1) / 10
    ens.capture()
    ens.step(3)
    torch.cuda.synchronize()
    ev0.record()
    ens.step(a.steps)
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / a.steps
    ens.check()
    peak = None
    try:
        with open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                               "MEASURED_PEAKS.json")) as f:
            peak = json.load(f).get("hbm_gbs")
    except (OSError, ValueError):
        pass
    peak_source = "measured" if peak else "fallback"
    peak = peak or 6650.0      # earlier STREAM-copy measurement on B200, GB/s
    gbs = ens.algorithmic_bytes_per_step() / (ms * 1e-3) / 1e9
    out = {"workload": "ensemble2d_%d_members" % a.members, "members": a.members,
           "dofs": info["dofs"], "steps": a.steps, "ms_per_step": ms,
           "dof_updates_per_s": ens.dof_updates_per_step() / (ms * 1e-3),
           "eager_ms_per_step": eager_ms, "achieved_gbs": gbs,
           "peak_gbs": peak, "peak_source": peak_source, "frac": gbs / peak,
           "launch": info, "tiles": {"%d,%d,%d" % k: v for k, v in TILE_TABLE.items()},
           "autotune_s": t_tune,
           "autotune_ms": {"%d,%d,%d" % k: v for k, v in (tuned or {}).items()}}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
