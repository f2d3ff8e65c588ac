"""Low-storage RK4 (Carpenter-Kennedy 5-stage, 2N storage).

Restates hedge/timestep/runge_kutta.py:34-131.  When ``rhs`` is a bound
operator of this backend, each stage is one fused device launch
(hb_lsrk_stage: RHS + residual update + state update); otherwise the stepper
calls ``rhs`` and combines on the device with hb_lincomb, as the reference's
linear combiner does (hedge/vector_primitives.py:58-77).
"""

from __future__ import annotations

import numpy as np

from . import _native

RK4A = [0.0,
        -567301805773 / 1357537059087,
        -2404267990393 / 2016746695238,
        -3550918686646 / 2091501179385,
        -1275806237668 / 842570457699]
RK4B = [1432997174477 / 9575080441755,
        5161836677717 / 13612068292357,
        1720146321549 / 2090206949498,
        3134564353537 / 4481467310338,
        2277821191437 / 14882151754819]
RK4C = [0.0,
        1432997174477 / 9575080441755,
        2526269341429 / 6820363962896,
        2006345519317 / 3224310063776,
        2802321613138 / 2924317926251]


class LSRK4TimeStepper:
    dt_fudge_factor = 1
    adaptive = False

    def __init__(self, dtype=np.float64, rcon=None, vector_primitive_factory=None):
        self.dtype = np.dtype(dtype)
        self.coeffs = np.array([RK4A, RK4B, RK4C], dtype=np.float64).T
        self.residual = None

    def __call__(self, y, t, dt, rhs):
        from .discretization import BoundRHS
        import torch
        if isinstance(rhs, BoundRHS):
            comp = rhs.compiled
            y = comp.as_state(y)
            if self.residual is None or self.residual.shape != y.shape:
                self.residual = torch.zeros_like(y)
            # ping-pong between two fresh buffers; the caller's y is not
            # written (the reference also returns a new state each step)
            bufs = [torch.empty_like(y), torch.empty_like(y)]
            cur = y
            for s, (a, b, c) in enumerate(self.coeffs):
                nxt = bufs[s % 2]
                comp.lsrk_stage(a, b, dt, cur, nxt, self.residual,
                                **rhs.context(t + c * dt))
                cur = nxt
            return cur
        lib = _native.load()
        if not isinstance(y, torch.Tensor):
            raise TypeError("state must be a CUDA tensor")
        for a, b, c in self.coeffs:
            this_rhs = rhs(t + c * dt, y)
            if self.residual is None:
                self.residual = torch.zeros_like(this_rhs)
            dtc = 0 if this_rhs.dtype == torch.float64 else 1
            stream = torch.cuda.current_stream(y.device).cuda_stream
            new_res = torch.empty_like(this_rhs)
            _native.check(lib.hb_lincomb(this_rhs.numel(), dtc, float(a),
                                         self.residual.data_ptr(), float(dt),
                                         this_rhs.data_ptr(), new_res.data_ptr(), stream))
            self.residual = new_res
            y_new = torch.empty_like(y)
            _native.check(lib.hb_lincomb(y.numel(), dtc, 1.0, y.data_ptr(), float(b),
                                         self.residual.data_ptr(), y_new.data_ptr(),
                                         stream))
            y = y_new
        return y


RK4TimeStepper = LSRK4TimeStepper


class GraphedLSRK4:
    """LSRK4 steps of a bound operator with a fixed time step, each step's 5
    fused stage launches recorded once as a CUDA graph on fixed device
    buffers and replayed: for small meshes, where launching the stages from
    Python costs more than running them.  The operator must not need data
    computed on the host per stage (a time-dependent inflow boundary), since
    a replay repeats the recorded launches as they are.

    ``g = GraphedLSRK4(rhs, y0, dt)``; ``y = g.step()`` advances the state by
    one step and returns the state buffer (overwritten by the next step);
    ``g.state`` is the same buffer.  Same kernels, same order and the same
    residual as ``LSRK4TimeStepper``, so the states agree bitwise.

    The recorded launches read the operator's coefficient field and source
    vector at their addresses at construction; this object keeps those two
    tensors alive, and ``step()`` raises if the operator has been given new
    ones since (``set_coefficient`` / ``set_source``): build a new
    GraphedLSRK4 then.  A replay does not read the operator's device error
    flag; ``check()`` does (it synchronises), so call it every so many steps
    to learn of bad input a kernel flagged (e.g. a halo face without halo
    data)."""

    def __init__(self, rhs, y0, dt):
        from .discretization import BoundRHS
        import torch
        if not isinstance(rhs, BoundRHS):
            raise TypeError("GraphedLSRK4 needs an operator bound to this backend")
        comp = rhs.compiled
        if comp.n_given:
            raise ValueError("the operator takes time-dependent boundary values; "
                             "use LSRK4TimeStepper")
        self.compiled = comp
        self.dt = float(dt)
        y = comp.as_state(y0)
        self.state = y.clone()
        self._tmp = [torch.empty_like(self.state), torch.empty_like(self.state)]
        self.residual = torch.zeros_like(self.state)
        # the graph holds these tensors' addresses: keep them alive here
        self._coeff, self._source = comp._coeff, comp._source
        coeffs = np.array([RK4A, RK4B], dtype=np.float64).T
        # stage s reads bufs[s] and writes bufs[s + 1] (never in place)
        bufs = [self.state, self._tmp[0], self._tmp[1], self._tmp[0], self._tmp[1],
                self.state]

        def stages():
            for s, (a, b) in enumerate(coeffs):
                comp.lsrk_stage(a, b, self.dt, bufs[s], bufs[s + 1], self.residual,
                                coeff=self._coeff, source=self._source)

        dev = self.state.device
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            stages()                   # one eager step first (lazy set-up)
        torch.cuda.current_stream(dev).wait_stream(side)
        torch.cuda.synchronize(dev)
        self.state.copy_(y)
        self.residual.zero_()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=side):
            stages()
        torch.cuda.synchronize(dev)

    def step(self):
        comp = self.compiled
        if comp._coeff is not self._coeff or comp._source is not self._source:
            raise RuntimeError("the operator's coefficient or source changed after the "
                               "step was recorded; build a new GraphedLSRK4")
        self.graph.replay()
        return self.state

    def check(self):
        """Synchronise and raise if a kernel of the replayed steps flagged bad
        input (the operator's device error flag)."""
        self.compiled.check()
