"""Benchmark: DG right-hand side + LSRK4 on the 3D Maxwell cavity workload.

Workload (one GPU): [-1,1]^3 split into 20^3 cubes x 6 tetrahedra
(K = 48000), interior vertices jittered +-0.05h (seed 1), order N = 4
(Np = 35, Nfp = 15), Maxwell with eps = mu = 1, upwind flux, PEC walls;
initial condition the (1,1,1) cavity mode plus 1e-3 uniform noise (seed 2).
A "step" is one LSRK4 time step = 5 fused RHS+stage launches.  The default
precision is the split (FP16x3 on the tensor cores, FP64 state) path; the
same run also times the plain FP64 path on the same workload and reports the
split path's relative L2 error against it after 1 RHS and after the timed
steps (the FP64 path matches the CPU oracle to 1e-12 in the tests).

  value  = DOF-updates/s with the state resident in HBM
           (DOF-update = one nodal value of one field through one RK stage)
  e2e    = the same metric through the public API with the state in pinned
           host memory: every step copies the state in, runs the step and
           copies the new state out (host<->device copies timed)

The three buffers of a stage (q_in, q_out, res: 3 x 80.6 MB in FP64) exceed
the 126 MB L2, so no flush is needed between iterations.

``--impl reference`` times the CPU oracle (a restatement of the reference jit
backend, which itself cannot be built in this image) on the host cores; each
of its steps is a bounded sample: one RK stage over the whole mesh.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# time-step factor of the split-vs-FP64 accuracy run (see run_ours)
ACC_DT_FACTOR = 0.5


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default="fp16x3",
                   choices=["fp64", "fp32", "fp32-simt", "bf16x3", "fp16x3"])
    p.add_argument("--workload", default="maxwell", choices=["maxwell", "wave7", "varadv2d"],
                   help="maxwell: 3D Maxwell N=4 cavity (default); wave7: 3D acoustic "
                        "wave N=7 Gaussian pulse (the high-order precision workload); "
                        "varadv2d: 2D variable-coefficient advection N=5 with "
                        "quadrature (the over-integration kernel; one GPU, FP64)")
    p.add_argument("--layout", default="partitioned", choices=["partitioned", "replicas"],
                   help="N > 1: partitioned = one mesh of N x the per-GPU size, "
                        "element-partitioned with a face-trace exchange every stage "
                        "(weak scaling); replicas = N independent copies")
    p.add_argument("--accuracy-steps", type=int, default=None,
                   help="steps of the split-vs-FP64 accuracy run (default steps+warmup)")
    p.add_argument("--no-compare", action="store_true",
                   help="skip the plain-FP64 comparison and the split accuracy check")
    p.add_argument("--n", type=int, default=20, help="cubes per axis")
    p.add_argument("--order", type=int, default=None, help="default 4 (maxwell), 7 (wave7)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    return p.parse_args()


WORKLOADS = {
    "maxwell": {"order": 4, "fields": 6,
                "metric": "DG RHS DOF-updates/s (3D Maxwell N=4, LSRK4)",
                "label": "maxwell3d_cavity_K%d_N%d"},
    "wave7": {"order": 7, "fields": 4,
              "metric": "DG RHS DOF-updates/s (3D acoustic wave N=7, LSRK4)",
              "label": "wave3d_pulse_K%d_N%d"},
    "varadv2d": {"order": 5, "fields": 1, "n": 400,
                 "metric": "DG RHS DOF-updates/s (2D variable-coefficient advection N=5, "
                           "quadrature degree 15, LSRK4)",
                 "label": "varadv2d_vortex_K%d_N%d"},
}


def build_problem(n, order, precision, device=None, workload="maxwell"):
    import hedge_b200 as hb
    from hedge_b200 import workloads
    mesh = workloads.box_mesh(n)
    discr = hb.Discretization(mesh, order=order, precision=precision, device=device)
    return hb, mesh, discr, workloads.operator(workload)


def initial_state(discr, workload="maxwell"):
    from hedge_b200 import workloads
    return workloads.initial_state(discr, workload)


def workload_config(args, K_total, K_rank, Np, F):
    """The workload as both arms report it (the implementation's precision
    and layout are reported beside it, in dtype and parallelism)."""
    W = WORKLOADS[args.workload]
    return {"workload": W["label"] % (K_rank, args.order), "K": K_total,
            "K_per_gpu": K_rank, "order": args.order, "Np": Np, "fields": F,
            "stepper": "LSRK4, one step = 5 RHS + stage updates",
            "l2": "working set of a stage (q_in, q_out, res) 3 x %.1f MB in FP64 > 126 MB L2, "
                  "no flush" % (K_rank * Np * F * 8 / 1e6)}


def algorithmic_bytes_per_dof_update(discr, state_bytes, F=6):
    """read q, read res, write q, write res per DOF-update, plus per-element
    geometry (d^2 metric + Nf (normal, Fscale)) and connectivity (Nf x
    (u32 neighbour, u8 face, u8 perm)) spread over Np*F DOF-updates."""
    d, nf = discr.dimensions, discr.Nfaces
    g_el = 8 * (d * d + nf * (d + 1)) + nf * 6
    return 4 * state_bytes + g_el / (discr.Np * F)


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            parts = [p.strip() for p in l.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus):
    import torch
    import torch.distributed as dist
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return rank, world, local


def max_over_ranks(x, world):
    import torch
    import torch.distributed as dist
    if world == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    import torch
    import torch.distributed as dist
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()


def load_traffic(kernel_key):
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(kernel_key)
    except (OSError, ValueError):
        return None


def cpu_baseline(discr, op, w0, dt, threads=None, F=6):
    """Oracle (CPU port of the jit backend) on a bounded sample: one LSRK
    stage over the whole mesh, all host threads (best of 3 after a warm-up),
    plus the same on one thread (the reference's generated loops are serial)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc_mod
    ncores = os.cpu_count() or 1
    orc = orc_mod.OracleRHS(discr, op.op_template())
    dofs = discr.K * discr.Np * F

    def stage_time(nthreads, reps):
        used = orc_mod.set_threads(nthreads)
        orc(w0)                     # warm-up
        best = None
        for _ in range(reps):
            t0 = time.perf_counter()
            r = orc(w0)
            res = dt * r
            _ = w0 + 0.149 * res
            el = time.perf_counter() - t0
            best = el if best is None else min(best, el)
        return used, best

    used, el = stage_time(threads or ncores, 3)
    _, el1 = stage_time(1, 1)
    orc_mod.set_threads(ncores)
    return {"value": dofs / el, "unit": "DOF-updates/s", "cores": used,
            "cpu_model": cpu_model(), "kind": "port", "single_thread_value": dofs / el1,
            "sample": "one LSRK stage (RHS + update) over the full K=%d mesh, "
                      "%d OpenMP threads, best of 3; C++ oracle -O3" % (discr.K, used)}, el


def cpu_model():
    """The host CPU's model name (Linux /proc/cpuinfo), else the platform's."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or platform.machine()


def run_reference(args):
    """The reference arm: the CPU oracle (the reference jit backend's loops,
    restated; the reference itself cannot be built here) on all host cores,
    on the same workload and metric as run_ours.  At N = 1 a step is one
    LSRK4 step (5 RHS + stage updates) over the whole mesh, as in run_ours.
    For N > 1 (a mesh N times larger) a step is a bounded sample, one LSRK
    stage over the whole mesh, so that the run ends within minutes."""
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if rank != 0:
        return
    W = WORKLOADS[args.workload]
    F = W["fields"]
    from hedge_b200 import workloads
    import hedge_b200 as hb
    stretch = world if (world > 1 and args.layout == "partitioned") else 1
    # the same mesh as our arm: world x the per-GPU workload when partitioned
    mesh = workloads.box_mesh(args.n, stretch=stretch)
    discr = hb.Discretization(mesh, order=args.order)
    op = workloads.operator(args.workload)
    w0 = initial_state(discr, args.workload)
    dt = op.estimate_timestep(discr)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc_mod
    ncores = os.cpu_count() or 1
    used = orc_mod.set_threads(ncores)
    orc = orc_mod.OracleRHS(discr, op.op_template())
    from hedge_b200.timestep import RK4A, RK4B, RK4C
    stages = 5 if stretch == 1 else 1
    y, res, t = w0.copy(), np.zeros_like(w0), 0.0

    def step(y, res, t):
        for s in range(stages):
            r = orc(y, t + RK4C[s] * dt)
            res = RK4A[s] * res + dt * r
            y = y + RK4B[s] * res
        return y, res, t + dt

    for _ in range(args.warmup):
        y, res, t = step(y, res, t)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        y, res, t = step(y, res, t)
    el = time.perf_counter() - t0
    v = discr.K * discr.Np * F * stages * args.steps / el
    K_rank = discr.K // world if stretch > 1 else discr.K
    sample = ("one LSRK4 step (5 RHS + stage updates) over the full K=%d mesh per step"
              % discr.K if stages == 5 else
              "one LSRK stage (RHS + update) over the full K=%d mesh per step" % discr.K)
    line = {
        "impl": "reference", "metric": W["metric"],
        "value": v, "unit": "DOF-updates/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": workload_config(args, discr.K, K_rank, discr.Np, F),
        "parallelism": "host cores (%d OpenMP threads)" % used,
        "cpu_baseline": {"value": v, "unit": "DOF-updates/s", "cores": used,
                         "cpu_model": cpu_model(), "kind": "port",
                         "sample": sample + "; C++ oracle (restated jit loops), OpenMP"},
        "e2e": {"value": v, "unit": "DOF-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "per_time_step": {"value": v / 5, "unit": "DOF-steps/s"},
    }
    print(json.dumps(line), flush=True)


def partitioned_problem(args, rank, world, dev):
    """One mesh of world x the per-GPU workload (the box stretched along x),
    element-partitioned across the ranks; this rank's operator exchanges its
    cut-face traces with its neighbours (NCCL point-to-point) every stage."""
    import torch
    import torch.distributed as dist
    import hedge_b200 as hb
    from hedge_b200.partition import DistExchange, PartitionPlan, PartitionedOperator
    from hedge_b200.timestep import RK4A, RK4B
    from hedge_b200 import workloads
    mesh = workloads.box_mesh(args.n, stretch=world)
    discr = hb.Discretization(mesh, order=args.order, precision=args.precision, device=dev)
    op = workloads.operator(args.workload)
    plan = PartitionPlan(discr, op.op_template(), world)
    part = PartitionedOperator(discr, op, plan, rank, precision=args.precision, device=dev,
                               exchange=DistExchange(plan, rank))
    dist.barrier()
    w0 = initial_state(discr, args.workload)
    dt = op.estimate_timestep(discr)
    res = torch.zeros((part.F, part.K * part.Np), dtype=part.dtype, device=dev)

    def stepper(y, t, dt_, rhs_):
        cur = y
        for s_ in range(5):
            nxt = torch.empty_like(cur)
            part.lsrk_stage(RK4A[s_], RK4B[s_], dt_, cur, nxt, res)
            cur = nxt
        return cur

    return hb, discr, op, part, part.scatter(w0), dt, stepper


def run_ours(args):
    import torch
    rank, world, local = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    W = WORKLOADS[args.workload]
    F = W["fields"]
    partitioned = world > 1 and args.layout == "partitioned"
    if partitioned:
        hb, discr, op, comp, y, dt, stepper = partitioned_problem(args, rank, world, dev)
        rhs = None
        w0 = y.cpu().numpy()
        K_rank, K_total = comp.K, discr.K
        args.no_compare = True
    else:
        hb, mesh, discr, op = build_problem(args.n, args.order, args.precision, device=dev,
                                            workload=args.workload)
        w0 = initial_state(discr, args.workload)
        dt = op.estimate_timestep(discr)
        rhs = op.bind(discr)
        comp = rhs.compiled
        stepper = hb.LSRK4TimeStepper()
        y = discr.to_device(w0).reshape(F, -1)
        K_rank, K_total = discr.K, discr.K * world
    # warm-up
    t = 0.0
    for _ in range(args.warmup):
        y = stepper(y, t, dt, rhs)
        t += dt
    comp.check()
    barrier(world)
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # An FP32 state's stage working set (3 x 40 MB at C2) nearly fits in the
    # 126 MB L2: those steps are timed one by one, with L2 flushed between
    # them (a 256 MB write outside the timed events).
    flush_l2 = args.precision in ("fp32", "fp32-simt")
    scratch = torch.empty(64 << 20, dtype=torch.float32, device=dev) if flush_l2 else None
    with ClockSampler(dev.index) as clk:
        barrier(world)
        if flush_l2:
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in range(args.steps)]
            for e_a, e_b in evs:
                scratch.fill_(1.0)
                e_a.record(stream)
                y = stepper(y, t, dt, rhs)
                t += dt
                e_b.record(stream)
            barrier(world)
            ms = sum(e_a.elapsed_time(e_b) for e_a, e_b in evs)
        else:
            ev0.record(stream)
            for _ in range(args.steps):
                y = stepper(y, t, dt, rhs)
                t += dt
            ev1.record(stream)
            barrier(world)
            ms = ev0.elapsed_time(ev1)
    comp.check()
    ms_max = max_over_ranks(ms, world)
    value = K_total * discr.Np * F * 5 * args.steps / (ms_max * 1e-3)
    launches = 5 * args.steps
    launch_ms = ms / launches
    state_bytes = 4 if args.precision in ("fp32", "fp32-simt") else 8
    bpd = algorithmic_bytes_per_dof_update(discr, state_bytes, F)
    bytes_per_launch = bpd * K_rank * discr.Np * F
    achieved = bytes_per_launch / (launch_ms * 1e-3) / 1e9
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs")
    peak_src = "measured" if peak else "fallback"
    peak = peak or 6650.0
    kernel_key = "rhs_stage_%s_%s_N%d" % (args.precision,
                                          "maxwell3d" if args.workload == "maxwell" else "wave3d",
                                          args.order)
    traffic = load_traffic(kernel_key)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                "algorithmic_bytes_per_dof_update": bpd,
                "kernel": kernel_key}

    # ---- the plain FP64 path on the same workload, and the split accuracy ----
    compare = None
    if not args.no_compare and args.precision != "fp64":
        d64 = hb.Discretization(mesh, order=args.order, precision="fp64", device=dev)
        rhs64 = op.bind(d64)
        y64 = d64.to_device(w0).reshape(F, -1)
        ys = discr.to_device(w0).reshape(F, -1)
        r_split = rhs(0.0, ys)
        r_64 = rhs64(0.0, y64)
        err_rhs = float(torch.linalg.norm(r_split - r_64) / torch.linalg.norm(r_64))
        st64 = hb.LSRK4TimeStepper()
        t64 = 0.0
        for _ in range(3):
            y64 = st64(y64, t64, dt, rhs64)
            t64 += dt
        barrier(world)
        n64 = max(2, args.steps // 2)
        ev0.record(stream)
        for _ in range(n64):
            y64 = st64(y64, t64, dt, rhs64)
            t64 += dt
        ev1.record(stream)
        barrier(world)
        ms64 = max_over_ranks(ev0.elapsed_time(ev1), world)
        v64 = discr.K * discr.Np * F * 5 * n64 * world / (ms64 * 1e-3)
        # same IC, same number of steps on both paths.  The accuracy run takes
        # half the CFL estimate: at the full estimate (no safety factor, as the
        # reference's) the upwind N=4 tet operator has eigenvalues outside the
        # LSRK4 stability region, and the FP64 run itself grows after ~100
        # steps; the timed steps' cost does not depend on dt.
        nacc = args.accuracy_steps or (args.steps + args.warmup)
        dt_acc = ACC_DT_FACTOR * dt
        ya, yb, ta = discr.to_device(w0).reshape(F, -1), d64.to_device(w0).reshape(F, -1), 0.0
        sa, sb = hb.LSRK4TimeStepper(), hb.LSRK4TimeStepper()
        for _ in range(nacc):
            ya = sa(ya, ta, dt_acc, rhs)
            yb = sb(yb, ta, dt_acc, rhs64)
            ta += dt_acc
        err_steps = float(torch.linalg.norm(ya - yb) / torch.linalg.norm(yb))
        growth = float(torch.linalg.norm(yb) / torch.linalg.norm(d64.to_device(w0)))
        compare = {"fp64_plain_value": v64, "unit": "DOF-updates/s",
                   "speedup_vs_fp64": value / v64,
                   "rel_l2_vs_fp64_after_1_rhs": err_rhs,
                   "rel_l2_vs_fp64_after_steps": err_steps, "accuracy_steps": nacc,
                   "accuracy_dt_factor": ACC_DT_FACTOR,
                   "fp64_norm_ratio_after_steps": growth,
                   "fp64_steps_timed": n64}

    # ---- end to end through the public API with host buffers ----
    e2e = None
    if not args.no_e2e:
        # Every step copies its input in from pinned host memory, advances it
        # one LSRK4 step and copies the result back.  The steps are independent
        # (the same host input each time), so they are pipelined: the copy in
        # of step i+1 and the copy out of step i-1 (the two PCIe directions,
        # each on its own stream) overlap the compute of step i.
        host_in = torch.from_numpy(np.ascontiguousarray(w0)).pin_memory()
        host_out = [torch.empty_like(host_in).pin_memory() for _ in range(2)]
        dev_in = [torch.empty(host_in.shape, dtype=host_in.dtype, device=dev) for _ in range(2)]
        s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
        ev = lambda: torch.cuda.Event()  # noqa: E731
        in_done, used, comp_done, out_done = ([ev(), ev()] for _ in range(4))

        def e2e_run(n):
            for i in range(n):
                b = i & 1
                with torch.cuda.stream(s_in):
                    s_in.wait_event(used[b])       # step i-2 is done with dev_in[b]
                    dev_in[b].copy_(host_in, non_blocking=True)
                    in_done[b].record(s_in)
                stream.wait_event(in_done[b])
                yd = stepper(dev_in[b], 0.0, dt, rhs)
                used[b].record(stream)
                comp_done[b].record(stream)
                with torch.cuda.stream(s_out):
                    s_out.wait_event(comp_done[b])
                    s_out.wait_event(out_done[b])  # host_out[b] of step i-2 was read
                    yd.record_stream(s_out)
                    host_out[b].copy_(yd, non_blocking=True)
                    out_done[b].record(s_out)
            stream.wait_stream(s_in)
            stream.wait_stream(s_out)

        # the same number of steps as the device-timed region: the pipeline's
        # fill (first copy in) and drain (last copy out) are amortised alike
        e2e_steps = max(1, args.steps)
        e2e_run(2)
        torch.cuda.synchronize(dev)
        barrier(world)
        ev0.record(stream)
        e2e_run(e2e_steps)
        ev1.record(stream)
        barrier(world)
        e_ms = max_over_ranks(ev0.elapsed_time(ev1), world)
        nbytes = host_in.numel() * host_in.element_size()
        e2e = {"value": K_total * discr.Np * F * 5 * e2e_steps / (e_ms * 1e-3),
               "unit": "DOF-updates/s", "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes, "steps": e2e_steps,
               "overlap": "copy in / compute / copy out of consecutive steps on three streams"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu, _ = cpu_baseline(discr, op, w0, dt, F=F)
        except Exception as exc:   # the baseline must not sink the GPU line
            cpu = {"value": None, "error": str(exc)}

    if rank == 0:
        line = {
            "metric": W["metric"],
            "value": value, "unit": "DOF-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp64": "f64", "fp32": "f32 state, fp16x3(scaled)+f32acc contractions",
                      "fp32-simt": "f32", "bf16x3": "bf16x3+f32acc, f64 state",
                      "fp16x3": "fp16x3(scaled)+f32acc, f64 state"}[args.precision],
            "data": "synthetic",
            "config": workload_config(args, K_total, K_rank, discr.Np, F),
            "precision": args.precision,
            "l2_flush": ("256 MB write before each timed step (FP32 state)" if flush_l2
                         else "none: working set > L2"),
            "parallelism": ("partitioned, face-trace exchange per stage (NCCL)"
                            if partitioned else "replicas" if world > 1 else "single GPU"),
            # the same rate per LSRK4 time step (5 stages): DOF-steps/s
            "per_time_step": {"value": value / 5, "unit": "DOF-steps/s"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "split_vs_fp64": compare,
            "gpu_launches": launches * (2 if partitioned else 1), "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def varadv_flops_per_element(discr, nq, nqf):
    """FP64 operations of the quadrature kernel per element (2 per FMA):
    u and v at the volume points, the chain rule and product with u, the
    projection, both traces at the face points and the lift (the flux
    arithmetic itself, ~10 per face point, is left out)."""
    d, np_, nfp, nf = discr.dimensions, discr.Np, discr.Nfp, discr.Nfaces
    nv = 1 + d
    fma = (nv * np_ * nq + nq * d * (d + 1) + d * nq * np_
           + nf * nqf * nfp * 2 * nv + nf * nqf * np_)
    return 2 * fma


def fp64_peak_tflops(dev):
    """cuBLAS DGEMM 8192^3 (the FP64 pipes' throughput), best of 5."""
    import torch
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    b = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    c = a @ b
    best = None
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        c = a @ b
        e1.record()
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del a, b, c
    return 2 * 8192 ** 3 / (best * 1e-3) / 1e12


def run_varadv(args):
    """The quadrature kernel on the 2D variable-coefficient advection
    workload (hedge_b200.workloads.varadv_problem), one GPU, FP64.  A step
    is one LSRK4 step (5 fused RHS + stage launches).  The kernel is bound by
    FP64 arithmetic (about 800 operations per DOF-update at N = 5), so the
    roofline is against cuBLAS DGEMM measured in the same run; the HBM
    fraction of the algorithmic bytes is reported beside it."""
    import torch
    import hedge_b200 as hb
    from hedge_b200 import workloads
    if args.gpus != 1:
        raise SystemExit("varadv2d: one GPU")
    dev = torch.device("cuda", torch.cuda.current_device())
    n = args.n if args.n != 20 else WORKLOADS["varadv2d"]["n"]
    d, op, u0 = workloads.varadv_problem(n, args.order, device=dev)
    rhs = op.bind(d)
    comp = rhs.compiled
    dt = 0.5 * op.estimate_timestep(d, t=0.0)
    stepper = hb.LSRK4TimeStepper()
    y = d.to_device(u0).reshape(1, -1)
    t = 0.0
    for _ in range(args.warmup):
        y = stepper(y, t, dt, rhs)
        t += dt
    comp.check()
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clk:
        torch.cuda.synchronize(dev)
        ev0.record(stream)
        for _ in range(args.steps):
            y = stepper(y, t, dt, rhs)
            t += dt
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        ms = ev0.elapsed_time(ev1)
    comp.check()
    dofs = d.K * d.Np
    value = dofs * 5 * args.steps / (ms * 1e-3)
    launches = 5 * args.steps
    launch_s = ms * 1e-3 / launches
    vi, vp, fi, fl = d.quadrature_matrices("quad", 3 * d.order - 1)
    nq, nqf = vi.shape[0], fi.shape[1]
    flops = varadv_flops_per_element(d, nq, nqf) * d.K
    g_el = 8 * (4 + 3 * 3) + 3 * 6
    bpd = 4 * 8 + 2 * 8 + g_el / d.Np     # q in/out, res r/w, velocity; geometry
    peak64 = fp64_peak_tflops(dev)
    hbm = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs", 6650.0)
    achieved = flops / launch_s / 1e12
    gbs = bpd * dofs / launch_s / 1e9
    roofline = {"bound": "fp64", "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                "frac": achieved / peak64,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
                "flops_per_element": flops / d.K, "volume_points": nq, "face_points": nqf,
                "hbm": {"achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                        "algorithmic_bytes_per_dof_update": bpd},
                "traffic": load_traffic("rhs_quad_varadv2d_N%d" % d.order),
                "kernel": "rhs_quad_kernel<2, double>"}
    # end to end: the state copied in from pinned host memory and out again
    # around every step (same stream, not overlapped)
    e2e = None
    if not args.no_e2e:
        host_in = torch.from_numpy(np.ascontiguousarray(u0.reshape(1, -1))).pin_memory()
        host_out = torch.empty_like(host_in).pin_memory()
        dev_in = torch.empty(host_in.shape, dtype=torch.float64, device=dev)
        for _ in range(2):
            dev_in.copy_(host_in, non_blocking=True)
            host_out.copy_(stepper(dev_in, 0.0, dt, rhs), non_blocking=True)
        torch.cuda.synchronize(dev)
        ev0.record(stream)
        for _ in range(args.steps):
            dev_in.copy_(host_in, non_blocking=True)
            host_out.copy_(stepper(dev_in, 0.0, dt, rhs), non_blocking=True)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        e_ms = ev0.elapsed_time(ev1)
        nbytes = host_in.numel() * 8
        e2e = {"value": dofs * 5 * args.steps / (e_ms * 1e-3), "unit": "DOF-updates/s",
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes}
    cpu = None
    if not args.no_cpu_baseline:
        cpu = varadv_cpu_baseline(args.order)
    line = {"metric": WORKLOADS["varadv2d"]["metric"], "value": value,
            "unit": "DOF-updates/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": varadv_config(d.K, d.order, d.Np),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches, "clocks": clk.summary(),
            "launch_config": comp.launch_info()}
    print(json.dumps(line), flush=True)


def varadv_cpu_baseline(order):
    """The template executor (oracle/optemplate_exec.py: the reference's
    quadrature integrals evaluated with numpy) on a bounded sample: one RHS
    of the same operator on a 24 x 24 mesh, best of 2, one thread of numpy."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from optemplate_exec import TemplateExecutor
    from hedge_b200 import workloads
    from hedge_b200.mesh import TAG_ALL
    d, op, u0 = workloads.varadv_problem(24, order)
    ex = TemplateExecutor(d)
    tpl = op.op_template()
    env = {"u": u0, "v": op.advec_v.f(d.nodes),
           "bc_u": op.bc_u_f.boundary_interpolant(0.0, d, TAG_ALL)}
    ex(tpl, **env)
    best = None
    for _ in range(2):
        t0 = time.perf_counter()
        ex(tpl, **env)
        el = time.perf_counter() - t0
        best = el if best is None else min(best, el)
    return {"value": d.K * d.Np / best, "unit": "DOF-updates/s", "cores": 1, "kind": "port",
            "sample": "one RHS of the operator on a K=%d mesh (24 x 24 squares), template "
                      "executor (numpy), best of 2" % d.K}


def varadv_config(K, order, Np):
    """The quadrature workload's config as both arms report it."""
    return {"workload": WORKLOADS["varadv2d"]["label"] % (K, order), "K": K, "order": order,
            "Np": Np, "quad_degree": 3 * order,
            "l2": "working set of a stage (q_in, q_out, res, v) 5 x %.1f MB > 126 "
                  "MB L2, no flush" % (K * Np * 8 / 1e6)}


def run_varadv_reference(args):
    """The reference arm of the quadrature workload: the template executor
    (oracle/optemplate_exec.py, the reference's quadrature integrals with
    numpy; no other CPU implementation of this operator exists here) on a
    bounded sample, one RHS of the same operator on a 24 x 24 mesh per step,
    on rank 0 only."""
    if int(os.environ.get("RANK", 0)) != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from optemplate_exec import TemplateExecutor
    from hedge_b200 import workloads
    from hedge_b200.mesh import TAG_ALL, make_regular_rect_mesh
    n = args.n if args.n != 20 else WORKLOADS["varadv2d"]["n"]
    K_full = len(make_regular_rect_mesh((-1, -1), (1, 1), (n, n)).elements)
    d, op, u0 = workloads.varadv_problem(24, args.order)
    ex = TemplateExecutor(d)
    tpl = op.op_template()
    env = {"u": u0, "v": op.advec_v.f(d.nodes),
           "bc_u": op.bc_u_f.boundary_interpolant(0.0, d, TAG_ALL)}
    for _ in range(args.warmup):
        ex(tpl, **env)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ex(tpl, **env)
    el = time.perf_counter() - t0
    v = d.K * d.Np * args.steps / el
    sample = ("one RHS of the operator on a K=%d mesh (24 x 24 squares) per step, template "
              "executor (numpy, the reference's quadrature integrals), one thread" % d.K)
    line = {"impl": "reference", "metric": WORKLOADS["varadv2d"]["metric"], "value": v,
            "unit": "DOF-updates/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * el / max(args.steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": varadv_config(K_full, args.order, d.Np),
            "cpu_baseline": {"value": v, "unit": "DOF-updates/s", "cores": 1,
                             "cpu_model": cpu_model(), "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "DOF-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.order is None:
        args.order = WORKLOADS[args.workload]["order"]
    if args.workload == "varadv2d":
        if args.impl == "reference":
            run_varadv_reference(args)
            return
        run_varadv(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
