"""Element partitions and the face-trace exchange (host side, no GPU).

* every element has one owner and the parts are contiguous along the Morton
  order; local face tables reproduce the global neighbours; a part's
  elements without halo faces come first;
* the halo a part receives (the owners' packed values, concatenated by
  source part) equals the ext values the global face-pair map gives for its
  cut faces, node by node in the receiver's face-node order;
* the same exchange through torch.distributed point-to-point on gloo,
  world size 2 and 3 (one process per part)."""
import os

import numpy as np
import pytest

import hedge_b200 as hb
from hedge_b200.partition import PartitionPlan, partition_elements


def _discr(dim=2, order=3):
    if dim == 2:
        m = hb.make_regular_rect_mesh((-1, -1), (1, 1), (7, 7), periodicity=(True, True),
                                      jitter=0.02, seed=1)
        return hb.Discretization(m, order=order), hb.StrongAdvectionOperator(
            np.array([1.0, 0.5]), flux_type="upwind")
    m = hb.make_box_tet_mesh(n=(2, 2, 2), jitter=0.02, seed=2)
    return hb.Discretization(m, order=order), hb.MaxwellOperator(1.0, 1.0, flux_type=1)


def _expected_halo(d, q, part):
    return q[:, part.halo_global].T


def _packed(plan, q, s, r):
    ps = plan.parts[s]
    nodes = (ps.elements[:, None] * (q.shape[1] // len(plan.owner)) +
             np.arange(q.shape[1] // len(plan.owner))).reshape(-1)
    ql = q[:, nodes]
    return ql[:, ps.send_idx[r]].T


@pytest.mark.parametrize("dim,nparts", [(2, 2), (2, 5), (3, 3)])
def test_plan_consistent(dim, nparts):
    d, op = _discr(dim)
    plan = PartitionPlan(d, op.op_template(), nparts)
    owner = plan.owner
    assert sorted(np.concatenate([p.elements for p in plan.parts]).tolist()) == list(range(d.K))
    from hedge_b200.discretization import build_face_table
    gconn, _, _ = build_face_table(d, op.op_template())
    rng = np.random.default_rng(0)
    F = op.descriptor().n_fields
    q = rng.standard_normal((F, len(d)))
    for r, p in enumerate(plan.parts):
        Kr = len(p.elements)
        for i, e in enumerate(p.elements):
            for f in range(d.Nfaces):
                nb, code = p.conn[i, f]
                gnb, gcode = gconn[e, f]
                assert code == gcode
                if gnb < 0:
                    assert nb == gnb
                elif owner[gnb] == r:
                    assert p.elements[nb] == gnb
                else:
                    assert Kr <= nb < Kr + p.n_halo_faces
        # halo assembled from the owners' packed values
        got = np.concatenate([_packed(plan, q, s, r) for s in sorted(p.recv_nodes)]) \
            if p.recv_nodes else np.zeros((0, F))
        np.testing.assert_array_equal(got, _expected_halo(d, q, p))


def test_halo_matches_global_gather():
    """The halo values equal q at the ext node the global face map gives."""
    d, op = _discr(2)
    plan = PartitionPlan(d, op.op_template(), 3)
    ld = d.ldis
    fmask, sh = np.asarray(ld.fmask), np.asarray(ld.face_shuffle_table)
    for r, p in enumerate(plan.parts):
        Kr = len(p.elements)
        for i, e in enumerate(p.elements):
            for f in range(d.Nfaces):
                nb, code = p.conn[i, f]
                if nb >= Kr:
                    h = nb - Kr
                    gnb = d.nbr[e, f]
                    c = d.nbr_code[e, f]
                    want = gnb * d.Np + fmask[c & 3][sh[c >> 2]]
                    np.testing.assert_array_equal(p.halo_global[h * d.Nfp:(h + 1) * d.Nfp], want)


@pytest.mark.parametrize("dim,nparts", [(2, 3), (3, 4)])
def test_interior_elements_first(dim, nparts):
    """A part lists its elements without halo faces first (the range the
    overlapped stage launches while the traces are exchanged): none of the
    first n_interior elements has a halo face, every later one has."""
    d, op = _discr(dim)
    plan = PartitionPlan(d, op.op_template(), nparts)
    for p in plan.parts:
        Kr = len(p.elements)
        halo_el = (p.conn[..., 0] >= Kr).any(1)
        assert not halo_el[:p.n_interior].any()
        assert halo_el[p.n_interior:].all()
        assert 0 < p.n_interior < Kr
        for grp in (p.elements[:p.n_interior], p.elements[p.n_interior:]):
            assert np.all(np.diff(grp) > 0)


def test_partition_is_balanced():
    d, _ = _discr(2)
    owner = partition_elements(d, 4)
    counts = np.bincount(owner, minlength=4)
    assert counts.max() - counts.min() <= 1


def _gloo_worker(rank, world, port, result_path):
    """One gloo rank: face-trace exchange and the rank sum of norms."""
    import torch
    import torch.distributed as dist
    from hedge_b200.partition import DistExchange
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        d, op = _discr(2)
        plan = PartitionPlan(d, op.op_template(), world)
        p = plan.parts[rank]
        F = op.descriptor().n_fields
        q = np.random.default_rng(7).standard_normal((F, len(d)))
        nodes = (p.elements[:, None] * d.Np + np.arange(d.Np)).reshape(-1)
        ql = q[:, nodes]
        send = torch.as_tensor(np.concatenate([ql[:, p.send_idx[x]].T
                                               for x in sorted(p.send_idx)]))
        halo = torch.zeros((p.n_halo_faces * d.Nfp, F), dtype=torch.float64)
        DistExchange(plan, rank)(send, halo)
        ok = np.array_equal(halo.numpy(), q[:, p.halo_global].T)
        # the norm reduction: every rank's share summed over the ranks
        from hedge_b200.partition import sum_over_ranks
        ok = ok and sum_over_ranks(float(rank + 1)) == world * (world + 1) / 2
        with open("%s.%d" % (result_path, rank), "w") as fh:
            fh.write("ok" if ok else "mismatch")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_gloo(tmp_path, world):
    import socket
    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    res = str(tmp_path / "res")
    mp.start_processes(_gloo_worker, args=(world, port, res), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        assert open("%s.%d" % (res, r)).read() == "ok"


def test_overlapped_stage_order():
    """With an exchange that can be started and finished separately, a part's
    stage packs, posts the exchange, launches the elements without halo
    faces, waits for the exchange, then launches the rest; without one (or
    after a LocalExchange) it launches all elements at once."""
    import types
    from hedge_b200.partition import PartitionedOperator
    log = []

    class Ex:
        def start(self, send, halo):
            log.append("start")
            return ["req"]

        def finish(self, reqs):
            log.append("finish")

    stub = types.SimpleNamespace(
        pack=lambda q: log.append("pack"), exchange=Ex(), send=np.zeros((4, 1)), n_send=3,
        halo=None, n_interior=7, K=10, _exchange=lambda q: log.append("exchange"))
    launch = lambda e0, e1: log.append((e0, e1))  # noqa: E731
    PartitionedOperator._run(stub, launch, None, exchanged=False, by_ranges=False)
    assert log == ["pack", "start", (0, 7), "finish", (7, 10)]
    log.clear()
    PartitionedOperator._run(stub, launch, None, exchanged=True, by_ranges=False)
    assert log == [(0, 10)]
    log.clear()
    PartitionedOperator._run(stub, launch, None, exchanged=True, by_ranges=True)
    assert log == [(0, 7), (7, 10)]
    log.clear()
    stub.exchange = lambda send, halo: log.append("blocking")
    PartitionedOperator._run(stub, launch, None, exchanged=False, by_ranges=False)
    assert log == ["exchange", (0, 10)]


def test_incident_walls_partition():
    """A Maxwell operator with incident walls partitions with its incident
    faces kept as boundary faces of that kind; incident data given per call
    (a given boundary vector) is refused, like every given boundary data."""
    from hedge_b200 import optemplate as ot
    from hedge_b200.models import BC_INCIDENT

    def tagger(fvi, el, fn, allv):
        return ["inc"] if allv[list(fvi)].mean(0)[0] > 0.99 else ["pec"]
    d = hb.Discretization(hb.make_box_tet_mesh(n=(2, 2, 2), jitter=0.03, seed=2,
                                               boundary_tagger=tagger), order=2)
    op = hb.MaxwellOperator(1.0, 1.0, flux_type=0.5, pec_tag="pec", incident_tag="inc")
    plan = PartitionPlan(d, op.op_template(), 3)
    n_inc = sum(int(np.count_nonzero((p.conn[..., 0] < 0) & (p.conn[..., 1] == BC_INCIDENT)))
                for p in plan.parts)
    assert n_inc == len(d.mesh.boundary_faces("inc")) > 0
    data = hb.MaxwellOperator(1.0, 1.0, flux_type=0.5, pec_tag="pec", incident_tag="inc",
                              incident_bc=lambda o, e, h: ot.make_sym_vector("inc", 6))
    with pytest.raises(NotImplementedError):
        PartitionPlan(d, data.op_template(), 3)
