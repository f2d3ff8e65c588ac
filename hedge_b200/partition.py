"""Element partitions of a discretization and the per-stage exchange of face
traces between them.

The reference partitions the mesh across MPI ranks (hedge/partition.py:
71-204, hedge/backends/mpi/__init__.py:82-118) and, once per right-hand
side, sends each rank's traces on the cut faces to the neighbouring rank
(hedge/backends/mpi/__init__.py:184-216, 284-340).  Here:

* ``partition_elements`` orders the elements along a Morton (Z-order) curve
  of their centroids and cuts it into equal contiguous pieces;
* ``PartitionPlan`` (host only, no device needed) builds, for every part,
  its local face table in which a face whose neighbour is owned by another
  part points to a halo slot (neighbour K_local + h), the number of halo
  nodes received from each other part, and the list of local volume nodes
  each part sends to each other part -- already in the receiver's face-node
  order, so the receiver reads its halo row h*Nfp + k for face node k;
* ``PartitionedOperator`` is one part's device operator: hb_pack gathers
  the values to send, an exchange object moves them into the halo buffer
  (``DistExchange``: torch.distributed point-to-point, NCCL between GPUs or
  gloo on CPU tensors; ``LocalExchange``: all parts in one process), and the
  right-hand side / LSRK stage kernels read the halo faces from it
  (hb_op_set_halo).  A part numbers its elements without halo faces first:
  with a ``DistExchange`` a stage packs the traces, posts the exchange,
  launches the kernel on those elements while the traces are in flight,
  makes the stream wait for the exchange and launches it on the elements
  with halo faces (hb_lsrk_stage_elements) -- the reference's futures
  (hedge/backends/mpi/__init__.py:184-216, hedge/compiler.py:414-467) on
  CUDA streams.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native
from .discretization import build_face_table, op_descriptor
from .lowering import as_descriptor
from .models import MODEL_VARWAVE


def _torch():
    import torch
    return torch


def _morton_key(x, bits=10):
    """Interleaved-bit key of points x [n, d] scaled into the unit cube."""
    lo, hi = x.min(0), x.max(0)
    q = ((x - lo) / np.maximum(hi - lo, 1e-300) * ((1 << bits) - 1)).astype(np.uint64)
    key = np.zeros(len(x), dtype=np.uint64)
    d = x.shape[1]
    for b in range(bits):
        for c in range(d):
            key |= ((q[:, c] >> np.uint64(b)) & np.uint64(1)) << np.uint64(b * d + c)
    return key


def partition_elements(discr, nparts):
    """Owner part of every element: equal contiguous pieces of the Morton
    order of the element centroids."""
    cent = discr.nodes.reshape(discr.K, discr.Np, -1).mean(1)
    order = np.argsort(_morton_key(cent), kind="stable")
    owner = np.empty(discr.K, dtype=np.int64)
    for r, chunk in enumerate(np.array_split(order, nparts)):
        owner[chunk] = r
    return owner


class PartPlan:
    """One part's view: owned elements (global ids; those without halo faces
    first, each group ascending), local face table, halo receive counts per
    source part and send lists per destination part (local volume node
    indices)."""

    def __init__(self, rank):
        self.rank = rank
        self.elements = None      # owned elements: without halo faces, then with
        self.n_interior = 0       # how many have no halo face
        self.conn = None
        self.n_halo_faces = 0
        self.recv_nodes = {}      # source part -> halo nodes received from it
        self.send_idx = {}        # destination part -> local volume node indices
        self.halo_global = None   # global volume index of every halo node (receiver order)


class PartitionPlan:
    def __init__(self, discr, ot, nparts, owner=None):
        ot = as_descriptor(ot, discr.dimensions, discr.mesh)
        conn, n_given, _ = build_face_table(discr, ot)
        if n_given:
            raise NotImplementedError("partitions with given boundary data")
        self.nparts = nparts
        self.owner = partition_elements(discr, nparts) if owner is None else np.asarray(owner)
        K, Np, Nfp, nf = discr.K, discr.Np, discr.Nfp, discr.Nfaces
        ld = discr.ldis
        fmask = np.asarray(ld.fmask)
        shuffle = np.asarray(ld.face_shuffle_table)
        local_index = np.empty(K, dtype=np.int64)
        self.parts = [PartPlan(r) for r in range(nparts)]
        nbr_all = conn[..., 0].astype(np.int64)
        cut = (nbr_all >= 0) & (self.owner[np.maximum(nbr_all, 0)] != self.owner[:, None])
        cut_el = cut.any(1)                       # elements with a halo face
        for r, p in enumerate(self.parts):
            own = np.nonzero(self.owner == r)[0]
            # elements without halo faces first (launched while the traces
            # are exchanged), then those with halo faces
            p.elements = np.concatenate([own[~cut_el[own]], own[cut_el[own]]])
            p.n_interior = int((~cut_el[own]).sum())
            local_index[p.elements] = np.arange(len(p.elements))
        for r, p in enumerate(self.parts):
            E = p.elements
            Kr = len(E)
            c = conn[E].astype(np.int64)                   # [Kr, nf, 2]
            nb, code = c[..., 0].copy(), c[..., 1].copy()
            interior = nb >= 0
            nbo = np.where(interior, self.owner[np.maximum(nb, 0)], -1)
            own = interior & (nbo == r)
            c[..., 0] = np.where(own, local_index[np.maximum(nb, 0)], c[..., 0])
            hi, hf = np.nonzero(interior & (nbo != r))     # halo faces (element, face)
            src = nbo[hi, hf]
            order = np.lexsort((hf, hi, src))              # by source part, then element, face
            hi, hf, src = hi[order], hf[order], src[order]
            c[hi, hf, 0] = Kr + np.arange(len(hi))
            p.conn = np.ascontiguousarray(c.astype(np.int32))
            p.n_halo_faces = len(hi)
            nbg = nb[hi, hf]
            hcode = code[hi, hf]
            nface, perm = hcode & 3, hcode >> 2
            # neighbour volume node of each halo face node, in this face's order
            nodes = fmask[nface[:, None], shuffle[perm][:, :]] if len(hi) else \
                np.zeros((0, Nfp), dtype=np.int64)
            p.halo_global = (nbg[:, None] * Np + nodes).reshape(-1)
            src_nodes = np.repeat(src, Nfp)
            for s in range(nparts):
                sel = src_nodes == s
                n = int(sel.sum())
                if n:
                    p.recv_nodes[s] = n
                    gidx = p.halo_global[sel]
                    el = gidx // Np
                    self.parts[s].send_idx[r] = local_index[el] * Np + (gidx - el * Np)

    def part(self, r):
        return self.parts[r]


class DistExchange:
    """Halo exchange between processes of a torch.distributed group:
    batched point-to-point sends of each destination's slice of the send
    buffer and receives into each source's slice of the halo buffer."""

    def __init__(self, plan, rank, group=None):
        self.plan, self.rank, self.group = plan, rank, group

    def start(self, send, halo):
        """Posts the sends and receives; returns their requests.  With NCCL
        the transfers run on NCCL's stream once the current stream's work
        (the pack) is done, so kernels launched meanwhile overlap them."""
        import torch.distributed as dist
        p = self.plan.parts[self.rank]
        ops = []
        off = 0
        for d in sorted(p.send_idx):
            n = len(p.send_idx[d])
            ops.append(dist.P2POp(dist.isend, send[off:off + n], d, group=self.group))
            off += n
        off = 0
        for s in sorted(p.recv_nodes):
            n = p.recv_nodes[s]
            ops.append(dist.P2POp(dist.irecv, halo[off:off + n], s, group=self.group))
            off += n
        return dist.batch_isend_irecv(ops) if ops else []

    @staticmethod
    def finish(reqs):
        """Waits for the requests (NCCL: the current stream waits; the host
        does not)."""
        for req in reqs:
            req.wait()

    def __call__(self, send, halo):
        self.finish(self.start(send, halo))


def sum_over_ranks(value, group=None, device=None):
    """A float summed over the ranks of ``group`` (all-reduce); the value
    itself without an initialised process group.  NCCL reduces a tensor on
    ``device``, other backends on the host."""
    import torch.distributed as dist
    torch = _torch()
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    on_dev = dist.get_backend(group) == "nccl"
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if on_dev else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t.item())


def partitioned_norm(parts, qs):
    """Energy norm of a field held as several parts in one process."""
    return sum(p.norm_sq(q) for p, q in zip(parts, qs)) ** 0.5


class LocalExchange:
    """All parts in one process (one device): copies each source's send
    slice into each destination's halo slice.  ``parts`` are the
    PartitionedOperators indexed by part."""

    def __init__(self, plan, parts):
        self.plan, self.parts = plan, parts

    def exchange_all(self):
        plan = self.plan
        for r, pr in enumerate(plan.parts):
            off = 0
            for s in sorted(pr.recv_nodes):
                n = pr.recv_nodes[s]
                ps = plan.parts[s]
                soff = 0
                for d in sorted(ps.send_idx):
                    if d == r:
                        break
                    soff += len(ps.send_idx[d])
                self.parts[r].halo[off:off + n].copy_(self.parts[s].send[soff:soff + n])
                off += n


class PartitionedOperator:
    """One part of an element-partitioned model operator on one device
    (any precision path)."""

    def __init__(self, discr, model, plan, rank, precision="fp64", device=None, exchange=None):
        torch = _torch()
        ot = as_descriptor(model.op_template(), discr.dimensions, discr.mesh)
        if ot.params.get("variable_material"):
            raise NotImplementedError("partitions of Maxwell with variable material "
                                      "(the halo carries no material values)")
        self.ot, self.plan, self.rank = ot, plan, rank
        self.part = p = plan.parts[rank]
        self.F = ot.n_fields
        self.Np = discr.Np
        self.K = len(p.elements)
        self.n_interior = p.n_interior
        self.device = torch.device(device) if device is not None else discr.device
        prec = {"fp64": _native.PREC_FP64, "fp32": _native.PREC_FP32,
                "fp32-simt": _native.PREC_FP32_SIMT,
                "bf16x3": _native.PREC_BF16X3, "fp16x3": _native.PREC_FP16X3}[precision]
        self.dtype = torch.float32 if precision in ("fp32", "fp32-simt") else torch.float64
        self.lib = lib = _native.load()
        ld = discr.ldis
        E = p.elements
        self._keep = dict(
            dmats=np.ascontiguousarray(np.stack(ld.differentiation_matrices)),
            lift=np.ascontiguousarray(ld.lifting_matrix),
            geo=np.ascontiguousarray(discr.geometry[E]),
            fmask=np.ascontiguousarray(ld.fmask, dtype=np.int32),
            shuffle=np.ascontiguousarray(ld.face_shuffle_table, dtype=np.int32),
            unit_nodes=np.ascontiguousarray(ld.unit_nodes, dtype=np.float64),
            mass=np.ascontiguousarray(ld.mass_matrix, dtype=np.float64),
            absjac=np.ascontiguousarray(np.abs(discr.mesh.jacobians[E]), dtype=np.float64),
            conn=p.conn)
        k = self._keep
        dd = _native.hb_discr_desc(
            discr.dimensions, discr.order, discr.Np, discr.Nfp, discr.Nfaces,
            len(ld.face_shuffle_perms), self.K, k["dmats"].ctypes.data, k["lift"].ctypes.data,
            k["geo"].ctypes.data, k["fmask"].ctypes.data, k["shuffle"].ctypes.data,
            int(self.device.index or 0), k["unit_nodes"].ctypes.data, k["mass"].ctypes.data,
            k["absjac"].ctypes.data)
        h = C.c_void_p()
        _native.check(lib.hb_discr_create(C.byref(dd), C.byref(h)))
        self._dh = h
        od = op_descriptor(ot, prec, p.conn, 0, p.n_halo_faces)
        h = C.c_void_p()
        _native.check(lib.hb_op_create(self._dh, C.byref(od), C.byref(h)))
        self._h = h
        n_send = sum(len(v) for v in p.send_idx.values())
        n_halo = p.n_halo_faces * discr.Nfp
        self.send = torch.zeros((max(n_send, 1), self.F), dtype=self.dtype, device=self.device)
        self.halo = torch.zeros((max(n_halo, 1), self.F), dtype=self.dtype, device=self.device)
        idx = np.concatenate([p.send_idx[d] for d in sorted(p.send_idx)]) if n_send else \
            np.zeros(1, dtype=np.int64)
        self.send_idx = torch.as_tensor(idx.astype(np.int64), device=self.device)
        self.n_send = n_send
        self.coeff = self.halo_c = None
        if ot.model == MODEL_VARWAVE:
            c = model.c
            cg = np.full(len(discr), float(c)) if np.isscalar(c) else np.asarray(c, dtype=np.float64)
            loc = (E[:, None] * discr.Np + np.arange(discr.Np)).reshape(-1)
            self.coeff = torch.as_tensor(cg[loc], device=self.device)
            hc = cg[p.halo_global] if n_halo else np.zeros(1)
            self.halo_c = torch.as_tensor(np.ascontiguousarray(hc), device=self.device)
        if p.n_halo_faces:
            _native.check(lib.hb_op_set_halo(
                self._h, self.halo.data_ptr(),
                self.halo_c.data_ptr() if self.halo_c is not None else None))
        self.exchange = exchange

    def __del__(self):
        try:
            if getattr(self, "_h", None) is not None:
                self.lib.hb_op_destroy(self._h)
                self._h = None
            if getattr(self, "_dh", None) is not None:
                self.lib.hb_discr_destroy(self._dh)
                self._dh = None
        except Exception:
            pass

    def _stream(self):
        return _torch().cuda.current_stream(self.device).cuda_stream

    # -- global <-> local ------------------------------------------------------
    def local_nodes(self):
        E = self.part.elements
        return (E[:, None] * self.Np + np.arange(self.Np)).reshape(-1)

    def scatter(self, q_global):
        """This part's slice [F, K_local*Np] of a global state (numpy or tensor)."""
        torch = _torch()
        q = torch.as_tensor(np.asarray(q_global)) if not isinstance(q_global, torch.Tensor) \
            else q_global
        idx = torch.as_tensor(self.local_nodes(), device=q.device)
        return q.reshape(self.F, -1)[:, idx].to(device=self.device, dtype=self.dtype).contiguous()

    # -- exchange and kernels ----------------------------------------------------
    def pack(self, q):
        if self.n_send:
            _native.check(self.lib.hb_pack(
                self.n_send, 0 if self.dtype == _torch().float64 else 1, self.F,
                self.K * self.Np, self.send_idx.data_ptr(), q.data_ptr(), self.send.data_ptr(),
                self._stream()))

    def _exchange(self, q):
        self.pack(q)
        if self.exchange is not None:
            self.exchange(self.send[:self.n_send], self.halo)

    def _run(self, launch, q, exchanged, by_ranges):
        """``launch(e0, e1)`` over this part's elements, the halo refreshed
        from ``q`` first unless ``exchanged`` (a LocalExchange already filled
        it).  A DistExchange overlaps the transfer with the launch on the
        elements without halo faces; ``by_ranges`` launches the two element
        ranges separately after an exchange that is already done."""
        if not exchanged and self.exchange is not None and hasattr(self.exchange, "start"):
            self.pack(q)
            reqs = self.exchange.start(self.send[:self.n_send], self.halo)
            launch(0, self.n_interior)
            self.exchange.finish(reqs)
            launch(self.n_interior, self.K)
            return
        if not exchanged:
            self._exchange(q)
        if by_ranges:
            launch(0, self.n_interior)
            launch(self.n_interior, self.K)
        else:
            launch(0, self.K)

    def rhs(self, q, exchanged=False, by_ranges=False):
        """RHS of this part's elements."""
        torch = _torch()
        out = torch.empty_like(q)
        coeff = self.coeff.data_ptr() if self.coeff is not None else None

        def launch(e0, e1):
            _native.check(self.lib.hb_rhs_elements(
                self._h, e0, e1, q.data_ptr(), out.data_ptr(), coeff, None, None,
                self._stream()))
        self._run(launch, q, exchanged, by_ranges)
        return out

    def lsrk_stage(self, a, b, dt, q_in, q_out, res, exchanged=False, by_ranges=False):
        coeff = self.coeff.data_ptr() if self.coeff is not None else None

        def launch(e0, e1):
            _native.check(self.lib.hb_lsrk_stage_elements(
                self._h, e0, e1, float(a), float(b), float(dt), q_in.data_ptr(),
                q_out.data_ptr(), res.data_ptr(), coeff, None, None, self._stream()))
        self._run(launch, q_in, exchanged, by_ranges)

    def check(self):
        _native.check(self.lib.hb_op_check(self._h, self._stream()))

    # -- reductions ------------------------------------------------------------
    def norm_sq(self, q):
        """Squared energy norm of this part's elements, all fields:
        sum_k |J_k| q_k^T M q_k, FP64 on the device (hb_norm)."""
        torch = _torch()
        qq = q.reshape(self.F, -1).contiguous()
        out = torch.empty(1, dtype=torch.float64, device=self.device)
        _native.check(self.lib.hb_norm(self._dh, self.F,
                                       0 if qq.dtype == torch.float64 else 1,
                                       qq.data_ptr(), out.data_ptr(), self._stream()))
        return float(out.item()) ** 2

    def norm(self, q, group=None):
        """Energy norm of the whole partitioned field: every rank's squared
        norm summed over the ranks (all-reduce; NCCL between GPUs), then the
        square root -- the reference's nodal sum plus allreduce
        (backends/mpi/__init__.py:266-280)."""
        return sum_over_ranks(self.norm_sq(q), group, self.device) ** 0.5
