"""One problem sharded over ranks: owner-computes partition, halo exchange, distributed CG.

pmsim solves one problem in one process (``src/fem/solver_implicit.rs``); this module has no
counterpart in the reference.  It splits one mesh over ``nparts`` ranks so that every rank holds
a disjoint set of CSR block rows of K and R:

* every node (block row) has one owner (``node_owner``: equal-count slabs along the longest axis);
* a rank computes every cell that touches a node it owns, so its owned rows of K and R are
  complete without exchanging element matrices (cells on a slab boundary are computed by both
  ranks); its local sub-mesh holds those cells and every node they touch: the owned nodes first,
  then the ghost nodes owned by other ranks;
* per Newton iteration the ranks exchange the ghost values of the displacement increment (and,
  inside the linear solve, of the search direction) with their neighbours only;
* the linear solve is this library's distributed block-Jacobi PCG (``DevicePcg`` over the
  ``pms_dpcg_*`` kernels): the exchange of the search direction's ghost values runs while the
  interior rows are multiplied, and each iteration needs two all-reduces of one scalar, read by
  the kernels from device memory (no host synchronisation inside an iteration).

The element work of a rank is the ordinary element path (``Elements`` / ``pms_elements_*``) on its
sub-mesh: its first ``n_owned`` block rows of K and entries of R are the owned ones.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .mesh import Mesh


def node_owner(mesh: Mesh, nparts: int, axis: int | None = None) -> np.ndarray:
    """Owner rank of every node: equal-count slabs of the node coordinates along ``axis`` (default:
    the axis of largest extent); ties keep the node order, so the result is deterministic."""
    if nparts < 1:
        raise ValueError("nparts must be >= 1")
    if axis is None:
        axis = int(np.argmax(np.ptp(mesh.coords, axis=0)))
    order = np.argsort(mesh.coords[:, axis], kind="stable")
    owner = np.empty(mesh.npoint, dtype=np.int32)
    owner[order] = (np.arange(mesh.npoint, dtype=np.int64) * nparts) // mesh.npoint
    return owner


@dataclass
class Shard:
    part: int
    nparts: int
    nodes: np.ndarray  # global node ids: owned (ascending), then ghosts (ascending)
    n_owned: int
    cells: np.ndarray  # global ids of the cells computed here (ascending)
    mesh: Mesh  # local sub-mesh over `nodes` and `cells`
    recv: dict = field(default_factory=dict)  # rank q -> local positions of the ghosts q owns
    send: dict = field(default_factory=dict)  # rank q -> local positions of owned nodes q needs

    @property
    def n_local(self) -> int:
        return len(self.nodes)


def build_shards(mesh: Mesh, owner: np.ndarray, nparts: int) -> list[Shard]:
    """The shards of every rank (each rank may build all and keep its own: the result is the same on
    every rank).  The ghost lists are sorted by global id on both sides, so rank p's recv[q] and
    rank q's send[p] name the same nodes in the same order."""
    owner = np.asarray(owner)
    if owner.shape != (mesh.npoint,) or owner.min() < 0 or owner.max() >= nparts:
        raise ValueError("owner must give a rank in [0, nparts) for every node")
    shards = []
    for p in range(nparts):
        owned = np.flatnonzero(owner == p)
        cells = np.flatnonzero(np.any(owner[mesh.cells] == p, axis=1))
        used = np.unique(mesh.cells[cells])
        ghosts = np.setdiff1d(used, owned)
        nodes = np.concatenate([owned, ghosts])
        g2l = np.full(mesh.npoint, -1, dtype=np.int64)
        g2l[nodes] = np.arange(len(nodes))
        sub = Mesh(mesh.ndim, mesh.coords[nodes], g2l[mesh.cells[cells]], mesh.kind)
        sh = Shard(p, nparts, nodes, len(owned), cells, sub)
        for q in np.unique(owner[ghosts]):
            sh.recv[int(q)] = g2l[ghosts[owner[ghosts] == q]]
        shards.append(sh)
    for sh in shards:  # send lists: what every other rank receives from this one, in its order
        g2l = {int(g): i for i, g in enumerate(sh.nodes[:sh.n_owned])}
        for other in shards:
            if sh.part in other.recv:
                need = other.nodes[other.recv[sh.part]]
                sh.send[other.part] = np.array([g2l[int(g)] for g in need], dtype=np.int64)
    return shards


def dof_index(node_positions: np.ndarray, ndim: int) -> np.ndarray:
    """Local DOF indices (node * ndim + d) of the given local node positions."""
    return (np.asarray(node_positions, dtype=np.int64)[:, None] * ndim + np.arange(ndim)).reshape(-1)


class Halo:
    """Exchange of ghost values over torch.distributed point-to-point calls (gloo on CPU, NCCL on
    GPUs): x holds the local vector (owned DOFs first); the ghost entries are overwritten with their
    owners' values.  Every rank posts its sends and receives in ascending neighbour order."""

    def __init__(self, shard: Shard, ndim: int):
        self.send = {q: dof_index(v, ndim) for q, v in sorted(shard.send.items())}
        self.recv = {q: dof_index(v, ndim) for q, v in sorted(shard.recv.items())}
        self._dev = {}  # device -> (send, recv) index tensors

    def _index(self, device):
        import torch
        key = str(device)
        if key not in self._dev:
            self._dev[key] = ({q: torch.as_tensor(i, device=device) for q, i in self.send.items()},
                              {q: torch.as_tensor(i, device=device) for q, i in self.recv.items()})
        return self._dev[key]

    def exchange(self, x):
        """Posts every send and receive of this rank as one group (torch.distributed's
        batch_isend_irecv): NCCL then issues them together, so two neighbours that both send
        first cannot wait on each other; gloo runs the same list."""
        import torch
        import torch.distributed as dist
        send, recv = self._index(x.device)
        ops, bufs = [], {}
        for q, idx in send.items():
            ops.append(dist.P2POp(dist.isend, x[idx].contiguous(), q))
        for q, idx in recv.items():
            bufs[q] = torch.empty(len(idx), dtype=x.dtype, device=x.device)
            ops.append(dist.P2POp(dist.irecv, bufs[q], q))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        for q, idx in recv.items():
            x[idx] = bufs[q]
        return x

    @property
    def send_dofs(self) -> np.ndarray:
        """Owned local DOFs sent to the neighbours, concatenated in ascending neighbour order."""
        return np.concatenate([v for _, v in sorted(self.send.items())] + [np.zeros(0, np.int64)])

    @property
    def recv_dofs(self) -> np.ndarray:
        """Ghost local DOFs received from the neighbours, concatenated in ascending neighbour order."""
        return np.concatenate([v for _, v in sorted(self.recv.items())] + [np.zeros(0, np.int64)])

    def segments(self):
        """(neighbour, send offset, send count, receive offset, receive count) in ascending order."""
        out, so, ro = [], 0, 0
        for q in sorted(set(self.send) | set(self.recv)):
            ns, nr = len(self.send.get(q, ())), len(self.recv.get(q, ()))
            out.append((q, so, ns, ro, nr))
            so += ns
            ro += nr
        return out

    def post(self, sendbuf, recvbuf):
        """Posts the exchange of packed buffers (send_dofs / recv_dofs order) as one group and
        returns its requests; on NCCL they run on the communicator's stream while the caller's
        stream goes on (finish makes it wait)."""
        import torch.distributed as dist
        ops = []
        for q, so, ns, ro, nr in self.segments():
            if ns:
                ops.append(dist.P2POp(dist.isend, sendbuf[so:so + ns], q))
            if nr:
                ops.append(dist.P2POp(dist.irecv, recvbuf[ro:ro + nr], q))
        return dist.batch_isend_irecv(ops) if ops else []

    @staticmethod
    def finish(requests):
        for r in requests:
            r.wait()


def owned_rows(indptr: np.ndarray, indices: np.ndarray, values: np.ndarray, n_owned_dof: int):
    """The owned rows of a local CSR matrix (the first n_owned_dof rows of the sub-mesh's K)."""
    end = int(indptr[n_owned_dof])
    return indptr[:n_owned_dof + 1].copy(), indices[:end].copy(), values[:end].copy()


# Slots of the PCG scalars (pms_dpcg_bind): the caller all-reduces RZN and PQ across ranks.
RZN, PQ, RZ, RZ0, DONE, ITERS = range(6)


class DevicePcg:
    """One rank's distributed block-Jacobi PCG on this library's kernels (``pms_dpcg_*``): the owned
    rows of K with the prescribed DOFs eliminated, split into interior and boundary rows so that the
    ghost exchange overlaps the interior SpMV; block-Jacobi preconditioner over the owned nodes;
    fixed-shape reductions.  CUDA tensors only: there is no host path.

    indptr/indices: pattern of the owned rows of the local K (local DOF numbering); fixed_local:
    prescribed flags of every local DOF; the values come with set_values every Newton iteration."""

    def __init__(self, indptr, indices, n_owned: int, n_local: int, fixed_local, halo: "Halo", ndim: int, device):
        import ctypes

        import torch

        from . import _lib
        dev = torch.device(device)
        if dev.type != "cuda":
            raise RuntimeError("DevicePcg runs on the library's CUDA kernels: give it a CUDA device")
        self.L = _lib.load()
        self.device = dev
        ip = np.ascontiguousarray(indptr[:n_owned + 1], dtype=np.int64)
        ix = np.ascontiguousarray(indices[:int(ip[-1])], dtype=np.int32)
        fx = np.ascontiguousarray(np.asarray(fixed_local, dtype=bool).astype(np.uint8))
        sd = np.ascontiguousarray(halo.send_dofs, dtype=np.int64)
        rd = np.ascontiguousarray(halo.recv_dofs, dtype=np.int64)
        h = ctypes.c_void_p()
        with torch.cuda.device(dev):
            rc = self.L.pms_dpcg_create(ndim, n_owned, n_local, _lib.ptr(ip), _lib.ptr(ix), _lib.ptr(fx), len(sd),
                                        _lib.ptr(sd), len(rd), _lib.ptr(rd), ctypes.byref(h))
        if rc != 0:
            raise _lib.PmsError(rc, (self.L.pms_dpcg_last_error(None) or b"").decode())
        self.h = h
        f64 = dict(dtype=torch.float64, device=dev)
        self.x = torch.zeros(n_owned, **f64)
        self.r = torch.zeros(n_owned, **f64)
        self.z = torch.zeros(n_owned, **f64)
        self.q = torch.zeros(n_owned, **f64)
        self.p = torch.zeros(n_local, **f64)
        self.sendbuf = torch.zeros(len(sd), **f64)
        self.recvbuf = torch.zeros(len(rd), **f64)
        self.scal = torch.zeros(6, **f64)
        self._values = None
        self._check(self.L.pms_dpcg_bind(self.h, *[_lib.ptr(t) if t.numel() else None for t in
                                                   (self.x, self.r, self.z, self.p, self.q, self.sendbuf,
                                                    self.recvbuf, self.scal)]))
        self._check(self.L.pms_dpcg_set_stream(self.h, torch.cuda.current_stream(dev).cuda_stream))

    def _check(self, rc):
        if rc != 0:
            from . import _lib
            raise _lib.PmsError(rc, (self.L.pms_dpcg_last_error(self.h) or b"").decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.pms_dpcg_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_values(self, values):
        """Values of the local K (host array or device tensor); the owned rows are taken."""
        import torch

        from . import _lib
        self._values = torch.as_tensor(values, dtype=torch.float64, device=self.device).contiguous()
        self._check(self.L.pms_dpcg_set_values(self.h, _lib.ptr(self._values)))

    def start(self, b):
        import torch

        from . import _lib
        self._b = torch.as_tensor(b, dtype=torch.float64, device=self.device).contiguous()
        self._check(self.L.pms_dpcg_start(self.h, _lib.ptr(self._b)))

    def init(self):
        self._check(self.L.pms_dpcg_init(self.h))

    def pack(self):
        self._check(self.L.pms_dpcg_pack(self.h))

    def unpack(self):
        self._check(self.L.pms_dpcg_unpack(self.h))

    def spmv(self, boundary: int):
        self._check(self.L.pms_dpcg_spmv(self.h, int(boundary)))

    def dot_pq(self):
        self._check(self.L.pms_dpcg_dot_pq(self.h))

    def update(self):
        self._check(self.L.pms_dpcg_update(self.h))

    def direction(self, rtol: float):
        self._check(self.L.pms_dpcg_direction(self.h, float(rtol)))

    def info(self):
        import ctypes
        c = (ctypes.c_int64 * 4)()
        self._check(self.L.pms_dpcg_info(self.h, c))
        return dict(nnz=c[0], interior_rows=c[1], boundary_rows=c[2], reduction_blocks=c[3])


class TorchComm:
    """The collectives of dist_cg over torch.distributed (NCCL on GPUs, gloo on CPU): in-place sums of
    the scalar slots and the halo's grouped point-to-point exchange."""

    def __init__(self, halo: "Halo"):
        self.halo = halo

    def allsum(self, t):
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.SUM)

    def post(self, sendbuf, recvbuf):
        return self.halo.post(sendbuf, recvbuf)

    def finish(self, requests):
        self.halo.finish(requests)


def dist_cg(pcg, comm, b_owned, rtol=1e-12, max_iterations=10000, check_every=8):
    """Block-Jacobi PCG over the ranks (the kernels of ``pcg``; the collectives of ``comm``, a
    TorchComm by default).  One iteration: pack the search direction's sent values, post the ghost
    exchange, multiply the interior rows while it is in flight, finish it, unpack the ghosts, multiply
    the boundary rows, then p.q (all-reduced), the update of x, r, z with r.z (all-reduced) and the
    new direction.  Convergence (r.z <= rtol^2 r0.z0) is decided on the device from the reduced
    value, the same on every rank, and freezes the iterates; the host reads the flag every
    ``check_every`` iterations, so the result does not depend on how often it looks.
    Returns (x_owned, iterations)."""
    if isinstance(comm, Halo):
        comm = TorchComm(comm)
    pcg.start(b_owned)
    comm.allsum(pcg.scal[RZN:RZN + 1])
    pcg.init()
    it = 0
    while it < max_iterations:
        for _ in range(min(check_every, max_iterations - it)):
            pcg.pack()
            req = comm.post(pcg.sendbuf, pcg.recvbuf)
            pcg.spmv(0)
            comm.finish(req)
            pcg.unpack()
            pcg.spmv(1)
            pcg.dot_pq()
            comm.allsum(pcg.scal[PQ:PQ + 1])
            pcg.update()
            comm.allsum(pcg.scal[RZN:RZN + 1])
            pcg.direction(rtol)
            it += 1
        if float(pcg.scal[DONE]) != 0.0:
            break
    return pcg.x, int(float(pcg.scal[ITERS]))


def _call(el, *names):
    for n in names:
        f = getattr(el, n, None)
        if f is not None:
            return f
    raise AttributeError(names[0])


def _local_kk(el):
    if hasattr(el, "assemble_kk_csr"):
        return el.assemble_kk_csr()
    indptr, indices = el.csr_pattern()
    return np.asarray(indptr), np.asarray(indices), np.asarray(el.assemble_kk())


def dist_newton(shard: Shard, ndim: int, elements, fixed_local, ff_ext_owned, nsteps, n_max_iterations=10,
                tol_rr_abs=1e-10, tol_mdu_rel=1e-8, cg_rtol=1e-13, on_step=None, device="cpu",
                prescribed_local=None, pcg_factory=None, comm=None):
    """The reference's implicit Newton loop (src/fem/solver_implicit.rs:187-272) over the ranks of a
    sharded problem.  ``elements`` runs the element calls on this rank's sub-mesh (the device
    ``Elements`` or any object with the same calls); ``ff_ext_owned(t)`` gives F_ext on the owned
    DOFs; ``fixed_local`` flags the prescribed DOFs of every local DOF.

    * ``prescribed_local`` None: reduced-system form with zero prescribed values
      (src/fem/bc_prescribed.rs:153-157).
    * ``prescribed_local(t)`` -> values at the local DOFs: Lagrange multipliers
      (src/fem/bc_prescribed.rs:99-134), solved by elimination, which gives the augmented direct
      solve's iterates: mdu_p = u_p - c, K_ff mdu_f = R_f - K_fp mdu_p, mdl = (R_p + l) - (K mdu)_p.
      The residual and rel(mdu) include the multiplier rows, as in the reference.

    Per iteration: R on the owned rows, max|R| over all ranks, K's owned rows, the correction by
    ``dist_cg``, rel(mdu) over all ranks, the owned dU update and the ghost exchange of dU before
    the stress update.  ``device`` holds the vectors that cross ranks ("cpu" for gloo, the rank's
    CUDA device for NCCL).  The linear solves run on ``pcg_factory(indptr, indices, n_owned, n_local,
    fixed_local, halo, ndim, device)``, built once from the pattern of the owned rows: DevicePcg
    (this library's kernels) unless another object with the same calls is given; ``comm`` (default
    TorchComm) carries its collectives.  Returns the per-step histories [(iteration, max|R|,
    rel(mdu))...] and the owned displacements."""
    import torch
    import torch.distributed as dist
    nl = shard.n_local * ndim
    n = shard.n_owned * ndim
    fixed_local = np.asarray(fixed_local, dtype=bool)
    fixed_own = fixed_local[:n]
    pres = np.flatnonzero(fixed_own)  # owned prescribed DOFs (one multiplier each in LMM form)
    lmm = prescribed_local is not None
    halo = Halo(shard, ndim)
    comm = comm if comm is not None else TorchComm(halo)
    pcg = None

    def allmax(x):
        t = torch.tensor([float(x)], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t[0])

    def kmul(rows, v_local):
        """(K v) on the owned rows for a local vector v (its ghost values exchanged first)."""
        vt = torch.as_tensor(v_local, device=device).clone()
        halo.exchange(vt)
        op, oi, ov = rows
        return np.bincount(np.repeat(np.arange(n), np.diff(op)), weights=ov * vt.cpu().numpy()[oi], minlength=n)

    _call(elements, "initialize_internal_values", "initialize")()
    u = np.zeros(n)
    lam = np.zeros(len(pres))
    histories = []
    for step in range(1, nsteps + 1):
        t = float(step)
        ddu = torch.zeros(nl, dtype=torch.float64, device=device)
        elements.reset_algorithmic_variables()
        ffe = np.asarray(ff_ext_owned(t), dtype=np.float64)
        if not lmm:
            ffe = np.where(fixed_own, 0.0, ffe)
        c = np.asarray(prescribed_local(t), dtype=np.float64)[:n][pres] if lmm else None
        hist, mdu0 = [], None
        for it in range(n_max_iterations):
            fi = np.asarray(elements.assemble_f_int())[:n]
            if lmm:
                rr = fi - ffe
                rr[pres] += lam
                rr_p = u[pres] - c
                norm_own = max(np.max(np.abs(rr)) if n else 0.0, np.max(np.abs(rr_p)) if len(pres) else 0.0)
            else:
                rr = np.where(fixed_own, 0.0, fi) - ffe
                norm_own = np.max(np.abs(rr)) if n else 0.0
            norm_rr = allmax(norm_own)
            if not np.isfinite(norm_rr):
                raise FloatingPointError("Found NaN or Inf")
            if norm_rr < tol_rr_abs:
                hist.append((it, norm_rr, None))
                break
            rows = owned_rows(*_local_kk(elements), n)
            if pcg is None:
                pcg = (pcg_factory or DevicePcg)(rows[0], rows[1], n, nl, fixed_local, halo, ndim, device)
            pcg.set_values(rows[2])
            if lmm:
                vp = np.zeros(nl)
                vp[pres] = rr_p  # mdu on the prescribed DOFs
                b = rr - kmul(rows, vp)
                mdu_f, _ = dist_cg(pcg, comm, b, rtol=cg_rtol)
                mdu = mdu_f.cpu().numpy().copy()
                mdu[pres] = rr_p
                full = np.zeros(nl)
                full[:n] = mdu
                mdl = rr[pres] - kmul(rows, full)[pres]
                mvec = np.concatenate([mdu, mdl])
            else:
                mdu_t, _ = dist_cg(pcg, comm, rr, rtol=cg_rtol)
                mdu = mdu_t.cpu().numpy().copy()
                mvec = mdu
            if it == 0:
                mdu0, rel = mvec.copy(), 1.0
            else:
                rel = allmax(np.max(np.abs(mvec) / (1.0 + np.abs(mdu0))) if len(mvec) else 0.0)
            hist.append((it, norm_rr, rel))
            if it > 0 and rel < tol_mdu_rel:
                break
            upd = np.ones(n, dtype=bool) if lmm else ~fixed_own
            u[upd] -= mdu[upd]
            if lmm:
                lam -= mdl
            ddu[:n][torch.as_tensor(upd, device=device)] -= torch.as_tensor(mdu[upd], device=device)
            halo.exchange(ddu)
            if it == 0:
                elements.backup_secondary_values()
            else:
                elements.restore_secondary_values()
            elements.update_secondary_values(ddu.cpu().numpy())
            if it == n_max_iterations - 1:
                raise RuntimeError("Newton-Raphson did not converge")
        histories.append(hist)
        if on_step is not None:
            on_step(step - 1, t, u.copy(), elements)
    return histories, u
