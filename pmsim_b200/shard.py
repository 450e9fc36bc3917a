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
* the conjugate-gradient solve over the owned rows needs two all-reduces per iteration.

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


def owned_rows(indptr: np.ndarray, indices: np.ndarray, values: np.ndarray, n_owned_dof: int):
    """The owned rows of a local CSR matrix (the first n_owned_dof rows of the sub-mesh's K)."""
    end = int(indptr[n_owned_dof])
    return indptr[:n_owned_dof + 1].copy(), indices[:end].copy(), values[:end].copy()


def _ell(rows, cols, vals, n):
    """Row-padded (ELL) form of a row-sorted coordinate matrix: cols/vals of shape (n, width),
    padding entries point at column 0 with value 0."""
    counts = np.bincount(rows, minlength=n)
    width = int(counts.max()) if n else 0
    start = np.concatenate([[0], np.cumsum(counts)[:-1]])
    slot = np.arange(len(rows)) - start[rows]
    ec = np.zeros((n, width), dtype=np.int64)
    ev = np.zeros((n, width))
    ec[rows, slot] = cols
    ev[rows, slot] = vals
    return ec, ev


def _spmv(ell_cols, ell_vals, x):
    """y = A x with A in row-padded form: a fixed-order sum over each row (no atomics), so the
    product, and the CG iterates built on it, are the same bits on every run."""
    return (ell_vals * x[ell_cols]).sum(dim=1)


def dist_cg(indptr, indices, values, b_owned, halo: Halo, n_local_dof: int, fixed_local: np.ndarray,
            rtol=1e-12, max_iterations=10000):
    """Jacobi-preconditioned CG on the owned rows of K with the prescribed DOFs eliminated (their
    rows and columns replaced by the identity, right-hand side zero there).  indptr/indices/values:
    the owned rows, columns in local DOF numbering; b_owned: owned right-hand side; fixed_local:
    prescribed flags of every local DOF (owned and ghost).  Two all-reduces per iteration (r.z and
    p.q); stops when r.z <= rtol^2 of its initial value.  Returns (x_owned, iterations)."""
    import torch
    import torch.distributed as dist
    n = len(b_owned)
    dev = b_owned.device
    fixed_local = np.asarray(fixed_local, dtype=bool)
    rows = np.repeat(np.arange(n), np.diff(indptr))
    keep = ~(fixed_local[rows] | fixed_local[indices])
    fr = np.flatnonzero(fixed_local[:n])
    r_all = np.concatenate([rows[keep], fr])
    c_all = np.concatenate([indices[keep], fr])
    v_all = np.concatenate([values[keep], np.ones(len(fr))])
    order = np.lexsort((c_all, r_all))
    r_all, c_all, v_all = r_all[order], c_all[order], v_all[order]
    diag = np.zeros(n)
    d = r_all == c_all
    np.add.at(diag, r_all[d], v_all[d])
    dinv = torch.as_tensor(1.0 / diag, device=dev)
    ec, ev = _ell(r_all, c_all.astype(np.int64), v_all, n)  # the device pattern is int32
    t_cols = torch.as_tensor(ec, device=dev)
    t_vals = torch.as_tensor(ev, device=dev)
    b = b_owned.clone()
    b[torch.as_tensor(fr, device=dev)] = 0.0

    def allsum(t):
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return t

    x = torch.zeros(n, dtype=b.dtype, device=dev)
    r = b.clone()
    z = dinv * r
    p_local = torch.zeros(n_local_dof, dtype=b.dtype, device=dev)
    p_local[:n] = z
    rz = allsum((r * z).sum().reshape(1))[0]
    rz0 = float(rz)
    it = 0
    while it < max_iterations and float(rz) > rtol * rtol * rz0:
        halo.exchange(p_local)
        q = _spmv(t_cols, t_vals, p_local)
        pq = allsum((p_local[:n] * q).sum().reshape(1))[0]
        alpha = rz / pq
        x += alpha * p_local[:n]
        r -= alpha * q
        z = dinv * r
        rz_new = allsum((r * z).sum().reshape(1))[0]
        p_local[:n] = z + (rz_new / rz) * p_local[:n]
        rz = rz_new
        it += 1
    return x, it


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
                prescribed_local=None):
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
    CUDA device for NCCL).  Returns the per-step histories [(iteration, max|R|, rel(mdu))...] and
    the owned displacements."""
    import torch
    import torch.distributed as dist
    nl = shard.n_local * ndim
    n = shard.n_owned * ndim
    fixed_local = np.asarray(fixed_local, dtype=bool)
    fixed_own = fixed_local[:n]
    pres = np.flatnonzero(fixed_own)  # owned prescribed DOFs (one multiplier each in LMM form)
    lmm = prescribed_local is not None
    halo = Halo(shard, ndim)

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
            if lmm:
                vp = np.zeros(nl)
                vp[pres] = rr_p  # mdu on the prescribed DOFs
                b = rr - kmul(rows, vp)
                mdu_f, _ = dist_cg(*rows, torch.as_tensor(b, device=device), halo, nl, fixed_local, rtol=cg_rtol)
                mdu = mdu_f.cpu().numpy()
                mdu[pres] = rr_p
                full = np.zeros(nl)
                full[:n] = mdu
                mdl = rr[pres] - kmul(rows, full)[pres]
                mvec = np.concatenate([mdu, mdl])
            else:
                mdu_t, _ = dist_cg(*rows, torch.as_tensor(rr, device=device), halo, nl, fixed_local, rtol=cg_rtol)
                mdu = mdu_t.cpu().numpy()
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
