"""Host stand-in of pmsim_b200.shard.DevicePcg for the multi-process gloo tests (test
infrastructure: the product's distributed PCG runs on the library's CUDA kernels only).

It restates what the pms_dpcg kernels do, call for call, in numpy on CPU tensors: the prescribed
DOFs eliminated (identity rows, dropped columns), the owned rows split into interior and boundary
rows, the inverse of each owned node's free diagonal block as preconditioner, and the convergence
flag that freezes the iterates once r.z <= rtol^2 r0.z0 (all on the all-reduced scalars)."""
import numpy as np
import torch

from pmsim_b200.shard import DONE, ITERS, PQ, RZ, RZ0, RZN


class HostPcg:
    def __init__(self, indptr, indices, n_owned, n_local, fixed_local, halo, ndim, device="cpu"):
        n, nd = int(n_owned), int(ndim)
        fx = np.asarray(fixed_local, dtype=bool)
        ptr, col, src, interior, boundary = [0], [], [], [], []
        for row in range(n):
            if fx[row]:
                kept = [(row, -1)]
            else:
                kept = [(int(indices[k]), k) for k in range(int(indptr[row]), int(indptr[row + 1]))
                        if not fx[int(indices[k])]]
            col += [c for c, _ in kept]
            src += [k for _, k in kept]
            ptr.append(len(col))
            (boundary if any(c >= n for c, _ in kept) else interior).append(row)
        self.n, self.nd, self.fixed = n, nd, fx[:n]
        self.ptr, self.col, self.src = np.array(ptr), np.array(col, dtype=np.int64), np.array(src, dtype=np.int64)
        self.rows = (np.array(interior, dtype=np.int64), np.array(boundary, dtype=np.int64))
        self.send, self.recv = halo.send_dofs, halo.recv_dofs
        f64 = dict(dtype=torch.float64)
        self.x, self.r, self.z, self.q = (torch.zeros(n, **f64) for _ in range(4))
        self.p = torch.zeros(int(n_local), **f64)
        self.sendbuf = torch.zeros(len(self.send), **f64)
        self.recvbuf = torch.zeros(len(self.recv), **f64)
        self.scal = torch.zeros(6, **f64)

    def _done(self):
        return float(self.scal[DONE]) != 0.0

    def set_values(self, values):
        import scipy.sparse as sp
        v = np.asarray(values, dtype=np.float64)
        self.val = np.where(self.src >= 0, v[np.maximum(self.src, 0)], 1.0)
        full = sp.csr_matrix((self.val, self.col, self.ptr), shape=(self.n, len(self.p)))
        self._mats = [full[rows] for rows in self.rows]
        nd = self.nd
        self.binv = np.zeros((self.n // nd, nd, nd))
        for node in range(self.n // nd):
            free = [i for i in range(nd) if not self.fixed[node * nd + i]]
            blk = np.zeros((len(free), len(free)))
            for a, i in enumerate(free):
                row = node * nd + i
                for k in range(self.ptr[row], self.ptr[row + 1]):
                    c = self.col[k]
                    if c // nd == node and (c % nd) in free:
                        blk[a, free.index(c % nd)] = self.val[k]
            if free:
                self.binv[node][np.ix_(free, free)] = np.linalg.inv(blk)

    def _precondition(self, r):
        return np.einsum("nij,nj->ni", self.binv, r.reshape(-1, self.nd)).reshape(-1)

    def start(self, b):
        b = np.asarray(b, dtype=np.float64)
        r = np.where(self.fixed, 0.0, b)
        z = self._precondition(r)
        self.x[:] = 0.0
        self.r[:] = torch.as_tensor(r)
        self.z[:] = torch.as_tensor(z)
        self.p[:self.n] = torch.as_tensor(z)
        self.scal[RZN] = float(r @ z)

    def init(self):
        self.scal[RZ] = self.scal[RZN]
        self.scal[RZ0] = self.scal[RZN]
        self.scal[ITERS] = 0.0
        self.scal[DONE] = 0.0 if float(self.scal[RZN]) > 0.0 else 1.0

    def pack(self):
        if not self._done():
            self.sendbuf[:] = self.p[torch.as_tensor(self.send)]

    def unpack(self):
        if not self._done():
            self.p[torch.as_tensor(self.recv)] = self.recvbuf

    def spmv(self, boundary):
        if self._done():
            return
        rows = self.rows[int(boundary)]
        if len(rows):
            self.q[torch.as_tensor(rows)] = torch.as_tensor(self._mats[int(boundary)] @ self.p.numpy())

    def dot_pq(self):
        self.scal[PQ] = 0.0 if self._done() else float(self.p[:self.n] @ self.q)

    def update(self):
        if self._done():
            self.scal[RZN] = 0.0
            return
        alpha = float(self.scal[RZ]) / float(self.scal[PQ])
        self.x += alpha * self.p[:self.n]
        self.r -= alpha * self.q
        z = self._precondition(self.r.numpy())
        self.z[:] = torch.as_tensor(z)
        self.scal[RZN] = float(self.r.numpy() @ z)

    def direction(self, rtol):
        if self._done():
            return
        beta = float(self.scal[RZN]) / float(self.scal[RZ])
        self.p[:self.n] = self.z + beta * self.p[:self.n]
        self.scal[RZ] = self.scal[RZN]
        self.scal[ITERS] += 1.0
        if float(self.scal[RZN]) <= rtol * rtol * float(self.scal[RZ0]):
            self.scal[DONE] = 1.0
