"""The distributed block-Jacobi PCG on this library's kernels (pms_dpcg_*, through
pmsim_b200.shard.dist_cg), with the ranks emulated in one process on one GPU: each rank's kernels
run on its own stream from its own host thread, and the collectives (the all-reduces of r.z and p.q,
the packed ghost exchange) are host-side reads and device copies between the ranks' buffers, met at
a barrier.  No kernel waits on another rank's kernel.  Checked against a direct solve of the whole
system, against the host stand-in of the same algorithm (tests/pcg_host.py), and for bit-identical
repeats."""
import threading

import numpy as np
import pytest
import torch

import oracle
from pcg_host import HostPcg
from pmsim_b200 import shard as S
from pmsim_b200.mesh import HEX8, QUA8, structured_2d, structured_3d

pytestmark = pytest.mark.gpu


class LocalComm:
    """Collectives between ranks that are host threads of one process."""

    def __init__(self, halos):
        self.halos = halos
        self.bar = threading.Barrier(len(halos))
        self.vals = [0.0] * len(halos)
        self.send = [None] * len(halos)

    def rank(self, p):
        return _RankComm(self, p)


class _RankComm:
    def __init__(self, shared, p):
        self.sh, self.p = shared, p

    @staticmethod
    def _sync(t):
        if t.is_cuda:
            torch.cuda.current_stream(t.device).synchronize()

    def allsum(self, t):
        sh = self.sh
        sh.vals[self.p] = float(t[0])  # reads after the rank's stream is done with it
        sh.bar.wait()
        total = 0.0
        for v in sh.vals:  # rank order, like a fixed reduction tree
            total += v
        sh.bar.wait()
        t.fill_(total)

    def post(self, sendbuf, recvbuf):
        sh = self.sh
        self._sync(sendbuf)
        sh.send[self.p] = sendbuf
        sh.bar.wait()
        for q, _, _, ro, nr in sh.halos[self.p].segments():
            if nr:
                so, ns = next((so, ns) for qq, so, ns, _, _ in sh.halos[q].segments() if qq == self.p)
                assert ns == nr
                recvbuf[ro:ro + nr].copy_(sh.send[q][so:so + ns])
        self._sync(recvbuf)
        sh.bar.wait()
        return None

    def finish(self, req):
        pass


def _setup(kind, ws):
    if kind == QUA8:
        m = structured_2d(QUA8, 12, 8, 4.0, 3.0)
        top = m.points_where(lambda x, y: np.abs(y - 3.0) < 1e-9)
        load_dof = 2 * top + 1
    else:
        m = structured_3d(HEX8, 6, 5, 4, 3.0, 2.5, 2.0)
        top = m.points_where(lambda x, y, z: np.abs(z - 2.0) < 1e-9)
        load_dof = 3 * top + 2
    nd = m.ndim
    fixed = np.zeros(m.ndof, dtype=bool)
    bottom = m.points_where(lambda *c: np.abs(c[-1]) < 1e-9)
    fixed[S.dof_index(bottom, nd)] = True
    f = np.zeros(m.ndof)
    f[load_dof] = -1.0 - 0.1 * m.coords[top, 0] ** 2
    shards = S.build_shards(m, S.node_owner(m, ws), ws)
    ranks = []
    for s in shards:
        loc = oracle.OracleElements(s.mesh, oracle.MODEL_LINEAR_ELASTIC, oracle.Params(1000.0, 0.3, 0.0, 1.0),
                                    sym_tol=-1.0)
        loc.initialize()
        lp, li, lv = loc.assemble_kk_csr()
        dof = S.dof_index(s.nodes, nd)
        n_own = s.n_owned * nd
        ranks.append(dict(shard=s, halo=S.Halo(s, nd), rows=S.owned_rows(lp, li, lv, n_own), dof=dof, n_own=n_own))
    # the whole system with the prescribed DOFs eliminated, solved directly
    g = oracle.OracleElements(m, oracle.MODEL_LINEAR_ELASTIC, oracle.Params(1000.0, 0.3, 0.0, 1.0), sym_tol=-1.0)
    g.initialize()
    gp, gi, gv = g.assemble_kk_csr()
    K = np.zeros((m.ndof, m.ndof))
    for r in range(m.ndof):
        K[r, gi[gp[r]:gp[r + 1]]] = gv[gp[r]:gp[r + 1]]
    free = ~fixed
    x = np.zeros(m.ndof)
    x[free] = np.linalg.solve(K[np.ix_(free, free)], f[free])
    return m, fixed, f, ranks, x


def _run(ranks, fixed, f, make, rtol=1e-13, cuda=True):
    comm = LocalComm([r["halo"] for r in ranks])
    out = [None] * len(ranks)
    errs = []

    def work(p):
        try:
            rk = ranks[p]
            import contextlib
            with torch.cuda.stream(torch.cuda.Stream()) if cuda else contextlib.nullcontext():
                op, oi, ov = rk["rows"]
                pcg = make(op, oi, rk["n_own"], len(rk["dof"]), fixed[rk["dof"]], rk["halo"], rk["shard"].mesh.ndim)
                pcg.set_values(ov)
                x, it = S.dist_cg(pcg, comm.rank(p), f[rk["dof"][:rk["n_own"]]], rtol=rtol)
                out[p] = (x.cpu().numpy().copy(), it)
        except Exception as e:  # noqa: BLE001 - reported below
            errs.append(e)
            comm.bar.abort()

    threads = [threading.Thread(target=work, args=(p,)) for p in range(len(ranks))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=120)
    assert not errs, errs
    return out


@pytest.mark.parametrize("kind,ws", [(QUA8, 2), (QUA8, 3), (HEX8, 2)])
def test_device_pcg_over_emulated_ranks(kind, ws):
    m, fixed, f, ranks, x_direct = _setup(kind, ws)
    dev = lambda *a: S.DevicePcg(*a, device="cuda:0")  # noqa: E731
    got = _run(ranks, fixed, f, dev)
    again = _run(ranks, fixed, f, dev)
    host = _run(ranks, fixed, f, HostPcg, cuda=False)
    scale = np.abs(x_direct).max()
    its = {it for _, it in got}
    assert len(its) == 1  # every rank stops at the same iteration (one reduced flag)
    for rk, (x, it), (x2, it2), (xh, ith) in zip(ranks, got, again, host):
        owned = rk["dof"][:rk["n_own"]]
        assert np.abs(x - x_direct[owned]).max() <= 1e-9 * scale
        assert np.array_equal(x, x2) and it == it2  # bit-identical repeat
        assert abs(it - ith) <= 1  # the same algorithm as the host stand-in
        assert np.abs(x - xh).max() <= 1e-10 * scale
    # the interior/boundary split is what the overlap relies on
    info = S.DevicePcg(*ranks[0]["rows"][:2], ranks[0]["n_own"], len(ranks[0]["dof"]), fixed[ranks[0]["dof"]],
                       ranks[0]["halo"], m.ndim, device="cuda:0").info()
    assert info["interior_rows"] > 0 and info["boundary_rows"] > 0
    assert info["interior_rows"] + info["boundary_rows"] == ranks[0]["n_own"]
