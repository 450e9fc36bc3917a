"""One problem sharded over ranks (pmsim_b200/shard.py), on the CPU: the owner-computes partition
gives every rank complete rows of K and R (checked against the whole-mesh assembly, with the oracle
standing in for the element calls), the halo lists of both sides agree, and the distributed CG over
two gloo ranks reproduces the single-process solution."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle
from pcg_host import HostPcg
from pmsim_b200 import shard as S
from pmsim_b200.mesh import HEX8, QUA4, QUA8, structured_2d, structured_3d

E, NU, H, Z0 = 1e4, 0.3, 500.0, 9.0


def _mesh(kind):
    m = structured_3d(HEX8, 3, 2, 4, 1.0, 1.0, 2.0) if kind == HEX8 else structured_2d(kind, 6, 4, 3.0, 2.0)
    rng = np.random.default_rng(kind)
    inner = np.all((m.coords > 1e-9) & (m.coords < m.coords.max(axis=0) - 1e-9), axis=1)
    m.coords[inner] += rng.uniform(-0.05, 0.05, (inner.sum(), m.ndim))
    return m


def _plastic_ddu(m, seed):
    rng = np.random.default_rng(seed)
    x = m.coords
    u = np.zeros((m.npoint, m.ndim))
    u[:, -1] = -0.004 * x[:, -1] * (1.0 + np.sin(2.0 * x[:, 0]))
    u += rng.normal(0.0, 2e-4, u.shape)
    return u.reshape(-1)


@pytest.mark.parametrize("kind,nparts", [(QUA8, 2), (QUA8, 3), (QUA4, 4), (HEX8, 2), (HEX8, 3)])
def test_owned_rows_equal_the_whole_mesh_rows(kind, nparts):
    m = _mesh(kind)
    nd = m.ndim
    owner = S.node_owner(m, nparts)
    shards = S.build_shards(m, owner, nparts)
    assert np.array_equal(np.sort(np.concatenate([s.nodes[:s.n_owned] for s in shards])), np.arange(m.npoint))
    prm = oracle.Params(E, NU, H, Z0)
    ddu = _plastic_ddu(m, kind + nparts)
    glob = oracle.OracleElements(m, oracle.MODEL_VON_MISES, prm, sym_tol=-1.0)
    glob.initialize()
    glob.update_secondary_values(ddu)
    assert glob.elastic.min() == 0  # plastic IPs present
    gp, gi, gv = glob.assemble_kk_csr()
    gf = glob.assemble_f_int()
    for s in shards:
        # every cell touching an owned node is computed here
        touch = np.flatnonzero(np.any(owner[m.cells] == s.part, axis=1))
        assert np.array_equal(touch, s.cells)
        loc = oracle.OracleElements(s.mesh, oracle.MODEL_VON_MISES, prm, sym_tol=-1.0)
        loc.initialize()
        loc.update_secondary_values(ddu.reshape(-1, nd)[s.nodes].reshape(-1))
        lp, li, lv = loc.assemble_kk_csr()
        lf = loc.assemble_f_int()
        dof_g = S.dof_index(s.nodes, nd)  # local DOF -> global DOF
        n_own = s.n_owned * nd
        np.testing.assert_allclose(lf[:n_own], gf[dof_g[:n_own]], rtol=0, atol=1e-12 * np.abs(gf).max())
        op, oi, ov = S.owned_rows(lp, li, lv, n_own)
        scale = np.abs(gv).max()
        for r in range(n_own):
            g = dof_g[r]
            want = dict(zip(gi[gp[g]:gp[g + 1]], gv[gp[g]:gp[g + 1]]))
            got = dict(zip(dof_g[oi[op[r]:op[r + 1]]], ov[op[r]:op[r + 1]]))
            assert set(got) == set(want), (s.part, r)
            assert max(abs(got[c] - want[c]) for c in want) <= 1e-13 * scale
    # halo lists: rank p receives from q exactly what q sends to p, in the same order
    for p in shards:
        for q, pos in p.recv.items():
            assert np.array_equal(p.nodes[pos], shards[q].nodes[shards[q].send[p.part]])
            assert np.all(owner[p.nodes[pos]] == q)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _problem():
    """Linear elastic Qua4 plate 8x6, bottom fixed, a parabolic downward load on the top nodes."""
    m = structured_2d(QUA4, 8, 6, 4.0, 3.0)
    fixed = np.zeros(m.ndof, dtype=bool)
    bottom = m.points_where(lambda x, y: np.abs(y) < 1e-9)
    fixed[S.dof_index(bottom, 2)] = True
    f = np.zeros(m.ndof)
    top = m.points_where(lambda x, y: np.abs(y - 3.0) < 1e-9)
    f[2 * top + 1] = -1.0 - 0.1 * m.coords[top, 0] ** 2
    return m, fixed, f


def _cg_rank(rank, ws, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(ws),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    import torch
    from pmsim_b200 import dist
    dist.init("gloo", timeout_s=60)
    torch.set_num_threads(1)  # two ranks share the cores
    try:
        m, fixed, f = _problem()
        shards = S.build_shards(m, S.node_owner(m, ws), ws)
        s = shards[rank]
        loc = oracle.OracleElements(s.mesh, oracle.MODEL_LINEAR_ELASTIC, oracle.Params(E, NU, 0.0, 1.0), sym_tol=-1.0)
        loc.initialize()
        lp, li, lv = loc.assemble_kk_csr()
        dof = S.dof_index(s.nodes, 2)
        n_own = s.n_owned * 2
        op, oi, ov = S.owned_rows(lp, li, lv, n_own)
        halo = S.Halo(s, 2)
        # the halo exchange returns the owners' values
        xg = np.arange(m.ndof, dtype=np.float64) * 0.5 + 1.0
        xl = torch.zeros(len(dof), dtype=torch.float64)
        xl[:n_own] = torch.as_tensor(xg[dof[:n_own]])
        halo.exchange(xl)
        halo_ok = bool(np.array_equal(xl.numpy(), xg[dof]))
        # packed exchange (the order DevicePcg's pack/unpack use) gives the same ghost values
        sb = torch.as_tensor(xl.numpy()[halo.send_dofs])
        rb = torch.zeros(len(halo.recv_dofs), dtype=torch.float64)
        halo.finish(halo.post(sb, rb))
        halo_ok = halo_ok and bool(np.array_equal(rb.numpy(), xg[dof][halo.recv_dofs]))
        pcg = HostPcg(op, oi, n_own, len(dof), fixed[dof], halo, 2)
        pcg.set_values(ov)
        x, it = S.dist_cg(pcg, S.TorchComm(halo), f[dof[:n_own]], rtol=1e-13)
        q.put((rank, halo_ok, it, dof[:n_own], x.numpy()))
    finally:
        dist.finalize()


@pytest.mark.timeout(180)
@pytest.mark.parametrize("ws", [2, 3])
def test_distributed_cg_over_gloo_ranks(ws):
    """Two ranks (one neighbour each) and three (the middle rank exchanges with two)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_cg_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    out = [q.get(timeout=150) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    # the single-process solution (oracle K, prescribed DOFs eliminated)
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    m, fixed, f = _problem()
    el = oracle.OracleElements(m, oracle.MODEL_LINEAR_ELASTIC, oracle.Params(E, NU, 0.0, 1.0), sym_tol=-1.0)
    el.initialize()
    gp, gi, gv = el.assemble_kk_csr()
    K = sp.csr_matrix((gv, gi, gp), shape=(m.ndof, m.ndof)).tocsc()
    free = ~fixed
    u = np.zeros(m.ndof)
    u[free] = spla.spsolve(K[free][:, free], f[free])
    got = np.zeros(m.ndof)
    seen = np.zeros(m.ndof, dtype=bool)
    iters = set()
    for rank, halo_ok, it, dofs, x in out:
        assert halo_ok, rank
        got[dofs] = x
        seen[dofs] = True
        iters.add(it)
    assert seen.all()
    assert len(iters) == 1  # every rank takes the same number of iterations (the reductions are global)
    np.testing.assert_allclose(got, u, rtol=0, atol=1e-9 * np.abs(u).max())


class _DeviceStyle:
    """The oracle behind the call names of the device ``Elements`` (initialize_internal_values,
    csr_pattern + assemble_kk), so the driver's other branch runs too."""

    def __init__(self, el):
        self.el = el

    def initialize_internal_values(self):
        self.el.initialize()

    def reset_algorithmic_variables(self):
        self.el.reset_algorithmic_variables()

    def backup_secondary_values(self):
        self.el.backup_secondary_values()

    def restore_secondary_values(self):
        self.el.restore_secondary_values()

    def update_secondary_values(self, ddu):
        self.el.update_secondary_values(ddu)

    def assemble_f_int(self):
        return self.el.assemble_f_int()

    def csr_pattern(self):
        ip, ix, _ = self.el.assemble_kk_csr()
        return ip, ix.astype(np.int32)  # the device pattern's column type

    def assemble_kk(self):
        return self.el.assemble_kk_csr()[2]

    @property
    def sig(self):
        return self.el.sig


def _newton_rank(rank, ws, port, q):
    import torch
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(ws),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    import problems
    from pmsim_b200 import dist
    dist.init("gloo", timeout_s=120)
    torch.set_num_threads(1)  # two ranks share the cores
    try:
        pb = problems.pres_cylin_751()
        m = pb["mesh"]
        fixed = np.zeros(m.ndof, dtype=bool)
        fixed[[e[0] for e in pb["essential"]]] = True
        s = S.build_shards(m, S.node_owner(m, ws), ws)[rank]
        dof = S.dof_index(s.nodes, 2)
        n_own = s.n_owned * 2
        el = oracle.OracleElements(s.mesh, oracle.MODEL_VON_MISES, oracle.Params(*pb["params"]), ngauss=4,
                                   sym_tol=-1.0)
        if rank == 1:
            el = _DeviceStyle(el)
        steps = []
        hist, u = S.dist_newton(s, 2, el, fixed[dof], lambda t: pb["natural"].ff_ext(t)[dof[:n_own]], pb["nsteps"],
                                tol_mdu_rel=1e-10, pcg_factory=HostPcg,
                                on_step=lambda k, t, u, e: steps.append((u.copy(), e.sig.copy())))
        q.put((rank, [len(h) for h in hist], dof[:n_own], s.cells, steps))
    finally:
        dist.finalize()


@pytest.mark.timeout(240)
def test_sharded_newton_replays_spo_751_over_two_gloo_ranks():
    """The reference's Newton loop over two ranks (owner-computes rows, dU halo exchange,
    distributed CG) on the SPO 7.5.1 pressurised cylinder (von Mises, reduced-system method,
    internal pressure): every step's displacements and IP stresses at the tolerances of the
    single-process replay, and pmsim's own logged Newton iteration counts.  Rank 1 drives its
    elements through the device call names."""
    import problems
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_newton_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=200) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    pb = problems.pres_cylin_751()
    m = pb["mesh"]
    g = pb["golden"]
    for rank, iters, dofs, cells, steps in out:
        assert iters == pb["iterations"], (rank, iters)
        for k, (u, sig) in enumerate(steps):
            gu = g["displacement"][k].reshape(-1)
            assert np.max(np.abs(u - gu[dofs])) <= pb["tol_u"], (rank, k)
            gs = np.array(g["stresses"][k], dtype=float)[cells]
            gs[..., 3:] *= np.sqrt(2.0)
            assert np.max(np.abs(sig.reshape(gs.shape) - gs)) <= pb["tol_s"], (rank, k)


def _footing_rank(rank, ws, port, q):
    import torch
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(ws),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    from pmsim_b200 import dist
    from pmsim_b200.footing import footing_problem
    dist.init("gloo", timeout_s=120)
    torch.set_num_threads(1)  # two ranks share the cores
    try:
        p = footing_problem(20, 10, 1e4, 9.0, 1.0, nsteps=10)
        m = p.mesh
        ess = {int(e[0]): e for e in p.essential}  # a later entry for the same equation wins
        fixed = np.zeros(m.ndof, dtype=bool)
        fixed[list(ess)] = True

        def values(t):
            c = np.zeros(m.ndof)
            for eq, (_, const, fn) in ess.items():
                c[eq] = const * fn(t) if fn is not None else const
            return c

        s = S.build_shards(m, S.node_owner(m, ws), ws)[rank]
        dof = S.dof_index(s.nodes, 2)
        n_own = s.n_owned * 2
        mt = p.material
        el = oracle.OracleElements(s.mesh, oracle.MODEL_VON_MISES, oracle.Params(mt.young, mt.poisson, mt.hh, mt.z_ini),
                                   ngauss=9, sym_tol=-1.0)
        steps = []
        hist, _ = S.dist_newton(s, 2, el, fixed[dof], lambda t: np.zeros(n_own), 10, n_max_iterations=20,
                                prescribed_local=lambda t: values(t)[dof], pcg_factory=HostPcg,
                                on_step=lambda k, t, u, e: steps.append(u.copy()))
        q.put((rank, [len(h) for h in hist], dof[:n_own], steps))
    finally:
        dist.finalize()


@pytest.mark.timeout(300)
def test_sharded_newton_with_multipliers_replays_the_footing():
    """Lagrange multipliers over two ranks: the 20x10 Qua8 footing (9 IP, von Mises, prescribed
    indentation, the reference's CPU-runnable configuration) takes the single-process oracle's Newton
    counts at every step (7,7,6,6,6,7,7,5,5,5) and its displacements within 1e-9 of the largest."""
    from oracle.driver import OracleSolver
    from pmsim_b200.footing import footing_problem
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_footing_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=280) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    p = footing_problem(20, 10, 1e4, 9.0, 1.0, nsteps=10)
    mt = p.material
    oel = oracle.OracleElements(p.mesh, oracle.MODEL_VON_MISES, oracle.Params(mt.young, mt.poisson, mt.hh, mt.z_ini),
                                ngauss=9, sym_tol=-1.0)
    ref = []
    osol = OracleSolver(oel, p.mesh.ndof, p.essential, n_max_iterations=20, t_fin=10.0)
    osol.solve(lambda k, t, u, e: ref.append(u.copy()))
    want = [len(h) for h in osol.history]
    assert want == [7, 7, 6, 6, 6, 7, 7, 5, 5, 5]
    for rank, iters, dofs, steps in out:
        assert iters == want, (rank, iters)
        for k, u in enumerate(steps):
            assert np.max(np.abs(u - ref[k][dofs])) <= 1e-9 * np.abs(ref[k]).max(), (rank, k)
