"""Batched device Newton + PCG (pms_batch_*): parity with the golden runs and with the oracle driver,
and results independent of the batch composition (same bits alone and in the mix).

Reference: SolverImplicit::iterate (src/fem/solver_implicit.rs:187-272) with LMM prescribed values
(src/fem/bc_prescribed.rs:99-134); golden data as in test_gpu_solver.py.
"""
import numpy as np
import pytest

import oracle
import problems
from oracle.driver import OracleSolver
from pmsim_b200 import mesh as M

pytestmark = pytest.mark.gpu


def as_problem(pb):
    from pmsim_b200.batch import Problem
    from pmsim_b200.elements import Material
    return Problem(pb["mesh"], Material.von_mises(*pb["params"]), pb["essential"], nsteps=pb["nsteps"],
                   ngauss=pb["ngauss"])


def footing(nx, ny, E, z0, width, nsteps=10, seed=0):
    """The plane-strain strip footing of the small benchmark configuration: 10 m x 5 m, Qua8, 3x3
    Gauss, von Mises nu=0.3 H=0, bottom fixed, sides roller, top nodes with x <= width pressed
    down by 0.005 m per step."""
    from pmsim_b200.batch import Problem
    from pmsim_b200.elements import Material
    m = M.structured_2d(M.QUA8, nx, ny, 10.0, 5.0)
    tol = 1e-8
    ess = []
    for p in m.points_where(lambda x, y: np.abs(y) < tol):
        ess += [(2 * p, 0.0, None), (2 * p + 1, 0.0, None)]
    for p in m.points_where(lambda x, y: (np.abs(x) < tol) | (np.abs(x - 10.0) < tol)):
        ess += [(2 * p, 0.0, None)]
    for p in m.points_where(lambda x, y: (np.abs(y - 5.0) < tol) & (x <= width + tol)):
        ess += [(2 * p + 1, -0.005, lambda t: t)]
    return Problem(m, Material.von_mises(E, 0.3, 0.0, z0), ess, nsteps=nsteps, ngauss=9)


@pytest.mark.parametrize("name", ["single_element_2d", "2x2_elements_2d", "tensile_755"])
def test_batch_spo_golden(name):
    from pmsim_b200.batch import BatchSolver
    pb = problems.SPO_PROBLEMS[name]()
    bs = BatchSolver([as_problem(pb)], n_max_iterations=20)
    worst = [0.0, 0.0]

    def cb(step, b):
        sig = b.state_of(0)[0]
        du, ds = problems.compare_step(pb["golden"], step, b.u_of(0), sig, pb["ngauss"])
        worst[0] = max(worst[0], du)
        worst[1] = max(worst[1], ds)

    bs.solve(cb)
    assert worst[0] <= pb["tol_u"], worst
    assert worst[1] <= pb["tol_s"], worst
    m = pb["mesh"]
    oel = oracle.OracleElements(m, 1, oracle.Params(*pb["params"]), ngauss=pb["ngauss"], sym_tol=-1.0)
    osol = OracleSolver(oel, m.ndof, pb["essential"], n_max_iterations=20, t_fin=float(pb["nsteps"]))
    osol.solve()
    assert bs.history[0] == [len(h) for h in osol.history]


def test_batch_footing_matches_oracle_driver():
    """Small footing (the CPU-runnable configuration at reduced size) against the oracle driver:
    displacements, IP stresses and the Newton iteration count of every step."""
    from pmsim_b200.batch import BatchSolver
    pb = footing(8, 4, 1e4, 9.0, 1.0, nsteps=10)
    bs = BatchSolver([pb], n_max_iterations=20)
    got = []
    bs.solve(lambda s, b: got.append((b.u_of(0).copy(), b.state_of(0)[0].copy())))
    m = pb.mesh
    oel = oracle.OracleElements(m, 1, oracle.Params(1e4, 0.3, 0.0, 9.0), ngauss=9, sym_tol=-1.0)
    ref = []
    osol = OracleSolver(oel, m.ndof, pb.essential, n_max_iterations=20, t_fin=10.0)
    osol.solve(lambda step, t, u, el: ref.append((u.copy(), el.sig.copy())))
    assert bs.history[0] == [len(h) for h in osol.history]
    for (ug, sg), (uo, so) in zip(got, ref):
        assert np.max(np.abs(ug - uo)) <= 1e-9 * max(np.max(np.abs(uo)), 1e-30)
        assert np.max(np.abs(sg - so)) <= 1e-7 * np.max(np.abs(so))


def test_batch_results_do_not_depend_on_the_mix():
    from pmsim_b200.batch import BatchSolver
    rng = np.random.default_rng(5)
    probs = [footing(int(rng.integers(4, 10)), int(rng.integers(2, 6)), float(1e4 * np.exp(rng.normal(0, 0.5))),
                     float(rng.uniform(5, 20)), float(rng.uniform(0.5, 2.0)), nsteps=4) for _ in range(5)]
    mix = BatchSolver(probs)
    mix.solve()
    u_mix = mix.u()
    st_mix = mix.elements.get_state()
    for i, p in enumerate(probs):
        alone = BatchSolver([p])
        alone.solve()
        assert np.array_equal(alone.u(), mix.u_of(i, u_mix)), f"problem {i}: U differs alone vs in the mix"
        a = alone.elements.get_state()
        b = mix.state_of(i, st_mix)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
        assert alone.history[0] == mix.history[i]


def test_independent_progress_matches_lock_step():
    """Ticks (each problem at its own step) give the same bits as lock-step load steps."""
    from pmsim_b200.batch import BatchSolver
    rng = np.random.default_rng(11)
    probs = [footing(int(rng.integers(4, 10)), int(rng.integers(2, 6)), float(1e4 * np.exp(rng.normal(0, 0.5))),
                     float(rng.uniform(5, 20)), float(rng.uniform(0.5, 2.0)), nsteps=int(rng.integers(2, 5)))
             for _ in range(4)]
    a = BatchSolver(probs)
    a.solve()
    b = BatchSolver(probs)
    b.solve_independent(on_fail="raise")
    assert np.array_equal(a.u(), b.u())
    for x, y in zip(a.elements.get_state(), b.elements.get_state()):
        assert np.array_equal(x, y)
    assert a.history == b.history


def _solve_with(probs, setting):
    from pmsim_b200.batch import BatchSolver
    bs = BatchSolver(probs)
    if setting == "wide":
        bs.set_tuning(team_max_ndof=0)
    elif setting == "teams1":  # one 128-node chunk per CTA: clusters of 1..16 CTAs
        bs.set_tuning(team_max_ndof=10 ** 12, team_threads=256, team_chunks=1, pcg_budget=7)
    elif setting == "teams4":
        bs.set_tuning(team_max_ndof=10 ** 12, team_threads=1024, team_chunks=4, pcg_budget=33)
    elif setting == "mixed":
        nd = sorted(p.mesh.ndof for p in probs)
        bs.set_tuning(team_max_ndof=nd[len(nd) // 2], team_threads=512, team_chunks=0, graph_iters=2, pcg_budget=16)
    else:
        bs.autotune()
    bs.solve_independent(on_fail="drop")
    out = (bs.u(), bs.elements.get_state(), bs.history, bs.pcg_history, dict(bs.failed))
    bs.close()
    return out


def _assert_same(runs):
    (n0, (u0, st0, h0, pc0, f0)) = runs[0]
    for name, (u, st, h, pc, f) in runs[1:]:
        assert f == f0, name
        assert np.array_equal(u, u0), f"{name}: U differs from {n0}"
        for x, y in zip(st, st0):
            assert np.array_equal(x, y), name
        assert h == h0, name
        assert pc == pc0, name


def test_pcg_engines_give_the_same_bits():
    """The team engine (a thread-block cluster per problem, vectors in shared memory) and the
    batch-wide engine run the same arithmetic: forcing either one, any team shape, or letting the
    autotuner choose gives identical U, IP state and Newton/PCG iteration histories."""
    rng = np.random.default_rng(21)
    probs = [footing(int(rng.integers(4, 16)), int(rng.integers(2, 8)), float(1e4 * np.exp(rng.normal(0, 0.5))),
                     float(rng.uniform(5, 20)), float(rng.uniform(0.5, 2.0)), nsteps=3) for _ in range(6)]
    _assert_same([(s, _solve_with(probs, s)) for s in ("wide", "teams1", "teams4", "mixed", "auto")])


def test_pcg_sixteen_cta_team_matches_batch_wide():
    """A 64x32 footing (50 chunks) on a 16-CTA cluster (4 chunks per CTA, p read across CTAs
    through distributed shared memory) next to a small one: same bits as the batch-wide engine."""
    probs = [footing(64, 32, 1e4, 9.0, 1.0, nsteps=2), footing(6, 3, 2e4, 12.0, 1.5, nsteps=2)]
    _assert_same([(s, _solve_with(probs, s)) for s in ("wide", "teams4")])


def test_device_resident_newton_loop_gives_the_same_bits():
    """pms_batch_solve_step_graph: the Newton loop of each load step on the device (one CUDA graph
    launch: conditional WHILE over iterations with a nested WHILE over PCG iterations) against the
    host-sequenced lock-step solve: identical U, IP state, iteration counts and PCG counts, and one
    host wait per load step instead of several per iteration."""
    from pmsim_b200.batch import BatchSolver
    rng = np.random.default_rng(17)
    probs = [footing(int(rng.integers(4, 10)), int(rng.integers(2, 6)), float(1e4 * np.exp(rng.normal(0, 0.5))),
                     float(rng.uniform(5, 20)), float(rng.uniform(0.5, 2.0)), nsteps=int(rng.integers(2, 5)))
             for _ in range(6)]
    a = BatchSolver(probs)
    a.solve()
    b = BatchSolver(probs)
    b.solve(device_loop=True)
    assert np.array_equal(a.u(), b.u())
    for x, y in zip(a.elements.get_state(), b.elements.get_state()):
        assert np.array_equal(x, y)
    assert a.history == b.history
    assert a.pcg_history == b.pcg_history
    nsteps = max(p.nsteps for p in probs)
    newton = sum(sum(h) for h in b.history)
    assert b.host_syncs() == nsteps  # one wait per load step
    assert a.host_syncs() > newton   # several per Newton iteration when the host drives the loop
    # the golden SPO run through the device loop, with the oracle driver's iteration counts
    pb = problems.SPO_PROBLEMS["2x2_elements_2d"]()
    c = BatchSolver([as_problem(pb)], n_max_iterations=20)
    worst = [0.0, 0.0]

    def cb(step, bs):
        du, ds = problems.compare_step(pb["golden"], step, bs.u_of(0), bs.state_of(0)[0], pb["ngauss"])
        worst[0], worst[1] = max(worst[0], du), max(worst[1], ds)

    c.solve(cb, device_loop=True)
    assert worst[0] <= pb["tol_u"] and worst[1] <= pb["tol_s"], worst


def test_device_resident_loop_stops_failing_problems_alone():
    """Failures inside the device loop (a NaN prescribed value, a reflected cell) stop their problems
    with the same step and message as the host-sequenced solve; the others keep their bits."""
    from pmsim_b200.batch import BatchSolver
    from test_gpu_errors import _footing
    import error_cases as C
    good = [_footing(6, 3, 1e4, 9.0, 1.0, 3), _footing(5, 4, 1.5e4, 12.0, 1.5, 3)]
    bad_nan = _footing(6, 3, 1e4, 9.0, 1.0, 3, nan_from=2.0)
    bad_jac = _footing(6, 3, 1e4, 9.0, 1.0, 3)
    bad_jac.mesh = C.inverted(bad_jac.mesh, 7)
    mix = [good[0], bad_nan, good[1], bad_jac]
    a = BatchSolver(mix)
    a.solve(on_fail="drop")
    b = BatchSolver(mix)
    b.solve(on_fail="drop", device_loop=True)
    assert a.failed == b.failed and set(b.failed) == {1, 3}
    ua, ub = a.u(), b.u()
    for i in (0, 2):
        assert np.array_equal(a.u_of(i, ua), b.u_of(i, ub))
        assert a.history[i] == b.history[i]


@pytest.mark.parametrize("name", ["single_element_2d", "2x2_elements_2d"])
def test_batch_constant_tangent_matches_oracle(name):
    """Config::constant_tangent (src/fem/solver_implicit.rs:216) in the batched solver: K assembled
    (and the block-Jacobi preconditioner formed) at the first Newton iteration of each load step only,
    the later iterations updating the IP state and R (element-pass mode 3).  Host-sequenced and
    with the Newton loop on the device: the oracle driver's iteration counts (more than full
    Newton's) and displacements at every step, and the same bits on both paths."""
    from pmsim_b200.batch import BatchSolver
    pb = problems.SPO_PROBLEMS[name]()
    m = pb["mesh"]
    oel = oracle.OracleElements(m, 1, oracle.Params(*pb["params"]), ngauss=pb["ngauss"], sym_tol=-1.0)
    ref = []
    osol = OracleSolver(oel, m.ndof, pb["essential"], n_max_iterations=60, t_fin=float(pb["nsteps"]),
                        constant_tangent=True)
    osol.solve(lambda s, t, u, e: ref.append(u[:m.ndof].copy()))
    runs = {}
    for device_loop in (False, True):
        bs = BatchSolver([as_problem(pb)], n_max_iterations=60, constant_tangent=True)
        got = []
        bs.solve(lambda step, b: got.append(b.u_of(0).copy()), device_loop=device_loop)
        assert bs.history[0] == [len(h) for h in osol.history], (device_loop, bs.history[0])
        for ug, uo in zip(got, ref):
            assert np.max(np.abs(ug - uo)) <= 1e-9 * max(np.max(np.abs(uo)), 1e-300)
        runs[device_loop] = got
        bs.close()
    for a, b in zip(runs[False], runs[True]):
        assert np.array_equal(a, b)
    assert sum(len(h) for h in osol.history) > pb["nsteps"] * 2  # modified Newton takes extra iterations
