"""Served path: continuous batching of solve requests (Poisson stream, memory-budget admission).

Each request's result must be the same alone and in the mix: the device solver's per-problem
arithmetic does not depend on the batch it shares or on when it was admitted.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def small_stream(n=8, seed=3):
    from pmsim_b200.footing import block_problem, footing_problem
    rng = np.random.default_rng(seed)
    probs = []
    for i in range(n):
        E = float(1e4 * np.exp(rng.normal(0, 0.5)))
        z0 = float(rng.uniform(5, 20))
        if i % 3 == 2:
            probs.append(block_problem(int(rng.integers(3, 6)), int(rng.integers(3, 6)), int(rng.integers(3, 6)),
                                       E, z0, nsteps=3))
        else:
            probs.append(footing_problem(int(rng.integers(6, 12)), int(rng.integers(3, 6)), E, z0,
                                         float(rng.uniform(0.5, 2)), nsteps=3))
    return probs


def test_serve_results_same_alone_and_in_mix():
    from pmsim_b200.batch import BatchSolver
    from pmsim_b200.serve import Request, Server, poisson_arrivals
    probs = small_stream()
    arr = poisson_arrivals(len(probs), rate=200.0, seed=5)
    reqs = [Request(i, p, float(a)) for i, (p, a) in enumerate(zip(probs, arr))]
    srv = Server(budget_bytes=4e9, keep_results=True)
    srv.serve(reqs)
    assert all(r.finished >= r.arrival for r in reqs)
    assert srv.batches >= 2  # arrivals spread over time -> several admission waves
    for r in reqs:
        alone = BatchSolver([r.problem])
        alone.solve_independent(on_fail="drop")
        if r.error is not None:
            assert 0 in alone.failed, f"request {r.rid} failed in the mix ({r.error}) but not alone"
            continue
        assert not alone.failed, f"request {r.rid} failed alone ({alone.failed}) but not in the mix"
        assert np.array_equal(alone.u(), r.u), f"request {r.rid}: U differs alone vs in the mix"
        for x, y in zip(alone.elements.get_state(), r.meta["state"]):
            assert np.array_equal(x, y)
        assert alone.history[0] == r.meta["history"]


def test_serve_respects_memory_budget():
    from pmsim_b200.serve import Request, Server, footprint_bytes
    probs = small_stream(6, seed=9)
    budget = 1.5 * max(footprint_bytes(p) for p in probs)
    reqs = [Request(i, p, 0.0) for i, p in enumerate(probs)]
    srv = Server(budget_bytes=budget)
    srv.serve(reqs)
    assert srv.peak_in_use <= budget
    assert all(r.finished > 0 for r in reqs)
