"""Host logic of the serving loop without a GPU: admission under the memory budget, grouping by
element kind, completion of every request (batches replaced by a timed stand-in)."""
import threading
import time

import numpy as np

from pmsim_b200 import serve
from pmsim_b200.batch import Problem
from pmsim_b200.elements import Material
from pmsim_b200.mesh import structured_2d, structured_3d, QUA8, HEX8


def fake_problem(kind, n):
    m = structured_2d(QUA8, n, n) if kind == "q" else structured_3d(HEX8, n, n, n)
    return Problem(m, Material.von_mises(1e4, 0.3, 0.0, 9.0), [], nsteps=1, ngauss=9 if kind == "q" else 8)


def test_admission_budget_and_grouping(monkeypatch):
    probs = [fake_problem("q" if i % 3 else "h", 4 + i % 5) for i in range(24)]
    sizes = [serve.footprint_bytes(p) for p in probs]
    budget = 3.2 * max(sizes)
    seen = []
    usage = []

    def fake_run(self, reqs, t0, dev=0):
        kinds = {(r.problem.mesh.kind, r.problem.ngauss) for r in reqs}
        seen.append(kinds)
        with self.lock:
            usage.append(self.in_use)
        time.sleep(0.01)
        for r in reqs:
            r.finished = time.perf_counter() - t0
        with self.lock:
            self.in_use_dev[dev] -= sum(r.bytes for r in reqs)
            self.live_dev[dev] -= 1
            self.live -= 1

    monkeypatch.setattr(serve.Server, "_run_batch", fake_run)
    arr = serve.poisson_arrivals(len(probs), rate=500.0, seed=1)
    reqs = [serve.Request(i, p, float(a)) for i, (p, a) in enumerate(zip(probs, arr))]
    srv = serve.Server(budget_bytes=budget)
    srv.serve(reqs)
    assert all(r.finished > 0 and r.admitted >= r.arrival - 1e-9 for r in reqs)
    assert all(len(k) == 1 for k in seen)  # one element kind per batch
    assert max(usage) <= budget
    assert srv.peak_in_use <= budget
    s = serve.summarize(reqs)
    assert s["converged"] == len(reqs) and s["latency_p99_s"] >= s["latency_p50_s"]


def test_request_population_matches_the_served_configuration():
    from pmsim_b200.footing import request_population
    ps = request_population(200, seed=7, nsteps=10)
    kinds = np.array([p.mesh.kind for p in ps])
    frac_q = float(np.mean(kinds == QUA8))
    assert 0.6 < frac_q < 0.8
    for p in ps:
        if p.mesh.kind == QUA8:
            assert 700 <= p.mesh.ndof <= 60000
        else:
            assert p.mesh.ndof <= 206763
        assert p.nsteps == 10


def test_requests_go_whole_to_the_least_loaded_device(monkeypatch):
    """Several devices (stand-ins: the batch runner is replaced, no GPU is touched): every request goes
    whole to one device, no device ever holds more than its budget, the devices share the work, and
    the placement rule picks the least-loaded device that fits."""
    from pmsim_b200 import placement
    probs = [fake_problem("q" if i % 3 else "h", 4 + i % 7) for i in range(60)]
    sizes = [serve.footprint_bytes(p) for p in probs]
    budget = 2.5 * max(sizes)
    log = []

    def fake_run(self, reqs, t0, dev=0):
        with self.lock:
            log.append((dev, list(self.in_use_dev)))
        time.sleep(0.005 * len(reqs))
        for r in reqs:
            r.finished = time.perf_counter() - t0
        with self.lock:
            self.in_use_dev[dev] -= sum(r.bytes for r in reqs)
            self.live_dev[dev] -= 1
            self.live -= 1

    monkeypatch.setattr(serve.Server, "_run_batch", fake_run)
    arr = serve.poisson_arrivals(len(probs), rate=2000.0, seed=3)
    reqs = [serve.Request(i, p, float(a)) for i, (p, a) in enumerate(zip(probs, arr))]
    srv = serve.Server(budget_bytes=budget, devices=[0, 1, 2], max_concurrent=2, admit_window=0.002)
    srv.serve(reqs)
    assert all(r.finished > 0 for r in reqs)
    assert all(r.meta["device"] in (0, 1, 2) for r in reqs)
    for dev, use in log:
        assert all(u <= budget + 1e-6 for u in use)
    assert all(n > 0 for n in srv.batches_dev), srv.batches_dev
    assert srv.in_use == 0.0 and srv.live == 0
    assert placement.least_loaded(5.0, [3.0, 1.0, 2.0], [10.0, 10.0, 10.0]) == 1
    assert placement.least_loaded(5.0, [3.0, 6.0, 2.0], [10.0, 10.0, 6.0]) == 0
    assert placement.least_loaded(5.0, [6.0, 6.0], [10.0, 10.0]) is None


def test_partition_balances_work_and_is_deterministic():
    from pmsim_b200 import placement
    from pmsim_b200.footing import population
    probs = population(64, seed=2024)
    parts = placement.partition(probs, 4)
    assert parts == placement.partition(probs, 4)
    assert sorted(set(parts)) == [0, 1, 2, 3]
    w = np.array([placement.work_estimate(p) for p in probs])
    load = np.array([w[np.array(parts) == k].sum() for k in range(4)])
    assert load.max() <= 1.15 * load.mean()
    assert placement.partition(probs, 1) == [0] * len(probs)
