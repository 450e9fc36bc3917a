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

    def fake_run(self, reqs, t0):
        kinds = {(r.problem.mesh.kind, r.problem.ngauss) for r in reqs}
        seen.append(kinds)
        with self.lock:
            usage.append(self.in_use)
        time.sleep(0.01)
        for r in reqs:
            r.finished = time.perf_counter() - t0
        with self.lock:
            self.in_use -= sum(r.bytes for r in reqs)
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
