"""Serving loop for solve requests: continuous batching of implicit Newton solves on one or more GPUs.

Requests arrive over time (e.g. a Poisson stream).  The server admits waiting requests while their
estimated device-memory footprint fits a device's budget and fewer than ``max_concurrent`` batches
are on that device; each request goes whole to the least-loaded device where it fits
(``placement.least_loaded``), and the requests admitted together on one device (per element kind)
become one device batch (``BatchSolver``: one element launch and one batched PCG per Newton
iteration, mesh/state/CSR resident on the device across Newton iterations and load steps).  Every
batch advances by ticks on its own CUDA stream and host thread, each request at its own load step
and iteration, so new batches start while earlier ones are still on the device and their work
overlaps; a batch releases its memory when its last request finishes.  Requests share nothing, so
there is no exchange between devices.  Latency = finish - arrival.
"""
from __future__ import annotations

import ctypes
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .batch import BatchSolver, Problem
from .placement import least_loaded


def footprint_bytes(problem: Problem) -> int:
    """Device bytes of a request: CSR values + indices, the per-cell assembly maps (slots and ranks),
    IP state (current + backup) and the solver vectors (from the CSR pattern built on the host)."""
    m = problem.mesh
    L = _lib.load()
    cm = _lib.Mesh_(m.ndim, m.kind, m.npoint, m.ncell, _lib.ptr(m.coords), _lib.ptr(m.cells), None)
    nnz = ctypes.c_int64()
    rc = L.pms_mesh_csr_pattern(ctypes.byref(cm), None, None, ctypes.byref(nnz))
    if rc != 0:
        raise _lib.PmsError(rc)
    nd, nn = m.ndim, m.nnode
    ng = problem.ngauss or 9
    nip = m.ncell * ng
    return int(nnz.value * 20 + m.ncell * nn * nn * 2 + m.ncell * nn * 4 + m.npoint * 12
               + nip * (2 * nd * 8 + 24) * 2 + m.ndof * 8 * 16 + m.ncell * nn * 12 + (64 << 20))


@dataclass
class Request:
    rid: int
    problem: Problem
    arrival: float
    admitted: float = -1.0
    finished: float = -1.0
    error: str | None = None
    u: np.ndarray | None = None
    bytes: int = 0
    meta: dict = field(default_factory=dict)


class Server:
    """``admit_window``: a waiting request is admitted once it has waited this long (seconds), together
    with everything that arrived since (one batch per element kind and device), so that bursts share a
    batch; ``devices`` lists the GPUs (each with ``budget_bytes``; None: the current device only);
    ``max_concurrent`` batches run at a time per device, each on its own stream and host thread;
    ``autotune`` picks each batch's PCG launch shapes (which change speed, never results)."""

    def __init__(self, budget_bytes=120e9, max_batch=256, max_concurrent=4, admit_window=0.1,
                 keep_results=False, autotune=True, devices=None, **solver_kw):
        self.devices = list(devices) if devices is not None else [None]
        self.budget = float(budget_bytes)
        self.max_batch = max_batch
        self.max_concurrent = max_concurrent
        self.admit_window = float(admit_window)
        self.autotune = autotune
        self.keep_results = keep_results
        self.solver_kw = solver_kw
        nd = len(self.devices)
        self.in_use_dev = [0.0] * nd
        self.live_dev = [0] * nd
        self.lock = threading.Lock()
        self.threads = []
        self.batches = 0
        self.batches_dev = [0] * nd
        self.peak_in_use = 0.0
        self.peak_concurrent = 0
        self.live = 0

    @property
    def in_use(self):
        return float(sum(self.in_use_dev))

    def _run_batch(self, reqs, t0, dev=0):
        try:
            if self.devices[dev] is not None:
                _lib.set_device(self.devices[dev])  # this thread's handles live on that device
            bs = BatchSolver([r.problem for r in reqs], **self.solver_kw)
            if self.autotune:
                bs.autotune()  # launch shapes only: the results do not depend on them
            clock = lambda: time.perf_counter() - t0  # noqa: E731
            bs.solve_independent(on_fail="drop", clock=clock)
            u = bs.u() if self.keep_results else None
            for i, r in enumerate(reqs):
                r.finished = bs.finish.get(i, clock())
                r.meta["newton"] = int(sum(bs.history[i]))
                r.meta["pcg"] = int(sum(bs.pcg_history[i]))
                r.meta["batch_size"] = len(reqs)
                if i in bs.failed:
                    r.error = bs.failed[i][1]
                if u is not None:
                    r.u = bs.u_of(i, u).copy()
                    r.meta["state"] = tuple(a.copy() for a in bs.state_of(i))
                    r.meta["history"] = list(bs.history[i])
            bs.close()
        except Exception as e:  # a failing batch fails its requests, not the server
            for r in reqs:
                r.error = f"batch error: {e}"
                r.finished = time.perf_counter() - t0
        finally:
            with self.lock:
                self.in_use_dev[dev] -= sum(r.bytes for r in reqs)
                self.live_dev[dev] -= 1
                self.live -= 1

    def serve(self, requests, realtime=True, poll=0.002):
        """Runs the stream to completion; returns the requests with admitted/finished times."""
        pending = sorted(requests, key=lambda r: r.arrival)
        for r in pending:
            r.bytes = footprint_bytes(r.problem)
            if r.bytes > self.budget:
                raise ValueError(f"request {r.rid} alone exceeds the memory budget")
        t0 = time.perf_counter()
        waiting = []
        k = 0
        while k < len(pending) or waiting:
            now = time.perf_counter() - t0
            while k < len(pending) and (pending[k].arrival <= now or not realtime):
                waiting.append(pending[k])
                k += 1
            # admit in arrival order: each request to the least-loaded device where it fits the budget,
            # grouped by element kind per device; devices already running max_concurrent batches take
            # no new batch, and their share of the arrivals waits for the next wave
            groups = {}
            with self.lock:
                keep = []
                # hold the wave until its oldest request has waited admit_window (or the stream ended)
                ready = bool(waiting) and (now - min(r.arrival for r in waiting) >= self.admit_window
                                           or k >= len(pending) or not realtime)
                open_dev = [self.live_dev[d] < self.max_concurrent for d in range(len(self.devices))]
                if not any(open_dev) or not ready:
                    keep, waiting = waiting, []
                budgets = [self.budget if open_dev[d] else -1.0 for d in range(len(self.devices))]
                for r in waiting:
                    kind = (r.problem.mesh.kind, r.problem.ngauss)
                    d = least_loaded(r.bytes, self.in_use_dev, budgets)
                    g = groups.setdefault((kind, d), []) if d is not None else None
                    if g is not None and len(g) < self.max_batch:
                        g.append(r)
                        self.in_use_dev[d] += r.bytes
                    else:
                        keep.append(r)
                waiting = keep
                self.peak_in_use = max(self.peak_in_use, self.in_use)
            for (kind, d), reqs in groups.items():
                if not reqs:
                    continue
                for r in reqs:
                    r.admitted = now
                    r.meta["device"] = d
                th = threading.Thread(target=self._run_batch, args=(reqs, t0, d), daemon=True)
                with self.lock:
                    self.live += 1
                    self.live_dev[d] += 1
                    self.peak_concurrent = max(self.peak_concurrent, self.live)
                th.start()
                self.threads.append(th)
                self.batches += 1
                self.batches_dev[d] += 1
            time.sleep(poll)
        for th in self.threads:
            th.join()
        return pending


def poisson_arrivals(n, rate, seed=11):
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def summarize(reqs):
    done = [r for r in reqs if r.error is None]
    lat = np.array([r.finished - r.arrival for r in done]) if done else np.array([np.nan])
    t_first = min(r.arrival for r in reqs)
    t_last = max(r.finished for r in reqs)
    return {"requests": len(reqs), "converged": len(done), "failed": len(reqs) - len(done),
            "seconds": t_last - t_first, "solves_per_s": len(done) / (t_last - t_first),
            "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
            "latency_mean_s": float(np.mean(lat))}
