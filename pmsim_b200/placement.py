"""Placement of independent problems on several GPUs: whole problems, no data exchange.

Problems of the batched and served configurations share nothing, so they go whole to one device
each; results do not depend on the placement (a problem's arithmetic is the same alone and in any
batch).  Two rules, both deterministic so that every process of a multi-GPU job computes the same
placement from the same list:

* ``least_loaded``: the device with the least device memory in use among those where the request
  still fits its budget (ties: the lowest device index) -- the serving loop's admission.
* ``partition``: the longest-processing-time rule on a work estimate -- each problem, largest first,
  goes to the part with the least work so far -- for splitting a batched population over ranks.
"""
from __future__ import annotations

import numpy as np


def least_loaded(nbytes: float, in_use, budgets):
    """Index of the device that takes a request of nbytes, or None when it fits nowhere now."""
    best = None
    for d, (u, b) in enumerate(zip(in_use, budgets)):
        if u + nbytes <= b and (best is None or u < in_use[best]):
            best = d
    return best


def work_estimate(problem) -> float:
    """Relative cost of solving a problem: the element work (IPs) and the PCG work (DOFs to the
    power 1.5, as the iteration count of a 2D/3D elliptic problem grows with its size), per step."""
    m = problem.mesh
    ng = problem.ngauss or {2: 9, 3: 8}[m.ndim]
    return float(problem.nsteps) * (m.ncell * ng + m.ndof ** 1.5 / 50.0)


def partition(problems, nparts: int, weight=work_estimate):
    """Longest-processing-time split: part index of every problem (a list of length len(problems))."""
    if nparts < 1:
        raise ValueError("nparts must be >= 1")
    w = np.array([weight(p) for p in problems], dtype=np.float64)
    order = sorted(range(len(problems)), key=lambda i: (-w[i], i))
    load = np.zeros(nparts)
    part = [0] * len(problems)
    for i in order:
        k = int(np.argmin(load))  # lowest index among equals
        part[i] = k
        load[k] += w[i]
    return part
