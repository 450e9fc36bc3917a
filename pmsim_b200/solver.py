"""Static implicit Newton solver over the B200 elements (mirror of pmsim's ``SolverImplicit``).

Sequencing follows ``SolverImplicit::solve`` / ``iterate`` (reference
``src/fem/solver_implicit.rs:56-272``): per step t += dt, dU = 0, lambda reset; per iteration
R = F_int - F_ext (+ Lagrange-multiplier rows, ``src/fem/bc_prescribed.rs:99-134``),
convergence on max|R| < tol_rr_abs, K, solve, convergence on rel(mdu) < tol_mdu_rel without
applying that last correction (``src/fem/convergence_control.rs:52-128``), U/dU update,
backup (iteration 0) / restore, stress update.

The element work of one iteration is a single fused library call
(``Elements.update_and_assemble``): the stress update of iteration k and the F_int / K
assembly of iteration k+1 happen in one pass over the cells.  The linear system is solved
on the host by a sparse direct LU (scipy SuperLU), which stands in for the reference's
UMFPACK call (``src/fem/linear_system.rs:185-201``).
"""
from __future__ import annotations

import time

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .elements import Elements


class NewtonError(RuntimeError):
    pass


class Essential:
    """Prescribed values keyed by equation (``src/base/essential.rs``); value = constant * f(t)."""

    def __init__(self):
        self.map = {}

    def set(self, eq, constant=0.0, fn=None):
        self.map[int(eq)] = (float(constant), fn)
        return self

    def points(self, point_ids, dof, ndim, constant=0.0, fn=None):
        for p in point_ids:
            self.set(ndim * int(p) + dof, constant, fn)
        return self

    @staticmethod
    def from_list(entries):
        e = Essential()
        for eq, c, fn in entries:
            e.set(eq, c, fn)
        return e

    def sorted(self):
        return sorted(self.map.items())


class SolverImplicit:
    def __init__(self, elements: Elements, essential, loads=(), lagrange_mult_method=True, n_max_iterations=10,
                 tol_rr_abs=1e-10, tol_mdu_rel=1e-8, t_ini=0.0, t_fin=1.0, ddt=1.0, verbose=False, natural=None,
                 constant_tangent=False):
        self.el = elements
        self.ndof = elements.ndof
        ess = essential if isinstance(essential, Essential) else Essential.from_list(essential)
        items = ess.sorted()
        self.eq_p = np.array([eq for eq, _ in items], dtype=np.int64)
        self.consts = np.array([c for _, (c, _) in items])
        self.fns = [fn for _, (_, fn) in items]
        self.loads = list(loads)
        self.lmm = lagrange_mult_method
        if not self.lmm and np.any(self.consts != 0.0):
            raise NewtonError("the Lagrange multiplier method is required for non-zero prescribed values")
        self.n_max_iterations = n_max_iterations
        self.tol_rr_abs, self.tol_mdu_rel = tol_rr_abs, tol_mdu_rel
        self.t_ini, self.t_fin, self.ddt = t_ini, t_fin, ddt
        self.np = len(items)
        self.neq_total = self.ndof + (self.np if self.lmm else 0)
        self.flags = np.zeros(self.ndof, dtype=bool)
        self.flags[self.eq_p] = True
        self.unknown = np.arange(self.neq_total) if self.lmm else np.nonzero(~self.flags)[0]
        self.indptr, self.indices = elements.csr_pattern()
        self.history = []
        self.timing = {"elements": 0.0, "solve": 0.0}
        self.verbose = verbose
        self.natural = natural  # object with ff_ext(t) -> F_ext over the DOFs (pmsim_b200.natural.Natural)
        # Config::constant_tangent (src/base/config.rs:38): K is assembled and factorised at the first
        # iteration of each step only (src/fem/solver_implicit.rs:216), later iterations reuse it
        self.constant_tangent = constant_tangent

    def _ff_ext(self, t):
        ffe = np.zeros(self.neq_total)
        for eq, v in self.loads:
            ffe[eq] += v
        if self.natural is not None:
            ffe[: self.ndof] += self.natural.ff_ext(t)
        if not self.lmm:
            ffe[: self.ndof][self.flags] = 0.0
        return ffe

    def _bc_values(self, t):
        return np.array([c * fn(t) if fn is not None else c for c, fn in zip(self.consts, self.fns)])

    def _factorize(self, kvals):
        kk = sp.csr_matrix((kvals, self.indices, self.indptr), shape=(self.ndof, self.ndof))
        if self.lmm:
            p = np.arange(self.np)
            a = sp.csr_matrix((np.ones(self.np), (p, self.eq_p)), shape=(self.np, self.ndof))
            kk = sp.bmat([[kk, a.T], [a, None]], format="csc")
        else:
            keep = sp.diags((~self.flags).astype(float))
            kk = (keep @ kk @ keep + sp.diags(self.flags.astype(float))).tocsc()
        return spla.splu(kk)

    def solve(self, on_step=None, on_iteration=None):
        """on_step(step, t, u, elements) after each load step; on_iteration(step, iteration) after each
        Newton iteration (a caller may raise there to stop the run)."""
        el = self.el
        u = np.zeros(self.neq_total)
        ddu = np.zeros(self.neq_total)
        ff = np.zeros(self.ndof)
        kv = np.zeros(el.nnz)
        t = self.t_ini
        el.initialize_internal_values()
        n_converged = 0
        while t + self.ddt <= self.t_fin:
            t += self.ddt
            ddu[:] = 0.0
            el.reset_algorithmic_variables()
            c = self._bc_values(t)
            ff_ext = self._ff_ext(t)
            hist = []
            t0 = time.perf_counter()
            el.assemble_f_int(ff)
            el.assemble_kk(kv)
            self.timing["elements"] += time.perf_counter() - t0
            mdu0 = None
            converged = False
            for it in range(self.n_max_iterations):
                rr = -ff_ext.copy()
                rr[: self.ndof] += np.where(self.flags, 0.0, ff) if not self.lmm else ff
                if self.lmm:
                    rr[self.eq_p] += u[self.ndof:]
                    rr[self.ndof:] = u[self.eq_p] - c
                norm_rr = float(np.max(np.abs(rr))) if rr.size else 0.0
                if not np.isfinite(norm_rr):
                    raise NewtonError("Found NaN or Inf")
                if norm_rr < self.tol_rr_abs:
                    hist.append((it, norm_rr, None))
                    converged = True
                    break
                t0 = time.perf_counter()
                if it == 0 or not self.constant_tangent:
                    lu = self._factorize(kv)
                mdu = lu.solve(rr)
                self.timing["solve"] += time.perf_counter() - t0
                if not np.all(np.isfinite(mdu)):
                    raise NewtonError("Found NaN or Inf in mdu")
                if it == 0:
                    mdu0 = mdu.copy()
                    rel = 1.0
                    conv = False
                else:
                    rel = float(np.max(np.abs(mdu) / (1.0 + np.abs(mdu0))))
                    conv = rel < self.tol_mdu_rel
                hist.append((it, norm_rr, rel))
                if self.verbose:
                    print(f"  t={t:g} it={it} max|R|={norm_rr:.3e} rel(mdu)={rel:.3e}")
                if conv:
                    converged = True
                    break
                u[self.unknown] -= mdu[self.unknown]
                ddu[self.unknown] -= mdu[self.unknown]
                if it == 0:
                    el.backup_secondary_values()
                t0 = time.perf_counter()
                el.update_and_assemble(ddu[: self.ndof], ff, None if self.constant_tangent else kv)
                self.timing["elements"] += time.perf_counter() - t0
                if on_iteration is not None:
                    on_iteration(len(self.history), it)
                if it == self.n_max_iterations - 1:
                    raise NewtonError("Newton-Raphson did not converge")
            if converged:
                n_converged += 1
            self.history.append(hist)
            if on_step is not None:
                on_step(len(self.history) - 1, t, u[: self.ndof].copy(), el)
            if t >= self.t_fin:
                break
        return n_converged
