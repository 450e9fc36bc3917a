"""Restatement of pmsim's implicit Newton/time loop -- TEST INFRASTRUCTURE.

Follows ``SolverImplicit::solve`` / ``iterate`` (reference ``src/fem/solver_implicit.rs:56-272``),
``SolverData`` (``src/fem/solver_data.rs:85-152``), ``BcPrescribed`` LMM/RSM
(``src/fem/bc_prescribed.rs:99-157``), ``ConvergenceControl`` (``src/fem/convergence_control.rs:52-128``)
and ``TimeControl::update`` (``src/fem/time_control.rs:78-91``), static analysis only.

The direct solver the reference calls through FFI (UMFPACK, ``src/fem/linear_system.rs:185-201``)
is not available here; scipy's SuperLU factorises the same (augmented) system.  The
Lagrange-multiplier rows follow a deterministic (point, dof) order instead of the
reference's HashMap order (``src/base/essential.rs:22``); only their row order differs.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


class NewtonError(RuntimeError):
    pass


class OracleSolver:
    """Static implicit solver over an elements object exposing the ElementTrait-like calls.

    ``essential``: list of (eq, constant, multiplier_fn or None); value = constant*fn(t).
    ``loads``: list of (eq, value) concentrated loads (constant in time, scaled by ell=1).
    """

    def __init__(self, elements, ndof, essential, loads=(), lagrange_mult_method=True, n_max_iterations=10,
                 tol_rr_abs=1e-10, tol_mdu_rel=1e-8, t_ini=0.0, t_fin=1.0, ddt=1.0, constant_tangent=False,
                 linear_problem=False, ff_ext_fn=None):
        self.el = elements
        self.ndof = ndof
        # Essential is a map keyed by (point, dof) (src/base/essential.rs:22): a later entry
        # for the same equation replaces the earlier one.
        uniq = {}
        for e in essential:
            uniq[int(e[0])] = e
        ess = sorted(uniq.values(), key=lambda e: e[0])
        self.eq_p = np.array([e[0] for e in ess], dtype=np.int64)
        self.consts = [e[1] for e in ess]
        self.fns = [e[2] for e in ess]
        self.loads = list(loads)
        self.ff_ext_fn = ff_ext_fn  # t -> F_ext over the DOFs (distributed loads), or None
        self.lmm = lagrange_mult_method
        if not self.lmm and any(c != 0.0 for c in self.consts):
            raise NewtonError("the Lagrange multiplier method is required for non-zero prescribed values")
        self.n_max_iterations = n_max_iterations
        self.tol_rr_abs = tol_rr_abs
        self.tol_mdu_rel = tol_mdu_rel
        self.t_ini, self.t_fin, self.ddt = t_ini, t_fin, ddt
        self.constant_tangent = constant_tangent
        self.linear_problem = linear_problem
        self.np = len(ess)
        self.neq_total = ndof + (self.np if self.lmm else 0)
        self.flags = np.zeros(ndof, dtype=bool)
        self.flags[self.eq_p] = True
        if self.lmm:
            self.unknown = np.arange(self.neq_total)
        else:
            self.unknown = np.nonzero(~self.flags)[0]
        self.history = []  # per step: list of (iteration, norm_rr, rel_mdu)

    def bc_value(self, p, t):
        f = self.fns[p]
        return self.consts[p] * f(t) if f is not None else self.consts[p]

    def _ff_ext(self, t):
        ff = np.zeros(self.neq_total)
        for eq, v in self.loads:
            ff[eq] += v
        if self.ff_ext_fn is not None:
            ff[: self.ndof] += self.ff_ext_fn(t)
        return ff

    def solve(self, on_step=None):
        el = self.el
        u = np.zeros(self.neq_total)
        ddu = np.zeros(self.neq_total)
        t = self.t_ini
        el.initialize()
        n_converged = 0
        for timestep in range(10 ** 9):
            if t + self.ddt > self.t_fin:
                break
            t += self.ddt
            ddu[:] = 0.0
            ell = 1.0
            if not self.linear_problem:
                el.reset_algorithmic_variables()
            hist = []
            converged = False
            mdu0 = None
            lu = None
            for it in range(self.n_max_iterations):
                # 1) F_int, F_ext; R = F_int - ell F_ext (+ LMM rows)
                rr = np.zeros(self.neq_total)
                fi = el.assemble_f_int()
                if self.lmm:
                    rr[: self.ndof] = fi
                else:
                    rr[: self.ndof] = np.where(self.flags, 0.0, fi)
                ffe = self._ff_ext(t)
                if not self.lmm:
                    ffe[: self.ndof][self.flags] = 0.0
                rr -= ell * ffe
                if self.lmm:
                    for p in range(self.np):
                        i = self.eq_p[p]
                        j = self.ndof + p
                        rr[i] += u[j]
                        rr[j] = u[i] - self.bc_value(p, t)
                norm_rr = float(np.max(np.abs(rr))) if rr.size else 0.0
                if not np.isfinite(norm_rr):
                    raise NewtonError("Found NaN or Inf")
                if norm_rr < self.tol_rr_abs:
                    hist.append((it, norm_rr, None))
                    converged = True
                    break
                # 2) K (only at it==0 if constant tangent)
                if it == 0 or not self.constant_tangent:
                    indptr, indices, data = el.assemble_kk_csr()
                    kk = sp.csr_matrix((data, indices, indptr), shape=(self.ndof, self.ndof))
                    if self.lmm:
                        p = np.arange(self.np)
                        a = sp.csr_matrix((np.ones(self.np), (p, self.eq_p)), shape=(self.np, self.ndof))
                        kk = sp.bmat([[kk, a.T], [a, None]], format="csc")
                    else:
                        keep = (~self.flags).astype(float)
                        dk = sp.diags(keep)
                        kk = (dk @ kk @ dk + sp.diags(self.flags.astype(float))).tocsc()
                    lu = spla.splu(kk)
                mdu = lu.solve(rr)
                norm_mdu = float(np.max(np.abs(mdu)))
                if not np.isfinite(norm_mdu):
                    raise NewtonError("Found NaN or Inf in mdu")
                if it == 0:
                    mdu0 = mdu.copy()
                    rel = 1.0
                    conv_mdu = False
                else:
                    rel = float(np.max(np.abs(mdu) / (1.0 + np.abs(mdu0))))
                    conv_mdu = rel < self.tol_mdu_rel
                hist.append((it, norm_rr, rel))
                if conv_mdu:
                    converged = True
                    break
                # 3) U, dU update on unknown equations
                u[self.unknown] -= mdu[self.unknown]
                ddu[self.unknown] -= mdu[self.unknown]
                # 4) backup / restore, then stress update from the step-start state
                if not self.linear_problem:
                    if it == 0:
                        el.backup_secondary_values()
                    else:
                        el.restore_secondary_values()
                el.update_secondary_values(ddu[: self.ndof])
                if self.linear_problem:
                    converged = True
                    break
                if it == self.n_max_iterations - 1:
                    raise NewtonError("Newton-Raphson did not converge")
            if converged:
                n_converged += 1
            self.history.append(hist)
            if on_step is not None:
                on_step(timestep, t, u[: self.ndof].copy(), el)
            if t >= self.t_fin:
                break
        return n_converged
