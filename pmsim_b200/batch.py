"""Batched static Newton solves on the device (many independent problems, one launch per iteration).

Each problem is a mesh, a material, prescribed values (``Essential``: equation -> constant * f(t)),
optional constant external forces, and a number of unit load steps (``set_incremental``,
reference ``src/base/config.rs:538-546``).  All problems are concatenated into one
``Elements`` handle (disjoint point and cell ranges, one material per problem) and solved together
by ``pms_batch_*`` (include/pms.h): per Newton iteration one element launch for all problems and
one batched FP64 block-Jacobi PCG, with the reference's Lagrange-multiplier iterates
(``src/fem/solver_implicit.rs:187-272``, ``src/fem/bc_prescribed.rs:99-134``).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .elements import Elements, Material
from .mesh import Mesh


@dataclass
class Problem:
    mesh: Mesh
    material: Material
    essential: list  # (local eq, constant, fn(t) or None)
    nsteps: int = 1
    ff_ext: np.ndarray | None = None
    ngauss: int = 0
    name: str = ""
    meta: dict = field(default_factory=dict)


class BatchSolver:
    def __init__(self, problems, tol_rr_abs=1e-10, tol_mdu_rel=1e-8, n_max_iterations=20, pcg_rtol=1e-12,
                 pcg_max_iterations=20000, constant_tangent=False):
        if not problems:
            raise ValueError("no problems")
        kinds = {p.mesh.kind for p in problems}
        if len(kinds) != 1:
            raise ValueError("one element kind per batch")
        ngs = {p.ngauss for p in problems}
        if len(ngs) != 1:
            raise ValueError("one integration rule per batch")
        self.L = _lib.load()
        self.problems = list(problems)
        nd = problems[0].mesh.ndim
        pts, cells, cmat, point_ptr, cell_ptr = [], [], [], [0], [0]
        for i, p in enumerate(problems):
            cells.append(p.mesh.cells + point_ptr[-1])
            pts.append(p.mesh.coords)
            cmat.append(np.full(p.mesh.ncell, i, np.int32))
            point_ptr.append(point_ptr[-1] + p.mesh.npoint)
            cell_ptr.append(cell_ptr[-1] + p.mesh.ncell)
        self.mesh = Mesh(nd, np.concatenate(pts), np.concatenate(cells), problems[0].mesh.kind)
        self.point_ptr = np.array(point_ptr, np.int64)
        self.cell_ptr = np.array(cell_ptr, np.int64)
        self.dof_ptr = self.point_ptr * nd
        self.elements = Elements(self.mesh, [p.material for p in problems], ngauss=problems[0].ngauss,
                                 cell_material=np.concatenate(cmat))
        # prescribed equations (map keyed by equation, later entries win), globally sorted
        pres = []
        for i, p in enumerate(problems):
            uniq = {}
            for eq, c, fn in p.essential:
                uniq[int(eq)] = (float(c), fn)
            for eq, (c, fn) in uniq.items():
                pres.append((int(self.dof_ptr[i]) + eq, i, c, fn))
        pres.sort(key=lambda x: x[0])
        self.pres_eq = np.array([x[0] for x in pres], np.int64)
        self.pres_prob = np.array([x[1] for x in pres], np.int32)
        self.pres_const = np.array([x[2] for x in pres])
        self.pres_fn = [x[3] for x in pres]
        ff_ext = None
        if any(p.ff_ext is not None for p in problems):
            ff_ext = np.zeros(self.mesh.ndof)
            for i, p in enumerate(problems):
                if p.ff_ext is not None:
                    ff_ext[self.dof_ptr[i]:self.dof_ptr[i + 1]] = p.ff_ext
        # constant_tangent: Config::constant_tangent (src/fem/solver_implicit.rs:216), K assembled only at the
        # first Newton iteration of each load step
        cfg = _lib.BatchConfig_(tol_rr_abs, tol_mdu_rel, n_max_iterations, pcg_rtol, pcg_max_iterations,
                                1 if constant_tangent else 0)
        h = ctypes.c_void_p()
        rc = self.L.pms_batch_create(self.elements.h, len(problems), _lib.ptr(self.point_ptr),
                                     _lib.ptr(self.cell_ptr), len(self.pres_eq), _lib.ptr(self.pres_eq),
                                     _lib.ptr(ff_ext), ctypes.byref(cfg), ctypes.byref(h))
        if rc != 0:
            raise _lib.PmsError(rc)
        self.h = h
        self.np = len(problems)
        self.t = np.zeros(self.np)
        self.step = np.zeros(self.np, np.int64)
        self.history = [[] for _ in problems]  # per problem: iterations per step
        self.pcg_history = [[] for _ in problems]

    def close(self):
        if getattr(self, "h", None):
            self.L.pms_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raw = self.L.pms_batch_last_error(self.h)
            raise _lib.PmsError(rc, raw.decode() if raw else None)

    def reset(self):
        self._check(self.L.pms_batch_reset(self.h))
        self.t[:] = 0.0
        self.step[:] = 0

    def c_values(self, t):
        """Prescribed values at each problem's time t[p] (constant * f(t))."""
        out = self.pres_const.copy()
        for k, fn in enumerate(self.pres_fn):
            if fn is not None:
                out[k] = self.pres_const[k] * fn(t[self.pres_prob[k]])
        return out

    def solve_step(self, active=None, device_loop=False):
        """Advance every active problem by one unit load step (t += 1) and solve it.

        device_loop: the whole Newton loop of the step runs on the device in one CUDA graph launch
        (pms_batch_solve_step_graph): the same results bit for bit, one host wait per load step."""
        act = np.ones(self.np, np.uint8) if active is None else np.ascontiguousarray(active, np.uint8)
        t_new = self.t + act
        c = self.c_values(t_new)
        iters = np.zeros(self.np, np.int32)
        norm = np.zeros(self.np)
        status = np.zeros(self.np, np.int32)
        pcg = np.zeros(self.np, np.int32)
        fn = self.L.pms_batch_solve_step_graph if device_loop else self.L.pms_batch_solve_step
        self._check(fn(self.h, _lib.ptr(c), _lib.ptr(act), _lib.ptr(iters), _lib.ptr(norm), _lib.ptr(status),
                       _lib.ptr(pcg)))
        self.t = t_new
        self.step += act
        for p in np.nonzero(act)[0]:
            self.history[p].append(int(iters[p]))
            self.pcg_history[p].append(int(pcg[p]))
        return iters, norm, status, pcg

    MESSAGES = {1: "Found NaN or Inf", 2: "Found NaN or Inf in mdu", 3: "Newton-Raphson did not converge",
                4: "von Mises plastic update must not lead to zero sigma_d (sigma_d < 1e-10)",
                5: "von Mises stiffness cannot be computed with zero deviatoric norm (norm_s < 1e-10)",
                6: "the determinant of the Jacobian must be positive"}

    def solve(self, on_step=None, on_fail="raise", device_loop=False):
        """Runs every problem through its load steps (problems with fewer steps drop out).

        on_fail="raise" stops at the first failing problem with the reference's message;
        on_fail="drop" removes failing problems and records them in ``self.failed``;
        device_loop: each load step's Newton loop runs on the device (one graph launch per step)."""
        self.reset()
        self.failed = {}
        nmax = max(p.nsteps for p in self.problems)
        for s in range(nmax):
            act = np.array([1 if (s < p.nsteps and i not in self.failed) else 0
                            for i, p in enumerate(self.problems)], np.uint8)
            if not act.any():
                break
            iters, norm, status, pcg = self.solve_step(act, device_loop=device_loop)
            for i in np.nonzero(status * act)[0]:
                msg = self.MESSAGES.get(int(status[i]), "error")
                if on_fail == "raise":
                    raise RuntimeError(f"problem {i}: {msg}")
                self.failed[int(i)] = (s, msg)
            if on_step is not None:
                on_step(s, self)

    def host_syncs(self):
        """Host waits for the device inside the Newton loops so far (pms_batch_host_syncs)."""
        return int(self.L.pms_batch_host_syncs(self.h))

    def tuning(self):
        t = _lib.BatchTuning_()
        self._check(self.L.pms_batch_get_tuning(self.h, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in t._fields_}

    def set_tuning(self, **kw):
        cur = self.tuning()
        cur.update(kw)
        t = _lib.BatchTuning_(**cur)
        self._check(self.L.pms_batch_set_tuning(self.h, ctypes.byref(t)))

    def autotune(self):
        """Times the PCG launch shapes on this batch (pms_batch_autotune) and keeps the fastest; the
        iterates do not depend on the choice.  Resets the batch."""
        t = _lib.BatchTuning_()
        self._check(self.L.pms_batch_autotune(self.h, ctypes.byref(t)))
        self.t[:] = 0.0
        self.step[:] = 0
        return {k: getattr(t, k) for k, _ in t._fields_}

    def tick(self, cmd):
        """One stage of the Newton iteration of every problem with cmd[p] != 0 (1: start its next
        load step, 2: continue).  Returns (result, iteration, norm_rr, pcg_iterations) per problem;
        result 2 means the problem's linear solve is still under way (send 2 again)."""
        cmd = np.ascontiguousarray(cmd, np.uint8)
        res = np.full(self.np, -1, np.int32)
        it = np.zeros(self.np, np.int32)
        norm = np.zeros(self.np)
        pcg = np.zeros(self.np, np.int32)
        c = self.c_values(self.t)
        self._check(self.L.pms_batch_tick(self.h, _lib.ptr(cmd), _lib.ptr(c), _lib.ptr(res), _lib.ptr(it),
                                          _lib.ptr(norm), _lib.ptr(pcg)))
        return res, it, norm, pcg

    def solve_independent(self, on_step=None, on_fail="drop", clock=None):
        """Every problem runs through its load steps at its own pace: each tick advances every running
        problem by one Newton iteration, and a problem that converges starts its next step at the next
        tick (no waiting for slower problems).  Records self.history / self.failed / self.finish."""
        import time as _time
        clock = clock or _time.perf_counter
        self.reset()
        self.failed, self.finish = {}, {}
        counts = np.zeros(self.np, np.int64)
        cmd = np.array([1 if p.nsteps > 0 else 0 for p in self.problems], np.uint8)
        self.t = cmd.astype(float)  # the first step's time
        self.step[:] = 0
        self.ticks = 0
        while cmd.any():
            res, it, norm, pcg = self.tick(cmd)
            self.ticks += 1
            for p in np.nonzero(cmd)[0]:
                r = int(res[p])
                if r == 2:  # linear solve still under way
                    continue
                counts[p] += 1
                if pcg[p]:
                    self.pcg_history[p].append(int(pcg[p]))
                if r == 0:
                    cmd[p] = 2
                elif r == 1:
                    self.history[p].append(int(counts[p]))
                    counts[p] = 0
                    self.step[p] += 1
                    if on_step is not None:
                        on_step(int(p), int(self.step[p]) - 1, self)
                    if self.step[p] < self.problems[p].nsteps:
                        self.t[p] += 1.0
                        cmd[p] = 1
                    else:
                        cmd[p] = 0
                        self.finish[int(p)] = clock()
                else:
                    msg = self.MESSAGES.get(r - 100, "error")
                    if on_fail == "raise":
                        raise RuntimeError(f"problem {p}: {msg}")
                    self.failed[int(p)] = (int(self.step[p]), msg)
                    cmd[p] = 0
                    self.finish[int(p)] = clock()

    def u(self):
        out = np.zeros(self.mesh.ndof)
        self._check(self.L.pms_batch_get_u(self.h, _lib.ptr(out)))
        return out

    def u_of(self, p, u=None):
        u = self.u() if u is None else u
        return u[self.dof_ptr[p]:self.dof_ptr[p + 1]]

    def state_of(self, p, state=None):
        sig, ivs, el = self.elements.get_state() if state is None else state
        ng = self.elements.ngauss
        a, b = self.cell_ptr[p] * ng, self.cell_ptr[p + 1] * ng
        return sig[a:b], ivs[a:b], el[a:b]
