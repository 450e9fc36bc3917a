"""Times the PCG engines of the batched solver on one problem (pms_batch_time_pcg).

    python -m pmsim_b200.pcg_time team foot 20 10            # team engine, 20x10 Qua8 footing
    python -m pmsim_b200.pcg_time team foot 20 10 --chunks 1 # one 128-node chunk per CTA (8 CTAs)
    python -m pmsim_b200.pcg_time wide hex 20 20 20          # batch-wide engine, 20^3 Hex8 block

Prints the device time per PCG iteration on the problem's initial tangent (unit right-hand side).
"""
from __future__ import annotations

import argparse
import ctypes

from . import _lib
from .batch import BatchSolver
from .footing import block_problem, footing_problem


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("engine", choices=["team", "wide"])
    ap.add_argument("problem", choices=["foot", "hex"])
    ap.add_argument("dims", type=int, nargs="+", help="nx ny (footing) or nx ny nz (Hex8 block)")
    ap.add_argument("--chunks", type=int, default=0, help="128-node chunks per CTA of a team (0: as many as fit)")
    ap.add_argument("--threads", type=int, default=1024)
    ap.add_argument("--iterations", type=int, default=64)
    a = ap.parse_args(argv)
    p = footing_problem(*a.dims[:2]) if a.problem == "foot" else block_problem(*a.dims[:3])
    bs = BatchSolver([p])
    t = _lib.BatchTuning_(10 ** 12 if a.engine == "team" else 0, a.threads, a.chunks, 128, 8)
    ms = ctypes.c_double()
    rc = bs.L.pms_batch_time_pcg(bs.h, ctypes.byref(t), a.iterations, ctypes.byref(ms))
    if rc != 0:
        raise _lib.PmsError(rc)
    print(f"{a.engine} {a.problem} {a.dims} ndof {p.mesh.ndof}: {ms.value / a.iterations * 1e3:.2f} us per iteration")
    bs.close()


if __name__ == "__main__":
    main()
