#!/usr/bin/env python
"""Accuracy of the large plume configurations against the f64 oracle.

The 128^3 x 200-step plumes (CG to 1e-6, and RB-SOR omega 1.7 x 80) and the
256^3 x 100-step plume (seed 1) take the single-threaded CPU oracle between a
quarter of an hour and well over an hour, too long for a test run.  The
comparison therefore runs in two halves:

  python tests/large_accuracy.py oracle c2_cg OUTDIR   # CPU, writes OUTDIR/oracle_c2_cg.npz
  python tests/large_accuracy.py gpu c2_cg OUTDIR      # B200, reads that file
  python tests/large_accuracy.py converged c2_cg OUTDIR  # B200 only, no oracle

The oracle's final fields are stored as float32 (relative resolution ~6e-8,
well below the 1e-5 / 1e-4 tolerances checked).  `gpu` runs each form of the
configuration on the device, stores its fields the same way and prints one
JSON line per form: relative L2 and max |error| of u, v, w, density and
temperature against the oracle, and whether the form's tolerance holds
(1e-5 relative L2 for the plain FP64 path, 1e-4 for the mixed path).
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "aether-core-engine_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

FIELDS = ("u", "v", "w", "density", "temperature")
TOL = {"fp64": 1e-5, "mixed": 1e-4}


def configs():
    from aether_fluid.plume import C2_CG, C2_SOR, C3
    return {"c2_cg": (C2_CG, ("fp64", "mixed")), "c2_sor": (C2_SOR, ("fp64", "mixed")),
            "c3": (C3, ("mixed", "fp64"))}


def run_oracle(name: str, out: str) -> None:
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from helpers import oracle_for
    O.build()
    plume, _ = configs()[name]
    s = oracle_for(plume, O)
    t0 = time.perf_counter()
    s.run(plume.steps, plume.dt, 0.0, plume.dt)
    el = time.perf_counter() - t0
    np.savez(os.path.join(out, f"oracle_{name}.npz"), seconds=el,
             **{f: s.field(f).astype(np.float32) for f in FIELDS})
    print(json.dumps({"config": name, "oracle_seconds": el}), flush=True)


def run_gpu(name: str, out: str) -> int:
    import aether_fluid as af
    from helpers import max_abs, rel_l2
    plume, forms = configs()[name]
    ref = np.load(os.path.join(out, f"oracle_{name}.npz"))
    ok = True
    for form in forms:
        s = plume.build(precision=af.Precision.FP64 if form == "fp64" else af.Precision.MIXED)
        _, infos = s.run(plume.steps, plume.dt, 0.0, plume.dt)
        got = {f: s.get_field(f) for f in FIELDS}
        s.close()
        row = {"config": name, "form": form, "grid": [plume.nx, plume.ny, plume.nz],
               "steps": plume.steps, "solver": plume.solver, "tolerance": TOL[form],
               "rel_l2": {f: rel_l2(got[f].astype(np.float32), ref[f]) for f in FIELDS},
               "max_abs": {f: max_abs(got[f].astype(np.float32), ref[f]) for f in FIELDS},
               "mean_solver_iters": float(np.mean([i.iterations for i in infos]))}
        row["within_tolerance"] = all(v <= TOL[form] for v in row["rel_l2"].values())
        ok &= row["within_tolerance"]
        print(json.dumps(row), flush=True)
    return 0 if ok else 1


def run_converged(name: str, iters: int = 5000) -> int:
    """The mixed form against the FP64 form when every solve converges (CG to
    the configuration's 1e-6 with an iteration cap high enough that it is
    never reached): separates the precision of the mixed form from the
    sensitivity of a solve truncated at 200 iterations."""
    import aether_fluid as af
    from helpers import max_abs, rel_l2
    plume, _ = configs()[name]
    if plume.solver != "cg":
        print("converged mode applies to CG configurations")
        return 2
    got, its = {}, {}
    for form in ("fp64", "mixed"):
        s = plume.build(precision=af.Precision.FP64 if form == "fp64" else af.Precision.MIXED)
        s.set_params(solver_iters=iters, mixed_inner_iters=iters)
        _, infos = s.run(plume.steps, plume.dt, 0.0, plume.dt)
        got[form] = {f: s.get_field(f) for f in FIELDS}
        its[form] = {"mean_solver_iters": float(np.mean([i.iterations for i in infos])),
                     "all_converged": bool(all(i.converged for i in infos))}
        s.close()
    row = {"config": name, "compare": "mixed vs fp64, converged solves", "iteration_cap": iters,
           "rel_l2": {f: rel_l2(got["mixed"][f], got["fp64"][f]) for f in FIELDS},
           "max_abs": {f: max_abs(got["mixed"][f], got["fp64"][f]) for f in FIELDS}, **its}
    row["within_mixed_tolerance"] = all(v <= TOL["mixed"] for v in row["rel_l2"].values())
    print(json.dumps(row), flush=True)
    return 0


def main() -> int:
    if len(sys.argv) == 4 and sys.argv[1] == "converged" and sys.argv[2] in configs():
        return run_converged(sys.argv[2])
    if len(sys.argv) != 4 or sys.argv[1] not in ("oracle", "gpu") or sys.argv[2] not in configs():
        print(__doc__)
        return 2
    mode, name, out = sys.argv[1:]
    os.makedirs(out, exist_ok=True)
    if mode == "oracle":
        run_oracle(name, out)
        return 0
    return run_gpu(name, out)


if __name__ == "__main__":
    sys.exit(main())
