"""Runs one plume workload on the CPU oracle and saves the result.

Usage: python oracle_plume_job.py <C2_CG|C2_SOR|C3> <steps> <out.npz>

Test infrastructure: the large-grid parity tests start one process per
workload so that the oracle runs (seconds to a minute each) overlap one
another and the GPU runs.  The output holds the u, v, w, density and
temperature fields after `steps` steps from the initial state, the per-step
Poisson iteration counts (CG) and the per-step telemetry.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (os.path.join(ROOT, "aether-core-engine_b200"), os.path.join(ROOT, "oracle"), HERE):
    if p not in sys.path:
        sys.path.insert(0, p)


def main(name: str, steps: int, out: str) -> None:
    import oracle as O
    from aether_fluid import plume
    from helpers import oracle_for
    p = getattr(plume, name)
    s = oracle_for(p, O)
    iters, tel = [], []
    for n in range(steps):
        tel.append(s.step(p.dt, n * p.dt))
        iters.append(s.last_cg_iters())
    fields = {f: s.field(f).copy() for f in ("u", "v", "w", "density", "temperature")}
    tmp = out + ".part.npz"
    np.savez(tmp, iters=np.array(iters), telemetry=np.array(tel), **fields)
    os.replace(tmp, out)


if __name__ == "__main__":
    main(sys.argv[1], int(sys.argv[2]), sys.argv[3])
