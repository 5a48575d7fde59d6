#!/usr/bin/env python
"""The 96^3 x 64-step adjoint gradient against central differences of the f64
CPU oracle (the adjoint workload: seed-0 velocity noise, seed-2 temperature
amplitude map, target source 8 cells further in x, checkpoints every 8 steps,
pressure solves to 1e-12).

One oracle run takes minutes, so the check runs in two halves:

  python tests/large_adjoint_fd.py gpu OUTDIR      # B200: adjoint directional derivatives
  python tests/large_adjoint_fd.py oracle OUTDIR   # CPU, all cores: oracle differences

`gpu` writes OUTDIR/adjoint_fd_gpu.json: the loss and <grad, d_k> for K seeded
unit directions d_k of the control space (velocity parts zero on the wall-BC
cells).  `oracle` runs the oracle at x +- eps*d_k in a process pool and prints
|fd - ad| / |ad| per direction.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "aether-core-engine_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

N, STEPS, EVERY = 96, 64, 8
DT = 0.5 / N
CENTER, RADIUS = (N / 2, 0.1 * N, N / 2), 5.0 * N / 64.0
SHIFT = 8.0
REL_TOL, ITERS = 1e-12, 4000
EPS = 1e-7
K = 8


def wall_masked(u, v, w):
    """enforce_wall_velocity_bc (src/fluid.rs:236-253) on flat arrays."""
    k, j, i = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
    edge = (i == 0) | (i + 1 >= N) | (j == 0) | (j + 1 >= N) | (k == 0) | (k + 1 >= N)
    masks = ((i <= 1) | edge, (j <= 1) | edge, (k <= 1) | edge)
    return tuple(np.where(m.ravel(), 0.0, a) for m, a in zip(masks, (u, v, w)))


def controls():
    from aether_fluid.ensemble import rng_f64
    cells = N ** 3
    noise = rng_f64(0, 0, 3 * cells)
    u, v, w = wall_masked(*(-0.01 + 0.02 * noise[a * cells:(a + 1) * cells] for a in range(3)))
    return u, v, w, 0.5 + rng_f64(2, 0, cells)


def directions():
    rng = np.random.default_rng(11)
    cells = N ** 3
    for _ in range(K):
        d = [rng.standard_normal(cells) for _ in range(4)]
        d[0], d[1], d[2] = wall_masked(d[0], d[1], d[2])
        nrm = np.sqrt(sum(float(np.dot(a, a)) for a in d))
        yield [a / nrm for a in d]


def run_gpu(out: str) -> None:
    from aether_fluid.adjoint import Adjoint

    def make(c):
        return Adjoint(N, N, N, center=c, radius=RADIUS, checkpoint_every=EVERY,
                       cg_rel_tol=REL_TOL, solver_iters=ITERS)
    ctl = controls()
    t = make((CENTER[0] + SHIFT, CENTER[1], CENTER[2]))
    tgt = t.forward(*ctl, STEPS, DT)
    t.close()
    adj = make(CENTER)
    rho = adj.forward(*ctl, STEPS, DT)
    g = adj.backward(rho - tgt)
    ad = [sum(float(np.dot(a, b)) for a, b in zip(g, d)) for d in directions()]
    rec = {"loss": 0.5 * float(np.sum((rho - tgt) ** 2)), "ad": ad, "eps": EPS,
           "gradient_norm": float(np.sqrt(sum(float(np.dot(a, a)) for a in g)))}
    np.save(os.path.join(out, "adjoint_fd_target.npy"), tgt)
    with open(os.path.join(out, "adjoint_fd_gpu.json"), "w") as f:
        json.dump(rec, f)
    print(json.dumps(rec))


def _oracle_loss(args):
    sign, k, tgt_path = args
    import oracle as O
    ctl = controls()
    d = list(directions())[k]
    x = [a + sign * EPS * b for a, b in zip(ctl, d)]
    s = O.OracleSolver(N, N, N)
    s.set_params(vorticity_eps=0.3, buoyancy_beta=0.4, gravity_alpha=0.08, solver_kind=O.CG,
                 solver_iters=ITERS, cg_rel_tol=REL_TOL)
    for name, arr in zip(("u", "v", "w"), x[:3]):
        s.field(name)[:] = arr
    s.set_sphere_source(CENTER, RADIUS, 1.0, 1.0, temp_amp=x[3])
    for n in range(STEPS):
        s.step(DT, n * DT)
    tgt = np.load(tgt_path)
    return sign, k, 0.5 * float(np.sum((s.field("density") - tgt) ** 2))


def run_oracle(out: str) -> None:
    import multiprocessing as mp
    import oracle as O
    O.build()
    with open(os.path.join(out, "adjoint_fd_gpu.json")) as f:
        rec = json.load(f)
    tgt_path = os.path.join(out, "adjoint_fd_target.npy")
    jobs = [(s, k, tgt_path) for k in range(K) for s in (1.0, -1.0)]
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(min(len(jobs), os.cpu_count() or 1)) as pool:
        res = pool.map(_oracle_loss, jobs)
    loss = {(s, k): v for s, k, v in res}
    rows = []
    for k in range(K):
        fd = (loss[(1.0, k)] - loss[(-1.0, k)]) / (2 * EPS)
        ad = rec["ad"][k]
        rows.append({"direction": k, "oracle_fd": fd, "adjoint": ad,
                     "rel_err": abs(fd - ad) / abs(ad)})
    errs = [r["rel_err"] for r in rows]
    print(json.dumps({"eps": EPS, "directions": K, "oracle_seconds": time.perf_counter() - t0,
                      "rel_err_median": float(np.median(errs)), "rel_err_max": float(max(errs)),
                      "rows": rows}))


if __name__ == "__main__":
    if len(sys.argv) != 3 or sys.argv[1] not in ("gpu", "oracle"):
        print(__doc__)
        sys.exit(2)
    os.makedirs(sys.argv[2], exist_ok=True)
    (run_gpu if sys.argv[1] == "gpu" else run_oracle)(sys.argv[2])
