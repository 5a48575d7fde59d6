"""Generates the golden fixtures of tests/golden/ from the CPU oracle.

The reference (Rust) cannot be built in this image, so the fixtures are the
oracle's outputs on small seeded cases; the oracle itself is pinned to the
reference's published known answer (README.md:54, produced by
src/verify.rs:229-250) and to the invariant tests of src/fluid.rs:917-968,
which tests/test_oracle.py re-checks.  Run:  python tests/golden/gen_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "aether-core-engine_b200"))

import oracle as O  # noqa: E402
from aether_fluid.plume import Plume  # noqa: E402

FIELDS = ("u", "v", "w", "density", "temperature", "pressure")


def _fields(s) -> dict:
    return {f: s.field(f).copy() for f in FIELDS}


def case_verify_check4() -> dict:
    """src/verify.rs:229-250: the projection known answer of README.md:54."""
    s = O.OracleSolver(16, 20, 16)
    s.set_params(solver_kind=O.CG, solver_iters=40)
    s.inject_cyberpunk_sources(0.5, 0.1)
    s.apply_buoyancy_and_vorticity_confinement(0.1)
    pre = s.compute_divergence_norm()
    iters = s.project()
    post = s.compute_divergence_norm()
    out = _fields(s)
    out.update(dims=np.array([16, 20, 16]), div_pre=pre, div_post=post, cg_iters=iters)
    return out


def burst_solver(kind: int):
    """src/fluid.rs:923-942: the divergent burst on 18x22x18."""
    s = O.OracleSolver(18, 22, 18)
    s.set_params(solver_kind=kind, solver_iters=45 if kind == O.CG else 90)
    u, v, w = s.field("u"), s.field("v"), s.field("w")
    for k in range(6, 12):
        for j in range(5, 11):
            for i in range(6, 12):
                c = s.idx(i, j, k)
                u[c] = (i - 8.5) * 3.0
                v[c] = (j - 7.5) * 4.5
                w[c] = (k - 8.5) * 2.5
    s.enforce_wall_velocity_bc()
    return s


def case_burst(kind: int) -> dict:
    s = burst_solver(kind)
    pre = s.compute_divergence_norm()
    s.project()
    post = s.compute_divergence_norm()
    out = _fields(s)
    out.update(dims=np.array([18, 22, 18]), div_pre=pre, div_post=post)
    return out


def case_two_steps() -> dict:
    """src/fluid.rs:959-968: two reference steps on 16x20x16 (cyberpunk jets)."""
    s = O.OracleSolver(16, 20, 16)
    t1 = s.step(0.08, 0.2)
    t2 = s.step(0.08, 0.4)
    out = _fields(s)
    out.update(dims=np.array([16, 20, 16]), telemetry=np.stack([t1, t2]))
    return out


def plume_case(p: Plume) -> dict:
    s = O.OracleSolver(p.nx, p.ny, p.nz)
    s.set_params(vorticity_eps=p.eps, buoyancy_beta=p.beta, gravity_alpha=p.alpha,
                 solver_kind=O.CG if p.solver == "cg" else O.RBGS, solver_iters=p.iters,
                 sor_omega=p.omega, cg_rel_tol=p.rel_tol if p.solver == "cg" else 0.0)
    s.init_velocity_noise(p.seed)
    s.set_sphere_source(p.center, p.radius)
    tel = []
    iters = []
    for n in range(p.steps):
        tel.append(s.step(p.dt, n * p.dt))
        iters.append(s.last_cg_iters())
    out = _fields(s)
    out.update(dims=np.array([p.nx, p.ny, p.nz]), telemetry=np.stack(tel),
               cg_iters=np.array(iters))
    return out


PLUME_CG = Plume(24, 20, 18, 8, seed=3)
PLUME_SOR = Plume(20, 24, 16, 6, seed=4, solver="sor", iters=20)


def case_rng() -> dict:
    out = {}
    for seed in (0, 1, 42):
        out[f"u64_{seed}"] = O.rng_u64(seed, 64)
        out[f"f64_{seed}"] = O.rng_f64(seed, 64)
    return out


CASES = {
    "verify_check4": case_verify_check4,
    "burst_cg": lambda: case_burst(O.CG),
    "burst_rbgs": lambda: case_burst(O.RBGS),
    "two_steps": case_two_steps,
    "plume_cg_24x20x18": lambda: plume_case(PLUME_CG),
    "plume_sor_20x24x16": lambda: plume_case(PLUME_SOR),
    "rng": case_rng,
}


def main():
    O.build()
    for name, fn in CASES.items():
        data = fn()
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **{k: np.asarray(v) for k, v in data.items()})
        print(f"{path}: {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
