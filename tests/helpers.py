"""Test helpers: the oracle set up for a plume configuration, field metrics."""
from __future__ import annotations

import numpy as np


def oracle_for(plume, O):
    """The CPU oracle configured and initialised like Plume.build()."""
    s = O.OracleSolver(plume.nx, plume.ny, plume.nz)
    s.set_params(vorticity_eps=plume.eps, buoyancy_beta=plume.beta,
                 gravity_alpha=plume.alpha,
                 solver_kind=O.CG if plume.solver == "cg" else O.RBGS,
                 solver_iters=plume.iters, sor_omega=plume.omega,
                 cg_rel_tol=plume.rel_tol if plume.solver == "cg" else 0.0)
    s.init_velocity_noise(plume.seed)
    s.set_sphere_source(plume.center, plume.radius)
    return s


def rel_l2(a, ref) -> float:
    a = np.asarray(a, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    den = np.linalg.norm(ref)
    num = np.linalg.norm(a - ref)
    return float(num / den) if den > 0 else float(num)


def max_abs(a, ref) -> float:
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(ref, np.float64))))
