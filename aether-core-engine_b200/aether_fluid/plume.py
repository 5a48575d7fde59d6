"""Seeded synthetic smoke-plume configurations shared by tests and bench.py.

Each configuration follows the workload definitions of the benchmark: a MAC
grid with h = 1/max(n), uniform velocity noise in [-0.01, 0.01] from a seed
(Rng::from_seed, u then v then w, x fastest, then the wall BC), a spherical
source that assigns density = temperature = 1 each step centred at
(nx/2, 0.1*ny, nz/2) with radius 5*nx/64 cells, alpha = 0.08, beta = 0.4,
eps = 0.3, dt = 0.5*h, CG to relative residual 1e-6 (max 200) or RB-SOR
omega = 1.7.
"""
from __future__ import annotations

from dataclasses import dataclass, field


@dataclass
class Plume:
    nx: int
    ny: int
    nz: int
    steps: int
    seed: int = 0
    solver: str = "cg"          # "cg" or "sor"
    iters: int = 200            # CG max iterations / SOR sweeps
    rel_tol: float = 1e-6
    omega: float = 1.7
    alpha: float = 0.08
    beta: float = 0.4
    eps: float = 0.3
    center: tuple = field(default=None)
    radius: float = None

    def __post_init__(self):
        if self.center is None:
            self.center = (self.nx / 2, 0.1 * self.ny, self.nz / 2)
        if self.radius is None:
            self.radius = 5.0 * self.nx / 64.0

    @property
    def h(self) -> float:
        return 1.0 / max(self.nx, self.ny, self.nz)

    @property
    def dt(self) -> float:
        return 0.5 * self.h

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    def build(self, precision=0):
        """A FluidSolver3D configured and initialised for this plume."""
        from .solver import FluidSolver3D
        s = FluidSolver3D(self.nx, self.ny, self.nz, precision=precision)
        s.set_params(vorticity_eps=self.eps, buoyancy_beta=self.beta,
                     gravity_alpha=self.alpha,
                     solver_kind=0 if self.solver == "cg" else 1,
                     solver_iters=self.iters, sor_omega=self.omega,
                     cg_rel_tol=self.rel_tol if self.solver == "cg" else 0.0)
        s.init_velocity_noise(self.seed)
        s.set_sphere_source(self.center, self.radius)
        return s


# The benchmark's configurations (the 48-plume ensemble is built elsewhere).
C1 = Plume(64, 64, 64, 50, seed=0)
C2_CG = Plume(128, 128, 128, 200, seed=0)
C2_SOR = Plume(128, 128, 128, 200, seed=0, solver="sor", iters=80)
C3 = Plume(256, 256, 256, 100, seed=1, center=(128, 25.6, 128), radius=20)
