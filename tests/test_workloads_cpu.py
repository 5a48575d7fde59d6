"""The plume workloads that the tests and bench.py run, pinned to their
definitions: grid, steps, seed, source centre and radius, physics constants,
time step and Poisson solver settings (64^3 x 50, 128^3 x 200 with CG or
RB-SOR, 256^3 x 100)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def check_common(p, n, steps, seed, center, radius):
    assert (p.nx, p.ny, p.nz) == (n, n, n)
    assert p.steps == steps and p.seed == seed
    assert p.center == pytest.approx(center) and p.radius == pytest.approx(radius)
    assert (p.alpha, p.beta, p.eps) == (0.08, 0.4, 0.3)
    assert p.h == 1.0 / n and p.dt == 0.5 / n
    assert p.cells == n ** 3


def test_64cube_plume():
    from aether_fluid.plume import C1
    check_common(C1, 64, 50, 0, (32, 6.4, 32), 5.0)
    assert (C1.solver, C1.iters, C1.rel_tol) == ("cg", 200, 1e-6)


def test_128cube_plumes():
    from aether_fluid.plume import C2_CG, C2_SOR
    check_common(C2_CG, 128, 200, 0, (64, 12.8, 64), 10.0)
    assert (C2_CG.solver, C2_CG.iters, C2_CG.rel_tol) == ("cg", 200, 1e-6)
    check_common(C2_SOR, 128, 200, 0, (64, 12.8, 64), 10.0)
    assert (C2_SOR.solver, C2_SOR.iters, C2_SOR.omega) == ("sor", 80, 1.7)


def test_256cube_plume():
    from aether_fluid.plume import C3
    check_common(C3, 256, 100, 1, (128, 25.6, 128), 20.0)
    assert (C3.solver, C3.iters, C3.rel_tol) == ("cg", 200, 1e-6)


def test_bench_runs_the_same_plumes():
    sys.path.insert(0, ROOT)
    import bench
    from aether_fluid.plume import C2_CG, C2_SOR
    for form, ref in (("mixed_cg", C2_CG), ("fp64_cg", C2_CG), ("fp64_sor", C2_SOR),
                      ("mixed_sor", C2_SOR)):
        assert bench.plume_for(form, 128, seed=0) == ref, form
