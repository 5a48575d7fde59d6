"""The batched ensemble against single-grid solvers with the same settings:
one launch per stage over all instances and one cooperative launch for all
pressure solves must evolve every instance like its own FluidSolver3D."""
import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "density", "temperature", "pressure")


def specs_small():
    from aether_fluid.ensemble import InstanceSpec
    return [
        InstanceSpec(24, 20, 18, seed=11, alpha=0.06, beta=0.35, center=(11.5, 2.5, 9.2),
                     radius=3.0),
        InstanceSpec(32, 32, 32, seed=12, alpha=0.09, beta=0.45),
        InstanceSpec(16, 24, 20, seed=13, alpha=0.07, beta=0.3, center=(8.3, 3.1, 10.0),
                     radius=2.5),
        InstanceSpec(40, 28, 24, seed=14),
    ]


def single(af, spec, precision, steps):
    s = af.FluidSolver3D(spec.nx, spec.ny, spec.nz, precision=precision)
    s.set_params(vorticity_eps=spec.eps, buoyancy_beta=spec.beta, gravity_alpha=spec.alpha,
                 solver_kind=0, solver_iters=200, cg_rel_tol=1e-6, poisson_kernel=1)
    s.init_velocity_noise(spec.seed, -spec.noise, spec.noise)
    s.set_sphere_source(spec.center, spec.radius)
    tel, infos = s.run(steps, spec.dt, 0.0, spec.dt)
    return s, tel, infos


@pytest.mark.parametrize("precision,tol", [(0, 1e-10), (1, 1e-5)])
def test_ensemble_matches_single_solvers(af, precision, tol):
    from aether_fluid.ensemble import Ensemble
    specs = specs_small()
    steps = 5
    ens = Ensemble(specs, precision=precision)
    info = ens.info()
    assert info["graph"], info
    assert sum(info["instance_ctas"]) == info["solver_ctas"] <= info["cta_budget"]
    tel, infos = ens.run(steps)
    for m, spec in enumerate(specs):
        s, tel1, infos1 = single(af, spec, precision, steps)
        for f in FIELDS:
            err = rel_l2(ens.field(m, f), s.get_field(f))
            assert err <= tol, (m, f, err)
        np.testing.assert_allclose(tel[:, m, 1:5], tel1[:, 1:5], rtol=max(tol, 1e-9))
        its = [infos[n][m].iterations for n in range(steps)]
        its1 = [i.iterations for i in infos1]
        assert all(abs(a - b) <= 1 for a, b in zip(its, its1)), (m, its, its1)


@pytest.mark.parametrize("persistent", [False, True])
@pytest.mark.parametrize("precision,tol", [(0, 1e-8), (1, 1e-4)])
def test_ensemble_matches_oracle(af, oracle, precision, tol, persistent):
    """Every instance of a batched ensemble of four grid sizes against its own
    run of the f64 CPU oracle (src/fluid.rs:598-611 with the sphere source):
    the fields after 5 steps within 1e-8 relative L2 (FP64; the batched CG
    sums in another order) or 1e-4 (mixed), and, in FP64, the per-step CG
    iteration counts within 1.  Both step forms: the graph of stage launches
    and the single persistent launch."""
    from aether_fluid.ensemble import Ensemble
    O = oracle
    specs = specs_small()
    steps = 5
    ens = Ensemble(specs, precision=precision)
    ens.set_persistent(persistent)
    assert ens.info()["persistent"] == persistent and ens.info()["graph"]
    tel, infos = ens.run(steps)
    for m, spec in enumerate(specs):
        o = O.OracleSolver(spec.nx, spec.ny, spec.nz)
        o.set_params(vorticity_eps=spec.eps, buoyancy_beta=spec.beta, gravity_alpha=spec.alpha,
                     solver_kind=O.CG, solver_iters=200, cg_rel_tol=1e-6)
        o.init_velocity_noise(spec.seed, -spec.noise, spec.noise)
        o.set_sphere_source(spec.center, spec.radius)
        its = []
        for n in range(steps):
            o.step(spec.dt, n * spec.dt)
            its.append(o.last_cg_iters())
        for f in ("u", "v", "w", "density", "temperature"):
            err = rel_l2(ens.field(m, f), o.field(f))
            assert err <= tol, (m, f, err)
        if precision == 0:
            got = [infos[n][m].iterations for n in range(steps)]
            assert all(abs(a - b) <= 1 for a, b in zip(got, its)), (m, got, its)


def test_ensemble_autotune_restores_state(af):
    from aether_fluid.ensemble import Ensemble
    specs = specs_small()
    a = Ensemble(specs, precision=1)
    choice = a.autotune()
    assert choice in (0, 1, 2)
    assert a.info()["autotune_choice"] == choice
    assert a.info()["tile_depth"] in (1, 2, 4)
    tel_a, _ = a.run(3)
    b = Ensemble(specs, precision=1)
    tel_b, _ = b.run(3)
    for m in range(len(specs)):
        for f in ("density", "u"):
            assert rel_l2(a.field(m, f), b.field(m, f)) <= 1e-5
    np.testing.assert_allclose(tel_a[:, :, 1:5], tel_b[:, :, 1:5], rtol=1e-4)


def test_plume48_runs(af):
    """The 48-plume ensemble (16 x 32^3, 16 x 48^3, 16 x 64x128x64), a few
    steps: every instance stays finite, its density non-negative, its
    projection reduces the residual."""
    from aether_fluid.ensemble import Ensemble, plume48
    specs = plume48()
    ens = Ensemble(specs, precision=1)
    tel, infos = ens.run(3)
    assert np.all(np.isfinite(tel))
    for m in (0, 16, 47):
        d = ens.field(m, "density")
        assert np.all(np.isfinite(d)) and d.min() >= 0.0 and d.max() > 0.5
    for n in range(3):
        for m in range(48):
            i = infos[n][m]
            assert i.final_residual < i.initial_residual, (n, m, i)


def test_sharded_api_single_rank_is_the_batched_ensemble(af):
    """run_sharded with one process runs the whole list as one ensemble: the
    gathered telemetry is the ensemble's, in the original instance order."""
    from aether_fluid.ensemble import Ensemble
    from aether_fluid.sharding import run_sharded
    specs = specs_small()
    tel, infos, parts = run_sharded(specs, 3, dist=None, precision=0, autotune=False)
    assert parts[0]["indices"] == list(range(len(specs)))
    assert parts[0]["run_seconds"] > 0
    ref_tel, ref_infos = Ensemble(specs, precision=0).run(3)
    np.testing.assert_array_equal(tel, ref_tel)
    assert [[i.iterations for i in row] for row in infos] == \
        [[i.iterations for i in row] for row in ref_infos]


@pytest.mark.parametrize("kz", [2, 4])
def test_tile_depth_does_not_change_the_evolution(af, kz):
    """Stage tiles of 1, 2 or 4 z planes run the same per-cell code: the FP64
    fields are identical; telemetry sums differ only in summation order."""
    from aether_fluid.ensemble import Ensemble
    specs = specs_small()
    a = Ensemble(specs, precision=0)
    tel_a, _ = a.run(3)
    b = Ensemble(specs, precision=0)
    b.set_tile_depth(kz)
    assert b.info()["tile_depth"] == kz and b.info()["graph"]
    tel_b, _ = b.run(3)
    for m in range(len(specs)):
        for f in FIELDS:
            assert np.array_equal(a.field(m, f), b.field(m, f)), (m, f)
    np.testing.assert_allclose(tel_b[:, :, 1:5], tel_a[:, :, 1:5], rtol=1e-12)
    # switching back mid-run keeps going from the current state
    b.set_tile_depth(1)
    a.run(2)
    b.run(2)
    for m in range(len(specs)):
        assert np.array_equal(a.field(m, "density"), b.field(m, "density"))


@pytest.mark.parametrize("precision,tol", [(0, 1e-10), (1, 1e-5)])
def test_persistent_step_matches_stage_graph(af, precision, tol):
    """One persistent launch per step against the graph of per-stage launches:
    the same per-cell code and CG body, so the fields agree to the summation
    order of the CG (its CTA split follows the step kernel's co-resident
    budget) and, in f32, to FMA contraction (the step kernel's unit is built
    without it).  Switching the form mid-run continues from the current state."""
    from aether_fluid.ensemble import Ensemble
    specs = specs_small()
    a = Ensemble(specs, precision=precision)
    a.set_persistent(False)
    tel_a, infos_a = a.run(5)
    b = Ensemble(specs, precision=precision)
    assert b.info()["persistent"]       # the default form
    b.set_persistent(True)
    info = b.info()
    assert info["persistent"] and info["graph"], info
    assert sum(info["instance_ctas"]) == info["solver_ctas"] <= info["cta_budget"]
    tel_b, infos_b = b.run(2)
    b.set_persistent(False)
    assert not b.info()["persistent"]
    tel_c, infos_c = b.run(1)
    b.set_persistent(True)
    tel_d, infos_d = b.run(2)
    tel_bd = np.concatenate([tel_b, tel_c, tel_d])
    infos_bd = infos_b + infos_c + infos_d
    for m in range(len(specs)):
        for f in FIELDS:
            err = rel_l2(b.field(m, f), a.field(m, f))
            assert err <= tol, (m, f, err)
        its_a = [infos_a[n][m].iterations for n in range(5)]
        its_b = [infos_bd[n][m].iterations for n in range(5)]
        assert all(abs(x - y) <= 1 for x, y in zip(its_a, its_b)), (m, its_a, its_b)
    # run() restarts the step count: each run's frames are numbered from 0
    np.testing.assert_allclose(tel_bd[:, :, 1:5], tel_a[:, :, 1:5], rtol=max(tol, 1e-9))


def test_persistent_autotune_restores_state(af):
    from aether_fluid.ensemble import Ensemble
    specs = specs_small()
    a = Ensemble(specs, precision=1)
    a.set_persistent(True)
    choice = a.autotune()
    info = a.info()
    assert choice in (0, 1, 2) and info["autotune_choice"] == choice and info["persistent"]
    tel_a, _ = a.run(3)
    b = Ensemble(specs, precision=1)
    b.set_persistent(True)
    tel_b, _ = b.run(3)
    for m in range(len(specs)):
        for f in ("density", "u"):
            assert rel_l2(a.field(m, f), b.field(m, f)) <= 1e-5
