"""CPU tests of the oracle: pinned to the reference's own known answers and
invariant tests, then to the committed golden fixtures."""
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR


def test_readme_known_answer(oracle):
    """README.md:54 (src/verify.rs:229-250): ||div u|| 2.5751e0 -> 6.7289e-3."""
    O = oracle
    s = O.OracleSolver(16, 20, 16)
    s.set_params(solver_kind=O.CG, solver_iters=40)
    s.inject_cyberpunk_sources(0.5, 0.1)
    s.apply_buoyancy_and_vorticity_confinement(0.1)
    pre = s.compute_divergence_norm()
    s.project()
    post = s.compute_divergence_norm()
    assert f"{pre:.4e}" == "2.5751e+00"
    assert f"{post:.4e}" == "6.7289e-03"
    assert f"{(1 - post / pre) * 100:.1f}" == "99.7"
    assert post <= 0.03 * pre  # src/verify.rs:239


@pytest.mark.parametrize("kind", ["cg", "rbgs"])
def test_projection_reduces_divergence(oracle, kind):
    """src/fluid.rs:918-956."""
    from golden.gen_golden import burst_solver
    O = oracle
    s = burst_solver(O.CG if kind == "cg" else O.RBGS)
    before = s.compute_divergence_norm()
    assert before > 1.0
    s.project()
    after = s.compute_divergence_norm()
    assert after < before * 0.02


def test_positivity_and_confinement(oracle):
    """src/fluid.rs:959-968."""
    s = oracle.OracleSolver(16, 20, 16)
    f1 = s.step(0.08, 0.2)
    f2 = s.step(0.08, 0.4)
    assert f1[1] > 0.0
    assert f2[2] > 0.0
    d = s.field("density")
    assert np.all(np.isfinite(d)) and np.all(d >= 0.0)


def test_grid_assert(oracle):
    """src/fluid.rs:54: every dimension must be >= 6."""
    with pytest.raises(ValueError):
        oracle.OracleSolver(5, 8, 8)


def test_rbgs_colour_order_independent(oracle):
    """Within one colour the SOR update reads only the other colour, so the
    sweep equals a Jacobi-style update of that colour from the same state."""
    O = oracle
    s = O.OracleSolver(10, 12, 9)
    rng = np.random.default_rng(5)
    s.field("divergence")[:] = rng.standard_normal(s.n)
    s.field("pressure")[:] = rng.standard_normal(s.n)
    p0 = s.field("pressure").copy()
    b = s.field("divergence").copy()
    s.set_params(sor_omega=1.7)
    s.solve_poisson_gauss_seidel(1)
    nx, ny, nz = 10, 12, 9
    p = p0.reshape(nz, ny, nx).copy()
    bb = b.reshape(nz, ny, nx)
    for color in (0, 1):
        new = p.copy()
        for k in range(1, nz - 1):
            for j in range(1, ny - 1):
                for i in range(1, nx - 1):
                    if (i + j + k) % 2 != color:
                        continue
                    diag = 0.0
                    nb = 0.0
                    for cond, val in ((i > 1, p[k, j, i - 1]), (i + 2 < nx, p[k, j, i + 1]),
                                      (j > 1, p[k, j - 1, i]), (j + 2 < ny, p[k, j + 1, i]),
                                      (k > 1, p[k - 1, j, i]), (k + 2 < nz, p[k + 1, j, i])):
                        if cond:
                            diag += 1.0
                            nb += val
                    new[k, j, i] = (1.0 - 1.7) * p[k, j, i] + 1.7 * ((bb[k, j, i] + nb) / diag)
        p = new
    assert np.array_equal(p.ravel(), s.field("pressure"))


def test_rng_golden(oracle):
    """Xoshiro256++/SplitMix64 (src/rng.rs:5-88) is integer arithmetic: bit exact."""
    d = np.load(os.path.join(GOLDEN_DIR, "rng.npz"))
    for seed in (0, 1, 42):
        assert np.array_equal(oracle.rng_u64(seed, 64), d[f"u64_{seed}"])
        assert np.array_equal(oracle.rng_f64(seed, 64), d[f"f64_{seed}"])
    f = oracle.rng_f64(42, 50_000)  # src/rng.rs:155-166
    assert np.all((f >= 0.0) & (f < 1.0)) and abs(f.mean() - 0.5) < 0.01


def test_rng_published_xoshiro_step(oracle):
    """The Xoshiro256++ output function on a known state, restated in numpy."""
    u = oracle.rng_u64(7, 3)
    M = (1 << 64) - 1

    def splitmix(st):
        st = (st + 0x9E3779B97F4A7C15) & M
        z = st
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        return st, z ^ (z >> 31)

    st = 7 ^ 0xA5A55A5AF0F00F0F
    s = []
    for _ in range(4):
        st, z = splitmix(st)
        s.append(z)
    rotl = lambda x, k: ((x << k) | (x >> (64 - k))) & M  # noqa: E731
    out = []
    for _ in range(3):
        out.append((rotl((s[0] + s[3]) & M, 23) + s[0]) & M)
        t = (s[1] << 17) & M
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = rotl(s[3], 45)
    assert [int(x) for x in u] == out


@pytest.mark.parametrize("name", ["verify_check4", "burst_cg", "burst_rbgs", "two_steps",
                                  "plume_cg_24x20x18", "plume_sor_20x24x16"])
def test_golden_fixtures_reproduce(oracle, name):
    """The oracle regenerates every committed fixture bit for bit."""
    from golden.gen_golden import CASES
    fresh = CASES[name]()
    gold = np.load(os.path.join(GOLDEN_DIR, f"{name}.npz"))
    assert set(gold.files) == set(fresh)
    for k in gold.files:
        assert np.array_equal(np.asarray(fresh[k]), gold[k]), k
