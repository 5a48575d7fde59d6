"""CPU checks of the ensemble's host logic: the product's copy of the reference
generator equals the oracle's bit for bit, and the 48-plume builder draws its
jitter and buoyancy from the documented ranges."""
import numpy as np


def test_product_rng_matches_oracle(oracle):
    from aether_fluid.ensemble import rng_f64
    for seed in (0, 7, 123):
        assert np.array_equal(rng_f64(seed, 0, 50), oracle.rng_f64(seed, 50))
    # skipping k draws equals dropping the first k values
    assert np.array_equal(rng_f64(5, 10, 20), oracle.rng_f64(5, 30)[10:])


def test_plume48_builder():
    from aether_fluid.ensemble import plume48
    specs = plume48()
    assert len(specs) == 48
    assert [s.seed for s in specs] == list(range(100, 148))
    shapes = [(s.nx, s.ny, s.nz) for s in specs]
    assert shapes == [(32, 32, 32)] * 16 + [(48, 48, 48)] * 16 + [(64, 128, 64)] * 16
    for s in specs:
        base = (s.nx / 2, 0.1 * s.ny, s.nz / 2)
        for a, ext in enumerate((s.nx, s.ny, s.nz)):
            assert abs(s.center[a] - base[a]) <= 0.1 * ext + 1e-12
        assert 0.05 <= s.alpha <= 0.1 and 0.3 <= s.beta <= 0.5
        assert s.radius == 5.0 * s.nx / 64.0 and s.dt == 0.5 / max(s.nx, s.ny, s.nz)
    assert len({round(s.alpha, 12) for s in specs}) == 48
