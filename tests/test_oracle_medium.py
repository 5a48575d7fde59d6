"""The oracle's restatement of FluidMedium's volume queries
(src/fluid.rs:687-874) on the CPU: the estimators against the optical depth
integrated along the ray, and the sampler's edge behaviour."""
import numpy as np
import pytest

SHAPE = (12, 14, 10)
LO, HI = (0.0, 0.0, 0.0), (1.0, 1.2, 0.8)


@pytest.fixture(scope="module")
def grids():
    rng = np.random.default_rng(3)
    n = SHAPE[0] * SHAPE[1] * SHAPE[2]
    return rng.uniform(0.0, 1.0, n), rng.uniform(0.0, 2.0, n)


def test_sampler_edges(oracle, grids):
    d, t = grids
    rho, tmp = oracle.medium_sample(d, t, SHAPE, LO, HI,
                                    [[-0.1, 0.5, 0.4], [0.5, 1.3, 0.4], [0.0, 0.5, 0.4],
                                     [0.5, 0.6, 0.4], [0.5, 1.2, 0.4]])
    assert rho[0] == 0.0 and rho[1] == 0.0          # outside the bounds
    assert rho[2] == 0.0                            # x feather is 0 on the face
    assert rho[3] > 0.0 and tmp[3] > 0.0
    assert rho[4] == 0.0                            # y feather is 0 at the top face


def test_bounds_are_ordered_like_aabb_new(oracle, grids):
    d, t = grids
    pts = np.random.default_rng(4).uniform(LO, HI, size=(200, 3))
    a = oracle.medium_sample(d, t, SHAPE, LO, HI, pts)
    b = oracle.medium_sample(d, t, SHAPE, HI, LO, pts)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_estimators_unbiased(oracle, grids):
    d, t = grids
    sigma = 2.5
    ray = np.array([0.5, -0.3, 0.4, 0.05, 1.0, 0.02, 0.0, 2.0])
    dirn = ray[3:6] / np.linalg.norm(ray[3:6])
    m = 20000
    ts = ray[6] + (np.arange(m) + 0.5) * (ray[7] - ray[6]) / m
    rho, _ = oracle.medium_sample(d, t, SHAPE, LO, HI, ray[:3] + ts[:, None] * dirn)
    expect = np.exp(-sigma * rho.sum() * (ray[7] - ray[6]) / m)
    n = 20000
    tr = oracle.medium_transmittance(d, t, SHAPE, LO, HI, sigma, np.tile(ray, (n, 1)), 11)
    assert abs(tr.mean() - expect) <= 4 * tr.std() / np.sqrt(n) + 1e-3
    hit = oracle.medium_interaction(d, t, SHAPE, LO, HI, sigma, np.tile(ray, (n, 1)), 12)[0]
    p = 1 - expect
    assert abs(hit.mean() - p) <= 4 * np.sqrt(p * (1 - p) / n) + 1e-3


def test_thin_medium_and_misses(oracle, grids):
    d, t = grids
    rays = np.array([[5.0, 5.0, 5.0, 1.0, 0.0, 0.0, 0.0, 10.0],     # misses the box
                     [0.5, 0.5, 0.4, 0.0, 1.0, 0.0, 3.0, 10.0]])    # starts past the exit
    tr = oracle.medium_transmittance(d, t, SHAPE, LO, HI, 2.0, rays, 1)
    assert np.all(tr == 1.0)
    z = np.zeros_like(d)
    tr0 = oracle.medium_transmittance(z, t, SHAPE, LO, HI, 2.0, np.tile(rays[0], (3, 1)), 1)
    assert np.all(tr0 == 1.0)
