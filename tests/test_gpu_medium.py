"""FluidMedium's volume queries on the GPU (afl_medium_*) against the oracle's
restatement of src/fluid.rs:687-874: the feathered sampler bit for bit, ratio
tracking and delta tracking ray by ray (the device `log` may differ from the
host's in the last bit, which can flip a rare decision), and both estimators
against the optical depth integrated along the ray."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPE = (32, 40, 32)
LO, HI = (-1.0, 0.0, -1.0), (1.0, 2.5, 1.0)
SIGMA = 40.0


@pytest.fixture(scope="module")
def plume(af):
    from aether_fluid.plume import Plume
    p = Plume(*SHAPE, 30, seed=4)
    out = {}
    for prec in (0, 1):
        s = p.build(precision=prec)
        s.run(p.steps, p.dt, 0.0, p.dt)
        out[prec] = s
    return out


def medium(af, solver, sigma=SIGMA, g=0.3):
    return af.DeviceMedium.from_solver(solver, af.Aabb(LO, HI), sigma, g)


def fields(solver):
    return solver.get_field("density"), solver.get_field("temperature")


def random_rays(n, seed, t_end=(0.5, 6.0)):
    rng = np.random.default_rng(seed)
    o = rng.uniform((-2.0, -1.0, -2.0), (2.0, 3.5, 2.0), size=(n, 3))
    target = rng.uniform(LO, HI, size=(n, 3))
    d = target - o
    t_min = rng.uniform(0.0, 0.2, size=n)
    t_end = rng.uniform(*t_end, size=n)
    return np.column_stack([o, d, t_min, t_end])


def test_create_matches_from_solver(af, plume):
    s = plume[0]
    m = medium(af, s, g=1.7)
    dens = s.get_field("density")
    assert m.max_density == max(0.0, float(dens.max()))
    assert m.majorant_sigma_t == max(m.max_density * SIGMA, 1e-4)
    assert m.phase_g == 0.9 and m.sigma_t_scale == SIGMA


@pytest.mark.parametrize("prec", [0, 1])
def test_sampler_bit_exact(af, oracle, plume, prec):
    s = plume[prec]
    m = medium(af, s)
    rng = np.random.default_rng(1)
    pts = np.concatenate([
        rng.uniform(LO, HI, size=(20000, 3)),                         # inside
        rng.uniform((-1.5, -0.5, -1.5), (1.5, 3.0, 1.5), size=(5000, 3)),  # around
        np.array([LO, HI, (0.0, 2.5, 0.0), (1.0, 1.0, 0.0), (0.0, 2.4, 0.0)]),  # faces
    ])
    rho, tmp = m.sample_density_and_temp(pts)
    d, t = fields(s)
    ref_rho, ref_tmp = oracle.medium_sample(d, t, SHAPE, LO, HI, pts)
    assert np.array_equal(rho, ref_rho)
    assert np.array_equal(tmp, ref_tmp)
    assert np.all(rho[20000:25000][np.any((pts[20000:25000] < LO) | (pts[20000:25000] > HI),
                                          axis=1)] == 0.0)


def test_transmittance_matches_oracle(af, oracle, plume):
    s = plume[0]
    m = medium(af, s)
    rays = random_rays(20000, 2)
    tr = m.transmittance(rays, seed=77)
    d, t = fields(s)
    ref = oracle.medium_transmittance(d, t, SHAPE, LO, HI, SIGMA, rays, 77)
    assert np.all((tr >= 0.0) & (tr <= 1.0))
    same = np.abs(tr - ref) <= 1e-12
    assert same.mean() >= 0.995, same.mean()
    assert abs(tr.mean() - ref.mean()) <= 5e-3
    # rays that miss the box, start past its end or end before it: exactly 1
    assert np.all(tr[ref == 1.0] == 1.0) or same.mean() >= 0.995


def test_interaction_matches_oracle(af, oracle, plume):
    s = plume[0]
    m = medium(af, s)
    rays = random_rays(20000, 3)
    hit, t, rho, tmp = m.sample_interaction(rays, seed=91)
    d, q = fields(s)
    rh, rt, rr, rq = oracle.medium_interaction(d, q, SHAPE, LO, HI, SIGMA, rays, 91)
    agree = (hit == rh) & np.where(hit == 1, np.abs(t - rt) <= 1e-9 * np.maximum(1, np.abs(rt)),
                                   True)
    assert agree.mean() >= 0.995, agree.mean()
    both = (hit == 1) & (rh == 1) & (np.abs(t - rt) <= 1e-12)
    assert np.allclose(rho[both], rr[both], rtol=1e-12, atol=0)
    assert np.allclose(tmp[both], rq[both], rtol=1e-12, atol=0)
    assert np.all(t[hit == 0] == 0.0)
    assert hit.sum() > 200  # interactions are exercised (the plume fills a small part of the box)


def optical_depth(m, ray, n=20000):
    """sigma * integral of the sampled density along the ray segment inside
    the box (midpoint rule on the device sampler)."""
    o, d = ray[:3], ray[3:6] / np.linalg.norm(ray[3:6])
    ts = ray[6] + (np.arange(n) + 0.5) * (ray[7] - ray[6]) / n
    rho, _ = m.sample_density_and_temp(o + ts[:, None] * d)
    return m.sigma_t_scale * rho.sum() * (ray[7] - ray[6]) / n


@pytest.mark.parametrize("which", [0, 1, 2])
def test_estimators_are_unbiased(af, plume, which):
    """Mean ratio-tracking transmittance over many independent streams equals
    exp(-optical depth); the delta-tracking interaction probability equals
    1 - that (within 4 standard errors)."""
    m = medium(af, plume[0])
    rays = [np.array([0.0, -0.5, 0.0, 0.02, 1.0, -0.01, 0.0, 3.5]),
            np.array([-1.5, 0.6, 0.1, 1.0, 0.05, 0.0, 0.0, 3.0]),
            np.array([0.3, 2.9, -1.4, -0.1, -1.0, 0.5, 0.2, 2.0])][which]
    n = 40000
    batch = np.tile(rays, (n, 1))
    expect = np.exp(-optical_depth(m, rays))
    tr = m.transmittance(batch, seed=1000 + which)
    assert abs(tr.mean() - expect) <= 4 * tr.std() / np.sqrt(n) + 1e-3, (tr.mean(), expect)
    hit = m.sample_interaction(batch, seed=2000 + which)[0]
    p = 1.0 - expect
    assert abs(hit.mean() - p) <= 4 * np.sqrt(p * (1 - p) / n) + 1e-3, (hit.mean(), p)


def test_empty_medium(af):
    s = af.FluidSolver3D(16, 16, 16)
    m = af.DeviceMedium.from_solver(s, af.Aabb(LO, HI), SIGMA, 0.0)
    assert m.max_density == 0.0 and m.majorant_sigma_t == 1e-4
    rays = random_rays(100, 5)
    assert np.all(m.transmittance(rays, 1) == 1.0)
    assert np.all(m.sample_interaction(rays, 1)[0] == 0)


def test_medium_outlives_later_steps(af, plume):
    """The medium is a snapshot, like the reference's cloned vectors."""
    from aether_fluid.plume import Plume
    p = Plume(*SHAPE, 5, seed=6)
    s = p.build()
    s.run(5, p.dt, 0.0, p.dt)
    m = medium(af, s)
    pts = np.random.default_rng(8).uniform(LO, HI, size=(1000, 3))
    before = m.sample_density_and_temp(pts)
    s.run(5, p.dt, 5 * p.dt, p.dt)
    after = m.sample_density_and_temp(pts)
    assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1])


def test_batch_independent_of_order(af, plume):
    m = medium(af, plume[0])
    rays = random_rays(2000, 9)
    a = m.transmittance(rays, seed=5)
    # ray r uses seed + r: the same ray at index r in a smaller batch gives the same value
    b = m.transmittance(rays[:500], seed=5)
    assert np.array_equal(a[:500], b)
    c = m.transmittance(rays[500:], seed=505)
    assert np.array_equal(a[500:], c)
