"""Reverse mode through the FP64 smoke step: gradients of
L = 0.5*sum((rho_final - rho_target)^2) with respect to the initial velocity
and the source's temperature amplitude map, checked against central finite
differences of the same forward, a dot-product test of the Jacobian, the
checkpoint interval, and finite differences of the CPU oracle.

The step is piecewise smooth (the MacCormack limiter clamps to the min or max
of 8 cells, scalars pass max(0, .), the near-wall fallback switches on the
backtrace position).  The adjoint differentiates the branch the forward took.
Finite-difference directions therefore live in the control space the solver
itself keeps: velocities vanish on the wall-BC cells (enforce_wall_velocity_bc,
src/fluid.rs:236-253).  A perturbation of those cells breaks ties between the
exact zeros the limiter compares, where central differences average the two
one-sided slopes.  With eps = 1e-6 the differences resolve the recorded
branch; larger eps steps across limiter switches, and the difference error
grows with eps."""
import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu

SHAPE = (20, 24, 18)
STEPS = 6


def wall_masked(u, v, w, shape):
    """enforce_wall_velocity_bc (src/fluid.rs:236-253) on numpy arrays."""
    nx, ny, nz = shape
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ib = (i == 0) | (i + 1 >= nx)
    jb = (j == 0) | (j + 1 >= ny)
    kb = (k == 0) | (k + 1 >= nz)
    mu = (i <= 1) | ib | jb | kb
    mv = (j <= 1) | ib | jb | kb
    mw = (k <= 1) | ib | jb | kb
    return (np.where(mu.ravel(), 0.0, u), np.where(mv.ravel(), 0.0, v),
            np.where(mw.ravel(), 0.0, w))


def controls(shape, seed):
    from aether_fluid.ensemble import rng_f64
    nx, ny, nz = shape
    n = nx * ny * nz
    x = rng_f64(seed, 0, 4 * n)
    u, v, w = (-0.01 + 0.02 * x[a * n:(a + 1) * n] for a in range(3))
    u, v, w = wall_masked(u, v, w, shape)
    amp = 0.5 + x[3 * n:]
    return u, v, w, amp


def source(shape, shift=0.0):
    nx, ny, nz = shape
    return (nx / 2 + shift, 0.1 * ny + 1.0, nz / 2), max(2.5, 5.0 * nx / 64.0)


CG_REL_TOL = 1e-13   # pressure solves well below the difference step
CG_ITERS = 4000
EPS = 1e-6


def make(af, shape, k=4, shift=0.0, poisson_kernel=0):
    from aether_fluid.adjoint import Adjoint
    c, r = source(shape, shift)
    return Adjoint(*shape, center=c, radius=r, checkpoint_every=k, cg_rel_tol=CG_REL_TOL,
                   solver_iters=CG_ITERS, poisson_kernel=poisson_kernel)


@pytest.fixture(scope="module")
def case(af):
    u, v, w, amp = controls(SHAPE, 5)
    dt = 0.5 / max(SHAPE)
    tgt = make(af, SHAPE, shift=3.0).forward(u, v, w, amp, STEPS, dt)
    adj = make(af, SHAPE)
    rho = adj.forward(u, v, w, amp, STEPS, dt)
    grads = adj.backward(rho - tgt)
    return {"x": (u, v, w, amp), "dt": dt, "tgt": tgt, "adj": adj, "rho": rho, "grads": grads}


def loss(adj, x, dt, tgt):
    rho = adj.forward(*x, STEPS, dt)
    return 0.5 * float(np.sum((rho - tgt) ** 2))


def directions(n, count, seed, shape=SHAPE):
    """Unit directions over (u0, v0, w0, amp), velocity parts wall-masked."""
    rng = np.random.default_rng(seed)
    for _ in range(count):
        d = [rng.standard_normal(n) for _ in range(4)]
        d[0], d[1], d[2] = wall_masked(d[0], d[1], d[2], shape)
        nrm = np.sqrt(sum(float(np.dot(a, a)) for a in d))
        yield [a / nrm for a in d]


def central(fun, x, d, eps):
    return (fun([a + eps * b for a, b in zip(x, d)]) -
            fun([a - eps * b for a, b in zip(x, d)])) / (2 * eps)


def test_gradient_matches_finite_differences(af, case):
    adj, x, dt, tgt, g = case["adj"], case["x"], case["dt"], case["tgt"], case["grads"]
    assert all(np.all(np.isfinite(a)) for a in g)
    gnorm = np.sqrt(sum(float(np.dot(a, a)) for a in g))
    assert gnorm > 0
    for d in directions(x[0].size, 6, 11):
        fd = central(lambda xx: loss(adj, xx, dt, tgt), x, d, EPS)
        ad = sum(float(np.dot(a, b)) for a, b in zip(g, d))
        assert abs(fd - ad) <= 1e-3 * max(abs(ad), 1e-3 * gnorm), (fd, ad)


def test_difference_error_shrinks_with_the_step(af, case):
    """Piecewise smoothness: the difference quotient approaches the adjoint
    as eps falls (fewer limiter switches inside the step)."""
    adj, x, dt, tgt, g = case["adj"], case["x"], case["dt"], case["tgt"], case["grads"]
    worst = {1e-4: 0.0, EPS: 0.0}
    for d in directions(x[0].size, 3, 23):
        ad = sum(float(np.dot(a, b)) for a, b in zip(g, d))
        for e in worst:
            fd = central(lambda xx: loss(adj, xx, dt, tgt), x, d, e)
            worst[e] = max(worst[e], abs(fd - ad))
    assert worst[EPS] < worst[1e-4], worst


def test_dot_product(af, case):
    """<J delta, w> (central differences of the final density) equals
    <delta, J^T w> (one backward pass) for a random cotangent w."""
    adj, x, dt = case["adj"], case["x"], case["dt"]
    rng = np.random.default_rng(3)
    wv = rng.standard_normal(x[0].size)
    adj.forward(*x, STEPS, dt)
    jtw = adj.backward(wv)
    for d in directions(x[0].size, 3, 17):
        rp = adj.forward(*[a + EPS * b for a, b in zip(x, d)], STEPS, dt)
        rm = adj.forward(*[a - EPS * b for a, b in zip(x, d)], STEPS, dt)
        lhs = float(np.dot((rp - rm) / (2 * EPS), wv))
        rhs = sum(float(np.dot(a, b)) for a, b in zip(jtw, d))
        assert abs(lhs - rhs) <= 1e-3 * max(abs(rhs), 1e-6), (lhs, rhs)


@pytest.mark.parametrize("k", [1, 3, STEPS])
def test_checkpoint_interval_does_not_change_the_gradient(af, case, k):
    x, dt, tgt = case["x"], case["dt"], case["tgt"]
    a = make(af, SHAPE, k=k)
    rho = a.forward(*x, STEPS, dt)
    assert np.array_equal(rho, case["rho"])
    g = a.backward(rho - tgt)
    for got, ref in zip(g, case["grads"]):
        assert rel_l2(got, ref) <= 1e-9


def test_poisson_kernel_choice_gives_the_same_gradient(af, case):
    """The forward and adjoint pressure solves run on the kernel the params
    name (AUTO takes the resident one at this grid).  The streaming and the
    resident kernel give iteration counts within one per solve of each other
    and the same gradient: they differ only in the order of the inner-product
    sums."""
    x, dt, tgt = case["x"], case["dt"], case["tgt"]
    runs = {}
    for kernel in (1, 2):   # STREAMING, RESIDENT
        a = make(af, SHAPE, poisson_kernel=kernel)
        rho = a.forward(*x, STEPS, dt)
        g = a.backward(rho - tgt)
        runs[kernel] = (rho, g, a.stats())
        a.close()
    (rs, gs, ss), (rr, gr, sr) = runs[1], runs[2]
    assert rel_l2(rs, rr) <= 1e-10 and rel_l2(rr, case["rho"]) <= 1e-12
    assert abs(ss["forward_cg_iters"] - sr["forward_cg_iters"]) <= 2 * STEPS
    assert abs(ss["adjoint_cg_iters"] - sr["adjoint_cg_iters"]) <= STEPS
    for a, b, want in zip(gs, gr, case["grads"]):
        assert rel_l2(a, b) <= 1e-8 and rel_l2(b, want) <= 1e-10


def test_forward_matches_oracle_and_oracle_fd(af, oracle, case):
    """The adjoint's forward is the reference step (oracle to 1e-9), and the
    adjoint gradient agrees with central differences of the f64 CPU oracle."""
    O = oracle
    x, dt, tgt, g = case["x"], case["dt"], case["tgt"], case["grads"]
    c, r = source(SHAPE)

    def oracle_rho(xx):
        s = O.OracleSolver(*SHAPE)
        s.set_params(vorticity_eps=0.3, buoyancy_beta=0.4, gravity_alpha=0.08,
                     solver_kind=O.CG, solver_iters=CG_ITERS, cg_rel_tol=CG_REL_TOL)
        for name, arr in zip(("u", "v", "w"), xx[:3]):
            s.field(name)[:] = arr
        s.set_sphere_source(c, r, 1.0, 1.0, temp_amp=xx[3])
        for n in range(STEPS):
            s.step(dt, n * dt)
        return s.field("density").copy()

    assert rel_l2(oracle_rho(x), case["rho"]) <= 1e-9
    gnorm = np.sqrt(sum(float(np.dot(a, a)) for a in g))
    for d in directions(x[0].size, 2, 29):
        fd = central(lambda xx: 0.5 * float(np.sum((oracle_rho(xx) - tgt) ** 2)), x, d, EPS)
        ad = sum(float(np.dot(a, b)) for a, b in zip(g, d))
        assert abs(fd - ad) <= 1e-3 * max(abs(ad), 1e-3 * gnorm), (fd, ad)


def test_torch_autograd_function(af, case):
    import torch
    from aether_fluid.adjoint import smoke_rollout
    f = smoke_rollout()
    x = [torch.tensor(a, dtype=torch.float64, requires_grad=True) for a in case["x"]]
    rho = f.apply(*x, case["adj"], STEPS, case["dt"])
    L = 0.5 * torch.sum((rho - torch.from_numpy(case["tgt"])) ** 2)
    L.backward()
    for t, ref in zip(x, case["grads"]):
        assert rel_l2(t.grad.numpy(), ref) <= 1e-9


# ---- the reference's jet source and the red-black SOR projection --------------
def oracle_rollout(O, shape, x, steps, dt, source_kind, solver, iters, omega=1.65,
                   center=None, radius=None):
    """The f64 CPU oracle from initial velocity x[:3] (amplitude x[3] for the
    sphere): the final density."""
    s = O.OracleSolver(*shape)
    s.set_params(vorticity_eps=0.3, buoyancy_beta=0.4, gravity_alpha=0.08,
                 solver_kind=O.CG if solver == "cg" else O.RBGS, solver_iters=iters,
                 cg_rel_tol=CG_REL_TOL if solver == "cg" else 0.0, sor_omega=omega)
    for name, arr in zip(("u", "v", "w"), x[:3]):
        s.field(name)[:] = arr
    if source_kind == "sphere":
        s.set_sphere_source(center, radius, 1.0, 1.0, temp_amp=x[3])
    else:
        s.set_source_kind(O.SOURCE_CYBERPUNK)
    for n in range(steps):
        s.step(dt, n * dt)
    return s.field("density").copy()


@pytest.mark.parametrize("source_kind,solver", [("cyberpunk", "cg"), ("sphere", "sor"),
                                                ("cyberpunk", "sor")])
def test_jet_and_sor_adjoints(af, oracle, source_kind, solver):
    """The adjoint through the reference's own source (inject_cyberpunk_sources,
    src/fluid.rs:532-595) and through the red-black SOR projection
    (src/fluid.rs:397-442): the forward equals the oracle's, and the gradient
    agrees with central differences of the GPU forward (3 directions) and of
    the oracle (1 direction).  The jets run at 1.5 cells per step."""
    from aether_fluid.adjoint import Adjoint
    u, v, w, amp = controls(SHAPE, 5)
    dt = (1.5 if source_kind == "cyberpunk" else 0.5) / max(SHAPE)
    center, radius = (SHAPE[0] / 2, 0.1 * SHAPE[1] + 1.0, SHAPE[2] / 2), 3.0
    iters = CG_ITERS if solver == "cg" else 30
    adj = Adjoint(*SHAPE, source=source_kind, solver=solver, checkpoint_every=4,
                  cg_rel_tol=CG_REL_TOL, solver_iters=iters, sor_omega=1.7, center=center,
                  radius=radius)
    x = (u, v, w, amp)
    tu, tv, tw, _ = controls(SHAPE, 6)
    tgt = adj.forward(tu, tv, tw, amp, STEPS, dt)
    rho = adj.forward(*x, STEPS, dt)
    ref = oracle_rollout(oracle, SHAPE, x, STEPS, dt, source_kind, solver, iters, 1.7, center,
                         radius)
    assert rel_l2(rho, ref) <= 1e-9
    g = adj.backward(rho - tgt)
    if source_kind == "cyberpunk":
        assert not np.any(g[3])           # the jets have no amplitude control
    gnorm = np.sqrt(sum(float(np.dot(a, a)) for a in g))
    assert gnorm > 0

    def loss_gpu(xx):
        return 0.5 * float(np.sum((adj.forward(*xx, STEPS, dt) - tgt) ** 2))

    def loss_oracle(xx):
        return 0.5 * float(np.sum((oracle_rollout(oracle, SHAPE, xx, STEPS, dt, source_kind,
                                                  solver, iters, 1.7, center, radius)
                                   - tgt) ** 2))

    for n, d in enumerate(directions(x[0].size, 4, 37)):
        if source_kind == "cyberpunk":
            d[3] = np.zeros_like(d[3])
        ad = sum(float(np.dot(a, b)) for a, b in zip(g, d))
        fd = central(loss_gpu if n < 3 else loss_oracle, x, d, EPS)
        assert abs(fd - ad) <= 1e-3 * max(abs(ad), 1e-3 * gnorm), (n, fd, ad)
    adj.close()


def test_adjoint_c4_reduced_against_oracle_fd(af, oracle):
    """The adjoint workload at reduced size: 32^3, 16 steps, a checkpoint every
    8; controls are the initial velocity (seed-0 noise in [-0.01, 0.01], wall
    BC) and the sphere's temperature amplitude (seed 2, uniform in [0.5, 1.5]);
    L = 0.5*|rho - rho_target|^2, the target's source 3 cells further in x;
    pressure solves to 1e-12.  The adjoint's directional derivative along 4
    seeded directions agrees with central differences (eps 1e-7) of the f64
    CPU oracle to 1e-3."""
    from aether_fluid.adjoint import Adjoint
    from aether_fluid.ensemble import rng_f64
    n, steps = 32, 16
    cells = n ** 3
    dt = 0.5 / n
    center, radius = (n / 2, 0.1 * n, n / 2), 5.0 * n / 64.0
    noise = rng_f64(0, 0, 3 * cells)

    def make_c4(cx):
        return Adjoint(n, n, n, center=(cx, center[1], center[2]), radius=radius,
                       checkpoint_every=8, cg_rel_tol=1e-12, solver_iters=4000)

    adj = make_c4(center[0])
    u, v, w = adj.wall_masked(*(-0.01 + 0.02 * noise[a * cells:(a + 1) * cells]
                                for a in range(3)))
    x = (u, v, w, 0.5 + rng_f64(2, 0, cells))
    t = make_c4(center[0] + 3.0)
    tgt = t.forward(*x, steps, dt)
    t.close()
    rho = adj.forward(*x, steps, dt)
    g = adj.backward(rho - tgt)

    def loss_oracle(xx):
        s = oracle.OracleSolver(n, n, n)
        s.set_params(vorticity_eps=0.3, buoyancy_beta=0.4, gravity_alpha=0.08,
                     solver_kind=oracle.CG, solver_iters=4000, cg_rel_tol=1e-12)
        for name, arr in zip(("u", "v", "w"), xx[:3]):
            s.field(name)[:] = arr
        s.set_sphere_source(center, radius, 1.0, 1.0, temp_amp=xx[3])
        for k in range(steps):
            s.step(dt, k * dt)
        return 0.5 * float(np.sum((s.field("density") - tgt) ** 2))

    rng = np.random.default_rng(11)
    for _ in range(4):
        d = [rng.standard_normal(cells) for _ in range(4)]
        d[0], d[1], d[2] = adj.wall_masked(d[0], d[1], d[2])
        nrm = np.sqrt(sum(float(np.dot(a, a)) for a in d))
        d = [a / nrm for a in d]
        ad = sum(float(np.dot(a, b)) for a, b in zip(g, d))
        fd = central(loss_oracle, x, d, 1e-7)
        assert abs(fd - ad) <= 1e-3 * abs(ad), (fd, ad)
    adj.close()
