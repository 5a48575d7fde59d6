"""Per-stage parity of the CUDA path against the oracle on small grids.

FP64: stages whose reference arithmetic is pointwise or a fixed-order stencil
(advection, wall BC, confinement/buoyancy, divergence field, projection
gradient, RB-SOR sweeps, sphere source, trilinear sampling, max) must match
bit for bit (the FP64 kernels are built without FMA contraction).  Stages with
a reduction (CG inner products, RMS, telemetry sums) or a libm call on the
device (exp in the cyberpunk jets) are compared within a stated tolerance.
MIXED: the same stages in f32 within 1e-5 relative L2 of the f64 oracle.
"""
import numpy as np
import pytest

from helpers import max_abs, rel_l2

pytestmark = pytest.mark.gpu

SHAPES = [(6, 6, 6), (18, 22, 18), (33, 17, 25)]
VEL = ("u", "v", "w")
SCAL = ("density", "temperature")


def seeded_state(shape, seed, vel_scale):
    nx, ny, nz = shape
    n = nx * ny * nz
    rng = np.random.default_rng(seed)
    st = {f: rng.uniform(-vel_scale, vel_scale, n) for f in VEL}
    st["density"] = rng.uniform(0.0, 2.0, n)
    st["temperature"] = rng.uniform(0.0, 1.5, n)
    st["pressure"] = rng.standard_normal(n) * 0.01
    # A right-hand side the singular Neumann operator can match: zero off the
    # interior and zero-mean on it (a divergence field of walled velocities
    # has both properties).
    b = np.zeros((nz, ny, nx))
    inner = rng.standard_normal((nz - 2, ny - 2, nx - 2)) * 0.01
    b[1:-1, 1:-1, 1:-1] = inner - inner.mean()
    st["divergence"] = b.ravel()
    return st


def pair(af, O, shape, seed=0, vel_scale=1.0, precision=0, **params):
    nx, ny, nz = shape
    g = af.FluidSolver3D(nx, ny, nz, precision=precision)
    o = O.OracleSolver(nx, ny, nz)
    if params:
        g.set_params(**params)
        o.set_params(**{k: v for k, v in params.items()
                        if k not in ("source_kind", "poisson_kernel")})
    st = seeded_state(shape, seed, vel_scale)
    for f, vals in st.items():
        g.set_field(f, vals)
        o.field(f)[:] = vals
    return g, o


def same(g, o, fields, precision=0, tol=1e-5):
    for f in fields:
        a, ref = g.get_field(f), o.field(f)
        if precision == 0:
            assert np.array_equal(a, ref), (f, max_abs(a, ref))
        else:
            assert rel_l2(a, ref) <= tol, (f, rel_l2(a, ref))


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("precision", [0, 1])
def test_advect_maccormack(af, oracle, shape, kind, precision):
    # dt/h * |u| reaches ~2 cells: exercises clamping, the near-wall fallback
    # and the extrema clamp.
    g, o = pair(af, oracle, shape, seed=kind, vel_scale=1.0, precision=precision)
    dt = 2.0 * g.h
    g.advect_maccormack_in_place(kind, dt, 0.985)
    o.advect_maccormack_in_place(kind, dt, 0.985)
    name = ("u", "v", "w", "density", "temperature")[kind]
    same(g, o, [name, "u", "v", "w"], precision, tol=2e-6)


# Grids of several 32 x 8 tiles and z chunks: rows 16-byte aligned or not (nx
# a multiple of 4, even, odd), ragged tiles in x and y.
TILE_SHAPES = [(64, 24, 40), (70, 36, 33), (45, 17, 50)]


@pytest.mark.parametrize("shape", TILE_SHAPES)
@pytest.mark.parametrize("steps_per_cell", [0.4, 3.0])
@pytest.mark.parametrize("precision", [0, 1])
def test_advection_tiles(af, oracle, shape, steps_per_cell, precision):
    """Advection of all five fields over many tiles, at 0.4 and 3 cells per
    step; FP64 matches the oracle bit for bit."""
    g, o = pair(af, oracle, shape, seed=41, vel_scale=1.0, precision=precision)
    dt = steps_per_cell * g.h
    for kind in range(5):
        g.advect_maccormack_in_place(kind, dt, 0.99)
        o.advect_maccormack_in_place(kind, dt, 0.99)
    same(g, o, ["u", "v", "w", "density", "temperature"], precision, tol=2e-6)


# Grids far larger than L2 for the shared-memory-staged forces kernel (many z
# chunks; 16-byte rows, and odd nx for the element-wise copies) and the x4
# divergence/projection kernels (nx a multiple of 128).
STREAM_FORCES = [((176, 160, 160), 0), ((177, 160, 160), 0), ((224, 200, 200), 1)]


@pytest.mark.parametrize("shape,precision", STREAM_FORCES,
                         ids=["176x160x160-fp64", "177x160x160-fp64", "224x200x200-mixed"])
def test_staged_forces_large(af, oracle, shape, precision):
    g, o = pair(af, oracle, shape, seed=43, vel_scale=0.5, precision=precision,
                vorticity_eps=0.3, buoyancy_beta=0.4, gravity_alpha=0.08)
    g.apply_buoyancy_and_vorticity_confinement(0.02)
    o.apply_buoyancy_and_vorticity_confinement(0.02)
    same(g, o, VEL, precision, tol=1e-5)


@pytest.mark.parametrize("precision", [0, 1])
def test_x4_divergence_and_projection_large(af, oracle, precision):
    """256 x 256 x 208: the divergence and the projection gradient on runs of
    4 cells per thread (FP64 bit for bit; mixed within 1e-5)."""
    shape = (256, 256, 208)
    g, o = pair(af, oracle, shape, seed=47, vel_scale=0.5, precision=precision,
                solver_kind=1, solver_iters=2, sor_omega=1.7)
    rg, ro = g.compute_divergence_norm(), o.compute_divergence_norm()
    assert abs(rg - ro) <= (1e-13 if precision == 0 else 1e-5) * ro
    same(g, o, ["divergence"], precision, tol=1e-5)
    g.project()
    o.project()
    same(g, o, ["u", "v", "w", "pressure"], precision, tol=1e-5)


@pytest.mark.parametrize("shape", SHAPES)
def test_wall_bc(af, oracle, shape):
    g, o = pair(af, oracle, shape, seed=7)
    g.enforce_wall_velocity_bc()
    o.enforce_wall_velocity_bc()
    same(g, o, VEL)


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("precision", [0, 1])
def test_buoyancy_vorticity(af, oracle, shape, precision):
    g, o = pair(af, oracle, shape, seed=11, vel_scale=0.3, precision=precision,
                vorticity_eps=0.3, buoyancy_beta=0.4, gravity_alpha=0.08)
    g.apply_buoyancy_and_vorticity_confinement(0.05)
    o.apply_buoyancy_and_vorticity_confinement(0.05)
    same(g, o, VEL, precision, tol=1e-5)


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("precision", [0, 1])
def test_divergence(af, oracle, shape, precision):
    g, o = pair(af, oracle, shape, seed=13, precision=precision)
    rg = g.compute_divergence_norm()
    ro = o.compute_divergence_norm()
    assert abs(rg - ro) <= 1e-13 * ro if precision == 0 else abs(rg - ro) <= 1e-5 * ro
    same(g, o, ["divergence"], precision, tol=1e-5)


@pytest.mark.parametrize("shape", SHAPES)
def test_rbsor_bit_exact(af, oracle, shape):
    g, o = pair(af, oracle, shape, seed=17, sor_omega=1.7)
    info = g.solve_poisson_gauss_seidel(25)
    o.solve_poisson_gauss_seidel(25)
    assert info.iterations == 25
    same(g, o, ["pressure"])


@pytest.mark.parametrize("shape", SHAPES)
def test_rbsor_mixed(af, oracle, shape):
    g, o = pair(af, oracle, shape, seed=17, precision=1, sor_omega=1.7)
    g.solve_poisson_gauss_seidel(25)
    o.solve_poisson_gauss_seidel(25)
    same(g, o, ["pressure"], precision=1, tol=1e-5)


KERNELS = {"streaming": 1, "resident": 2}


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("kernel", ["streaming", "resident"])
def test_cg_fixed_iterations(af, oracle, shape, kernel):
    """Reference stopping rule (absolute), fixed iteration budget: the only
    difference is the summation order of the two inner products."""
    g, o = pair(af, oracle, shape, seed=19, poisson_kernel=KERNELS[kernel])
    info = g.solve_poisson_conjugate_gradient(30)
    it = o.solve_poisson_conjugate_gradient(30)
    assert info.iterations == it
    a, ref = g.get_field("pressure"), o.field("pressure")
    assert rel_l2(a, ref) <= 1e-11, rel_l2(a, ref)


@pytest.mark.parametrize("shape", [(18, 22, 18), (33, 17, 25)])
@pytest.mark.parametrize("kernel", ["streaming", "resident"])
def test_cg_relative_tolerance(af, oracle, shape, kernel):
    g, o = pair(af, oracle, shape, seed=23, cg_rel_tol=1e-6, poisson_kernel=KERNELS[kernel])
    info = g.solve_poisson_conjugate_gradient(500)
    it = o.solve_poisson_conjugate_gradient(500)
    assert info.converged and abs(info.iterations - it) <= 1
    assert info.final_residual <= 1e-6 * info.rhs_norm * (1 + 1e-12)
    assert rel_l2(g.get_field("pressure"), o.field("pressure")) <= 1e-8


@pytest.mark.parametrize("shape", [(18, 22, 18), (33, 17, 25)])
@pytest.mark.parametrize("kernel", ["streaming", "resident"])
def test_cg_mixed_refinement(af, oracle, shape, kernel):
    """The mixed solve reaches the f64 tolerance in f64 (true residual)."""
    g, o = pair(af, oracle, shape, seed=29, precision=1, cg_rel_tol=1e-6, solver_iters=2000,
                poisson_kernel=KERNELS[kernel])
    info = g.solve_poisson_conjugate_gradient(2000)
    assert info.converged, info
    assert info.final_residual <= 1e-6 * info.rhs_norm
    o.solve_poisson_conjugate_gradient(2000)
    # Both solutions satisfy the same residual bound; the Neumann operator is
    # singular, so compare modulo the mean.
    a = g.get_field("pressure")
    ref = o.field("pressure").copy()
    assert rel_l2(a - a.mean(), ref - ref.mean()) <= 1e-4


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("kind", ["cg", "rbgs"])
def test_project(af, oracle, shape, kind):
    k = 0 if kind == "cg" else 1
    g, o = pair(af, oracle, shape, seed=31, solver_kind=k, solver_iters=20)
    g.project()
    o.project()
    if kind == "rbgs":
        same(g, o, VEL + ("pressure",))
    else:
        for f in VEL + ("pressure",):
            assert rel_l2(g.get_field(f), o.field(f)) <= 1e-11, f


@pytest.mark.parametrize("shape", SHAPES)
def test_inject_cyberpunk(af, oracle, shape):
    g, o = pair(af, oracle, shape, seed=37)
    for t in (0.0, 0.5, 3.7):
        g.inject_cyberpunk_sources(t, 0.1)
        o.inject_cyberpunk_sources(t, 0.1)
    # the device exp() may differ from glibc's in the last bit
    for f in VEL + SCAL:
        assert max_abs(g.get_field(f), o.field(f)) <= 1e-14, f


@pytest.mark.parametrize("shape", SHAPES)
def test_inject_sphere(af, oracle, shape):
    g, o = pair(af, oracle, shape, seed=41)
    c = (shape[0] / 2 + 0.3, 0.1 * shape[1], shape[2] / 2 - 0.2)
    r = max(1.5, 5.0 * shape[0] / 64)
    amp = np.random.default_rng(3).uniform(0.5, 1.5, g.n)
    g.set_sphere_source(c, r, 1.0, 1.0, amplitude=amp)
    o.set_sphere_source(c, r, 1.0, 1.0, temp_amp=amp)
    g.inject_sphere()
    o.inject_sphere()
    same(g, o, SCAL)


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("precision", [0, 1])
def test_telemetry(af, oracle, shape, precision):
    g, o = pair(af, oracle, shape, seed=43, precision=precision)
    tg = g.compute_telemetry(1.25).as_array()
    to = o.compute_telemetry(1.25)
    tol = 1e-12 if precision == 0 else 1e-6
    assert tg[0] == to[0]
    assert np.allclose(tg[1:], to[1:], rtol=tol, atol=1e-300), (tg, to)


@pytest.mark.parametrize("shape", SHAPES)
def test_max_density_and_handoff(af, oracle, shape):
    g, o = pair(af, oracle, shape, seed=47)
    assert g.max_density() == o.max_density()
    m = af.FluidMedium.from_solver(g, af.Aabb((-2, 0.2, -2), (2, 4.8, 1.3)), 0.85, 0.32)
    assert m.max_density == o.max_density()
    assert np.array_equal(m.density, o.field("density"))
    assert np.array_equal(m.temperature, o.field("temperature"))
    assert m.majorant_sigma_t == max(o.max_density() * 0.85, 1e-4)


@pytest.mark.parametrize("shape", SHAPES)
def test_sample_trilinear(af, oracle, shape):
    """sample_trilinear (src/fluid.rs:94-128) at points inside, on and outside
    the clamped range, against a numpy restatement over the oracle's field."""
    g, o = pair(af, oracle, shape, seed=53)
    nx, ny, nz = shape
    rng = np.random.default_rng(1)
    pts = np.stack([rng.uniform(-2, nx + 2, 500), rng.uniform(-2, ny + 2, 500),
                    rng.uniform(-2, nz + 2, 500)], axis=1)
    got = g.sample_trilinear("density", pts)
    f = o.field("density")
    want = []
    for x, y, z in pts:
        xc = min(max(x, 0.5), nx - 1.500001)
        yc = min(max(y, 0.5), ny - 1.500001)
        zc = min(max(z, 0.5), nz - 1.500001)
        i0, j0, k0 = int(np.floor(xc)), int(np.floor(yc)), int(np.floor(zc))
        tx, ty, tz = xc - i0, yc - j0, zc - k0
        c = lambda i, j, k: f[(k * ny + j) * nx + i]  # noqa: E731
        c00 = c(i0, j0, k0) * (1.0 - tx) + c(i0 + 1, j0, k0) * tx
        c10 = c(i0, j0 + 1, k0) * (1.0 - tx) + c(i0 + 1, j0 + 1, k0) * tx
        c01 = c(i0, j0, k0 + 1) * (1.0 - tx) + c(i0 + 1, j0, k0 + 1) * tx
        c11 = c(i0, j0 + 1, k0 + 1) * (1.0 - tx) + c(i0 + 1, j0 + 1, k0 + 1) * tx
        c0 = c00 * (1.0 - ty) + c10 * ty
        c1 = c01 * (1.0 - ty) + c11 * ty
        want.append(c0 * (1.0 - tz) + c1 * tz)
    assert np.array_equal(got, np.array(want))


@pytest.mark.parametrize("shape", [(128, 128, 128), (96, 96, 96), (64, 128, 64), (48, 48, 48)])
@pytest.mark.parametrize("precision", [0, 1])
def test_resident_matches_streaming_at_full_size(af, shape, precision):
    """At the workload sizes the resident and streaming kernels solve the same
    system: 60 fixed iterations agree to summation-order rounding."""
    nx, ny, nz = shape
    st = seeded_state(shape, 61, 1.0)
    out = {}
    for kernel in ("streaming", "resident"):
        g = af.FluidSolver3D(nx, ny, nz, precision=precision, poisson_kernel=KERNELS[kernel],
                             mixed_inner_iters=60, mixed_max_refinements=1)
        g.set_field("divergence", st["divergence"])
        g.set_field("pressure", st["pressure"])
        info = g.solve_poisson_conjugate_gradient(60)
        assert info.iterations == 60, info
        out[kernel] = (g.get_field("pressure"), info)
    tol = 1e-10 if precision == 0 else 1e-4
    assert rel_l2(out["resident"][0], out["streaming"][0]) <= tol
    fr, fs = out["resident"][1].final_residual, out["streaming"][1].final_residual
    assert abs(fr - fs) <= (1e-8 if precision == 0 else 1e-2) * fs


# Shapes that reach every tile plan of the resident kernel (16 x TY columns,
# CPT z cells per thread): TY = 16 needs a wide grid (TY = 4 and 8 would need
# more tiles than SMs), ragged x/y tile edges, and a shallow grid.
PLAN_SHAPES = {(160, 200, 32): 16, (100, 90, 120): 8, (130, 12, 7): 8, (37, 45, 29): 4}


@pytest.mark.parametrize("shape", sorted(PLAN_SHAPES))
@pytest.mark.parametrize("precision", [0, 1])
def test_resident_tile_plans(af, shape, precision):
    """Every tile plan solves the same system as the streaming kernel."""
    nx, ny, nz = shape
    st = seeded_state(shape, 67, 1.0)
    out = {}
    for kernel in ("streaming", "resident"):
        g = af.FluidSolver3D(nx, ny, nz, precision=precision, poisson_kernel=KERNELS[kernel],
                             mixed_inner_iters=40, mixed_max_refinements=1)
        if kernel == "resident":
            plan = g.poisson_plan()
            assert plan["resident"] and plan["tile"][1] == PLAN_SHAPES[shape], plan
        g.set_field("divergence", st["divergence"])
        g.set_field("pressure", st["pressure"])
        info = g.solve_poisson_conjugate_gradient(40)
        assert info.iterations == 40, info
        out[kernel] = g.get_field("pressure")
    tol = 1e-10 if precision == 0 else 1e-4
    assert rel_l2(out["resident"], out["streaming"]) <= tol


@pytest.mark.parametrize("shape", sorted(PLAN_SHAPES) + [(128, 128, 128)])
@pytest.mark.parametrize("precision", [0, 1])
def test_resident_sor_matches_streaming(af, shape, precision):
    """RB-SOR on the resident tiles equals the streaming sweep: bit for bit in
    FP64 (each colour reads only the other colour, so the visiting order does
    not matter); the mixed form to f32 rounding."""
    nx, ny, nz = shape
    st = seeded_state(shape, 71, 1.0)
    out = {}
    for kernel in ("streaming", "resident"):
        g = af.FluidSolver3D(nx, ny, nz, precision=precision, poisson_kernel=KERNELS[kernel])
        g.set_params(solver_kind=1, sor_omega=1.7)
        g.set_field("divergence", st["divergence"])
        g.set_field("pressure", st["pressure"])
        g.solve_poisson_gauss_seidel(25)
        out[kernel] = g.get_field("pressure")
    if precision == 0:
        assert np.array_equal(out["resident"], out["streaming"])
    else:
        assert rel_l2(out["resident"], out["streaming"]) <= 1e-5


@pytest.mark.parametrize("shape", [(40, 36, 30), (64, 24, 40)])
@pytest.mark.parametrize("kind", [0, 3])
def test_nan_velocity_cell_matches_oracle(af, oracle, shape, kind):
    """A velocity field that has blown up (a NaN at an interior cell): the
    backtrace of that cell has a NaN position, which the reference's
    `floor() as usize` turns into cell 0.  FP64 advection gives the oracle's
    fields, NaNs in the same places, and the handle stays usable."""
    g, o = pair(af, oracle, shape, seed=7, vel_scale=1.0)
    nx, ny, nz = shape
    c = ((nz // 2) * ny + ny // 2) * nx + nx // 2
    for s in (g, o):
        if s is g:
            u = g.get_field("u")
            u[c] = np.nan
            g.set_field("u", u)
        else:
            o.field("u")[c] = np.nan
    dt = 1.5 * g.h
    g.advect_maccormack_in_place(kind, dt, 0.985)
    o.advect_maccormack_in_place(kind, dt, 0.985)
    name = ("u", "v", "w", "density", "temperature")[kind]
    for f in (name, "u", "v", "w"):
        a, ref = g.get_field(f), o.field(f)
        assert np.array_equal(a, ref, equal_nan=True), (f, np.isnan(a).sum(), np.isnan(ref).sum())
    g.advect_maccormack_in_place(1, dt, 0.985)   # the handle still runs kernels


@pytest.mark.parametrize("kind", [0, 3])
def test_nan_velocity_cell_mixed_runs(af, kind):
    """The same in the mixed form (its f32 backtrace takes the corner from the
    displacement): the kernels run, and the NaN reaches only the cells whose
    samples include it."""
    shape = (40, 36, 30)
    g = af.FluidSolver3D(*shape, precision=1)
    st = seeded_state(shape, 7, 1.0)
    for f, vals in st.items():
        g.set_field(f, vals)
    u = g.get_field("u")
    c = (15 * 36 + 18) * 40 + 20
    u[c] = np.nan
    g.set_field("u", u)
    g.advect_maccormack_in_place(kind, 1.5 * g.h, 0.985)
    name = ("u", "v", "w", "density", "temperature")[kind]
    out = g.get_field(name)
    assert np.isnan(out).sum() < out.size // 100
    g.advect_maccormack_in_place(1, 1.5 * g.h, 0.985)
