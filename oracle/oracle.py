"""ctypes view of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is the f64 C++ restatement of the reference smoke solver
(`src/fluid.rs:23-673`, `src/rng.rs:5-88` of vanovri/aether-core-engine) in
`oracle/fluid_oracle.cpp`.  Only `tests/`, `__graft_entry__.smoke()` and the
CPU-baseline leg of `bench.py` import this module, and only to check results;
the product library never calls it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_fluid.so")
SRC = os.path.join(HERE, "fluid_oracle.cpp")

FIELDS = ("u", "v", "w", "density", "temperature", "pressure", "divergence")
CG, RBGS = 0, 1
SOURCE_CYBERPUNK, SOURCE_SPHERE, SOURCE_NONE = 0, 1, 2

_c_double_p = ctypes.POINTER(ctypes.c_double)


def build(force: bool = False) -> str:
    """Compile the oracle with the flags that keep rustc's f64 semantics."""
    if force or not os.path.exists(LIB_PATH) or (
        os.path.getmtime(LIB_PATH) < os.path.getmtime(SRC)
    ):
        cmd = [
            "g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math",
            "-fPIC", "-shared", "-Wall", "-o", LIB_PATH, SRC,
        ]
        subprocess.check_call(cmd, cwd=HERE)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        sz = ctypes.c_size_t
        vp = ctypes.c_void_p
        d = ctypes.c_double
        i = ctypes.c_int
        L.ofl_create.restype = vp
        L.ofl_create.argtypes = [sz, sz, sz]
        L.ofl_destroy.argtypes = [vp]
        L.ofl_h.restype = d
        L.ofl_h.argtypes = [vp]
        L.ofl_cells.restype = sz
        L.ofl_cells.argtypes = [vp]
        L.ofl_field.restype = _c_double_p
        L.ofl_field.argtypes = [vp, i]
        L.ofl_set_params.argtypes = [vp, d, d, d, i, i, d, d]
        L.ofl_set_sphere_source.argtypes = [vp, d, d, d, d, d, d, _c_double_p]
        L.ofl_set_source_kind.argtypes = [vp, i]
        L.ofl_advect_maccormack.argtypes = [vp, i, d, d]
        L.ofl_enforce_wall_bc.argtypes = [vp]
        L.ofl_buoyancy_vorticity.argtypes = [vp, d]
        L.ofl_divergence_norm.restype = d
        L.ofl_divergence_norm.argtypes = [vp]
        L.ofl_solve_cg.restype = i
        L.ofl_solve_cg.argtypes = [vp, i, _c_double_p]
        L.ofl_solve_rbgs.argtypes = [vp, i]
        L.ofl_project.restype = i
        L.ofl_project.argtypes = [vp]
        L.ofl_inject_cyberpunk.argtypes = [vp, d, d]
        L.ofl_inject_sphere.argtypes = [vp]
        L.ofl_step.argtypes = [vp, d, d, _c_double_p]
        L.ofl_compute_telemetry.argtypes = [vp, d, _c_double_p]
        L.ofl_max_density.restype = d
        L.ofl_max_density.argtypes = [vp]
        L.ofl_last_cg_iters.restype = i
        L.ofl_last_cg_iters.argtypes = [vp]
        L.ofl_run.restype = ctypes.c_long
        L.ofl_run.argtypes = [vp, i, d, d, d, _c_double_p]
        L.ofl_init_velocity_noise.argtypes = [vp, ctypes.c_uint64, d, d]
        L.ofl_rng_u64.argtypes = [ctypes.c_uint64, sz, ctypes.POINTER(ctypes.c_uint64)]
        L.ofl_rng_f64.argtypes = [ctypes.c_uint64, sz, _c_double_p]
        L.ofl_medium_sample.argtypes = [_c_double_p, _c_double_p, sz, sz, sz, _c_double_p,
                                        _c_double_p, _c_double_p, sz, _c_double_p, _c_double_p]
        L.ofl_medium_transmittance.argtypes = [_c_double_p, _c_double_p, sz, sz, sz, _c_double_p,
                                               _c_double_p, d, _c_double_p, sz, ctypes.c_uint64,
                                               _c_double_p]
        L.ofl_medium_interaction.argtypes = [_c_double_p, _c_double_p, sz, sz, sz, _c_double_p,
                                             _c_double_p, d, _c_double_p, sz, ctypes.c_uint64,
                                             ctypes.POINTER(ctypes.c_int32), _c_double_p,
                                             _c_double_p, _c_double_p]
        _lib = L
    return _lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_c_double_p)


class OracleSolver:
    """Mirror of `FluidSolver3D` over the C++ restatement (src/fluid.rs:52-85)."""

    def __init__(self, nx: int, ny: int, nz: int):
        L = lib()
        self._h = L.ofl_create(nx, ny, nz)
        if not self._h:
            raise ValueError("grid dimensions must all be >= 6 (src/fluid.rs:54)")
        self.nx, self.ny, self.nz = nx, ny, nz
        self.h = L.ofl_h(self._h)
        self.n = nx * ny * nz
        self.vorticity_eps, self.buoyancy_beta, self.gravity_alpha = 5.5, 6.8, 0.45
        self.solver_kind, self.solver_iters = CG, 32
        self.sor_omega, self.cg_rel_tol = 1.65, 0.0
        self._push()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().ofl_destroy(h)
            self._h = None

    def _push(self):
        lib().ofl_set_params(
            self._h, self.vorticity_eps, self.buoyancy_beta, self.gravity_alpha,
            self.solver_kind, self.solver_iters, self.sor_omega, self.cg_rel_tol,
        )

    def set_params(self, **kw):
        for k, v in kw.items():
            if not hasattr(self, k):
                raise AttributeError(k)
            setattr(self, k, v)
        self._push()

    def field(self, name: str) -> np.ndarray:
        """Writable numpy view of a public field (x fastest)."""
        ptr = lib().ofl_field(self._h, FIELDS.index(name))
        return np.ctypeslib.as_array(ptr, shape=(self.n,))

    def idx(self, i, j, k):
        return (k * self.ny + j) * self.nx + i

    def set_sphere_source(self, center, radius, rho=1.0, temp=1.0, temp_amp=None):
        amp = None
        if temp_amp is not None:
            self._amp = np.ascontiguousarray(temp_amp, dtype=np.float64)
            amp = _dptr(self._amp)
        lib().ofl_set_sphere_source(self._h, *map(float, center), float(radius),
                                    float(rho), float(temp), amp)
        lib().ofl_set_source_kind(self._h, SOURCE_SPHERE)

    def set_source_kind(self, kind: int):
        lib().ofl_set_source_kind(self._h, kind)

    def advect_maccormack_in_place(self, field_kind, dt, dissipation):
        lib().ofl_advect_maccormack(self._h, field_kind, dt, dissipation)

    def enforce_wall_velocity_bc(self):
        lib().ofl_enforce_wall_bc(self._h)

    def apply_buoyancy_and_vorticity_confinement(self, dt):
        lib().ofl_buoyancy_vorticity(self._h, dt)

    def compute_divergence_norm(self) -> float:
        return lib().ofl_divergence_norm(self._h)

    def solve_poisson_conjugate_gradient(self, max_iters) -> int:
        return lib().ofl_solve_cg(self._h, max_iters, None)

    def solve_poisson_gauss_seidel(self, iterations):
        lib().ofl_solve_rbgs(self._h, iterations)

    def project(self) -> int:
        return lib().ofl_project(self._h)

    def inject_cyberpunk_sources(self, time_sec, dt):
        lib().ofl_inject_cyberpunk(self._h, time_sec, dt)

    def inject_sphere(self):
        lib().ofl_inject_sphere(self._h)

    def step(self, dt, time_sec) -> np.ndarray:
        t = np.zeros(8)
        lib().ofl_step(self._h, dt, time_sec, _dptr(t))
        return t

    def compute_telemetry(self, time_sec) -> np.ndarray:
        t = np.zeros(8)
        lib().ofl_compute_telemetry(self._h, time_sec, _dptr(t))
        return t

    def max_density(self) -> float:
        return lib().ofl_max_density(self._h)

    def last_cg_iters(self) -> int:
        return lib().ofl_last_cg_iters(self._h)

    def run(self, steps, dt, t0=0.0, dt_time=None, telemetry=False):
        dt_time = dt if dt_time is None else dt_time
        tel = np.zeros((steps, 8)) if telemetry else None
        total = lib().ofl_run(self._h, steps, dt, t0, dt_time,
                              _dptr(tel) if tel is not None else None)
        return (total, tel) if telemetry else total

    def init_velocity_noise(self, seed, lo=-0.01, hi=0.01):
        lib().ofl_init_velocity_noise(self._h, seed, lo, hi)


def rng_u64(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, dtype=np.uint64)
    lib().ofl_rng_u64(seed, n, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
    return out


def rng_f64(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n)
    lib().ofl_rng_f64(seed, n, _dptr(out))
    return out


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def medium_sample(dens, temp, shape, bmin, bmax, points):
    """FluidMedium::sample_density_and_temp (src/fluid.rs:739-786) at points [n, 3]."""
    dens, temp, pts = _f64(dens).ravel(), _f64(temp).ravel(), _f64(points).reshape(-1, 3)
    n = pts.shape[0]
    rho, tmp = np.zeros(n), np.zeros(n)
    lib().ofl_medium_sample(_dptr(dens), _dptr(temp), *shape, _dptr(_f64(bmin)),
                            _dptr(_f64(bmax)), _dptr(pts), n, _dptr(rho), _dptr(tmp))
    return rho, tmp


def medium_transmittance(dens, temp, shape, bmin, bmax, sigma_t_scale, rays, seed):
    """FluidMedium::transmittance (src/fluid.rs:840-874) per ray; rays [n, 8] =
    origin, dir, t_min, t_end; ray r uses Rng::from_seed(seed + r)."""
    dens, temp, r = _f64(dens).ravel(), _f64(temp).ravel(), _f64(rays).reshape(-1, 8)
    n = r.shape[0]
    tr = np.zeros(n)
    lib().ofl_medium_transmittance(_dptr(dens), _dptr(temp), *shape, _dptr(_f64(bmin)),
                                   _dptr(_f64(bmax)), sigma_t_scale, _dptr(r), n, seed, _dptr(tr))
    return tr


def medium_interaction(dens, temp, shape, bmin, bmax, sigma_t_scale, rays, seed):
    """FluidMedium::sample_interaction (src/fluid.rs:792-838) per ray: (hit, t,
    density, temperature)."""
    dens, temp, r = _f64(dens).ravel(), _f64(temp).ravel(), _f64(rays).reshape(-1, 8)
    n = r.shape[0]
    hit = np.zeros(n, dtype=np.int32)
    t, rho, tmp = np.zeros(n), np.zeros(n), np.zeros(n)
    lib().ofl_medium_interaction(_dptr(dens), _dptr(temp), *shape, _dptr(_f64(bmin)),
                                 _dptr(_f64(bmax)), sigma_t_scale, _dptr(r), n, seed,
                                 hit.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), _dptr(t),
                                 _dptr(rho), _dptr(tmp))
    return hit, t, rho, tmp
