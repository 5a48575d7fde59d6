"""Host-side mirror of the reference's `FluidSolver3D` / `FluidMedium` API.

`FluidSolver3D` keeps the reference's names, argument meanings and method
order (src/fluid.rs:52-672) over the C ABI of libaether_fluid.so; state lives
in device memory.  The reference's public `Vec<f64>` fields become properties
that download on read and upload on assignment (the reference test at
src/fluid.rs:935-938 writes `solver.u[id]` directly; here: `u = solver.u;
u[id] = ...; solver.u = u`).  Failed preconditions raise `AetherFluidError`
where the reference panics.
"""
from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import AetherFluidError, AflParams, AflSolveInfo, AflTelemetry, check

_dp = ctypes.POINTER(ctypes.c_double)


class PoissonSolverKind(enum.IntEnum):
    """src/fluid.rs:17-21."""
    ConjugateGradient = 0
    RedBlackGaussSeidel = 1


class Precision(enum.IntEnum):
    FP64 = 0
    MIXED = 1


class SourceKind(enum.IntEnum):
    CYBERPUNK = 0
    SPHERE = 1
    NONE = 2


@dataclass
class FluidTelemetryFrame:
    """src/fluid.rs:7-15."""
    time_sec: float
    kinetic_energy: float
    enstrophy: float
    peak_vorticity: float
    total_mass: float
    center_of_mass: tuple

    @staticmethod
    def from_c(t: AflTelemetry) -> "FluidTelemetryFrame":
        return FluidTelemetryFrame(t.time_sec, t.kinetic_energy, t.enstrophy,
                                   t.peak_vorticity, t.total_mass, tuple(t.center_of_mass))

    def as_array(self) -> np.ndarray:
        return np.array([self.time_sec, self.kinetic_energy, self.enstrophy,
                         self.peak_vorticity, self.total_mass, *self.center_of_mass])


@dataclass
class SolveInfo:
    iterations: int
    refinements: int
    converged: bool
    status: int
    initial_residual: float
    final_residual: float
    rhs_norm: float

    @staticmethod
    def from_c(s: AflSolveInfo) -> "SolveInfo":
        return SolveInfo(s.iterations, s.refinements, bool(s.converged), s.status,
                         s.initial_residual, s.final_residual, s.rhs_norm)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class FluidSolver3D:
    """B200 implementation of `FluidSolver3D` (src/fluid.rs:23-673)."""

    _KNOBS = ("vorticity_eps", "buoyancy_beta", "gravity_alpha", "solver_iters",
              "sor_omega", "cg_rel_tol", "sphere_radius", "sphere_density",
              "sphere_temperature", "fail_on_not_converged", "mixed_inner_iters",
              "mixed_inner_rel_tol", "mixed_max_refinements", "poisson_kernel")

    def __init__(self, nx: int, ny: int, nz: int, precision: Precision = Precision.FP64,
                 **params):
        lib = _lib.load()
        p = _lib.default_params()
        p.precision = int(precision)
        handle = ctypes.c_void_p()
        check(lib.afl_create(nx, ny, nz, ctypes.byref(p), ctypes.byref(handle)))
        self._h = handle
        self._lib = lib
        self.nx, self.ny, self.nz = nx, ny, nz
        self.n = nx * ny * nz
        h = ctypes.c_double()
        check(lib.afl_get_dims(handle, None, None, None, ctypes.byref(h)))
        self.h = h.value
        self.precision = Precision(precision)
        if params:
            self.set_params(**params)

    # -- lifecycle -----------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.afl_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- parameters (public fields of src/fluid.rs:45-49 + extensions) -------
    def _params(self) -> AflParams:
        p = AflParams()
        check(self._lib.afl_get_params(self._h, ctypes.byref(p)))
        return p

    def set_params(self, **kw):
        p = self._params()
        for k, v in kw.items():
            if k == "solver_kind":
                p.solver_kind = int(v)
            elif k == "source_kind":
                p.source_kind = int(v)
            elif k == "sphere_center":
                for a in range(3):
                    p.sphere_center[a] = float(v[a])
            elif k in self._KNOBS:
                setattr(p, k, type(getattr(p, k))(v))
            else:
                raise AttributeError(f"unknown solver parameter {k!r}")
        check(self._lib.afl_set_params(self._h, ctypes.byref(p)))

    def get_params(self) -> dict:
        p = self._params()
        out = {k: getattr(p, k) for k in self._KNOBS}
        out["solver_kind"] = PoissonSolverKind(p.solver_kind)
        out["source_kind"] = SourceKind(p.source_kind)
        out["sphere_center"] = tuple(p.sphere_center)
        out["precision"] = Precision(p.precision)
        return out

    def __getattr__(self, name):
        if name in FluidSolver3D._KNOBS or name in ("solver_kind", "source_kind"):
            return self.get_params()[name]
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name in FluidSolver3D._KNOBS or name in ("solver_kind", "source_kind",
                                                    "sphere_center"):
            self.set_params(**{name: value})
        else:
            object.__setattr__(self, name, value)

    def set_sphere_source(self, center, radius, density=1.0, temperature=1.0,
                          amplitude=None):
        """Switches step() to the sphere source (assignment inside the sphere)."""
        self.set_params(source_kind=SourceKind.SPHERE, sphere_center=center,
                        sphere_radius=radius, sphere_density=density,
                        sphere_temperature=temperature)
        if amplitude is None:
            check(self._lib.afl_set_source_amplitude(self._h, None, 0))
        else:
            a = np.ascontiguousarray(amplitude, dtype=np.float64).ravel()
            check(self._lib.afl_set_source_amplitude(self._h, _ptr(a), a.size))

    # -- fields ----------------------------------------------------------------
    def idx(self, i, j, k):
        """src/fluid.rs:88-90."""
        return (k * self.ny + j) * self.nx + i

    def get_field(self, name: str) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float64)
        check(self._lib.afl_download_field(self._h, _lib.FIELD_IDS[name], _ptr(out), self.n))
        return out

    def set_field(self, name: str, values) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64).ravel()
        if a.size != self.n:
            raise AetherFluidError(1, f"field {name} needs {self.n} values, got {a.size}")
        check(self._lib.afl_upload_field(self._h, _lib.FIELD_IDS[name], _ptr(a), self.n))

    def init_velocity_noise(self, seed: int, lo: float = -0.01, hi: float = 0.01):
        check(self._lib.afl_init_velocity_noise(self._h, seed, lo, hi))

    # -- reference methods -----------------------------------------------------
    def sample_trilinear(self, field, x, y=None, z=None):
        """src/fluid.rs:94-128; `field` is a field name, x may be an (n,3) array."""
        if y is None:
            pts = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
        else:
            pts = np.array([[x, y, z]], dtype=np.float64)
        out = np.empty(pts.shape[0])
        check(self._lib.afl_sample_trilinear(self._h, _lib.FIELD_IDS[field], _ptr(pts),
                                             pts.shape[0], _ptr(out)))
        return out if y is None else float(out[0])

    def advect_maccormack_in_place(self, field_kind: int, dt: float, dissipation: float):
        check(self._lib.afl_advect_maccormack(self._h, field_kind, dt, dissipation))

    def enforce_wall_velocity_bc(self):
        check(self._lib.afl_enforce_wall_bc(self._h))

    def apply_buoyancy_and_vorticity_confinement(self, dt: float):
        check(self._lib.afl_buoyancy_vorticity(self._h, dt))

    def compute_divergence_norm(self) -> float:
        out = ctypes.c_double()
        check(self._lib.afl_divergence_norm(self._h, ctypes.byref(out)))
        return out.value

    def solve_poisson_conjugate_gradient(self, max_iters: int) -> SolveInfo:
        info = AflSolveInfo()
        check(self._lib.afl_solve_cg(self._h, max_iters, ctypes.byref(info)))
        return SolveInfo.from_c(info)

    def solve_poisson_gauss_seidel(self, iterations: int) -> SolveInfo:
        info = AflSolveInfo()
        check(self._lib.afl_solve_rbsor(self._h, iterations, ctypes.byref(info)))
        return SolveInfo.from_c(info)

    def project(self) -> SolveInfo:
        info = AflSolveInfo()
        check(self._lib.afl_project(self._h, ctypes.byref(info)))
        return SolveInfo.from_c(info)

    def inject_cyberpunk_sources(self, time_sec: float, dt: float):
        check(self._lib.afl_inject_cyberpunk(self._h, time_sec, dt))

    def inject_sphere(self):
        check(self._lib.afl_inject_sphere(self._h))

    def step(self, sim_dt: float, timeline_sec: float) -> FluidTelemetryFrame:
        t = AflTelemetry()
        check(self._lib.afl_step(self._h, sim_dt, timeline_sec, ctypes.byref(t), None))
        return FluidTelemetryFrame.from_c(t)

    def step_with_info(self, sim_dt: float, timeline_sec: float):
        t = AflTelemetry()
        info = AflSolveInfo()
        check(self._lib.afl_step(self._h, sim_dt, timeline_sec, ctypes.byref(t),
                                 ctypes.byref(info)))
        return FluidTelemetryFrame.from_c(t), SolveInfo.from_c(info)

    def run(self, steps: int, sim_dt: float, t0: float = 0.0, dt_time: float | None = None):
        """`steps` calls of step() without a host sync between them.  Returns
        (telemetry array [steps, 8], list of SolveInfo)."""
        dt_time = sim_dt if dt_time is None else dt_time
        tel = (AflTelemetry * max(steps, 1))()
        infos = (AflSolveInfo * max(steps, 1))()
        check(self._lib.afl_run(self._h, steps, sim_dt, t0, dt_time, tel, infos))
        arr = np.array([tel[n].as_tuple() for n in range(steps)]).reshape(steps, 8)
        return arr, [SolveInfo.from_c(infos[n]) for n in range(steps)]

    def compute_telemetry(self, timeline_sec: float) -> FluidTelemetryFrame:
        t = AflTelemetry()
        check(self._lib.afl_compute_telemetry(self._h, timeline_sec, ctypes.byref(t)))
        return FluidTelemetryFrame.from_c(t)

    def max_density(self) -> float:
        out = ctypes.c_double()
        check(self._lib.afl_max_density(self._h, ctypes.byref(out)))
        return out.value

    def synchronize(self):
        check(self._lib.afl_synchronize(self._h))

    # -- tracing -----------------------------------------------------------------
    def set_stage_timing(self, enable: bool = True):
        check(self._lib.afl_set_stage_timing(self._h, 1 if enable else 0))

    def stage_timing(self) -> dict:
        """{stage: (device ms, timed calls)} accumulated since set_stage_timing."""
        n = len(_lib.STAGES)
        ms = (ctypes.c_double * n)()
        calls = (ctypes.c_int64 * n)()
        check(self._lib.afl_get_stage_timing(self._h, ms, calls))
        return {name: (ms[i], calls[i]) for i, name in enumerate(_lib.STAGES)}

    def poisson_plan(self) -> dict:
        out = (ctypes.c_int32 * 4)()
        check(self._lib.afl_get_poisson_plan(self._h, out))
        return {"resident": bool(out[0]), "tile": (16, out[1]), "cells_per_thread": out[2],
                "ctas": out[3]}

    def launch_count(self) -> int:
        out = ctypes.c_uint64()
        check(self._lib.afl_get_launch_count(self._h, ctypes.byref(out)))
        return out.value

    @property
    def stream(self) -> int:
        return self._lib.afl_stream(self._h) or 0


def _field_property(name):
    def get(self):
        return self.get_field(name)

    def put(self, values):
        self.set_field(name, values)

    return property(get, put, doc=f"public field `{name}` (download on read, upload on write)")


for _name in _lib.FIELD_IDS:
    setattr(FluidSolver3D, _name, _field_property(_name))


@dataclass
class Aabb:
    min: tuple
    max: tuple


class FluidMedium:
    """The density/temperature hand-off of `FluidMedium::from_solver`
    (src/fluid.rs:703-732): host copies of the two grids, the max density and
    the delta-tracking majorant.  Sampling stays with the CPU renderer."""

    def __init__(self, bounds, nx, ny, nz, density, temperature, max_density,
                 sigma_t_scale, phase_g):
        self.bounds = bounds
        self.nx, self.ny, self.nz = nx, ny, nz
        self.density = density
        self.temperature = temperature
        self.max_density = max_density
        self.sigma_t_scale = sigma_t_scale
        self.majorant_sigma_t = max(max_density * sigma_t_scale, 1e-4)
        self.phase_g = min(max(phase_g, -0.9), 0.9)

    @staticmethod
    def from_solver(solver: FluidSolver3D, bounds, sigma_t_scale: float,
                    phase_g: float) -> "FluidMedium":
        n = solver.n
        dens = np.empty(n)
        temp = np.empty(n)
        mx = ctypes.c_double()
        check(solver._lib.afl_medium_handoff(solver._h, _ptr(dens), _ptr(temp), n,
                                             ctypes.byref(mx)))
        return FluidMedium(bounds, solver.nx, solver.ny, solver.nz, dens, temp, mx.value,
                           sigma_t_scale, phase_g)
