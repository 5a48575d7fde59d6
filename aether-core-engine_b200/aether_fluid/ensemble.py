"""Batched ensembles of independent smoke plumes (include/aether_fluid.h,
afl_ensemble_*): by default a step is one persistent cooperative launch over
all instances; the other form runs every stage as one launch over all
instances with the pressure solves in one cooperative launch.  Either way a
step is a replayed CUDA graph."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import AflInstance, AflSolveInfo, AflTelemetry, check
from .solver import Precision, SolveInfo


@dataclass
class InstanceSpec:
    nx: int
    ny: int
    nz: int
    seed: int
    alpha: float = 0.08
    beta: float = 0.4
    eps: float = 0.3
    center: tuple = None
    radius: float = None
    noise: float = 0.01

    def __post_init__(self):
        if self.center is None:
            self.center = (self.nx / 2, 0.1 * self.ny, self.nz / 2)
        if self.radius is None:
            self.radius = 5.0 * self.nx / 64.0

    @property
    def h(self) -> float:
        return 1.0 / max(self.nx, self.ny, self.nz)

    @property
    def dt(self) -> float:
        return 0.5 * self.h

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    def to_c(self) -> AflInstance:
        c = AflInstance()
        c.nx, c.ny, c.nz = self.nx, self.ny, self.nz
        c.seed = self.seed
        c.noise_lo, c.noise_hi = -self.noise, self.noise
        c.dt = self.dt
        c.vorticity_eps, c.buoyancy_beta, c.gravity_alpha = self.eps, self.beta, self.alpha
        for a in range(3):
            c.sphere_center[a] = float(self.center[a])
        c.sphere_radius = float(self.radius)
        c.sphere_density = 1.0
        c.sphere_temperature = 1.0
        return c


def rng_f64(seed: int, skip: int, n: int) -> np.ndarray:
    out = np.empty(n)
    check(_lib.load().afl_rng_f64(seed, skip, n, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return out


def plume48() -> list[InstanceSpec]:
    """The 48-plume ensemble: 16 at 32^3, 16 at 48^3, 16 at 64x128x64, seeds
    100..147.  Per instance, after the 3*N velocity-noise draws of its seed,
    the same generator gives the source-centre jitter (uniform +-10 % of the
    extent in x, y, z) and then alpha in [0.05, 0.1] and beta in [0.3, 0.5]."""
    shapes = [(32, 32, 32)] * 16 + [(48, 48, 48)] * 16 + [(64, 128, 64)] * 16
    out = []
    for m, (nx, ny, nz) in enumerate(shapes):
        seed = 100 + m
        n = nx * ny * nz
        x = rng_f64(seed, 3 * n, 5)
        base = (nx / 2, 0.1 * ny, nz / 2)
        ext = (nx, ny, nz)
        center = tuple(base[a] + (2.0 * x[a] - 1.0) * 0.1 * ext[a] for a in range(3))
        alpha = 0.05 + 0.05 * x[3]
        beta = 0.3 + 0.2 * x[4]
        out.append(InstanceSpec(nx, ny, nz, seed, alpha=alpha, beta=beta, center=center))
    return out


class Ensemble:
    def __init__(self, specs: list[InstanceSpec], precision: Precision = Precision.MIXED,
                 solver_iters: int = 200, cg_rel_tol: float = 1e-6):
        lib = _lib.load()
        self._lib = lib
        self.specs = list(specs)
        arr = (AflInstance * len(specs))(*[s.to_c() for s in specs])
        p = _lib.default_params()
        p.precision = int(precision)
        p.solver_kind = 0
        p.solver_iters = solver_iters
        p.cg_rel_tol = cg_rel_tol
        h = ctypes.c_void_p()
        check(lib.afl_ensemble_create(arr, len(specs), ctypes.byref(p), ctypes.byref(h)))
        self._h = h
        self.count = len(specs)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.afl_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, steps: int):
        """Returns (telemetry [steps, count, 8], solve infos [steps][count])."""
        rows = max(steps * self.count, 1)
        tel = (AflTelemetry * rows)()
        infos = (AflSolveInfo * rows)()
        check(self._lib.afl_ensemble_run(self._h, steps, tel, infos))
        arr = np.array([tel[r].as_tuple() for r in range(steps * self.count)])
        arr = arr.reshape(steps, self.count, 8)
        inf = [[SolveInfo.from_c(infos[n * self.count + m]) for m in range(self.count)]
               for n in range(steps)]
        return arr, inf

    def field(self, instance: int, name: str) -> np.ndarray:
        s = self.specs[instance]
        out = np.empty(s.cells)
        check(self._lib.afl_ensemble_download_field(
            self._h, instance, _lib.FIELD_IDS[name],
            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), s.cells))
        return out

    def autotune(self) -> int:
        c = ctypes.c_int32()
        check(self._lib.afl_ensemble_autotune(self._h, ctypes.byref(c)))
        return c.value

    def info(self) -> dict:
        out = (ctypes.c_int32 * 6)()
        check(self._lib.afl_ensemble_info(self._h, out))
        ctas = (ctypes.c_int32 * self.count)()
        check(self._lib.afl_ensemble_instance_ctas(self._h, ctas, self.count))
        kz = ctypes.c_int32()
        check(self._lib.afl_ensemble_tile_depth(self._h, ctypes.byref(kz)))
        pers = ctypes.c_int32()
        check(self._lib.afl_ensemble_persistent(self._h, ctypes.byref(pers)))
        return {"instances": out[0], "graph": bool(out[1]), "solver_ctas": out[2],
                "cta_budget": out[3], "vector_width": out[4], "autotune_choice": out[5],
                "instance_ctas": list(ctas), "tile_depth": kz.value,
                "persistent": bool(pers.value)}

    def set_tile_depth(self, kz: int):
        """z planes per CTA tile of the batched stage kernels (1, 2 or 4)."""
        check(self._lib.afl_ensemble_set_tile_depth(self._h, kz))

    def set_persistent(self, on: bool):
        """Step form: True (the default) = one persistent cooperative launch
        per step (instances meet only at their own barriers); False = the
        captured graph of per-stage batched launches and the cooperative solve.  Re-splits the CTAs
        for the form's co-resident budget and clears the autotune choice."""
        check(self._lib.afl_ensemble_set_persistent(self._h, 1 if on else 0))
