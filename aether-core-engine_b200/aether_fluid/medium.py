"""FluidMedium's volume queries on the GPU (afl_medium_* of
include/aether_fluid.h): the renderer's medium calls (src/renderer.rs:236,
258, 306) as batched kernels over a device snapshot of a solver's density and
temperature.

    m = DeviceMedium.from_solver(solver, Aabb(lo, hi), sigma_t_scale, phase_g)
    rho, temp = m.sample_density_and_temp(points)            # [n, 3]
    tr = m.transmittance(rays, seed)                         # [n, 8]
    hit, t, rho, temp = m.sample_interaction(rays, seed)     # [n, 8]

A ray row is origin (3), direction (3, normalised inside as Ray::new does),
t_min and the end of the segment: `surface_t` for sample_interaction,
`max_dist` for transmittance.  Ray r draws from Rng::from_seed(seed + r).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check

_dp = ctypes.POINTER(ctypes.c_double)


def _p(a):
    return a.ctypes.data_as(_dp)


def _rays(rays) -> np.ndarray:
    r = np.ascontiguousarray(rays, dtype=np.float64).reshape(-1, 8)
    assert ctypes.sizeof(_lib.AflRay) == 64
    return r


class DeviceMedium:
    def __init__(self, handle, lib, info):
        self._h = handle
        self._lib = lib
        self.max_density, self.majorant_sigma_t, self.phase_g, self.sigma_t_scale = info

    @staticmethod
    def from_solver(solver, bounds, sigma_t_scale: float, phase_g: float) -> "DeviceMedium":
        """FluidMedium::from_solver (src/fluid.rs:703-732), kept on the device."""
        lib = _lib.load()
        lo = np.ascontiguousarray(bounds.min, dtype=np.float64)
        hi = np.ascontiguousarray(bounds.max, dtype=np.float64)
        h = ctypes.c_void_p()
        check(lib.afl_medium_create(solver._h, _p(lo), _p(hi), sigma_t_scale, phase_g,
                                    ctypes.byref(h)))
        out = (ctypes.c_double * 4)()
        check(lib.afl_medium_info(h, out))
        return DeviceMedium(h, lib, tuple(out))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.afl_medium_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sample_density_and_temp(self, points):
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        n = pts.shape[0]
        rho, tmp = np.empty(n), np.empty(n)
        check(self._lib.afl_medium_sample_density_temp(self._h, _p(pts), n, _p(rho), _p(tmp)))
        return rho, tmp

    def transmittance(self, rays, seed: int) -> np.ndarray:
        r = _rays(rays)
        out = np.empty(r.shape[0])
        check(self._lib.afl_medium_transmittance(self._h, r.ctypes.data_as(ctypes.c_void_p),
                                                 r.shape[0], seed, _p(out)))
        return out

    def sample_interaction(self, rays, seed: int):
        r = _rays(rays)
        n = r.shape[0]
        hit = np.empty(n, dtype=np.int32)
        t, rho, tmp = np.empty(n), np.empty(n), np.empty(n)
        check(self._lib.afl_medium_sample_interaction(
            self._h, r.ctypes.data_as(ctypes.c_void_p), n, seed,
            hit.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), _p(t), _p(rho), _p(tmp)))
        return hit, t, rho, tmp
