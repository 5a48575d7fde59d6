"""Reverse mode through the FP64 smoke step (afl_adjoint_* of
include/aether_fluid.h): controls are the initial velocity and the per-cell
temperature amplitude of the sphere source, the output is the final density.
The step's source is the sphere, the reference's cyberpunk jets
(inject_cyberpunk_sources, step n at time n*dt) or none; its pressure solve
is CG or red-black SOR.  `SmokeRollout` wraps one forward/backward pair with
the contract of a torch.autograd.Function (host tensors)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check

_dp = ctypes.POINTER(ctypes.c_double)


def _p(a):
    return a.ctypes.data_as(_dp) if a is not None else None


class Adjoint:
    SOURCES = {"cyberpunk": 0, "sphere": 1, "none": 2}
    SOLVERS = {"cg": 0, "sor": 1}

    def __init__(self, nx, ny, nz, center=(0.0, 0.0, 0.0), radius=0.0, eps=0.3, beta=0.4,
                 alpha=0.08, cg_rel_tol=1e-10, solver_iters=2000, checkpoint_every=8,
                 density=1.0, temperature=1.0, poisson_kernel=0, source="sphere", solver="cg",
                 sor_omega=1.65):
        lib = _lib.load()
        self._lib = lib
        p = _lib.default_params()
        p.vorticity_eps, p.buoyancy_beta, p.gravity_alpha = eps, beta, alpha
        p.solver_kind, p.solver_iters, p.cg_rel_tol = self.SOLVERS[solver], solver_iters, cg_rel_tol
        p.sor_omega = sor_omega
        p.source_kind = self.SOURCES[source]
        p.poisson_kernel = poisson_kernel
        for a in range(3):
            p.sphere_center[a] = float(center[a])
        p.sphere_radius = float(radius)
        p.sphere_density, p.sphere_temperature = density, temperature
        h = ctypes.c_void_p()
        check(lib.afl_adjoint_create(nx, ny, nz, ctypes.byref(p), checkpoint_every,
                                     ctypes.byref(h)))
        self._h = h
        self.nx, self.ny, self.nz = nx, ny, nz
        self.n = nx * ny * nz

    def close(self):
        if getattr(self, "_h", None):
            self._lib.afl_adjoint_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, u0, v0, w0, amp, steps, dt) -> np.ndarray:
        arrs = [np.ascontiguousarray(x, dtype=np.float64).ravel() for x in (u0, v0, w0)]
        a = None if amp is None else np.ascontiguousarray(amp, dtype=np.float64).ravel()
        rho = np.empty(self.n)
        check(self._lib.afl_adjoint_forward(self._h, _p(arrs[0]), _p(arrs[1]), _p(arrs[2]),
                                            _p(a), steps, dt, _p(rho)))
        return rho

    def backward(self, rho_bar):
        rb = np.ascontiguousarray(rho_bar, dtype=np.float64).ravel()
        outs = [np.empty(self.n) for _ in range(4)]
        check(self._lib.afl_adjoint_backward(self._h, _p(rb), *[_p(o) for o in outs]))
        return tuple(outs)

    def wall_masked(self, u, v, w):
        """Copies of (u, v, w) with the wall-BC cells zeroed
        (enforce_wall_velocity_bc, src/fluid.rs:236-253): the velocity
        subspace every step leaves the state in."""
        nx, ny, nz = self.nx, self.ny, self.nz
        k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        edge = (i == 0) | (i + 1 >= nx) | (j == 0) | (j + 1 >= ny) | (k == 0) | (k + 1 >= nz)
        masks = ((i <= 1) | edge, (j <= 1) | edge, (k <= 1) | edge)
        return tuple(np.where(m.ravel(), 0.0, np.asarray(a, dtype=np.float64).ravel())
                     for m, a in zip(masks, (u, v, w)))

    def stats(self) -> dict:
        out = (ctypes.c_double * 4)()
        check(self._lib.afl_adjoint_stats(self._h, out))
        return {"forward_ms": out[0], "backward_ms": out[1], "forward_cg_iters": int(out[2]),
                "adjoint_cg_iters": int(out[3])}


def _torch_function():
    import torch

    class SmokeRollout(torch.autograd.Function):
        """rho_final = SmokeRollout.apply(u0, v0, w0, amp, adjoint, steps, dt)."""

        @staticmethod
        def forward(ctx, u0, v0, w0, amp, adjoint, steps, dt):
            rho = adjoint.forward(u0.detach().cpu().numpy(), v0.detach().cpu().numpy(),
                                  w0.detach().cpu().numpy(), amp.detach().cpu().numpy(),
                                  steps, dt)
            ctx.adjoint = adjoint
            return torch.from_numpy(rho)

        @staticmethod
        def backward(ctx, grad_rho):
            ub, vb, wb, ab = ctx.adjoint.backward(grad_rho.detach().cpu().numpy())
            t = torch.from_numpy
            return t(ub), t(vb), t(wb), t(ab), None, None, None

    return SmokeRollout


def smoke_rollout():
    """The torch.autograd.Function of a rollout (imports torch on first use)."""
    return _torch_function()
