"""ctypes binding of include/aether_fluid.h (libaether_fluid.so).

This is the reference-side binding a Python caller uses; a Rust caller would
declare the same entry points in an `extern "C"` block.  Loading fails loudly
when the library has not been built: there is no CPU path.
"""
from __future__ import annotations

import ctypes
import os

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "libaether_fluid.so")

AFL_OK = 0
STATUS_NAMES = {
    0: "AFL_OK",
    1: "AFL_ERR_INVALID_ARGUMENT",
    2: "AFL_ERR_CUDA",
    3: "AFL_ERR_OUT_OF_MEMORY",
    4: "AFL_ERR_NONFINITE",
    5: "AFL_ERR_TIMEOUT",
    6: "AFL_ERR_NOT_CONVERGED",
}

STAGES = ("advect", "source", "forces", "divergence", "poisson", "project", "telemetry")

FIELD_IDS = {"u": 0, "v": 1, "w": 2, "density": 3, "temperature": 4,
             "pressure": 5, "divergence": 6}


class AflParams(ctypes.Structure):
    _fields_ = [
        ("vorticity_eps", ctypes.c_double),
        ("buoyancy_beta", ctypes.c_double),
        ("gravity_alpha", ctypes.c_double),
        ("solver_kind", ctypes.c_int32),
        ("solver_iters", ctypes.c_int32),
        ("sor_omega", ctypes.c_double),
        ("cg_rel_tol", ctypes.c_double),
        ("precision", ctypes.c_int32),
        ("source_kind", ctypes.c_int32),
        ("sphere_center", ctypes.c_double * 3),
        ("sphere_radius", ctypes.c_double),
        ("sphere_density", ctypes.c_double),
        ("sphere_temperature", ctypes.c_double),
        ("fail_on_not_converged", ctypes.c_int32),
        ("mixed_inner_iters", ctypes.c_int32),
        ("mixed_inner_rel_tol", ctypes.c_double),
        ("mixed_max_refinements", ctypes.c_int32),
        ("poisson_kernel", ctypes.c_int32),
        ("reserved_f64", ctypes.c_double * 4),
    ]


class AflTelemetry(ctypes.Structure):
    _fields_ = [
        ("time_sec", ctypes.c_double),
        ("kinetic_energy", ctypes.c_double),
        ("enstrophy", ctypes.c_double),
        ("peak_vorticity", ctypes.c_double),
        ("total_mass", ctypes.c_double),
        ("center_of_mass", ctypes.c_double * 3),
    ]

    def as_tuple(self):
        return (self.time_sec, self.kinetic_energy, self.enstrophy, self.peak_vorticity,
                self.total_mass, *self.center_of_mass)


class AflSolveInfo(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int32),
        ("refinements", ctypes.c_int32),
        ("converged", ctypes.c_int32),
        ("status", ctypes.c_int32),
        ("initial_residual", ctypes.c_double),
        ("final_residual", ctypes.c_double),
        ("rhs_norm", ctypes.c_double),
    ]


class AflInstance(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_size_t), ("ny", ctypes.c_size_t), ("nz", ctypes.c_size_t),
        ("seed", ctypes.c_uint64),
        ("noise_lo", ctypes.c_double), ("noise_hi", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("vorticity_eps", ctypes.c_double), ("buoyancy_beta", ctypes.c_double),
        ("gravity_alpha", ctypes.c_double),
        ("sphere_center", ctypes.c_double * 3), ("sphere_radius", ctypes.c_double),
        ("sphere_density", ctypes.c_double), ("sphere_temperature", ctypes.c_double),
    ]


class AetherFluidError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


# (name, restype, argtypes) for every entry point declared in the header.
_vp = ctypes.c_void_p
_d = ctypes.c_double
_i = ctypes.c_int
_sz = ctypes.c_size_t
_dp = ctypes.POINTER(ctypes.c_double)
_st = ctypes.c_int
class AflRay(ctypes.Structure):
    _fields_ = [("origin", ctypes.c_double * 3), ("dir", ctypes.c_double * 3),
                ("t_min", ctypes.c_double), ("t_end", ctypes.c_double)]


SIGNATURES = [
    ("afl_last_error", ctypes.c_char_p, []),
    ("afl_abi_version", ctypes.c_int, []),
    ("afl_params_default", _st, [ctypes.POINTER(AflParams)]),
    ("afl_create", _st, [_sz, _sz, _sz, ctypes.POINTER(AflParams), ctypes.POINTER(_vp)]),
    ("afl_destroy", _st, [_vp]),
    ("afl_get_dims", _st, [_vp, ctypes.POINTER(_sz), ctypes.POINTER(_sz),
                           ctypes.POINTER(_sz), _dp]),
    ("afl_set_params", _st, [_vp, ctypes.POINTER(AflParams)]),
    ("afl_get_params", _st, [_vp, ctypes.POINTER(AflParams)]),
    ("afl_set_source_amplitude", _st, [_vp, _dp, _sz]),
    ("afl_upload_field", _st, [_vp, _i, _dp, _sz]),
    ("afl_download_field", _st, [_vp, _i, _dp, _sz]),
    ("afl_init_velocity_noise", _st, [_vp, ctypes.c_uint64, _d, _d]),
    ("afl_advect_maccormack", _st, [_vp, _i, _d, _d]),
    ("afl_enforce_wall_bc", _st, [_vp]),
    ("afl_buoyancy_vorticity", _st, [_vp, _d]),
    ("afl_divergence_norm", _st, [_vp, _dp]),
    ("afl_solve_cg", _st, [_vp, _i, ctypes.POINTER(AflSolveInfo)]),
    ("afl_solve_rbsor", _st, [_vp, _i, ctypes.POINTER(AflSolveInfo)]),
    ("afl_project", _st, [_vp, ctypes.POINTER(AflSolveInfo)]),
    ("afl_inject_cyberpunk", _st, [_vp, _d, _d]),
    ("afl_inject_sphere", _st, [_vp]),
    ("afl_step", _st, [_vp, _d, _d, ctypes.POINTER(AflTelemetry),
                       ctypes.POINTER(AflSolveInfo)]),
    ("afl_run", _st, [_vp, _i, _d, _d, _d, ctypes.POINTER(AflTelemetry),
                      ctypes.POINTER(AflSolveInfo)]),
    ("afl_compute_telemetry", _st, [_vp, _d, ctypes.POINTER(AflTelemetry)]),
    ("afl_max_density", _st, [_vp, _dp]),
    ("afl_medium_handoff", _st, [_vp, _dp, _dp, _sz, _dp]),
    ("afl_sample_trilinear", _st, [_vp, _i, _dp, _sz, _dp]),
    ("afl_set_stage_timing", _st, [_vp, _i]),
    ("afl_get_stage_timing", _st, [_vp, _dp, ctypes.POINTER(ctypes.c_int64)]),
    ("afl_get_poisson_plan", _st, [_vp, ctypes.POINTER(ctypes.c_int32)]),
    ("afl_get_launch_count", _st, [_vp, ctypes.POINTER(ctypes.c_uint64)]),
    ("afl_ensemble_create", _st, [ctypes.POINTER(AflInstance), _i, ctypes.POINTER(AflParams),
                                   ctypes.POINTER(_vp)]),
    ("afl_ensemble_destroy", _st, [_vp]),
    ("afl_ensemble_run", _st, [_vp, _i, ctypes.POINTER(AflTelemetry),
                               ctypes.POINTER(AflSolveInfo)]),
    ("afl_ensemble_download_field", _st, [_vp, _i, _i, _dp, _sz]),
    ("afl_ensemble_autotune", _st, [_vp, ctypes.POINTER(ctypes.c_int32)]),
    ("afl_ensemble_info", _st, [_vp, ctypes.POINTER(ctypes.c_int32)]),
    ("afl_ensemble_instance_ctas", _st, [_vp, ctypes.POINTER(ctypes.c_int32), _i]),
    ("afl_ensemble_set_tile_depth", _st, [_vp, ctypes.c_int32]),
    ("afl_ensemble_tile_depth", _st, [_vp, ctypes.POINTER(ctypes.c_int32)]),
    ("afl_ensemble_set_persistent", _st, [_vp, ctypes.c_int32]),
    ("afl_ensemble_persistent", _st, [_vp, ctypes.POINTER(ctypes.c_int32)]),
    ("afl_rng_f64", _st, [ctypes.c_uint64, ctypes.c_uint64, _sz, _dp]),
    ("afl_adjoint_create", _st, [_sz, _sz, _sz, ctypes.POINTER(AflParams), _i,
                                 ctypes.POINTER(_vp)]),
    ("afl_adjoint_destroy", _st, [_vp]),
    ("afl_adjoint_forward", _st, [_vp, _dp, _dp, _dp, _dp, _i, _d, _dp]),
    ("afl_adjoint_backward", _st, [_vp, _dp, _dp, _dp, _dp, _dp]),
    ("afl_adjoint_stats", _st, [_vp, _dp]),
    ("afl_solve_cg_noalloc", _st, [_vp, _vp, _sz, _sz, _sz, _i, _d, _vp,
                                    ctypes.POINTER(AflSolveInfo)]),
    ("afl_medium_create", _st, [_vp, _dp, _dp, _d, _d, ctypes.POINTER(_vp)]),
    ("afl_medium_destroy", _st, [_vp]),
    ("afl_medium_info", _st, [_vp, _dp]),
    ("afl_medium_sample_density_temp", _st, [_vp, _dp, _sz, _dp, _dp]),
    ("afl_medium_transmittance", _st, [_vp, _vp, _sz, ctypes.c_uint64, _dp]),
    ("afl_medium_sample_interaction", _st, [_vp, _vp, _sz, ctypes.c_uint64,
                                            ctypes.POINTER(ctypes.c_int32), _dp, _dp, _dp]),
    ("afl_synchronize", _st, [_vp]),
    ("afl_stream", _vp, [_vp]),
]

_lib = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads the CUDA library; raises if it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with aether_fluid.build.build() "
            "(nvcc, sm_100a); this package has no CPU implementation")
    lib = ctypes.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != AFL_OK:
        msg = load().afl_last_error()
        raise AetherFluidError(status, msg.decode() if msg else "")


def default_params() -> AflParams:
    p = AflParams()
    check(load().afl_params_default(ctypes.byref(p)))
    return p
