"""aether_fluid -- B200-native (sm_100a) smoke step of vanovri/aether-core-engine.

The numerical work runs in libaether_fluid.so (hand-written CUDA kernels behind
the C ABI of include/aether_fluid.h); this package is the host-side mirror of
the reference's `FluidSolver3D` / `FluidMedium` interface (src/fluid.rs).
"""
from ._lib import AetherFluidError, LIB_PATH, load  # noqa: F401
from .medium import DeviceMedium  # noqa: F401
from .solver import (  # noqa: F401
    Aabb,
    FluidMedium,
    FluidSolver3D,
    FluidTelemetryFrame,
    PoissonSolverKind,
    Precision,
    SolveInfo,
    SourceKind,
)
