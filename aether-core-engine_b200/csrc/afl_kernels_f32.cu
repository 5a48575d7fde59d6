// afl_kernels_f32.cu -- f32 instantiation of the stage kernels for the mixed
// form (advection, curl, confinement, buoyancy and projection updates in f32;
// divergence, telemetry and the pressure gradient accumulate in f64).
#include "afl_stage_fused.cuh"

namespace afl {
AFL_INSTANTIATE_STAGES(float)
AFL_INSTANTIATE_FUSED(float)
}  // namespace afl
