// afl_ensemble_f32.cu -- f32 instantiation of the batched ensemble kernels
// (the mixed form), built like the single-grid f32 kernels.
#include "afl_ensemble_kernels.cuh"

namespace afl {
AFL_INSTANTIATE_ENSEMBLE(float)
}  // namespace afl
