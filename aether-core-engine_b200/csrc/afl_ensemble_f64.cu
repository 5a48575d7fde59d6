// afl_ensemble_f64.cu -- FP64 instantiation of the batched ensemble kernels,
// built without FMA contraction like the single-grid FP64 kernels.
#include "afl_ensemble_kernels.cuh"

namespace afl {

__global__ void kb_step_advance(int *step_counter) {
  if (threadIdx.x == 0) *step_counter += 1;
}

void ens_step_advance(int *step_counter, cudaStream_t st) {
  kb_step_advance<<<1, 32, 0, st>>>(step_counter);
}

AFL_INSTANTIATE_ENSEMBLE(double)

}  // namespace afl
