// afl_kernels_f64.cu -- FP64 instantiation of the stage kernels, plus the
// type-independent finalize/convert kernels.  Built with -fmad=false: the
// reference's f64 arithmetic is never contracted into FMAs (rustc emits none
// without an explicit mul_add), so the pointwise and stencil stages here
// reproduce the reference's f64 results bit for bit.
#include "afl_stage_fused.cuh"

namespace afl {

__global__ void __launch_bounds__(kBlock)
    k_divergence_finalize(const double *__restrict__ partials, int nparts,
                          double interior_cells, double *__restrict__ out2) {
  __shared__ double scratch[kWarps * 2];
  double tot[2];
  reduce_partials<2>(partials, nparts, tot, scratch);
  if (threadIdx.x == 0) {
    out2[0] = sqrt(tot[0] / interior_cells);  // src/fluid.rs:351-352
    out2[1] = sqrt(tot[1]);
  }
}

__global__ void __launch_bounds__(kBlock)
    k_telemetry_finalize(const double *__restrict__ partials, int nparts, double time_sec,
                         double *__restrict__ out8) {
  __shared__ double scratch[kWarps * 6];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  double peak = 0.0;
  for (int b = threadIdx.x; b < nparts; b += blockDim.x) {
#pragma unroll
    for (int a = 0; a < 6; ++a) acc[a] += partials[b * 7 + a];
    peak = fmax(peak, partials[b * 7 + 6]);
  }
  block_sum<6>(acc, scratch);
  peak = block_max(peak, scratch);
  if (threadIdx.x == 0) {
    const double mass = acc[2];
    double com[3] = {acc[3], acc[4], acc[5]};
    if (mass > 1e-12) {  // src/fluid.rs:661-663 (Vec3 /= m multiplies by 1/m)
      const double inv = 1.0 / mass;
      for (int a = 0; a < 3; ++a) com[a] = com[a] * inv;
    }
    out8[0] = time_sec;
    out8[1] = acc[0];
    out8[2] = acc[1];
    out8[3] = peak;
    out8[4] = mass;
    for (int a = 0; a < 3; ++a) out8[5 + a] = rs_clamp(com[a], -1.0, 1.0);
  }
}

__global__ void __launch_bounds__(kBlock)
    k_max_finalize(const double *__restrict__ partials, int nparts, double *__restrict__ out1) {
  __shared__ double scratch[kWarps];
  double m = 0.0;
  for (int b = threadIdx.x; b < nparts; b += blockDim.x) m = fmax(m, partials[b]);
  m = block_max(m, scratch);
  if (threadIdx.x == 0) out1[0] = m;
}

__global__ void k_f64_to_f32(const double *__restrict__ s, float *__restrict__ d, int n) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    d[c] = float(s[c]);
}
__global__ void k_f32_to_f64(const float *__restrict__ s, double *__restrict__ d, int n) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    d[c] = double(s[c]);
}

void launch_convert_f64_to_f32(const double *src, float *dst, int n, cudaStream_t st) {
  k_f64_to_f32<<<kReduceBlocks, kBlock, 0, st>>>(src, dst, n);
}
void launch_convert_f32_to_f64(const float *src, double *dst, int n, cudaStream_t st) {
  k_f32_to_f64<<<kReduceBlocks, kBlock, 0, st>>>(src, dst, n);
}

void launch_telemetry_finalize(const double *partials, int nparts, double time_sec,
                               double *out8, cudaStream_t st) {
  k_telemetry_finalize<<<1, kBlock, 0, st>>>(partials, nparts, time_sec, out8);
}

int fused_ctas(const Dims &g) { return fused_ctas_of(g); }

AFL_INSTANTIATE_STAGES(double)
AFL_INSTANTIATE_FUSED(double)

}  // namespace afl
