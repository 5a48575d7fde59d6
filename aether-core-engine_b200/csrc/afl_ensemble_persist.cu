// afl_ensemble_persist.cu -- one persistent launch per ensemble step.
//
// The alternative to the captured graph of per-stage launches
// (afl_ensemble.cu): a single cooperative kernel runs the whole step
// (src/fluid.rs:598-611) for every instance.  Its CTAs are split between the
// instances exactly as the batched pressure solve splits them; the CTAs of
// one instance loop over that instance's plane blocks stage by stage and meet
// at the instance's own bounded grid barrier between stages, then run the
// instance's CG (the body of the batched streaming solve) on the same
// barrier.  Instances never wait for one another.  The per-cell code is the
// batched kernels' code (afl_ensemble_kernels.cuh), compiled here without
// __restrict__ so that every load of a field written earlier in the launch is
// an ordinary coherent load, ordered after the writes by the barrier's
// acquire.  The MacCormack ping-pong swaps a CTA-local copy of the instance
// descriptor; the instance's first CTA writes the final pointers back.
//
// Built with -fmad=false, like the other f64 units; the f32 (mixed) stages
// therefore round each product and sum separately here, where the batched
// f32 kernels may contract them.
//
// Every stage runs at the solve's occupancy (4 CTAs per SM at 64 registers;
// 5 per SM spills 300-480 bytes), and the solve gets 592 CTAs instead of the
// graph form's 740.  Its CG body therefore prefetches the runs two steps ahead
// into L2.  Measured on the 48-plume ensemble (mixed, 100 steps, autotuned):
// 645-650 Mcell-steps/s against 632-633 for the graph of stage launches (593
// without the prefetch), so this is the default form.
#define AFL_RESTRICT
#include <type_traits>

#include "afl_cg_stream_body.cuh"
#include "afl_ensemble_kernels.cuh"

namespace afl {
namespace {

// CTAs per SM the step kernel is built for (64 registers per thread).
constexpr int kStepCtasPerSm = 4;
constexpr int kStepScratch = kWarps * 6 + 4;  // telemetry sums and CG partials

template <typename T, int V>
__global__ void __launch_bounds__(kST, kStepCtasPerSm) kp_ens_step(EnsStepArgs a) {
  __shared__ EnsInstance<T> d;
  __shared__ double scratch[kStepScratch];
  const int m = a.cta_inst[blockIdx.x];
  const MultiCgSystem &s = a.sys[m];
  const int vb = static_cast<int>(blockIdx.x) - s.cta_begin, nv = s.ctas;
  const GridSync gs = s.gs;
  if (threadIdx.x == 0) d = static_cast<EnsInstance<T> *>(a.inst)[m];
  const int step = *a.step_counter;
  __syncthreads();
  // every plane block of the instance, CTA vb taking blocks vb, vb + nv, ...
  auto each = [&](auto &&body) {
    for (int lb = vb; lb < d.blk_count; lb += nv) body(lb);
  };
  // the advected field becomes current, its old buffer the next output
  auto swap_out = [&](int f) {
    if (threadIdx.x == 0) {
      T *t = d.fld[f];
      d.fld[f] = d.tmp_out;
      d.tmp_out = t;
    }
    __syncthreads();
  };
  auto advect = [&](int f, double diss) {
    each([&](int lb) { blk_advect_fwd(d, lb, f); });
    if (!grid_sync(gs)) return false;
    each([&](int lb) { blk_advect_mc(d, lb, f, diss); });
    if (!grid_sync(gs)) return false;
    swap_out(f);
    return true;
  };
  for (int f = 0; f < 3; ++f)
    if (!advect(f, 0.996)) return;
  each([&](int lb) { blk_curl(d, lb); });
  if (!grid_sync(gs)) return;
  each([&](int lb) { blk_source_confine_buoy(d, lb); });
  if (!grid_sync(gs)) return;
  each([&](int lb) { blk_divergence(d, lb); });
  if (!grid_sync(gs)) return;
  bool ok;
  if constexpr (std::is_same<T, double>::value) {
    const Ring3 pr{s.partials, 2 * nv};
    ok = cg_stream_f64_body<V, false, true>(s.f64, gs, pr, vb, nv, scratch);
  } else {
    const Ring3 pr{s.partials, 3 * nv};
    ok = cg_stream_mixed_body<V, false, true>(s.mixed, gs, pr, vb, nv, scratch);
  }
  // The solve ends at a barrier after its last pressure write; this one also
  // separates its last read of the partials from the stages' writes.
  if (!ok || !grid_sync(gs)) return;
  each([&](int lb) { blk_project(d, lb); });
  if (!grid_sync(gs)) return;
  if (!advect(3, 0.996)) return;
  if (!advect(4, 0.985)) return;
  each([&](int lb) {
    blk_telemetry(d, lb, a.tel_partials, scratch);
  });
  if (!grid_sync(gs)) return;
  if (vb == 0) {
    ens_finalize(d, m, a.tel_partials, step, a.tel_out, a.rep_cur, a.reports, a.count,
                 a.capacity, scratch);
    if (threadIdx.x == 0) {
      EnsInstance<T> &out = static_cast<EnsInstance<T> *>(a.inst)[m];
      for (int f = 0; f < 5; ++f) out.fld[f] = d.fld[f];
      out.tmp_out = d.tmp_out;
    }
  }
}

template <typename T, int V>
const void *step_kernel() {
  return reinterpret_cast<const void *>(&kp_ens_step<T, V>);
}

const void *pick(bool f64, int v) {
  if (f64) return v == 2 ? step_kernel<double, 2>() : step_kernel<double, 1>();
  return v == 4 ? step_kernel<float, 4>() : step_kernel<float, 1>();
}

}  // namespace

int persistent_blocks_ens_step(bool f64, int v) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pick(f64, v), kST, 0);
  return sms * (per_sm < 1 ? 1 : per_sm);
}

int launch_ens_step(const EnsStepArgs &a, bool f64, int v, int total_ctas, cudaStream_t st) {
  EnsStepArgs args = a;
  void *params[] = {&args};
  const cudaError_t err =
      cudaLaunchCooperativeKernel(pick(f64, v), dim3(total_ctas), dim3(kST), params, 0, st);
  return err == cudaSuccess ? total_ctas : -static_cast<int>(err);
}

}  // namespace afl
