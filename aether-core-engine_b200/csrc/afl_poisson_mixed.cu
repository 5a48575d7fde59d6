// afl_poisson_mixed.cu -- mixed-precision red-black SOR (the mixed CG with
// its f64 iterative refinement lives in afl_poisson_stream.cu and
// afl_poisson_resident.cu).
#include "afl_launch.h"

namespace afl {
namespace {

template <typename R, typename X>
__device__ __forceinline__ R lap7(const Dims &g, int c, int i, int j, int k, const X &x) {
  R diag = R(0), nb = R(0);
  if (i > 1) { diag += R(1); nb += x(c - 1); }
  if (i + 2 < g.nx) { diag += R(1); nb += x(c + 1); }
  if (j > 1) { diag += R(1); nb += x(c - g.nx); }
  if (j + 2 < g.ny) { diag += R(1); nb += x(c + g.nx); }
  if (k > 1) { diag += R(1); nb += x(c - g.nxy); }
  if (k + 2 < g.nz) { diag += R(1); nb += x(c + g.nxy); }
  return diag * x(c) - nb;
}

// Mixed RB-SOR: the f64 residual r = b - A p is formed once, the sweeps run in
// f32 on the correction (A e = r, e0 = 0 -- the same linear iteration as
// sweeping p itself), and p += e in f64.
__global__ void __launch_bounds__(kBlock) k_rbsor_mixed(SorMixedArgs a, GridSync gs) {
  const Dims g = a.g;
  const int t0 = blockIdx.x * kBlock + threadIdx.x;
  const int stride = gridDim.x * kBlock;
  float *e = a.p32;
  const float *rb = a.b32;
  for (int c = t0; c < g.n; c += stride) {
    int i, j, k;
    decode(g, c, i, j, k);
    double ap = 0.0;
    if (interior(g, i, j, k)) ap = lap7<double>(g, c, i, j, k, [&](int x) { return a.p[x]; });
    a.b32[c] = float(__ldg(a.b + c) - ap);
    e[c] = 0.0f;
  }
  if (!grid_sync(gs)) return;
  const float omega = float(a.omega);
  const ColorWalk walk(g);
  for (int sweep = 0; sweep < a.sweeps; ++sweep) {
    for (int color = 0; color < 2; ++color) {
      for (int q = t0; q < walk.total; q += stride) {
        int i, j, k;
        if (!walk.cell(g, q, color, i, j, k)) continue;
        const int c = (k * g.ny + j) * g.nx + i;
        float diag = 0.0f, nb = 0.0f;
        if (i > 1) { diag += 1.0f; nb += e[c - 1]; }
        if (i + 2 < g.nx) { diag += 1.0f; nb += e[c + 1]; }
        if (j > 1) { diag += 1.0f; nb += e[c - g.nx]; }
        if (j + 2 < g.ny) { diag += 1.0f; nb += e[c + g.nx]; }
        if (k > 1) { diag += 1.0f; nb += e[c - g.nxy]; }
        if (k + 2 < g.nz) { diag += 1.0f; nb += e[c + g.nxy]; }
        const float target = (rb[c] + nb) / diag;
        e[c] = (1.0f - omega) * e[c] + omega * target;
      }
      if (!grid_sync(gs)) return;
    }
  }
  for (int c = t0; c < g.n; c += stride) a.p[c] = a.p[c] + double(e[c]);
  if (blockIdx.x == 0 && threadIdx.x == 0 && a.report) {
    SolveReport rep;
    rep.iterations = a.sweeps;
    rep.refinements = 1;
    rep.converged = 0;
    rep.status = 0;
    rep.initial_residual = 0.0;
    rep.final_residual = 0.0;
    rep.rhs_norm = 0.0;
    *a.report = rep;
  }
}

int blocks_for(const void *kernel) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, 0);
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

GridSync make_sync(const PersistentState &ps, int blocks) {
  GridSync gs;
  gs.count = ps.count;
  gs.gen = ps.gen;
  gs.abort_flag = ps.abort_flag;
  gs.nblocks = static_cast<unsigned int>(blocks);
  gs.timeout_ns = ps.timeout_ns;
  return gs;
}

}  // namespace

int persistent_blocks_cg_mixed() { return persistent_blocks_stream(); }
int persistent_blocks_sor_mixed() {
  return blocks_for(reinterpret_cast<const void *>(&k_rbsor_mixed));
}

int launch_cg_mixed(const MixedCgArgs &a, const PersistentState &ps, cudaStream_t st) {
  return launch_cg_stream_mixed(a, ps, st);
}

int launch_rbsor_mixed(const SorMixedArgs &a, const PersistentState &ps, cudaStream_t st) {
  int blocks = persistent_blocks_sor_mixed();
  if (blocks > ps.max_blocks) blocks = ps.max_blocks;
  cudaMemsetAsync(ps.count, 0, sizeof(unsigned int), st);
  cudaMemsetAsync(ps.gen, 0, sizeof(unsigned int), st);
  cudaMemsetAsync(ps.abort_flag, 0, sizeof(int), st);
  SorMixedArgs args = a;
  GridSync gs = make_sync(ps, blocks);
  void *params[] = {&args, &gs};
  const cudaError_t err = cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(&k_rbsor_mixed), dim3(blocks),
                              dim3(kBlock), params, 0, st);
  return err == cudaSuccess ? blocks : -static_cast<int>(err);
}

}  // namespace afl
