// afl_poisson_f64.cu -- FP64 red-black SOR as one persistent launch (the FP64
// CG lives in afl_poisson_stream.cu and afl_poisson_resident.cu).
//
// Built with -fmad=false: every update is the reference's un-fused expression,
// and an RB-SOR sweep reproduces the reference bit for bit (each colour reads
// only the other colour, so the visiting order does not matter).  Colours are
// separated by the bounded grid barrier of afl_device.cuh.
#include "afl_launch.h"

namespace afl {
namespace {

// solve_poisson_gauss_seidel (src/fluid.rs:397-442): colour 0 then colour 1
// per sweep, in place.  The update reads only the other colour, so the result
// does not depend on the order cells are visited and equals the reference's.
__global__ void __launch_bounds__(kBlock) k_rbsor_f64(SorArgs a, GridSync gs) {
  const Dims g = a.g;
  const int t0 = blockIdx.x * kBlock + threadIdx.x;
  const int stride = gridDim.x * kBlock;
  double *p = a.p;
  const double omega = a.omega;
  const ColorWalk walk(g);
  for (int sweep = 0; sweep < a.sweeps; ++sweep) {
    for (int color = 0; color < 2; ++color) {
      for (int q = t0; q < walk.total; q += stride) {
        int i, j, k;
        if (!walk.cell(g, q, color, i, j, k)) continue;
        const int c = (k * g.ny + j) * g.nx + i;
        double diag = 0.0, nb = 0.0;
        if (i > 1) { diag += 1.0; nb += p[c - 1]; }
        if (i + 2 < g.nx) { diag += 1.0; nb += p[c + 1]; }
        if (j > 1) { diag += 1.0; nb += p[c - g.nx]; }
        if (j + 2 < g.ny) { diag += 1.0; nb += p[c + g.nx]; }
        if (k > 1) { diag += 1.0; nb += p[c - g.nxy]; }
        if (k + 2 < g.nz) { diag += 1.0; nb += p[c + g.nxy]; }
        const double gs_target = (__ldg(a.b + c) + nb) / diag;
        p[c] = (1.0 - omega) * p[c] + omega * gs_target;
      }
      if (!grid_sync(gs)) return;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && a.report) {
    SolveReport rep;
    rep.iterations = a.sweeps;
    rep.refinements = 0;
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

int persistent_blocks_cg_f64() { return persistent_blocks_stream(); }
int persistent_blocks_sor_f64() {
  return blocks_for(reinterpret_cast<const void *>(&k_rbsor_f64));
}

int launch_cg_f64(const CgArgs &a, const PersistentState &ps, cudaStream_t st) {
  return launch_cg_stream_f64(a, ps, st);
}

int launch_rbsor_f64(const SorArgs &a, const PersistentState &ps, cudaStream_t st) {
  int blocks = persistent_blocks_sor_f64();
  if (blocks > ps.max_blocks) blocks = ps.max_blocks;
  cudaMemsetAsync(ps.count, 0, sizeof(unsigned int), st);
  cudaMemsetAsync(ps.gen, 0, sizeof(unsigned int), st);
  cudaMemsetAsync(ps.abort_flag, 0, sizeof(int), st);
  SorArgs args = a;
  GridSync gs = make_sync(ps, blocks);
  void *params[] = {&args, &gs};
  const cudaError_t err = cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(&k_rbsor_f64), dim3(blocks),
                              dim3(kBlock), params, 0, st);
  return err == cudaSuccess ? blocks : -static_cast<int>(err);
}

}  // namespace afl
