// afl_poisson_mixed.cu -- the mixed-precision pressure solves.
//
// Iterative refinement: the Poisson residual r = b - A p and its norm are
// formed in f64 from the f64 pressure; an f32 CG solves A e = r (f32 vectors
// and f32 matrix-vector products, every inner product accumulated in f64);
// p += e in f64; repeat until ||r||_2 <= rel_tol*||b||_2 in f64.  The whole
// refinement loop is one persistent cooperative launch.
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

struct Ring {
  double *base;
  int stride;
  __device__ double *buf(int phase) const { return base + (phase & 1) * stride; }
};

__global__ void __launch_bounds__(kBlock) k_cg_mixed(MixedCgArgs a, GridSync gs, Ring pr) {
  __shared__ double scratch[kWarps * 3];
  const Dims g = a.g;
  const int t0 = blockIdx.x * kBlock + threadIdx.x;
  const int stride = gridDim.x * kBlock;
  double *p = a.p;
  const double *b = a.b;
  float *r = a.r, *e = a.e, *q = a.q;
  int phase = 0;

  // Outer residual in f64; its f32 copy seeds the inner CG (e = 0).  Partials:
  // (||r||^2 in f64, ||b||^2, ||float(r)||^2 -- where the inner CG starts).
  auto outer_residual = [&](bool with_b) {
    double acc[3] = {0.0, 0.0, 0.0};
    for (int c = t0; c < g.n; c += stride) {
      int i, j, k;
      decode(g, c, i, j, k);
      double ap = 0.0;
      if (interior(g, i, j, k)) ap = lap7<double>(g, c, i, j, k, [&](int x) { return p[x]; });
      const double bc = __ldg(b + c);
      const double rv = bc - ap;
      const float rf = float(rv);
      r[c] = rf;
      e[c] = 0.0f;
      acc[0] += rv * rv;
      if (with_b) acc[1] += bc * bc;
      acc[2] += double(rf) * double(rf);
    }
    block_sum<3>(acc, scratch);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int v = 0; v < 3; ++v) pr.buf(phase)[blockIdx.x * 3 + v] = acc[v];
    }
  };

  outer_residual(true);
  if (!grid_sync(gs)) return;
  double tot[3];
  reduce_partials<3>(pr.buf(phase), gridDim.x, tot, scratch);
  ++phase;
  const double bb = tot[1];
  double rr = tot[0];
  const double rr0 = rr;
  double tol2 = -1.0;
  if (a.rel_tol > 0.0) {
    const double tl = a.rel_tol * sqrt(bb);
    tol2 = tl * tl;
  }
  int total = 0, passes = 0, converged = 0;
  if (!(rr > 1e-24) || (tol2 >= 0.0 && rr <= tol2)) converged = 1;

  while (!converged && passes < a.max_refine && total < a.max_total && isfinite(rr)) {
    // Inner target: the reduction still needed, with margin, but no tighter
    // than f32 arithmetic can deliver.
    double inner_rel = a.inner_rel_tol;
    if (tol2 >= 0.0) inner_rel = fmax(inner_rel, 0.5 * sqrt(tol2 / rr));
    double delta = tot[2];  // ||float(r)||^2, from the outer residual pass
    const double inner_tol2 = inner_rel * inner_rel * delta;
    double beta = 0.0;
    float *dold = a.d0, *dnew = a.d1;
    int it = 0;
    while (it < a.max_inner && total < a.max_total) {
      double acc[1] = {0.0};
      const bool first = (it == 0);
      const float bf = float(beta);
      auto dn_at = [&](int x) { return first ? r[x] : r[x] + bf * dold[x]; };
      for (int c = t0; c < g.n; c += stride) {
        int i, j, k;
        decode(g, c, i, j, k);
        const float dc = dn_at(c);
        float qv = 0.0f;
        if (interior(g, i, j, k)) qv = lap7<float>(g, c, i, j, k, dn_at);
        dnew[c] = dc;
        q[c] = qv;
        acc[0] += double(dc) * double(qv);
      }
      block_sum<1>(acc, scratch);
      if (threadIdx.x == 0) pr.buf(phase)[blockIdx.x] = acc[0];
      if (!grid_sync(gs)) return;
      double dq[1];
      reduce_partials<1>(pr.buf(phase), gridDim.x, dq, scratch);
      ++phase;
      if (!(fabs(dq[0]) >= 1e-30)) break;
      const float af = float(delta / dq[0]);
      double acc2[1] = {0.0};
      for (int c = t0; c < g.n; c += stride) {
        const float dc = dnew[c];
        e[c] = e[c] + af * dc;
        const float rv = r[c] - af * q[c];
        r[c] = rv;
        acc2[0] += double(rv) * double(rv);
      }
      block_sum<1>(acc2, scratch);
      if (threadIdx.x == 0) pr.buf(phase)[blockIdx.x] = acc2[0];
      if (!grid_sync(gs)) return;
      double dn[1];
      reduce_partials<1>(pr.buf(phase), gridDim.x, dn, scratch);
      ++phase;
      ++it;
      ++total;
      if (!isfinite(dn[0]) || dn[0] <= inner_tol2 || dn[0] < 1e-30) break;
      beta = dn[0] / delta;
      delta = dn[0];
      float *t = dold;
      dold = dnew;
      dnew = t;
    }
    // p += e (f64), then the true residual again.
    for (int c = t0; c < g.n; c += stride) p[c] = p[c] + double(e[c]);
    if (!grid_sync(gs)) return;
    outer_residual(false);
    if (!grid_sync(gs)) return;
    reduce_partials<3>(pr.buf(phase), gridDim.x, tot, scratch);
    ++phase;
    rr = tot[0];
    ++passes;
    if (rr < 1e-20 || (tol2 >= 0.0 && rr <= tol2)) converged = 1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && a.report) {
    SolveReport rep;
    rep.iterations = total;
    rep.refinements = passes;
    rep.converged = converged;
    rep.status = isfinite(rr) ? 0 : 4;
    rep.initial_residual = sqrt(rr0);
    rep.final_residual = sqrt(rr);
    rep.rhs_norm = sqrt(bb);
    *a.report = rep;
  }
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
  for (int sweep = 0; sweep < a.sweeps; ++sweep) {
    for (int color = 0; color < 2; ++color) {
      for (int c = t0; c < g.n; c += stride) {
        int i, j, k;
        decode(g, c, i, j, k);
        if (!interior(g, i, j, k) || ((i + j + k) & 1) != color) continue;
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

int persistent_blocks_cg_mixed() {
  return blocks_for(reinterpret_cast<const void *>(&k_cg_mixed));
}
int persistent_blocks_sor_mixed() {
  return blocks_for(reinterpret_cast<const void *>(&k_rbsor_mixed));
}

int launch_cg_mixed(const MixedCgArgs &a, const PersistentState &ps, cudaStream_t st) {
  int blocks = persistent_blocks_cg_mixed();
  if (blocks > ps.max_blocks) blocks = ps.max_blocks;
  cudaMemsetAsync(ps.count, 0, sizeof(unsigned int), st);
  cudaMemsetAsync(ps.gen, 0, sizeof(unsigned int), st);
  cudaMemsetAsync(ps.abort_flag, 0, sizeof(int), st);
  MixedCgArgs args = a;
  GridSync gs = make_sync(ps, blocks);
  Ring pr{ps.partials, 3 * ps.max_blocks};
  void *params[] = {&args, &gs, &pr};
  const cudaError_t err = cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(&k_cg_mixed), dim3(blocks),
                              dim3(kBlock), params, 0, st);
  return err == cudaSuccess ? blocks : -static_cast<int>(err);
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
