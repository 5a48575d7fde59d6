// afl_poisson_f64.cu -- FP64 pressure solves as single persistent launches.
//
// Built with -fmad=false: every update is the reference's un-fused
// expression, so the CG iterates differ from the reference only through the
// summation order of the two inner products, and an RB-SOR sweep reproduces
// the reference bit for bit (each colour reads only the other colour).
//
// One cooperative launch runs the whole solve.  All CTAs stay resident; phases
// are separated by the bounded grid barrier of afl_device.cuh, and every CTA
// reduces the per-CTA partials itself, in the same order, so all of them take
// identical decisions (alpha, beta, the stopping tests) with no extra barrier.
#include "afl_launch.h"

namespace afl {
namespace {

// 7-point pure-Neumann -Laplacian of src/fluid.rs:356-394 at interior cell c;
// the neighbour sum keeps the reference's order (i-1, i+1, j-1, j+1, k-1,
// k+1).  `X` returns the operand value at a cell.
template <typename X>
__device__ __forceinline__ double spd_lap(const Dims &g, int c, int i, int j, int k,
                                          const X &x) {
  double diag = 0.0, nb = 0.0;
  if (i > 1) { diag += 1.0; nb += x(c - 1); }
  if (i + 2 < g.nx) { diag += 1.0; nb += x(c + 1); }
  if (j > 1) { diag += 1.0; nb += x(c - g.nx); }
  if (j + 2 < g.ny) { diag += 1.0; nb += x(c + g.nx); }
  if (k > 1) { diag += 1.0; nb += x(c - g.nxy); }
  if (k + 2 < g.nz) { diag += 1.0; nb += x(c + g.nxy); }
  return diag * x(c) - nb;
}

struct PartialRing {
  double *base;
  int stride;  // doubles per buffer
  __device__ double *buf(int phase) const { return base + (phase & 1) * stride; }
};

// solve_poisson_conjugate_gradient (src/fluid.rs:445-493) with the relative
// tolerance extension.  The direction update d = r + beta*d (:483-485) is
// folded into the next matrix-vector product: each thread forms the new
// direction at its cell and its six neighbours from r and the previous
// direction (double-buffered d0/d1), so an iteration needs two barriers.
__global__ void __launch_bounds__(kBlock)
    k_cg_f64(CgArgs a, GridSync gs, PartialRing pr) {
  __shared__ double scratch[kWarps * 2];
  const Dims g = a.g;
  const int t0 = blockIdx.x * kBlock + threadIdx.x;
  const int stride = gridDim.x * kBlock;
  double *p = a.p;
  double *r = a.r;
  double *q = a.q;
  const double *b = a.b;
  int phase = 0;

  // r = b - A p (q = 0 off the interior), delta = r.r, and ||b||^2.
  {
    double acc[2] = {0.0, 0.0};
    for (int c = t0; c < g.n; c += stride) {
      int i, j, k;
      decode(g, c, i, j, k);
      double ap = 0.0;
      if (interior(g, i, j, k)) ap = spd_lap(g, c, i, j, k, [&](int x) { return p[x]; });
      const double bc = __ldg(b + c);
      const double rv = bc - ap;
      r[c] = rv;
      acc[0] += rv * rv;
      acc[1] += bc * bc;
    }
    block_sum<2>(acc, scratch);
    if (threadIdx.x == 0) {
      pr.buf(phase)[blockIdx.x * 2 + 0] = acc[0];
      pr.buf(phase)[blockIdx.x * 2 + 1] = acc[1];
    }
  }
  if (!grid_sync(gs)) return;
  double tot[2];
  reduce_partials<2>(pr.buf(phase), gridDim.x, tot, scratch);
  ++phase;
  double delta = tot[0];
  const double bb = tot[1];
  double tol2 = -1.0;
  if (a.rel_tol > 0.0) {
    const double tl = a.rel_tol * sqrt(bb);
    tol2 = tl * tl;
  }
  const double delta0 = delta;
  int it = 0;
  int converged = 0;
  double last = delta;
  if (!(delta > 1e-24) || (tol2 >= 0.0 && delta <= tol2)) {
    converged = 1;
  } else {
    double beta = 0.0;
    double *dold = a.d0, *dnew = a.d1;
    while (it < a.max_iters) {
      // q = A dn with dn = r + beta*dold formed on the fly; partial d.q.
      double acc[1] = {0.0};
      const bool first = (it == 0);
      auto dn_at = [&](int x) { return first ? r[x] : r[x] + beta * dold[x]; };
      for (int c = t0; c < g.n; c += stride) {
        int i, j, k;
        decode(g, c, i, j, k);
        const double dc = dn_at(c);
        double qv = 0.0;
        if (interior(g, i, j, k)) qv = spd_lap(g, c, i, j, k, dn_at);
        dnew[c] = dc;
        q[c] = qv;
        acc[0] += dc * qv;
      }
      block_sum<1>(acc, scratch);
      if (threadIdx.x == 0) pr.buf(phase)[blockIdx.x] = acc[0];
      if (!grid_sync(gs)) return;
      double dq[1];
      reduce_partials<1>(pr.buf(phase), gridDim.x, dq, scratch);
      ++phase;
      if (fabs(dq[0]) < 1e-28) break;  // src/fluid.rs:469
      const double alpha = delta / dq[0];
      // p += alpha d; r -= alpha q; partial r.r  (src/fluid.rs:473-478)
      double acc2[1] = {0.0};
      for (int c = t0; c < g.n; c += stride) {
        const double dc = dnew[c];
        p[c] = p[c] + alpha * dc;
        const double rv = r[c] - alpha * q[c];
        r[c] = rv;
        acc2[0] += rv * rv;
      }
      block_sum<1>(acc2, scratch);
      if (threadIdx.x == 0) pr.buf(phase)[blockIdx.x] = acc2[0];
      if (!grid_sync(gs)) return;
      double dn[1];
      reduce_partials<1>(pr.buf(phase), gridDim.x, dn, scratch);
      ++phase;
      ++it;
      last = dn[0];
      if (!isfinite(dn[0])) break;  // NaN/Inf: nothing further can converge
      if (dn[0] < 1e-20) { converged = 1; break; }             // src/fluid.rs:479
      if (tol2 >= 0.0 && dn[0] <= tol2) { converged = 1; break; }
      beta = dn[0] / delta;                                     // src/fluid.rs:482
      delta = dn[0];
      double *t = dold;
      dold = dnew;
      dnew = t;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && a.report) {
    SolveReport rep;
    rep.iterations = it;
    rep.refinements = 0;
    rep.converged = converged;
    rep.status = isfinite(last) ? 0 : 4;
    rep.initial_residual = sqrt(delta0);
    rep.final_residual = sqrt(last);
    rep.rhs_norm = sqrt(bb);
    *a.report = rep;
  }
}

// solve_poisson_gauss_seidel (src/fluid.rs:397-442): colour 0 then colour 1
// per sweep, in place.  The update reads only the other colour, so the result
// does not depend on the order cells are visited and equals the reference's.
__global__ void __launch_bounds__(kBlock) k_rbsor_f64(SorArgs a, GridSync gs) {
  const Dims g = a.g;
  const int t0 = blockIdx.x * kBlock + threadIdx.x;
  const int stride = gridDim.x * kBlock;
  double *p = a.p;
  const double omega = a.omega;
  for (int sweep = 0; sweep < a.sweeps; ++sweep) {
    for (int color = 0; color < 2; ++color) {
      for (int c = t0; c < g.n; c += stride) {
        int i, j, k;
        decode(g, c, i, j, k);
        if (!interior(g, i, j, k) || ((i + j + k) & 1) != color) continue;
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

int persistent_blocks_cg_f64() { return blocks_for(reinterpret_cast<const void *>(&k_cg_f64)); }
int persistent_blocks_sor_f64() {
  return blocks_for(reinterpret_cast<const void *>(&k_rbsor_f64));
}

int launch_cg_f64(const CgArgs &a, const PersistentState &ps, cudaStream_t st) {
  int blocks = persistent_blocks_cg_f64();
  if (blocks > ps.max_blocks) blocks = ps.max_blocks;
  cudaMemsetAsync(ps.count, 0, sizeof(unsigned int), st);
  cudaMemsetAsync(ps.gen, 0, sizeof(unsigned int), st);
  cudaMemsetAsync(ps.abort_flag, 0, sizeof(int), st);
  CgArgs args = a;
  GridSync gs = make_sync(ps, blocks);
  PartialRing pr{ps.partials, 2 * ps.max_blocks};
  void *params[] = {&args, &gs, &pr};
  const cudaError_t err = cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(&k_cg_f64), dim3(blocks),
                              dim3(kBlock), params, 0, st);
  return err == cudaSuccess ? blocks : -static_cast<int>(err);
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
