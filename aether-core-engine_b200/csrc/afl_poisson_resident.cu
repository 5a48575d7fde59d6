// afl_poisson_resident.cu -- on-chip resident CG solves for grids that fit.
//
// One 1024-thread CTA per SM owns a column tile of 16 x TY cells in x-y that
// spans every z plane.  During the solve nothing of the tile leaves the SM:
//   * the search direction d lives in shared memory (tile + one-cell halo
//     ring in x and y), because the 7-point operator reads it at neighbours;
//   * the residual r (and, in the mixed form, the f32 correction e) live in
//     registers, CPT consecutive z cells per thread.
// Per iteration only the tile-edge values cross L2: each CTA publishes the
// r and d of its edge cells, and rebuilds its halo ring from its neighbours'
// published values.  The direction update d = r + beta*d (src/fluid.rs:483-485)
// is evaluated for halo cells from the neighbours' published r and previous d
// with the same expression the owner uses, so halo and owner agree bit for bit
// and an iteration needs two grid barriers, as in the streaming kernel.
//
// Built with -fmad=false: the FP64 kernel keeps the reference's un-fused
// arithmetic; the mixed kernel writes its FMAs explicitly (__fmaf_rn), so
// owner and halo evaluate identical operations.
#include "afl_launch.h"

namespace afl {
namespace {

constexpr int kRT = 1024;       // threads per CTA
constexpr int kRW = kRT / 32;   // warps per CTA
constexpr int kTX = 16;         // tile width in x (cells): one half-warp reads one row

// CTA-wide sum of NV values, valid in every thread.  Warp butterflies, then
// warp 0 combines the 32 warp sums with another butterfly: a fixed order, so
// CTAs reducing the same data get the same bits.  `scratch` holds
// kRW*NV + NV doubles.
template <int NV>
__device__ __forceinline__ void bsum(double (&v)[NV], double *scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < NV; ++a) v[a] = warp_sum(v[a]);
  if (lane == 0)
#pragma unroll
    for (int a = 0; a < NV; ++a) scratch[warp * NV + a] = v[a];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int a = 0; a < NV; ++a) {
      const double x = warp_sum(scratch[lane * NV + a]);
      if (lane == 0) scratch[kRW * NV + a] = x;
    }
  }
  __syncthreads();
#pragma unroll
  for (int a = 0; a < NV; ++a) v[a] = scratch[kRW * NV + a];
}

// Fixed-order sum of NV interleaved per-CTA partials, read by warp 0 and
// broadcast through `slot` (NV doubles); identical in every CTA.
template <int NV>
__device__ __forceinline__ void reduce_parts(const double *parts, int nparts,
                                             double (&out)[NV], double *slot) {
  if (threadIdx.x < 32) {
    double acc[NV];
#pragma unroll
    for (int a = 0; a < NV; ++a) acc[a] = 0.0;
    for (int b = threadIdx.x; b < nparts; b += 32)
#pragma unroll
      for (int a = 0; a < NV; ++a) acc[a] += __ldcg(parts + b * NV + a);
#pragma unroll
    for (int a = 0; a < NV; ++a) {
      acc[a] = warp_sum(acc[a]);
      if (threadIdx.x == 0) slot[a] = acc[a];
    }
  }
  __syncthreads();
#pragma unroll
  for (int a = 0; a < NV; ++a) out[a] = slot[a];
}

// Sums NV values over the CTA (same fixed order as bsum) and stores the CTA's
// partials to parts[blockIdx.x*NV + a]; only warp 0 sees the sum, so one CTA
// barrier suffices (the grid barrier that follows starts with another).
template <int NV>
__device__ __forceinline__ void publish_sum(double *parts, double (&v)[NV], double *scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < NV; ++a) v[a] = warp_sum(v[a]);
  if (lane == 0)
#pragma unroll
    for (int a = 0; a < NV; ++a) scratch[warp * NV + a] = v[a];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int a = 0; a < NV; ++a) {
      const double x = warp_sum(scratch[lane * NV + a]);
      if (lane == 0) parts[blockIdx.x * NV + a] = x;
    }
  }
}

// Where this thread's cells sit: column (ii, jj) of the tile, planes
// k0 .. k0+CPT-1, and the operator's x/y neighbour tests, which are the same
// for all of the thread's cells.
// Shared-memory plane stride: the (kTX+2) x (TY+2) plane padded to an odd
// number of words, so that the two half-warps (which work CPT planes apart)
// hit disjoint banks.
template <int TY>
struct Plane {
  static constexpr int SX = kTX + 2;
  static constexpr int kRaw = (kTX + 2) * (TY + 2);
  static constexpr int SXY = kRaw | 1;
};

template <int TY, int CPT>
struct Cells {
  static constexpr int kCols = kTX * TY;
  static_assert(kRT % (2 * kCols) == 0, "a CTA must cover whole pairs of column groups");
  static constexpr int SX = Plane<TY>::SX;
  static constexpr int SXY = Plane<TY>::SXY;
  static constexpr int kPlanes = (kRT / kCols) * CPT;  // planes the threads cover (>= nz)
  int i, j, k0;
  int c0, s0;        // global / shared index of plane k0
  bool in_ij;        // column inside the grid
  bool ij_interior;  // 1 <= i <= nx-2 and 1 <= j <= ny-2
  bool edge;         // value needed by a neighbouring tile
  bool xl, xh, yl, yh;  // i > 1, i+2 < nx, j > 1, j+2 < ny
  int diag_xy;          // x/y neighbours present (the operator's diagonal part)
  __device__ Cells(const Dims &g, int tiles_x) {
    // lane bits 0-3: x in the tile; bit 4: which of a pair of plane groups;
    // then the row jj, then the group pair.
    const int t = threadIdx.x;
    const int ii = t & (kTX - 1);
    const int half = (t >> 4) & 1;
    const int row_pair = t >> 5;
    const int jj = row_pair % TY;
    const int grp = 2 * (row_pair / TY) + half;
    const int bx = blockIdx.x % tiles_x, by = blockIdx.x / tiles_x;
    i = bx * kTX + ii;
    j = by * TY + jj;
    k0 = grp * CPT;
    in_ij = i < g.nx && j < g.ny;
    ij_interior = i >= 1 && i <= g.nx - 2 && j >= 1 && j <= g.ny - 2;
    edge = ii == 0 || ii == kTX - 1 || jj == 0 || jj == TY - 1;
    xl = i > 1;
    xh = i + 2 < g.nx;
    yl = j > 1;
    yh = j + 2 < g.ny;
    diag_xy = int(xl) + int(xh) + int(yl) + int(yh);
    c0 = (k0 * g.ny + j) * g.nx + i;
    s0 = k0 * SXY + (jj + 1) * SX + ii + 1;
  }
  __device__ bool valid(const Dims &g, int m) const { return in_ij && k0 + m < g.nz; }
  __device__ bool interior(const Dims &g, int m) const {
    const int k = k0 + m;
    return ij_interior && k >= 1 && k <= g.nz - 2;
  }
};

// The reference operator (src/fluid.rs:356-394) on the shared-memory tile,
// without branches: a missing neighbour contributes a selected 0 to the sum
// (the reference skips it; the sum is the same value), the diagonal is the
// count of present neighbours.  Shared slots of missing neighbours are never
// used, whatever they hold.
template <typename R, int SX, int SXY, typename Cl>
__device__ __forceinline__ R lap_smem(const Dims &g, const R *D, int s, const Cl &cl, int k) {
  const bool zl = k > 1, zh = k + 2 < g.nz;
  R nb = cl.xl ? D[s - 1] : R(0);
  nb += cl.xh ? D[s + 1] : R(0);
  nb += cl.yl ? D[s - SX] : R(0);
  nb += cl.yh ? D[s + SX] : R(0);
  nb += zl ? D[s - SXY] : R(0);
  nb += zh ? D[s + SXY] : R(0);
  const R diag = R(cl.diag_xy + int(zl) + int(zh));
  return diag * D[s] - nb;
}

// The same operator on the f64 pressure in global memory (L2 reads: the
// pressure is written by other CTAs between passes).
__device__ __forceinline__ double lap_global(const Dims &g, const double *x, int c, int i, int j,
                                             int k) {
  double diag = 0.0, nb = 0.0;
  if (i > 1) { diag += 1.0; nb += __ldcg(x + c - 1); }
  if (i + 2 < g.nx) { diag += 1.0; nb += __ldcg(x + c + 1); }
  if (j > 1) { diag += 1.0; nb += __ldcg(x + c - g.nx); }
  if (j + 2 < g.ny) { diag += 1.0; nb += __ldcg(x + c + g.nx); }
  if (k > 1) { diag += 1.0; nb += __ldcg(x + c - g.nxy); }
  if (k + 2 < g.nz) { diag += 1.0; nb += __ldcg(x + c + g.nxy); }
  return diag * __ldcg(x + c) - nb;
}

// The halo ring (x and y neighbours of the tile, every plane): 2*TY + 2*kTX
// cells per plane, padded to kPad so that each thread keeps one ring position
// (computed once) and serves it in every kLanes-th plane.  Ring positions
// outside the grid are skipped (the operator never reads them).  The ring
// keeps last iteration's directions, so a new ring direction needs only the
// neighbour's published residual: d = r + beta*d_ring, the owner's expression
// on the owner's operands.
template <int TY>
struct Halo {
  static constexpr int kPerPlane = 2 * TY + 2 * kTX;
  static constexpr int kPad = kPerPlane <= 64 ? 64 : 128;
  static constexpr int kLanes = kRT / kPad;
  bool active;
  int col_c, col_s, k_first;
  __device__ Halo(const Dims &g, int tiles_x) {
    constexpr int SX = Plane<TY>::SX;
    const int q = threadIdx.x % kPad;
    k_first = threadIdx.x / kPad;
    const int bx0 = (blockIdx.x % tiles_x) * kTX, by0 = (blockIdx.x / tiles_x) * TY;
    int ii, jj;
    if (q < 2 * kTX) {  // the rows below and above the tile
      jj = q < kTX ? -1 : TY;
      ii = q < kTX ? q : q - kTX;
    } else {            // the columns left and right of the tile
      const int r = q - 2 * kTX;
      ii = r < TY ? -1 : kTX;
      jj = r < TY ? r : r - TY;
    }
    const int i = bx0 + ii, j = by0 + jj;
    active = q < kPerPlane && i >= 0 && i < g.nx && j >= 0 && j < g.ny;
    col_c = j * g.nx + i;
    col_s = (jj + 1) * SX + ii + 1;
  }
  // D[ring cell] = value_at(global cell, D[ring cell]) for every plane.
  template <typename R, typename F>
  __device__ __forceinline__ void fill(const Dims &g, R *D, const F &value_at) const {
    constexpr int SXY = Plane<TY>::SXY;
    if (!active) return;
#pragma unroll 4
    for (int k = k_first; k < g.nz; k += kLanes) {
      R &slot = D[k * SXY + col_s];
      slot = value_at(k * g.nxy + col_c, slot);
    }
  }
};

struct Ring2 {
  double *base;
  int stride;
  __device__ double *buf(int phase) const { return base + (phase & 1) * stride; }
};

// Shared scratch of the reductions: per-warp values, the CTA result, and the
// broadcast slot of the grid-wide sums.
constexpr int kScratch = kRW * 3 + 3 + 3;

// ---------------------------------------------------------------- FP64 ------
// solve_poisson_conjugate_gradient (src/fluid.rs:445-493) with the relative
// tolerance extension.  d in shared memory, r in registers, p in global memory
// (updated once per iteration, never read by the operator).
template <int TY, int CPT>
__global__ void __launch_bounds__(kRT, 1)
    k_cg_res_f64(ResidentCgArgs a, GridSync gs, Ring2 pr) {
  using C = Cells<TY, CPT>;
  extern __shared__ double Dbase[];
  double *D = Dbase + C::SXY;  // one padding plane below plane 0
  __shared__ double scratch[kScratch];
  double *slot = scratch + kRW * 3 + 3;
  const Dims g = a.g;
  const C cl(g, a.tiles_x);
  const Halo<TY> halo(g, a.tiles_x);
  double *p = a.p;
  double *rpub = static_cast<double *>(a.rpub);
  double r[CPT];
  int phase = 0;
  {
    double acc[2] = {0.0, 0.0};
#pragma unroll
    for (int m = 0; m < CPT; ++m) {
      r[m] = 0.0;
      if (!cl.valid(g, m)) continue;
      const int c = cl.c0 + m * g.nxy;
      const double ap = cl.interior(g, m) ? lap_global(g, p, c, cl.i, cl.j, cl.k0 + m) : 0.0;
      const double bc = __ldg(a.b + c);
      const double rv = bc - ap;
      r[m] = rv;
      if (cl.edge) rpub[c] = rv;
      acc[0] += rv * rv;
      acc[1] += bc * bc;
    }
    publish_sum<2>(pr.buf(phase), acc, scratch);
  }
  if (!grid_sync(gs)) return;
  double tot[2];
  reduce_parts<2>(pr.buf(phase), gridDim.x, tot, slot);
  ++phase;
  double delta = tot[0];
  const double bb = tot[1];
  double tol2 = -1.0;
  if (a.rel_tol > 0.0) {
    const double tl = a.rel_tol * sqrt(bb);
    tol2 = tl * tl;
  }
  const double delta0 = delta;
  double last = delta;
  int it = 0, converged = 0;
  if (!(delta > 1e-24) || (tol2 >= 0.0 && delta <= tol2)) {
    converged = isfinite(delta) ? 1 : 0;
  } else {
    double beta = 0.0;
    while (it < a.max_iters) {
      const bool first = it == 0;
      // d = r + beta*d on the tile and its halo ring (src/fluid.rs:483-485).
      // Cells past the grid hold r = 0, so their d stays 0: the loops below
      // need no per-cell branches (padding planes keep every slot in bounds).
#pragma unroll
      for (int m = 0; m < CPT; ++m) {
        const int s = cl.s0 + m * C::SXY;
        D[s] = first ? r[m] : r[m] + beta * D[s];
      }
      halo.fill(g, D, [&](int c, double dprev) {
        const double rv = __ldcg(rpub + c);
        return first ? rv : rv + beta * dprev;
      });
      __syncthreads();
      double acc[1] = {0.0};
#pragma unroll
      for (int m = 0; m < CPT; ++m) {
        const int s = cl.s0 + m * C::SXY;
        const double qv = lap_smem<double, C::SX, C::SXY>(g, D, s, cl, cl.k0 + m);
        acc[0] += cl.interior(g, m) ? D[s] * qv : 0.0;
      }
      publish_sum<1>(pr.buf(phase), acc, scratch);
      if (!grid_sync(gs)) return;
      double dq[1];
      reduce_parts<1>(pr.buf(phase), gridDim.x, dq, slot);
      ++phase;
      if (fabs(dq[0]) < 1e-28) break;  // src/fluid.rs:469
      const double alpha = delta / dq[0];
      double acc2[1] = {0.0};
#pragma unroll
      for (int m = 0; m < CPT; ++m) {
        const int s = cl.s0 + m * C::SXY;
        const int c = cl.c0 + m * g.nxy;
        const double lq = lap_smem<double, C::SX, C::SXY>(g, D, s, cl, cl.k0 + m);
        const double qv = cl.interior(g, m) ? lq : 0.0;
        const bool v = cl.valid(g, m);
        if (v) p[c] = p[c] + alpha * D[s];
        const double rv = r[m] - alpha * qv;
        r[m] = rv;
        if (v && cl.edge) rpub[c] = rv;
        acc2[0] += rv * rv;
      }
      publish_sum<1>(pr.buf(phase), acc2, scratch);
      if (!grid_sync(gs)) return;
      double dn[1];
      reduce_parts<1>(pr.buf(phase), gridDim.x, dn, slot);
      ++phase;
      ++it;
      last = dn[0];
      if (!isfinite(dn[0])) break;
      if (dn[0] < 1e-20) { converged = 1; break; }  // src/fluid.rs:479
      if (tol2 >= 0.0 && dn[0] <= tol2) { converged = 1; break; }
      beta = dn[0] / delta;  // src/fluid.rs:482
      delta = dn[0];
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

// ---------------------------------------------------------------- mixed -----
// f64 refinement around an f32 CG whose vectors never leave the SM: d and the
// correction e in shared memory (same tile layout), r in registers.
template <int TY, int CPT>
__global__ void __launch_bounds__(kRT, 1)
    k_cg_res_mixed(ResidentCgArgs a, GridSync gs, Ring2 pr) {
  using C = Cells<TY, CPT>;
  extern __shared__ float Dfbase[];
  float *Df = Dfbase + C::SXY;  // one padding plane below plane 0
  __shared__ double scratch[kScratch];
  double *slot = scratch + kRW * 3 + 3;
  const Dims g = a.g;
  const C cl(g, a.tiles_x);
  const Halo<TY> halo(g, a.tiles_x);
  float *E = Df + C::SXY * (C::kPlanes + 2);  // the correction, same tile layout
  double *p = a.p;
  float *rpub = static_cast<float *>(a.rpub);
  float r[CPT];
  int phase = 0;

  // r = b - A p in f64, rounded once to f32; e = 0.
  auto outer_residual = [&](bool with_b) {
    double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int m = 0; m < CPT; ++m) {
      r[m] = 0.0f;
      E[cl.s0 + m * C::SXY] = 0.0f;
      if (!cl.valid(g, m)) continue;
      const int c = cl.c0 + m * g.nxy;
      const double ap = cl.interior(g, m) ? lap_global(g, p, c, cl.i, cl.j, cl.k0 + m) : 0.0;
      const double bc = __ldg(a.b + c);
      const double rv = bc - ap;
      const float rf = float(rv);
      r[m] = rf;
      if (cl.edge) rpub[c] = rf;
      acc[0] += rv * rv;
      if (with_b) acc[1] += bc * bc;
      acc[2] += double(rf) * double(rf);
    }
    publish_sum<3>(pr.buf(phase), acc, scratch);
  };

  outer_residual(true);
  if (!grid_sync(gs)) return;
  double tot[3];
  reduce_parts<3>(pr.buf(phase), gridDim.x, tot, slot);
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
  if (!(rr > 1e-24) || (tol2 >= 0.0 && rr <= tol2)) converged = isfinite(rr) ? 1 : 0;

  while (!converged && passes < a.max_refine && total < a.max_iters && isfinite(rr)) {
    double inner_rel = a.inner_rel_tol;
    if (tol2 >= 0.0) inner_rel = fmax(inner_rel, 0.5 * sqrt(tol2 / rr));
    double delta = tot[2];
    const double inner_tol2 = inner_rel * inner_rel * delta;
    double beta = 0.0;
    int it = 0;
    while (it < a.max_inner && total < a.max_iters) {
      const bool first = it == 0;
      const float bf = float(beta);
#pragma unroll
      for (int m = 0; m < CPT; ++m) {
        const int s = cl.s0 + m * C::SXY;
        Df[s] = first ? r[m] : __fmaf_rn(bf, Df[s], r[m]);
      }
      halo.fill(g, Df, [&](int c, float dprev) {
        const float rv = __ldcg(rpub + c);
        return first ? rv : __fmaf_rn(bf, dprev, rv);
      });
      __syncthreads();
      double acc[1] = {0.0};
#pragma unroll
      for (int m = 0; m < CPT; ++m) {
        const int s = cl.s0 + m * C::SXY;
        const float qv = lap_smem<float, C::SX, C::SXY>(g, Df, s, cl, cl.k0 + m);
        acc[0] += cl.interior(g, m) ? double(Df[s]) * double(qv) : 0.0;
      }
      publish_sum<1>(pr.buf(phase), acc, scratch);
      if (!grid_sync(gs)) return;
      double dq[1];
      reduce_parts<1>(pr.buf(phase), gridDim.x, dq, slot);
      ++phase;
      if (!(fabs(dq[0]) >= 1e-30)) break;
      const float af = float(delta / dq[0]);
      double acc2[1] = {0.0};
#pragma unroll
      for (int m = 0; m < CPT; ++m) {
        const int s = cl.s0 + m * C::SXY;
        const float lq = lap_smem<float, C::SX, C::SXY>(g, Df, s, cl, cl.k0 + m);
        const float qv = cl.interior(g, m) ? lq : 0.0f;
        E[s] = __fmaf_rn(af, Df[s], E[s]);
        const float rv = __fmaf_rn(-af, qv, r[m]);
        r[m] = rv;
        if (cl.edge && cl.valid(g, m)) rpub[cl.c0 + m * g.nxy] = rv;
        acc2[0] += double(rv) * double(rv);
      }
      publish_sum<1>(pr.buf(phase), acc2, scratch);
      if (!grid_sync(gs)) return;
      double dn[1];
      reduce_parts<1>(pr.buf(phase), gridDim.x, dn, slot);
      ++phase;
      ++it;
      ++total;
      if (!isfinite(dn[0]) || dn[0] <= inner_tol2 || dn[0] < 1e-30) break;
      beta = dn[0] / delta;
      delta = dn[0];
    }
    // p += e in f64, then the true residual again.
#pragma unroll
    for (int m = 0; m < CPT; ++m) {
      if (!cl.valid(g, m)) continue;
      const int c = cl.c0 + m * g.nxy;
      p[c] = p[c] + double(E[cl.s0 + m * C::SXY]);
    }
    if (!grid_sync(gs)) return;
    outer_residual(false);
    if (!grid_sync(gs)) return;
    reduce_parts<3>(pr.buf(phase), gridDim.x, tot, slot);
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

// ---------------------------------------------------------------- dispatch --
using KernelFn = void (*)(ResidentCgArgs, GridSync, Ring2);

template <int TY, int CPT>
KernelFn pick_kernel(bool f64) {
  return f64 ? &k_cg_res_f64<TY, CPT> : &k_cg_res_mixed<TY, CPT>;
}

KernelFn kernel_for(bool f64, int ty, int cpt) {
#define AFL_RES_CASE(TY_, CPT_) \
  if (ty == TY_ && cpt == CPT_) return pick_kernel<TY_, CPT_>(f64);
  AFL_RES_CASE(4, 1) AFL_RES_CASE(4, 2) AFL_RES_CASE(4, 4) AFL_RES_CASE(4, 8) AFL_RES_CASE(4, 16)
  AFL_RES_CASE(8, 1) AFL_RES_CASE(8, 2) AFL_RES_CASE(8, 4) AFL_RES_CASE(8, 8) AFL_RES_CASE(8, 16)
  AFL_RES_CASE(16, 1) AFL_RES_CASE(16, 2) AFL_RES_CASE(16, 4) AFL_RES_CASE(16, 8)
  AFL_RES_CASE(16, 16)
#undef AFL_RES_CASE
  return nullptr;
}

}  // namespace

size_t resident_smem_bytes(const Dims &g, int ty, int cpt, bool f64) {
  // FP64: the direction tile.  Mixed: direction and correction tiles (f32).
  // Planes: those the threads cover (groups*cpt >= nz) plus one padding plane
  // on each side, so every shared access of the branch-free loops is in bounds.
  (void)g;
  const size_t plane = static_cast<size_t>((kTX + 2) * (ty + 2)) | 1u;
  const size_t planes = static_cast<size_t>(kRT / (kTX * ty)) * cpt + 2;
  const size_t tile = plane * planes;
  return f64 ? tile * sizeof(double) : 2 * tile * sizeof(float);
}

bool plan_resident(const Dims &g, bool f64, ResidentPlan *plan) {
  int dev = 0, sms = 0, smem_optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const size_t static_smem = 2048;  // reduction scratch + barrier flag, rounded up
  bool found = false;
  ResidentPlan best{};
  for (int ty : {4, 8, 16}) {
    const int groups = kRT / (kTX * ty);
    int cpt = (g.nz + groups - 1) / groups;
    int rounded = 1;
    while (rounded < cpt) rounded *= 2;
    if (rounded > 16) continue;
    const int tiles_x = (g.nx + kTX - 1) / kTX;
    const int tiles_y = (g.ny + ty - 1) / ty;
    const int tiles = tiles_x * tiles_y;
    if (tiles > sms) continue;
    const size_t smem = resident_smem_bytes(g, ty, rounded, f64);
    if (smem + static_smem > static_cast<size_t>(smem_optin)) continue;
    ResidentPlan cand{ty, rounded, tiles_x, tiles_y, static_cast<int>(smem)};
    // fewest cells per thread first, then the smaller halo (larger tile)
    if (!found || cand.cpt < best.cpt || (cand.cpt == best.cpt && cand.ty > best.ty)) {
      best = cand;
      found = true;
    }
  }
  if (found && plan) *plan = best;
  return found;
}

int launch_cg_resident(const ResidentCgArgs &a, const ResidentPlan &plan, bool f64,
                       const PersistentState &ps, cudaStream_t st) {
  KernelFn fn = kernel_for(f64, plan.ty, plan.cpt);
  if (!fn) return -static_cast<int>(cudaErrorInvalidConfiguration);
  const int blocks = plan.tiles_x * plan.tiles_y;
  if (blocks > ps.max_blocks) return -static_cast<int>(cudaErrorInvalidConfiguration);
  cudaError_t err = cudaFuncSetAttribute(reinterpret_cast<const void *>(fn),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         plan.smem_bytes);
  if (err != cudaSuccess) return -static_cast<int>(err);
  cudaMemsetAsync(ps.count, 0, sizeof(unsigned int), st);
  cudaMemsetAsync(ps.gen, 0, sizeof(unsigned int), st);
  cudaMemsetAsync(ps.abort_flag, 0, sizeof(int), st);
  ResidentCgArgs args = a;
  args.tiles_x = plan.tiles_x;
  args.tiles_y = plan.tiles_y;
  GridSync gs;
  gs.count = ps.count;
  gs.gen = ps.gen;
  gs.abort_flag = ps.abort_flag;
  gs.nblocks = static_cast<unsigned int>(blocks);
  gs.timeout_ns = ps.timeout_ns;
  Ring2 pr{ps.partials, 3 * ps.max_blocks};
  void *params[] = {&args, &gs, &pr};
  err = cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(fn), dim3(blocks), dim3(kRT),
                                    params, static_cast<size_t>(plan.smem_bytes), st);
  return err == cudaSuccess ? blocks : -static_cast<int>(err);
}

}  // namespace afl
