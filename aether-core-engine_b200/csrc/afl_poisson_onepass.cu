// afl_poisson_onepass.cu -- the mixed form's f32 CG for grids that do not fit
// on chip, at one pass over the grid and one grid barrier per iteration.
//
// The two-pass streaming CG (afl_poisson_stream.cu) reads and writes its
// vectors twice per iteration, around two grid-wide sums.  Here an
// iteration's update is deferred into the next iteration's pass:
//   pass m (coefficients alpha, beta of iteration m-1, stored r, d, e of
//   iteration m-1):  q' = A d (recomputed), r = r - alpha q', d = r + beta d,
//   e = e + alpha d_old, q = A d, and the sums d.q, r.q, q.q, r.r.
// After the sum, alpha = (r.r)/(d.q) and the next r.r is the same number
// expanded, r.r - 2 alpha r.q + alpha^2 q.q, which gives beta without a
// second sum (src/fluid.rs:465-485).  d at a cell's neighbours needs q' at
// theirs, so each CTA stages the old d with a two-cell halo and the old r with
// a one-cell halo in shared memory (asynchronous copies, several planes
// ahead), computes q' and the new d on its tile plus a one-cell ring, and
// then q on its tile.  HBM sees r, d and e read once and written once per
// iteration: 24 bytes per cell, against 28-32 for the two-pass form.
//
// Work is a list of (32 x 8 column tile, chunk of z planes) items that the
// persistent CTAs walk in a fixed order; r and d alternate between two
// buffers by pass parity, because neighbouring CTAs read the old values at
// tile edges while this one writes the new.  The f64 refinement around the
// f32 solve (residual b - A p in f64, p += e) is the two-pass kernel's.
// Built with -fmad=false; the f32 updates use explicit FMAs.
#include "afl_launch.h"
#include "afl_stage_fused.cuh"

namespace afl {
namespace {

constexpr int kOT = kFThreads;  // 256 threads: one per cell of a 32 x 8 plane tile
constexpr int kOS = 6;          // staged planes: d at k-2 .. k+2 for plane k, one ahead
constexpr int kOKz = 16;        // z planes per work item

using G = Staged<float>;
constexpr int kORW = G::RW;          // 40 floats: x halo of 4 (16 bytes)
constexpr int kOXH = G::XH;
constexpr int kODRows = kFy + 4;     // d: y halo 2
constexpr int kORRows = kFy + 2;     // r: y halo 1
constexpr int kODPlane = kODRows * kORW;
constexpr int kORPlane = kORRows * kORW;
constexpr int kOTile1 = kFh * kFw;   // tile + one-cell ring (34 x 10)
constexpr int kOSmemFloats = kOS * (kODPlane + kORPlane) + 2 * 3 * kOTile1;

struct OnePassArgs {
  MixedCgArgs a;
  float *rbuf[2];  // r by pass parity (a.r and a.q)
  float *dbuf[2];  // d by pass parity (a.d0 and a.d1)
  int tiles_x, tiles_y, chunks;
};

template <int NV>
__device__ __forceinline__ void publish(double *parts, double (&v)[NV], double *scratch) {
  constexpr int W = kOT / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int x = 0; x < NV; ++x) v[x] = warp_sum(v[x]);
  if (lane == 0)
#pragma unroll
    for (int x = 0; x < NV; ++x) scratch[warp * NV + x] = v[x];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int x = 0; x < NV; ++x) {
      const double s = warp_sum(lane < W ? scratch[lane * NV + x] : 0.0);
      if (lane == 0) parts[blockIdx.x * NV + x] = s;
    }
  }
}

template <int NV>
__device__ __forceinline__ void total(const double *parts, int nparts, double (&out)[NV],
                                      double *slot) {
  if (threadIdx.x < 32) {
    double acc[NV];
#pragma unroll
    for (int x = 0; x < NV; ++x) acc[x] = 0.0;
    for (int b = threadIdx.x; b < nparts; b += 32)
#pragma unroll
      for (int x = 0; x < NV; ++x) acc[x] += __ldcg(parts + b * NV + x);
#pragma unroll
    for (int x = 0; x < NV; ++x) {
      acc[x] = warp_sum(acc[x]);
      if (threadIdx.x == 0) slot[x] = acc[x];
    }
  }
  __syncthreads();
#pragma unroll
  for (int x = 0; x < NV; ++x) out[x] = slot[x];
}

// The reference operator (src/fluid.rs:356-394) in f64 on the pressure, for
// the refinement's residual.
__device__ __forceinline__ double lap_p(const Dims &g, const double *p, int c, int i, int j,
                                        int k) {
  double diag = 0.0, nb = 0.0;
  if (i > 1) { diag += 1.0; nb += __ldcg(p + c - 1); }
  if (i + 2 < g.nx) { diag += 1.0; nb += __ldcg(p + c + 1); }
  if (j > 1) { diag += 1.0; nb += __ldcg(p + c - g.nx); }
  if (j + 2 < g.ny) { diag += 1.0; nb += __ldcg(p + c + g.nx); }
  if (k > 1) { diag += 1.0; nb += __ldcg(p + c - g.nxy); }
  if (k + 2 < g.nz) { diag += 1.0; nb += __ldcg(p + c + g.nxy); }
  return diag * __ldcg(p + c) - nb;
}

// One work item of pass m: `first` (m = 0) forms d = r and q = A d only.
template <bool VEC>
__device__ __forceinline__ void pass_item(const OnePassArgs &o, int item, bool first, float af,
                                          float bf, const float *rin, const float *din,
                                          float *rout, float *dout, float *smem,
                                          double (&acc)[4]) {
  const Dims &g = o.a.g;
  const int tid = threadIdx.x;
  const int tile = item % (o.tiles_x * o.tiles_y);
  const int chunk = item / (o.tiles_x * o.tiles_y);
  const int i0 = (tile % o.tiles_x) * kFx, j0 = (tile / o.tiles_x) * kFy;
  const int k0 = chunk * kOKz;
  const int k1 = min(k0 + kOKz, g.nz);
  const int mi = i0 + (tid & (kFx - 1)), mj = j0 + tid / kFx;
  const bool mine = mi < g.nx && mj < g.ny;
  float *dring = smem;                        // kOS planes of d (tile + 2)
  float *rring = dring + kOS * kODPlane;      // kOS planes of r (tile + 1)
  float *qring = rring + kOS * kORPlane;      // 3 planes of q' = A d_old (tile + 1)
  float *nring = qring + 3 * kOTile1;         // 3 planes of the new d (tile + 1)
  auto slot = [](int p) { return (p + 2 * kOS) % kOS; };
  auto dpl = [&](int p) -> const float * { return dring + slot(p) * kODPlane; };
  auto rpl = [&](int p) -> const float * { return rring + slot(p) * kORPlane; };
  auto qpl = [&](int p) -> float * { return qring + ((p + 3) % 3) * kOTile1; };
  auto npl = [&](int p) -> float * { return nring + ((p + 3) % 3) * kOTile1; };
  auto stage = [&](int p) {
    if (!first) stage_rows<float, VEC>(dring + slot(p) * kODPlane, din, g, i0, j0, 2, p);
    stage_rows<float, VEC>(rring + slot(p) * kORPlane, rin, g, i0, j0, 1, p);
    cp_async_commit();
  };
  // q' = A d_old and the new d at (ci, cj, p) of the tile + ring
  auto ring_cell = [&](int ci, int cj, int p) {
    const int ro = (cj - j0 + 1) * kORW + (ci - i0 + kOXH);
    const int to = (cj - j0 + 1) * kFw + (ci - i0 + 1);
    const float rv = rpl(p)[ro];
    float dn;
    if (first) {
      dn = rv;
    } else {
      float q = 0.0f;
      const int o = (cj - j0 + 2) * kORW + (ci - i0 + kOXH);
      const float *D = dpl(p) + o;
      const float dc = D[0];
      if (interior(g, ci, cj, p)) {
        const int diag = int(ci > 1) + int(ci + 2 < g.nx) + int(cj > 1) + int(cj + 2 < g.ny) +
                         int(p > 1) + int(p + 2 < g.nz);
        float nb = D[-1];
        nb += D[1];
        nb += D[-kORW];
        nb += D[kORW];
        nb += dpl(p - 1)[o];
        nb += dpl(p + 1)[o];
        q = float(diag) * dc - nb;
      }
      qpl(p)[to] = q;
      dn = __fmaf_rn(bf, dc, __fmaf_rn(-af, q, rv));
    }
    npl(p)[to] = dn;
  };
  auto ring_plane = [&](int p) {
    if (p < 0 || p >= g.nz) return;  // never read: the operator stays inside the grid
    if (mine) ring_cell(mi, mj, p);
    if (tid < kFHalo) {
      int hi_, hj;
      halo_cell(tid, i0, j0, hi_, hj);
      if (hi_ >= 0 && hi_ < g.nx && hj >= 0 && hj < g.ny) ring_cell(hi_, hj, p);
    }
  };

  for (int p = k0 - 2; p <= k0 + kOS - 3; ++p) stage(p);
  cp_async_wait<kOS - 4>();  // planes k0-2 .. k0+1
  __syncthreads();
  ring_plane(k0 - 1);
  ring_plane(k0);
  for (int k = k0; k < k1; ++k) {
    cp_async_wait<kOS - 5>();  // plane k+2
    __syncthreads();
    ring_plane(k + 1);
    __syncthreads();
    stage(k + kOS - 2);        // into the slot of plane k-2, last read in iteration k-1
    if (mine) {
      const int to = (mj - j0 + 1) * kFw + (mi - i0 + 1);
      const int c = (k * g.ny + mj) * g.nx + mi;
      const float *N = npl(k) + to;
      const float dn = N[0];
      float q = 0.0f;
      if (interior(g, mi, mj, k)) {
        const int diag = int(mi > 1) + int(mi + 2 < g.nx) + int(mj > 1) + int(mj + 2 < g.ny) +
                         int(k > 1) + int(k + 2 < g.nz);
        float nb = N[-1];
        nb += N[1];
        nb += N[-kFw];
        nb += N[kFw];
        nb += npl(k - 1)[to];
        nb += npl(k + 1)[to];
        q = float(diag) * dn - nb;
      }
      const float rv = rpl(k)[(mj - j0 + 1) * kORW + (mi - i0 + kOXH)];
      const float rnew = first ? rv : __fmaf_rn(-af, qpl(k)[to], rv);
      if (!first) {
        const float dold = dpl(k)[(mj - j0 + 2) * kORW + (mi - i0 + kOXH)];
        o.a.e[c] = __fmaf_rn(af, dold, o.a.e[c]);
      }
      rout[c] = rnew;
      dout[c] = dn;
      acc[0] += double(dn) * double(q);
      acc[1] += double(rnew) * double(q);
      acc[2] += double(q) * double(q);
      acc[3] += double(rnew) * double(rnew);
    }
  }
  cp_async_wait<0>();
  __syncthreads();  // the rings are reused by the next item
}

template <bool VEC>
__global__ void __launch_bounds__(kOT, 3)
    k_cg_onepass_mixed(const __grid_constant__ OnePassArgs o, const __grid_constant__ GridSync gs,
                       double *partials) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float *smem = reinterpret_cast<float *>(smem_raw);
  __shared__ double scratch[(kOT / 32) * 4 + 4];
  double *slot = scratch + (kOT / 32) * 4;
  const MixedCgArgs &a = o.a;
  const Dims g = a.g;
  const int items = o.tiles_x * o.tiles_y * o.chunks;
  const int t0 = blockIdx.x * kOT + threadIdx.x, stride = gridDim.x * kOT;
  double *p = a.p;
  int phase = 0;
  auto parts = [&](int ph) { return partials + (ph & 1) * 4 * gridDim.x; };

  // r = b - A p in f64, rounded once to f32 (into rbuf[1], which pass 0
  // reads); e = 0
  auto outer_residual = [&](bool with_b) {
    double acc[3] = {0.0, 0.0, 0.0};
    for (int c = t0; c < g.n; c += stride) {
      int i, j, k;
      decode(g, c, i, j, k);
      const double ap = interior(g, i, j, k) ? lap_p(g, p, c, i, j, k) : 0.0;
      const double bc = __ldg(a.b + c);
      const double rv = bc - ap;
      const float rf = float(rv);
      o.rbuf[1][c] = rf;
      a.e[c] = 0.0f;
      acc[0] += rv * rv;
      if (with_b) acc[1] += bc * bc;
      acc[2] += double(rf) * double(rf);
    }
    publish<3>(parts(phase), acc, scratch);
  };

  outer_residual(true);
  if (!grid_sync(gs)) return;
  double tot[3];
  total<3>(parts(phase), gridDim.x, tot, slot);
  ++phase;
  const double bb = tot[1];
  double rr = tot[0];
  const double rr0 = rr;
  double tol2 = -1.0;
  if (a.rel_tol > 0.0) {
    const double tl = a.rel_tol * sqrt(bb);
    tol2 = tl * tl;
  }
  int all = 0, passes = 0, converged = 0;
  if (!(rr > 1e-24) || (tol2 >= 0.0 && rr <= tol2)) converged = isfinite(rr) ? 1 : 0;

  while (!converged && passes < a.max_refine && all < a.max_total && isfinite(rr)) {
    double inner_rel = a.inner_rel_tol;
    if (tol2 >= 0.0) inner_rel = fmax(inner_rel, 0.5 * sqrt(tol2 / rr));
    const double inner_tol2 = inner_rel * inner_rel * tot[2];
    double delta = tot[2];
    float af = 0.0f, bf = 0.0f;
    int it = 0;
    for (int m = 0;; ++m) {
      const bool first = m == 0;
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
      const float *rin = o.rbuf[(m + 1) & 1];
      const float *din = o.dbuf[(m + 1) & 1];
      float *rout = o.rbuf[m & 1];
      float *dout = o.dbuf[m & 1];
      for (int item = blockIdx.x; item < items; item += gridDim.x)
        pass_item<VEC>(o, item, first, af, bf, rin, din, rout, dout, smem, acc);
      publish<4>(parts(phase), acc, scratch);
      if (!grid_sync(gs)) return;
      double s4[4];
      total<4>(parts(phase), gridDim.x, s4, slot);
      ++phase;
      if (!first) {  // the tests after update m (the two-pass kernel's order)
        ++it;
        ++all;
        if (!isfinite(s4[3]) || s4[3] <= inner_tol2 || s4[3] < 1e-30) break;
        delta = s4[3];
      }
      if (it >= a.max_inner || all >= a.max_total) break;
      if (!(fabs(s4[0]) >= 1e-30)) break;
      const double alpha = delta / s4[0];
      const double dnext = delta - 2.0 * alpha * s4[1] + alpha * alpha * s4[2];
      af = float(alpha);
      bf = float(dnext / delta);
    }
    // p += e in f64, then the true residual again
    for (int c = t0; c < g.n; c += stride) p[c] = p[c] + double(a.e[c]);
    if (!grid_sync(gs)) return;
    outer_residual(false);
    if (!grid_sync(gs)) return;
    total<3>(parts(phase), gridDim.x, tot, slot);
    ++phase;
    rr = tot[0];
    ++passes;
    if (rr < 1e-20 || (tol2 >= 0.0 && rr <= tol2)) converged = 1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && a.report) {
    SolveReport rep;
    rep.iterations = all;
    rep.refinements = passes;
    rep.converged = converged;
    rep.status = isfinite(rr) ? 0 : 4;
    rep.initial_residual = sqrt(rr0);
    rep.final_residual = sqrt(rr);
    rep.rhs_norm = sqrt(bb);
    *a.report = rep;
  }
}

template <bool VEC>
int blocks_onepass() {
  const size_t smem = sizeof(float) * kOSmemFloats;
  cudaFuncSetAttribute(reinterpret_cast<const void *>(&k_cg_onepass_mixed<VEC>),
                       cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, reinterpret_cast<const void *>(&k_cg_onepass_mixed<VEC>), kOT, smem);
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

}  // namespace

int persistent_blocks_onepass() {
  const int a = blocks_onepass<true>(), b = blocks_onepass<false>();
  return a > b ? a : b;
}

int launch_cg_onepass_mixed(const MixedCgArgs &a, const PersistentState &ps, cudaStream_t st) {
  const bool vec = a.g.nx % Staged<float>::V == 0;
  int blocks = vec ? blocks_onepass<true>() : blocks_onepass<false>();
  if (blocks > ps.max_blocks) blocks = ps.max_blocks;
  OnePassArgs o{};
  o.a = a;
  o.rbuf[0] = a.r;
  o.rbuf[1] = a.q;
  o.dbuf[0] = a.d0;
  o.dbuf[1] = a.d1;
  o.tiles_x = (a.g.nx + kFx - 1) / kFx;
  o.tiles_y = (a.g.ny + kFy - 1) / kFy;
  o.chunks = (a.g.nz + kOKz - 1) / kOKz;
  const int items = o.tiles_x * o.tiles_y * o.chunks;
  if (blocks > items) blocks = items;
  cudaMemsetAsync(ps.count, 0, sizeof(unsigned int), st);
  cudaMemsetAsync(ps.gen, 0, sizeof(unsigned int), st);
  cudaMemsetAsync(ps.abort_flag, 0, sizeof(int), st);
  GridSync gs;
  gs.count = ps.count;
  gs.gen = ps.gen;
  gs.abort_flag = ps.abort_flag;
  gs.nblocks = static_cast<unsigned int>(blocks);
  gs.timeout_ns = ps.timeout_ns;
  double *partials = ps.partials;
  void *params[] = {&o, &gs, &partials};
  const size_t smem = sizeof(float) * kOSmemFloats;
  const void *fn = vec ? reinterpret_cast<const void *>(&k_cg_onepass_mixed<true>)
                       : reinterpret_cast<const void *>(&k_cg_onepass_mixed<false>);
  const cudaError_t err =
      cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(kOT), params, smem, st);
  return err == cudaSuccess ? blocks : -static_cast<int>(err);
}

}  // namespace afl
