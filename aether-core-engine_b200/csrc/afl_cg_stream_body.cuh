// afl_cg_stream_body.cuh -- the streaming CG iteration bodies (FP64 and the
// mixed f32-in-f64-refinement form) shared by the streaming solve kernels
// (afl_poisson_stream.cu) and the persistent ensemble step
// (afl_ensemble_persist.cu).  A body runs as CTA `vblock` of `vgrid` CTAs on
// one system; every grid-level wait is a bounded GridSync barrier.  Included
// only by units built with -fmad=false.
#pragma once

#include "afl_launch.h"

namespace afl {
namespace {


constexpr int kST = 256;  // threads per CTA

template <typename T, int V>
struct alignas(sizeof(T) * V) Vec {
  T v[V];
};

template <typename T, int V>
__device__ __forceinline__ Vec<T, V> ldv(const T *p) {
  return *reinterpret_cast<const Vec<T, V> *>(p);
}
template <typename T, int V>
__device__ __forceinline__ void stv(T *p, const Vec<T, V> &x) {
  *reinterpret_cast<Vec<T, V> *>(p) = x;
}

// A run: V cells starting at x = i0 in row (j, k).
struct Run {
  int i0, j, k, c;
};

template <int V>
__device__ __forceinline__ Run decode_run(const Dims &g, int run) {
  const int rx = g.nx / V;
  const int row = run / rx;
  Run r;
  r.i0 = (run - row * rx) * V;
  r.k = row / g.ny;
  r.j = row - r.k * g.ny;
  r.c = row * g.nx + r.i0;
  return r;
}

// The last of a thread's runs t0, t0 + stride, ... (t0 - stride when it has
// none), where a backward walk starts.
__device__ __forceinline__ int last_run(int t0, int stride, int runs) {
  return t0 < runs ? t0 + ((runs - 1 - t0) / stride) * stride : t0 - stride;
}

// L2 prefetch of run `run`'s V cells of array a, when that run exists: the
// loop over a thread's runs asks for the run kPfAhead steps further along its
// walk, so more HBM requests are in flight without holding registers.  The
// bodies' PF flag turns it on; only the persistent ensemble step uses it
// (48-plume ensemble 593 -> 608-626 Mcell-steps/s).  For one large grid it
// measured slower (256^3: FP64 353 -> 337, mixed 679 -> 671), and the
// graph-form batched solve gained nothing.
constexpr int kPfAhead = 2;
template <int V, typename T>
__device__ __forceinline__ void pf_run(const T *a, int run, int runs) {
  if (run >= 0 && run < runs)
    asm volatile("prefetch.global.L2 [%0];" ::"l"(a + static_cast<size_t>(run) * V));
}

// Direction value at a cell, formed from r and the previous direction with
// the owner's expression (first iteration: d = r).
template <typename T>
struct DirF64 {
  __device__ static T make(bool first, T r, T beta, T d) { return first ? r : r + beta * d; }
};
struct DirF32 {
  __device__ static float make(bool first, float r, float beta, float d) {
    return first ? r : __fmaf_rn(beta, d, r);
  }
};

// q = A dn over one run, dn formed on the fly from (r, dold); also returns the
// run's dn (written by the caller) -- src/fluid.rs:356-394 per cell, with the
// neighbour sum in the reference's order.  The loads may hit in L1: neighbour
// rows of a CTA's runs are loaded by the same CTA.  r and dold were written
// before the grid barrier that precedes this pass, and the barrier's acquire
// and GPU-scope fence order these loads after those writes.
template <typename T, int V, typename Dir>
__device__ __forceinline__ void spmv_run(const Dims &g, const Run &ru, const T *r, const T *dold,
                                         bool first, T beta, Vec<T, V> &dn, Vec<T, V> &q) {
  const Vec<T, V> rc = ldv<T, V>(r + ru.c);
  Vec<T, V> dc;
  if (!first) dc = ldv<T, V>(dold + ru.c);
#pragma unroll
  for (int a = 0; a < V; ++a) dn.v[a] = Dir::make(first, rc.v[a], beta, first ? T(0) : dc.v[a]);
  const bool row_in = ru.j >= 1 && ru.j <= g.ny - 2 && ru.k >= 1 && ru.k <= g.nz - 2;
  if (!row_in) {
#pragma unroll
    for (int a = 0; a < V; ++a) q.v[a] = T(0);
    return;
  }
  auto dn_at = [&](int c) {
    const T rv = r[c];
    return Dir::make(first, rv, beta, first ? T(0) : dold[c]);
  };
  auto dn_vec = [&](int c) {
    Vec<T, V> out;
    const Vec<T, V> rv = ldv<T, V>(r + c);
    if (first) return rv;
    const Vec<T, V> dv = ldv<T, V>(dold + c);
#pragma unroll
    for (int a = 0; a < V; ++a) out.v[a] = Dir::make(false, rv.v[a], beta, dv.v[a]);
    return out;
  };
  const T left = ru.i0 > 0 ? dn_at(ru.c - 1) : T(0);
  const T right = ru.i0 + V < g.nx ? dn_at(ru.c + V) : T(0);
  const Vec<T, V> ym = dn_vec(ru.c - g.nx), yp = dn_vec(ru.c + g.nx);
  const Vec<T, V> zm = dn_vec(ru.c - g.nxy), zp = dn_vec(ru.c + g.nxy);
  const bool yl = ru.j > 1, yh = ru.j + 2 < g.ny, zl = ru.k > 1, zh = ru.k + 2 < g.nz;
#pragma unroll
  for (int a = 0; a < V; ++a) {
    const int i = ru.i0 + a;
    if (i < 1 || i > g.nx - 2) {
      q.v[a] = T(0);
      continue;
    }
    T diag = T(0), nb = T(0);
    if (i > 1) { diag += T(1); nb += a == 0 ? left : dn.v[a - 1]; }
    if (i + 2 < g.nx) { diag += T(1); nb += a == V - 1 ? right : dn.v[a + 1]; }
    if (yl) { diag += T(1); nb += ym.v[a]; }
    if (yh) { diag += T(1); nb += yp.v[a]; }
    if (zl) { diag += T(1); nb += zm.v[a]; }
    if (zh) { diag += T(1); nb += zp.v[a]; }
    q.v[a] = diag * dn.v[a] - nb;
  }
}

// q = A d over one run from the stored direction d, with spmv_run's
// arithmetic and neighbour order, so it reproduces that pass's q bit for bit.
template <typename T, int V>
__device__ __forceinline__ void lap_run(const Dims &g, const Run &ru, const T *d,
                                        const Vec<T, V> &dc, Vec<T, V> &q) {
  const bool row_in = ru.j >= 1 && ru.j <= g.ny - 2 && ru.k >= 1 && ru.k <= g.nz - 2;
  if (!row_in) {
#pragma unroll
    for (int a = 0; a < V; ++a) q.v[a] = T(0);
    return;
  }
  const T left = ru.i0 > 0 ? d[ru.c - 1] : T(0);
  const T right = ru.i0 + V < g.nx ? d[ru.c + V] : T(0);
  const Vec<T, V> ym = ldv<T, V>(d + ru.c - g.nx), yp = ldv<T, V>(d + ru.c + g.nx);
  const Vec<T, V> zm = ldv<T, V>(d + ru.c - g.nxy), zp = ldv<T, V>(d + ru.c + g.nxy);
  const bool yl = ru.j > 1, yh = ru.j + 2 < g.ny, zl = ru.k > 1, zh = ru.k + 2 < g.nz;
#pragma unroll
  for (int a = 0; a < V; ++a) {
    const int i = ru.i0 + a;
    if (i < 1 || i > g.nx - 2) {
      q.v[a] = T(0);
      continue;
    }
    T diag = T(0), nb = T(0);
    if (i > 1) { diag += T(1); nb += a == 0 ? left : dc.v[a - 1]; }
    if (i + 2 < g.nx) { diag += T(1); nb += a == V - 1 ? right : dc.v[a + 1]; }
    if (yl) { diag += T(1); nb += ym.v[a]; }
    if (yh) { diag += T(1); nb += yp.v[a]; }
    if (zl) { diag += T(1); nb += zm.v[a]; }
    if (zh) { diag += T(1); nb += zp.v[a]; }
    q.v[a] = diag * dc.v[a] - nb;
  }
}

// The operator on the f64 pressure (outer residual of the mixed form and the
// FP64 initial residual).
template <int V>
__device__ __forceinline__ void lap_p_run(const Dims &g, const Run &ru, const double *p,
                                          Vec<double, V> &out) {
  const bool row_in = ru.j >= 1 && ru.j <= g.ny - 2 && ru.k >= 1 && ru.k <= g.nz - 2;
#pragma unroll
  for (int a = 0; a < V; ++a) {
    const int i = ru.i0 + a;
    const int c = ru.c + a;
    double v = 0.0;
    if (row_in && i >= 1 && i <= g.nx - 2) {
      double diag = 0.0, nb = 0.0;
      if (i > 1) { diag += 1.0; nb += __ldcg(p + c - 1); }
      if (i + 2 < g.nx) { diag += 1.0; nb += __ldcg(p + c + 1); }
      if (ru.j > 1) { diag += 1.0; nb += __ldcg(p + c - g.nx); }
      if (ru.j + 2 < g.ny) { diag += 1.0; nb += __ldcg(p + c + g.nx); }
      if (ru.k > 1) { diag += 1.0; nb += __ldcg(p + c - g.nxy); }
      if (ru.k + 2 < g.nz) { diag += 1.0; nb += __ldcg(p + c + g.nxy); }
      v = diag * __ldcg(p + c) - nb;
    }
    out.v[a] = v;
  }
}

template <int NV>
__device__ __forceinline__ void cta_publish(double *parts, int vblock, double (&v)[NV],
                                            double *scratch) {
  constexpr int W = kST / 32;
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
      const double x = warp_sum(lane < W ? scratch[lane * NV + a] : 0.0);
      if (lane == 0) parts[vblock * NV + a] = x;
    }
  }
}

template <int NV>
__device__ __forceinline__ void grid_total(const double *parts, int nparts, double (&out)[NV],
                                           double *slot) {
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

struct Ring3 {
  double *base;
  int stride;
  __device__ double *buf(int phase) const { return base + (phase & 1) * stride; }
};

// ------------------------------------------------------------------ FP64 ----
// The solve run by CTA `vblock` of `vgrid` CTAs working on this system (the
// whole launch for a single grid, a slice of it in the batched launch).
// Returns false when a grid barrier gave up (timeout or another CTA's abort):
// every thread of the CTA returns at the same barrier.
//
// SINGLE (one grid larger than L2, the whole launch):
//  - the update pass recomputes q = A d from the stored direction instead of
//    storing q in the matrix-vector pass and reading it back (8 / 4 bytes
//    less per cell written and read);
//  - the matrix-vector pass walks its runs backward and the other passes
//    forward, so each pass starts on the runs the previous one touched last,
//    which are still in L2.
// The batched solves (many small grids side by side) measured slower in this
// form (48-plume ensemble 560 -> 537 Mcell-steps/s) and keep the plain one.
template <int V, bool SINGLE, bool PF = false>
__device__ __forceinline__ bool cg_stream_f64_body(const CgArgs &a, const GridSync &gs,
                                                   const Ring3 &pr, int vblock, int vgrid,
                                                   double *scratch) {
  double *slot = scratch + (kST / 32) * 2;
  const Dims g = a.g;
  const int runs = g.n / V;
  const int t0 = vblock * kST + threadIdx.x, stride = vgrid * kST;
  double *p = a.p, *r = a.r, *q = a.q;
  const double *b = a.b;
  int phase = 0;
  {
    double acc[2] = {0.0, 0.0};
    for (int run = t0; run < runs; run += stride) {
      const Run ru = decode_run<V>(g, run);
      Vec<double, V> ap;
      lap_p_run<V>(g, ru, p, ap);
      const Vec<double, V> bv = ldv<double, V>(b + ru.c);
      Vec<double, V> rv;
#pragma unroll
      for (int e = 0; e < V; ++e) {
        rv.v[e] = bv.v[e] - ap.v[e];
        acc[0] += rv.v[e] * rv.v[e];
        acc[1] += bv.v[e] * bv.v[e];
      }
      stv<double, V>(r + ru.c, rv);
    }
    cta_publish<2>(pr.buf(phase), vblock, acc, scratch);
  }
  if (!grid_sync(gs)) return false;
  double tot[2];
  grid_total<2>(pr.buf(phase), vgrid, tot, slot);
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
    double *dold = a.d0, *dnew = a.d1;
    while (it < a.max_iters) {
      const bool first = it == 0;
      double acc[1] = {0.0};
      for (int run = SINGLE ? last_run(t0, stride, runs) : t0;
           SINGLE ? run >= t0 : run < runs; run += SINGLE ? -stride : stride) {
        const Run ru = decode_run<V>(g, run);
        if (PF) {
          const int ahead = run + kPfAhead * stride;
          pf_run<V>(r, ahead, runs);
          if (!first) pf_run<V>(dold, ahead, runs);
        }
        Vec<double, V> dn, qv;
        spmv_run<double, V, DirF64<double>>(g, ru, r, dold, first, beta, dn, qv);
        stv<double, V>(dnew + ru.c, dn);
        if (!SINGLE) stv<double, V>(q + ru.c, qv);
#pragma unroll
        for (int e = 0; e < V; ++e) acc[0] += dn.v[e] * qv.v[e];
      }
      cta_publish<1>(pr.buf(phase), vblock, acc, scratch);
      if (!grid_sync(gs)) return false;
      double dq[1];
      grid_total<1>(pr.buf(phase), vgrid, dq, slot);
      ++phase;
      if (fabs(dq[0]) < 1e-28) break;  // src/fluid.rs:469
      const double alpha = delta / dq[0];
      double acc2[1] = {0.0};
      for (int run = t0; run < runs; run += stride) {
        const Run ru = decode_run<V>(g, run);
        const int c = ru.c;
        if (PF) {
          const int ahead = run + kPfAhead * stride;
          pf_run<V>(p, ahead, runs);
          pf_run<V>(dnew, ahead, runs);
          pf_run<V>(r, ahead, runs);
          pf_run<V>(q, ahead, runs);
        }
        Vec<double, V> pv = ldv<double, V>(p + c);
        const Vec<double, V> dv = ldv<double, V>(dnew + c);
        Vec<double, V> qv;
        if (!SINGLE) qv = ldv<double, V>(q + c);
        else lap_run<double, V>(g, ru, dnew, dv, qv);
        Vec<double, V> rv = ldv<double, V>(r + c);
#pragma unroll
        for (int e = 0; e < V; ++e) {
          pv.v[e] = pv.v[e] + alpha * dv.v[e];
          rv.v[e] = rv.v[e] - alpha * qv.v[e];
          acc2[0] += rv.v[e] * rv.v[e];
        }
        stv<double, V>(p + c, pv);
        stv<double, V>(r + c, rv);
      }
      cta_publish<1>(pr.buf(phase), vblock, acc2, scratch);
      if (!grid_sync(gs)) return false;
      double dn[1];
      grid_total<1>(pr.buf(phase), vgrid, dn, slot);
      ++phase;
      ++it;
      last = dn[0];
      if (!isfinite(dn[0])) break;
      if (dn[0] < 1e-20) { converged = 1; break; }  // src/fluid.rs:479
      if (tol2 >= 0.0 && dn[0] <= tol2) { converged = 1; break; }
      beta = dn[0] / delta;  // src/fluid.rs:482
      delta = dn[0];
      double *t = dold;
      dold = dnew;
      dnew = t;
    }
  }
  if (vblock == 0 && threadIdx.x == 0 && a.report) {
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
  return true;
}

// ----------------------------------------------------------------- mixed ----
// f32 CG on the correction e inside f64 iterative refinement; SINGLE as for
// the FP64 body.
template <int V, bool SINGLE, bool PF = false>
__device__ __forceinline__ bool cg_stream_mixed_body(const MixedCgArgs &a, const GridSync &gs,
                                                     const Ring3 &pr, int vblock, int vgrid,
                                                     double *scratch) {
  double *slot = scratch + (kST / 32) * 3;
  const Dims g = a.g;
  const int runs = g.n / V;
  const int t0 = vblock * kST + threadIdx.x, stride = vgrid * kST;
  double *p = a.p;
  const double *b = a.b;
  float *r = a.r, *e = a.e, *q = a.q;
  int phase = 0;

  auto outer_residual = [&](bool with_b) {
    double acc[3] = {0.0, 0.0, 0.0};
    for (int run = t0; run < runs; run += stride) {
      const Run ru = decode_run<V>(g, run);
      Vec<double, V> ap;
      lap_p_run<V>(g, ru, p, ap);
      const Vec<double, V> bv = ldv<double, V>(b + ru.c);
      Vec<float, V> rf, zero;
#pragma unroll
      for (int x = 0; x < V; ++x) {
        const double rv = bv.v[x] - ap.v[x];
        rf.v[x] = float(rv);
        zero.v[x] = 0.0f;
        acc[0] += rv * rv;
        if (with_b) acc[1] += bv.v[x] * bv.v[x];
        acc[2] += double(rf.v[x]) * double(rf.v[x]);
      }
      stv<float, V>(r + ru.c, rf);
      stv<float, V>(e + ru.c, zero);
    }
    cta_publish<3>(pr.buf(phase), vblock, acc, scratch);
  };

  outer_residual(true);
  if (!grid_sync(gs)) return false;
  double tot[3];
  grid_total<3>(pr.buf(phase), vgrid, tot, slot);
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

  while (!converged && passes < a.max_refine && total < a.max_total && isfinite(rr)) {
    double inner_rel = a.inner_rel_tol;
    if (tol2 >= 0.0) inner_rel = fmax(inner_rel, 0.5 * sqrt(tol2 / rr));
    double delta = tot[2];
    const double inner_tol2 = inner_rel * inner_rel * delta;
    double beta = 0.0;
    float *dold = a.d0, *dnew = a.d1;
    int it = 0;
    while (it < a.max_inner && total < a.max_total) {
      const bool first = it == 0;
      const float bf = float(beta);
      double acc[1] = {0.0};
      for (int run = SINGLE ? last_run(t0, stride, runs) : t0;
           SINGLE ? run >= t0 : run < runs; run += SINGLE ? -stride : stride) {
        const Run ru = decode_run<V>(g, run);
        if (PF) {
          const int ahead = run + kPfAhead * stride;
          pf_run<V>(r, ahead, runs);
          if (!first) pf_run<V>(dold, ahead, runs);
        }
        Vec<float, V> dn, qv;
        spmv_run<float, V, DirF32>(g, ru, r, dold, first, bf, dn, qv);
        stv<float, V>(dnew + ru.c, dn);
        if (!SINGLE) stv<float, V>(q + ru.c, qv);
        {  // the run's products summed in f32, the runs in f64 (256^3: 706 -> 722)
          float part = 0.0f;
#pragma unroll
          for (int x = 0; x < V; ++x) part = __fmaf_rn(dn.v[x], qv.v[x], part);
          acc[0] += double(part);
        }
      }
      cta_publish<1>(pr.buf(phase), vblock, acc, scratch);
      if (!grid_sync(gs)) return false;
      double dq[1];
      grid_total<1>(pr.buf(phase), vgrid, dq, slot);
      ++phase;
      if (!(fabs(dq[0]) >= 1e-30)) break;
      const float af = float(delta / dq[0]);
      double acc2[1] = {0.0};
      for (int run = t0; run < runs; run += stride) {
        const Run ru = decode_run<V>(g, run);
        const int c = ru.c;
        if (PF) {
          const int ahead = run + kPfAhead * stride;
          pf_run<V>(e, ahead, runs);
          pf_run<V>(dnew, ahead, runs);
          pf_run<V>(r, ahead, runs);
          pf_run<V>(q, ahead, runs);
        }
        Vec<float, V> ev = ldv<float, V>(e + c);
        const Vec<float, V> dv = ldv<float, V>(dnew + c);
        Vec<float, V> qv;
        if (!SINGLE) qv = ldv<float, V>(q + c);
        else lap_run<float, V>(g, ru, dnew, dv, qv);
        Vec<float, V> rv = ldv<float, V>(r + c);
        float part = 0.0f;
#pragma unroll
        for (int x = 0; x < V; ++x) {
          ev.v[x] = __fmaf_rn(af, dv.v[x], ev.v[x]);
          rv.v[x] = __fmaf_rn(-af, qv.v[x], rv.v[x]);
          part = __fmaf_rn(rv.v[x], rv.v[x], part);
        }
        acc2[0] += double(part);
        stv<float, V>(e + c, ev);
        stv<float, V>(r + c, rv);
      }
      cta_publish<1>(pr.buf(phase), vblock, acc2, scratch);
      if (!grid_sync(gs)) return false;
      double dn[1];
      grid_total<1>(pr.buf(phase), vgrid, dn, slot);
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
    // p += e (f64), then the true residual again
    for (int run = SINGLE ? last_run(t0, stride, runs) : t0;
         SINGLE ? run >= t0 : run < runs; run += SINGLE ? -stride : stride) {
      const int c = decode_run<V>(g, run).c;
      Vec<double, V> pv = ldv<double, V>(p + c);
      const Vec<float, V> ev = ldv<float, V>(e + c);
#pragma unroll
      for (int x = 0; x < V; ++x) pv.v[x] = pv.v[x] + double(ev.v[x]);
      stv<double, V>(p + c, pv);
    }
    if (!grid_sync(gs)) return false;
    outer_residual(false);
    if (!grid_sync(gs)) return false;
    grid_total<3>(pr.buf(phase), vgrid, tot, slot);
    ++phase;
    rr = tot[0];
    ++passes;
    if (rr < 1e-20 || (tol2 >= 0.0 && rr <= tol2)) converged = 1;
  }
  if (vblock == 0 && threadIdx.x == 0 && a.report) {
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
  return true;
}

}  // namespace
}  // namespace afl
