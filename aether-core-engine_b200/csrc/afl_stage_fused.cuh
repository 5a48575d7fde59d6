// afl_stage_fused.cuh -- the shared-memory-staged stage kernels, templated
// on the field type T (double: FP64 form; float: mixed form).  Included by
// afl_kernels_f64.cu (built with -fmad=false) and afl_kernels_f32.cu.
//
// Launch shape: one CTA of 256 threads owns a 32 x 8 tile of the x-y plane
// (one thread per cell) and marches up a chunk of z planes.  Every plane it
// reads is copied into a ring of S shared-memory slots with asynchronous
// copies (cp.async; 16-byte copies along x when the rows are 16-byte
// aligned), S-4 planes ahead of the plane being computed, so the HBM stream
// stays in flight while the stencil runs on the staged copies.  The staged
// rows reach 16 bytes past the tile on each side in x and two cells in y;
// cells outside the grid read as 0.
//
// k_maccormack_fused: advect_maccormack_in_place (src/fluid.rs:170-234) in
// one pass.  The forward semi-Lagrangian field `fwd` (:183) is computed on the
// tile plus a one-cell halo into a ring of three shared planes; the backward
// sample `bwd` (:184) reads that ring, and the clamp's 8-cell min/max
// (:196-209) comes from the same staged corners as the cell's own `fwd`.  A
// footprint that leaves the staged region (a backtrace longer than about one
// cell) is evaluated from global memory with the same arithmetic.  The solver
// uses it for the end of a step: density and temperature advected in one
// launch that reads the velocity once, with the telemetry sums of the final
// state (compute_telemetry, :613-672) accumulated in the same pass.
//
// k_forces_fused: apply_buoyancy_and_vorticity_confinement
// (src/fluid.rs:256-330).  The curl and |w| of the tile plus a one-cell halo
// exist only in shared memory and registers; the new velocities go to a
// second set of arrays, because neighbouring CTAs still read the old ones.
// Each cell's arithmetic is the expression of the per-cell kernels of
// afl_stage.cuh, so the FP64 results are the same bits as theirs.
#pragma once

#include "afl_stage.cuh"

namespace afl {

constexpr int kFx = 32, kFy = 8, kFThreads = kFx * kFy;
constexpr int kFHalo = 2 * (kFx + 2) + 2 * kFy;  // cells of the one-cell ring: 84
constexpr int kFw = kFx + 2, kFh = kFy + 2;      // tile plus a one-cell halo

template <typename T>
struct Staged {
  static constexpr int V = 16 / int(sizeof(T));  // elements of one 16-byte copy
  static constexpr int XH = V;                   // x halo: rows stay 16-byte aligned
  static constexpr int RW = kFx + 2 * XH;        // staged row width
};

__device__ __forceinline__ void cp_async16(void *s, const void *gsrc, bool ok) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(s));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gsrc),
               "r"(ok ? 16 : 0)
               : "memory");
}
template <int B>
__device__ __forceinline__ void cp_async_small(void *s, const void *gsrc, bool ok) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(s));
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(sa), "l"(gsrc), "n"(B),
               "r"(ok ? B : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// One thread's part of staging a (kFy + 2*yh) x RW block of a plane: up to
// two copies (RW / V chunks per row), their shared-memory offsets and their
// offsets inside a plane, worked out once per CTA; per plane only the plane
// offset and the plane's bounds change.
template <typename T, bool VEC>
struct StageDesc {
  static constexpr int V = VEC ? Staged<T>::V : 1;
  int soff[2], goff[2];
  bool ok[2];
  int n;
  __device__ __forceinline__ StageDesc(const Dims &g, int i0, int j0, int yh) {
    constexpr int RW = Staged<T>::RW, XH = Staged<T>::XH, CPR = RW / V;
    const int total = (kFy + 2 * yh) * CPR;
    n = 0;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int t = threadIdx.x + q * kFThreads;
      soff[q] = 0;
      goff[q] = 0;
      ok[q] = false;
      if (t < total) {
        const int r = t / CPR;
        const int m = t - r * CPR;
        const int j = j0 - yh + r, i = i0 - XH + m * V;
        soff[q] = r * RW + m * V;
        ok[q] = j >= 0 && j < g.ny && i >= 0 && i < g.nx;
        goff[q] = ok[q] ? j * g.nx + i : 0;
        n = q + 1;
      }
    }
  }
  // Copies plane p of src into dst (cells outside the grid read 0).
  __device__ __forceinline__ void copy(T *dst, const T *__restrict__ src, const Dims &g,
                                       int p) const {
    const bool pin = p >= 0 && p < g.nz;
    const T *plane = src + (pin ? p * g.nxy : 0);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      if (q >= n) break;
      const bool okq = pin && ok[q];
      if constexpr (VEC) cp_async16(dst + soff[q], okq ? plane + goff[q] : src, okq);
      else cp_async_small<int(sizeof(T))>(dst + soff[q], okq ? plane + goff[q] : src, okq);
    }
  }
};

// Clamp bounds of sample_trilinear (src/fluid.rs:95-97) per axis, n - 1.500001,
// computed once per CTA with the expression footprint3 uses.
template <typename T>
struct FpBounds {
  T hx, hy, hz;
  __device__ __forceinline__ explicit FpBounds(const Dims &g)
      : hx(T(g.nx) - T(1.500001)), hy(T(g.ny) - T(1.500001)), hz(T(g.nz) - T(1.500001)) {}
};

// footprint3_at with the bounds precomputed: the same operations, so the same
// corner and weights bit for bit.
__device__ __forceinline__ void fp_axis(int i, double hi, double d, int &i0, double &t) {
  const double xc = rs_clamp(double(i) - d, 0.5, hi);
  i0 = floor_index(xc);
  t = xc - double(i0);
}
__device__ __forceinline__ void fp_axis(int i, float hi, float d, int &i0, float &t) {
  const float p = float(i) - d;
  if (!(p == p)) {  // NaN displacement: cell 0, as floor_index
    i0 = 0;
    t = p;
  } else if (p < 0.5f) {
    i0 = 0;
    t = 0.5f;
  } else if (p > hi) {
    const float f = floorf(hi);
    i0 = static_cast<int>(f);
    t = hi - f;
  } else {
    const float f = floorf(-d);
    i0 = i + static_cast<int>(f);
    t = -d - f;
  }
}
template <typename T>
__device__ __forceinline__ Footprint3<T> fp_at(const FpBounds<T> &b, int i, int j, int k, T dx,
                                               T dy, T dz) {
  Footprint3<T> f;
  fp_axis(i, b.hx, dx, f.i, f.tx);
  fp_axis(j, b.hy, dy, f.j, f.ty);
  fp_axis(k, b.hz, dz, f.k, f.tz);
  return f;
}

// Cell t of the one-cell ring around the tile at (i0, j0).
__device__ __forceinline__ void halo_cell(int t, int i0, int j0, int &i, int &j) {
  if (t < kFw) {
    i = i0 - 1 + t;
    j = j0 - 1;
  } else if (t < 2 * kFw) {
    i = i0 - 1 + (t - kFw);
    j = j0 + kFy;
  } else if (t < 2 * kFw + kFy) {
    i = i0 - 1;
    j = j0 + (t - 2 * kFw);
  } else {
    i = i0 + kFx;
    j = j0 + (t - 2 * kFw - kFy);
  }
}

// ---- MacCormack advection ----------------------------------------------------
template <typename T>
struct McArgs {
  Dims g;
  const T *u, *v, *w;  // velocity (not written by the launch)
  const T *src[2];     // advected fields
  T *out[2];           // their new values (distinct arrays)
  T scale_f, scale_b;  // dt/h and -dt/h
  T diss[2];           // dissipation per field
  int nonneg;          // density/temperature: max(0, .)
  int vel_src;         // the advected field is velocity component vel_src (NF = 1)
  int kz;              // z planes per CTA
  double *tel;         // telemetry partials, 7 per CTA (TEL only)
  double dv, inv_2h;   // telemetry: cell volume h^3 and 1/(2h)
};

template <typename T, int NF, bool SRC_IS_VEL>
struct McLayout {
  static constexpr int RW = Staged<T>::RW;
  static constexpr int VYH = SRC_IS_VEL ? 2 : 1;       // y halo of the velocity rows
  static constexpr int VROWS = kFy + 2 * VYH;
  static constexpr int SROWS = kFy + 4;                // advected fields: y halo 2
  static constexpr int VPL = 3 * VROWS * RW;           // one staged velocity plane
  static constexpr int SPL = SRC_IS_VEL ? 0 : NF * SROWS * RW;
  static constexpr int FPL = NF * kFh * kFw;           // one fwd plane
  static constexpr int elems(int S) { return S * (VPL + SPL) + 3 * FPL; }
};

// One launch advects NF fields of the same velocity.  SRC_IS_VEL: the field
// is a velocity component, read from the staged velocity (kept for
// single-field use; the solver advects velocity with the fwd + mc pair of
// afl_stage.cuh, which measured faster).  TEL (NF = 2, field 0 = density):
// the telemetry sums over this CTA's cells go to a.tel[7 * cta] as
// k_telemetry's partials.
// Ring slots are tracked as plane offsets that advance by one slot per
// iteration (no division); the plane pointers of an iteration are set once.
template <typename T, int NF, bool SRC_IS_VEL, bool TEL, int S, bool VEC>
__global__ void __launch_bounds__(kFThreads, NF == 1 ? 3 : 2)
    k_maccormack_fused(const __grid_constant__ McArgs<T> a) {
  static_assert(S >= 5, "the ring holds planes k-2 .. k+2 plus at least one ahead");
  using L = McLayout<T, NF, SRC_IS_VEL>;
  constexpr int RW = L::RW, XH = Staged<T>::XH, VYH = L::VYH, VROWS = L::VROWS;
  constexpr int SROWS = L::SROWS, VPL = L::VPL, SPL = L::SPL, FPL = L::FPL;
  constexpr int PL = VPL + SPL;  // one ring slot: the velocity, then the fields
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *ring = reinterpret_cast<T *>(smem_raw);
  T *fring = ring + S * PL;
  const Dims &g = a.g;
  const int tid = threadIdx.x;
  const int i0 = blockIdx.x * kFx, j0 = blockIdx.y * kFy;
  const int k0 = blockIdx.z * a.kz;
  const int k1 = min(k0 + a.kz, g.nz);
  const int mi = i0 + (tid & (kFx - 1)), mj = j0 + tid / kFx;
  const bool mine = mi < g.nx && mj < g.ny;
  const FpBounds<T> fb_bounds(g);
  const T wxl = T(1.5), wxh = T(g.nx) - T(2.5), wyh = T(g.ny) - T(2.5), wzh = T(g.nz) - T(2.5);
  // field f of a slot starts SROWS*RW apart (velocity component vel_src when
  // the field is a velocity component); rows start at y = j0 - 2
  const int foff = SRC_IS_VEL ? a.vel_src * VROWS * RW : VPL;
  constexpr int FSTRIDE = SROWS * RW;

  const StageDesc<T, VEC> dvel(g, i0, j0, VYH);
  const StageDesc<T, VEC> dsrc(g, i0, j0, 2);
  auto stage = [&](T *slotp, int p) {
    dvel.copy(slotp, a.u, g, p);
    dvel.copy(slotp + VROWS * RW, a.v, g, p);
    dvel.copy(slotp + 2 * VROWS * RW, a.w, g, p);
    if constexpr (!SRC_IS_VEL) {
#pragma unroll
      for (int f = 0; f < NF; ++f) dsrc.copy(slotp + VPL + f * FSTRIDE, a.src[f], g, p);
    }
    cp_async_commit();
  };
  auto next_slot = [&](T *sp) { return sp + PL == ring + S * PL ? ring : sp + PL; };

  // fwd = SL(src, dt) at cell (ci, cj) of plane p (advect_semi_lagrangian,
  // src/fluid.rs:153-167) into fo of the fwd plane F.  vp: the staged plane
  // p; vm, vq: planes p-1 and p+1 (for the field corners).  For the thread's
  // own cell (own), also the min/max of the same 8 corners (stencil_minmax,
  // :131-150), the bounds of its clamp.
  auto fwd_cell = [&](int ci, int cj, int p, const T *vm, const T *vp, const T *vq, T *F,
                      bool own, T (&lo)[NF], T (&hi)[NF]) {
    T res[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) res[f] = T(0);
    if (interior(g, ci, cj, p)) {
      const int vo = (cj - j0 + VYH) * RW + (ci - i0 + XH);
      const T uc = vp[vo], vc = vp[VROWS * RW + vo], wc = vp[2 * VROWS * RW + vo];
      const Footprint3<T> fp =
          fp_at(fb_bounds, ci, cj, p, a.scale_f * uc, a.scale_f * vc, a.scale_f * wc);
      const bool staged = fp.i >= i0 - XH && fp.i + 1 < i0 + kFx + XH && fp.j >= j0 - 2 &&
                          fp.j + 1 < j0 + kFy + 2 && fp.k >= p - 1 && fp.k <= p;
      const int o = (fp.j - j0 + 2) * RW + (fp.i - i0 + XH) + foff;
      const T *z0 = (fp.k == p - 1 ? vm : vp) + o;
      const T *z1 = (fp.k == p - 1 ? vp : vq) + o;
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        T c[8];
        if (staged) {
          const T *s0 = z0 + f * FSTRIDE, *s1 = z1 + f * FSTRIDE;
          c[0] = s0[0]; c[1] = s0[1]; c[2] = s0[RW]; c[3] = s0[RW + 1];
          c[4] = s1[0]; c[5] = s1[1]; c[6] = s1[RW]; c[7] = s1[RW + 1];
        } else {
          const T *sg = a.src[f] + fp.base(g);
          c[0] = __ldg(sg); c[1] = __ldg(sg + 1); c[2] = __ldg(sg + g.nx);
          c[3] = __ldg(sg + g.nx + 1); c[4] = __ldg(sg + g.nxy); c[5] = __ldg(sg + g.nxy + 1);
          c[6] = __ldg(sg + g.nxy + g.nx); c[7] = __ldg(sg + g.nxy + g.nx + 1);
        }
        res[f] = lerp8(c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], fp.tx, fp.ty, fp.tz);
        if (own) {
          T l = T(INFINITY), h = T(-INFINITY);
#pragma unroll
          for (int q = 0; q < 8; ++q) {  // minmax8's corner order
            l = fmin(l, c[q]);
            h = fmax(h, c[q]);
          }
          lo[f] = l;
          hi[f] = h;
        }
      }
    }
    const int fo = (cj - j0 + 1) * kFw + (ci - i0 + 1);
#pragma unroll
    for (int f = 0; f < NF; ++f) F[f * kFh * kFw + fo] = res[f];
  };

  // This thread's ring cell (threads below kFHalo), found once.
  int hi_i = 0, hi_j = 0;
  if (tid < kFHalo) halo_cell(tid, i0, j0, hi_i, hi_j);
  // fwd of plane p on the tile and its one-cell ring (planes outside the grid
  // are never sampled: every footprint lies inside it).
  auto fwd_plane = [&](int p, const T *vm, const T *vp, const T *vq, T *F, T (&lo)[NF],
                       T (&hi)[NF]) {
    if (p < 0 || p >= g.nz) return;
    if (mine) fwd_cell(mi, mj, p, vm, vp, vq, F, true, lo, hi);
    if (tid < kFHalo) {
      T dl[NF], dh[NF];
      fwd_cell(hi_i, hi_j, p, vm, vp, vq, F, false, dl, dh);
    }
  };

  // fwd at one cell from global memory: the fallback of a long backtrace.
  auto fwd_global = [&](int f, int qi, int qj, int qk) -> T {
    if (!interior(g, qi, qj, qk)) return T(0);
    const int q = (qk * g.ny + qj) * g.nx + qi;
    const T uq = __ldg(a.u + q), vq = __ldg(a.v + q), wq = __ldg(a.w + q);
    return trilinear(a.src[f], g,
                     footprint_at(g, qi, qj, qk, a.scale_f * uq, a.scale_f * vq, a.scale_f * wq));
  };

  T lo_cur[NF], hi_cur[NF], lo_nxt[NF], hi_nxt[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) lo_cur[f] = hi_cur[f] = lo_nxt[f] = hi_nxt[f] = T(0);
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  double peak = 0.0;

  // slot of plane k0-2 is ring[0]; plane k0-2+t sits in slot t mod S
  {
    T *sp = ring;
    for (int p = k0 - 2; p <= k0 + S - 3; ++p) {
      stage(sp, p);
      sp += PL;
    }
  }
  T *sm2 = ring;                 // plane k-2 (k = k0)
  T *sm1 = ring + PL;            // k-1
  T *s0 = ring + 2 * PL;         // k
  T *s1 = ring + 3 * PL;         // k+1
  T *s2 = ring + 4 * PL;         // k+2
  T *F0 = fring, *F1 = fring + FPL, *F2 = fring + 2 * FPL;  // fwd of planes k-1, k, k+1
  cp_async_wait<S - 4>();  // planes k0-2 .. k0+1 have landed
  __syncthreads();
  fwd_plane(k0 - 1, sm2, sm1, s0, F0, lo_nxt, hi_nxt);  // ring plane only
  fwd_plane(k0, sm1, s0, s1, F1, lo_cur, hi_cur);

  for (int k = k0; k < k1; ++k) {
    cp_async_wait<S - 5>();  // plane k+2 has landed
    __syncthreads();         // ... for every thread; iteration k-1 is done with its planes
    fwd_plane(k + 1, s0, s1, s2, F2, lo_nxt, hi_nxt);
    __syncthreads();         // fwd of plane k+1 is visible
    {
      // plane k+S-2 goes into the slot of plane k-2, last read in iteration k-1
      T *sp = sm2;
      stage(sp, k + S - 2);
    }
    if (mine) {
      T res[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) res[f] = T(0);
      const int vo = (mj - j0 + VYH) * RW + (mi - i0 + XH);
      const bool inner = interior(g, mi, mj, k);
      if (inner) {
        const T uc = s0[vo], vc = s0[VROWS * RW + vo], wc = s0[2 * VROWS * RW + vo];
        const T bx = T(mi) - a.scale_f * uc;
        const T by = T(mj) - a.scale_f * vc;
        const T bz = T(k) - a.scale_f * wc;
        const bool near_wall = bx < wxl || bx > wxh || by < wxl || by > wyh || bz < wxl ||
                               bz > wzh;
        const int fo = (mj - j0 + 1) * kFw + (mi - i0 + 1);
        if (near_wall) {
#pragma unroll
          for (int f = 0; f < NF; ++f) res[f] = F1[f * kFh * kFw + fo] * a.diss[f];
        } else {
          const Footprint3<T> fb =
              fp_at(fb_bounds, mi, mj, k, a.scale_b * uc, a.scale_b * vc, a.scale_b * wc);
          const bool staged = fb.i >= i0 - 1 && fb.i + 1 <= i0 + kFx && fb.j >= j0 - 1 &&
                              fb.j + 1 <= j0 + kFy && fb.k >= k - 1 && fb.k <= k;
          const int o = (fb.j - j0 + 1) * kFw + (fb.i - i0 + 1);
          const T *z0 = (fb.k == k - 1 ? F0 : F1) + o;
          const T *z1 = (fb.k == k - 1 ? F1 : F2) + o;
          const int so = (mj - j0 + 2) * RW + (mi - i0 + XH) + foff;
#pragma unroll
          for (int f = 0; f < NF; ++f) {
            T bwd;
            if (staged) {
              const T *f0 = z0 + f * kFh * kFw, *f1 = z1 + f * kFh * kFw;
              bwd = lerp8(f0[0], f0[1], f0[kFw], f0[kFw + 1], f1[0], f1[1], f1[kFw],
                          f1[kFw + 1], fb.tx, fb.ty, fb.tz);
            } else {
              bwd = lerp8(fwd_global(f, fb.i, fb.j, fb.k), fwd_global(f, fb.i + 1, fb.j, fb.k),
                          fwd_global(f, fb.i, fb.j + 1, fb.k),
                          fwd_global(f, fb.i + 1, fb.j + 1, fb.k),
                          fwd_global(f, fb.i, fb.j, fb.k + 1),
                          fwd_global(f, fb.i + 1, fb.j, fb.k + 1),
                          fwd_global(f, fb.i, fb.j + 1, fb.k + 1),
                          fwd_global(f, fb.i + 1, fb.j + 1, fb.k + 1), fb.tx, fb.ty, fb.tz);
            }
            const T fc = F1[f * kFh * kFw + fo];
            const T mc = fc + T(0.5) * (s0[so + f * FSTRIDE] - bwd);
            res[f] = rs_clamp(mc, lo_cur[f], hi_cur[f]) * a.diss[f];
          }
        }
      }
      const int c = (k * g.ny + mj) * g.nx + mi;
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        if (a.nonneg) res[f] = fmax(res[f], T(0));
        a.out[f][c] = res[f];
      }
      if constexpr (TEL) {
        if (inner) {  // compute_telemetry (src/fluid.rs:613-672) at this cell
          const T *U = s0, *Vv = s0 + VROWS * RW, *W = s0 + 2 * VROWS * RW;
          const double uc = U[vo], vc = Vv[vo], wc = W[vo];
          const double u2 = uc * uc + vc * vc + wc * wc;
          acc[0] += 0.5 * u2 * a.dv;
          const double dw_dy = (double(W[vo + RW]) - double(W[vo - RW])) * a.inv_2h;
          const double dv_dz =
              (double(s1[VROWS * RW + vo]) - double(sm1[VROWS * RW + vo])) * a.inv_2h;
          const double du_dz = (double(s1[vo]) - double(sm1[vo])) * a.inv_2h;
          const double dw_dx = (double(W[vo + 1]) - double(W[vo - 1])) * a.inv_2h;
          const double dv_dx = (double(Vv[vo + 1]) - double(Vv[vo - 1])) * a.inv_2h;
          const double du_dy = (double(U[vo + RW]) - double(U[vo - RW])) * a.inv_2h;
          const double ox = dw_dy - dv_dz;
          const double oy = du_dz - dw_dx;
          const double oz = dv_dx - du_dy;
          const double w2 = ox * ox + oy * oy + oz * oz;
          acc[1] += 0.5 * w2 * a.dv;
          peak = fmax(peak, sqrt(w2));
          const double r = double(res[0]);
          if (r > 1e-8) {
            acc[2] += r * a.dv;
            const double nxn = 2.0 * (double(mi) / double(g.nx - 1)) - 1.0;
            const double nyn = 2.0 * (double(mj) / double(g.ny - 1)) - 1.0;
            const double nzn = 2.0 * (double(k) / double(g.nz - 1)) - 1.0;
            const double wgt = r * a.dv;
            acc[3] += nxn * wgt;
            acc[4] += nyn * wgt;
            acc[5] += nzn * wgt;
          }
        }
      }
    }
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      lo_cur[f] = lo_nxt[f];
      hi_cur[f] = hi_nxt[f];
    }
    // advance the ring by one plane
    T *old = sm2;
    sm2 = sm1;
    sm1 = s0;
    s0 = s1;
    s1 = s2;
    s2 = next_slot(s2);
    (void)old;
    T *ft = F0;
    F0 = F1;
    F1 = F2;
    F2 = ft;
  }
  cp_async_wait<0>();  // no copy outlives the CTA
  if constexpr (TEL) {
    __shared__ double scratch[kWarps * 6];
    block_sum<6>(acc, scratch);
    const double pk = block_max(peak, scratch);
    if (tid == 0) {
      const int cta = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
#pragma unroll
      for (int q = 0; q < 6; ++q) a.tel[cta * 7 + q] = acc[q];
      a.tel[cta * 7 + 6] = pk;
    }
  }
}

// ---- vorticity confinement + buoyancy -----------------------------------------
template <typename T>
struct ForcesArgs {
  Dims g;
  const T *u, *v, *w, *rho, *temp;
  T *uo, *vo, *wo;  // new velocity (distinct from u, v, w)
  T dt, eps_h, inv_2h, beta, alpha;
  int kz;
};

template <typename T>
struct ForcesLayout {
  static constexpr int RW = Staged<T>::RW;
  static constexpr int VROWS = kFy + 4;       // y halo 2: the curl of the one-cell ring
  static constexpr int VPL = 3 * VROWS * RW;
  static constexpr int MPL = kFh * kFw;       // one |w| plane
  static constexpr int elems(int S) { return S * VPL + 3 * MPL; }
};

template <typename T, int S, bool VEC>
__global__ void __launch_bounds__(kFThreads, 3)
    k_forces_fused(const __grid_constant__ ForcesArgs<T> a) {
  static_assert(S >= 5, "the ring holds planes k-2 .. k+2 plus at least one ahead");
  using L = ForcesLayout<T>;
  constexpr int RW = L::RW, XH = Staged<T>::XH, VROWS = L::VROWS, VPL = L::VPL, MPL = L::MPL;
  constexpr int CS = VROWS * RW;  // one velocity component of a slot
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *ring = reinterpret_cast<T *>(smem_raw);
  T *mring = ring + S * VPL;
  const Dims &g = a.g;
  const int tid = threadIdx.x;
  const int i0 = blockIdx.x * kFx, j0 = blockIdx.y * kFy;
  const int k0 = blockIdx.z * a.kz;
  const int k1 = min(k0 + a.kz, g.nz);
  const int mi = i0 + (tid & (kFx - 1)), mj = j0 + tid / kFx;
  const bool mine = mi < g.nx && mj < g.ny;

  const StageDesc<T, VEC> dvel(g, i0, j0, 2);
  auto stage = [&](T *sp, int p) {
    dvel.copy(sp, a.u, g, p);
    dvel.copy(sp + CS, a.v, g, p);
    dvel.copy(sp + 2 * CS, a.w, g, p);
    cp_async_commit();
  };
  auto next_slot = [&](T *sp) { return sp + VPL == ring + S * VPL ? ring : sp + VPL; };

  // Central-difference curl and |w| at (ci, cj) of plane p on the interior
  // (src/fluid.rs:260-281), 0 elsewhere; vm, vp, vq: staged planes p-1, p, p+1.
  auto curl_cell = [&](int ci, int cj, int p, const T *vm, const T *vp, const T *vq, T &ox,
                       T &oy, T &oz) -> T {
    if (!interior(g, ci, cj, p)) {
      ox = oy = oz = T(0);
      return T(0);
    }
    const int o = (cj - j0 + 2) * RW + (ci - i0 + XH);
    const T *U = vp + o, *Vv = vp + CS + o, *W = vp + 2 * CS + o;
    const T dw_dy = (W[RW] - W[-RW]) * a.inv_2h;
    const T dv_dz = (vq[CS + o] - vm[CS + o]) * a.inv_2h;
    const T du_dz = (vq[o] - vm[o]) * a.inv_2h;
    const T dw_dx = (W[1] - W[-1]) * a.inv_2h;
    const T dv_dx = (Vv[1] - Vv[-1]) * a.inv_2h;
    const T du_dy = (U[RW] - U[-RW]) * a.inv_2h;
    ox = dw_dy - dv_dz;
    oy = du_dz - dw_dx;
    oz = dv_dx - du_dy;
    return sqrt(ox * ox + oy * oy + oz * oz);
  };
  int hi_i = 0, hi_j = 0;
  if (tid < kFHalo) halo_cell(tid, i0, j0, hi_i, hi_j);
  auto curl_plane = [&](int p, const T *vm, const T *vp, const T *vq, T *M, T &ox, T &oy,
                        T &oz) {
    if (p < 0 || p >= g.nz) return;  // never read: confinement touches planes 1..nz-2
    if (mine) M[(mj - j0 + 1) * kFw + (mi - i0 + 1)] = curl_cell(mi, mj, p, vm, vp, vq, ox, oy, oz);
    if (tid < kFHalo) {
      T x_, y_, z_;
      M[(hi_j - j0 + 1) * kFw + (hi_i - i0 + 1)] = curl_cell(hi_i, hi_j, p, vm, vp, vq, x_, y_, z_);
    }
  };

  T ox = T(0), oy = T(0), oz = T(0), nox = T(0), noy = T(0), noz = T(0);
  {
    T *sp = ring;
    for (int p = k0 - 2; p <= k0 + S - 3; ++p) {
      stage(sp, p);
      sp += VPL;
    }
  }
  T *sm2 = ring, *sm1 = ring + VPL, *s0 = ring + 2 * VPL, *s1 = ring + 3 * VPL,
    *s2 = ring + 4 * VPL;
  T *M0 = mring, *M1 = mring + MPL, *M2 = mring + 2 * MPL;  // |w| of planes k-1, k, k+1
  cp_async_wait<S - 4>();
  __syncthreads();
  curl_plane(k0 - 1, sm2, sm1, s0, M0, nox, noy, noz);
  curl_plane(k0, sm1, s0, s1, M1, ox, oy, oz);

  for (int k = k0; k < k1; ++k) {
    const int c = (k * g.ny + mj) * g.nx + mi;
    T rho_c = T(0), temp_c = T(0);
    if (mine) {
      rho_c = __ldg(a.rho + c);
      temp_c = __ldg(a.temp + c);
    }
    cp_async_wait<S - 5>();
    __syncthreads();
    curl_plane(k + 1, s0, s1, s2, M2, nox, noy, noz);
    __syncthreads();
    stage(sm2, k + S - 2);
    if (mine) {  // cell_confine_buoy at (mi, mj, k)
      const int o = (mj - j0 + 2) * RW + (mi - i0 + XH);
      T uu = s0[o], vv = s0[CS + o], ww = s0[2 * CS + o];
      if (mi >= 2 && mi <= g.nx - 3 && mj >= 2 && mj <= g.ny - 3 && k >= 2 && k <= g.nz - 3) {
        const int mo = (mj - j0 + 1) * kFw + (mi - i0 + 1);
        const T *M = M1 + mo;
        const T gx = (M[1] - M[-1]) * a.inv_2h;
        const T gy = (M[kFw] - M[-kFw]) * a.inv_2h;
        const T gz = (M2[mo] - M0[mo]) * a.inv_2h;
        const T glen = sqrt(gx * gx + gy * gy + gz * gz) + T(1e-10);
        const T nx_ = gx / glen, ny_ = gy / glen, nz_ = gz / glen;
        const T fx = a.eps_h * (ny_ * oz - nz_ * oy);
        const T fy = a.eps_h * (nz_ * ox - nx_ * oz);
        const T fz = a.eps_h * (nx_ * oy - ny_ * ox);
        uu = uu + a.dt * fx;
        vv = vv + a.dt * fy;
        ww = ww + a.dt * fz;
      }
      if (interior(g, mi, mj, k)) {
        const T lift = a.beta * temp_c - a.alpha * rho_c;
        vv = vv + a.dt * lift;
      }
      a.uo[c] = wall_u(g, mi, mj, k) ? T(0) : uu;
      a.vo[c] = wall_v(g, mi, mj, k) ? T(0) : vv;
      a.wo[c] = wall_w(g, mi, mj, k) ? T(0) : ww;
    }
    ox = nox;
    oy = noy;
    oz = noz;
    sm2 = sm1;
    sm1 = s0;
    s0 = s1;
    s1 = s2;
    s2 = next_slot(s2);
    T *mt = M0;
    M0 = M1;
    M1 = M2;
    M2 = mt;
  }
  cp_async_wait<0>();
}

// ---- launchers ------------------------------------------------------------------
// Ring depths: six planes, two ahead of the stencils' reach.
constexpr int kRingScalar = 6, kRingForces = 6;

// z planes per CTA: about four waves of two resident CTAs per SM over the
// grid, and at least 8 planes per CTA (the ring is primed with two planes
// below the chunk).
inline int fused_kz(const Dims &g) {
  const int ctas_per_sm = 2;
  const int tiles = ((g.nx + kFx - 1) / kFx) * ((g.ny + kFy - 1) / kFy);
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0)
      sms = v;
  }
  long want = 4L * sms * ctas_per_sm;
  long chunks = (want + tiles - 1) / tiles;
  const long max_chunks = g.nz / 8 > 0 ? g.nz / 8 : 1;
  if (chunks > max_chunks) chunks = max_chunks;
  if (chunks < 1) chunks = 1;
  return static_cast<int>((g.nz + chunks - 1) / chunks);
}

inline dim3 fused_grid(const Dims &g, int kz) {
  return dim3((g.nx + kFx - 1) / kFx, (g.ny + kFy - 1) / kFy, (g.nz + kz - 1) / kz);
}

// Opts a kernel in to its dynamic shared memory (above the 48 KB default) on
// the current device, once per device.
template <typename K>
inline void fused_prepare(K kernel, size_t smem, unsigned long long &done_mask) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  if (done_mask & (1ull << dev)) return;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(smem)) == cudaSuccess)
    done_mask |= 1ull << dev;
}

template <typename T, bool VEC>
void launch_scalars_variant(McArgs<T> a, cudaStream_t st) {
  auto kern = k_maccormack_fused<T, 2, false, true, kRingScalar, VEC>;
  const size_t smem = sizeof(T) * McLayout<T, 2, false>::elems(kRingScalar);
  static unsigned long long prepared = 0;
  fused_prepare(kern, smem, prepared);
  a.kz = fused_kz(a.g);
  kern<<<fused_grid(a.g, a.kz), kFThreads, smem, st>>>(a);
}

template <typename T, bool VEC>
void launch_forces_variant(ForcesArgs<T> a, cudaStream_t st) {
  auto kern = k_forces_fused<T, kRingForces, VEC>;
  const size_t smem = sizeof(T) * ForcesLayout<T>::elems(kRingForces);
  static unsigned long long prepared = 0;
  fused_prepare(kern, smem, prepared);
  a.kz = fused_kz(a.g);
  kern<<<fused_grid(a.g, a.kz), kFThreads, smem, st>>>(a);
}

template <typename T>
void launch_forces_fused(const Dims &g, const T *u, const T *v, const T *w, const T *rho,
                         const T *temp, T *uo, T *vo, T *wo, double dt, double eps, double beta,
                         double alpha, cudaStream_t st) {
  ForcesArgs<T> a{};
  a.g = g;
  a.u = u;
  a.v = v;
  a.w = w;
  a.rho = rho;
  a.temp = temp;
  a.uo = uo;
  a.vo = vo;
  a.wo = wo;
  a.dt = T(dt);
  a.eps_h = T(eps * g.h);
  a.inv_2h = T(0.5 / g.h);
  a.beta = T(beta);
  a.alpha = T(alpha);
  if (g.nx % Staged<T>::V == 0) launch_forces_variant<T, true>(a, st);
  else launch_forces_variant<T, false>(a, st);
}

// CTAs of the fused density/temperature advection on this grid: the number
// of telemetry partials it writes.
inline int fused_ctas_of(const Dims &g) {
  const dim3 gr = fused_grid(g, fused_kz(g));
  return static_cast<int>(gr.x * gr.y * gr.z);
}

// advect_maccormack_in_place of density (dissipation diss[0]) and temperature
// (diss[1]) by (u, v, w) in one launch, into out[0], out[1] (arrays distinct
// from the inputs), max(0, .) applied; the telemetry partials of the final
// state go to tel, 7 per CTA (fused_ctas of them).
template <typename T>
void launch_scalars_fused(const Dims &g, const T *u, const T *v, const T *w,
                          const T *const src[2], T *const out[2], const double diss[2],
                          double dt, double *tel, cudaStream_t st) {
  McArgs<T> a{};
  a.g = g;
  a.u = u;
  a.v = v;
  a.w = w;
  for (int f = 0; f < 2; ++f) {
    a.src[f] = src[f];
    a.out[f] = out[f];
    a.diss[f] = T(diss[f]);
  }
  a.scale_f = T(dt / g.h);
  a.scale_b = T((-dt) / g.h);
  a.nonneg = 1;
  a.vel_src = -1;
  a.tel = tel;
  a.dv = g.h * g.h * g.h;
  a.inv_2h = 0.5 / g.h;
  if (g.nx % Staged<T>::V == 0) launch_scalars_variant<T, true>(a, st);
  else launch_scalars_variant<T, false>(a, st);
}

#define AFL_INSTANTIATE_FUSED(T)                                                           \
  template void launch_scalars_fused<T>(const Dims &, const T *, const T *, const T *,      \
                                        const T *const *, T *const *, const double *,       \
                                        double, double *, cudaStream_t);                    \
  template void launch_forces_fused<T>(const Dims &, const T *, const T *, const T *,       \
                                       const T *, const T *, T *, T *, T *, double, double, \
                                       double, double, cudaStream_t);

}  // namespace afl
