// afl_stage.cuh -- the per-stage kernels of one smoke step, templated on the
// field type T (double: FP64 drop-in; float: mixed form).  Included by
// afl_kernels_f64.cu (built with -fmad=false so every f64 expression rounds
// exactly like the reference's un-fused Rust arithmetic) and
// afl_kernels_f32.cu.
//
// Launch shape: the streaming/stencil kernels put one thread on one cell with
// CTAs of 32x8 cells in an x-y plane (a warp reads 32 consecutive doubles, one
// 256-byte line), grid.z walking the z planes.  Reductions run a fixed grid of
// kReduceBlocks CTAs so every sum is reproducible from run to run.
#pragma once

#include "afl_launch.h"

// Pointer qualifier of the per-cell code.  A unit that runs several stages in
// one launch, reading in a later stage what an earlier one wrote, defines it
// empty before including this header, so that no load of such data can be
// taken through the read-only (non-coherent) data path.
#ifndef AFL_RESTRICT
#define AFL_RESTRICT __restrict__
#endif

namespace afl {

constexpr int kTx = 32, kTy = 8;

inline dim3 plane_grid(const Dims &g) {
  return dim3((g.nx + kTx - 1) / kTx, (g.ny + kTy - 1) / kTy, g.nz);
}

// Cell coordinates of a thread in a plane_grid launch; false when outside.
__device__ __forceinline__ bool cell_of_thread(const Dims &g, int &i, int &j, int &k) {
  i = blockIdx.x * kTx + threadIdx.x;
  j = blockIdx.y * kTy + threadIdx.y;
  k = blockIdx.z;
  return i < g.nx && j < g.ny;
}

// The forward stage kernels give each thread kKz consecutive z planes of its
// (i, j) column: independent cells, so their loads are in flight together.
constexpr int kKz = 2;
inline dim3 column_grid(const Dims &g) {
  return dim3((g.nx + kTx - 1) / kTx, (g.ny + kTy - 1) / kTy, (g.nz + kKz - 1) / kKz);
}

// Runs body(i, j, k) for the thread's cells of a column_grid launch.
template <typename F>
__device__ __forceinline__ void for_column_cells(const Dims &g, F &&body) {
  const int i = blockIdx.x * kTx + threadIdx.x;
  const int j = blockIdx.y * kTy + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  const int k0 = blockIdx.z * kKz;
#pragma unroll
  for (int t = 0; t < kKz; ++t)
    if (k0 + t < g.nz) body(i, j, k0 + t);
}

// Each stage is a per-cell device function (shared by the single-grid kernels
// below and the batched ensemble kernels of afl_ensemble.cu, so both run the
// same arithmetic) plus a thin kernel over one grid.

// ---- MacCormack advection (src/fluid.rs:153-234) ---------------------------
// Pass 1: fwd = SL(src, dt) -- advect_semi_lagrangian (src/fluid.rs:153-167).
template <typename T>
__device__ __forceinline__ void cell_advect_fwd(const Dims &g, const T *AFL_RESTRICT u,
                                                const T *AFL_RESTRICT v,
                                                const T *AFL_RESTRICT w,
                                                const T *AFL_RESTRICT src, T *AFL_RESTRICT fwd,
                                                T scale, int i, int j, int k) {
  const int c = (k * g.ny + j) * g.nx + i;
  T out = T(0);
  if (interior(g, i, j, k)) {
    out = trilinear(src, g, footprint_at(g, i, j, k, scale * u[c], scale * v[c], scale * w[c]));
  }
  fwd[c] = out;
}

template <typename T>
__global__ void __launch_bounds__(kTx *kTy)
    k_advect_fwd(Dims g, const T *AFL_RESTRICT u, const T *AFL_RESTRICT v,
                 const T *AFL_RESTRICT w, const T *AFL_RESTRICT src, T *AFL_RESTRICT fwd,
                 T scale) {
  for_column_cells(g, [&](int i, int j, int k) {
    cell_advect_fwd(g, u, v, w, src, fwd, scale, i, j, k);
  });
}

// Pass 2: the reference's bwd = SL(fwd, -dt) (:184) is evaluated on the fly at
// each cell, then the MacCormack correction with the 8-cell clamp, the
// near-wall fallback, dissipation and max(0) for scalars (:186-229).  The
// result goes to a separate buffer: src is read at data-dependent cells.
template <typename T>
__device__ __forceinline__ void cell_advect_mc(const Dims &g, const T *AFL_RESTRICT u,
                                               const T *AFL_RESTRICT v,
                                               const T *AFL_RESTRICT w,
                                               const T *AFL_RESTRICT src,
                                               const T *AFL_RESTRICT fwd, T *AFL_RESTRICT out,
                                               T scale_f, T scale_b, T dissipation, int nonneg,
                                               int i, int j, int k) {
  const int c = (k * g.ny + j) * g.nx + i;
  T res = T(0);
  if (interior(g, i, j, k)) {
    const T uc = u[c], vc = v[c], wc = w[c];
    const T bx = T(i) - scale_f * uc;
    const T by = T(j) - scale_f * vc;
    const T bz = T(k) - scale_f * wc;
    const bool near_wall = bx < T(1.5) || bx > T(g.nx) - T(2.5) || by < T(1.5) ||
                           by > T(g.ny) - T(2.5) || bz < T(1.5) || bz > T(g.nz) - T(2.5);
    const T fc = fwd[c];
    T val;
    if (near_wall) {
      val = fc;
    } else {
      // bwd[c] = sample of fwd at the forward-traced point (scale_b = -dt/h)
      const T bwd = trilinear(fwd, g, footprint_at(g, i, j, k, scale_b * uc, scale_b * vc,
                                                    scale_b * wc));
      const T mc = fc + T(0.5) * (src[c] - bwd);
      T lo, hi;
      minmax8(src, g, footprint_at(g, i, j, k, scale_f * uc, scale_f * vc, scale_f * wc).base,
              lo, hi);
      val = rs_clamp(mc, lo, hi);
    }
    res = val * dissipation;
  }
  if (nonneg) res = fmax(res, T(0));
  out[c] = res;
}

template <typename T>
__global__ void __launch_bounds__(kTx *kTy)
    k_advect_mc(Dims g, const T *AFL_RESTRICT u, const T *AFL_RESTRICT v,
                const T *AFL_RESTRICT w, const T *AFL_RESTRICT src,
                const T *AFL_RESTRICT fwd, T *AFL_RESTRICT out, T scale_f, T scale_b,
                T dissipation, int nonneg) {
  for_column_cells(g, [&](int i, int j, int k) {
    cell_advect_mc(g, u, v, w, src, fwd, out, scale_f, scale_b, dissipation, nonneg, i, j, k);
  });
}

// ---- enforce_wall_velocity_bc (src/fluid.rs:236-253) -----------------------
template <typename T>
__global__ void __launch_bounds__(kTx *kTy)
    k_wall_bc(Dims g, T *AFL_RESTRICT u, T *AFL_RESTRICT v, T *AFL_RESTRICT w) {
  for_column_cells(g, [&](int i, int j, int k) {
    const int c = (k * g.ny + j) * g.nx + i;
    if (wall_u(g, i, j, k)) u[c] = T(0);
    if (wall_v(g, i, j, k)) v[c] = T(0);
    if (wall_w(g, i, j, k)) w[c] = T(0);
  });
}

// ---- vorticity confinement + buoyancy (src/fluid.rs:256-330) ---------------
// Pass 1: central-difference curl and |omega| on the interior (:260-281).
template <typename T>
__device__ __forceinline__ void cell_curl(const Dims &g, const T *AFL_RESTRICT u,
                                          const T *AFL_RESTRICT v, const T *AFL_RESTRICT w,
                                          T *AFL_RESTRICT cx, T *AFL_RESTRICT cy,
                                          T *AFL_RESTRICT cz, T *AFL_RESTRICT cmag, T inv_2h,
                                          int i, int j, int k) {
  const int c = (k * g.ny + j) * g.nx + i;
  if (!interior(g, i, j, k)) {
    cx[c] = T(0);
    cy[c] = T(0);
    cz[c] = T(0);
    cmag[c] = T(0);
    return;
  }
  const int sy = g.nx, sz = g.nxy;
  const T dw_dy = (w[c + sy] - w[c - sy]) * inv_2h;
  const T dv_dz = (v[c + sz] - v[c - sz]) * inv_2h;
  const T du_dz = (u[c + sz] - u[c - sz]) * inv_2h;
  const T dw_dx = (w[c + 1] - w[c - 1]) * inv_2h;
  const T dv_dx = (v[c + 1] - v[c - 1]) * inv_2h;
  const T du_dy = (u[c + sy] - u[c - sy]) * inv_2h;
  const T ox = dw_dy - dv_dz;
  const T oy = du_dz - dw_dx;
  const T oz = dv_dx - du_dy;
  cx[c] = ox;
  cy[c] = oy;
  cz[c] = oz;
  cmag[c] = sqrt(ox * ox + oy * oy + oz * oz);
}

template <typename T>
__global__ void __launch_bounds__(kTx *kTy)
    k_curl(Dims g, const T *AFL_RESTRICT u, const T *AFL_RESTRICT v,
           const T *AFL_RESTRICT w, T *AFL_RESTRICT cx, T *AFL_RESTRICT cy,
           T *AFL_RESTRICT cz, T *AFL_RESTRICT cmag, T inv_2h) {
  for_column_cells(g, [&](int i, int j, int k) {
    cell_curl(g, u, v, w, cx, cy, cz, cmag, inv_2h, i, j, k);
  });
}

// Pass 2: confinement force on 2..n-3 (:284-316), buoyancy lift on 1..n-2
// (:318-327) and the wall BC (:329), fused; pointwise in u/v/w, so in place.
// `rho_c`/`temp_c` are the density and temperature at the cell.
template <typename T>
__device__ __forceinline__ void cell_confine_buoy(const Dims &g, T *AFL_RESTRICT u,
                                                  T *AFL_RESTRICT v, T *AFL_RESTRICT w,
                                                  T rho_c, T temp_c, const T *AFL_RESTRICT cx,
                                                  const T *AFL_RESTRICT cy,
                                                  const T *AFL_RESTRICT cz,
                                                  const T *AFL_RESTRICT cmag, T dt, T eps_h,
                                                  T inv_2h, T beta, T alpha, int i, int j,
                                                  int k) {
  const int c = (k * g.ny + j) * g.nx + i;
  T uu = u[c], vv = v[c], ww = w[c];
  if (i >= 2 && i <= g.nx - 3 && j >= 2 && j <= g.ny - 3 && k >= 2 && k <= g.nz - 3) {
    const int sy = g.nx, sz = g.nxy;
    const T gx = (cmag[c + 1] - cmag[c - 1]) * inv_2h;
    const T gy = (cmag[c + sy] - cmag[c - sy]) * inv_2h;
    const T gz = (cmag[c + sz] - cmag[c - sz]) * inv_2h;
    const T glen = sqrt(gx * gx + gy * gy + gz * gz) + T(1e-10);
    const T nx = gx / glen, ny = gy / glen, nz = gz / glen;
    const T ox = cx[c], oy = cy[c], oz = cz[c];
    const T fx = eps_h * (ny * oz - nz * oy);
    const T fy = eps_h * (nz * ox - nx * oz);
    const T fz = eps_h * (nx * oy - ny * ox);
    uu = uu + dt * fx;
    vv = vv + dt * fy;
    ww = ww + dt * fz;
  }
  if (interior(g, i, j, k)) {
    const T lift = beta * temp_c - alpha * rho_c;
    vv = vv + dt * lift;
  }
  u[c] = wall_u(g, i, j, k) ? T(0) : uu;
  v[c] = wall_v(g, i, j, k) ? T(0) : vv;
  w[c] = wall_w(g, i, j, k) ? T(0) : ww;
}

template <typename T>
__global__ void __launch_bounds__(kTx *kTy)
    k_confine_buoy(Dims g, T *AFL_RESTRICT u, T *AFL_RESTRICT v, T *AFL_RESTRICT w,
                   const T *AFL_RESTRICT rho, const T *AFL_RESTRICT temp,
                   const T *AFL_RESTRICT cx, const T *AFL_RESTRICT cy,
                   const T *AFL_RESTRICT cz, const T *AFL_RESTRICT cmag, T dt, T eps_h,
                   T inv_2h, T beta, T alpha) {
  for_column_cells(g, [&](int i, int j, int k) {
    const int c = (k * g.ny + j) * g.nx + i;
    cell_confine_buoy(g, u, v, w, rho[c], temp[c], cx, cy, cz, cmag, dt, eps_h, inv_2h, beta,
                      alpha, i, j, k);
  });
}

// ---- compute_divergence_norm (src/fluid.rs:333-353) ------------------------
// Always evaluated in f64 (the mixed form recomputes the divergence in f64
// from its f32 velocities).  Flat grid-stride over the cells with a fixed CTA
// count; per-CTA partials of (sum div^2, sum b^2).
template <typename T>
__global__ void __launch_bounds__(kBlock)
    k_divergence(Dims g, const T *AFL_RESTRICT u, const T *AFL_RESTRICT v,
                 const T *AFL_RESTRICT w, double *AFL_RESTRICT b,
                 double *AFL_RESTRICT partials, double inv_h, double h) {
  __shared__ double scratch[kWarps * 2];
  double acc[2] = {0.0, 0.0};
#pragma unroll 2
  for (int c = blockIdx.x * kBlock + threadIdx.x; c < g.n; c += gridDim.x * kBlock) {
    int i, j, k;
    decode(g, c, i, j, k);
    double bv = 0.0;
    if (interior(g, i, j, k)) {
      const double du = double(u[c + 1]) - double(u[c]);
      const double dv = double(v[c + g.nx]) - double(v[c]);
      const double dw = double(w[c + g.nxy]) - double(w[c]);
      const double div_val = (du + dv + dw) * inv_h;
      bv = -h * (du + dv + dw);
      acc[0] += div_val * div_val;
      acc[1] += bv * bv;
    }
    b[c] = bv;
  }
  block_sum<2>(acc, scratch);
  if (threadIdx.x == 0) {
    partials[blockIdx.x * 2 + 0] = acc[0];
    partials[blockIdx.x * 2 + 1] = acc[1];
  }
}

// The same stage with four cells per thread (grids with nx % 128 == 0): a
// warp covers 128 consecutive cells of a row and lane l takes cells l, l+32,
// l+64 and l+96, so every load and store is coalesced and each thread has
// four cells' loads in flight; the per-cell arithmetic is k_divergence's.  A
// fixed grid of kReduceBlocks CTAs walks the rows, so the sums stay
// reproducible.
template <typename T>
__global__ void __launch_bounds__(kBlock)
    k_divergence_x4(Dims g, const T *AFL_RESTRICT u, const T *AFL_RESTRICT v,
                    const T *AFL_RESTRICT w, double *AFL_RESTRICT b,
                    double *AFL_RESTRICT partials, double inv_h, double h) {
  __shared__ double scratch[kWarps * 2];
  double acc[2] = {0.0, 0.0};
  const int lane = threadIdx.x & 31;
  const int segs = g.n / 128, sx = g.nx / 128;
  for (int sgi = (blockIdx.x * kBlock + threadIdx.x) / 32; sgi < segs;
       sgi += gridDim.x * kWarps) {
    const int row = sgi / sx;
    const int i0 = (sgi - row * sx) * 128 + lane;
    const int k = row / g.ny, j = row - k * g.ny;
    const int c0 = row * g.nx + i0;
    const bool rin = j >= 1 && j <= g.ny - 2 && k >= 1 && k <= g.nz - 2;
    double bv[4] = {0.0, 0.0, 0.0, 0.0};
    if (rin) {
      T uc[4], un[4], vc[4], vn[4], wc[4], wn[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const int c = c0 + 32 * a;
        const bool in_x = i0 + 32 * a + 1 < g.nx;
        uc[a] = u[c];
        un[a] = in_x ? u[c + 1] : T(0);
        vc[a] = v[c];
        vn[a] = v[c + g.nx];
        wc[a] = w[c];
        wn[a] = w[c + g.nxy];
      }
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const int i = i0 + 32 * a;
        if (i < 1 || i > g.nx - 2) continue;
        const double du = double(un[a]) - double(uc[a]);
        const double dv = double(vn[a]) - double(vc[a]);
        const double dw = double(wn[a]) - double(wc[a]);
        const double div_val = (du + dv + dw) * inv_h;
        bv[a] = -h * (du + dv + dw);
        acc[0] += div_val * div_val;
        acc[1] += bv[a] * bv[a];
      }
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) b[c0 + 32 * a] = bv[a];
  }
  block_sum<2>(acc, scratch);
  if (threadIdx.x == 0) {
    partials[blockIdx.x * 2 + 0] = acc[0];
    partials[blockIdx.x * 2 + 1] = acc[1];
  }
}

// Finishes k_divergence: out2 = {RMS divergence, ||b||_2}.
__global__ void __launch_bounds__(kBlock)
    k_divergence_finalize(const double *AFL_RESTRICT partials, int nparts,
                          double interior_cells, double *AFL_RESTRICT out2);

// ---- projection (src/fluid.rs:509-528) -------------------------------------
// u -= (p[i]-p[i-1])/h where i > 1 (likewise v, w), then the wall BC.  The
// gradient is formed in f64; in the mixed form the f32 velocity is updated in
// f64 and rounded once.
template <typename T>
__device__ __forceinline__ void cell_project(const Dims &g, T *AFL_RESTRICT u,
                                             T *AFL_RESTRICT v, T *AFL_RESTRICT w,
                                             const double *AFL_RESTRICT p, double inv_h, int i,
                                             int j, int k) {
  const int c = (k * g.ny + j) * g.nx + i;
  if (interior(g, i, j, k)) {
    const double pc = p[c];
    if (i > 1) u[c] = T(double(u[c]) - (pc - p[c - 1]) * inv_h);
    if (j > 1) v[c] = T(double(v[c]) - (pc - p[c - g.nx]) * inv_h);
    if (k > 1) w[c] = T(double(w[c]) - (pc - p[c - g.nxy]) * inv_h);
  }
  if (wall_u(g, i, j, k)) u[c] = T(0);
  if (wall_v(g, i, j, k)) v[c] = T(0);
  if (wall_w(g, i, j, k)) w[c] = T(0);
}

template <typename T>
__global__ void __launch_bounds__(kTx *kTy)
    k_project(Dims g, T *AFL_RESTRICT u, T *AFL_RESTRICT v, T *AFL_RESTRICT w,
              const double *AFL_RESTRICT p, double inv_h) {
  for_column_cells(g, [&](int i, int j, int k) {
    cell_project(g, u, v, w, p, inv_h, i, j, k);
  });
}

// The same stage with four cells per thread (nx % 128 == 0): a warp covers
// 128 consecutive cells of a row, lane l takes cells l, l+32, l+64 and
// l+96, so every load and store is coalesced; cell_project's arithmetic.
template <typename T>
__global__ void __launch_bounds__(kBlock)
    k_project_x4(Dims g, T *AFL_RESTRICT u, T *AFL_RESTRICT v, T *AFL_RESTRICT w,
                 const double *AFL_RESTRICT p, double inv_h) {
  const int lane = threadIdx.x & 31;
  const int sgi = (blockIdx.x * kBlock + threadIdx.x) / 32;
  if (sgi >= g.n / 128) return;
  const int sx = g.nx / 128;
  const int row = sgi / sx;
  const int i0 = (sgi - row * sx) * 128 + lane;
  const int k = row / g.ny, j = row - k * g.ny;
  const int c0 = row * g.nx + i0;
  const bool rin = j >= 1 && j <= g.ny - 2 && k >= 1 && k <= g.nz - 2;
  T uu[4], vv[4], ww[4];
  double pc[4], pxm[4], pym[4], pzm[4];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int c = c0 + 32 * a;
    uu[a] = u[c];
    vv[a] = v[c];
    ww[a] = w[c];
    if (rin) {
      pc[a] = p[c];
      pxm[a] = i0 + 32 * a > 0 ? p[c - 1] : 0.0;
      pym[a] = p[c - g.nx];
      pzm[a] = p[c - g.nxy];
    }
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int i = i0 + 32 * a;
    if (rin && i >= 1 && i <= g.nx - 2) {
      if (i > 1) uu[a] = T(double(uu[a]) - (pc[a] - pxm[a]) * inv_h);
      if (j > 1) vv[a] = T(double(vv[a]) - (pc[a] - pym[a]) * inv_h);
      if (k > 1) ww[a] = T(double(ww[a]) - (pc[a] - pzm[a]) * inv_h);
    }
    const int c = c0 + 32 * a;
    u[c] = wall_u(g, i, j, k) ? T(0) : uu[a];
    v[c] = wall_v(g, i, j, k) ? T(0) : vv[a];
    w[c] = wall_w(g, i, j, k) ? T(0) : ww[a];
  }
}

// ---- sources -----------------------------------------------------------------
// One jet of inject_cyberpunk_sources (src/fluid.rs:573-593) over its clamped
// bounding box; the two jets are launched in order because their boxes can
// overlap.  pulse and the jet geometry are computed on the host.
template <typename T>
__global__ void __launch_bounds__(kTx *kTy)
    k_inject_jet(Dims g, int i0, int j0, int k0, int ni, int nj, T *AFL_RESTRICT rho,
                 T *AFL_RESTRICT temp, T *AFL_RESTRICT u, T *AFL_RESTRICT v,
                 T *AFL_RESTRICT w, double jx, double jy, double jz, double vx, double vy,
                 double vz, double r2, double dt, double pulse) {
  const int ii = blockIdx.x * kTx + threadIdx.x;
  const int jj = blockIdx.y * kTy + threadIdx.y;
  if (ii >= ni || jj >= nj) return;
  const int i = i0 + ii, j = j0 + jj, k = k0 + blockIdx.z;
  const double dx = double(i) - jx;
  const double dy = double(j) - jy;
  const double dz = double(k) - jz;
  const double d2 = dx * dx + dy * dy + dz * dz;
  if (!(d2 < r2)) return;
  const double wf = exp(-2.2 * d2 / r2);
  const int c = (k * g.ny + j) * g.nx + i;
  rho[c] = T(fmin(double(rho[c]) + dt * 9.5 * pulse * wf, 3.8));
  temp[c] = T(fmin(double(temp[c]) + dt * 8.2 * pulse * wf, 4.5));
  u[c] = T(double(u[c]) + dt * vx * wf * 4.2);
  v[c] = T(double(v[c]) + dt * vy * wf * 4.2);
  w[c] = T(double(w[c]) + dt * vz * wf * 4.2);
}

// Sphere source: density/temperature assignment inside the sphere.
template <typename T>
__global__ void __launch_bounds__(kTx *kTy)
    k_inject_sphere(Dims g, int i0, int j0, int k0, int ni, int nj, T *AFL_RESTRICT rho,
                    T *AFL_RESTRICT temp, const double *AFL_RESTRICT amp, double cx,
                    double cy, double cz, double r2, double rho_val, double temp_val) {
  const int ii = blockIdx.x * kTx + threadIdx.x;
  const int jj = blockIdx.y * kTy + threadIdx.y;
  if (ii >= ni || jj >= nj) return;
  const int i = i0 + ii, j = j0 + jj, k = k0 + blockIdx.z;
  const double dx = double(i) - cx;
  const double dy = double(j) - cy;
  const double dz = double(k) - cz;
  const double d2 = dx * dx + dy * dy + dz * dz;
  if (!(d2 < r2)) return;
  const int c = (k * g.ny + j) * g.nx + i;
  rho[c] = T(rho_val);
  temp[c] = T(amp ? temp_val * amp[c] : temp_val);
}

// ---- compute_telemetry (src/fluid.rs:613-672) -------------------------------
// Per-CTA partials of (KE, enstrophy, mass, com x, com y, com z, peak |w|).
template <typename T>
__global__ void __launch_bounds__(kBlock)
    k_telemetry(Dims g, const T *AFL_RESTRICT u, const T *AFL_RESTRICT v,
                const T *AFL_RESTRICT w, const T *AFL_RESTRICT rho,
                double *AFL_RESTRICT partials, double dv, double inv_2h) {
  __shared__ double scratch[kWarps * 6];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  double peak = 0.0;
  const double sx = 1.0 / double(g.nx - 1), sy = 1.0 / double(g.ny - 1),
               sz = 1.0 / double(g.nz - 1);
  (void)sx;
  (void)sy;
  (void)sz;
#pragma unroll 2
  for (int c = blockIdx.x * kBlock + threadIdx.x; c < g.n; c += gridDim.x * kBlock) {
    int i, j, k;
    decode(g, c, i, j, k);
    if (!interior(g, i, j, k)) continue;
    const double uc = u[c], vc = v[c], wc = w[c];
    const double u2 = uc * uc + vc * vc + wc * wc;
    acc[0] += 0.5 * u2 * dv;
    const int ny_ = g.nx, nz_ = g.nxy;
    const double dw_dy = (double(w[c + ny_]) - double(w[c - ny_])) * inv_2h;
    const double dv_dz = (double(v[c + nz_]) - double(v[c - nz_])) * inv_2h;
    const double du_dz = (double(u[c + nz_]) - double(u[c - nz_])) * inv_2h;
    const double dw_dx = (double(w[c + 1]) - double(w[c - 1])) * inv_2h;
    const double dv_dx = (double(v[c + 1]) - double(v[c - 1])) * inv_2h;
    const double du_dy = (double(u[c + ny_]) - double(u[c - ny_])) * inv_2h;
    const double ox = dw_dy - dv_dz;
    const double oy = du_dz - dw_dx;
    const double oz = dv_dx - du_dy;
    const double w2 = ox * ox + oy * oy + oz * oz;
    acc[1] += 0.5 * w2 * dv;
    peak = fmax(peak, sqrt(w2));
    const double r = rho[c];
    if (r > 1e-8) {
      acc[2] += r * dv;
      const double nxn = 2.0 * (double(i) / double(g.nx - 1)) - 1.0;
      const double nyn = 2.0 * (double(j) / double(g.ny - 1)) - 1.0;
      const double nzn = 2.0 * (double(k) / double(g.nz - 1)) - 1.0;
      const double wgt = r * dv;
      acc[3] += nxn * wgt;
      acc[4] += nyn * wgt;
      acc[5] += nzn * wgt;
    }
  }
  block_sum<6>(acc, scratch);
  const double pk = block_max(peak, scratch);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int a = 0; a < 6; ++a) partials[blockIdx.x * 7 + a] = acc[a];
    partials[blockIdx.x * 7 + 6] = pk;
  }
}

__global__ void __launch_bounds__(kBlock)
    k_telemetry_finalize(const double *AFL_RESTRICT partials, int nparts, double time_sec,
                         double *AFL_RESTRICT out8);

template <typename T>
__global__ void __launch_bounds__(kBlock)
    k_max(int n, const T *AFL_RESTRICT x, double *AFL_RESTRICT partials) {
  __shared__ double scratch[kWarps];
  double m = 0.0;  // max_density starts at 0 (src/fluid.rs:704)
  for (int c = blockIdx.x * kBlock + threadIdx.x; c < n; c += gridDim.x * kBlock)
    m = fmax(m, double(x[c]));
  m = block_max(m, scratch);
  if (threadIdx.x == 0) partials[blockIdx.x] = m;
}

__global__ void __launch_bounds__(kBlock)
    k_max_finalize(const double *AFL_RESTRICT partials, int nparts, double *AFL_RESTRICT out1);

// Batched sample_trilinear (src/fluid.rs:94-128) at caller-given points.
template <typename T>
__global__ void __launch_bounds__(kBlock)
    k_sample(Dims g, const T *AFL_RESTRICT f, const double *AFL_RESTRICT xyz, int npts,
             double *AFL_RESTRICT out) {
  const int t = blockIdx.x * kBlock + threadIdx.x;
  if (t >= npts) return;
  const T x = T(xyz[3 * t]), y = T(xyz[3 * t + 1]), z = T(xyz[3 * t + 2]);
  out[t] = double(trilinear(f, g, footprint(g, x, y, z)));
}

// ---- launchers ------------------------------------------------------------
template <typename T>
void launch_advect_fwd(const Dims &g, const T *u, const T *v, const T *w, const T *src,
                       T *fwd, double dt, cudaStream_t st) {
  const double scale = dt / g.h;
  k_advect_fwd<T><<<column_grid(g), dim3(kTx, kTy), 0, st>>>(g, u, v, w, src, fwd, T(scale));
}

template <typename T>
void launch_advect_mc(const Dims &g, const T *u, const T *v, const T *w, const T *src,
                      const T *fwd, T *out, double dt, double dissipation, bool nonneg,
                      cudaStream_t st) {
  const double scale_f = dt / g.h;
  const double scale_b = (-dt) / g.h;
  k_advect_mc<T><<<column_grid(g), dim3(kTx, kTy), 0, st>>>(
      g, u, v, w, src, fwd, out, T(scale_f), T(scale_b), T(dissipation), nonneg ? 1 : 0);
}

template <typename T>
void launch_wall_bc(const Dims &g, T *u, T *v, T *w, cudaStream_t st) {
  k_wall_bc<T><<<column_grid(g), dim3(kTx, kTy), 0, st>>>(g, u, v, w);
}

template <typename T>
void launch_curl(const Dims &g, const T *u, const T *v, const T *w, T *cx, T *cy, T *cz,
                 T *cmag, cudaStream_t st) {
  const double inv_2h = 0.5 / g.h;
  k_curl<T><<<column_grid(g), dim3(kTx, kTy), 0, st>>>(g, u, v, w, cx, cy, cz, cmag,
                                                      T(inv_2h));
}

template <typename T>
void launch_confine_buoy(const Dims &g, T *u, T *v, T *w, const T *rho, const T *temp,
                         const T *cx, const T *cy, const T *cz, const T *cmag, double dt,
                         double eps, double beta, double alpha, cudaStream_t st) {
  const double inv_2h = 0.5 / g.h;
  const double eps_h = eps * g.h;
  k_confine_buoy<T><<<column_grid(g), dim3(kTx, kTy), 0, st>>>(
      g, u, v, w, rho, temp, cx, cy, cz, cmag, T(dt), T(eps_h), T(inv_2h), T(beta),
      T(alpha));
}

template <typename T>
void launch_divergence(const Dims &g, const T *u, const T *v, const T *w, double *b,
                       double *partials, double *out2, cudaStream_t st) {
  const double inv_h = 1.0 / g.h;
  if (g.nx % 128 == 0)
    k_divergence_x4<T><<<kReduceBlocks, kBlock, 0, st>>>(g, u, v, w, b, partials, inv_h, g.h);
  else
    k_divergence<T><<<kReduceBlocks, kBlock, 0, st>>>(g, u, v, w, b, partials, inv_h, g.h);
  const double interior_cells = double(g.nx - 2) * double(g.ny - 2) * double(g.nz - 2);
  k_divergence_finalize<<<1, kBlock, 0, st>>>(partials, kReduceBlocks, interior_cells, out2);
}

template <typename T>
void launch_project(const Dims &g, T *u, T *v, T *w, const double *p, cudaStream_t st) {
  if (g.nx % 128 == 0)
    k_project_x4<T><<<(g.n / 128 + kWarps - 1) / kWarps, kBlock, 0, st>>>(g, u, v, w, p,
                                                                          1.0 / g.h);
  else
    k_project<T><<<column_grid(g), dim3(kTx, kTy), 0, st>>>(g, u, v, w, p, 1.0 / g.h);
}

template <typename T>
void launch_inject_jet(const Dims &g, const int lo[3], const int hi[3], T *rho, T *temp,
                       T *u, T *v, T *w, const double jet[6], double r2, double dt,
                       double pulse, cudaStream_t st) {
  const int ni = hi[0] - lo[0] + 1, nj = hi[1] - lo[1] + 1, nk = hi[2] - lo[2] + 1;
  if (ni <= 0 || nj <= 0 || nk <= 0) return;
  dim3 grid((ni + kTx - 1) / kTx, (nj + kTy - 1) / kTy, nk);
  k_inject_jet<T><<<grid, dim3(kTx, kTy), 0, st>>>(g, lo[0], lo[1], lo[2], ni, nj, rho,
                                                   temp, u, v, w, jet[0], jet[1], jet[2],
                                                   jet[3], jet[4], jet[5], r2, dt, pulse);
}

template <typename T>
void launch_inject_sphere(const Dims &g, const int lo[3], const int hi[3], T *rho,
                          T *temp, const double *amp, const double c[3], double r2,
                          double rho_val, double temp_val, cudaStream_t st) {
  const int ni = hi[0] - lo[0] + 1, nj = hi[1] - lo[1] + 1, nk = hi[2] - lo[2] + 1;
  if (ni <= 0 || nj <= 0 || nk <= 0) return;
  dim3 grid((ni + kTx - 1) / kTx, (nj + kTy - 1) / kTy, nk);
  k_inject_sphere<T><<<grid, dim3(kTx, kTy), 0, st>>>(g, lo[0], lo[1], lo[2], ni, nj, rho,
                                                      temp, amp, c[0], c[1], c[2], r2,
                                                      rho_val, temp_val);
}

template <typename T>
void launch_telemetry(const Dims &g, const T *u, const T *v, const T *w, const T *rho,
                      double time_sec, double *partials, double *out8, cudaStream_t st) {
  const double dv = g.h * g.h * g.h;
  const double inv_2h = 0.5 / g.h;
  k_telemetry<T><<<kReduceBlocks, kBlock, 0, st>>>(g, u, v, w, rho, partials, dv, inv_2h);
  k_telemetry_finalize<<<1, kBlock, 0, st>>>(partials, kReduceBlocks, time_sec, out8);
}

template <typename T>
void launch_max(const Dims &g, const T *x, double *partials, double *out1, cudaStream_t st) {
  k_max<T><<<kReduceBlocks, kBlock, 0, st>>>(g.n, x, partials);
  k_max_finalize<<<1, kBlock, 0, st>>>(partials, kReduceBlocks, out1);
}

template <typename T>
void launch_sample(const Dims &g, const T *f, const double *xyz, int npts, double *out,
                   cudaStream_t st) {
  if (npts <= 0) return;
  k_sample<T><<<(npts + kBlock - 1) / kBlock, kBlock, 0, st>>>(g, f, xyz, npts, out);
}

#define AFL_INSTANTIATE_STAGES(T)                                                        \
  template void launch_advect_fwd<T>(const Dims &, const T *, const T *, const T *,      \
                                     const T *, T *, double, cudaStream_t);              \
  template void launch_advect_mc<T>(const Dims &, const T *, const T *, const T *,       \
                                    const T *, const T *, T *, double, double, bool,     \
                                    cudaStream_t);                                       \
  template void launch_wall_bc<T>(const Dims &, T *, T *, T *, cudaStream_t);            \
  template void launch_curl<T>(const Dims &, const T *, const T *, const T *, T *, T *,  \
                               T *, T *, cudaStream_t);                                  \
  template void launch_confine_buoy<T>(const Dims &, T *, T *, T *, const T *, const T *, \
                                       const T *, const T *, const T *, const T *,       \
                                       double, double, double, double, cudaStream_t);    \
  template void launch_divergence<T>(const Dims &, const T *, const T *, const T *,      \
                                     double *, double *, double *, cudaStream_t);        \
  template void launch_project<T>(const Dims &, T *, T *, T *, const double *,           \
                                  cudaStream_t);                                         \
  template void launch_inject_jet<T>(const Dims &, const int *, const int *, T *, T *,   \
                                     T *, T *, T *, const double *, double, double,      \
                                     double, cudaStream_t);                              \
  template void launch_inject_sphere<T>(const Dims &, const int *, const int *, T *, T *, \
                                        const double *, const double *, double, double,  \
                                        double, cudaStream_t);                           \
  template void launch_telemetry<T>(const Dims &, const T *, const T *, const T *,       \
                                    const T *, double, double *, double *,               \
                                    cudaStream_t);                                       \
  template void launch_max<T>(const Dims &, const T *, double *, double *, cudaStream_t); \
  template void launch_sample<T>(const Dims &, const T *, const double *, int, double *, \
                                 cudaStream_t);

}  // namespace afl
