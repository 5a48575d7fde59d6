// afl_ensemble_kernels.cuh -- batched stage kernels for an ensemble of
// independent smoke plumes of different grid sizes.
//
// One launch covers every instance: the plane blocks (32 x 8 cells of kz z
// planes, one 256-thread CTA each) of all instances are numbered
// consecutively and a block table maps a CTA to its instance.  Each kernel calls the same per-cell functions as the
// single-grid kernels of afl_stage.cuh, so an instance evolves exactly like a
// single-grid solver with the same settings (up to the summation order of its
// reductions).  Field pointers live in the device-side instance descriptors;
// the MacCormack ping-pong swaps them on the device, so a captured step graph
// stays valid from step to step.  Included by afl_ensemble_f64.cu (built
// without FMA contraction, like afl_kernels_f64.cu) and afl_ensemble_f32.cu.
#pragma once

#include "afl_stage.cuh"

namespace afl {

// The cells of plane block `local` of an instance: a 32 x 8 tile of d.kz
// consecutive z planes (the tile depth is the tuner's choice); body(i, j, k)
// per cell, one cell per thread and plane.
template <typename T, typename F>
__device__ __forceinline__ void ens_cells_at(const EnsInstance<T> &d, int local, F &&body) {
  const int gx = (d.g.nx + kTx - 1) / kTx, gy = (d.g.ny + kTy - 1) / kTy;
  const int bx = local % gx, t = local / gx;
  const int by = t % gy;
  const int k0 = (t / gy) * d.kz;
  // 1-D CTAs of kTx*kTy threads: lane = x offset, warp = y offset
  const int i = bx * kTx + static_cast<int>(threadIdx.x & (kTx - 1));
  const int j = by * kTy + static_cast<int>(threadIdx.x / kTx);
  if (i >= d.g.nx || j >= d.g.ny) return;
  const int k1 = min(k0 + d.kz, d.g.nz);
  for (int k = k0; k < k1; ++k) body(i, j, k);
}

// The cells of this CTA's plane block (its index in the block table).
template <typename T, typename F>
__device__ __forceinline__ void ens_cells(const EnsInstance<T> &d, F &&body) {
  ens_cells_at(d, static_cast<int>(blockIdx.x) - d.blk_begin, body);
}

// ---- per-block bodies ---------------------------------------------------------
// Each body does one plane block (`local` within its instance); the batched
// kernels below run one block per CTA, the persistent step kernel
// (afl_ensemble_persist.cu) loops its CTAs over the blocks of their instance.
template <typename T>
__device__ __forceinline__ void blk_advect_fwd(const EnsInstance<T> &d, int local, int f) {
  ens_cells_at(d, local, [&](int i, int j, int k) {
    cell_advect_fwd(d.g, d.fld[0], d.fld[1], d.fld[2], d.fld[f], d.tmp_fwd, d.scale_f, i, j, k);
  });
}

template <typename T>
__device__ __forceinline__ void blk_advect_mc(const EnsInstance<T> &d, int local, int f,
                                              double dissipation) {
  ens_cells_at(d, local, [&](int i, int j, int k) {
    cell_advect_mc(d.g, d.fld[0], d.fld[1], d.fld[2], d.fld[f], d.tmp_fwd, d.tmp_out, d.scale_f,
                   d.scale_b, T(dissipation), f >= 3 ? 1 : 0, i, j, k);
  });
}

template <typename T>
__device__ __forceinline__ void blk_curl(const EnsInstance<T> &d, int local) {
  ens_cells_at(d, local, [&](int i, int j, int k) {
    cell_curl(d.g, d.fld[0], d.fld[1], d.fld[2], d.curl[0], d.curl[1], d.curl[2], d.curl[3],
              d.inv_2h, i, j, k);
  });
}

// Sphere source (density/temperature assignment) fused with the confinement
// and buoyancy pass that follows it in the step: the pass reads density and
// temperature only at its own cell, after the assignment, as the separate
// kernels do.
template <typename T>
__device__ __forceinline__ void blk_source_confine_buoy(const EnsInstance<T> &d, int local) {
  ens_cells_at(d, local, [&](int i, int j, int k) {
    const int c = (k * d.g.ny + j) * d.g.nx + i;
    T rho = d.fld[3][c], temp = d.fld[4][c];
    if (d.src_on && i >= d.src_lo[0] && i <= d.src_hi[0] && j >= d.src_lo[1] &&
        j <= d.src_hi[1] && k >= d.src_lo[2] && k <= d.src_hi[2]) {
      const double dx = double(i) - d.src_c[0];
      const double dy = double(j) - d.src_c[1];
      const double dz = double(k) - d.src_c[2];
      const double d2 = dx * dx + dy * dy + dz * dz;
      if (d2 < d.src_r2) {
        rho = T(d.src_rho);
        temp = T(d.src_temp);
        d.fld[3][c] = rho;
        d.fld[4][c] = temp;
      }
    }
    cell_confine_buoy(d.g, d.fld[0], d.fld[1], d.fld[2], rho, temp, d.curl[0], d.curl[1],
                      d.curl[2], d.curl[3], d.dt, d.eps_h, d.inv_2h, d.beta, d.alpha, i, j, k);
  });
}

// Right-hand side b = -h*(du+dv+dw) (src/fluid.rs:341-346), in f64.
template <typename T>
__device__ __forceinline__ void blk_divergence(const EnsInstance<T> &d, int local) {
  ens_cells_at(d, local, [&](int i, int j, int k) {
    const int c = (k * d.g.ny + j) * d.g.nx + i;
    double bv = 0.0;
    if (interior(d.g, i, j, k)) {
      const T *u = d.fld[0], *v = d.fld[1], *w = d.fld[2];
      const double du = double(u[c + 1]) - double(u[c]);
      const double dv = double(v[c + d.g.nx]) - double(v[c]);
      const double dw = double(w[c + d.g.nxy]) - double(w[c]);
      bv = -d.h * (du + dv + dw);
    }
    d.b[c] = bv;
  });
}

template <typename T>
__device__ __forceinline__ void blk_project(const EnsInstance<T> &d, int local) {
  ens_cells_at(d, local, [&](int i, int j, int k) {
    cell_project(d.g, d.fld[0], d.fld[1], d.fld[2], d.p, d.inv_h, i, j, k);
  });
}

// compute_telemetry (src/fluid.rs:613-672): the block's partials of
// (KE, enstrophy, mass, com x, com y, com z, peak |w|) into
// partials[(blk_begin + local) * 7 ...].  Block-wide: every thread of the CTA
// calls it.
template <typename T>
__device__ __forceinline__ void blk_telemetry(const EnsInstance<T> &d, int local,
                                              double *partials, double *scratch) {
  double acc[6] = {0, 0, 0, 0, 0, 0};
  double peak = 0.0;
  ens_cells_at(d, local, [&](int i, int j, int k) {
    if (!interior(d.g, i, j, k)) return;
    const Dims &g = d.g;
    const int c = (k * g.ny + j) * g.nx + i;
    const T *u = d.fld[0], *v = d.fld[1], *w = d.fld[2], *rho = d.fld[3];
    const double uc = u[c], vc = v[c], wc = w[c];
    const double u2 = uc * uc + vc * vc + wc * wc;
    acc[0] += 0.5 * u2 * d.dv;
    const double inv_2h = d.inv_2h_d;
    const double dw_dy = (double(w[c + g.nx]) - double(w[c - g.nx])) * inv_2h;
    const double dv_dz = (double(v[c + g.nxy]) - double(v[c - g.nxy])) * inv_2h;
    const double du_dz = (double(u[c + g.nxy]) - double(u[c - g.nxy])) * inv_2h;
    const double dw_dx = (double(w[c + 1]) - double(w[c - 1])) * inv_2h;
    const double dv_dx = (double(v[c + 1]) - double(v[c - 1])) * inv_2h;
    const double du_dy = (double(u[c + g.nx]) - double(u[c - g.nx])) * inv_2h;
    const double ox = dw_dy - dv_dz;
    const double oy = du_dz - dw_dx;
    const double oz = dv_dx - du_dy;
    const double w2 = ox * ox + oy * oy + oz * oz;
    acc[1] += 0.5 * w2 * d.dv;
    peak = fmax(peak, sqrt(w2));
    const double r = rho[c];
    if (r > 1e-8) {
      acc[2] += r * d.dv;
      const double wgt = r * d.dv;
      acc[3] += (2.0 * (double(i) / double(g.nx - 1)) - 1.0) * wgt;
      acc[4] += (2.0 * (double(j) / double(g.ny - 1)) - 1.0) * wgt;
      acc[5] += (2.0 * (double(k) / double(g.nz - 1)) - 1.0) * wgt;
    }
  });
  block_sum<6>(acc, scratch);
  const double pk = block_max(peak, scratch);
  if (threadIdx.x == 0) {
    double *out = partials + static_cast<size_t>(d.blk_begin + local) * 7;
#pragma unroll
    for (int a = 0; a < 6; ++a) out[a] = acc[a];
    out[6] = pk;
  }
}

// Sums instance m's block partials in block order into its telemetry frame of
// step `step`, and files the step's solve report.  Block-wide, kBlock threads.
template <typename T>
__device__ __forceinline__ void ens_finalize(const EnsInstance<T> &d, int m,
                                             const double *partials, int step, double *tel_out,
                                             const SolveReport *rep_cur, SolveReport *reports,
                                             int count, int capacity, double *scratch) {
  double acc[6] = {0, 0, 0, 0, 0, 0};
  double peak = 0.0;
  for (int b = threadIdx.x; b < d.blk_count; b += kBlock) {
    const double *pp = partials + (d.blk_begin + b) * 7;
#pragma unroll
    for (int a = 0; a < 6; ++a) acc[a] += pp[a];
    peak = fmax(peak, pp[6]);
  }
  block_sum<6>(acc, scratch);
  peak = block_max(peak, scratch);
  if (threadIdx.x == 0 && step < capacity) {
    double *out = tel_out + (static_cast<size_t>(step) * count + m) * 8;
    const double mass = acc[2];
    double com[3] = {acc[3], acc[4], acc[5]};
    if (mass > 1e-12) {
      const double inv = 1.0 / mass;
      for (int a = 0; a < 3; ++a) com[a] = com[a] * inv;
    }
    out[0] = double(step) * d.dt_time;
    out[1] = acc[0];
    out[2] = acc[1];
    out[3] = peak;
    out[4] = mass;
    for (int a = 0; a < 3; ++a) out[5 + a] = rs_clamp(com[a], -1.0, 1.0);
    reports[static_cast<size_t>(step) * count + m] = rep_cur[m];
  }
}

// ---- batched kernels: one plane block per CTA ---------------------------------
template <typename T>
__global__ void __launch_bounds__(kTx *kTy)
    kb_advect_fwd(const EnsInstance<T> *inst, const int *blk_inst, int f) {
  const EnsInstance<T> &d = inst[blk_inst[blockIdx.x]];
  blk_advect_fwd(d, static_cast<int>(blockIdx.x) - d.blk_begin, f);
}

template <typename T>
__global__ void __launch_bounds__(kTx *kTy)
    kb_advect_mc(const EnsInstance<T> *inst, const int *blk_inst, int f, double dissipation) {
  const EnsInstance<T> &d = inst[blk_inst[blockIdx.x]];
  blk_advect_mc(d, static_cast<int>(blockIdx.x) - d.blk_begin, f, dissipation);
}

// The advected field becomes current; its old buffer becomes the next output.
template <typename T>
__global__ void kb_swap(EnsInstance<T> *inst, int count, int f) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= count) return;
  T *t = inst[m].fld[f];
  inst[m].fld[f] = inst[m].tmp_out;
  inst[m].tmp_out = t;
}

template <typename T>
__global__ void __launch_bounds__(kTx *kTy) kb_curl(const EnsInstance<T> *inst, const int *blk_inst) {
  const EnsInstance<T> &d = inst[blk_inst[blockIdx.x]];
  blk_curl(d, static_cast<int>(blockIdx.x) - d.blk_begin);
}

template <typename T>
__global__ void __launch_bounds__(kTx *kTy)
    kb_source_confine_buoy(const EnsInstance<T> *inst, const int *blk_inst) {
  const EnsInstance<T> &d = inst[blk_inst[blockIdx.x]];
  blk_source_confine_buoy(d, static_cast<int>(blockIdx.x) - d.blk_begin);
}

template <typename T>
__global__ void __launch_bounds__(kTx *kTy)
    kb_divergence(const EnsInstance<T> *inst, const int *blk_inst) {
  const EnsInstance<T> &d = inst[blk_inst[blockIdx.x]];
  blk_divergence(d, static_cast<int>(blockIdx.x) - d.blk_begin);
}

template <typename T>
__global__ void __launch_bounds__(kTx *kTy)
    kb_project(const EnsInstance<T> *inst, const int *blk_inst) {
  const EnsInstance<T> &d = inst[blk_inst[blockIdx.x]];
  blk_project(d, static_cast<int>(blockIdx.x) - d.blk_begin);
}

template <typename T>
__global__ void __launch_bounds__(kTx *kTy)
    kb_telemetry(const EnsInstance<T> *inst, const int *blk_inst, double *partials) {
  __shared__ double scratch[kWarps * 6];
  const EnsInstance<T> &d = inst[blk_inst[blockIdx.x]];
  blk_telemetry(d, static_cast<int>(blockIdx.x) - d.blk_begin, partials, scratch);
}

// One CTA per instance.
template <typename T>
__global__ void __launch_bounds__(kBlock)
    kb_telemetry_finalize(const EnsInstance<T> *inst, const double *partials,
                          const int *step_counter, double *tel_out,
                          const SolveReport *rep_cur, SolveReport *reports, int count,
                          int capacity) {
  __shared__ double scratch[kWarps * 6];
  const int m = blockIdx.x;
  ens_finalize(inst[m], m, partials, *step_counter, tel_out, rep_cur, reports, count, capacity,
               scratch);
}

// ---- launchers -------------------------------------------------------------
template <typename T>
void ens_advect(const EnsLaunch<T> &L, int f, double diss, cudaStream_t st) {
  kb_advect_fwd<T><<<L.blocks, kTx * kTy, 0, st>>>(L.inst, L.blk_inst, f);
  kb_advect_mc<T><<<L.blocks, kTx * kTy, 0, st>>>(L.inst, L.blk_inst, f, diss);
  kb_swap<T><<<(L.count + 127) / 128, 128, 0, st>>>(L.inst, L.count, f);
}

template <typename T>
void ens_forces(const EnsLaunch<T> &L, cudaStream_t st) {
  kb_curl<T><<<L.blocks, kTx * kTy, 0, st>>>(L.inst, L.blk_inst);
  kb_source_confine_buoy<T><<<L.blocks, kTx * kTy, 0, st>>>(L.inst, L.blk_inst);
}

template <typename T>
void ens_divergence(const EnsLaunch<T> &L, cudaStream_t st) {
  kb_divergence<T><<<L.blocks, kTx * kTy, 0, st>>>(L.inst, L.blk_inst);
}

template <typename T>
void ens_project(const EnsLaunch<T> &L, cudaStream_t st) {
  kb_project<T><<<L.blocks, kTx * kTy, 0, st>>>(L.inst, L.blk_inst);
}

template <typename T>
void ens_telemetry(const EnsLaunch<T> &L, double *partials, const int *step_counter,
                   double *tel_out, const SolveReport *rep_cur, SolveReport *reports,
                   int capacity, cudaStream_t st) {
  kb_telemetry<T><<<L.blocks, kTx * kTy, 0, st>>>(L.inst, L.blk_inst, partials);
  kb_telemetry_finalize<T><<<L.count, kBlock, 0, st>>>(L.inst, partials, step_counter, tel_out,
                                                        rep_cur, reports, L.count, capacity);
}

#define AFL_INSTANTIATE_ENSEMBLE(T)                                                        \
  template void ens_advect<T>(const EnsLaunch<T> &, int, double, cudaStream_t);            \
  template void ens_forces<T>(const EnsLaunch<T> &, cudaStream_t);                         \
  template void ens_divergence<T>(const EnsLaunch<T> &, cudaStream_t);                     \
  template void ens_project<T>(const EnsLaunch<T> &, cudaStream_t);                        \
  template void ens_telemetry<T>(const EnsLaunch<T> &, double *, const int *, double *,    \
                                 const SolveReport *, SolveReport *, int, cudaStream_t);

}  // namespace afl
