// afl_stage_fused.cuh -- the shared-memory-staged form of the forces stage,
// templated on the field type T (double: FP64 form; float: mixed form).
// Included by afl_kernels_f64.cu (built with -fmad=false) and
// afl_kernels_f32.cu.  The solver runs it on grids whose stage arrays exceed
// twice the L2 cache, where the stage streams from HBM; smaller grids keep the
// one-thread-per-cell kernels of afl_stage.cuh, which L2 serves faster.
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
// k_forces_fused: apply_buoyancy_and_vorticity_confinement
// (src/fluid.rs:256-330).  The curl and |w| of the tile plus a one-cell halo
// exist only in shared memory and registers; the new velocities go to a
// second set of arrays, because neighbouring CTAs still read the old ones.
// Each cell's arithmetic is the expression of cell_curl and
// cell_confine_buoy (afl_stage.cuh), so the FP64 results are the same bits.
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
constexpr int kRingForces = 6;  // six planes: two ahead of the stencil's reach

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

#define AFL_INSTANTIATE_FUSED(T)                                                           \
  template void launch_forces_fused<T>(const Dims &, const T *, const T *, const T *,       \
                                       const T *, const T *, T *, T *, T *, double, double, \
                                       double, double, cudaStream_t);

}  // namespace afl
