// afl_device.cuh -- device-side building blocks shared by every kernel.
//
// Layout: one scalar per cell, x fastest, idx = (k*ny + j)*nx + i, the
// reference's layout (src/fluid.rs:88-90); u/v/w share the cell index
// (src/fluid.rs:160-162, 341-343, 517-523).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace afl {

struct Dims {
  int nx, ny, nz;
  int n;       // nx*ny*nz
  int nxy;     // nx*ny
  double h;
};

constexpr int kBlock = 256;          // threads per CTA of the flat kernels
constexpr int kWarps = kBlock / 32;

__host__ __device__ inline bool interior(const Dims &g, int i, int j, int k) {
  return i >= 1 && i <= g.nx - 2 && j >= 1 && j <= g.ny - 2 && k >= 1 && k <= g.nz - 2;
}

__device__ inline void decode(const Dims &g, int c, int &i, int &j, int &k) {
  k = c / g.nxy;
  const int r = c - k * g.nxy;
  j = r / g.nx;
  i = r - j * g.nx;
}

// f64::clamp / f32::clamp: "if x < lo {lo}; if x > hi {hi}".
template <typename T>
__device__ __forceinline__ T rs_clamp(T x, T lo, T hi) {
  x = x < lo ? lo : x;
  x = x > hi ? hi : x;
  return x;
}

// Wall masks of enforce_wall_velocity_bc (src/fluid.rs:241-249): true where
// the component is forced to zero.
__device__ __forceinline__ bool wall_u(const Dims &g, int i, int j, int k) {
  return i <= 1 || i + 1 >= g.nx || j == 0 || j + 1 >= g.ny || k == 0 || k + 1 >= g.nz;
}
__device__ __forceinline__ bool wall_v(const Dims &g, int i, int j, int k) {
  return j <= 1 || j + 1 >= g.ny || i == 0 || i + 1 >= g.nx || k == 0 || k + 1 >= g.nz;
}
__device__ __forceinline__ bool wall_w(const Dims &g, int i, int j, int k) {
  return k <= 1 || k + 1 >= g.nz || i == 0 || i + 1 >= g.nx || j == 0 || j + 1 >= g.ny;
}

// Corner cell and weights of the clamped trilinear footprint
// (src/fluid.rs:95-108).
template <typename T>
struct Footprint {
  int base;  // idx(i0, j0, k0)
  T tx, ty, tz;
};

// The same footprint with the corner as three indices (the fused stage
// kernels test whether it lies inside their shared-memory tile).
// floor(x) as a cell index.  A NaN position (a field that has blown up)
// gives cell 0, as the reference's `as usize` does, instead of an index that
// the float-to-int conversion leaves undefined.
template <typename T>
__device__ __forceinline__ int floor_index(T x) {
  return x == x ? static_cast<int>(floor(x)) : 0;
}

template <typename T>
struct Footprint3 {
  int i, j, k;  // corner (i0, j0, k0)
  T tx, ty, tz;
  __device__ __forceinline__ int base(const Dims &g) const { return (k * g.ny + j) * g.nx + i; }
};

template <typename T>
__device__ __forceinline__ Footprint3<T> footprint3(const Dims &g, T x, T y, T z) {
  const T xc = rs_clamp(x, T(0.5), T(g.nx) - T(1.500001));
  const T yc = rs_clamp(y, T(0.5), T(g.ny) - T(1.500001));
  const T zc = rs_clamp(z, T(0.5), T(g.nz) - T(1.500001));
  Footprint3<T> f;
  f.i = floor_index(xc);
  f.j = floor_index(yc);
  f.k = floor_index(zc);
  f.tx = xc - T(f.i);
  f.ty = yc - T(f.j);
  f.tz = zc - T(f.k);
  return f;
}

template <typename T>
__device__ __forceinline__ Footprint<T> footprint(const Dims &g, T x, T y, T z) {
  const Footprint3<T> f3 = footprint3(g, x, y, z);
  Footprint<T> f;
  f.base = f3.base(g);
  f.tx = f3.tx;
  f.ty = f3.ty;
  f.tz = f3.tz;
  return f;
}

// The interior cells of one red-black colour ((i + j + k) & 1 == color) by a
// flat index q: rows (j, k) of the interior and, in each row, every second x
// from the row's first interior cell of that colour.  `half` slots per row
// cover the longer of the two parities; a slot past the row's last cell of the
// colour is skipped.
struct ColorWalk {
  int half, rows_y, total;
  __device__ explicit ColorWalk(const Dims &g)
      : half((g.nx - 1) / 2), rows_y(g.ny - 2), total(((g.nx - 1) / 2) * (g.ny - 2) * (g.nz - 2)) {}
  __device__ __forceinline__ bool cell(const Dims &g, int q, int color, int &i, int &j,
                                       int &k) const {
    const int row = q / half;
    const int m = q - row * half;
    const int kk = row / rows_y;
    j = 1 + (row - kk * rows_y);
    k = 1 + kk;
    i = 1 + 2 * m + ((1 + j + k + color) & 1);
    return i <= g.nx - 2;
  }
};

// The footprint of the point (i, j, k) - (dx, dy, dz), a cell index moved by a
// displacement.  In f64 this is footprint() of the moved position, the
// reference's own expression (src/fluid.rs:160-162), bit for bit.
template <typename T>
__device__ __forceinline__ Footprint3<T> footprint3_at(const Dims &g, int i, int j, int k, T dx,
                                                       T dy, T dz) {
  return footprint3(g, T(i) - dx, T(j) - dy, T(k) - dz);
}

// In f32 the moved position i - d, formed as one number near i, keeps only
// ~1e-5 cell of the displacement at i ~ 100 (a relative error of 1e-3 in a
// 0.005-cell step of the smoke).  Unclamped, the corner and weight follow from
// the displacement alone: floor(i - d) = i + floor(-d) and the weight is
// -d - floor(-d), both at the displacement's own precision.  The clamp test
// still uses the moved position; near the clamp bounds the two agree to a few
// ulps, which keeps the corner inside [0, n-2].
__device__ __forceinline__ void axis_at(int i, int n, float d, int &i0, float &t) {
  const float p = float(i) - d;
  const float hi = float(n) - 1.500001f;
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

template <>
__device__ __forceinline__ Footprint3<float> footprint3_at<float>(const Dims &g, int i, int j,
                                                                  int k, float dx, float dy,
                                                                  float dz) {
  Footprint3<float> f;
  axis_at(i, g.nx, dx, f.i, f.tx);
  axis_at(j, g.ny, dy, f.j, f.ty);
  axis_at(k, g.nz, dz, f.k, f.tz);
  return f;
}

template <typename T>
__device__ __forceinline__ Footprint<T> footprint_at(const Dims &g, int i, int j, int k, T dx,
                                                     T dy, T dz) {
  const Footprint3<T> f3 = footprint3_at(g, i, j, k, dx, dy, dz);
  Footprint<T> f;
  f.base = f3.base(g);
  f.tx = f3.tx;
  f.ty = f3.ty;
  f.tz = f3.tz;
  return f;
}

// Rng::from_seed / next_u64 / next_f64 (src/rng.rs:20-88): SplitMix64 of the
// seed xor a constant fills the four Xoshiro256++ words; next_f64 keeps the top
// 53 bits.  Integer work, identical on host and device.
struct XoshiroRng {
  unsigned long long s[4];
  __host__ __device__ static unsigned long long rotl(unsigned long long x, int k) {
    return (x << k) | (x >> (64 - k));
  }
  __host__ __device__ explicit XoshiroRng(unsigned long long seed) {
    unsigned long long sm = seed ^ 0xA5A55A5AF0F00F0Full;
    for (int a = 0; a < 4; ++a) {
      sm += 0x9E3779B97F4A7C15ull;
      unsigned long long z = sm;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      s[a] = z ^ (z >> 31);
    }
    if ((s[0] | s[1] | s[2] | s[3]) == 0) s[0] = 1;
  }
  __host__ __device__ unsigned long long next_u64() {
    const unsigned long long out = rotl(s[0] + s[3], 23) + s[0];
    const unsigned long long t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return out;
  }
  __host__ __device__ double next_f64() {
    return static_cast<double>(next_u64() >> 11) * (1.0 / 9007199254740992.0);
  }
};

// sample_trilinear (src/fluid.rs:110-127): x-lerps, then y, then z, each as
// a*(1-t) + b*t.  lerp8 takes the 8 corner values; trilinear loads them.
template <typename T>
__device__ __forceinline__ T lerp8(T c000, T c100, T c010, T c110, T c001, T c101, T c011,
                                   T c111, T tx, T ty, T tz) {
  const T ox = T(1) - tx, oy = T(1) - ty, oz = T(1) - tz;
  const T c00 = c000 * ox + c100 * tx;
  const T c10 = c010 * ox + c110 * tx;
  const T c01 = c001 * ox + c101 * tx;
  const T c11 = c011 * ox + c111 * tx;
  const T c0 = c00 * oy + c10 * ty;
  const T c1 = c01 * oy + c11 * ty;
  return c0 * oz + c1 * tz;
}

template <typename T>
__device__ __forceinline__ T trilinear(const T *__restrict__ f, const Dims &g,
                                       const Footprint<T> &p) {
  const int b = p.base, sx = 1, sy = g.nx, sz = g.nxy;
  const T c000 = __ldg(f + b), c100 = __ldg(f + b + sx);
  const T c010 = __ldg(f + b + sy), c110 = __ldg(f + b + sy + sx);
  const T c001 = __ldg(f + b + sz), c101 = __ldg(f + b + sz + sx);
  const T c011 = __ldg(f + b + sz + sy), c111 = __ldg(f + b + sz + sy + sx);
  return lerp8(c000, c100, c010, c110, c001, c101, c011, c111, p.tx, p.ty, p.tz);
}

// stencil_minmax (src/fluid.rs:131-150): same 8 corners, fmin/fmax keep the
// non-NaN operand like f64::min/max.
template <typename T>
__device__ __forceinline__ void minmax8(const T *__restrict__ f, const Dims &g,
                                        int base, T &lo, T &hi) {
  const int sy = g.nx, sz = g.nxy;
  lo = T(INFINITY);
  hi = T(-INFINITY);
#pragma unroll
  for (int dk = 0; dk <= 1; ++dk)
#pragma unroll
    for (int dj = 0; dj <= 1; ++dj)
#pragma unroll
      for (int di = 0; di <= 1; ++di) {
        const T v = __ldg(f + base + dk * sz + dj * sy + di);
        lo = fmin(lo, v);
        hi = fmax(hi, v);
      }
}

// ---- deterministic reductions ---------------------------------------------
// Butterfly inside the warp, then the warp sums in warp order: the result is a
// pure function of the per-thread inputs, so every CTA that reduces the same
// data gets the same bits.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Sums NV values across the CTA; the result is valid in every thread.
// `scratch` needs kWarps*NV doubles.  Ends with a __syncthreads.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < NV; ++a) v[a] = warp_sum(v[a]);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int a = 0; a < NV; ++a) scratch[warp * NV + a] = v[a];
  __syncthreads();
#pragma unroll
  for (int a = 0; a < NV; ++a) {
    double s = 0.0;
    for (int w = 0; w < kWarps; ++w) s += scratch[w * NV + a];
    v[a] = s;
  }
  __syncthreads();
}

__device__ __forceinline__ double block_max(double v, double *scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double m = scratch[0];
  for (int w = 1; w < kWarps; ++w) m = fmax(m, scratch[w]);
  __syncthreads();
  return m;
}

// Sums NV interleaved partials (parts[b*NV + a], b < nparts) in a fixed order;
// every CTA calling this on the same data gets identical results.
template <int NV>
__device__ __forceinline__ void reduce_partials(const double *parts, int nparts,
                                                double (&out)[NV], double *scratch) {
#pragma unroll
  for (int a = 0; a < NV; ++a) out[a] = 0.0;
  for (int b = threadIdx.x; b < nparts; b += blockDim.x)
#pragma unroll
    for (int a = 0; a < NV; ++a) out[a] += __ldcg(parts + b * NV + a);
  block_sum<NV>(out, scratch);
}

// ---- bounded grid barrier for the persistent (cooperative) kernels ---------
// Sense-reversing barrier over `nblocks` co-resident CTAs.  The wait is
// bounded by `timeout_ns` of %globaltimer; a CTA that gives up, or that sees
// another CTA's abort, returns false and the kernel unwinds.  No wait in this
// library is unbounded.
struct GridSync {
  unsigned int *count;   // arrivals in the current generation
  unsigned int *gen;     // generation number
  int *abort_flag;       // set to a non-zero code by the first CTA to give up
  unsigned int nblocks;
  unsigned long long timeout_ns;
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int ld_relaxed_i32(const int *p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(unsigned int *p, unsigned int v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned int atom_add_release(unsigned int *p, unsigned int v) {
  unsigned int old;
  asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;"
               : "=r"(old)
               : "l"(p), "r"(v)
               : "memory");
  return old;
}

// Returns true when every CTA arrived; false on timeout/abort (code 1 =
// timeout is recorded in abort_flag).  Arrival is a release atomic and the
// wait an acquire load, so writes made before the barrier by any CTA are
// visible to every CTA after it; the abort flag and the clock are polled every
// 256 spins (measured on B200: ~2.0 us per barrier over 128-592 CTAs).
__device__ inline bool grid_sync(const GridSync &gs) {
  __shared__ int ok_shared;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned int g0 = ld_acquire(gs.gen);
    const unsigned int arrived = atom_add_release(gs.count, 1u);
    if (arrived == gs.nblocks - 1) {
      *gs.count = 0;
      st_release(gs.gen, g0 + 1u);
    } else {
      const unsigned long long t0 = global_ns();
      unsigned int spins = 0;
      while (ld_acquire(gs.gen) == g0) {
        if ((spins++ & 255u) == 0u) {
          if (ld_relaxed_i32(gs.abort_flag) != 0) { ok = 0; break; }
          // a limit of 0 means: give up at the first wait
          if (gs.timeout_ns == 0 || global_ns() - t0 > gs.timeout_ns) {
            atomicCAS(gs.abort_flag, 0, 1);
            ok = 0;
            break;
          }
        }
      }
    }
    // Plain (L1-cached) loads after the barrier must see the other CTAs'
    // writes: order them after the acquire at GPU scope.
    __threadfence();
    ok_shared = ok;
  }
  __syncthreads();
  return ok_shared != 0;
}

}  // namespace afl
