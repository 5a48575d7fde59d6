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

// ---- tagged partials: the grid-wide sums without a central barrier ---------
// Every grid-wide sum of the solve is "each CTA contributes its partial, every
// CTA needs the fixed-order total".  Instead of a counter barrier followed by
// a read of the partials, each CTA stores its partial as two 64-bit words,
// each carrying the number of the sum in its upper half and one half of the
// double in its lower half (aligned 64-bit stores are single-copy atomic).
// A reader polls a CTA's two words until both carry the expected number, so
// arrival and data come in one L2 round trip and no CTA waits on an atomic.
// Sum number k uses buffer k & 1: a CTA can publish sum k+1 only after it has
// read all of sum k, and sum k+2 only after every CTA published k+1, so a
// buffer is never rewritten while a CTA may still read it.  Tags start at 1;
// the slots are zeroed before each launch.
constexpr int kMaxNV = 4;

struct TagSync {
  unsigned long long *slots;  // 2 buffers x nblocks x 2*kMaxNV words
  int nblocks;
};

__device__ __forceinline__ void st_relaxed_u64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long *tag_slot(const TagSync &ts, unsigned int tag,
                                                       int block) {
  return ts.slots + (static_cast<size_t>(tag & 1u) * ts.nblocks + block) * (2 * kMaxNV);
}

// Sums NV values over the CTA (warp butterflies, then warp 0 over the 32 warp
// sums: a fixed order) and publishes the CTA's partials as sum number `tag`.
// Writes made by any thread of the CTA before the call are released with it.
template <int NV>
__device__ __forceinline__ void tag_publish(const TagSync &ts, unsigned int tag,
                                            double (&v)[NV], double *scratch) {
  static_assert(NV <= kMaxNV, "too many values");
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < NV; ++a) v[a] = warp_sum(v[a]);
  if (lane == 0)
#pragma unroll
    for (int a = 0; a < NV; ++a) scratch[warp * NV + a] = v[a];
  __syncthreads();
  if (warp == 0) {
    double x[NV];
#pragma unroll
    for (int a = 0; a < NV; ++a) x[a] = warp_sum(scratch[lane * NV + a]);
    if (lane == 0) {
      unsigned long long *dst = tag_slot(ts, tag, blockIdx.x);
      const unsigned long long hi_tag = static_cast<unsigned long long>(tag) << 32;
      __threadfence();  // release: the CTA's writes before the sum (fence + relaxed stores)
#pragma unroll
      for (int a = 0; a < NV; ++a) {
        const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(x[a]));
        st_relaxed_u64(dst + 2 * a, hi_tag | (bits & 0xffffffffull));
        st_relaxed_u64(dst + 2 * a + 1, hi_tag | (bits >> 32));
      }
    }
  }
}

// The fixed-order total of sum number `tag` over all CTAs, in every thread.
// Thread b waits for CTA b's words (relaxed loads; an acquire load after the
// wait makes it an acquire of what CTA b released) and parks the value in shared
// `vals`; then warp 0 lane l adds CTAs l, l+32, ... in that order and a
// butterfly combines the lanes, so every CTA computes the same bits.  Waits
// are bounded like grid_sync's (abort flag and clock polled every 256 spins; a
// limit of 0 gives up at the first wait).  Returns false when a wait gave up;
// the abort flag then holds the reason.
constexpr int kMaxTagBlocks = 160;  // >= the SM count: one CTA per SM

template <int NV>
__device__ __forceinline__ bool tag_gather(const TagSync &ts, const GridSync &gs, unsigned int tag,
                                           double (&out)[NV], double *slot, double *vals) {
  int ok = 1;
  const int b = threadIdx.x;
  if (b < ts.nblocks) {
    const unsigned long long *src = tag_slot(ts, tag, b);
    unsigned long long w[2 * NV];
    unsigned int spins = 0;
    const unsigned long long t0 = global_ns();
    for (;;) {
      bool ready = true;
#pragma unroll
      for (int x = 0; x < 2 * NV; ++x) {
        w[x] = ld_relaxed_u64(src + x);
        ready &= static_cast<unsigned int>(w[x] >> 32) == tag;
      }
      if (ready) break;
      if ((spins++ & 255u) == 0u) {
        if (ld_relaxed_i32(gs.abort_flag) != 0) { ok = 0; break; }
        if (gs.timeout_ns == 0 || global_ns() - t0 > gs.timeout_ns) {
          atomicCAS(gs.abort_flag, 0, 1);
          ok = 0;
          break;
        }
      }
    }
#pragma unroll
    for (int a = 0; a < NV; ++a)
      vals[b * NV + a] = __longlong_as_double(
          static_cast<long long>((w[2 * a + 1] << 32) | (w[2 * a] & 0xffffffffull)));
    // acquire: loads after the sum (halo values of other CTAs) must see the
    // writes released with it.  An acquire load of a word already seen with
    // this tag synchronises with CTA b's release without the full fence,
    // which would also wait for this thread's own outstanding stores.
    {
      unsigned long long t;
      asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(t) : "l"(src) : "memory");
    }
  }
  ok = __syncthreads_and(ok);
  if (threadIdx.x < 32) {
    double acc[NV];
#pragma unroll
    for (int a = 0; a < NV; ++a) acc[a] = 0.0;
    for (int bb = threadIdx.x; bb < ts.nblocks; bb += 32)
#pragma unroll
      for (int a = 0; a < NV; ++a) acc[a] += vals[bb * NV + a];
#pragma unroll
    for (int a = 0; a < NV; ++a) {
      acc[a] = warp_sum(acc[a]);
      if (threadIdx.x == 0) slot[a] = acc[a];
    }
  }
  __syncthreads();
#pragma unroll
  for (int a = 0; a < NV; ++a) out[a] = slot[a];
  return ok != 0;
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

// The reference operator (src/fluid.rs:356-394) on the thread's column of
// CPT cells, marching up in z with the z neighbours in registers.  No
// branches or selects: a neighbour the reference skips is a cell outside the
// interior, where the direction is exactly 0 (r = b - A p = 0 on every
// non-interior cell, and d = r + beta*d keeps it 0), so adding it leaves the
// neighbour sum's value unchanged; the sum keeps the reference's order
// (x-, x+, y-, y+, z-, z+).  The diagonal is the count of interior
// neighbours.  Only interior cells keep the result; their neighbours all lie
// in the grid, so slots that hold no grid cell (halo outside the grid,
// padding planes) never reach a kept result.
// use(m, s, d_m, (A d)_m) is called for every cell of the column.
template <typename R, int SX, int SXY, int CPT, typename Cl, typename F>
__device__ __forceinline__ void lap_column(const Dims &g, const R *D, const Cl &cl, F &&use) {
  int s = cl.s0;
  R below = D[s - SXY];
  R mid = D[s];
#pragma unroll
  for (int m = 0; m < CPT; ++m) {
    const R above = D[s + SXY];
    const int k = cl.k0 + m;
    const int diag = cl.diag_xy + int(k > 1) + int(k + 2 < g.nz);
    R nb = D[s - 1];
    nb += D[s + 1];
    nb += D[s - SX];
    nb += D[s + SX];
    nb += below;
    nb += above;
    use(m, s, mid, R(diag) * mid - nb);
    below = mid;
    mid = above;
    s += SXY;
  }
}

// The FP64 kernel's form of the same operator, one cell at a time with the
// reference's neighbour tests as selects: its 16 f64 residuals per thread
// leave too few registers for the column march above.
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
  int par;  // (i + j) & 1 of the ring column: a ring cell's colour is (par + k) & 1
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
    par = (i + j) & 1;
    col_c = j * g.nx + i;
    col_s = (jj + 1) * SX + ii + 1;
  }
  // D[ring cell] = value_at(global cell, D[ring cell]) for every plane.  The
  // trip count is a constant (the planes the tile covers), so every L2 load of
  // the ring is issued before the first use.
  // The FP64 kernel's form: a rolled loop (its registers are taken by the
  // f64 residuals).
  template <typename R, typename F>
  __device__ __forceinline__ void fill_rolled(const Dims &g, R *D, const F &value_at) const {
    constexpr int SXY = Plane<TY>::SXY;
    if (!active) return;
#pragma unroll 4
    for (int k = k_first; k < g.nz; k += kLanes) {
      R &slot = D[k * SXY + col_s];
      slot = value_at(k * g.nxy + col_c, slot);
    }
  }
  // The red-black form: only ring cells of one colour ((i + j + k) & 1).
  template <typename R, typename F>
  __device__ __forceinline__ void fill_color(const Dims &g, R *D, int color,
                                             const F &value_at) const {
    constexpr int SXY = Plane<TY>::SXY;
    if (!active) return;
#pragma unroll 4
    for (int k = k_first; k < g.nz; k += kLanes) {
      if (((par + k) & 1) != color) continue;
      R &slot = D[k * SXY + col_s];
      slot = value_at(k * g.nxy + col_c, slot);
    }
  }
  template <int kTrips, typename R, typename F>
  __device__ __forceinline__ void fill(const Dims &g, R *D, const F &value_at) const {
    constexpr int SXY = Plane<TY>::SXY;
    if (!active) return;
#pragma unroll
    for (int t = 0; t < kTrips; ++t) {
      const int k = k_first + t * kLanes;
      if (k < g.nz) {
        R &slot = D[k * SXY + col_s];
        slot = value_at(k * g.nxy + col_c, slot);
      }
    }
  }
};


// Shared scratch of the reductions: per-warp values, the CTA result, and the
// broadcast slot of the grid-wide sums.
constexpr int kScratch = kRW * kMaxNV + 2 * kMaxNV;
constexpr int kScratchSlot = kRW * kMaxNV + kMaxNV;  // broadcast slot of the grid sums

// ---- tensor memory as per-thread storage -----------------------------------
// The FP64 kernel keeps two of its per-cell vectors in the SM's tensor memory
// (TMEM: 128 lanes x 512 columns of 32 bits, 256 KB beside the register file
// and shared memory).  With 1024 threads, warp w reaches lanes 32*(w%4) ..
// +31 and owns 64 columns of them: 32 doubles per thread.  No tensor-core
// instruction runs; 32x32b loads and stores move a thread's own columns
// between TMEM and its registers.  The CTA allocates all 512 columns (one CTA
// per SM) and frees them on every exit path.
constexpr unsigned kTmCols = 512;

__device__ __forceinline__ void tm_alloc_all(unsigned *dst_smem) {  // one whole warp
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(dst_smem));
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sa),
               "r"(kTmCols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tm_dealloc_all(unsigned taddr) {  // the allocating warp
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr),
               "r"(kTmCols)
               : "memory");
}
__device__ __forceinline__ void tm_sync_threads() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// 4 doubles (8 columns) of this thread's lane at column address taddr; the
// load waits for its data inside the same statement, the store for its
// completion, so no register is used before it is valid or reused early.
__device__ __forceinline__ void tm_ld4(unsigned taddr, double (&v)[4]) {
  unsigned x0, x1, x2, x3, x4, x5, x6, x7;
  __syncwarp();  // the .sync.aligned forms need the whole warp converged
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(x0), "=r"(x1), "=r"(x2), "=r"(x3), "=r"(x4), "=r"(x5), "=r"(x6), "=r"(x7)
      : "r"(taddr)
      : "memory");
  v[0] = __hiloint2double(static_cast<int>(x1), static_cast<int>(x0));
  v[1] = __hiloint2double(static_cast<int>(x3), static_cast<int>(x2));
  v[2] = __hiloint2double(static_cast<int>(x5), static_cast<int>(x4));
  v[3] = __hiloint2double(static_cast<int>(x7), static_cast<int>(x6));
}
__device__ __forceinline__ void tm_st4(unsigned taddr, const double (&v)[4]) {
  __syncwarp();
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};\n"
      "tcgen05.wait::st.sync.aligned;\n" ::"r"(taddr),
      "r"(__double2loint(v[0])), "r"(__double2hiint(v[0])), "r"(__double2loint(v[1])),
      "r"(__double2hiint(v[1])), "r"(__double2loint(v[2])), "r"(__double2hiint(v[2])),
      "r"(__double2loint(v[3])), "r"(__double2hiint(v[3]))
      : "memory");
}

// ---------------------------------------------------------------- FP64 ------
// solve_poisson_conjugate_gradient (src/fluid.rs:445-493) with the relative
// tolerance extension, one grid-wide sum per iteration.
//  * d lives in shared memory (tile + halo ring); the residual r and the
//    pressure p live in tensor memory (TMEM); q = A d goes to global memory
//    (L2) with r as a (r, q) pair by iteration parity, where the neighbours
//    also read the tile-edge pairs.  With r and p off the register file the
//    kernel does not spill.
//  * One sum carries d.q, r.q, q.q and the r.r of the current residual.
//    alpha = delta/(d.q) takes the true delta = r.r; the next r.r, which the
//    reference sums after r -= alpha q, is the same number expanded,
//    delta - 2 alpha r.q + alpha^2 q.q, and gives beta = delta'/delta
//    (src/fluid.rs:482) without a second sum.  The stopping tests after an
//    update (:479, relative tolerance) read the true r.r, which arrives with
//    the next iteration's sum: the test runs there, before any further update,
//    so the iterations done and the stopping iteration are the reference's.
//  * The halo ring of d' = (r - alpha q) + beta d is rebuilt from the
//    neighbours' published (r, q) pairs (written before the sum) with the
//    owner's expression, bit for bit.  The pairs are kept by iteration parity.
//  * The stencil marches up each thread's column with the z neighbours in
//    registers and no selects (d is exactly 0 off the interior).
// The arguments are __grid_constant__: they stay in the constant bank.
template <int TY, int CPT>
__device__ __forceinline__ void cg_f64_body(const ResidentCgArgs &a, const GridSync &gs,
                                            const TagSync &ts, double *D, double *scratch,
                                            double *slot, double *vals, unsigned t_r,
                                            unsigned t_p) {
  using C = Cells<TY, CPT>;
  constexpr int NCH = (CPT + 3) / 4;  // chunks of 4 doubles in TMEM
  const Dims g = a.g;
  const C cl(g, a.tiles_x);
  const Halo<TY> halo(g, a.tiles_x);
  double *p = a.p;
  // (r, q) of every cell by iteration parity: the stencil pass publishes the
  // pair once (one 16-byte store), the update reloads its own q from it and
  // the ring rebuild reads both halves with one load
  double2 *const pr0 = static_cast<double2 *>(a.rpub);
  double2 *const pr1 = pr0 + g.n;
  int phase = 0;
  {
    // r = b - A p (src/fluid.rs:455-458) and p into TMEM, d = r.  The chunk
    // loops stay rolled: unrolled over 16 cells they spill.
    double acc[2] = {0.0, 0.0};
#pragma unroll 1
    for (int ch = 0; ch < NCH; ++ch) {
      double rv4[4] = {0.0, 0.0, 0.0, 0.0}, pv4[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int m = ch * 4 + q;
        if (m >= CPT) break;
        if (cl.valid(g, m)) {
          const int c = cl.c0 + m * g.nxy;
          const double ap = cl.interior(g, m) ? lap_global(g, p, c, cl.i, cl.j, cl.k0 + m) : 0.0;
          const double bc = __ldg(a.b + c);
          const double rv = bc - ap;
          rv4[q] = rv;
          pv4[q] = __ldcg(p + c);
          if (cl.edge) pr0[c].x = rv;
          acc[0] += rv * rv;
          acc[1] += bc * bc;
        }
        D[cl.s0 + m * C::SXY] = rv4[q];
      }
      tm_st4(t_r + 8u * ch, rv4);
      tm_st4(t_p + 8u * ch, pv4);
    }
    tag_publish<2>(ts, unsigned(phase + 1), acc, scratch);
  }
  double tot[2];
  if (!tag_gather<2>(ts, gs, unsigned(phase + 1), tot, slot, vals)) return;
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
  if (!(delta > 1e-24) || (tol2 >= 0.0 && delta <= tol2)) {  // src/fluid.rs:462
    converged = isfinite(delta) ? 1 : 0;
  } else {
    // the first direction on the halo ring: the neighbours' r
    halo.fill_rolled(g, D, [&](int c, double) { return __ldcg(&pr0[c].x); });
    __syncthreads();
    double rr_next = 0.0;
    for (;;) {
      const bool odd = (it & 1) != 0;
      double2 *const pw = odd ? pr1 : pr0;
      // q = A d (src/fluid.rs:465) marching up the column (the z neighbours in
      // registers, the neighbour sum in the reference's order x-, x+, y-, y+,
      // z-, z+, no selects); d.q, r.q, q.q; this residual's r.r
      double acc[4] = {0.0, 0.0, 0.0, rr_next};
      {
        int s = cl.s0;
        double below = D[s - C::SXY];
        double mid = D[s];
#pragma unroll 1
        for (int ch = 0; ch < NCH; ++ch) {
          double rc[4];
          tm_ld4(t_r + 8u * ch, rc);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int m = ch * 4 + q;
            if (m >= CPT) break;
            const double above = D[s + C::SXY];
            const int k = cl.k0 + m;
            const int diag = cl.diag_xy + int(k > 1) + int(k + 2 < g.nz);
            double nb = D[s - 1];
            nb += D[s + 1];
            nb += D[s - C::SX];
            nb += D[s + C::SX];
            nb += below;
            nb += above;
            const double qk = cl.interior(g, m) ? double(diag) * mid - nb : 0.0;
            acc[0] += mid * qk;
            acc[1] += rc[q] * qk;
            acc[2] += qk * qk;
            if (cl.valid(g, m)) pw[cl.c0 + m * g.nxy] = make_double2(rc[q], qk);
            below = mid;
            mid = above;
            s += C::SXY;
          }
        }
      }
      tag_publish<4>(ts, unsigned(phase + 1), acc, scratch);
      double sum[4];
      if (!tag_gather<4>(ts, gs, unsigned(phase + 1), sum, slot, vals)) return;
      ++phase;
      if (it > 0) {  // the tests after the previous update (src/fluid.rs:478-481)
        last = sum[3];
        if (!isfinite(last)) break;
        if (last < 1e-20) { converged = 1; break; }
        if (tol2 >= 0.0 && last <= tol2) { converged = 1; break; }
        delta = last;
      }
      if (it >= a.max_iters) break;
      if (fabs(sum[0]) < 1e-28) break;  // src/fluid.rs:469
      const double alpha = delta / sum[0];
      const double dnext = delta - 2.0 * alpha * sum[1] + alpha * alpha * sum[2];
      const double beta = dnext / delta;
      // p += alpha d, r -= alpha q, d = r + beta d (src/fluid.rs:472-485)
      rr_next = 0.0;
      // r and q of a chunk come from this thread's published pairs in L2 (r
      // as in TMEM, bit for bit); the next chunk's loads are issued after this
      // chunk's TMEM stores, when its registers are free, so their latency
      // overlaps the next TMEM load (holding them longer spills)
      double2 qn[4];
#pragma unroll
      for (int q = 0; q < 4; ++q)
        qn[q] = (q < CPT && cl.valid(g, q)) ? __ldcg(&pw[cl.c0 + q * g.nxy]) : make_double2(0.0, 0.0);
#pragma unroll 1
      for (int ch = 0; ch < NCH; ++ch) {
        double rv4[4], pv4[4], qv4[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) { rv4[q] = qn[q].x; qv4[q] = qn[q].y; }
        tm_ld4(t_p + 8u * ch, pv4);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int m = ch * 4 + q;
          if (m >= CPT) continue;
          const int s = cl.s0 + m * C::SXY;
          const double dv = D[s];
          pv4[q] = pv4[q] + alpha * dv;
          const double rv = rv4[q] - alpha * qv4[q];
          rv4[q] = rv;
          D[s] = rv + beta * dv;
          rr_next += rv * rv;
        }
        tm_st4(t_r + 8u * ch, rv4);
        tm_st4(t_p + 8u * ch, pv4);
        if (ch + 1 < NCH) {
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int m = (ch + 1) * 4 + q;
            qn[q] = (m < CPT && cl.valid(g, m)) ? __ldcg(&pw[cl.c0 + m * g.nxy]) : make_double2(0.0, 0.0);
          }
        }
      }

      halo.fill_rolled(g, D, [&](int c, double dprev) {
        const double2 v = __ldcg(pw + c);
        const double rv = v.x - alpha * v.y;
        return rv + beta * dprev;
      });
      __syncthreads();
      ++it;
    }
  }
  // the pressure back to global memory
#pragma unroll 1
  for (int ch = 0; ch < NCH; ++ch) {
    double pv4[4];
    tm_ld4(t_p + 8u * ch, pv4);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int m = ch * 4 + q;
      if (m < CPT && cl.valid(g, m)) p[cl.c0 + m * g.nxy] = pv4[q];
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

template <int TY, int CPT>
__global__ void __launch_bounds__(kRT, 1)
    k_cg_res_f64(const __grid_constant__ ResidentCgArgs a, const __grid_constant__ GridSync gs,
                 const __grid_constant__ TagSync ts) {
  using C = Cells<TY, CPT>;
  extern __shared__ double Dbase[];
  __shared__ double scratch[kScratch];
  __shared__ double vals[kMaxTagBlocks * kMaxNV];
  __shared__ unsigned tm_base;
  const int warp = threadIdx.x >> 5;
  if (warp == 0) tm_alloc_all(&tm_base);
  tm_sync_threads();
  // this thread's 64 columns: r in the first 32, p in the next 32
  const unsigned t_r = tm_base + ((32u * unsigned(warp & 3)) << 16) + 64u * unsigned(warp >> 2);
  cg_f64_body<TY, CPT>(a, gs, ts, Dbase + C::SXY, scratch, scratch + kScratchSlot, vals, t_r,
                       t_r + 32u);
  tm_sync_threads();  // every TMEM access of the CTA is complete
  if (warp == 0) tm_dealloc_all(tm_base);
}

// ---------------------------------------------------------------- mixed -----
// f64 refinement around an f32 CG whose vectors never leave the SM: d and
// q = A d in shared memory (same tile layout), r and the correction e in
// registers.  q is stored by the first pass of an iteration and read by the
// second, so the stencil runs once per iteration.
template <int TY, int CPT>
__global__ void __launch_bounds__(kRT, 1)
    k_cg_res_mixed(ResidentCgArgs a, GridSync gs, TagSync ts) {
  using C = Cells<TY, CPT>;
  constexpr int kRingTrips = (C::kPlanes + Halo<TY>::kLanes - 1) / Halo<TY>::kLanes;
  extern __shared__ float Dfbase[];
  float *Df = Dfbase + C::SXY;  // one padding plane below plane 0
  __shared__ double scratch[kScratch];
  __shared__ double vals[kMaxTagBlocks * kMaxNV];
  double *slot = scratch + kScratchSlot;
  const Dims g = a.g;
  const C cl(g, a.tiles_x);
  const Halo<TY> halo(g, a.tiles_x);
  float *Q = Df + C::SXY * (C::kPlanes + 2);  // q = A d, same tile layout
  double *p = a.p;
  float *rpub = static_cast<float *>(a.rpub);
  float r[CPT], e[CPT];
  int phase = 0;

  // r = b - A p in f64, rounded once to f32; e = 0.
  auto outer_residual = [&](bool with_b) {
    double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int m = 0; m < CPT; ++m) {
      r[m] = 0.0f;
      e[m] = 0.0f;
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
    tag_publish<3>(ts, unsigned(phase + 1), acc, scratch);
  };

  outer_residual(true);
  double tot[3];
  if (!tag_gather<3>(ts, gs, unsigned(phase + 1), tot, slot, vals)) return;
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
      halo.template fill<kRingTrips>(g, Df, [&](int c, float dprev) {
        const float rv = __ldcg(rpub + c);
        return first ? rv : __fmaf_rn(bf, dprev, rv);
      });
#pragma unroll
      for (int m = 0; m < CPT; ++m) {
        const int s = cl.s0 + m * C::SXY;
        Df[s] = first ? r[m] : __fmaf_rn(bf, Df[s], r[m]);
      }
      __syncthreads();
      double acc[1] = {0.0};
      lap_column<float, C::SX, C::SXY, CPT>(g, Df, cl, [&](int m, int s, float dv, float lq) {
        const float qv = cl.interior(g, m) ? lq : 0.0f;
        Q[s] = qv;
        acc[0] += double(dv) * double(qv);
      });
      tag_publish<1>(ts, unsigned(phase + 1), acc, scratch);
      double dq[1];
      if (!tag_gather<1>(ts, gs, unsigned(phase + 1), dq, slot, vals)) return;
      ++phase;
      if (!(fabs(dq[0]) >= 1e-30)) break;
      const float af = float(delta / dq[0]);
      double acc2[1] = {0.0};
#pragma unroll
      for (int m = 0; m < CPT; ++m) {
        const int s = cl.s0 + m * C::SXY;
        const float qv = Q[s];
        e[m] = __fmaf_rn(af, Df[s], e[m]);
        const float rv = __fmaf_rn(-af, qv, r[m]);
        r[m] = rv;
        if (cl.edge && cl.valid(g, m)) rpub[cl.c0 + m * g.nxy] = rv;
        acc2[0] += double(rv) * double(rv);
      }
      tag_publish<1>(ts, unsigned(phase + 1), acc2, scratch);
      double dn[1];
      if (!tag_gather<1>(ts, gs, unsigned(phase + 1), dn, slot, vals)) return;
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
      p[c] = p[c] + double(e[m]);
    }
    if (!grid_sync(gs)) return;
    outer_residual(false);
    if (!tag_gather<3>(ts, gs, unsigned(phase + 1), tot, slot, vals)) return;
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

// ------------------------------------------------------------- RB-SOR ----
// solve_poisson_gauss_seidel (src/fluid.rs:397-442) with the tile on chip: the
// pressure (FP64) or the f32 correction (mixed) in shared memory with its halo
// ring.  A half-sweep updates the cells of one colour in place (each reads only
// the other colour), writes the tile-edge cells it changed to global memory,
// and after one grid barrier the ring cells of that colour are reloaded from
// there.  The FP64 update is the reference's expression with its neighbour
// order, so a sweep equals the reference's bit for bit.
template <typename R, int SX, int SXY, typename Cl>
__device__ __forceinline__ void sor_terms(const Dims &g, const R *P, int s, const Cl &cl, int k,
                                          R &nb, R &diag) {
  const bool zl = k > 1, zh = k + 2 < g.nz;
  nb = cl.xl ? P[s - 1] : R(0);
  nb += cl.xh ? P[s + 1] : R(0);
  nb += cl.yl ? P[s - SX] : R(0);
  nb += cl.yh ? P[s + SX] : R(0);
  nb += zl ? P[s - SXY] : R(0);
  nb += zh ? P[s + SXY] : R(0);
  diag = R(cl.diag_xy + int(zl) + int(zh));
}

template <int TY, int CPT>
__global__ void __launch_bounds__(kRT, 1) k_sor_res_f64(ResidentSorArgs a, GridSync gs) {
  using C = Cells<TY, CPT>;
  extern __shared__ double Pbase[];
  double *P = Pbase + C::SXY;  // one padding plane below plane 0
  const Dims g = a.g;
  const C cl(g, a.tiles_x);
  const Halo<TY> halo(g, a.tiles_x);
  double *p = a.p;
#pragma unroll
  for (int m = 0; m < CPT; ++m)
    P[cl.s0 + m * C::SXY] = cl.valid(g, m) ? __ldcg(p + cl.c0 + m * g.nxy) : 0.0;
  halo.fill_rolled(g, P, [&](int c, double) { return __ldcg(p + c); });
  __syncthreads();
  const double omega = a.omega;
  const int par0 = (cl.i + cl.j + cl.k0) & 1;
  for (int sweep = 0; sweep < a.sweeps; ++sweep) {
    for (int color = 0; color < 2; ++color) {
#pragma unroll
      for (int m = 0; m < CPT; ++m) {
        if (((par0 + m) & 1) != color || !cl.interior(g, m)) continue;
        const int s = cl.s0 + m * C::SXY;
        const int c = cl.c0 + m * g.nxy;
        double nb, diag;
        sor_terms<double, C::SX, C::SXY>(g, P, s, cl, cl.k0 + m, nb, diag);
        const double target = (__ldg(a.b + c) + nb) / diag;
        const double v = (1.0 - omega) * P[s] + omega * target;
        P[s] = v;
        if (cl.edge) p[c] = v;
      }
      if (!grid_sync(gs)) return;
      halo.fill_color(g, P, color, [&](int c, double) { return __ldcg(p + c); });
      __syncthreads();
    }
  }
#pragma unroll
  for (int m = 0; m < CPT; ++m)
    if (cl.valid(g, m)) p[cl.c0 + m * g.nxy] = P[cl.s0 + m * C::SXY];
  if (blockIdx.x == 0 && threadIdx.x == 0 && a.report) {
    SolveReport rep{};
    rep.iterations = a.sweeps;
    *a.report = rep;
  }
}

// Mixed RB-SOR: r = b - A p once in f64 (rounded to f32, kept in registers),
// the sweeps on the f32 correction (A e = r from e = 0, the same linear
// iteration as sweeping p), then p += e in f64.  Published edge values go
// through a.e32.
template <int TY, int CPT>
__global__ void __launch_bounds__(kRT, 1) k_sor_res_mixed(ResidentSorArgs a, GridSync gs) {
  using C = Cells<TY, CPT>;
  extern __shared__ float Ebase[];
  float *E = Ebase + C::SXY;
  const Dims g = a.g;
  const C cl(g, a.tiles_x);
  const Halo<TY> halo(g, a.tiles_x);
  double *p = a.p;
  float *epub = a.e32;
  float rb[CPT];
#pragma unroll
  for (int m = 0; m < CPT; ++m) {
    rb[m] = 0.0f;
    E[cl.s0 + m * C::SXY] = 0.0f;
    if (!cl.valid(g, m)) continue;
    const int c = cl.c0 + m * g.nxy;
    const double ap = cl.interior(g, m) ? lap_global(g, p, c, cl.i, cl.j, cl.k0 + m) : 0.0;
    rb[m] = float(__ldg(a.b + c) - ap);
  }
  halo.fill_rolled(g, E, [&](int, float) { return 0.0f; });
  __syncthreads();
  const float omega = float(a.omega);
  const int par0 = (cl.i + cl.j + cl.k0) & 1;
  for (int sweep = 0; sweep < a.sweeps; ++sweep) {
    for (int color = 0; color < 2; ++color) {
#pragma unroll
      for (int m = 0; m < CPT; ++m) {
        if (((par0 + m) & 1) != color || !cl.interior(g, m)) continue;
        const int s = cl.s0 + m * C::SXY;
        float nb, diag;
        sor_terms<float, C::SX, C::SXY>(g, E, s, cl, cl.k0 + m, nb, diag);
        const float target = (rb[m] + nb) / diag;
        const float v = (1.0f - omega) * E[s] + omega * target;
        E[s] = v;
        if (cl.edge) epub[cl.c0 + m * g.nxy] = v;
      }
      if (!grid_sync(gs)) return;
      halo.fill_color(g, E, color, [&](int c, float) { return __ldcg(epub + c); });
      __syncthreads();
    }
  }
#pragma unroll
  for (int m = 0; m < CPT; ++m) {
    if (!cl.valid(g, m)) continue;
    const int c = cl.c0 + m * g.nxy;
    p[c] = p[c] + double(E[cl.s0 + m * C::SXY]);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && a.report) {
    SolveReport rep{};
    rep.iterations = a.sweeps;
    rep.refinements = 1;
    *a.report = rep;
  }
}

// ---------------------------------------------------------------- dispatch --
using KernelFn = void (*)(ResidentCgArgs, GridSync, TagSync);

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

using SorFn = void (*)(ResidentSorArgs, GridSync);

template <int TY, int CPT>
SorFn pick_sor(bool f64) {
  return f64 ? &k_sor_res_f64<TY, CPT> : &k_sor_res_mixed<TY, CPT>;
}

SorFn sor_kernel_for(bool f64, int ty, int cpt) {
#define AFL_SOR_CASE(TY_, CPT_) \
  if (ty == TY_ && cpt == CPT_) return pick_sor<TY_, CPT_>(f64);
  AFL_SOR_CASE(4, 1) AFL_SOR_CASE(4, 2) AFL_SOR_CASE(4, 4) AFL_SOR_CASE(4, 8) AFL_SOR_CASE(4, 16)
  AFL_SOR_CASE(8, 1) AFL_SOR_CASE(8, 2) AFL_SOR_CASE(8, 4) AFL_SOR_CASE(8, 8) AFL_SOR_CASE(8, 16)
  AFL_SOR_CASE(16, 1) AFL_SOR_CASE(16, 2) AFL_SOR_CASE(16, 4) AFL_SOR_CASE(16, 8)
  AFL_SOR_CASE(16, 16)
#undef AFL_SOR_CASE
  return nullptr;
}

}  // namespace

int launch_sor_resident(const ResidentSorArgs &a, const ResidentPlan &plan, bool f64,
                        const PersistentState &ps, cudaStream_t st) {
  SorFn fn = sor_kernel_for(f64, plan.ty, plan.cpt);
  if (!fn) return -static_cast<int>(cudaErrorInvalidConfiguration);
  const int blocks = plan.tiles_x * plan.tiles_y;
  if (blocks > ps.max_blocks) return -static_cast<int>(cudaErrorInvalidConfiguration);
  // one tile of the solved quantity: f64 pressure or f32 correction
  const size_t tile = resident_smem_bytes(a.g, plan.ty, plan.cpt, true) / sizeof(double);
  const int smem = static_cast<int>(tile * (f64 ? sizeof(double) : sizeof(float)));
  cudaError_t err = cudaFuncSetAttribute(reinterpret_cast<const void *>(fn),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (err != cudaSuccess) return -static_cast<int>(err);
  cudaMemsetAsync(ps.count, 0, sizeof(unsigned int), st);
  cudaMemsetAsync(ps.gen, 0, sizeof(unsigned int), st);
  cudaMemsetAsync(ps.abort_flag, 0, sizeof(int), st);
  ResidentSorArgs args = a;
  args.tiles_x = plan.tiles_x;
  args.tiles_y = plan.tiles_y;
  GridSync gs;
  gs.count = ps.count;
  gs.gen = ps.gen;
  gs.abort_flag = ps.abort_flag;
  gs.nblocks = static_cast<unsigned int>(blocks);
  gs.timeout_ns = ps.timeout_ns;
  void *params[] = {&args, &gs};
  err = cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(fn), dim3(blocks), dim3(kRT),
                                    params, static_cast<size_t>(smem), st);
  return err == cudaSuccess ? blocks : -static_cast<int>(err);
}

size_t resident_smem_bytes(const Dims &g, int ty, int cpt, bool f64) {
  // FP64: the direction tile.  Mixed: direction and q = A d tiles (f32).
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
  const size_t static_smem = 6400;  // reduction scratch, tagged-sum values, flags, rounded up
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
    if (tiles > sms || tiles > kMaxTagBlocks) continue;
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
  // the tagged slots must fit the persistent state's partials (12 per CTA)
  if (2 * 2 * kMaxNV * blocks > 12 * ps.max_blocks)
    return -static_cast<int>(cudaErrorInvalidConfiguration);
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
  // the tagged-partial slots (2 buffers x blocks x 2*kMaxNV words) start at 0
  TagSync ts{reinterpret_cast<unsigned long long *>(ps.partials), blocks};
  cudaMemsetAsync(ts.slots, 0, sizeof(unsigned long long) * 2 * kMaxNV * 2 * blocks, st);
  void *params[] = {&args, &gs, &ts};
  err = cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(fn), dim3(blocks), dim3(kRT),
                                    params, static_cast<size_t>(plan.smem_bytes), st);
  return err == cudaSuccess ? blocks : -static_cast<int>(err);
}

}  // namespace afl
