// afl_poisson_stream.cu -- streaming persistent CG for grids that do not fit
// on chip (256^3 and up), vectorised along x.
//
// Each thread handles runs of V consecutive x cells (the widest of 4 / 2 / 1
// doubles or 8 / 4 / 1 floats that divides nx) and walks the runs of the
// whole grid with a stride of the CTA grid, so every array is streamed from
// HBM once per phase while the y neighbour rows of a run hit in L1 and the z
// neighbour planes in L2.  The solve is one cooperative launch
// with two bounded grid barriers per iteration; the direction update
// d = r + beta*d (src/fluid.rs:483-485) is formed on the fly inside the next
// matrix-vector product (double-buffered d), and for a single large grid
// q = A d is recomputed in the update pass rather than stored; passes
// alternate their walking direction so each starts in L2.  Built with
// -fmad=false: the FP64
// path keeps the reference's un-fused expressions (the mixed path writes its
// FMAs explicitly).
#include "afl_cg_stream_body.cuh"

namespace afl {
namespace {

// Register caps (CTAs per SM).  Uncapped, 4-double runs with the recomputed
// q take ~93 registers (2 CTAs per SM), 2- and 1-double runs 108 / 90;
// capped at 80 / 64 they fit 3 / 4 without spilling more than a few bytes
// (256^3: 323 -> 359; 258 x 256^2: 243 -> 310; 257 x 256^2: 172 -> 234
// Mcell-steps/s).
template <int V>
__global__ void __launch_bounds__(kST, (V == 4 ? 3 : 4))
    k_cg_stream_f64(CgArgs a, GridSync gs, Ring3 pr) {
  __shared__ double scratch[(kST / 32) * 3 + 4];
  cg_stream_f64_body<V, true>(a, gs, pr, blockIdx.x, gridDim.x, scratch);
}

// Uncapped, 8-float runs take 127 registers (2 CTAs per SM), 4- and 1-float
// runs ~150 (1 CTA per SM); capped at 80 / 64 they fit 3 / 4 without
// spilling (256^3: 602 -> 635; 260 x 256^2: 287 -> 612; 257 x 256^2:
// 106 -> 275 Mcell-steps/s).
template <int V>
__global__ void __launch_bounds__(kST, (V == 8 ? 3 : 4))
    k_cg_stream_mixed(MixedCgArgs a, GridSync gs, Ring3 pr) {
  __shared__ double scratch[(kST / 32) * 3 + 4];
  cg_stream_mixed_body<V, true>(a, gs, pr, blockIdx.x, gridDim.x, scratch);
}

// Many independent solves in one cooperative launch: CTA b works on system
// cta_inst[b] as its (b - first CTA of that system)-th CTA; each system has its
// own barrier, partials and stopping decisions, so systems finish at their
// own iteration counts.
// Capped at 48 registers: 5 CTAs per SM instead of 3 (at 80) for ~70 bytes of
// spill; the 48-plume ensemble 560 -> 596 (4 per SM) -> 605-624 Mcell-steps/s
// (FP64 ensemble: 338 -> 342).  At 6 per SM (40 registers) the spill doubles.
template <int V, bool F64>
__global__ void __launch_bounds__(kST, 5) k_cg_stream_multi(const MultiCgSystem *sys,
                                                            const int *cta_inst) {
  __shared__ double scratch[(kST / 32) * 3 + 4];
  const MultiCgSystem &s = sys[cta_inst[blockIdx.x]];
  const int vblock = blockIdx.x - s.cta_begin;
  const Ring3 pr{s.partials, (F64 ? 2 : 3) * s.ctas};
  if constexpr (F64) {
    const CgArgs a = s.f64;
    cg_stream_f64_body<V, false>(a, s.gs, pr, vblock, s.ctas, scratch);
  } else {
    const MixedCgArgs a = s.mixed;
    cg_stream_mixed_body<V, false>(a, s.gs, pr, vblock, s.ctas, scratch);
  }
}

template <typename K>
int blocks_of(K kernel) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reinterpret_cast<const void *>(kernel),
                                                kST, 0);
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

template <typename Args, typename K>
int launch_persistent(K kernel, const Args &a, const PersistentState &ps, int nvals,
                      cudaStream_t st) {
  int blocks = blocks_of(kernel);
  if (blocks > ps.max_blocks) blocks = ps.max_blocks;
  cudaMemsetAsync(ps.count, 0, sizeof(unsigned int), st);
  cudaMemsetAsync(ps.gen, 0, sizeof(unsigned int), st);
  cudaMemsetAsync(ps.abort_flag, 0, sizeof(int), st);
  Args args = a;
  GridSync gs;
  gs.count = ps.count;
  gs.gen = ps.gen;
  gs.abort_flag = ps.abort_flag;
  gs.nblocks = static_cast<unsigned int>(blocks);
  gs.timeout_ns = ps.timeout_ns;
  Ring3 pr{ps.partials, nvals * ps.max_blocks};
  void *params[] = {&args, &gs, &pr};
  const cudaError_t err = cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(kernel),
                                                      dim3(blocks), dim3(kST), params, 0, st);
  return err == cudaSuccess ? blocks : -static_cast<int>(err);
}

}  // namespace

int persistent_blocks_multi(bool f64, int v) {
  if (f64) return v == 2 ? blocks_of(&k_cg_stream_multi<2, true>)
                         : blocks_of(&k_cg_stream_multi<1, true>);
  return v == 4 ? blocks_of(&k_cg_stream_multi<4, false>) : blocks_of(&k_cg_stream_multi<1, false>);
}

int launch_cg_multi(const MultiCgSystem *d_sys, const int *d_cta_inst, int total_ctas, bool f64,
                    int v, cudaStream_t st) {
  const void *fn;
  if (f64)
    fn = v == 2 ? reinterpret_cast<const void *>(&k_cg_stream_multi<2, true>)
                : reinterpret_cast<const void *>(&k_cg_stream_multi<1, true>);
  else
    fn = v == 4 ? reinterpret_cast<const void *>(&k_cg_stream_multi<4, false>)
                : reinterpret_cast<const void *>(&k_cg_stream_multi<1, false>);
  void *params[] = {const_cast<MultiCgSystem **>(&d_sys), const_cast<int **>(&d_cta_inst)};
  const cudaError_t err =
      cudaLaunchCooperativeKernel(fn, dim3(total_ctas), dim3(kST), params, 0, st);
  return err == cudaSuccess ? total_ctas : -static_cast<int>(err);
}

int persistent_blocks_stream() {
  const int counts[] = {blocks_of(&k_cg_stream_f64<1>), blocks_of(&k_cg_stream_f64<2>),
                        blocks_of(&k_cg_stream_f64<4>), blocks_of(&k_cg_stream_mixed<1>),
                        blocks_of(&k_cg_stream_mixed<4>), blocks_of(&k_cg_stream_mixed<8>)};
  int most = 0;
  for (int c : counts) most = c > most ? c : most;
  return most;
}

// Cells per run: the widest of 4 / 2 / 1 doubles or 8 / 4 / 1 floats that
// divides nx (wider runs keep more bytes in flight per thread).
int stream_vector_width(const Dims &g, bool f64) {
  const int widths[2][3] = {{8, 4, 1}, {4, 2, 1}};
  for (int v : widths[f64 ? 1 : 0])
    if (g.nx % v == 0) return v;
  return 1;
}

int launch_cg_stream_f64(const CgArgs &a, const PersistentState &ps, cudaStream_t st) {
  switch (stream_vector_width(a.g, true)) {
    case 4: return launch_persistent(&k_cg_stream_f64<4>, a, ps, 2, st);
    case 2: return launch_persistent(&k_cg_stream_f64<2>, a, ps, 2, st);
    default: return launch_persistent(&k_cg_stream_f64<1>, a, ps, 2, st);
  }
}

int launch_cg_stream_mixed(const MixedCgArgs &a, const PersistentState &ps, cudaStream_t st) {
  switch (stream_vector_width(a.g, false)) {
    case 8: return launch_persistent(&k_cg_stream_mixed<8>, a, ps, 3, st);
    case 4: return launch_persistent(&k_cg_stream_mixed<4>, a, ps, 3, st);
    default: return launch_persistent(&k_cg_stream_mixed<1>, a, ps, 3, st);
  }
}

}  // namespace afl
