// afl_noalloc.cu -- a CG pressure solve for callers that cannot allocate.
//
// Some callers may not call cudaMalloc at all: real-time or render threads
// that must never block on the driver's allocator (cudaMalloc can wait for
// the device and takes driver locks), and hosts whose device memory is owned
// entirely by their own pool or arena (a game engine's or a renderer's
// budgeted heap), where a hidden allocation by a library breaks the budget.
// For them afl_solve_cg_noalloc runs the streaming persistent FP64 CG kernel
// (the kernel afl_solve_cg runs with AFL_POISSON_KERNEL_STREAMING; its AUTO
// choice may run the on-chip resident kernel instead, whose sums are ordered
// differently) on device buffers the caller already owns, and takes the
// solver's working memory from one fixed array compiled into this library
// instead of allocating it.  The call synchronises its stream before it
// returns, to read the solve's report.
//
// The array below is that working memory.  Every GPU that loads the library
// holds it (kNoAllocBytes, about 8.1 MiB) until the process exits.  All calls
// on a device share it and it keeps what the last call left there, so this
// file clears what must start at zero on every call, and calls whose work
// overlaps on the same GPU (for instance on two streams) race on it: a caller
// must order them.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/aether_fluid.h"
#include "afl_launch.h"

namespace {

// Grids of at most 64^3 cells; the four CG vectors take 32 bytes per cell.
constexpr size_t kNoAllocMaxCells = 262144;
constexpr size_t kVecBytes = kNoAllocMaxCells * sizeof(double);
constexpr size_t kHeaderBytes = 256;             // barrier words + report
constexpr int kMaxPartialBlocks = 2048;          // persistent CTAs the partials can hold
constexpr size_t kPartialBytes = 6 * kMaxPartialBlocks * sizeof(double);
constexpr size_t kNoAllocBytes = kHeaderBytes + kPartialBytes + 4 * kVecBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char *g_scratch_addr[kMaxDevices] = {};  // device address, per device

afl_status fail(afl_status st, const char *msg) {
  afl::set_last_error_text(msg);  // read back through afl_last_error()
  return st;
}

// The host-side name g_noalloc_scratch is not a device address; each device's
// address of the array is looked up once, with that device current.
afl_status scratch_address(int device, unsigned char **out) {
  if (device < 0 || device >= kMaxDevices)
    return fail(AFL_ERR_CUDA, "device ordinal outside the supported range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[device]) {
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) {
      char msg[200];
      snprintf(msg, sizeof msg, "cudaGetSymbolAddress of the solver scratch failed: %s",
               cudaGetErrorString(e));
      return fail(AFL_ERR_CUDA, msg);
    }
    g_scratch_addr[device] = static_cast<unsigned char *>(ptr);
  }
  *out = g_scratch_addr[device];
  return AFL_OK;
}

}  // namespace

extern "C" afl_status afl_solve_cg_noalloc(const double *d_rhs, double *d_pressure, size_t nx,
                                           size_t ny, size_t nz, int max_iters, double rel_tol,
                                           void *stream, afl_solve_info *info) {
  if (!d_rhs || !d_pressure)
    return fail(AFL_ERR_INVALID_ARGUMENT, "null device buffer");
  if (nx < 6 || ny < 6 || nz < 6)
    return fail(AFL_ERR_INVALID_ARGUMENT, "every grid dimension must be >= 6");
  // Each dimension is at least 6, so a grid within the limit has every
  // dimension below kNoAllocMaxCells / 36; checking them one by one first
  // keeps the product from wrapping around.
  if (nx > kNoAllocMaxCells / 36 || ny > kNoAllocMaxCells / 36 || nz > kNoAllocMaxCells / 36 ||
      nx * ny * nz > kNoAllocMaxCells) {
    char msg[240];
    snprintf(msg, sizeof msg,
             "grid %zux%zux%zu exceeds the no-allocation limit of %zu cells (64^3); "
             "use afl_solve_cg on a solver handle", nx, ny, nz, kNoAllocMaxCells);
    return fail(AFL_ERR_INVALID_ARGUMENT, msg);
  }
  if (max_iters < 0 || !(rel_tol >= 0.0))
    return fail(AFL_ERR_INVALID_ARGUMENT, "max_iters and rel_tol must be >= 0");

  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return fail(AFL_ERR_CUDA, cudaGetErrorString(e));
  unsigned char *base = nullptr;
  afl_status st = scratch_address(device, &base);
  if (st != AFL_OK) return st;

  const int blocks = afl::persistent_blocks_cg_f64();
  if (blocks > kMaxPartialBlocks)
    return fail(AFL_ERR_CUDA, "this GPU needs more persistent CTAs than the scratch holds");

  // Carve the array: barrier words and report, partials, then r, d0, d1, q.
  auto *words = reinterpret_cast<unsigned int *>(base);
  auto *report = reinterpret_cast<afl::SolveReport *>(base + 64);
  auto *partials = reinterpret_cast<double *>(base + kHeaderBytes);
  auto *vec = reinterpret_cast<double *>(base + kHeaderBytes + kPartialBytes);
  const size_t n = nx * ny * nz;

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // Zero what a call must not inherit from the previous one: the barrier
  // words and the report (the partials and vectors are written before read).
  e = cudaMemsetAsync(base, 0, kHeaderBytes, s);
  if (e != cudaSuccess) return fail(AFL_ERR_CUDA, cudaGetErrorString(e));

  afl::Dims g{};
  g.nx = static_cast<int>(nx);
  g.ny = static_cast<int>(ny);
  g.nz = static_cast<int>(nz);
  g.nxy = static_cast<int>(nx * ny);
  g.n = static_cast<int>(n);
  g.h = 1.0 / static_cast<double>(nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz));

  afl::PersistentState ps{};
  ps.count = words;
  ps.gen = words + 1;
  ps.abort_flag = reinterpret_cast<int *>(words + 2);
  ps.partials = partials;
  ps.max_blocks = kMaxPartialBlocks;
  ps.timeout_ns = 5000000000ull;

  afl::CgArgs a{g, d_pressure, d_rhs, vec, vec + n, vec + 2 * n, vec + 3 * n, max_iters,
                rel_tol, report};
  const int used = afl::launch_cg_f64(a, ps, s);
  if (used <= 0) {
    cudaGetLastError();
    return fail(AFL_ERR_CUDA, "cooperative launch of the CG kernel failed");
  }

  afl::SolveReport rep{};
  int abort_flag = 0;
  e = cudaMemcpyAsync(&rep, report, sizeof rep, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&abort_flag, words + 2, sizeof abort_flag, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(AFL_ERR_CUDA, cudaGetErrorString(e));
  if (abort_flag != 0)
    return fail(AFL_ERR_TIMEOUT, "the CG kernel gave up waiting at a grid barrier");
  if (info) {
    info->iterations = rep.iterations;
    info->refinements = rep.refinements;
    info->converged = rep.converged;
    info->status = rep.status;
    info->initial_residual = rep.initial_residual;
    info->final_residual = rep.final_residual;
    info->rhs_norm = rep.rhs_norm;
  }
  if (rep.status != 0) return fail(AFL_ERR_NONFINITE, "non-finite residual in the CG solve");
  return AFL_OK;
}
