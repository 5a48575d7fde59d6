// afl_solver.cu -- the C ABI of include/aether_fluid.h: the handle, its
// device buffers and stream, and the order of kernels in each reference
// method.  No CPU fallback exists: every numerical entry point runs kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/aether_fluid.h"
#include "afl_launch.h"

using afl::Dims;

namespace {

thread_local std::string g_last_error;

afl_status set_error(afl_status st, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return st;
}

#define AFL_CUDA(call)                                                              \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      return set_error(e_ == cudaErrorMemoryAllocation ? AFL_ERR_OUT_OF_MEMORY      \
                                                       : AFL_ERR_CUDA,              \
                       "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),     \
                       __FILE__, __LINE__);                                         \
    }                                                                               \
  } while (0)

#define AFL_TRY(expr)                  \
  do {                                 \
    afl_status s_ = (expr);            \
    if (s_ != AFL_OK) return s_;       \
  } while (0)

// f64::clamp, f64::floor/ceil and saturating `as usize` for the source boxes
// (src/fluid.rs:566-571), evaluated on the host exactly as the reference does.
int box_lo(double c, double r, int n) {
  const double v = std::fmax(std::floor(c - r - 1.0), 1.0);
  return v < static_cast<double>(n) ? static_cast<int>(v) : n;  // empty box beyond n-2
}
int box_hi(double c, double r, int n) {
  const double v = std::fmin(std::ceil(c + r + 1.0), static_cast<double>(n - 2));
  return v > 0.0 ? static_cast<int>(v) : 0;
}

// SplitMix64-seeded Xoshiro256++ (src/rng.rs:5-88), for the seeded initial
// velocity noise.
struct Xoshiro256pp {
  uint64_t s[4];
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  explicit Xoshiro256pp(uint64_t seed) {
    uint64_t sm = seed ^ 0xA5A55A5AF0F00F0Full;
    for (auto &w : s) {
      sm += 0x9E3779B97F4A7C15ull;
      uint64_t z = sm;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      w = z ^ (z >> 31);
    }
    if ((s[0] | s[1] | s[2] | s[3]) == 0) s[0] = 1;
  }
  uint64_t next() {
    const uint64_t out = rotl(s[0] + s[3], 23) + s[0];
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return out;
  }
  double next_f64() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }
};

// Folds the persistent kernels' abort flag and the solve report into the
// handle's sticky status word (read at the next synchronising call).
__global__ void k_fold_status(const int *abort_flag, const afl::SolveReport *rep,
                              int *sticky) {
  if (threadIdx.x != 0) return;
  int st = 0;
  if (*abort_flag != 0) st = AFL_ERR_TIMEOUT;
  else if (rep && rep->status != 0) st = rep->status;
  if (st != 0 && *sticky == 0) *sticky = st;
}

}  // namespace

struct afl_solver {
  int device = 0;
  cudaStream_t stream = nullptr;
  Dims g{};
  afl_params params{};
  int precision = AFL_PRECISION_FP64;
  size_t esize = 8;        // bytes per velocity/density/temperature value
  void *fld[5] = {};       // u, v, w, density, temperature (T)
  void *tmp_fwd = nullptr, *tmp_out = nullptr;
  void *curl[4] = {};      // curl x, y, z, |curl| (T)
  double *p = nullptr, *b = nullptr;
  // Poisson vectors: FP64 -> r, d0, d1, q (double); MIXED -> r, e, d0, d1, q (float)
  void *cg[5] = {};
  double *partials = nullptr;     // kReduceBlocks * kReduceMaxVals
  double *tel_partials = nullptr; // 7 per CTA of the fused density/temperature advection
  double *scal = nullptr;         // [0..1] divergence {rms,||b||}, [2..9] telemetry, [10] max
  double *tel = nullptr;          // run telemetry, 8 doubles per step
  afl::SolveReport *reports = nullptr;  // run reports, one per step
  int run_cap = 0;
  int *sticky = nullptr;
  afl::PersistentState ps{};
  bool resident_ok = false;       // the grid fits the on-chip resident CG
  afl::ResidentPlan resident{};
  double *amp = nullptr;          // sphere amplitude map (optional)
  double *stage = nullptr;        // f64 staging for the mixed form's transfers
  double *sample_buf = nullptr;   // 4 doubles per point
  size_t sample_cap = 0;
  double *h_scal = nullptr;       // pinned host mirror for scalars
  std::vector<void *> allocs;
  // tracing
  bool timing = false;
  struct Timed { int stage; cudaEvent_t start, stop; };
  std::vector<Timed> pending;
  std::vector<cudaEvent_t> event_pool;
  double stage_ms[AFL_STAGE_COUNT] = {};
  int64_t stage_calls[AFL_STAGE_COUNT] = {};
  uint64_t launches = 0;

  template <typename T>
  T *F(int f) const { return static_cast<T *>(fld[f]); }
};

namespace {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

cudaEvent_t pool_event(afl_solver *s) {
  if (!s->event_pool.empty()) {
    cudaEvent_t e = s->event_pool.back();
    s->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Records CUDA events around one stage on the handle's stream when timing is
// enabled; `kernels` is the number of kernels the stage launches.
struct StageTimer {
  afl_solver *s;
  int stage;
  cudaEvent_t start = nullptr;
  StageTimer(afl_solver *s_, int stage_, int kernels) : s(s_), stage(stage_) {
    s->launches += static_cast<uint64_t>(kernels);
    if (s->timing) {
      start = pool_event(s);
      cudaEventRecord(start, s->stream);
    }
  }
  ~StageTimer() {
    if (start) {
      cudaEvent_t stop = pool_event(s);
      cudaEventRecord(stop, s->stream);
      s->pending.push_back({stage, start, stop});
    }
  }
};

// Folds recorded event pairs into the per-stage totals (stream must be idle).
void resolve_timing(afl_solver *s) {
  for (auto &t : s->pending) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, t.start, t.stop) == cudaSuccess) {
      s->stage_ms[t.stage] += ms;
      s->stage_calls[t.stage] += 1;
    }
    s->event_pool.push_back(t.start);
    s->event_pool.push_back(t.stop);
  }
  s->pending.clear();
}

afl_status check_handle(const afl_solver *s) {
  if (!s) return set_error(AFL_ERR_INVALID_ARGUMENT, "null solver handle");
  return AFL_OK;
}

afl_status dev_alloc(afl_solver *s, void **out, size_t bytes) {
  void *ptr = nullptr;
  AFL_CUDA(cudaMalloc(&ptr, bytes));
  s->allocs.push_back(ptr);
  *out = ptr;
  return AFL_OK;
}

template <typename P>
afl_status alloc_as(afl_solver *s, P **out, size_t bytes) {
  void *v = nullptr;
  AFL_TRY(dev_alloc(s, &v, bytes));
  *out = static_cast<P *>(v);
  return AFL_OK;
}

afl_status validate_params(const afl_params &p) {
  if (p.solver_kind != AFL_POISSON_CG && p.solver_kind != AFL_POISSON_RBSOR)
    return set_error(AFL_ERR_INVALID_ARGUMENT, "solver_kind must be 0 (CG) or 1 (RB-SOR)");
  if (p.solver_iters < 0)
    return set_error(AFL_ERR_INVALID_ARGUMENT, "solver_iters must be >= 0");
  if (p.precision != AFL_PRECISION_FP64 && p.precision != AFL_PRECISION_MIXED)
    return set_error(AFL_ERR_INVALID_ARGUMENT, "precision must be 0 (FP64) or 1 (MIXED)");
  if (p.source_kind < AFL_SOURCE_CYBERPUNK || p.source_kind > AFL_SOURCE_NONE)
    return set_error(AFL_ERR_INVALID_ARGUMENT, "source_kind must be 0, 1 or 2");
  if (!(p.cg_rel_tol >= 0.0))
    return set_error(AFL_ERR_INVALID_ARGUMENT, "cg_rel_tol must be >= 0");
  if (p.mixed_inner_iters < 1 || p.mixed_max_refinements < 1 || !(p.mixed_inner_rel_tol > 0.0))
    return set_error(AFL_ERR_INVALID_ARGUMENT, "mixed solver settings must be positive");
  if (p.poisson_kernel < AFL_POISSON_KERNEL_AUTO || p.poisson_kernel > AFL_POISSON_KERNEL_RESIDENT)
    return set_error(AFL_ERR_INVALID_ARGUMENT, "poisson_kernel must be 0, 1 or 2");
  return AFL_OK;
}

// Synchronises the stream and reports (then clears) a sticky device error.
afl_status sync_and_check(afl_solver *s) {
  AFL_CUDA(cudaStreamSynchronize(s->stream));
  AFL_CUDA(cudaGetLastError());
  int st = 0;
  AFL_CUDA(cudaMemcpy(&st, s->sticky, sizeof(int), cudaMemcpyDeviceToHost));
  if (st != 0) {
    AFL_CUDA(cudaMemset(s->sticky, 0, sizeof(int)));
    if (st == AFL_ERR_TIMEOUT)
      return set_error(AFL_ERR_TIMEOUT,
                       "a persistent Poisson kernel gave up waiting at a grid barrier");
    return set_error(static_cast<afl_status>(st),
                     "non-finite residual in the Poisson solve (status %d)", st);
  }
  return AFL_OK;
}

afl_status launch_check() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_error(AFL_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
  return AFL_OK;
}

// ---- stages, generic over the field type ------------------------------------
template <typename T>
afl_status stage_advect(afl_solver *s, int kind, double dt, double diss) {
  const int f = (kind >= 0 && kind <= 3) ? kind : 4;  // `_ =>` arm: temperature
  const T *u = s->F<T>(0), *v = s->F<T>(1), *w = s->F<T>(2);
  const T *src = s->F<T>(f);
  T *fwd = static_cast<T *>(s->tmp_fwd), *out = static_cast<T *>(s->tmp_out);
  StageTimer timer(s, AFL_STAGE_ADVECT, 2);
  afl::launch_advect_fwd<T>(s->g, u, v, w, src, fwd, dt, s->stream);
  afl::launch_advect_mc<T>(s->g, u, v, w, src, fwd, out, dt, diss, f >= 3, s->stream);
  std::swap(s->fld[f], s->tmp_out);
  return launch_check();
}

template <typename T>
afl_status stage_wall_bc(afl_solver *s) {
  StageTimer timer(s, AFL_STAGE_FORCES, 1);
  afl::launch_wall_bc<T>(s->g, s->F<T>(0), s->F<T>(1), s->F<T>(2), s->stream);
  return launch_check();
}

// apply_buoyancy_and_vorticity_confinement (src/fluid.rs:256-330): one
// shared-memory-staged launch writes the new velocity into three spare
// buffers, which then become u, v, w (the curl never reaches memory).
template <typename T>
afl_status stage_buoyancy_vorticity(afl_solver *s, double dt) {
  StageTimer timer(s, AFL_STAGE_FORCES, 1);
  afl::launch_forces_fused<T>(s->g, s->F<T>(0), s->F<T>(1), s->F<T>(2), s->F<T>(3), s->F<T>(4),
                              static_cast<T *>(s->curl[0]), static_cast<T *>(s->curl[1]),
                              static_cast<T *>(s->curl[2]), dt, s->params.vorticity_eps,
                              s->params.buoyancy_beta, s->params.gravity_alpha, s->stream);
  for (int f = 0; f < 3; ++f) std::swap(s->fld[f], s->curl[f]);
  return launch_check();
}

// The end of step() (src/fluid.rs:607-610): density (dissipation 0.996) and
// temperature (0.985) advected in one shared-memory-staged launch that reads
// the velocity once and sums the telemetry of the final state; the finalize
// kernel writes its 8 doubles.
template <typename T>
afl_status stage_advect_scalars_telemetry(afl_solver *s, double dt, double time_sec,
                                          double *out8) {
  const T *src[2] = {s->F<T>(3), s->F<T>(4)};
  T *out[2] = {static_cast<T *>(s->tmp_out), static_cast<T *>(s->tmp_fwd)};
  const double diss[2] = {0.996, 0.985};
  {
    StageTimer timer(s, AFL_STAGE_ADVECT, 1);
    afl::launch_scalars_fused<T>(s->g, s->F<T>(0), s->F<T>(1), s->F<T>(2), src, out, diss, dt,
                                 s->tel_partials, s->stream);
  }
  std::swap(s->fld[3], s->tmp_out);
  std::swap(s->fld[4], s->tmp_fwd);
  AFL_TRY(launch_check());
  StageTimer timer(s, AFL_STAGE_TELEMETRY, 1);
  afl::launch_telemetry_finalize(s->tel_partials, afl::fused_ctas(s->g), time_sec, out8,
                                 s->stream);
  return launch_check();
}

template <typename T>
afl_status stage_divergence(afl_solver *s) {
  StageTimer timer(s, AFL_STAGE_DIVERGENCE, 2);
  afl::launch_divergence<T>(s->g, s->F<T>(0), s->F<T>(1), s->F<T>(2), s->b, s->partials,
                            s->scal, s->stream);
  return launch_check();
}

afl_status stage_solve(afl_solver *s, int kind, int iters, afl::SolveReport *rep) {
  const Dims &g = s->g;
  StageTimer timer(s, AFL_STAGE_POISSON, 2);
  int blocks = 0;
  const bool want_resident = kind == AFL_POISSON_CG &&
                             s->params.poisson_kernel != AFL_POISSON_KERNEL_STREAMING;
  if (kind == AFL_POISSON_CG && s->params.poisson_kernel == AFL_POISSON_KERNEL_RESIDENT &&
      !s->resident_ok)
    return set_error(AFL_ERR_INVALID_ARGUMENT,
                     "the %dx%dx%d grid does not fit the resident CG kernel", g.nx, g.ny, g.nz);
  if (want_resident && s->resident_ok) {
    const bool f64 = s->precision == AFL_PRECISION_FP64;
    afl::ResidentCgArgs a{};
    a.g = g;
    a.p = s->p;
    a.b = s->b;
    a.rpub = s->cg[0];
    a.dpub0 = f64 ? s->cg[1] : s->cg[2];
    a.dpub1 = f64 ? s->cg[2] : s->cg[3];
    a.max_iters = std::max(f64 ? 0 : 1, iters);
    a.max_inner = std::max(1, s->params.mixed_inner_iters);
    a.max_refine = s->params.mixed_max_refinements;
    a.inner_rel_tol = s->params.mixed_inner_rel_tol;
    a.rel_tol = s->params.cg_rel_tol;
    a.report = rep;
    blocks = afl::launch_cg_resident(a, s->resident, f64, s->ps, s->stream);
  } else if (kind != AFL_POISSON_CG && s->resident_ok &&
             (s->params.poisson_kernel == AFL_POISSON_KERNEL_RESIDENT ||
              (s->params.poisson_kernel == AFL_POISSON_KERNEL_AUTO &&
               s->precision != AFL_PRECISION_FP64))) {
    // RB-SOR on chip: the automatic choice for the mixed form only.  The FP64
    // sweep re-reads its f64 right-hand side from L2 every half-sweep (no room
    // on chip beside the f64 tile), and the streaming colour walk is faster.
    const bool f64 = s->precision == AFL_PRECISION_FP64;
    afl::ResidentSorArgs a{};
    a.g = g;
    a.p = s->p;
    a.b = s->b;
    a.e32 = f64 ? nullptr : static_cast<float *>(s->cg[0]);
    a.sweeps = iters;
    a.omega = s->params.sor_omega;
    a.report = rep;
    blocks = afl::launch_sor_resident(a, s->resident, f64, s->ps, s->stream);
  } else if (s->precision == AFL_PRECISION_FP64) {
    if (kind == AFL_POISSON_CG) {
      afl::CgArgs a{g, s->p, s->b, static_cast<double *>(s->cg[0]),
                    static_cast<double *>(s->cg[1]), static_cast<double *>(s->cg[2]),
                    static_cast<double *>(s->cg[3]), iters, s->params.cg_rel_tol, rep};
      blocks = afl::launch_cg_f64(a, s->ps, s->stream);
    } else {
      afl::SorArgs a{g, s->p, s->b, iters, s->params.sor_omega, rep};
      blocks = afl::launch_rbsor_f64(a, s->ps, s->stream);
    }
  } else {
    if (kind == AFL_POISSON_CG) {
      afl::MixedCgArgs a{};
      a.g = g;
      a.p = s->p;
      a.b = s->b;
      a.r = static_cast<float *>(s->cg[0]);
      a.e = static_cast<float *>(s->cg[1]);
      a.d0 = static_cast<float *>(s->cg[2]);
      a.d1 = static_cast<float *>(s->cg[3]);
      a.q = static_cast<float *>(s->cg[4]);
      a.max_inner = std::max(1, s->params.mixed_inner_iters);
      a.max_total = std::max(1, iters);
      a.max_refine = s->params.mixed_max_refinements;
      a.inner_rel_tol = s->params.mixed_inner_rel_tol;
      a.rel_tol = s->params.cg_rel_tol;
      a.report = rep;
      blocks = afl::launch_cg_mixed(a, s->ps, s->stream);
    } else {
      afl::SorMixedArgs a{g, s->p, s->b, static_cast<float *>(s->cg[0]),
                          static_cast<float *>(s->cg[1]), iters, s->params.sor_omega, rep};
      blocks = afl::launch_rbsor_mixed(a, s->ps, s->stream);
    }
  }
  if (blocks <= 0) {
    cudaGetLastError();  // clear it: the handle stays usable
    return set_error(AFL_ERR_CUDA, "cooperative launch of the Poisson kernel failed: %s",
                     cudaGetErrorString(static_cast<cudaError_t>(-blocks)));
  }
  AFL_TRY(launch_check());
  k_fold_status<<<1, 32, 0, s->stream>>>(s->ps.abort_flag, rep, s->sticky);
  return launch_check();
}

template <typename T>
afl_status stage_project(afl_solver *s, bool leading_bc, afl::SolveReport *rep) {
  // project (src/fluid.rs:496-529): wall BC, divergence, solve, gradient, BC.
  if (leading_bc) AFL_TRY(stage_wall_bc<T>(s));
  AFL_TRY(stage_divergence<T>(s));
  AFL_TRY(stage_solve(s, s->params.solver_kind, s->params.solver_iters, rep));
  StageTimer timer(s, AFL_STAGE_PROJECT, 1);
  afl::launch_project<T>(s->g, s->F<T>(0), s->F<T>(1), s->F<T>(2), s->p, s->stream);
  return launch_check();
}

template <typename T>
afl_status stage_inject_cyberpunk(afl_solver *s, double time_sec, double dt) {
  const afl::JetPair jp = afl::cyberpunk_jets(s->g, time_sec);
  StageTimer timer(s, AFL_STAGE_SOURCE, 2);
  for (int q = 0; q < 2; ++q)
    afl::launch_inject_jet<T>(s->g, jp.lo[q], jp.hi[q], s->F<T>(3), s->F<T>(4), s->F<T>(0),
                              s->F<T>(1), s->F<T>(2), jp.jet[q], jp.r2, dt, jp.pulse, s->stream);
  return launch_check();
}

template <typename T>
afl_status stage_inject_sphere(afl_solver *s) {
  const Dims &g = s->g;
  const double *c = s->params.sphere_center;
  const double r = s->params.sphere_radius;
  const int lo[3] = {box_lo(c[0], r, g.nx), box_lo(c[1], r, g.ny), box_lo(c[2], r, g.nz)};
  const int hi[3] = {box_hi(c[0], r, g.nx), box_hi(c[1], r, g.ny), box_hi(c[2], r, g.nz)};
  StageTimer timer(s, AFL_STAGE_SOURCE, 1);
  afl::launch_inject_sphere<T>(g, lo, hi, s->F<T>(3), s->F<T>(4), s->amp, c, r * r,
                               s->params.sphere_density, s->params.sphere_temperature,
                               s->stream);
  return launch_check();
}

template <typename T>
afl_status stage_telemetry(afl_solver *s, double time_sec, double *out8) {
  StageTimer timer(s, AFL_STAGE_TELEMETRY, 2);
  afl::launch_telemetry<T>(s->g, s->F<T>(0), s->F<T>(1), s->F<T>(2), s->F<T>(3), time_sec,
                           s->partials, out8, s->stream);
  return launch_check();
}

template <typename T>
afl_status stage_step(afl_solver *s, double dt, double time_sec, double *tel8,
                      afl::SolveReport *rep) {
  // step (src/fluid.rs:598-611)
  AFL_TRY(stage_advect<T>(s, 0, dt, 0.996));
  AFL_TRY(stage_advect<T>(s, 1, dt, 0.996));
  AFL_TRY(stage_advect<T>(s, 2, dt, 0.996));
  if (s->params.source_kind == AFL_SOURCE_CYBERPUNK)
    AFL_TRY(stage_inject_cyberpunk<T>(s, time_sec, dt));
  else if (s->params.source_kind == AFL_SOURCE_SPHERE)
    AFL_TRY(stage_inject_sphere<T>(s));
  AFL_TRY(stage_buoyancy_vorticity<T>(s, dt));
  // The confinement kernel ends with the wall BC, so project's leading
  // enforce_wall_velocity_bc (src/fluid.rs:497) is a no-op here and skipped.
  AFL_TRY(stage_project<T>(s, false, rep));
  return stage_advect_scalars_telemetry<T>(s, dt, time_sec, tel8);
}

template <typename Fn>
afl_status dispatch(afl_solver *s, Fn &&fn) {
  if (s->precision == AFL_PRECISION_FP64) return fn(static_cast<double *>(nullptr));
  return fn(static_cast<float *>(nullptr));
}

afl_status ensure_run_capacity(afl_solver *s, int steps) {
  if (steps <= s->run_cap) return AFL_OK;
  int cap = std::max(steps, 2 * s->run_cap);
  double *tel = nullptr;
  afl::SolveReport *rep = nullptr;
  AFL_CUDA(cudaMalloc(&tel, sizeof(double) * 8 * static_cast<size_t>(cap)));
  cudaError_t e = cudaMalloc(&rep, sizeof(afl::SolveReport) * static_cast<size_t>(cap));
  if (e != cudaSuccess) {
    cudaFree(tel);
    return set_error(AFL_ERR_OUT_OF_MEMORY, "cudaMalloc of run buffers failed: %s",
                     cudaGetErrorString(e));
  }
  AFL_CUDA(cudaStreamSynchronize(s->stream));
  if (s->tel) cudaFree(s->tel);
  if (s->reports) cudaFree(s->reports);
  s->tel = tel;
  s->reports = rep;
  s->run_cap = cap;
  return AFL_OK;
}

void to_info(const afl::SolveReport &r, afl_solve_info *info) {
  info->iterations = r.iterations;
  info->refinements = r.refinements;
  info->converged = r.converged;
  info->status = r.status;
  info->initial_residual = r.initial_residual;
  info->final_residual = r.final_residual;
  info->rhs_norm = r.rhs_norm;
}

void to_telemetry(const double *t8, afl_telemetry *t) {
  t->time_sec = t8[0];
  t->kinetic_energy = t8[1];
  t->enstrophy = t8[2];
  t->peak_vorticity = t8[3];
  t->total_mass = t8[4];
  t->center_of_mass[0] = t8[5];
  t->center_of_mass[1] = t8[6];
  t->center_of_mass[2] = t8[7];
}

afl_status check_field(const afl_solver *s, int field, size_t n) {
  if (field < AFL_FIELD_U || field > AFL_FIELD_DIVERGENCE)
    return set_error(AFL_ERR_INVALID_ARGUMENT, "field id %d out of range 0..6", field);
  if (n != static_cast<size_t>(s->g.n))
    return set_error(AFL_ERR_INVALID_ARGUMENT, "field length %zu != nx*ny*nz = %d", n, s->g.n);
  return AFL_OK;
}

}  // namespace

namespace afl {
void set_last_error_text(const char *msg) { g_last_error = msg ? msg : ""; }

// Scalars and jet geometry of src/fluid.rs:533-571, on the host.
JetPair cyberpunk_jets(const Dims &g, double time_sec) {
  constexpr double kTau = 6.283185307179586;
  const double cx = 0.5 * static_cast<double>(g.nx);
  const double cz = 0.5 * static_cast<double>(g.nz);
  const int base_j = std::min(3, g.ny - 3);
  JetPair jp{};
  jp.pulse = 0.65 + 0.35 * std::sin(time_sec * kTau * 0.55) +
             0.25 * std::fmax(std::cos(time_sec * kTau * 1.35), 0.0);
  const double angle = time_sec * 1.85;
  const double orbit_r = static_cast<double>(g.nx) * 0.14;
  const double ca = std::cos(angle), sa = std::sin(angle);
  const double jets[2][6] = {
      {cx + orbit_r * ca, static_cast<double>(base_j) + 1.5, cz + orbit_r * sa, -2.6 * sa,
       7.2 * jp.pulse, 2.6 * ca},
      {cx - orbit_r * ca, static_cast<double>(base_j) + 2.0, cz - orbit_r * sa, 2.6 * sa,
       6.4 * jp.pulse, -2.6 * ca},
  };
  const double r_cells = std::fmax(static_cast<double>(g.nx) * 0.105, 2.2);
  jp.r2 = r_cells * r_cells;
  const int n[3] = {g.nx, g.ny, g.nz};
  for (int q = 0; q < 2; ++q) {
    for (int a = 0; a < 6; ++a) jp.jet[q][a] = jets[q][a];
    for (int a = 0; a < 3; ++a) {
      jp.lo[q][a] = box_lo(jets[q][a], r_cells, n[a]);
      jp.hi[q][a] = box_hi(jets[q][a], r_cells, n[a]);
    }
  }
  return jp;
}
}  // namespace afl

// ============================================================================
namespace afl {
bool solver_view(const afl_solver *s, SolverView *out) {
  if (!s || !out) return false;
  out->g = s->g;
  out->device = s->device;
  out->stream = s->stream;
  out->f64 = s->precision == AFL_PRECISION_FP64;
  out->density = s->fld[3];
  out->temperature = s->fld[4];
  return true;
}
}  // namespace afl

extern "C" {

const char *afl_last_error(void) { return g_last_error.c_str(); }
int afl_abi_version(void) { return AFL_ABI_VERSION; }

afl_status afl_params_default(afl_params *p) {
  if (!p) return set_error(AFL_ERR_INVALID_ARGUMENT, "null params");
  std::memset(p, 0, sizeof *p);
  p->vorticity_eps = 5.5;  // src/fluid.rs:79-83
  p->buoyancy_beta = 6.8;
  p->gravity_alpha = 0.45;
  p->solver_kind = AFL_POISSON_CG;
  p->solver_iters = 32;
  p->sor_omega = 1.65;  // src/fluid.rs:398
  p->cg_rel_tol = 0.0;
  p->precision = AFL_PRECISION_FP64;
  p->source_kind = AFL_SOURCE_CYBERPUNK;
  p->sphere_radius = 0.0;
  p->sphere_density = 1.0;
  p->sphere_temperature = 1.0;
  p->fail_on_not_converged = 0;
  p->mixed_inner_iters = 200;
  p->mixed_inner_rel_tol = 1e-4;
  p->mixed_max_refinements = 8;
  p->poisson_kernel = AFL_POISSON_KERNEL_AUTO;
  return AFL_OK;
}

afl_status afl_create(size_t nx, size_t ny, size_t nz, const afl_params *params,
                      afl_solver **out) {
  if (!out) return set_error(AFL_ERR_INVALID_ARGUMENT, "null output handle pointer");
  *out = nullptr;
  if (nx < 6 || ny < 6 || nz < 6)  // src/fluid.rs:54
    return set_error(AFL_ERR_INVALID_ARGUMENT,
                     "grid %zux%zux%zu: every dimension must be >= 6", nx, ny, nz);
  const size_t n = nx * ny * nz;
  if (n > (static_cast<size_t>(1) << 30))
    return set_error(AFL_ERR_INVALID_ARGUMENT, "grid of %zu cells exceeds 2^30", n);
  afl_params p;
  if (params) p = *params; else afl_params_default(&p);
  AFL_TRY(validate_params(p));
  int dev_count = 0;
  cudaError_t ce = cudaGetDeviceCount(&dev_count);
  if (ce != cudaSuccess || dev_count == 0)
    return set_error(AFL_ERR_CUDA, "no CUDA device available (%s); this library has no "
                     "CPU path", cudaGetErrorString(ce));

  auto *s = new afl_solver();
  cudaGetDevice(&s->device);
  s->params = p;
  s->precision = p.precision;
  s->esize = p.precision == AFL_PRECISION_FP64 ? sizeof(double) : sizeof(float);
  s->g.nx = static_cast<int>(nx);
  s->g.ny = static_cast<int>(ny);
  s->g.nz = static_cast<int>(nz);
  s->g.nxy = static_cast<int>(nx * ny);
  s->g.n = static_cast<int>(n);
  s->g.h = 1.0 / static_cast<double>(std::max(nx, std::max(ny, nz)));  // src/fluid.rs:56

  auto fail = [&](afl_status st) {
    std::string msg = g_last_error;
    afl_destroy(s);
    g_last_error = msg;
    return st;
  };
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(set_error(AFL_ERR_CUDA, "cudaStreamCreate failed"));
  const size_t fb = n * s->esize;
  afl_status st = AFL_OK;
  for (int f = 0; f < 5 && st == AFL_OK; ++f) st = dev_alloc(s, &s->fld[f], fb);
  if (st == AFL_OK) st = dev_alloc(s, &s->tmp_fwd, fb);
  if (st == AFL_OK) st = dev_alloc(s, &s->tmp_out, fb);
  for (int f = 0; f < 4 && st == AFL_OK; ++f) st = dev_alloc(s, &s->curl[f], fb);
  if (st == AFL_OK) st = alloc_as(s, &s->p, n * sizeof(double));
  if (st == AFL_OK) st = alloc_as(s, &s->b, n * sizeof(double));
  const int ncg = s->precision == AFL_PRECISION_FP64 ? 4 : 5;
  // one block: the resident FP64 CG reads cg[0..3] as four consecutive arrays
  void *cg_block = nullptr;
  if (st == AFL_OK) st = dev_alloc(s, &cg_block, fb * static_cast<size_t>(ncg));
  for (int f = 0; f < ncg && st == AFL_OK; ++f)
    s->cg[f] = static_cast<unsigned char *>(cg_block) + fb * static_cast<size_t>(f);
  if (st == AFL_OK && s->precision == AFL_PRECISION_MIXED)
    st = alloc_as(s, &s->stage, n * sizeof(double));
  if (st == AFL_OK)
    st = alloc_as(s, &s->partials, sizeof(double) * afl::kReduceBlocks * afl::kReduceMaxVals);
  if (st == AFL_OK) st = alloc_as(s, &s->scal, sizeof(double) * 16);
  if (st == AFL_OK)
    st = alloc_as(s, &s->tel_partials, sizeof(double) * 7 * afl::fused_ctas(s->g));
  if (st == AFL_OK) st = alloc_as(s, &s->sticky, sizeof(int) * 4);
  // persistent-kernel state: the CTA bound is the largest co-resident grid
  int maxb = std::max(std::max(afl::persistent_blocks_cg_f64(), afl::persistent_blocks_sor_f64()),
                      std::max(afl::persistent_blocks_cg_mixed(),
                               afl::persistent_blocks_sor_mixed()));
  s->ps.max_blocks = maxb;
  s->resident_ok = afl::plan_resident(s->g, s->precision == AFL_PRECISION_FP64, &s->resident);
  s->ps.timeout_ns = 5000000000ull;  // 5 s per barrier wait
  if (const char *env = std::getenv("AFL_BARRIER_TIMEOUT_NS")) s->ps.timeout_ns = std::strtoull(env, nullptr, 10);
  unsigned int *bar = nullptr;
  if (st == AFL_OK) st = alloc_as(s, &bar, sizeof(unsigned int) * 4);
  if (st == AFL_OK) {
    s->ps.count = bar;
    s->ps.gen = bar + 1;
    s->ps.abort_flag = reinterpret_cast<int *>(bar + 2);
    st = alloc_as(s, &s->ps.partials, sizeof(double) * 12 * static_cast<size_t>(maxb));
  }
  if (st == AFL_OK && cudaMallocHost(&s->h_scal, sizeof(double) * 16) != cudaSuccess)
    st = set_error(AFL_ERR_OUT_OF_MEMORY, "cudaMallocHost failed");
  if (st != AFL_OK) return fail(st);
  // FluidSolver3D::new zero-initialises every field (src/fluid.rs:62-78).
  for (int f = 0; f < 5; ++f) cudaMemsetAsync(s->fld[f], 0, fb, s->stream);
  cudaMemsetAsync(s->tmp_fwd, 0, fb, s->stream);
  cudaMemsetAsync(s->tmp_out, 0, fb, s->stream);
  for (int f = 0; f < 4; ++f) cudaMemsetAsync(s->curl[f], 0, fb, s->stream);
  for (int f = 0; f < ncg; ++f) cudaMemsetAsync(s->cg[f], 0, fb, s->stream);
  cudaMemsetAsync(s->p, 0, n * sizeof(double), s->stream);
  cudaMemsetAsync(s->b, 0, n * sizeof(double), s->stream);
  cudaMemsetAsync(s->sticky, 0, sizeof(int) * 4, s->stream);
  cudaMemsetAsync(bar, 0, sizeof(unsigned int) * 4, s->stream);
  if (cudaStreamSynchronize(s->stream) != cudaSuccess)
    return fail(set_error(AFL_ERR_CUDA, "initialisation failed: %s",
                          cudaGetErrorString(cudaGetLastError())));
  *out = s;
  return AFL_OK;
}

afl_status afl_destroy(afl_solver *s) {
  if (!s) return AFL_OK;
  DeviceGuard guard(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (void *p : s->allocs) cudaFree(p);
  if (s->tel) cudaFree(s->tel);
  if (s->reports) cudaFree(s->reports);
  if (s->amp) cudaFree(s->amp);
  if (s->sample_buf) cudaFree(s->sample_buf);
  if (s->h_scal) cudaFreeHost(s->h_scal);
  for (auto &t : s->pending) {
    cudaEventDestroy(t.start);
    cudaEventDestroy(t.stop);
  }
  for (cudaEvent_t e : s->event_pool) cudaEventDestroy(e);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return AFL_OK;
}

afl_status afl_get_dims(const afl_solver *s, size_t *nx, size_t *ny, size_t *nz, double *h) {
  AFL_TRY(check_handle(s));
  if (nx) *nx = static_cast<size_t>(s->g.nx);
  if (ny) *ny = static_cast<size_t>(s->g.ny);
  if (nz) *nz = static_cast<size_t>(s->g.nz);
  if (h) *h = s->g.h;
  return AFL_OK;
}

afl_status afl_set_params(afl_solver *s, const afl_params *params) {
  AFL_TRY(check_handle(s));
  if (!params) return set_error(AFL_ERR_INVALID_ARGUMENT, "null params");
  afl_params p = *params;
  p.precision = s->precision;  // fixed at creation
  AFL_TRY(validate_params(p));
  s->params = p;
  return AFL_OK;
}

afl_status afl_get_params(const afl_solver *s, afl_params *params) {
  AFL_TRY(check_handle(s));
  if (!params) return set_error(AFL_ERR_INVALID_ARGUMENT, "null params");
  *params = s->params;
  return AFL_OK;
}

afl_status afl_set_source_amplitude(afl_solver *s, const double *amp, size_t n) {
  AFL_TRY(check_handle(s));
  DeviceGuard guard(s->device);
  if (!amp) {
    if (s->amp) {
      AFL_CUDA(cudaStreamSynchronize(s->stream));
      cudaFree(s->amp);
      s->amp = nullptr;
    }
    return AFL_OK;
  }
  if (n != static_cast<size_t>(s->g.n))
    return set_error(AFL_ERR_INVALID_ARGUMENT, "amplitude length %zu != %d", n, s->g.n);
  if (!s->amp) AFL_CUDA(cudaMalloc(&s->amp, n * sizeof(double)));
  AFL_CUDA(cudaMemcpyAsync(s->amp, amp, n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  return AFL_OK;
}

afl_status afl_upload_field(afl_solver *s, int field, const double *host, size_t n) {
  AFL_TRY(check_handle(s));
  AFL_TRY(check_field(s, field, n));
  if (!host) return set_error(AFL_ERR_INVALID_ARGUMENT, "null host buffer");
  DeviceGuard guard(s->device);
  const size_t bytes = n * sizeof(double);
  if (field == AFL_FIELD_PRESSURE || field == AFL_FIELD_DIVERGENCE) {
    double *dst = field == AFL_FIELD_PRESSURE ? s->p : s->b;
    AFL_CUDA(cudaMemcpyAsync(dst, host, bytes, cudaMemcpyHostToDevice, s->stream));
  } else if (s->precision == AFL_PRECISION_FP64) {
    AFL_CUDA(cudaMemcpyAsync(s->fld[field], host, bytes, cudaMemcpyHostToDevice, s->stream));
  } else {
    AFL_CUDA(cudaMemcpyAsync(s->stage, host, bytes, cudaMemcpyHostToDevice, s->stream));
    afl::launch_convert_f64_to_f32(s->stage, static_cast<float *>(s->fld[field]),
                                   static_cast<int>(n), s->stream);
    s->launches += 1;
    AFL_TRY(launch_check());
  }
  // The host buffer may be reused as soon as this returns.
  AFL_CUDA(cudaStreamSynchronize(s->stream));
  return AFL_OK;
}

afl_status afl_download_field(afl_solver *s, int field, double *host, size_t n) {
  AFL_TRY(check_handle(s));
  AFL_TRY(check_field(s, field, n));
  if (!host) return set_error(AFL_ERR_INVALID_ARGUMENT, "null host buffer");
  DeviceGuard guard(s->device);
  const size_t bytes = n * sizeof(double);
  const void *src = nullptr;
  if (field == AFL_FIELD_PRESSURE) {
    src = s->p;
  } else if (field == AFL_FIELD_DIVERGENCE) {
    src = s->b;
  } else if (s->precision == AFL_PRECISION_FP64) {
    src = s->fld[field];
  } else {
    afl::launch_convert_f32_to_f64(static_cast<const float *>(s->fld[field]), s->stage,
                                   static_cast<int>(n), s->stream);
    s->launches += 1;
    AFL_TRY(launch_check());
    src = s->stage;
  }
  AFL_CUDA(cudaMemcpyAsync(host, src, bytes, cudaMemcpyDeviceToHost, s->stream));
  return sync_and_check(s);
}

afl_status afl_init_velocity_noise(afl_solver *s, uint64_t seed, double lo, double hi) {
  AFL_TRY(check_handle(s));
  DeviceGuard guard(s->device);
  const size_t n = static_cast<size_t>(s->g.n);
  Xoshiro256pp rng(seed);
  std::vector<double> buf(n);
  for (int f = 0; f < 3; ++f) {
    for (size_t i = 0; i < n; ++i) buf[i] = lo + (hi - lo) * rng.next_f64();  // range_f64
    AFL_TRY(afl_upload_field(s, f, buf.data(), n));
  }
  for (int f = 3; f < 5; ++f) AFL_CUDA(cudaMemsetAsync(s->fld[f], 0, n * s->esize, s->stream));
  AFL_CUDA(cudaMemsetAsync(s->p, 0, n * sizeof(double), s->stream));
  AFL_TRY(dispatch(s, [&](auto tag) {
    using T = std::remove_pointer_t<decltype(tag)>;
    return stage_wall_bc<T>(s);
  }));
  return sync_and_check(s);
}

afl_status afl_advect_maccormack(afl_solver *s, int field_kind, double dt, double dissipation) {
  AFL_TRY(check_handle(s));
  DeviceGuard guard(s->device);
  return dispatch(s, [&](auto tag) {
    using T = std::remove_pointer_t<decltype(tag)>;
    return stage_advect<T>(s, field_kind, dt, dissipation);
  });
}

afl_status afl_enforce_wall_bc(afl_solver *s) {
  AFL_TRY(check_handle(s));
  DeviceGuard guard(s->device);
  return dispatch(s, [&](auto tag) {
    using T = std::remove_pointer_t<decltype(tag)>;
    return stage_wall_bc<T>(s);
  });
}

afl_status afl_buoyancy_vorticity(afl_solver *s, double dt) {
  AFL_TRY(check_handle(s));
  DeviceGuard guard(s->device);
  return dispatch(s, [&](auto tag) {
    using T = std::remove_pointer_t<decltype(tag)>;
    return stage_buoyancy_vorticity<T>(s, dt);
  });
}

afl_status afl_divergence_norm(afl_solver *s, double *rms) {
  AFL_TRY(check_handle(s));
  DeviceGuard guard(s->device);
  AFL_TRY(dispatch(s, [&](auto tag) {
    using T = std::remove_pointer_t<decltype(tag)>;
    return stage_divergence<T>(s);
  }));
  AFL_CUDA(cudaMemcpyAsync(s->h_scal, s->scal, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                           s->stream));
  AFL_TRY(sync_and_check(s));
  if (rms) *rms = s->h_scal[0];
  return AFL_OK;
}

static afl_status solve_common(afl_solver *s, int kind, int iters, afl_solve_info *info) {
  AFL_TRY(check_handle(s));
  if (iters < 0) return set_error(AFL_ERR_INVALID_ARGUMENT, "iteration count must be >= 0");
  DeviceGuard guard(s->device);
  AFL_TRY(ensure_run_capacity(s, 1));
  AFL_TRY(stage_solve(s, kind, iters, s->reports));
  afl::SolveReport rep{};
  AFL_CUDA(cudaMemcpyAsync(&rep, s->reports, sizeof rep, cudaMemcpyDeviceToHost, s->stream));
  AFL_TRY(sync_and_check(s));
  if (info) to_info(rep, info);
  if (kind == AFL_POISSON_CG && s->params.fail_on_not_converged && !rep.converged)
    return set_error(AFL_ERR_NOT_CONVERGED, "CG stopped at max_iters=%d without converging",
                     iters);
  return AFL_OK;
}

afl_status afl_solve_cg(afl_solver *s, int max_iters, afl_solve_info *info) {
  return solve_common(s, AFL_POISSON_CG, max_iters, info);
}

afl_status afl_solve_rbsor(afl_solver *s, int iterations, afl_solve_info *info) {
  return solve_common(s, AFL_POISSON_RBSOR, iterations, info);
}

afl_status afl_project(afl_solver *s, afl_solve_info *info) {
  AFL_TRY(check_handle(s));
  DeviceGuard guard(s->device);
  AFL_TRY(ensure_run_capacity(s, 1));
  AFL_TRY(dispatch(s, [&](auto tag) {
    using T = std::remove_pointer_t<decltype(tag)>;
    return stage_project<T>(s, true, s->reports);
  }));
  if (!info && !s->params.fail_on_not_converged) return AFL_OK;
  afl::SolveReport rep{};
  AFL_CUDA(cudaMemcpyAsync(&rep, s->reports, sizeof rep, cudaMemcpyDeviceToHost, s->stream));
  AFL_TRY(sync_and_check(s));
  if (info) to_info(rep, info);
  if (s->params.solver_kind == AFL_POISSON_CG && s->params.fail_on_not_converged &&
      !rep.converged)
    return set_error(AFL_ERR_NOT_CONVERGED, "projection CG did not converge");
  return AFL_OK;
}

afl_status afl_inject_cyberpunk(afl_solver *s, double time_sec, double dt) {
  AFL_TRY(check_handle(s));
  DeviceGuard guard(s->device);
  return dispatch(s, [&](auto tag) {
    using T = std::remove_pointer_t<decltype(tag)>;
    return stage_inject_cyberpunk<T>(s, time_sec, dt);
  });
}

afl_status afl_inject_sphere(afl_solver *s) {
  AFL_TRY(check_handle(s));
  DeviceGuard guard(s->device);
  return dispatch(s, [&](auto tag) {
    using T = std::remove_pointer_t<decltype(tag)>;
    return stage_inject_sphere<T>(s);
  });
}

afl_status afl_step(afl_solver *s, double dt, double time_sec, afl_telemetry *out,
                    afl_solve_info *info) {
  AFL_TRY(check_handle(s));
  DeviceGuard guard(s->device);
  AFL_TRY(ensure_run_capacity(s, 1));
  AFL_TRY(dispatch(s, [&](auto tag) {
    using T = std::remove_pointer_t<decltype(tag)>;
    return stage_step<T>(s, dt, time_sec, s->tel, s->reports);
  }));
  if (!out && !info) return launch_check();
  AFL_CUDA(cudaMemcpyAsync(s->h_scal, s->tel, 8 * sizeof(double), cudaMemcpyDeviceToHost,
                           s->stream));
  afl::SolveReport rep{};
  if (info)
    AFL_CUDA(cudaMemcpyAsync(&rep, s->reports, sizeof rep, cudaMemcpyDeviceToHost, s->stream));
  AFL_TRY(sync_and_check(s));
  if (out) to_telemetry(s->h_scal, out);
  if (info) to_info(rep, info);
  return AFL_OK;
}

afl_status afl_run(afl_solver *s, int steps, double dt, double t0, double dt_time,
                   afl_telemetry *telemetry, afl_solve_info *infos) {
  AFL_TRY(check_handle(s));
  if (steps < 0) return set_error(AFL_ERR_INVALID_ARGUMENT, "steps must be >= 0");
  DeviceGuard guard(s->device);
  AFL_TRY(ensure_run_capacity(s, std::max(1, steps)));
  for (int n = 0; n < steps; ++n) {
    const double t = t0 + static_cast<double>(n) * dt_time;
    AFL_TRY(dispatch(s, [&](auto tag) {
      using T = std::remove_pointer_t<decltype(tag)>;
      return stage_step<T>(s, dt, t, s->tel + 8 * static_cast<size_t>(n), s->reports + n);
    }));
  }
  std::vector<double> t8;
  std::vector<afl::SolveReport> reps;
  if (telemetry && steps > 0) {
    t8.resize(8 * static_cast<size_t>(steps));
    AFL_CUDA(cudaMemcpyAsync(t8.data(), s->tel, t8.size() * sizeof(double),
                             cudaMemcpyDeviceToHost, s->stream));
  }
  if (infos && steps > 0) {
    reps.resize(static_cast<size_t>(steps));
    AFL_CUDA(cudaMemcpyAsync(reps.data(), s->reports, reps.size() * sizeof(afl::SolveReport),
                             cudaMemcpyDeviceToHost, s->stream));
  }
  AFL_TRY(sync_and_check(s));
  for (int n = 0; n < steps; ++n) {
    if (telemetry) to_telemetry(&t8[8 * static_cast<size_t>(n)], &telemetry[n]);
    if (infos) to_info(reps[n], &infos[n]);
  }
  return AFL_OK;
}

afl_status afl_compute_telemetry(afl_solver *s, double time_sec, afl_telemetry *out) {
  AFL_TRY(check_handle(s));
  if (!out) return set_error(AFL_ERR_INVALID_ARGUMENT, "null telemetry output");
  DeviceGuard guard(s->device);
  AFL_TRY(dispatch(s, [&](auto tag) {
    using T = std::remove_pointer_t<decltype(tag)>;
    return stage_telemetry<T>(s, time_sec, s->scal + 2);
  }));
  AFL_CUDA(cudaMemcpyAsync(s->h_scal, s->scal + 2, 8 * sizeof(double), cudaMemcpyDeviceToHost,
                           s->stream));
  AFL_TRY(sync_and_check(s));
  to_telemetry(s->h_scal, out);
  return AFL_OK;
}

afl_status afl_max_density(afl_solver *s, double *out) {
  AFL_TRY(check_handle(s));
  if (!out) return set_error(AFL_ERR_INVALID_ARGUMENT, "null output");
  DeviceGuard guard(s->device);
  AFL_TRY(dispatch(s, [&](auto tag) {
    using T = std::remove_pointer_t<decltype(tag)>;
    afl::launch_max<T>(s->g, s->F<T>(3), s->partials, s->scal + 10, s->stream);
    s->launches += 2;
    return launch_check();
  }));
  AFL_CUDA(cudaMemcpyAsync(s->h_scal, s->scal + 10, sizeof(double), cudaMemcpyDeviceToHost,
                           s->stream));
  AFL_TRY(sync_and_check(s));
  *out = s->h_scal[0];
  return AFL_OK;
}

afl_status afl_medium_handoff(afl_solver *s, double *density, double *temperature, size_t n,
                              double *max_density) {
  AFL_TRY(check_handle(s));
  if (n != static_cast<size_t>(s->g.n))
    return set_error(AFL_ERR_INVALID_ARGUMENT, "length %zu != %d", n, s->g.n);
  if (density) AFL_TRY(afl_download_field(s, AFL_FIELD_DENSITY, density, n));
  if (temperature) AFL_TRY(afl_download_field(s, AFL_FIELD_TEMPERATURE, temperature, n));
  if (max_density) AFL_TRY(afl_max_density(s, max_density));
  return AFL_OK;
}

afl_status afl_sample_trilinear(afl_solver *s, int field, const double *xyz, size_t npts,
                                double *out) {
  AFL_TRY(check_handle(s));
  if (field < AFL_FIELD_U || field > AFL_FIELD_DIVERGENCE)
    return set_error(AFL_ERR_INVALID_ARGUMENT, "field id %d out of range", field);
  if (npts == 0) return AFL_OK;
  if (!xyz || !out) return set_error(AFL_ERR_INVALID_ARGUMENT, "null point/output buffer");
  if (npts > (static_cast<size_t>(1) << 28))
    return set_error(AFL_ERR_INVALID_ARGUMENT, "too many points");
  DeviceGuard guard(s->device);
  if (npts > s->sample_cap) {
    AFL_CUDA(cudaStreamSynchronize(s->stream));
    if (s->sample_buf) cudaFree(s->sample_buf);
    s->sample_buf = nullptr;
    s->sample_cap = 0;
    AFL_CUDA(cudaMalloc(&s->sample_buf, npts * 4 * sizeof(double)));
    s->sample_cap = npts;
  }
  double *d_xyz = s->sample_buf, *d_out = s->sample_buf + 3 * npts;
  AFL_CUDA(cudaMemcpyAsync(d_xyz, xyz, npts * 3 * sizeof(double), cudaMemcpyHostToDevice,
                           s->stream));
  const int np = static_cast<int>(npts);
  if (field == AFL_FIELD_PRESSURE || field == AFL_FIELD_DIVERGENCE) {
    afl::launch_sample<double>(s->g, field == AFL_FIELD_PRESSURE ? s->p : s->b, d_xyz, np,
                               d_out, s->stream);
  } else {
    AFL_TRY(dispatch(s, [&](auto tag) {
      using T = std::remove_pointer_t<decltype(tag)>;
      afl::launch_sample<T>(s->g, s->F<T>(field), d_xyz, np, d_out, s->stream);
      return AFL_OK;
    }));
  }
  s->launches += 1;
  AFL_TRY(launch_check());
  AFL_CUDA(cudaMemcpyAsync(out, d_out, npts * sizeof(double), cudaMemcpyDeviceToHost,
                           s->stream));
  return sync_and_check(s);
}

afl_status afl_synchronize(afl_solver *s) {
  AFL_TRY(check_handle(s));
  DeviceGuard guard(s->device);
  return sync_and_check(s);
}

afl_status afl_set_stage_timing(afl_solver *s, int enable) {
  AFL_TRY(check_handle(s));
  DeviceGuard guard(s->device);
  AFL_CUDA(cudaStreamSynchronize(s->stream));
  resolve_timing(s);
  for (int i = 0; i < AFL_STAGE_COUNT; ++i) {
    s->stage_ms[i] = 0.0;
    s->stage_calls[i] = 0;
  }
  s->timing = enable != 0;
  return AFL_OK;
}

afl_status afl_get_stage_timing(afl_solver *s, double *ms, int64_t *calls) {
  AFL_TRY(check_handle(s));
  DeviceGuard guard(s->device);
  AFL_CUDA(cudaStreamSynchronize(s->stream));
  resolve_timing(s);
  for (int i = 0; i < AFL_STAGE_COUNT; ++i) {
    if (ms) ms[i] = s->stage_ms[i];
    if (calls) calls[i] = s->stage_calls[i];
  }
  return AFL_OK;
}

afl_status afl_get_poisson_plan(const afl_solver *s, int32_t out[4]) {
  AFL_TRY(check_handle(s));
  if (!out) return set_error(AFL_ERR_INVALID_ARGUMENT, "null output");
  out[0] = s->resident_ok ? 1 : 0;
  out[1] = s->resident_ok ? s->resident.ty : 0;
  out[2] = s->resident_ok ? s->resident.cpt : 0;
  out[3] = s->resident_ok ? s->resident.tiles_x * s->resident.tiles_y : 0;
  return AFL_OK;
}

afl_status afl_get_launch_count(const afl_solver *s, uint64_t *count) {
  AFL_TRY(check_handle(s));
  if (!count) return set_error(AFL_ERR_INVALID_ARGUMENT, "null output");
  *count = s->launches;
  return AFL_OK;
}

void *afl_stream(afl_solver *s) { return s ? static_cast<void *>(s->stream) : nullptr; }

}  // extern "C"
