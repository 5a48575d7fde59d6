// afl_ensemble.cu -- many independent smoke plumes of different grid sizes
// advanced together (no counterpart in the reference, which runs one solver).
//
// Every stage of a step is one batched launch over all instances (block table
// -> instance descriptor -> the single-grid per-cell code), and the pressure
// solves of all instances run in one cooperative launch whose CTAs are split
// between the instances (afl_poisson_stream.cu, k_cg_stream_multi).  One step
// is captured once into a CUDA graph and replayed.  By default the whole step
// instead runs as one persistent cooperative launch (afl_ensemble_persist.cu),
// itself captured in the graph; it measured 0-5 % faster on the 48-plume
// ensemble.  The autotuner chooses the CTA split of the
// solve by timing candidate splits on a snapshot of the state, which it then
// restores.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <vector>

#include "../../include/aether_fluid.h"
#include "afl_launch.h"

namespace {

afl_status fail(afl_status st, const char *msg) {
  afl::set_last_error_text(msg);
  return st;
}

afl_status cuda_fail(cudaError_t e, const char *what) {
  char buf[256];
  snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
  return fail(e == cudaErrorMemoryAllocation ? AFL_ERR_OUT_OF_MEMORY : AFL_ERR_CUDA, buf);
}

#define ENS_CUDA(call)                              \
  do {                                              \
    cudaError_t e_ = (call);                        \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

#define ENS_TRY(expr)                \
  do {                               \
    afl_status s_ = (expr);          \
    if (s_ != AFL_OK) return s_;     \
  } while (0)

// The jets' bounding-box rule of src/fluid.rs:566-571 for the sphere source.
int box_lo(double c, double r, int n) {
  const double v = std::fmax(std::floor(c - r - 1.0), 1.0);
  return v < static_cast<double>(n) ? static_cast<int>(v) : n;
}
int box_hi(double c, double r, int n) {
  const double v = std::fmin(std::ceil(c + r + 1.0), static_cast<double>(n - 2));
  return v > 0.0 ? static_cast<int>(v) : 0;
}

// SplitMix64-seeded Xoshiro256++ (src/rng.rs:5-88).
struct Rng {
  uint64_t s[4];
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  explicit Rng(uint64_t seed) {
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

struct Bufs {
  void *fld[5] = {};
  void *tmp_fwd = nullptr, *tmp_out = nullptr;
  void *curl[4] = {};
  double *p = nullptr, *b = nullptr;
  void *cg[5] = {};
};

}  // namespace

struct afl_ensemble {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool f64 = true;
  size_t esize = 8;
  int count = 0;
  afl_params common{};
  std::vector<afl_instance> inst;
  std::vector<afl::Dims> dims;
  std::vector<Bufs> bufs;
  std::vector<void *> allocs;
  // batched stages
  void *d_inst = nullptr;  // EnsInstance<T>[count]
  int *d_blk_inst = nullptr;
  int blocks = 0;
  int kz = 1;              // z planes per stage block (tile depth)
  double *d_tel_partials = nullptr;
  int *d_step = nullptr;
  double *d_tel_out = nullptr;
  afl::SolveReport *d_reports = nullptr, *d_rep_cur = nullptr;
  int capacity = 0;
  // batched solve
  int vec = 1;
  int budget = 0;            // co-resident CTAs of the batched solve
  int budget_step = 0;       // co-resident CTAs of the persistent step kernel
  bool persistent = false;   // one persistent launch per step (default) or the stage graph
  std::vector<int> ctas;     // per instance
  afl::MultiCgSystem *d_sys = nullptr;
  int *d_cta_inst = nullptr;
  int total_ctas = 0;
  unsigned int *d_bar = nullptr;  // count/gen per instance + shared abort flag
  double *d_cg_partials = nullptr;
  // graph
  cudaGraphExec_t graph = nullptr;
  bool graph_ok = false;
  int tune_choice = -1;
  double *staging = nullptr;
};

namespace {

afl_status ens_alloc(afl_ensemble *e, void **out, size_t bytes) {
  void *p = nullptr;
  ENS_CUDA(cudaMalloc(&p, bytes));
  e->allocs.push_back(p);
  *out = p;
  return AFL_OK;
}

template <typename P>
afl_status ens_alloc_as(afl_ensemble *e, P **out, size_t bytes) {
  void *v = nullptr;
  ENS_TRY(ens_alloc(e, &v, bytes));
  *out = static_cast<P *>(v);
  return AFL_OK;
}

// Stage blocks of one instance: 32 x 8 tiles of kz z planes.
int tile_blocks(const afl::Dims &g, int kz) {
  return ((g.nx + 31) / 32) * ((g.ny + 7) / 8) * ((g.nz + kz - 1) / kz);
}

template <typename T>
afl_status build_descriptors(afl_ensemble *e, std::vector<int> &blk_inst) {
  std::vector<afl::EnsInstance<T>> h(e->count);
  blk_inst.clear();
  for (int m = 0; m < e->count; ++m) {
    const afl::Dims &g = e->dims[m];
    const afl_instance &in = e->inst[m];
    afl::EnsInstance<T> &d = h[m];
    std::memset(&d, 0, sizeof d);
    d.g = g;
    for (int f = 0; f < 5; ++f) d.fld[f] = static_cast<T *>(e->bufs[m].fld[f]);
    d.tmp_fwd = static_cast<T *>(e->bufs[m].tmp_fwd);
    d.tmp_out = static_cast<T *>(e->bufs[m].tmp_out);
    for (int f = 0; f < 4; ++f) d.curl[f] = static_cast<T *>(e->bufs[m].curl[f]);
    d.p = e->bufs[m].p;
    d.b = e->bufs[m].b;
    d.scale_f = T(in.dt / g.h);
    d.scale_b = T((-in.dt) / g.h);
    d.dt = T(in.dt);
    d.eps_h = T(in.vorticity_eps * g.h);
    d.inv_2h = T(0.5 / g.h);
    d.beta = T(in.buoyancy_beta);
    d.alpha = T(in.gravity_alpha);
    d.h = g.h;
    d.inv_h = 1.0 / g.h;
    d.dv = g.h * g.h * g.h;
    d.inv_2h_d = 0.5 / g.h;
    d.dt_time = in.dt;
    d.src_on = in.sphere_radius > 0.0 ? 1 : 0;
    const double *c = in.sphere_center;
    const double r = in.sphere_radius;
    d.src_lo[0] = box_lo(c[0], r, g.nx);
    d.src_lo[1] = box_lo(c[1], r, g.ny);
    d.src_lo[2] = box_lo(c[2], r, g.nz);
    d.src_hi[0] = box_hi(c[0], r, g.nx);
    d.src_hi[1] = box_hi(c[1], r, g.ny);
    d.src_hi[2] = box_hi(c[2], r, g.nz);
    for (int a = 0; a < 3; ++a) d.src_c[a] = c[a];
    d.src_r2 = r * r;
    d.src_rho = in.sphere_density;
    d.src_temp = in.sphere_temperature;
    d.kz = e->kz;
    d.blk_begin = static_cast<int>(blk_inst.size());
    d.blk_count = tile_blocks(g, e->kz);
    blk_inst.insert(blk_inst.end(), static_cast<size_t>(d.blk_count), m);
  }
  ENS_CUDA(cudaMemcpyAsync(e->d_inst, h.data(), sizeof(afl::EnsInstance<T>) * e->count,
                           cudaMemcpyHostToDevice, e->stream));
  ENS_CUDA(cudaStreamSynchronize(e->stream));
  return AFL_OK;
}

// Changes the tile depth of the stage kernels in place: the descriptors on the
// device keep their current field pointers (the ping-pong state); only the
// block ranges change, and the block table is rewritten.
template <typename T>
afl_status set_tile_depth_t(afl_ensemble *e, int kz) {
  std::vector<afl::EnsInstance<T>> h(e->count);
  ENS_CUDA(cudaStreamSynchronize(e->stream));
  ENS_CUDA(cudaMemcpy(h.data(), e->d_inst, sizeof(afl::EnsInstance<T>) * e->count,
                      cudaMemcpyDeviceToHost));
  std::vector<int> blk_inst;
  for (int m = 0; m < e->count; ++m) {
    h[m].kz = kz;
    h[m].blk_begin = static_cast<int>(blk_inst.size());
    h[m].blk_count = tile_blocks(e->dims[m], kz);
    blk_inst.insert(blk_inst.end(), static_cast<size_t>(h[m].blk_count), m);
  }
  ENS_CUDA(cudaMemcpy(e->d_inst, h.data(), sizeof(afl::EnsInstance<T>) * e->count,
                      cudaMemcpyHostToDevice));
  ENS_CUDA(cudaMemcpy(e->d_blk_inst, blk_inst.data(), sizeof(int) * blk_inst.size(),
                      cudaMemcpyHostToDevice));
  e->blocks = static_cast<int>(blk_inst.size());
  e->kz = kz;
  return AFL_OK;
}

afl_status set_tile_depth(afl_ensemble *e, int kz) {
  return e->f64 ? set_tile_depth_t<double>(e, kz) : set_tile_depth_t<float>(e, kz);
}

// CTA split of the batched solve: proportional to the weights, at least one
// CTA per instance, at most `budget` in total.
std::vector<int> split_ctas(const std::vector<double> &w, int budget) {
  const int n = static_cast<int>(w.size());
  std::vector<int> out(n, 1);
  const double total = std::accumulate(w.begin(), w.end(), 0.0);
  int left = budget - n;
  if (left <= 0 || total <= 0.0) return out;
  std::vector<double> frac(n);
  int used = 0;
  for (int m = 0; m < n; ++m) {
    const double share = left * w[m] / total;
    const int whole = static_cast<int>(share);
    out[m] += whole;
    used += whole;
    frac[m] = share - whole;
  }
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return frac[a] > frac[b]; });
  for (int t = 0; t < left - used && t < n; ++t) out[order[t]] += 1;
  return out;
}

// Co-resident CTAs of the launch that runs the solves in the current form.
int active_budget(const afl_ensemble *e) { return e->persistent ? e->budget_step : e->budget; }

afl_status build_systems(afl_ensemble *e, const std::vector<int> &ctas) {
  e->ctas = ctas;
  std::vector<afl::MultiCgSystem> sys(e->count);
  std::vector<int> cta_inst;
  size_t part_off = 0;
  const int nv = e->f64 ? 2 : 3;
  for (int m = 0; m < e->count; ++m) {
    afl::MultiCgSystem &s = sys[m];
    std::memset(&s, 0, sizeof s);
    const afl::Dims &g = e->dims[m];
    const Bufs &B = e->bufs[m];
    const int iters = e->common.solver_iters;
    if (e->f64) {
      s.f64 = afl::CgArgs{g, B.p, B.b, static_cast<double *>(B.cg[0]), static_cast<double *>(B.cg[1]),
                          static_cast<double *>(B.cg[2]), static_cast<double *>(B.cg[3]), iters,
                          e->common.cg_rel_tol, e->d_rep_cur + m};
    } else {
      afl::MixedCgArgs &a = s.mixed;
      a.g = g;
      a.p = B.p;
      a.b = B.b;
      a.r = static_cast<float *>(B.cg[0]);
      a.e = static_cast<float *>(B.cg[1]);
      a.d0 = static_cast<float *>(B.cg[2]);
      a.d1 = static_cast<float *>(B.cg[3]);
      a.q = static_cast<float *>(B.cg[4]);
      a.max_inner = std::max(1, e->common.mixed_inner_iters);
      a.max_total = std::max(1, iters);
      a.max_refine = e->common.mixed_max_refinements;
      a.inner_rel_tol = e->common.mixed_inner_rel_tol;
      a.rel_tol = e->common.cg_rel_tol;
      a.report = e->d_rep_cur + m;
    }
    s.gs.count = e->d_bar + 2 * m;
    s.gs.gen = e->d_bar + 2 * m + 1;
    s.gs.abort_flag = reinterpret_cast<int *>(e->d_bar + 2 * e->count);
    s.gs.nblocks = static_cast<unsigned int>(ctas[m]);
    s.gs.timeout_ns = 5000000000ull;
    s.partials = e->d_cg_partials + part_off;
    part_off += static_cast<size_t>(2 * nv * ctas[m]);
    s.cta_begin = static_cast<int>(cta_inst.size());
    s.ctas = ctas[m];
    cta_inst.insert(cta_inst.end(), static_cast<size_t>(ctas[m]), m);
  }
  e->total_ctas = static_cast<int>(cta_inst.size());
  ENS_CUDA(cudaMemcpyAsync(e->d_sys, sys.data(), sizeof(afl::MultiCgSystem) * e->count,
                           cudaMemcpyHostToDevice, e->stream));
  ENS_CUDA(cudaMemcpyAsync(e->d_cta_inst, cta_inst.data(), sizeof(int) * cta_inst.size(),
                           cudaMemcpyHostToDevice, e->stream));
  ENS_CUDA(cudaStreamSynchronize(e->stream));
  return AFL_OK;
}

template <typename T>
afl_status enqueue_step(afl_ensemble *e) {
  afl::EnsLaunch<T> L{static_cast<afl::EnsInstance<T> *>(e->d_inst), e->d_blk_inst, e->blocks,
                      e->count};
  cudaStream_t st = e->stream;
  if (e->persistent) {
    ENS_CUDA(cudaMemsetAsync(e->d_bar, 0, sizeof(unsigned int) * (2 * e->count + 1), st));
    afl::EnsStepArgs a{e->d_inst, e->d_sys,       e->d_cta_inst, e->d_tel_partials, e->d_step,
                       e->d_tel_out, e->d_rep_cur, e->d_reports,  e->count,          e->capacity};
    const int used = afl::launch_ens_step(a, e->f64, e->vec, e->total_ctas, st);
    if (used <= 0) return cuda_fail(static_cast<cudaError_t>(-used), "persistent step launch");
    afl::ens_step_advance(e->d_step, st);
    ENS_CUDA(cudaGetLastError());
    return AFL_OK;
  }
  // step (src/fluid.rs:598-611) for every instance at once
  afl::ens_advect<T>(L, 0, 0.996, st);
  afl::ens_advect<T>(L, 1, 0.996, st);
  afl::ens_advect<T>(L, 2, 0.996, st);
  afl::ens_forces<T>(L, st);  // sphere source + curl + confinement/buoyancy/wall BC
  afl::ens_divergence<T>(L, st);
  ENS_CUDA(cudaMemsetAsync(e->d_bar, 0, sizeof(unsigned int) * (2 * e->count + 1), st));
  const int used = afl::launch_cg_multi(e->d_sys, e->d_cta_inst, e->total_ctas, e->f64, e->vec, st);
  if (used <= 0)
    return cuda_fail(static_cast<cudaError_t>(-used), "batched pressure solve launch");
  afl::ens_project<T>(L, st);
  afl::ens_advect<T>(L, 3, 0.996, st);
  afl::ens_advect<T>(L, 4, 0.985, st);
  afl::ens_telemetry<T>(L, e->d_tel_partials, e->d_step, e->d_tel_out, e->d_rep_cur,
                        e->d_reports, e->capacity, st);
  afl::ens_step_advance(e->d_step, st);
  ENS_CUDA(cudaGetLastError());
  return AFL_OK;
}

afl_status enqueue(afl_ensemble *e) {
  return e->f64 ? enqueue_step<double>(e) : enqueue_step<float>(e);
}

void drop_graph(afl_ensemble *e) {
  if (e->graph) cudaGraphExecDestroy(e->graph);
  e->graph = nullptr;
  e->graph_ok = false;
}

// Captures one step into a graph; on any capture failure the steps are
// launched directly instead.
void build_graph(afl_ensemble *e) {
  drop_graph(e);
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  const afl_status st = enqueue(e);
  const cudaError_t end = cudaStreamEndCapture(e->stream, &g);
  if (st == AFL_OK && end == cudaSuccess && g) {
    if (cudaGraphInstantiate(&e->graph, g, 0) == cudaSuccess) e->graph_ok = true;
  }
  if (g) cudaGraphDestroy(g);
  cudaGetLastError();
}

afl_status ensure_capacity(afl_ensemble *e, int steps) {
  if (steps <= e->capacity) return AFL_OK;
  ENS_CUDA(cudaStreamSynchronize(e->stream));
  if (e->d_tel_out) cudaFree(e->d_tel_out);
  if (e->d_reports) cudaFree(e->d_reports);
  e->d_tel_out = nullptr;
  e->d_reports = nullptr;
  const int cap = std::max(steps, 2 * e->capacity);
  ENS_CUDA(cudaMalloc(&e->d_tel_out, sizeof(double) * 8 * static_cast<size_t>(cap) * e->count));
  ENS_CUDA(cudaMalloc(&e->d_reports,
                      sizeof(afl::SolveReport) * static_cast<size_t>(cap) * e->count));
  e->capacity = cap;
  build_graph(e);  // the step writes into the new buffers
  return AFL_OK;
}

template <typename T>
afl_status init_instance(afl_ensemble *e, int m) {
  const afl::Dims &g = e->dims[m];
  const afl_instance &in = e->inst[m];
  const size_t n = static_cast<size_t>(g.n);
  Rng rng(in.seed);
  std::vector<double> buf(n);
  std::vector<T> conv(n);
  for (int f = 0; f < 3; ++f) {
    for (size_t c = 0; c < n; ++c)
      buf[c] = in.noise_lo + (in.noise_hi - in.noise_lo) * rng.next_f64();  // range_f64
    for (size_t c = 0; c < n; ++c) conv[c] = T(buf[c]);
    ENS_CUDA(cudaMemcpyAsync(e->bufs[m].fld[f], conv.data(), n * sizeof(T), cudaMemcpyHostToDevice,
                             e->stream));
    ENS_CUDA(cudaStreamSynchronize(e->stream));
  }
  for (int f = 3; f < 5; ++f) ENS_CUDA(cudaMemsetAsync(e->bufs[m].fld[f], 0, n * sizeof(T), e->stream));
  ENS_CUDA(cudaMemsetAsync(e->bufs[m].p, 0, n * sizeof(double), e->stream));
  afl::launch_wall_bc<T>(g, static_cast<T *>(e->bufs[m].fld[0]), static_cast<T *>(e->bufs[m].fld[1]),
                         static_cast<T *>(e->bufs[m].fld[2]), e->stream);
  ENS_CUDA(cudaGetLastError());
  return AFL_OK;
}

// Current device pointer of field f of instance m (the ping-pong moves it).
afl_status current_field(afl_ensemble *e, int m, int f, void **out) {
  if (f == AFL_FIELD_PRESSURE) { *out = e->bufs[m].p; return AFL_OK; }
  if (f == AFL_FIELD_DIVERGENCE) { *out = e->bufs[m].b; return AFL_OK; }
  const size_t stride = e->f64 ? sizeof(afl::EnsInstance<double>) : sizeof(afl::EnsInstance<float>);
  const size_t off = e->f64 ? offsetof(afl::EnsInstance<double>, fld) : offsetof(afl::EnsInstance<float>, fld);
  void *ptr = nullptr;
  ENS_CUDA(cudaMemcpy(&ptr, static_cast<char *>(e->d_inst) + stride * m + off + sizeof(void *) * f,
                      sizeof ptr, cudaMemcpyDeviceToHost));
  *out = ptr;
  return AFL_OK;
}

afl_status sync_status(afl_ensemble *e) {
  ENS_CUDA(cudaStreamSynchronize(e->stream));
  unsigned int abort_flag = 0;
  ENS_CUDA(cudaMemcpy(&abort_flag, e->d_bar + 2 * e->count, sizeof abort_flag,
                      cudaMemcpyDeviceToHost));
  if (abort_flag) return fail(AFL_ERR_TIMEOUT, "the batched pressure solve gave up at a grid barrier");
  return AFL_OK;
}

}  // namespace

extern "C" {

afl_status afl_rng_f64(uint64_t seed, uint64_t skip, size_t n, double *out) {
  if (n && !out) return fail(AFL_ERR_INVALID_ARGUMENT, "null output");
  Rng rng(seed);
  for (uint64_t s = 0; s < skip; ++s) rng.next();
  for (size_t i = 0; i < n; ++i) out[i] = rng.next_f64();
  return AFL_OK;
}

afl_status afl_ensemble_create(const afl_instance *inst, int count, const afl_params *common,
                               afl_ensemble **out) {
  if (!out || !inst || count < 1) return fail(AFL_ERR_INVALID_ARGUMENT, "need count >= 1 instances");
  *out = nullptr;
  afl_params p;
  if (common) p = *common; else afl_params_default(&p);
  if (p.solver_kind != AFL_POISSON_CG)
    return fail(AFL_ERR_INVALID_ARGUMENT, "the ensemble solves pressure with CG only");
  if (p.precision != AFL_PRECISION_FP64 && p.precision != AFL_PRECISION_MIXED)
    return fail(AFL_ERR_INVALID_ARGUMENT, "precision must be 0 or 1");
  for (int m = 0; m < count; ++m) {
    if (inst[m].nx < 6 || inst[m].ny < 6 || inst[m].nz < 6)
      return fail(AFL_ERR_INVALID_ARGUMENT, "every instance dimension must be >= 6");
    if (inst[m].nx * inst[m].ny * inst[m].nz > (static_cast<size_t>(1) << 28))
      return fail(AFL_ERR_INVALID_ARGUMENT, "instance grid too large");
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(AFL_ERR_CUDA, "no CUDA device available; this library has no CPU path");
  }
  auto *e = new afl_ensemble();
  auto bail = [&](afl_status st) {
    afl_ensemble_destroy(e);
    return st;
  };
  cudaGetDevice(&e->device);
  e->common = p;
  e->f64 = p.precision == AFL_PRECISION_FP64;
  e->esize = e->f64 ? sizeof(double) : sizeof(float);
  e->count = count;
  e->inst.assign(inst, inst + count);
  if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(AFL_ERR_CUDA, "cudaStreamCreate failed"));
  e->dims.resize(count);
  e->bufs.resize(count);
  bool all_vec = true;
  const int want_vec = e->f64 ? 2 : 4;
  size_t max_n = 0;
  for (int m = 0; m < count; ++m) {
    afl::Dims &g = e->dims[m];
    g.nx = static_cast<int>(inst[m].nx);
    g.ny = static_cast<int>(inst[m].ny);
    g.nz = static_cast<int>(inst[m].nz);
    g.nxy = g.nx * g.ny;
    g.n = g.nxy * g.nz;
    g.h = 1.0 / static_cast<double>(std::max(g.nx, std::max(g.ny, g.nz)));
    if (g.nx % want_vec) all_vec = false;
    max_n = std::max(max_n, static_cast<size_t>(g.n));
    const size_t fb = static_cast<size_t>(g.n) * e->esize;
    Bufs &B = e->bufs[m];
    afl_status st = AFL_OK;
    for (int f = 0; f < 5 && st == AFL_OK; ++f) st = ens_alloc(e, &B.fld[f], fb);
    if (st == AFL_OK) st = ens_alloc(e, &B.tmp_fwd, fb);
    if (st == AFL_OK) st = ens_alloc(e, &B.tmp_out, fb);
    for (int f = 0; f < 4 && st == AFL_OK; ++f) st = ens_alloc(e, &B.curl[f], fb);
    if (st == AFL_OK) st = ens_alloc_as(e, &B.p, static_cast<size_t>(g.n) * sizeof(double));
    if (st == AFL_OK) st = ens_alloc_as(e, &B.b, static_cast<size_t>(g.n) * sizeof(double));
    const int ncg = e->f64 ? 4 : 5;
    for (int f = 0; f < ncg && st == AFL_OK; ++f) st = ens_alloc(e, &B.cg[f], fb);
    if (st != AFL_OK) return bail(st);
  }
  e->vec = all_vec ? want_vec : 1;
  afl_status st = ens_alloc(e, &e->d_inst, (e->f64 ? sizeof(afl::EnsInstance<double>)
                                                   : sizeof(afl::EnsInstance<float>)) * count);
  if (st == AFL_OK) st = ens_alloc_as(e, &e->d_rep_cur, sizeof(afl::SolveReport) * count);
  if (st == AFL_OK) st = ens_alloc_as(e, &e->d_step, sizeof(int));
  if (st == AFL_OK) st = ens_alloc_as(e, &e->d_bar, sizeof(unsigned int) * (2 * count + 1));
  if (st == AFL_OK) st = ens_alloc_as(e, &e->d_sys, sizeof(afl::MultiCgSystem) * count);
  if (st == AFL_OK) st = ens_alloc_as(e, &e->staging, max_n * sizeof(double));
  if (st != AFL_OK) return bail(st);
  // initial condition of every instance
  for (int m = 0; m < count && st == AFL_OK; ++m)
    st = e->f64 ? init_instance<double>(e, m) : init_instance<float>(e, m);
  if (st != AFL_OK) return bail(st);
  std::vector<int> blk_inst;
  st = e->f64 ? build_descriptors<double>(e, blk_inst) : build_descriptors<float>(e, blk_inst);
  if (st != AFL_OK) return bail(st);
  e->blocks = static_cast<int>(blk_inst.size());
  st = ens_alloc_as(e, &e->d_blk_inst, sizeof(int) * blk_inst.size());
  if (st == AFL_OK) st = ens_alloc_as(e, &e->d_tel_partials, sizeof(double) * 7 * blk_inst.size());
  if (st != AFL_OK) return bail(st);
  cudaMemcpy(e->d_blk_inst, blk_inst.data(), sizeof(int) * blk_inst.size(), cudaMemcpyHostToDevice);
  cudaMemset(e->d_step, 0, sizeof(int));
  // batched solve: every CTA co-resident; at least one CTA per instance
  e->budget = afl::persistent_blocks_multi(e->f64, e->vec);
  e->budget_step = afl::persistent_blocks_ens_step(e->f64, e->vec);
  if (e->budget < count)
    return bail(fail(AFL_ERR_INVALID_ARGUMENT, "more instances than co-resident solver CTAs"));
  const int nv = e->f64 ? 2 : 3;
  const int most = std::max(e->budget, e->budget_step);
  st = ens_alloc_as(e, &e->d_cta_inst, sizeof(int) * most);
  if (st == AFL_OK) st = ens_alloc_as(e, &e->d_cg_partials, sizeof(double) * 2 * nv * most);
  if (st != AFL_OK) return bail(st);
  std::vector<double> w(count);
  for (int m = 0; m < count; ++m) w[m] = static_cast<double>(e->dims[m].n);
  // the persistent step is the default form when every instance gets a CTA
  e->persistent = e->budget_step >= count;
  st = build_systems(e, split_ctas(w, active_budget(e)));
  if (st == AFL_OK) st = ensure_capacity(e, 1);
  if (st != AFL_OK) return bail(st);
  if (!e->graph_ok) build_graph(e);
  *out = e;
  return AFL_OK;
}

afl_status afl_ensemble_destroy(afl_ensemble *e) {
  if (!e) return AFL_OK;
  if (e->stream) cudaStreamSynchronize(e->stream);
  drop_graph(e);
  for (void *p : e->allocs) cudaFree(p);
  if (e->d_tel_out) cudaFree(e->d_tel_out);
  if (e->d_reports) cudaFree(e->d_reports);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return AFL_OK;
}

afl_status afl_ensemble_run(afl_ensemble *e, int steps, afl_telemetry *telemetry,
                            afl_solve_info *infos) {
  if (!e) return fail(AFL_ERR_INVALID_ARGUMENT, "null ensemble");
  if (steps < 0) return fail(AFL_ERR_INVALID_ARGUMENT, "steps must be >= 0");
  ENS_TRY(ensure_capacity(e, std::max(1, steps)));
  ENS_CUDA(cudaMemsetAsync(e->d_step, 0, sizeof(int), e->stream));
  for (int n = 0; n < steps; ++n) {
    if (e->graph_ok) {
      ENS_CUDA(cudaGraphLaunch(e->graph, e->stream));
    } else {
      ENS_TRY(enqueue(e));
    }
  }
  ENS_TRY(sync_status(e));
  const size_t rows = static_cast<size_t>(steps) * e->count;
  if (telemetry && rows) {
    std::vector<double> t8(rows * 8);
    ENS_CUDA(cudaMemcpy(t8.data(), e->d_tel_out, t8.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (size_t r = 0; r < rows; ++r) {
      afl_telemetry &t = telemetry[r];
      t.time_sec = t8[8 * r];
      t.kinetic_energy = t8[8 * r + 1];
      t.enstrophy = t8[8 * r + 2];
      t.peak_vorticity = t8[8 * r + 3];
      t.total_mass = t8[8 * r + 4];
      for (int a = 0; a < 3; ++a) t.center_of_mass[a] = t8[8 * r + 5 + a];
    }
  }
  if (infos && rows) {
    std::vector<afl::SolveReport> reps(rows);
    ENS_CUDA(cudaMemcpy(reps.data(), e->d_reports, rows * sizeof(afl::SolveReport),
                        cudaMemcpyDeviceToHost));
    for (size_t r = 0; r < rows; ++r) {
      infos[r].iterations = reps[r].iterations;
      infos[r].refinements = reps[r].refinements;
      infos[r].converged = reps[r].converged;
      infos[r].status = reps[r].status;
      infos[r].initial_residual = reps[r].initial_residual;
      infos[r].final_residual = reps[r].final_residual;
      infos[r].rhs_norm = reps[r].rhs_norm;
    }
  }
  return AFL_OK;
}

afl_status afl_ensemble_download_field(afl_ensemble *e, int instance, int field, double *host,
                                       size_t n) {
  if (!e || !host) return fail(AFL_ERR_INVALID_ARGUMENT, "null ensemble or buffer");
  if (instance < 0 || instance >= e->count) return fail(AFL_ERR_INVALID_ARGUMENT, "bad instance");
  if (field < AFL_FIELD_U || field > AFL_FIELD_DIVERGENCE)
    return fail(AFL_ERR_INVALID_ARGUMENT, "bad field id");
  if (n != static_cast<size_t>(e->dims[instance].n))
    return fail(AFL_ERR_INVALID_ARGUMENT, "length does not match the instance grid");
  ENS_CUDA(cudaStreamSynchronize(e->stream));
  void *src = nullptr;
  ENS_TRY(current_field(e, instance, field, &src));
  if (field >= AFL_FIELD_PRESSURE || e->f64) {
    ENS_CUDA(cudaMemcpy(host, src, n * sizeof(double), cudaMemcpyDeviceToHost));
  } else {
    afl::launch_convert_f32_to_f64(static_cast<const float *>(src), e->staging,
                                   static_cast<int>(n), e->stream);
    ENS_CUDA(cudaGetLastError());
    ENS_CUDA(cudaMemcpyAsync(host, e->staging, n * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    ENS_CUDA(cudaStreamSynchronize(e->stream));
  }
  return AFL_OK;
}

// Times candidate layouts, one step each (after one untimed step), on a
// snapshot of the state that is restored before every candidate and at the
// end; keeps the fastest.  Candidates: CTA splits of the batched solve --
// proportional to cells, proportional to cells x observed iterations, and the
// cell split on 3/4 of the co-resident CTAs -- and then, with the best split,
// stage tiles of 2 and 4 z planes besides 1.
afl_status afl_ensemble_autotune(afl_ensemble *e, int32_t *choice) {
  if (!e) return fail(AFL_ERR_INVALID_ARGUMENT, "null ensemble");
  ENS_CUDA(cudaStreamSynchronize(e->stream));
  const int kz0 = e->kz;
  const size_t desc_bytes = (e->f64 ? sizeof(afl::EnsInstance<double>)
                                    : sizeof(afl::EnsInstance<float>)) * e->count;
  std::vector<char> desc(desc_bytes);
  ENS_CUDA(cudaMemcpy(desc.data(), e->d_inst, desc_bytes, cudaMemcpyDeviceToHost));
  // snapshot: the five current fields and the pressure of every instance
  std::vector<void *> snap;
  std::vector<std::pair<void *, size_t>> live;
  for (int m = 0; m < e->count; ++m) {
    for (int f = 0; f < 6; ++f) {
      void *src = nullptr;
      ENS_TRY(current_field(e, m, f, &src));
      const size_t bytes = static_cast<size_t>(e->dims[m].n) * (f == 5 ? sizeof(double) : e->esize);
      void *dst = nullptr;
      const cudaError_t err = cudaMalloc(&dst, bytes);
      if (err != cudaSuccess) {
        for (void *sp : snap) cudaFree(sp);
        return cuda_fail(err, "autotune snapshot");
      }
      cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToDevice);
      snap.push_back(dst);
      live.push_back({src, bytes});
    }
  }
  // the state and the descriptors as they were (tile depth kz0)
  auto restore = [&]() {
    for (size_t k = 0; k < snap.size(); ++k)
      cudaMemcpy(live[k].first, snap[k], live[k].second, cudaMemcpyDeviceToDevice);
    cudaMemcpy(e->d_inst, desc.data(), desc_bytes, cudaMemcpyHostToDevice);
    cudaMemset(e->d_step, 0, sizeof(int));
  };
  std::vector<double> cells(e->count), work(e->count);
  for (int m = 0; m < e->count; ++m) cells[m] = static_cast<double>(e->dims[m].n);
  std::vector<std::vector<int>> cands;
  const int budget = active_budget(e);
  cands.push_back(split_ctas(cells, budget));
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  // one timed step of (split, tile depth); restores the state first
  auto time_one = [&](const std::vector<int> &split, int kz, float *ms) -> afl_status {
    ENS_TRY(build_systems(e, split));
    restore();
    ENS_TRY(set_tile_depth(e, kz));
    ENS_TRY(enqueue(e));  // untimed
    cudaEventRecord(t0, e->stream);
    ENS_TRY(enqueue(e));
    cudaEventRecord(t1, e->stream);
    ENS_TRY(sync_status(e));
    cudaEventElapsedTime(ms, t0, t1);
    return AFL_OK;
  };
  float best_ms = 1e30f;
  int best = 0, best_kz = kz0;
  afl_status st = AFL_OK;
  for (size_t c = 0; c < 3 && st == AFL_OK; ++c) {
    if (c == 1) cands.push_back(split_ctas(work, budget));
    if (c == 2) cands.push_back(split_ctas(cells, std::max(e->count, (3 * budget) / 4)));
    float ms = 0.0f;
    st = time_one(cands[c], 1, &ms);
    if (st != AFL_OK) break;
    if (c == 0) {  // observed iterations of the timed step
      std::vector<afl::SolveReport> reps(e->count);
      cudaMemcpy(reps.data(), e->d_rep_cur, sizeof(afl::SolveReport) * e->count,
                 cudaMemcpyDeviceToHost);
      for (int m = 0; m < e->count; ++m)
        work[m] = cells[m] * std::max(1, reps[m].iterations + reps[m].refinements);
    }
    if (ms < best_ms) {
      best_ms = ms;
      best = static_cast<int>(c);
      best_kz = 1;
    }
  }
  for (int kz : {2, 4}) {
    if (st != AFL_OK) break;
    float ms = 0.0f;
    st = time_one(cands[best], kz, &ms);
    if (st == AFL_OK && ms < best_ms) {
      best_ms = ms;
      best_kz = kz;
    }
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  restore();
  for (void *sp : snap) cudaFree(sp);
  e->kz = kz0;  // the restored descriptors carry kz0
  if (st != AFL_OK) {
    set_tile_depth(e, kz0);  // the block table of the last candidate goes too
    build_graph(e);
    return st;
  }
  ENS_TRY(build_systems(e, cands[best]));
  ENS_TRY(set_tile_depth(e, best_kz));
  build_graph(e);
  e->tune_choice = best;
  if (choice) *choice = best;
  return AFL_OK;
}

afl_status afl_ensemble_set_tile_depth(afl_ensemble *e, int32_t kz) {
  if (!e) return fail(AFL_ERR_INVALID_ARGUMENT, "null ensemble");
  if (kz != 1 && kz != 2 && kz != 4) return fail(AFL_ERR_INVALID_ARGUMENT, "tile depth must be 1, 2 or 4");
  ENS_TRY(set_tile_depth(e, kz));
  build_graph(e);
  return AFL_OK;
}

afl_status afl_ensemble_tile_depth(const afl_ensemble *e, int32_t *kz) {
  if (!e || !kz) return fail(AFL_ERR_INVALID_ARGUMENT, "null argument");
  *kz = e->kz;
  return AFL_OK;
}

afl_status afl_ensemble_set_persistent(afl_ensemble *e, int32_t on) {
  if (!e) return fail(AFL_ERR_INVALID_ARGUMENT, "null ensemble");
  if (on != 0 && on != 1) return fail(AFL_ERR_INVALID_ARGUMENT, "step form must be 0 or 1");
  if (on && e->budget_step < e->count)
    return fail(AFL_ERR_INVALID_ARGUMENT, "more instances than co-resident step-kernel CTAs");
  ENS_CUDA(cudaStreamSynchronize(e->stream));
  e->persistent = on != 0;
  std::vector<double> w(e->count);
  for (int m = 0; m < e->count; ++m) w[m] = static_cast<double>(e->dims[m].n);
  ENS_TRY(build_systems(e, split_ctas(w, active_budget(e))));
  e->tune_choice = -1;
  build_graph(e);
  return AFL_OK;
}

afl_status afl_ensemble_persistent(const afl_ensemble *e, int32_t *on) {
  if (!e || !on) return fail(AFL_ERR_INVALID_ARGUMENT, "null argument");
  *on = e->persistent ? 1 : 0;
  return AFL_OK;
}

afl_status afl_ensemble_info(const afl_ensemble *e, int32_t out[6]) {
  if (!e || !out) return fail(AFL_ERR_INVALID_ARGUMENT, "null argument");
  out[0] = e->count;
  out[1] = e->graph_ok ? 1 : 0;
  out[2] = e->total_ctas;
  out[3] = active_budget(e);
  out[4] = e->vec;
  out[5] = e->tune_choice;
  return AFL_OK;
}

afl_status afl_ensemble_instance_ctas(const afl_ensemble *e, int32_t *out, int count) {
  if (!e || !out || count != e->count) return fail(AFL_ERR_INVALID_ARGUMENT, "bad arguments");
  for (int m = 0; m < count; ++m) out[m] = e->ctas[m];
  return AFL_OK;
}

}  // extern "C"
