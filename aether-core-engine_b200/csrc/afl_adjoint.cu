// afl_adjoint.cu -- checkpointed reverse mode through the FP64 smoke step.
//
// No counterpart in the reference.  Controls: the initial velocity (u, v, w)
// and the per-cell temperature amplitude of the sphere source; output: the
// density after `steps` steps.  The step's source is the sphere, the
// reference's cyberpunk jets (inject_cyberpunk_sources at time n*dt of step
// n; their caps are recorded) or none; its pressure solve is CG (taken as an
// exact solve) or red-black SOR with a fixed sweep count (transposed sweep by
// sweep; the warm start carries an adjoint from step to step).  The forward keeps the state every k steps.
// The backward walks the segments from the last: it restores the segment's
// checkpoint, recomputes the segment's steps recording each stage's inputs,
// forward-sample arrays and MacCormack clamp masks (k_advect_mc_record, the
// same arithmetic as the plain forward), then applies the stage adjoints of
// afl_adjoint_kernels.cu step by step in reverse.  The adjoint pressure solve
// uses the same symmetric-operator CG (solves taken as exact).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/aether_fluid.h"
#include "afl_launch.h"

namespace afl {
void adj_advect_mc_record(const Dims &g, const double *u, const double *v, const double *w,
                          const double *src, const double *fwd, double *out, double dt,
                          double diss, bool nonneg, unsigned char *mask, cudaStream_t st);
void adj_advect_bwd(const Dims &g, const double *u, const double *v, const double *w,
                    const double *src, const double *fwd, const unsigned char *mask, double dt,
                    double diss, bool nonneg, const double *ob, double *fb, double *sb,
                    double *ub, double *vb, double *wb, cudaStream_t st);
void adj_source_bwd(const Dims &g, const int lo[3], const int hi[3], const double c[3], double r2,
                    double temp_val, double *rhob, double *tempb, double *ampb, cudaStream_t st);
void adj_confine_bwd(const Dims &g, const double *cx, const double *cy, const double *cz,
                     const double *cm, const double *u2b, const double *v2b, const double *w2b,
                     double dt, double eps, double beta, double alpha, double *gb[3],
                     double *ob[3], double *u1b, double *v1b, double *w1b, double *rhob,
                     double *tempb, cudaStream_t st);
void adj_project_bwd_p(const Dims &g, double *u3b, double *v3b, double *w3b, double *pb,
                       cudaStream_t st);
void adj_project_bwd_b(const Dims &g, const double *u3b, const double *v3b, const double *w3b,
                       const double *bb, double *u2b, double *v2b, double *w2b, cudaStream_t st);
void adj_jet_record(const Dims &g, double time_sec, double dt, double *rho, double *temp,
                    double *u, double *v, double *w, unsigned char *mask, cudaStream_t st);
void adj_jet_bwd(const Dims &g, const unsigned char *mask, double *rhob, double *tempb,
                 cudaStream_t st);
void adj_sor_bwd(const Dims &g, int sweeps, double omega, double *pb, double *bb,
                 cudaStream_t st);
void adj_add(const Dims &g, const double *x, double *y, cudaStream_t st);
}  // namespace afl

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

#define ADJ_CUDA(call)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)
#define ADJ_TRY(expr)              \
  do {                             \
    afl_status s_ = (expr);        \
    if (s_ != AFL_OK) return s_;   \
  } while (0)

int box_lo(double c, double r, int n) {
  const double v = std::fmax(std::floor(c - r - 1.0), 1.0);
  return v < static_cast<double>(n) ? static_cast<int>(v) : n;
}
int box_hi(double c, double r, int n) {
  const double v = std::fmin(std::ceil(c + r + 1.0), static_cast<double>(n - 2));
  return v > 0.0 ? static_cast<int>(v) : 0;
}

// Everything one step's adjoint needs from its forward.
struct Rec {
  double *u0, *v0, *w0;        // input velocity
  double *u1, *v1, *w1;        // after the three velocity advections
  double *rhos, *temps;        // density/temperature after the source
  double *u3, *v3, *w3;        // after projection (advects the scalars)
  double *u1s, *v1s, *w1s;     // jets: the velocity after the source (the curl's input)
  unsigned char *jmask;        // jets: the caps each cell's density/temperature reached
  double *fwd[5];              // semi-Lagrangian samples of the five advections
  unsigned char *mask[5];      // MacCormack branch of every cell
};

}  // namespace

struct afl_adjoint {
  int device = 0;
  cudaStream_t stream = nullptr;
  afl::Dims g{};
  afl_params params{};
  int k = 8;
  int steps = 0;
  double dt = 0.0;
  std::vector<void *> allocs;
  double *F[5] = {};  // u, v, w, density, temperature (ping-pong with tmp_out)
  double *p = nullptr, *b = nullptr, *tmp_fwd = nullptr, *tmp_out = nullptr;
  double *curl[4] = {}, *cg[4] = {};
  double *amp = nullptr;
  double *partials = nullptr, *scal = nullptr;
  afl::SolveReport *rep = nullptr;
  afl::PersistentState ps{};
  afl::ResidentPlan res{};  // on-chip CG tiles, when the grid fits
  bool resident = false;
  std::vector<std::array<double *, 6>> ckpt;
  std::vector<Rec> rec;
  // adjoint work arrays
  double *ub0 = nullptr, *vb0 = nullptr, *wb0 = nullptr, *rhob = nullptr, *tempb = nullptr;
  double *ub1 = nullptr, *vb1 = nullptr, *wb1 = nullptr, *ub2 = nullptr, *vb2 = nullptr,
         *wb2 = nullptr;
  double *rhobs = nullptr, *tempbs = nullptr, *fb = nullptr, *pb = nullptr, *bb = nullptr;
  double *gb[3] = {}, *ob[3] = {};
  double *ampb = nullptr;
  double *pcarry = nullptr;  // SOR: the adjoint of the next step's warm start
  int src_lo[3] = {}, src_hi[3] = {};
  float fwd_ms = 0.0f, bwd_ms = 0.0f;
  long fwd_iters = 0, adj_iters = 0;
  bool have_forward = false;
};

namespace {

size_t nbytes(const afl_adjoint *a) { return static_cast<size_t>(a->g.n) * sizeof(double); }

afl_status dalloc(afl_adjoint *a, double **out) {
  void *p = nullptr;
  ADJ_CUDA(cudaMalloc(&p, nbytes(a)));
  a->allocs.push_back(p);
  *out = static_cast<double *>(p);
  return AFL_OK;
}

afl_status balloc(afl_adjoint *a, unsigned char **out) {
  void *p = nullptr;
  ADJ_CUDA(cudaMalloc(&p, static_cast<size_t>(a->g.n)));
  a->allocs.push_back(p);
  *out = static_cast<unsigned char *>(p);
  return AFL_OK;
}

afl_status zero(afl_adjoint *a, double *x) {
  ADJ_CUDA(cudaMemsetAsync(x, 0, nbytes(a), a->stream));
  return AFL_OK;
}

afl_status copy(afl_adjoint *a, double *dst, const double *src) {
  ADJ_CUDA(cudaMemcpyAsync(dst, src, nbytes(a), cudaMemcpyDeviceToDevice, a->stream));
  return AFL_OK;
}

// The FP64 CG of afl_solve_cg (warm start from x): the on-chip resident
// kernel when the grid fits, else the streaming one.
afl_status solve(afl_adjoint *a, double *x, const double *rhs, long *iters) {
  int used;
  if (a->params.solver_kind == AFL_POISSON_RBSOR) {
    afl::SorArgs sa{a->g, x, rhs, a->params.solver_iters, a->params.sor_omega, a->rep};
    used = afl::launch_rbsor_f64(sa, a->ps, a->stream);
  } else if (a->resident) {
    afl::ResidentCgArgs ra{};
    ra.g = a->g;
    ra.p = x;
    ra.b = rhs;
    ra.rpub = a->cg[0];
    ra.max_iters = a->params.solver_iters;
    ra.rel_tol = a->params.cg_rel_tol;
    ra.report = a->rep;
    used = afl::launch_cg_resident(ra, a->res, true, a->ps, a->stream);
  } else {
    afl::CgArgs args{a->g, x, rhs, a->cg[0], a->cg[1], a->cg[2], a->cg[3],
                     a->params.solver_iters, a->params.cg_rel_tol, a->rep};
    used = afl::launch_cg_f64(args, a->ps, a->stream);
  }
  if (used <= 0) return cuda_fail(static_cast<cudaError_t>(-used), "CG launch");
  afl::SolveReport r{};
  ADJ_CUDA(cudaMemcpyAsync(&r, a->rep, sizeof r, cudaMemcpyDeviceToHost, a->stream));
  ADJ_CUDA(cudaStreamSynchronize(a->stream));
  int abort_flag = 0;
  ADJ_CUDA(cudaMemcpy(&abort_flag, a->ps.abort_flag, sizeof abort_flag, cudaMemcpyDeviceToHost));
  if (abort_flag) return fail(AFL_ERR_TIMEOUT, "the CG kernel gave up at a grid barrier");
  if (r.status != 0) return fail(AFL_ERR_NONFINITE, "non-finite residual in a CG solve");
  *iters += r.iterations;
  return AFL_OK;
}

bool jets(const afl_adjoint *a) { return a->params.source_kind == AFL_SOURCE_CYBERPUNK; }
bool sphere_on(const afl_adjoint *a) { return a->params.source_kind == AFL_SOURCE_SPHERE; }

// The step's source on (rho, temp, u, v, w); step n runs at time n*dt.
void source(afl_adjoint *a, int step, double *rho, double *temp, double *u, double *v,
            double *w) {
  if (sphere_on(a)) {
    afl::launch_inject_sphere<double>(a->g, a->src_lo, a->src_hi, rho, temp, a->amp,
                                      a->params.sphere_center,
                                      a->params.sphere_radius * a->params.sphere_radius,
                                      a->params.sphere_density, a->params.sphere_temperature,
                                      a->stream);
  } else if (jets(a)) {
    const afl::JetPair jp = afl::cyberpunk_jets(a->g, step * a->dt);
    for (int q = 0; q < 2; ++q)
      afl::launch_inject_jet<double>(a->g, jp.lo[q], jp.hi[q], rho, temp, u, v, w, jp.jet[q],
                                     jp.r2, a->dt, jp.pulse, a->stream);
  }
}

// One plain FP64 step (src/fluid.rs:598-611), state in F/p.
afl_status step_plain(afl_adjoint *a, int step) {
  const afl::Dims &g = a->g;
  for (int f = 0; f < 5; ++f) {
    if (f == 3) {
      source(a, step, a->F[3], a->F[4], a->F[0], a->F[1], a->F[2]);
      afl::launch_curl<double>(g, a->F[0], a->F[1], a->F[2], a->curl[0], a->curl[1], a->curl[2],
                               a->curl[3], a->stream);
      afl::launch_confine_buoy<double>(g, a->F[0], a->F[1], a->F[2], a->F[3], a->F[4], a->curl[0],
                                       a->curl[1], a->curl[2], a->curl[3], a->dt,
                                       a->params.vorticity_eps, a->params.buoyancy_beta,
                                       a->params.gravity_alpha, a->stream);
      afl::launch_divergence<double>(g, a->F[0], a->F[1], a->F[2], a->b, a->partials, a->scal,
                                     a->stream);
      ADJ_TRY(solve(a, a->p, a->b, &a->fwd_iters));
      afl::launch_project<double>(g, a->F[0], a->F[1], a->F[2], a->p, a->stream);
    }
    afl::launch_advect_fwd<double>(g, a->F[0], a->F[1], a->F[2], a->F[f], a->tmp_fwd, a->dt,
                                   a->stream);
    afl::launch_advect_mc<double>(g, a->F[0], a->F[1], a->F[2], a->F[f], a->tmp_fwd, a->tmp_out,
                                  a->dt, f == 4 ? 0.985 : 0.996, f >= 3, a->stream);
    std::swap(a->F[f], a->tmp_out);
  }
  ADJ_CUDA(cudaGetLastError());
  return AFL_OK;
}

// The same step, keeping what its adjoint needs in R.
afl_status step_record(afl_adjoint *a, Rec &R, int step) {
  const afl::Dims &g = a->g;
  cudaStream_t st = a->stream;
  ADJ_TRY(copy(a, R.u0, a->F[0]));
  ADJ_TRY(copy(a, R.v0, a->F[1]));
  ADJ_TRY(copy(a, R.w0, a->F[2]));
  const double *vel_u[3] = {R.u0, R.v0, R.w0};
  double *outs[3] = {R.u1, R.v1, R.w1};
  const double *srcs[3] = {R.u0, R.v0, R.w0};
  for (int f = 0; f < 3; ++f) {
    // velocity used by component f: components before f are already advected
    const double *vu = f > 0 ? R.u1 : vel_u[0];
    const double *vv = f > 1 ? R.v1 : vel_u[1];
    const double *vw = vel_u[2];
    afl::launch_advect_fwd<double>(g, vu, vv, vw, srcs[f], R.fwd[f], a->dt, st);
    afl::adj_advect_mc_record(g, vu, vv, vw, srcs[f], R.fwd[f], outs[f], a->dt, 0.996, false,
                              R.mask[f], st);
  }
  ADJ_TRY(copy(a, R.rhos, a->F[3]));
  ADJ_TRY(copy(a, R.temps, a->F[4]));
  ADJ_TRY(copy(a, R.u3, R.u1));
  ADJ_TRY(copy(a, R.v3, R.v1));
  ADJ_TRY(copy(a, R.w3, R.w1));
  if (jets(a)) {
    ADJ_CUDA(cudaMemsetAsync(R.jmask, 0, static_cast<size_t>(g.n), st));
    afl::adj_jet_record(g, step * a->dt, a->dt, R.rhos, R.temps, R.u3, R.v3, R.w3, R.jmask, st);
    ADJ_TRY(copy(a, R.u1s, R.u3));
    ADJ_TRY(copy(a, R.v1s, R.v3));
    ADJ_TRY(copy(a, R.w1s, R.w3));
  } else {
    source(a, step, R.rhos, R.temps, R.u3, R.v3, R.w3);
  }
  afl::launch_curl<double>(g, R.u3, R.v3, R.w3, a->curl[0], a->curl[1], a->curl[2], a->curl[3], st);
  afl::launch_confine_buoy<double>(g, R.u3, R.v3, R.w3, R.rhos, R.temps, a->curl[0], a->curl[1],
                                   a->curl[2], a->curl[3], a->dt, a->params.vorticity_eps,
                                   a->params.buoyancy_beta, a->params.gravity_alpha, st);
  afl::launch_divergence<double>(g, R.u3, R.v3, R.w3, a->b, a->partials, a->scal, st);
  long dummy = 0;
  ADJ_TRY(solve(a, a->p, a->b, &dummy));
  afl::launch_project<double>(g, R.u3, R.v3, R.w3, a->p, st);
  for (int f = 3; f < 5; ++f) {
    const double *src = f == 3 ? R.rhos : R.temps;
    afl::launch_advect_fwd<double>(g, R.u3, R.v3, R.w3, src, R.fwd[f], a->dt, st);
    afl::adj_advect_mc_record(g, R.u3, R.v3, R.w3, src, R.fwd[f], a->F[f], a->dt,
                              f == 4 ? 0.985 : 0.996, true, R.mask[f], st);
  }
  ADJ_TRY(copy(a, a->F[0], R.u3));
  ADJ_TRY(copy(a, a->F[1], R.v3));
  ADJ_TRY(copy(a, a->F[2], R.w3));
  ADJ_CUDA(cudaGetLastError());
  return AFL_OK;
}

// Adjoint of one step: on entry (ub0, vb0, wb0, rhob, tempb) is the adjoint of
// the step's output state, on exit that of its input state; ampb accumulates.
afl_status step_adjoint(afl_adjoint *a, const Rec &R) {
  const afl::Dims &g = a->g;
  cudaStream_t st = a->stream;
  ADJ_TRY(zero(a, a->rhobs));
  ADJ_TRY(zero(a, a->tempbs));
  // scalars (advected by the projected velocity u3; its adjoint is ub0..)
  afl::adj_advect_bwd(g, R.u3, R.v3, R.w3, R.temps, R.fwd[4], R.mask[4], a->dt, 0.985, true,
                      a->tempb, a->fb, a->tempbs, a->ub0, a->vb0, a->wb0, st);
  afl::adj_advect_bwd(g, R.u3, R.v3, R.w3, R.rhos, R.fwd[3], R.mask[3], a->dt, 0.996, true,
                      a->rhob, a->fb, a->rhobs, a->ub0, a->vb0, a->wb0, st);
  // projection
  afl::adj_project_bwd_p(g, a->ub0, a->vb0, a->wb0, a->pb, st);
  if (a->params.solver_kind == AFL_POISSON_RBSOR) {
    // the pressure this step solved for is also the next step's warm start
    afl::adj_add(g, a->pcarry, a->pb, st);
    afl::adj_sor_bwd(g, a->params.solver_iters, a->params.sor_omega, a->pb, a->bb, st);
    std::swap(a->pcarry, a->pb);
  } else {
    ADJ_TRY(solve(a, a->bb, a->pb, &a->adj_iters));
  }
  afl::adj_project_bwd_b(g, a->ub0, a->vb0, a->wb0, a->bb, a->ub2, a->vb2, a->wb2, st);
  // confinement + buoyancy (curl of the velocity after the source, recomputed)
  const double *cu = jets(a) ? R.u1s : R.u1, *cv = jets(a) ? R.v1s : R.v1,
               *cw = jets(a) ? R.w1s : R.w1;
  afl::launch_curl<double>(g, cu, cv, cw, a->curl[0], a->curl[1], a->curl[2], a->curl[3], st);
  ADJ_TRY(zero(a, a->ub1));
  ADJ_TRY(zero(a, a->vb1));
  ADJ_TRY(zero(a, a->wb1));
  afl::adj_confine_bwd(g, a->curl[0], a->curl[1], a->curl[2], a->curl[3], a->ub2, a->vb2, a->wb2,
                       a->dt, a->params.vorticity_eps, a->params.buoyancy_beta,
                       a->params.gravity_alpha, a->gb, a->ob, a->ub1, a->vb1, a->wb1, a->rhobs,
                       a->tempbs, st);
  // source: the sphere's assignment, or the jets' caps (their velocity
  // increments pass the velocity adjoint through)
  if (sphere_on(a))
    afl::adj_source_bwd(g, a->src_lo, a->src_hi, a->params.sphere_center,
                        a->params.sphere_radius * a->params.sphere_radius,
                        a->params.sphere_temperature, a->rhobs, a->tempbs, a->ampb, st);
  else if (jets(a))
    afl::adj_jet_bwd(g, R.jmask, a->rhobs, a->tempbs, st);
  // velocity advections, last first
  ADJ_TRY(zero(a, a->ub0));
  ADJ_TRY(zero(a, a->vb0));
  ADJ_TRY(zero(a, a->wb0));
  afl::adj_advect_bwd(g, R.u1, R.v1, R.w0, R.w0, R.fwd[2], R.mask[2], a->dt, 0.996, false, a->wb1,
                      a->fb, a->wb0, a->ub1, a->vb1, a->wb0, st);
  afl::adj_advect_bwd(g, R.u1, R.v0, R.w0, R.v0, R.fwd[1], R.mask[1], a->dt, 0.996, false, a->vb1,
                      a->fb, a->vb0, a->ub1, a->vb0, a->wb0, st);
  afl::adj_advect_bwd(g, R.u0, R.v0, R.w0, R.u0, R.fwd[0], R.mask[0], a->dt, 0.996, false, a->ub1,
                      a->fb, a->ub0, a->ub0, a->vb0, a->wb0, st);
  std::swap(a->rhob, a->rhobs);
  std::swap(a->tempb, a->tempbs);
  ADJ_CUDA(cudaGetLastError());
  return AFL_OK;
}

afl_status upload(afl_adjoint *a, double *dst, const double *host) {
  ADJ_CUDA(cudaMemcpyAsync(dst, host, nbytes(a), cudaMemcpyHostToDevice, a->stream));
  ADJ_CUDA(cudaStreamSynchronize(a->stream));
  return AFL_OK;
}

afl_status download(afl_adjoint *a, double *host, const double *src) {
  ADJ_CUDA(cudaMemcpyAsync(host, src, nbytes(a), cudaMemcpyDeviceToHost, a->stream));
  ADJ_CUDA(cudaStreamSynchronize(a->stream));
  return AFL_OK;
}

}  // namespace

extern "C" {

afl_status afl_adjoint_create(size_t nx, size_t ny, size_t nz, const afl_params *params,
                              int checkpoint_every, afl_adjoint **out) {
  if (!out || !params) return fail(AFL_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (nx < 6 || ny < 6 || nz < 6) return fail(AFL_ERR_INVALID_ARGUMENT, "dimensions must be >= 6");
  if (checkpoint_every < 1) return fail(AFL_ERR_INVALID_ARGUMENT, "checkpoint_every must be >= 1");
  if (params->solver_kind != AFL_POISSON_CG && params->solver_kind != AFL_POISSON_RBSOR)
    return fail(AFL_ERR_INVALID_ARGUMENT, "solver_kind must be 0 (CG) or 1 (RB-SOR)");
  if (params->source_kind < AFL_SOURCE_CYBERPUNK || params->source_kind > AFL_SOURCE_NONE)
    return fail(AFL_ERR_INVALID_ARGUMENT, "source_kind must be 0, 1 or 2");
  if (params->solver_iters < 0)
    return fail(AFL_ERR_INVALID_ARGUMENT, "solver_iters must be >= 0");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(AFL_ERR_CUDA, "no CUDA device available; this library has no CPU path");
  }
  auto *a = new afl_adjoint();
  auto bail = [&](afl_status st) {
    afl_adjoint_destroy(a);
    return st;
  };
  cudaGetDevice(&a->device);
  a->params = *params;
  a->k = checkpoint_every;
  a->g.nx = static_cast<int>(nx);
  a->g.ny = static_cast<int>(ny);
  a->g.nz = static_cast<int>(nz);
  a->g.nxy = a->g.nx * a->g.ny;
  a->g.n = a->g.nxy * a->g.nz;
  a->g.h = 1.0 / static_cast<double>(std::max(nx, std::max(ny, nz)));
  const double *c = params->sphere_center;
  const double r = params->sphere_radius;
  a->src_lo[0] = box_lo(c[0], r, a->g.nx);
  a->src_lo[1] = box_lo(c[1], r, a->g.ny);
  a->src_lo[2] = box_lo(c[2], r, a->g.nz);
  a->src_hi[0] = box_hi(c[0], r, a->g.nx);
  a->src_hi[1] = box_hi(c[1], r, a->g.ny);
  a->src_hi[2] = box_hi(c[2], r, a->g.nz);
  if (cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(AFL_ERR_CUDA, "cudaStreamCreate failed"));
  afl_status st = AFL_OK;
  for (int f = 0; f < 5 && st == AFL_OK; ++f) st = dalloc(a, &a->F[f]);
  double **singles[] = {&a->p, &a->b, &a->tmp_fwd, &a->tmp_out, &a->amp, &a->ub0, &a->vb0,
                        &a->wb0, &a->rhob, &a->tempb, &a->ub1, &a->vb1, &a->wb1, &a->ub2,
                        &a->vb2, &a->wb2, &a->rhobs, &a->tempbs, &a->fb, &a->pb, &a->bb,
                        &a->ampb, &a->pcarry};
  for (double **x : singles)
    if (st == AFL_OK) st = dalloc(a, x);
  for (int f = 0; f < 4 && st == AFL_OK; ++f) st = dalloc(a, &a->curl[f]);
  // one block: the resident FP64 CG reads cg[0..3] as four consecutive arrays
  if (st == AFL_OK) {
    void *blk = nullptr;
    if (cudaMalloc(&blk, 4 * nbytes(a)) != cudaSuccess) {
      st = fail(AFL_ERR_OUT_OF_MEMORY, "CG vectors");
    } else {
      a->allocs.push_back(blk);
      for (int f = 0; f < 4; ++f) a->cg[f] = static_cast<double *>(blk) + f * static_cast<size_t>(a->g.n);
    }
  }
  for (int f = 0; f < 3 && st == AFL_OK; ++f) st = dalloc(a, &a->gb[f]);
  for (int f = 0; f < 3 && st == AFL_OK; ++f) st = dalloc(a, &a->ob[f]);
  if (st != AFL_OK) return bail(st);
  // reductions and the persistent CG's barrier/partials
  void *v = nullptr;
  if (cudaMalloc(&v, sizeof(double) * afl::kReduceBlocks * afl::kReduceMaxVals) != cudaSuccess)
    return bail(fail(AFL_ERR_OUT_OF_MEMORY, "partials"));
  a->allocs.push_back(v);
  a->partials = static_cast<double *>(v);
  if (cudaMalloc(&v, sizeof(double) * 16) != cudaSuccess)
    return bail(fail(AFL_ERR_OUT_OF_MEMORY, "scalars"));
  a->allocs.push_back(v);
  a->scal = static_cast<double *>(v);
  if (cudaMalloc(&v, sizeof(afl::SolveReport)) != cudaSuccess)
    return bail(fail(AFL_ERR_OUT_OF_MEMORY, "report"));
  a->allocs.push_back(v);
  a->rep = static_cast<afl::SolveReport *>(v);
  const int maxb = afl::persistent_blocks_cg_f64();
  if (cudaMalloc(&v, sizeof(unsigned int) * 4) != cudaSuccess)
    return bail(fail(AFL_ERR_OUT_OF_MEMORY, "barrier"));
  a->allocs.push_back(v);
  a->ps.count = static_cast<unsigned int *>(v);
  a->ps.gen = a->ps.count + 1;
  a->ps.abort_flag = reinterpret_cast<int *>(a->ps.count + 2);
  // partials of the streaming CG (2 x 2 per CTA) or tagged slots of the resident one
  // (2 buffers x 2 words x up to 3 values per tile)
  if (cudaMalloc(&v, sizeof(double) * 12 * static_cast<size_t>(maxb)) != cudaSuccess)
    return bail(fail(AFL_ERR_OUT_OF_MEMORY, "CG partials"));
  a->allocs.push_back(v);
  a->ps.partials = static_cast<double *>(v);
  a->ps.max_blocks = maxb;
  a->ps.timeout_ns = 5000000000ull;
  // The Poisson kernel follows params->poisson_kernel as afl_create's does:
  // AUTO takes the on-chip resident CG when the grid fits, STREAMING never,
  // RESIDENT always (an error when the grid does not fit).
  const bool fits = afl::plan_resident(a->g, true, &a->res) &&
                    a->res.tiles_x * a->res.tiles_y <= maxb;
  if (params->poisson_kernel == AFL_POISSON_KERNEL_RESIDENT && !fits)
    return bail(fail(AFL_ERR_INVALID_ARGUMENT,
                     "the grid does not fit the resident CG kernel"));
  a->resident = fits && params->poisson_kernel != AFL_POISSON_KERNEL_STREAMING;
  // one segment of recorded steps
  a->rec.resize(static_cast<size_t>(a->k));
  for (Rec &R : a->rec) {
    double **arrs[] = {&R.u0, &R.v0, &R.w0, &R.u1, &R.v1, &R.w1, &R.rhos, &R.temps,
                       &R.u3, &R.v3, &R.w3};
    for (double **x : arrs)
      if (st == AFL_OK) st = dalloc(a, x);
    for (int f = 0; f < 5 && st == AFL_OK; ++f) st = dalloc(a, &R.fwd[f]);
    for (int f = 0; f < 5 && st == AFL_OK; ++f) st = balloc(a, &R.mask[f]);
    if (jets(a)) {
      for (double **x : {&R.u1s, &R.v1s, &R.w1s})
        if (st == AFL_OK) st = dalloc(a, x);
      if (st == AFL_OK) st = balloc(a, &R.jmask);
    }
  }
  if (st != AFL_OK) return bail(st);
  *out = a;
  return AFL_OK;
}

afl_status afl_adjoint_destroy(afl_adjoint *a) {
  if (!a) return AFL_OK;
  if (a->stream) cudaStreamSynchronize(a->stream);
  for (void *p : a->allocs) cudaFree(p);
  for (auto &cp : a->ckpt)
    for (double *x : cp) cudaFree(x);
  if (a->stream) cudaStreamDestroy(a->stream);
  delete a;
  return AFL_OK;
}

afl_status afl_adjoint_forward(afl_adjoint *a, const double *u0, const double *v0,
                               const double *w0, const double *amp, int steps, double dt,
                               double *rho_final) {
  if (!a || !u0 || !v0 || !w0) return fail(AFL_ERR_INVALID_ARGUMENT, "null argument");
  if (steps < 1) return fail(AFL_ERR_INVALID_ARGUMENT, "steps must be >= 1");
  a->steps = steps;
  a->dt = dt;
  a->fwd_iters = 0;
  const int nck = (steps + a->k - 1) / a->k;
  while (static_cast<int>(a->ckpt.size()) < nck) {
    std::array<double *, 6> cp{};
    for (double *&x : cp) {
      void *v = nullptr;
      ADJ_CUDA(cudaMalloc(&v, nbytes(a)));
      x = static_cast<double *>(v);
    }
    a->ckpt.push_back(cp);
  }
  ADJ_TRY(upload(a, a->F[0], u0));
  ADJ_TRY(upload(a, a->F[1], v0));
  ADJ_TRY(upload(a, a->F[2], w0));
  ADJ_TRY(zero(a, a->F[3]));
  ADJ_TRY(zero(a, a->F[4]));
  ADJ_TRY(zero(a, a->p));
  if (amp) {
    ADJ_TRY(upload(a, a->amp, amp));
  } else {
    std::vector<double> ones(static_cast<size_t>(a->g.n), 1.0);
    ADJ_TRY(upload(a, a->amp, ones.data()));
  }
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventRecord(t0, a->stream);
  for (int s = 0; s < steps; ++s) {
    if (s % a->k == 0) {
      auto &cp = a->ckpt[static_cast<size_t>(s / a->k)];
      for (int f = 0; f < 5; ++f) ADJ_TRY(copy(a, cp[f], a->F[f]));
      ADJ_TRY(copy(a, cp[5], a->p));
    }
    ADJ_TRY(step_plain(a, s));
  }
  cudaEventRecord(t1, a->stream);
  ADJ_CUDA(cudaStreamSynchronize(a->stream));
  cudaEventElapsedTime(&a->fwd_ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  a->have_forward = true;
  if (rho_final) ADJ_TRY(download(a, rho_final, a->F[3]));
  return AFL_OK;
}

afl_status afl_adjoint_backward(afl_adjoint *a, const double *rho_bar, double *u0_bar,
                                double *v0_bar, double *w0_bar, double *amp_bar) {
  if (!a || !rho_bar) return fail(AFL_ERR_INVALID_ARGUMENT, "null argument");
  if (!a->have_forward) return fail(AFL_ERR_INVALID_ARGUMENT, "run afl_adjoint_forward first");
  a->adj_iters = 0;
  ADJ_TRY(upload(a, a->rhob, rho_bar));
  for (double *x : {a->ub0, a->vb0, a->wb0, a->tempb, a->ampb, a->bb, a->pcarry})
    ADJ_TRY(zero(a, x));
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventRecord(t0, a->stream);
  const int nseg = (a->steps + a->k - 1) / a->k;
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int first = seg * a->k;
    const int count = std::min(a->k, a->steps - first);
    auto &cp = a->ckpt[static_cast<size_t>(seg)];
    for (int f = 0; f < 5; ++f) ADJ_TRY(copy(a, a->F[f], cp[f]));
    ADJ_TRY(copy(a, a->p, cp[5]));
    for (int s = 0; s < count; ++s)
      ADJ_TRY(step_record(a, a->rec[static_cast<size_t>(s)], first + s));
    for (int s = count - 1; s >= 0; --s) ADJ_TRY(step_adjoint(a, a->rec[static_cast<size_t>(s)]));
  }
  cudaEventRecord(t1, a->stream);
  ADJ_CUDA(cudaStreamSynchronize(a->stream));
  cudaEventElapsedTime(&a->bwd_ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (u0_bar) ADJ_TRY(download(a, u0_bar, a->ub0));
  if (v0_bar) ADJ_TRY(download(a, v0_bar, a->vb0));
  if (w0_bar) ADJ_TRY(download(a, w0_bar, a->wb0));
  if (amp_bar) ADJ_TRY(download(a, amp_bar, a->ampb));
  return AFL_OK;
}

// out = {forward ms, backward ms (recompute included), forward CG iterations,
//        adjoint CG iterations}
afl_status afl_adjoint_stats(const afl_adjoint *a, double out[4]) {
  if (!a || !out) return fail(AFL_ERR_INVALID_ARGUMENT, "null argument");
  out[0] = a->fwd_ms;
  out[1] = a->bwd_ms;
  out[2] = static_cast<double>(a->fwd_iters);
  out[3] = static_cast<double>(a->adj_iters);
  return AFL_OK;
}

}  // extern "C"
