// afl_launch.h -- host-side launchers for the stage kernels.
//
// T is the storage/arithmetic type of velocity, density and temperature:
// double for the FP64 drop-in form, float for the mixed form.  Pressure and
// the Poisson right-hand side are always double.  Every launcher is
// asynchronous on `st`.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "afl_device.cuh"

struct afl_solver;  // include/aether_fluid.h

namespace afl {

// Device-resident per-step report written by the Poisson kernels (mirrors
// afl_solve_info field for field).
struct SolveReport {
  int32_t iterations;
  int32_t refinements;
  int32_t converged;
  int32_t status;
  double initial_residual;
  double final_residual;
  double rhs_norm;
};

// Barrier + scratch state of the persistent kernels.
struct PersistentState {
  unsigned int *count;
  unsigned int *gen;
  int *abort_flag;
  double *partials;      // >= 12 * max_blocks doubles (streaming kernels: 2 buffers x 3
                         // values; resident kernels: 2 buffers x 3 tagged values x 2 words)
  int max_blocks;
  unsigned long long timeout_ns;
};

// Number of CTAs the reduction kernels use (fixed, so sums are reproducible).
constexpr int kReduceBlocks = 1184;  // 8 per SM on a 148-SM B200 (full occupancy at 256 threads)
constexpr int kReduceMaxVals = 8;

template <typename T>
void launch_advect_fwd(const Dims &g, const T *u, const T *v, const T *w, const T *src,
                       T *fwd, double dt, cudaStream_t st);
template <typename T>
void launch_advect_mc(const Dims &g, const T *u, const T *v, const T *w, const T *src,
                      const T *fwd, T *out, double dt, double dissipation, bool nonneg,
                      cudaStream_t st);
// The shared-memory-staged stage kernels (afl_stage_fused.cuh).
// Density and temperature advected by (u, v, w) in one launch into out[]
// (arrays distinct from the inputs), with the telemetry partials of the final
// state in tel, 7 per CTA (fused_ctas of them).
template <typename T>
void launch_scalars_fused(const Dims &g, const T *u, const T *v, const T *w,
                          const T *const src[2], T *const out[2], const double diss[2],
                          double dt, double *tel, cudaStream_t st);
// Curl, confinement, buoyancy and the wall BC in one launch; the new velocity
// goes to (uo, vo, wo), arrays distinct from (u, v, w).
template <typename T>
void launch_forces_fused(const Dims &g, const T *u, const T *v, const T *w, const T *rho,
                         const T *temp, T *uo, T *vo, T *wo, double dt, double eps, double beta,
                         double alpha, cudaStream_t st);
int fused_ctas(const Dims &g);
// Sums telemetry partials (7 per CTA) into the 8 doubles of compute_telemetry.
void launch_telemetry_finalize(const double *partials, int nparts, double time_sec,
                               double *out8, cudaStream_t st);
template <typename T>
void launch_wall_bc(const Dims &g, T *u, T *v, T *w, cudaStream_t st);
template <typename T>
void launch_curl(const Dims &g, const T *u, const T *v, const T *w, T *cx, T *cy, T *cz,
                 T *cmag, cudaStream_t st);
template <typename T>
void launch_confine_buoy(const Dims &g, T *u, T *v, T *w, const T *rho, const T *temp,
                         const T *cx, const T *cy, const T *cz, const T *cmag, double dt,
                         double eps, double beta, double alpha, cudaStream_t st);
// b = -h*(du+dv+dw) on the interior (0 elsewhere); partials get
// (sum div^2, sum b^2) per CTA; finalize writes {rms, ||b||} to out2.
template <typename T>
void launch_divergence(const Dims &g, const T *u, const T *v, const T *w, double *b,
                       double *partials, double *out2, cudaStream_t st);
template <typename T>
void launch_project(const Dims &g, T *u, T *v, T *w, const double *p, cudaStream_t st);
template <typename T>
void launch_inject_jet(const Dims &g, const int lo[3], const int hi[3], T *rho, T *temp,
                       T *u, T *v, T *w, const double jet[6], double r2, double dt,
                       double pulse, cudaStream_t st);
template <typename T>
void launch_inject_sphere(const Dims &g, const int lo[3], const int hi[3], T *rho,
                          T *temp, const double *amp, const double c[3], double r2,
                          double rho_val, double temp_val, cudaStream_t st);
// Writes 8 doubles (time, KE, enstrophy, peak, mass, com xyz) to out8.
template <typename T>
void launch_telemetry(const Dims &g, const T *u, const T *v, const T *w, const T *rho,
                      double time_sec, double *partials, double *out8, cudaStream_t st);
template <typename T>
void launch_max(const Dims &g, const T *x, double *partials, double *out1, cudaStream_t st);
template <typename T>
void launch_sample(const Dims &g, const T *f, const double *xyz, int npts, double *out,
                   cudaStream_t st);
// Precision conversions for the mixed form's uploads/downloads.
void launch_convert_f64_to_f32(const double *src, float *dst, int n, cudaStream_t st);
void launch_convert_f32_to_f64(const float *src, double *dst, int n, cudaStream_t st);

// ---- Poisson ---------------------------------------------------------------
struct CgArgs {
  Dims g;
  double *p;        // pressure (warm start in, solution out)
  const double *b;  // right-hand side
  double *r, *d0, *d1, *q;
  int max_iters;
  double rel_tol;
  SolveReport *report;
};
// Returns the number of CTAs used (for tests/diagnostics).
int launch_cg_f64(const CgArgs &a, const PersistentState &ps, cudaStream_t st);

struct SorArgs {
  Dims g;
  double *p;
  const double *b;
  int sweeps;
  double omega;
  SolveReport *report;
};
int launch_rbsor_f64(const SorArgs &a, const PersistentState &ps, cudaStream_t st);

struct MixedCgArgs {
  Dims g;
  double *p;          // f64 pressure
  const double *b;    // f64 right-hand side
  float *r, *e, *d0, *d1, *q;  // f32 inner-CG vectors
  int max_inner;      // inner iterations per pass
  int max_total;      // cap on inner iterations over all passes
  int max_refine;
  double inner_rel_tol;
  double rel_tol;     // outer (f64) target
  SolveReport *report;
};
int launch_cg_mixed(const MixedCgArgs &a, const PersistentState &ps, cudaStream_t st);

struct SorMixedArgs {
  Dims g;
  double *p;
  const double *b;
  float *p32;
  float *b32;
  int sweeps;
  double omega;
  SolveReport *report;
};
int launch_rbsor_mixed(const SorMixedArgs &a, const PersistentState &ps, cudaStream_t st);

// On-chip resident CG (afl_poisson_resident.cu): one 1024-thread CTA per SM
// owns a 16 x ty column tile spanning all z planes.
struct ResidentPlan {
  int ty;          // tile height in y (cells)
  int cpt;         // z cells per thread
  int tiles_x, tiles_y;
  int smem_bytes;  // dynamic shared memory per CTA
};
struct ResidentCgArgs {
  Dims g;
  int tiles_x, tiles_y;
  double *p;            // f64 pressure
  const double *b;      // f64 right-hand side
  void *rpub;           // mixed: published tile-edge residual (f32, n cells).
                        // FP64: 4n doubles: the (r, q = A d) pair of every
                        // cell, by iteration parity (0, 1)
  void *dpub0, *dpub1;  // mixed: published tile-edge direction, by iteration parity
  int max_iters;        // FP64: CG iterations; mixed: inner iterations, all passes
  int max_inner;        // mixed: inner iterations per refinement pass
  int max_refine;       // mixed: refinement passes
  double inner_rel_tol; // mixed
  double rel_tol;
  SolveReport *report;
};
struct ResidentSorArgs {
  Dims g;
  int tiles_x, tiles_y;
  double *p;            // f64 pressure (read, written)
  const double *b;      // f64 right-hand side
  float *e32;           // mixed: published tile-edge correction (n cells)
  int sweeps;
  double omega;
  SolveReport *report;
};
// RB-SOR on the resident tile plan of the CG (the tile of one solved quantity
// fits wherever the CG's does).
int launch_sor_resident(const ResidentSorArgs &a, const ResidentPlan &plan, bool f64,
                        const PersistentState &ps, cudaStream_t st);
// False when the grid does not fit on chip (too many tiles, too much shared
// memory, or more than 16 z cells per thread).
bool plan_resident(const Dims &g, bool f64, ResidentPlan *plan);
size_t resident_smem_bytes(const Dims &g, int ty, int cpt, bool f64);
int launch_cg_resident(const ResidentCgArgs &a, const ResidentPlan &plan, bool f64,
                       const PersistentState &ps, cudaStream_t st);

// The two orbiting jets of inject_cyberpunk_sources (src/fluid.rs:533-571) at
// time_sec: centre and velocity of each jet, its cell box clamped as the
// reference clamps it, the squared radius in cells and the pulse.
struct JetPair {
  double jet[2][6];  // centre x, y, z; velocity x, y, z
  int lo[2][3], hi[2][3];
  double r2, pulse;
};
JetPair cyberpunk_jets(const Dims &g, double time_sec);

// Sets the text afl_last_error() returns on the calling thread.
void set_last_error_text(const char *msg);

// Streaming CG (afl_poisson_stream.cu): x runs of 2 doubles / 4 floats per
// thread when nx allows, else single cells.
int stream_vector_width(const Dims &g, bool f64);
int launch_cg_stream_f64(const CgArgs &a, const PersistentState &ps, cudaStream_t st);
int launch_cg_stream_mixed(const MixedCgArgs &a, const PersistentState &ps, cudaStream_t st);
int persistent_blocks_stream();

// One system of the batched (multi-grid) streaming CG: its arguments, its own
// barrier and partials (2 buffers x 3 values x ctas), and its CTA range.
struct MultiCgSystem {
  CgArgs f64;          // used by the FP64 form
  MixedCgArgs mixed;   // used by the mixed form
  GridSync gs;         // nblocks = ctas
  double *partials;
  int cta_begin, ctas;
};
// d_sys / d_cta_inst live in device memory; every system's grid must allow the
// vector width v (nx % v == 0).
int launch_cg_multi(const MultiCgSystem *d_sys, const int *d_cta_inst, int total_ctas, bool f64,
                    int v, cudaStream_t st);
int persistent_blocks_multi(bool f64, int v);

// ---- ensemble (afl_ensemble_kernels.cuh) ------------------------------------
// Device-side descriptor of one instance of a batched ensemble.
template <typename T>
struct EnsInstance {
  Dims g;
  T *fld[5];        // current u, v, w, density, temperature
  T *tmp_fwd, *tmp_out;
  T *curl[4];
  double *p, *b;
  T scale_f, scale_b, dt, eps_h, inv_2h, beta, alpha;
  double h, inv_h, dv, inv_2h_d, dt_time;
  int src_on;                 // sphere source active
  int src_lo[3], src_hi[3];   // clamped bounding box (src/fluid.rs:566-571 rule)
  double src_c[3], src_r2, src_rho, src_temp;
  int blk_begin, blk_count;   // plane blocks of this instance in the block table
  int kz;                     // z planes per block (the tile depth chosen by the tuner)
};

template <typename T>
struct EnsLaunch {
  EnsInstance<T> *inst;  // device descriptors
  const int *blk_inst;   // device block table: plane block -> instance
  int blocks;            // plane blocks of all instances
  int count;             // instances
};

template <typename T>
void ens_advect(const EnsLaunch<T> &L, int f, double diss, cudaStream_t st);
template <typename T>
void ens_forces(const EnsLaunch<T> &L, cudaStream_t st);
template <typename T>
void ens_divergence(const EnsLaunch<T> &L, cudaStream_t st);
template <typename T>
void ens_project(const EnsLaunch<T> &L, cudaStream_t st);
template <typename T>
void ens_telemetry(const EnsLaunch<T> &L, double *partials, const int *step_counter,
                   double *tel_out, const SolveReport *rep_cur, SolveReport *reports,
                   int capacity, cudaStream_t st);
void ens_step_advance(int *step_counter, cudaStream_t st);

// One persistent cooperative launch for a whole ensemble step
// (afl_ensemble_persist.cu): CTA b works on instance cta_inst[b] with the CTA
// range, barrier and partials of sys[cta_inst[b]].
struct EnsStepArgs {
  void *inst;                 // EnsInstance<T>[count] (device)
  const MultiCgSystem *sys;   // per instance: solve arguments, barrier, CTA range
  const int *cta_inst;        // CTA -> instance
  double *tel_partials;       // 7 per plane block
  const int *step_counter;
  double *tel_out;
  const SolveReport *rep_cur;
  SolveReport *reports;
  int count, capacity;
};
// Co-resident CTAs of the step kernel for the precision and run width v.
int persistent_blocks_ens_step(bool f64, int v);
int launch_ens_step(const EnsStepArgs &a, bool f64, int v, int total_ctas, cudaStream_t st);

// Occupancy-derived CTA count of each persistent kernel (co-residency bound).
int persistent_blocks_cg_f64();
int persistent_blocks_sor_f64();
int persistent_blocks_cg_mixed();
int persistent_blocks_sor_mixed();

// Read-only view of a solver's device state for other units of the library
// (afl_medium.cu): the grid, the device, the stream and the density and
// temperature fields (f64 or f32 by precision).
struct SolverView {
  Dims g;
  int device;
  cudaStream_t stream;
  bool f64;
  const void *density;
  const void *temperature;
};
bool solver_view(const afl_solver *s, SolverView *out);

}  // namespace afl
