/*
 * aether_fluid.h -- C ABI of the B200 (sm_100a) smoke solver.
 *
 * Drop-in boundary for the `FluidSolver3D` method surface of
 * vanovri/aether-core-engine (src/fluid.rs:23-673) and for the
 * density/temperature hand-off of `FluidMedium::from_solver`
 * (src/fluid.rs:703-732).  The reference has no FFI of its own; these entry
 * points are what its Rust side would bind with `extern "C"` declarations in
 * place of the method calls cited beside each one.
 *
 * Conventions
 *  - Every entry point returns an afl_status (0 = AFL_OK).  A non-zero status
 *    corresponds to a panic in the reference (failed assert, index out of
 *    range); afl_last_error() returns the text for the calling thread.
 *  - A handle owns its device memory and one CUDA stream on the device that
 *    was current when it was created.  Handles are not thread-safe (the
 *    reference takes `&mut self`); distinct handles may be used from distinct
 *    threads.
 *  - Fields are nx*ny*nz doubles, x fastest: idx = (k*ny + j)*nx + i
 *    (src/fluid.rs:88-90).  The caller owns the host memory passed in.
 *  - Stage calls are asynchronous on the handle's stream; downloads and calls
 *    that return a scalar synchronise the stream.
 *  - No entry point falls back to the CPU.  Without a usable CUDA device,
 *    afl_create fails with AFL_ERR_CUDA.
 */
#ifndef AETHER_FLUID_H
#define AETHER_FLUID_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AFL_ABI_VERSION 1

typedef enum afl_status {
  AFL_OK = 0,
  AFL_ERR_INVALID_ARGUMENT = 1, /* bad handle, size, field id or parameter  */
  AFL_ERR_CUDA = 2,             /* CUDA runtime error (text has the detail) */
  AFL_ERR_OUT_OF_MEMORY = 3,
  AFL_ERR_NONFINITE = 4,        /* NaN/Inf met in a residual or a reduction */
  AFL_ERR_TIMEOUT = 5,          /* a grid barrier exceeded its spin limit   */
  AFL_ERR_NOT_CONVERGED = 6     /* only when afl_params.fail_on_not_converged */
} afl_status;

/* Field ids: the public Vec<f64> fields of FluidSolver3D (src/fluid.rs:28-34). */
typedef enum afl_field {
  AFL_FIELD_U = 0,
  AFL_FIELD_V = 1,
  AFL_FIELD_W = 2,
  AFL_FIELD_DENSITY = 3,
  AFL_FIELD_TEMPERATURE = 4,
  AFL_FIELD_PRESSURE = 5,
  AFL_FIELD_DIVERGENCE = 6
} afl_field;

/* PoissonSolverKind (src/fluid.rs:17-21). */
typedef enum afl_poisson_kind {
  AFL_POISSON_CG = 0,
  AFL_POISSON_RBSOR = 1
} afl_poisson_kind;

/* Arithmetic of the handle, fixed at creation.
 * FP64: every stage in f64, the drop-in form.
 * MIXED: velocity/density/temperature stored and advanced in f32 (advection,
 *   confinement, buoyancy, CG matrix-vector products); divergence, Poisson
 *   residual, pressure and every inner product in f64, with an outer
 *   iterative-refinement loop in f64 around an f32 CG. */
typedef enum afl_precision {
  AFL_PRECISION_FP64 = 0,
  AFL_PRECISION_MIXED = 1
} afl_precision;

/* Poisson kernel choice.  CG, AUTO: the on-chip resident kernel when the grid
 * fits (tiles <= SMs, tile + halo in shared memory), else the streaming
 * kernel; the two differ only in the summation order of the inner products.
 * RB-SOR, AUTO: the resident kernel for the mixed form when the grid fits,
 * else the streaming sweep; RESIDENT selects the resident sweep for FP64 too
 * (same result bit for bit, since a colour reads only the other colour). */
typedef enum afl_poisson_kernel {
  AFL_POISSON_KERNEL_AUTO = 0,
  AFL_POISSON_KERNEL_STREAMING = 1,
  AFL_POISSON_KERNEL_RESIDENT = 2  /* fails with INVALID_ARGUMENT if it does not fit */
} afl_poisson_kernel;

/* What step() injects between velocity advection and the forces.
 * CYBERPUNK: inject_cyberpunk_sources (src/fluid.rs:532-595), the reference.
 * SPHERE: assign density/temperature inside a sphere (see afl_params).
 * NONE: inject nothing. */
typedef enum afl_source_kind {
  AFL_SOURCE_CYBERPUNK = 0,
  AFL_SOURCE_SPHERE = 1,
  AFL_SOURCE_NONE = 2
} afl_source_kind;

/* Solver knobs.  The first five are the reference's public fields
 * (src/fluid.rs:45-49, defaults :79-83); the rest are extensions whose
 * defaults reproduce the reference. */
typedef struct afl_params {
  double vorticity_eps;   /* 5.5  */
  double buoyancy_beta;   /* 6.8  */
  double gravity_alpha;   /* 0.45 */
  int32_t solver_kind;    /* afl_poisson_kind, AFL_POISSON_CG */
  int32_t solver_iters;   /* 32: CG max iterations or SOR sweeps */
  double sor_omega;       /* 1.65 (src/fluid.rs:398) */
  double cg_rel_tol;      /* 0: reference's absolute stopping rule only.
                             > 0: also stop at ||r||_2 <= cg_rel_tol*||b||_2 */
  int32_t precision;      /* afl_precision; read only by afl_create */
  int32_t source_kind;    /* afl_source_kind, AFL_SOURCE_CYBERPUNK */
  double sphere_center[3];/* cell-index coordinates */
  double sphere_radius;   /* cells */
  double sphere_density;  /* value assigned inside the sphere */
  double sphere_temperature; /* value (times the amplitude map, if set) */
  int32_t fail_on_not_converged; /* 0: a solve that hits max iterations is
                             reported in afl_solve_info only (reference) */
  int32_t mixed_inner_iters;  /* MIXED: max f32 CG iterations per refinement
                                 pass (default 200) */
  double mixed_inner_rel_tol; /* MIXED: inner f32 CG relative tolerance
                                 (default 1e-4) */
  int32_t mixed_max_refinements; /* MIXED: max outer passes (default 8) */
  int32_t poisson_kernel; /* afl_poisson_kernel: which Poisson kernel runs */
  double reserved_f64[4];
} afl_params;

/* FluidTelemetryFrame (src/fluid.rs:7-15). */
typedef struct afl_telemetry {
  double time_sec;
  double kinetic_energy;
  double enstrophy;
  double peak_vorticity;
  double total_mass;
  double center_of_mass[3];
} afl_telemetry;

/* Report of one Poisson solve (no counterpart in the reference, which
 * returns nothing from its solvers). */
typedef struct afl_solve_info {
  int32_t iterations;       /* CG p/r updates (all passes), or SOR sweeps */
  int32_t refinements;      /* MIXED: outer f64 passes; 0 otherwise */
  int32_t converged;        /* 1 when a stopping test (not max_iters) fired */
  int32_t status;           /* afl_status of the solve */
  double initial_residual;  /* ||b - A p0||_2 */
  double final_residual;    /* ||b - A p||_2 (f64) at exit */
  double rhs_norm;          /* ||b||_2 */
} afl_solve_info;

typedef struct afl_solver afl_solver;

/* ---- errors / params --------------------------------------------------- */
const char *afl_last_error(void);
int afl_abi_version(void);
/* Fills *p with the reference defaults (src/fluid.rs:79-83). */
afl_status afl_params_default(afl_params *p);

/* ---- lifecycle: FluidSolver3D::new (src/fluid.rs:53-85) ----------------- */
/* Fails with AFL_ERR_INVALID_ARGUMENT when any dimension is < 6
 * (the assert at src/fluid.rs:54). params may be NULL for the defaults. */
afl_status afl_create(size_t nx, size_t ny, size_t nz, const afl_params *params,
                      afl_solver **out);
afl_status afl_destroy(afl_solver *s);
afl_status afl_get_dims(const afl_solver *s, size_t *nx, size_t *ny, size_t *nz,
                        double *h);
/* Public-field writes (src/fluid.rs:45-49); precision is ignored here. */
afl_status afl_set_params(afl_solver *s, const afl_params *params);
afl_status afl_get_params(const afl_solver *s, afl_params *params);
/* Optional per-cell temperature amplitude for the sphere source (N doubles,
 * copied to the device); NULL clears it. */
afl_status afl_set_source_amplitude(afl_solver *s, const double *amp, size_t n);

/* ---- public fields: direct reads/writes of solver.u etc. ---------------- */
afl_status afl_upload_field(afl_solver *s, int field, const double *host, size_t n);
afl_status afl_download_field(afl_solver *s, int field, double *host, size_t n);
/* Seeded initial condition: Rng::from_seed(seed) (src/rng.rs:21-33), then for
 * u, v, w in turn and id in 0..N, range_f64(lo, hi) (src/rng.rs:86-88); then
 * enforce_wall_velocity_bc.  density/temperature/pressure are zeroed. */
afl_status afl_init_velocity_noise(afl_solver *s, uint64_t seed, double lo, double hi);

/* ---- stage calls -------------------------------------------------------- */
/* advect_maccormack_in_place (src/fluid.rs:170-234); field_kind 0..4 =
 * u, v, w, density, temperature (any other value means temperature). */
afl_status afl_advect_maccormack(afl_solver *s, int field_kind, double dt,
                                 double dissipation);
/* enforce_wall_velocity_bc (src/fluid.rs:236-253). */
afl_status afl_enforce_wall_bc(afl_solver *s);
/* apply_buoyancy_and_vorticity_confinement (src/fluid.rs:256-330). */
afl_status afl_buoyancy_vorticity(afl_solver *s, double dt);
/* compute_divergence_norm (src/fluid.rs:333-353): writes the divergence
 * field (the Poisson right-hand side) and returns the RMS divergence. */
afl_status afl_divergence_norm(afl_solver *s, double *rms);
/* solve_poisson_conjugate_gradient (src/fluid.rs:445-493). */
afl_status afl_solve_cg(afl_solver *s, int max_iters, afl_solve_info *info);
/* solve_poisson_gauss_seidel (src/fluid.rs:397-442), omega = sor_omega. */
afl_status afl_solve_rbsor(afl_solver *s, int iterations, afl_solve_info *info);
/* project (src/fluid.rs:496-529). info may be NULL. */
afl_status afl_project(afl_solver *s, afl_solve_info *info);
/* inject_cyberpunk_sources (src/fluid.rs:532-595). */
afl_status afl_inject_cyberpunk(afl_solver *s, double time_sec, double dt);
/* Sphere source of afl_params (extension, no reference counterpart). */
afl_status afl_inject_sphere(afl_solver *s);
/* step (src/fluid.rs:598-611); out may be NULL.  Synchronises when out or
 * info is non-NULL. */
afl_status afl_step(afl_solver *s, double dt, double time_sec, afl_telemetry *out,
                    afl_solve_info *info);
/* `steps` calls of step() with time = t0 + n*dt_time, without a host sync
 * between steps; telemetry (steps entries) and per-step Poisson reports
 * (steps entries) are gathered on the device and copied out once at the end.
 * Either array may be NULL. */
afl_status afl_run(afl_solver *s, int steps, double dt, double t0, double dt_time,
                   afl_telemetry *telemetry, afl_solve_info *infos);
/* compute_telemetry (src/fluid.rs:613-672). */
afl_status afl_compute_telemetry(afl_solver *s, double time_sec, afl_telemetry *out);

/* ---- hand-off to FluidMedium::from_solver (src/fluid.rs:703-732) -------- */
/* max over the density field (src/fluid.rs:704-707). */
afl_status afl_max_density(afl_solver *s, double *out);
/* Copies density and temperature (N doubles each, either may be NULL) and
 * the max density in one synchronisation. */
afl_status afl_medium_handoff(afl_solver *s, double *density, double *temperature,
                              size_t n, double *max_density);

/* Batched trilinear sampling of a field at continuous index coordinates
 * (sample_trilinear, src/fluid.rs:94-128): xyz holds npts triples (host),
 * out receives npts doubles (host). */
afl_status afl_sample_trilinear(afl_solver *s, int field, const double *xyz,
                                size_t npts, double *out);

/* ---- tracing (no reference counterpart: the reference only wall-times the
 * whole fluid stage, src/main.rs:82-113) ------------------------------------ */
typedef enum afl_stage {
  AFL_STAGE_ADVECT = 0,      /* MacCormack passes of u, v, w, density, temperature */
  AFL_STAGE_SOURCE = 1,      /* source injection */
  AFL_STAGE_FORCES = 2,      /* curl, confinement, buoyancy, wall BC */
  AFL_STAGE_DIVERGENCE = 3,  /* divergence / Poisson right-hand side */
  AFL_STAGE_POISSON = 4,     /* the persistent CG / RB-SOR solve */
  AFL_STAGE_PROJECT = 5,     /* pressure-gradient subtraction + wall BC */
  AFL_STAGE_TELEMETRY = 6,   /* telemetry reduction */
  AFL_STAGE_COUNT = 7
} afl_stage;
/* Enables (1) or disables (0) CUDA-event timing of every stage on the
 * handle's stream and resets the accumulated times. */
afl_status afl_set_stage_timing(afl_solver *s, int enable);
/* Synchronises, then returns the accumulated device milliseconds and the
 * number of timed calls per stage (arrays of AFL_STAGE_COUNT; either may be
 * NULL). */
afl_status afl_get_stage_timing(afl_solver *s, double *ms, int64_t *calls);
/* The CG kernel plan chosen for this grid: out[0] = 1 when the on-chip
 * resident kernel fits (else the streaming kernel runs), out[1] = tile height
 * in y (tiles are 16 wide in x and span all z), out[2] = z cells per thread,
 * out[3] = CTAs (one per SM). */
afl_status afl_get_poisson_plan(const afl_solver *s, int32_t out[4]);
/* Kernels this handle has launched since creation. */
afl_status afl_get_launch_count(const afl_solver *s, uint64_t *count);

/* ---- batched ensemble (no reference counterpart) -----------------------------
 * Many independent plumes of different grid sizes advanced together: every
 * stage of a step is one batched launch over all instances, the pressure
 * solves run in one cooperative launch whose CTAs are split between the
 * instances, and one step is captured once in a CUDA graph and replayed.
 * Each instance follows step() with the sphere source (the same arithmetic
 * as a single solver with the same settings; only reduction order differs). */
typedef struct afl_instance {
  size_t nx, ny, nz;
  uint64_t seed;           /* velocity noise: Rng::from_seed(seed), range_f64 */
  double noise_lo, noise_hi;
  double dt;               /* time step of this instance */
  double vorticity_eps, buoyancy_beta, gravity_alpha;
  double sphere_center[3]; /* cell-index coordinates */
  double sphere_radius;    /* cells; 0 = no source */
  double sphere_density, sphere_temperature;
} afl_instance;

typedef struct afl_ensemble afl_ensemble;

/* common: precision, solver_iters, cg_rel_tol and the mixed_* knobs apply to
 * every instance (CG only); NULL for the defaults. */
afl_status afl_ensemble_create(const afl_instance *instances, int count,
                               const afl_params *common, afl_ensemble **out);
afl_status afl_ensemble_destroy(afl_ensemble *e);
/* `steps` steps of every instance; telemetry and infos (either may be NULL)
 * receive steps*count entries, step-major.  Telemetry time is n*dt. */
afl_status afl_ensemble_run(afl_ensemble *e, int steps, afl_telemetry *telemetry,
                            afl_solve_info *infos);
afl_status afl_ensemble_download_field(afl_ensemble *e, int instance, int field, double *host,
                                       size_t n);
/* Picks the CTA split of the batched solve by timing candidates on a snapshot
 * of the state (restored afterwards); *choice gets the candidate index. */
afl_status afl_ensemble_autotune(afl_ensemble *e, int32_t *choice);
/* out = {instances, step graph captured (1/0), solver CTAs, co-resident CTA
 * budget, vector width, autotune choice (-1 = not tuned)} */
afl_status afl_ensemble_info(const afl_ensemble *e, int32_t out[6]);
afl_status afl_ensemble_instance_ctas(const afl_ensemble *e, int32_t *out, int count);
/* Tile depth of the batched stage kernels: each CTA covers a 32 x 8 tile of
 * kz consecutive z planes (1, 2 or 4).  afl_ensemble_autotune chooses it with
 * the solver's CTA split; these set and read it directly. */
afl_status afl_ensemble_set_tile_depth(afl_ensemble *e, int32_t kz);
afl_status afl_ensemble_tile_depth(const afl_ensemble *e, int32_t *kz);
/* Step form: 1 = one persistent cooperative launch per step, the CTAs of
 * each instance meeting at the instance's own bounded barrier between stages
 * (the default when the step kernel's co-resident CTAs outnumber the
 * instances); 0 = the captured graph of per-stage batched launches plus the
 * cooperative solve.  Setting it re-splits the CTAs for the form's
 * co-resident budget, clears the autotune choice and captures the step again. */
afl_status afl_ensemble_set_persistent(afl_ensemble *e, int32_t on);
afl_status afl_ensemble_persistent(const afl_ensemble *e, int32_t *on);
/* The reference generator (src/rng.rs:21-88): n values of next_f64 after
 * skipping `skip` next_u64 draws from Rng::from_seed(seed). */
afl_status afl_rng_f64(uint64_t seed, uint64_t skip, size_t n, double *out);

/* ---- reverse mode (no reference counterpart) --------------------------------
 * Gradient of a function of the final density with respect to the initial
 * velocity and the per-cell temperature amplitude of the sphere source, through
 * `steps` FP64 steps.  Hand-written adjoints of every stage; MacCormack clamp
 * branches and the jets' caps are recorded.  Sources: the sphere
 * (AFL_SOURCE_SPHERE), the reference's cyberpunk jets (step n at time n*dt)
 * or none.  Pressure solves: CG, whose adjoint solve uses the same
 * symmetric-operator CG (solves treated as exact, so use a tight cg_rel_tol),
 * or red-black SOR with solver_iters sweeps, transposed sweep by sweep (its
 * warm start from the previous step's pressure carries an adjoint between
 * steps).  The state is checkpointed every `checkpoint_every` steps and each
 * segment is recomputed during the backward pass.  FP64 only
 * (params.precision is ignored). */
typedef struct afl_adjoint afl_adjoint;
/* params: source_kind and solver_kind as above; poisson_kernel picks the CG
 * kernel as in afl_create. */
afl_status afl_adjoint_create(size_t nx, size_t ny, size_t nz, const afl_params *params,
                              int checkpoint_every, afl_adjoint **out);
afl_status afl_adjoint_destroy(afl_adjoint *a);
/* Host arrays of nx*ny*nz doubles; amp may be NULL (all 1); rho_final may be
 * NULL.  Density, temperature and pressure start at zero. */
afl_status afl_adjoint_forward(afl_adjoint *a, const double *u0, const double *v0,
                               const double *w0, const double *amp, int steps, double dt,
                               double *rho_final);
/* rho_bar: the gradient of the function with respect to the final density.
 * Any output may be NULL. */
afl_status afl_adjoint_backward(afl_adjoint *a, const double *rho_bar, double *u0_bar,
                                double *v0_bar, double *w0_bar, double *amp_bar);
/* out = {last forward ms, last backward ms (recompute included), forward CG
 * iterations, adjoint CG iterations} */
afl_status afl_adjoint_stats(const afl_adjoint *a, double out[4]);

/* ---- FluidMedium on the device (src/fluid.rs:687-874) ----------------------
 * The renderer's medium queries over a snapshot of a solver's density and
 * temperature, kept on the GPU.  afl_medium_create replaces
 * FluidMedium::from_solver (src/fluid.rs:703-732): it copies the two fields
 * (as f64), takes the max density and the majorant
 * max(max_density * sigma_t_scale, 1e-4), clamps phase_g to [-0.9, 0.9] and
 * orders the bounds as Aabb::new does.  Later steps of the solver do not change
 * the medium.
 *
 * Queries take host arrays and return host arrays; the medium keeps device
 * staging buffers that grow to the largest batch seen.  A ray is given as in
 * Ray::new (the direction is normalised inside, src/math.rs:763-774) plus the
 * end of its segment: `surface_t` of sample_interaction (src/fluid.rs:793-799) or
 * `max_dist` of transmittance (src/fluid.rs:841).  Each ray draws from its own
 * Rng::from_seed(seed + ray index) stream, so results do not depend on batch
 * order or size (the reference threads one generator through a path). */
typedef struct afl_medium afl_medium;
typedef struct afl_ray {
  double origin[3];
  double dir[3];
  double t_min; /* Ray::t_min */
  double t_end; /* surface_t (interaction) or max_dist (transmittance) */
} afl_ray;
afl_status afl_medium_create(afl_solver *s, const double bounds_min[3],
                             const double bounds_max[3], double sigma_t_scale, double phase_g,
                             afl_medium **out);
afl_status afl_medium_destroy(afl_medium *m);
/* out = {max_density, majorant_sigma_t, phase_g, sigma_t_scale} */
afl_status afl_medium_info(const afl_medium *m, double out[4]);
/* sample_density_and_temp (src/fluid.rs:739-786) at n points (x, y, z). */
afl_status afl_medium_sample_density_temp(afl_medium *m, const double *points, size_t n,
                                          double *density, double *temperature);
/* Ratio-tracking transmittance in [0, 1] (src/fluid.rs:840-874) per ray. */
afl_status afl_medium_transmittance(afl_medium *m, const afl_ray *rays, size_t n,
                                    uint64_t seed, double *transmittance);
/* Delta-tracking free flight (src/fluid.rs:792-838) per ray: hit[r] = 1 and the
 * distance t, density and temperature at ray.at(t) when the ray interacts
 * before t_end, else hit[r] = 0 (t, density, temperature = 0).  Any of t,
 * density, temperature may be NULL. */
afl_status afl_medium_sample_interaction(afl_medium *m, const afl_ray *rays, size_t n,
                                         uint64_t seed, int32_t *hit, double *t,
                                         double *density, double *temperature);

/* ---- a pressure solve that allocates nothing --------------------------------
 * No counterpart in the reference.  For callers that may not allocate device
 * memory -- real-time/render threads that must not block on the driver's
 * allocator, hosts whose device memory is one budgeted pool -- this runs the
 * streaming FP64 CG kernel (the one afl_solve_cg runs with
 * AFL_POISSON_KERNEL_STREAMING; same stopping rules, warm start from
 * *d_pressure) on device buffers the caller owns: d_rhs (read) and d_pressure
 * (read and written), nx*ny*nz doubles each, x fastest.  Its working memory is
 * a fixed array inside the library (about 8.1 MiB, held on every GPU that
 * loads the library until exit), so grids larger than 262144 cells (64^3) are
 * rejected with AFL_ERR_INVALID_ARGUMENT.  The first call on each device looks
 * up that array's device address (with the device current) and should come
 * before any stream capture.  All calls share the array: calls whose work
 * overlaps on one GPU race and must be ordered by the caller.  Runs on
 * `stream` (a cudaStream_t, NULL = legacy default) and synchronises it before
 * returning, to read the solve's report; info may be NULL; errors are
 * reported through afl_last_error(). */
afl_status afl_solve_cg_noalloc(const double *d_rhs, double *d_pressure, size_t nx, size_t ny,
                                size_t nz, int max_iters, double rel_tol, void *stream,
                                afl_solve_info *info);

afl_status afl_synchronize(afl_solver *s);
/* The handle's cudaStream_t, for callers that order their own work on it. */
void *afl_stream(afl_solver *s);

#ifdef __cplusplus
}
#endif
#endif /* AETHER_FLUID_H */
