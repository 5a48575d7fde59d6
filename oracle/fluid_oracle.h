/*
 * fluid_oracle.h -- CPU restatement of the reference smoke solver.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle: a scalar, single-threaded,
 * f64 restatement of `FluidSolver3D` (src/fluid.rs:23-673), of the volume
 * queries of `FluidMedium` (src/fluid.rs:687-874) and of the
 * SplitMix64/Xoshiro256++ generator (src/rng.rs:5-88) of
 * vanovri/aether-core-engine.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it, and only to check results.  The
 * product path (libaether_fluid.so) never links or calls it.
 *
 * Parity pin: the reference is Rust and cannot be built in this image, so the
 * restatement is pinned by the reference's only published numeric output for
 * this path -- the projection known answer printed in README.md:54 (produced
 * by src/verify.rs:229-250: RMS divergence 2.5751e0 -> 6.7289e-3) -- and by
 * the invariant tests of src/fluid.rs:917-968.  Everything else the oracle
 * emits (the golden fields under tests/golden/) is generated from this
 * restatement.
 *
 * Compile with -O2 -ffp-contract=off: rustc never contracts a*b+c into an FMA
 * unless `mul_add` is written, and the reference writes none.
 */
#ifndef AETHER_FLUID_ORACLE_H
#define AETHER_FLUID_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ofl_solver ofl_solver;

/* Field ids: the order of the public Vec<f64> fields of FluidSolver3D
 * (src/fluid.rs:28-34). */
enum {
  OFL_U = 0, OFL_V = 1, OFL_W = 2, OFL_DENSITY = 3, OFL_TEMPERATURE = 4,
  OFL_PRESSURE = 5, OFL_DIVERGENCE = 6
};

/* Source kinds used by ofl_step.  CYBERPUNK is the reference's hard-wired
 * inject_cyberpunk_sources (src/fluid.rs:532-595); SPHERE is the documented
 * extension that assigns density/temperature inside a sphere; NONE skips the
 * injection. */
enum { OFL_SOURCE_CYBERPUNK = 0, OFL_SOURCE_SPHERE = 1, OFL_SOURCE_NONE = 2 };

/* Poisson solver kind (src/fluid.rs:17-21). */
enum { OFL_CG = 0, OFL_RBGS = 1 };

ofl_solver *ofl_create(size_t nx, size_t ny, size_t nz);
void ofl_destroy(ofl_solver *s);

double ofl_h(const ofl_solver *s);
size_t ofl_cells(const ofl_solver *s);
/* Direct view of a field's storage (x fastest, nx*ny*nz doubles). */
double *ofl_field(ofl_solver *s, int field);

/* Solver knobs.  The reference fields are vorticity_eps, buoyancy_beta,
 * gravity_alpha, solver_kind, solver_iters (src/fluid.rs:45-49); sor_omega
 * (reference constant 1.65, src/fluid.rs:398) and cg_rel_tol (0 = the
 * reference's absolute-only stopping rule) are the extensions. */
void ofl_set_params(ofl_solver *s, double vorticity_eps, double buoyancy_beta,
                    double gravity_alpha, int solver_kind, int solver_iters,
                    double sor_omega, double cg_rel_tol);

/* Sphere source: cells with integer-index distance^2 < r^2 inside the
 * [1, n-2] box get density = rho_value and temperature = temp_value (times
 * temp_amp[id] when temp_amp is non-NULL; the array is copied). */
void ofl_set_sphere_source(ofl_solver *s, double cx, double cy, double cz,
                           double radius, double rho_value, double temp_value,
                           const double *temp_amp);
void ofl_set_source_kind(ofl_solver *s, int kind);

/* Stage calls mirroring the reference's methods. */
void ofl_advect_maccormack(ofl_solver *s, int field_kind, double dt,
                           double dissipation);
void ofl_enforce_wall_bc(ofl_solver *s);
void ofl_buoyancy_vorticity(ofl_solver *s, double dt);
double ofl_divergence_norm(ofl_solver *s);
/* Returns iterations executed; *final_delta gets the last r.r. */
int ofl_solve_cg(ofl_solver *s, int max_iters, double *final_delta);
void ofl_solve_rbgs(ofl_solver *s, int iterations);
int ofl_project(ofl_solver *s);
void ofl_inject_cyberpunk(ofl_solver *s, double time_sec, double dt);
void ofl_inject_sphere(ofl_solver *s);
/* telemetry[8] = time, KE, enstrophy, peak |w|, mass, com.x, com.y, com.z */
void ofl_step(ofl_solver *s, double dt, double time_sec, double *telemetry);
void ofl_compute_telemetry(const ofl_solver *s, double time_sec,
                           double *telemetry);
double ofl_max_density(const ofl_solver *s);
/* CG iterations spent by the last projection (or -1 for RB-GS). */
int ofl_last_cg_iters(const ofl_solver *s);

/* Runs `steps` steps with constant dt and time = t0 + n*dt_time; returns the
 * summed CG iterations and, when telemetry is non-NULL, writes 8 doubles per
 * step. */
long ofl_run(ofl_solver *s, int steps, double dt, double t0, double dt_time,
             double *telemetry);

/* Seeded initial condition: Rng::from_seed(seed), then for u, v, w in that
 * order and id in 0..N: range_f64(lo, hi); then enforce_wall_velocity_bc. */
void ofl_init_velocity_noise(ofl_solver *s, uint64_t seed, double lo,
                             double hi);

/* Generator access for tests (src/rng.rs:21-88). */
void ofl_rng_u64(uint64_t seed, size_t n, uint64_t *out);
void ofl_rng_f64(uint64_t seed, size_t n, double *out);

/* FluidMedium volume queries (src/fluid.rs:687-874) over host arrays of
 * nx*ny*nz doubles.  Bounds are ordered as Aabb::new does; the max density
 * and the majorant are taken as FluidMedium::from_solver does.  A ray is 8
 * doubles: origin[3], dir[3] (normalised as Ray::new does), t_min, t_end.
 * Ray r draws from Rng::from_seed(seed + r). */
void ofl_medium_sample(const double *dens, const double *temp, size_t nx, size_t ny, size_t nz,
                       const double *bmin, const double *bmax, const double *pts, size_t n,
                       double *rho, double *tmp);
void ofl_medium_transmittance(const double *dens, const double *temp, size_t nx, size_t ny,
                              size_t nz, const double *bmin, const double *bmax,
                              double sigma_t_scale, const double *rays, size_t n, uint64_t seed,
                              double *tr);
void ofl_medium_interaction(const double *dens, const double *temp, size_t nx, size_t ny,
                            size_t nz, const double *bmin, const double *bmax,
                            double sigma_t_scale, const double *rays, size_t n, uint64_t seed,
                            int32_t *hit, double *t, double *rho, double *tmp);

#ifdef __cplusplus
}
#endif
#endif
