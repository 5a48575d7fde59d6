// fluid_oracle.cpp -- TEST INFRASTRUCTURE: the f64 CPU oracle.
//
// A scalar restatement of FluidSolver3D (src/fluid.rs:23-673) and Rng
// (src/rng.rs:5-88) of vanovri/aether-core-engine.  Every loop keeps the
// reference's iteration order (k outer, j, i inner) and every expression keeps
// the reference's operation order, so that the f64 results agree bit for bit
// with a rustc build (no FMA contraction: build with -ffp-contract=off).
// Rust semantics that C++ does not share are spelled out:
//   * f64::min / f64::max return the non-NaN operand -> std::fmin / std::fmax
//   * f64::clamp(lo, hi) is "if x < lo {lo} else if x > hi {hi} else {x}"
//   * `as usize` on a double saturates (negative / NaN -> 0)
// Only tests/, the smoke check and bench.py's CPU-baseline leg load this file.

#include "fluid_oracle.h"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr double kTau = 6.283185307179586;  // std::f64::consts::TAU

inline double rs_clamp(double x, double lo, double hi) {
  // f64::clamp (core::f64): lower bound checked first, then the upper one.
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}

inline size_t rs_as_usize(double x) {
  // `f as usize`: saturating, NaN -> 0.
  if (!(x > 0.0)) return 0;
  if (x >= 18446744073709551616.0) return SIZE_MAX;
  return static_cast<size_t>(x);
}

// ---------------------------------------------------------------- RNG ------
// src/rng.rs:5-11 (splitmix64) and :20-88 (from_seed, next_u64, next_f64,
// range_f64).  Integer work, bit exact.
inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

inline uint64_t splitmix_next(uint64_t &state) {
  state += 0x9E3779B97F4A7C15ull;
  uint64_t z = state;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct Xoshiro {
  uint64_t s[4];
  explicit Xoshiro(uint64_t seed) {
    uint64_t sm = seed ^ 0xA5A55A5AF0F00F0Full;
    for (int i = 0; i < 4; ++i) s[i] = splitmix_next(sm);
    if ((s[0] | s[1] | s[2] | s[3]) == 0) s[0] = 1;
  }
  uint64_t next_u64() {
    const uint64_t result = rotl64(s[0] + s[3], 23) + s[0];
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl64(s[3], 45);
    return result;
  }
  double next_f64() {
    const double scale = 1.0 / 9007199254740992.0;  // 1 / 2^53
    return static_cast<double>(next_u64() >> 11) * scale;
  }
  double range_f64(double lo, double hi) { return lo + (hi - lo) * next_f64(); }
};

}  // namespace

struct ofl_solver {
  size_t nx, ny, nz;
  double h;
  // public fields (src/fluid.rs:28-34)
  std::vector<double> f[7];
  // private scratch (src/fluid.rs:35-44)
  std::vector<double> curl_x, curl_y, curl_z, curl_mag;
  std::vector<double> tmp_fwd, tmp_bwd, tmp_out;
  std::vector<double> cg_r, cg_d, cg_q;
  // knobs (src/fluid.rs:45-49 + extensions)
  double vorticity_eps = 5.5, buoyancy_beta = 6.8, gravity_alpha = 0.45;
  int solver_kind = OFL_CG;
  int solver_iters = 32;
  double sor_omega = 1.65;
  double cg_rel_tol = 0.0;
  // source extension
  int source_kind = OFL_SOURCE_CYBERPUNK;
  double sph_c[3] = {0, 0, 0}, sph_r = 0, sph_rho = 1, sph_temp = 1;
  std::vector<double> sph_amp;
  int last_cg_iters = -1;
  double last_cg_delta = 0.0;

  size_t idx(size_t i, size_t j, size_t k) const { return (k * ny + j) * nx + i; }
  std::vector<double> &U() { return f[OFL_U]; }
  std::vector<double> &V() { return f[OFL_V]; }
  std::vector<double> &W() { return f[OFL_W]; }
  std::vector<double> &P() { return f[OFL_PRESSURE]; }
  std::vector<double> &B() { return f[OFL_DIVERGENCE]; }
};

namespace {

// src/fluid.rs:94-128
double sample_trilinear(const ofl_solver &s, const std::vector<double> &field,
                        double x, double y, double z) {
  const double xc = rs_clamp(x, 0.5, static_cast<double>(s.nx) - 1.500001);
  const double yc = rs_clamp(y, 0.5, static_cast<double>(s.ny) - 1.500001);
  const double zc = rs_clamp(z, 0.5, static_cast<double>(s.nz) - 1.500001);
  const size_t i0 = rs_as_usize(std::floor(xc));
  const size_t j0 = rs_as_usize(std::floor(yc));
  const size_t k0 = rs_as_usize(std::floor(zc));
  const size_t i1 = i0 + 1, j1 = j0 + 1, k1 = k0 + 1;
  const double tx = xc - static_cast<double>(i0);
  const double ty = yc - static_cast<double>(j0);
  const double tz = zc - static_cast<double>(k0);
  const double c000 = field[s.idx(i0, j0, k0)];
  const double c100 = field[s.idx(i1, j0, k0)];
  const double c010 = field[s.idx(i0, j1, k0)];
  const double c110 = field[s.idx(i1, j1, k0)];
  const double c001 = field[s.idx(i0, j0, k1)];
  const double c101 = field[s.idx(i1, j0, k1)];
  const double c011 = field[s.idx(i0, j1, k1)];
  const double c111 = field[s.idx(i1, j1, k1)];
  const double c00 = c000 * (1.0 - tx) + c100 * tx;
  const double c10 = c010 * (1.0 - tx) + c110 * tx;
  const double c01 = c001 * (1.0 - tx) + c101 * tx;
  const double c11 = c011 * (1.0 - tx) + c111 * tx;
  const double c0 = c00 * (1.0 - ty) + c10 * ty;
  const double c1 = c01 * (1.0 - ty) + c11 * ty;
  return c0 * (1.0 - tz) + c1 * tz;
}

// src/fluid.rs:131-150
void stencil_minmax(const ofl_solver &s, const std::vector<double> &field,
                    double x, double y, double z, double &lo, double &hi) {
  const double xc = rs_clamp(x, 0.5, static_cast<double>(s.nx) - 1.500001);
  const double yc = rs_clamp(y, 0.5, static_cast<double>(s.ny) - 1.500001);
  const double zc = rs_clamp(z, 0.5, static_cast<double>(s.nz) - 1.500001);
  const size_t i0 = rs_as_usize(std::floor(xc));
  const size_t j0 = rs_as_usize(std::floor(yc));
  const size_t k0 = rs_as_usize(std::floor(zc));
  lo = INFINITY;
  hi = -INFINITY;
  for (size_t dk = 0; dk <= 1; ++dk)
    for (size_t dj = 0; dj <= 1; ++dj)
      for (size_t di = 0; di <= 1; ++di) {
        const double v = field[s.idx(i0 + di, j0 + dj, k0 + dk)];
        lo = std::fmin(lo, v);
        hi = std::fmax(hi, v);
      }
}

// src/fluid.rs:153-167
void advect_semi_lagrangian(const ofl_solver &s, const std::vector<double> &src,
                            std::vector<double> &dst, double dt) {
  const double scale = dt / s.h;
  std::fill(dst.begin(), dst.end(), 0.0);
  const std::vector<double> &u = s.f[OFL_U], &v = s.f[OFL_V], &w = s.f[OFL_W];
  for (size_t k = 1; k < s.nz - 1; ++k)
    for (size_t j = 1; j < s.ny - 1; ++j)
      for (size_t i = 1; i < s.nx - 1; ++i) {
        const size_t id = s.idx(i, j, k);
        const double bx = static_cast<double>(i) - scale * u[id];
        const double by = static_cast<double>(j) - scale * v[id];
        const double bz = static_cast<double>(k) - scale * w[id];
        dst[id] = sample_trilinear(s, src, bx, by, bz);
      }
}

// src/fluid.rs:236-253
void enforce_wall_bc(ofl_solver &s) {
  std::vector<double> &u = s.U(), &v = s.V(), &w = s.W();
  const size_t nx = s.nx, ny = s.ny, nz = s.nz;
  for (size_t k = 0; k < nz; ++k)
    for (size_t j = 0; j < ny; ++j)
      for (size_t i = 0; i < nx; ++i) {
        const size_t id = s.idx(i, j, k);
        if (i <= 1 || i + 1 >= nx || j == 0 || j + 1 >= ny || k == 0 || k + 1 >= nz) u[id] = 0.0;
        if (j <= 1 || j + 1 >= ny || i == 0 || i + 1 >= nx || k == 0 || k + 1 >= nz) v[id] = 0.0;
        if (k <= 1 || k + 1 >= nz || i == 0 || i + 1 >= nx || j == 0 || j + 1 >= ny) w[id] = 0.0;
      }
}

// src/fluid.rs:356-394
void apply_spd_laplacian(const ofl_solver &s, const std::vector<double> &x,
                         std::vector<double> &out) {
  std::fill(out.begin(), out.end(), 0.0);
  for (size_t k = 1; k < s.nz - 1; ++k)
    for (size_t j = 1; j < s.ny - 1; ++j)
      for (size_t i = 1; i < s.nx - 1; ++i) {
        const size_t id = s.idx(i, j, k);
        double diag = 0.0, nb = 0.0;
        if (i > 1) { diag += 1.0; nb += x[s.idx(i - 1, j, k)]; }
        if (i + 2 < s.nx) { diag += 1.0; nb += x[s.idx(i + 1, j, k)]; }
        if (j > 1) { diag += 1.0; nb += x[s.idx(i, j - 1, k)]; }
        if (j + 2 < s.ny) { diag += 1.0; nb += x[s.idx(i, j + 1, k)]; }
        if (k > 1) { diag += 1.0; nb += x[s.idx(i, j, k - 1)]; }
        if (k + 2 < s.nz) { diag += 1.0; nb += x[s.idx(i, j, k + 1)]; }
        out[id] = diag * x[id] - nb;
      }
}

// Sphere-source bounding box, same rule as the jets' box of
// src/fluid.rs:566-571 (floor/ceil +-(r+1), clamped to [1, n-2]).
void source_box(const ofl_solver &s, double cx, double cy, double cz, double r,
                size_t lo[3], size_t hi[3]) {
  lo[2] = rs_as_usize(std::fmax(std::floor(cz - r - 1.0), 1.0));
  hi[2] = rs_as_usize(std::fmin(std::ceil(cz + r + 1.0), static_cast<double>(s.nz - 2)));
  lo[1] = rs_as_usize(std::fmax(std::floor(cy - r - 1.0), 1.0));
  hi[1] = rs_as_usize(std::fmin(std::ceil(cy + r + 1.0), static_cast<double>(s.ny - 2)));
  lo[0] = rs_as_usize(std::fmax(std::floor(cx - r - 1.0), 1.0));
  hi[0] = rs_as_usize(std::fmin(std::ceil(cx + r + 1.0), static_cast<double>(s.nx - 2)));
}

}  // namespace

extern "C" {

ofl_solver *ofl_create(size_t nx, size_t ny, size_t nz) {
  // src/fluid.rs:53-85 (the assert at :54 becomes a NULL return)
  if (nx < 6 || ny < 6 || nz < 6) return nullptr;
  auto *s = new ofl_solver();
  s->nx = nx;
  s->ny = ny;
  s->nz = nz;
  const size_t nmax = std::max(nx, std::max(ny, nz));
  s->h = 1.0 / static_cast<double>(nmax);
  const size_t n = nx * ny * nz;
  for (auto &v : s->f) v.assign(n, 0.0);
  for (auto *v : {&s->curl_x, &s->curl_y, &s->curl_z, &s->curl_mag, &s->tmp_fwd,
                  &s->tmp_bwd, &s->tmp_out, &s->cg_r, &s->cg_d, &s->cg_q})
    v->assign(n, 0.0);
  return s;
}

void ofl_destroy(ofl_solver *s) { delete s; }
double ofl_h(const ofl_solver *s) { return s->h; }
size_t ofl_cells(const ofl_solver *s) { return s->nx * s->ny * s->nz; }
double *ofl_field(ofl_solver *s, int field) {
  if (field < 0 || field > 6) return nullptr;
  return s->f[field].data();
}

void ofl_set_params(ofl_solver *s, double eps, double beta, double alpha,
                    int kind, int iters, double omega, double rel_tol) {
  s->vorticity_eps = eps;
  s->buoyancy_beta = beta;
  s->gravity_alpha = alpha;
  s->solver_kind = kind;
  s->solver_iters = iters;
  s->sor_omega = omega;
  s->cg_rel_tol = rel_tol;
}

void ofl_set_sphere_source(ofl_solver *s, double cx, double cy, double cz,
                           double radius, double rho_value, double temp_value,
                           const double *temp_amp) {
  s->sph_c[0] = cx;
  s->sph_c[1] = cy;
  s->sph_c[2] = cz;
  s->sph_r = radius;
  s->sph_rho = rho_value;
  s->sph_temp = temp_value;
  if (temp_amp)
    s->sph_amp.assign(temp_amp, temp_amp + ofl_cells(s));
  else
    s->sph_amp.clear();
}

void ofl_set_source_kind(ofl_solver *s, int kind) { s->source_kind = kind; }

// src/fluid.rs:170-234
void ofl_advect_maccormack(ofl_solver *s, int field_kind, double dt,
                           double dissipation) {
  const int fid = (field_kind >= 0 && field_kind <= 3) ? field_kind : 4;  // `_ =>` arm
  const std::vector<double> src = s->f[fid];  // the snapshot clone (:171-177)
  std::vector<double> &fwd = s->tmp_fwd, &bwd = s->tmp_bwd, &out = s->tmp_out;
  advect_semi_lagrangian(*s, src, fwd, dt);
  advect_semi_lagrangian(*s, fwd, bwd, -dt);
  std::fill(out.begin(), out.end(), 0.0);
  const double scale = dt / s->h;
  const std::vector<double> &u = s->f[OFL_U], &v = s->f[OFL_V], &w = s->f[OFL_W];
  const double xhi = static_cast<double>(s->nx) - 2.5;
  const double yhi = static_cast<double>(s->ny) - 2.5;
  const double zhi = static_cast<double>(s->nz) - 2.5;
  for (size_t k = 1; k < s->nz - 1; ++k)
    for (size_t j = 1; j < s->ny - 1; ++j)
      for (size_t i = 1; i < s->nx - 1; ++i) {
        const size_t id = s->idx(i, j, k);
        const double bx = static_cast<double>(i) - scale * u[id];
        const double by = static_cast<double>(j) - scale * v[id];
        const double bz = static_cast<double>(k) - scale * w[id];
        const bool near_wall = bx < 1.5 || bx > xhi || by < 1.5 || by > yhi ||
                               bz < 1.5 || bz > zhi;
        double val;
        if (near_wall) {
          val = fwd[id];
        } else {
          const double mc = fwd[id] + 0.5 * (src[id] - bwd[id]);
          double lo, hi;
          stencil_minmax(*s, src, bx, by, bz, lo, hi);
          val = rs_clamp(mc, lo, hi);
        }
        out[id] = val * dissipation;
      }
  std::vector<double> &dst = s->f[fid];
  if (fid <= 2) {
    dst = out;
  } else {
    for (size_t id = 0; id < dst.size(); ++id) dst[id] = std::fmax(out[id], 0.0);
  }
}

void ofl_enforce_wall_bc(ofl_solver *s) { enforce_wall_bc(*s); }

// src/fluid.rs:256-330
void ofl_buoyancy_vorticity(ofl_solver *s, double dt) {
  const double inv_2h = 0.5 / s->h;
  std::vector<double> &u = s->U(), &v = s->V(), &w = s->W();
  const std::vector<double> &rho = s->f[OFL_DENSITY], &temp = s->f[OFL_TEMPERATURE];
  std::fill(s->curl_mag.begin(), s->curl_mag.end(), 0.0);
  for (size_t k = 1; k < s->nz - 1; ++k)
    for (size_t j = 1; j < s->ny - 1; ++j)
      for (size_t i = 1; i < s->nx - 1; ++i) {
        const size_t id = s->idx(i, j, k);
        const double dw_dy = (w[s->idx(i, j + 1, k)] - w[s->idx(i, j - 1, k)]) * inv_2h;
        const double dv_dz = (v[s->idx(i, j, k + 1)] - v[s->idx(i, j, k - 1)]) * inv_2h;
        const double du_dz = (u[s->idx(i, j, k + 1)] - u[s->idx(i, j, k - 1)]) * inv_2h;
        const double dw_dx = (w[s->idx(i + 1, j, k)] - w[s->idx(i - 1, j, k)]) * inv_2h;
        const double dv_dx = (v[s->idx(i + 1, j, k)] - v[s->idx(i - 1, j, k)]) * inv_2h;
        const double du_dy = (u[s->idx(i, j + 1, k)] - u[s->idx(i, j - 1, k)]) * inv_2h;
        const double ox = dw_dy - dv_dz;
        const double oy = du_dz - dw_dx;
        const double oz = dv_dx - du_dy;
        s->curl_x[id] = ox;
        s->curl_y[id] = oy;
        s->curl_z[id] = oz;
        s->curl_mag[id] = std::sqrt(ox * ox + oy * oy + oz * oz);
      }
  const double eps_h = s->vorticity_eps * s->h;
  const std::vector<double> &cm = s->curl_mag;
  for (size_t k = 2; k < s->nz - 2; ++k)
    for (size_t j = 2; j < s->ny - 2; ++j)
      for (size_t i = 2; i < s->nx - 2; ++i) {
        const size_t id = s->idx(i, j, k);
        const double gx = (cm[s->idx(i + 1, j, k)] - cm[s->idx(i - 1, j, k)]) * inv_2h;
        const double gy = (cm[s->idx(i, j + 1, k)] - cm[s->idx(i, j - 1, k)]) * inv_2h;
        const double gz = (cm[s->idx(i, j, k + 1)] - cm[s->idx(i, j, k - 1)]) * inv_2h;
        const double glen = std::sqrt(gx * gx + gy * gy + gz * gz) + 1e-10;
        const double nx = gx / glen, ny = gy / glen, nz = gz / glen;
        const double ox = s->curl_x[id], oy = s->curl_y[id], oz = s->curl_z[id];
        const double fx = eps_h * (ny * oz - nz * oy);
        const double fy = eps_h * (nz * ox - nx * oz);
        const double fz = eps_h * (nx * oy - ny * ox);
        u[id] += dt * fx;
        v[id] += dt * fy;
        w[id] += dt * fz;
      }
  for (size_t k = 1; k < s->nz - 1; ++k)
    for (size_t j = 1; j < s->ny - 1; ++j)
      for (size_t i = 1; i < s->nx - 1; ++i) {
        const size_t id = s->idx(i, j, k);
        const double lift = s->buoyancy_beta * temp[id] - s->gravity_alpha * rho[id];
        v[id] += dt * lift;
      }
  enforce_wall_bc(*s);
}

// src/fluid.rs:333-353
double ofl_divergence_norm(ofl_solver *s) {
  const double inv_h = 1.0 / s->h;
  double sum_sq = 0.0;
  std::vector<double> &b = s->B();
  const std::vector<double> &u = s->f[OFL_U], &v = s->f[OFL_V], &w = s->f[OFL_W];
  std::fill(b.begin(), b.end(), 0.0);
  for (size_t k = 1; k < s->nz - 1; ++k)
    for (size_t j = 1; j < s->ny - 1; ++j)
      for (size_t i = 1; i < s->nx - 1; ++i) {
        const size_t id = s->idx(i, j, k);
        const double du = u[s->idx(i + 1, j, k)] - u[id];
        const double dv = v[s->idx(i, j + 1, k)] - v[id];
        const double dw = w[s->idx(i, j, k + 1)] - w[id];
        const double div_val = (du + dv + dw) * inv_h;
        b[id] = -s->h * (du + dv + dw);
        sum_sq += div_val * div_val;
      }
  const double interior = static_cast<double>((s->nx - 2) * (s->ny - 2) * (s->nz - 2));
  return std::sqrt(sum_sq / interior);
}


// src/fluid.rs:445-493.  Extension: with cg_rel_tol > 0 the solve also stops
// when sqrt(r.r) <= cg_rel_tol * ||b||_2, tested in the position of the
// reference's absolute test r.r < 1e-20 (:479); the warm-start skip (:462)
// likewise also fires when sqrt(r0.r0) <= cg_rel_tol * ||b||_2.  With
// cg_rel_tol == 0 the loop is exactly the reference's.  Returns the number of
// executed p/r updates.
int ofl_solve_cg(ofl_solver *s, int max_iters, double *final_delta) {
  std::vector<double> &r = s->cg_r, &d = s->cg_d, &q = s->cg_q;
  std::vector<double> &p = s->P();
  const std::vector<double> &b = s->B();
  const size_t n = p.size();
  apply_spd_laplacian(*s, p, q);  // warm start from the previous pressure
  double delta_new = 0.0;
  for (size_t i = 0; i < n; ++i) {
    const double ri = b[i] - q[i];
    r[i] = ri;
    d[i] = ri;
    delta_new += ri * ri;
  }
  double tol2 = -1.0;
  if (s->cg_rel_tol > 0.0) {
    double bb = 0.0;
    for (size_t i = 0; i < n; ++i) bb += b[i] * b[i];
    const double t = s->cg_rel_tol * std::sqrt(bb);
    tol2 = t * t;
  }
  double last = delta_new;
  int it = 0;
  const bool rel_done = tol2 >= 0.0 && delta_new <= tol2;
  if (delta_new > 1e-24 && !rel_done) {
    while (it < max_iters) {
      apply_spd_laplacian(*s, d, q);
      double dq = 0.0;
      for (size_t i = 0; i < n; ++i) dq += d[i] * q[i];
      if (std::fabs(dq) < 1e-28) break;
      const double alpha = delta_new / dq;
      double delta_next = 0.0;
      for (size_t i = 0; i < n; ++i) {
        p[i] += alpha * d[i];
        r[i] -= alpha * q[i];
        delta_next += r[i] * r[i];
      }
      ++it;
      last = delta_next;
      if (delta_next < 1e-20) break;
      if (tol2 >= 0.0 && delta_next <= tol2) break;
      const double beta = delta_next / delta_new;
      for (size_t i = 0; i < n; ++i) d[i] = r[i] + beta * d[i];
      delta_new = delta_next;
    }
  }
  s->last_cg_iters = it;
  s->last_cg_delta = last;
  if (final_delta) *final_delta = last;
  return it;
}

// src/fluid.rs:397-442, with the SOR factor taken from sor_omega (the
// reference's constant is 1.65, :398).
void ofl_solve_rbgs(ofl_solver *s, int iterations) {
  const double omega = s->sor_omega;
  std::vector<double> &p = s->P();
  const std::vector<double> &b = s->B();
  for (int it = 0; it < iterations; ++it)
    for (size_t color = 0; color < 2; ++color)
      for (size_t k = 1; k < s->nz - 1; ++k)
        for (size_t j = 1; j < s->ny - 1; ++j)
          for (size_t i = 1; i < s->nx - 1; ++i) {
            if ((i + j + k) % 2 != color) continue;
            const size_t id = s->idx(i, j, k);
            double diag = 0.0, nb = 0.0;
            if (i > 1) { diag += 1.0; nb += p[s->idx(i - 1, j, k)]; }
            if (i + 2 < s->nx) { diag += 1.0; nb += p[s->idx(i + 1, j, k)]; }
            if (j > 1) { diag += 1.0; nb += p[s->idx(i, j - 1, k)]; }
            if (j + 2 < s->ny) { diag += 1.0; nb += p[s->idx(i, j + 1, k)]; }
            if (k > 1) { diag += 1.0; nb += p[s->idx(i, j, k - 1)]; }
            if (k + 2 < s->nz) { diag += 1.0; nb += p[s->idx(i, j, k + 1)]; }
            const double gs_target = (b[id] + nb) / diag;
            p[id] = (1.0 - omega) * p[id] + omega * gs_target;
          }
}

// src/fluid.rs:496-529
int ofl_project(ofl_solver *s) {
  enforce_wall_bc(*s);
  (void)ofl_divergence_norm(s);
  int iters = -1;
  if (s->solver_kind == OFL_CG)
    iters = ofl_solve_cg(s, s->solver_iters, nullptr);
  else {
    ofl_solve_rbgs(s, s->solver_iters);
    s->last_cg_iters = -1;
  }
  const double inv_h = 1.0 / s->h;
  std::vector<double> &u = s->U(), &v = s->V(), &w = s->W();
  const std::vector<double> &p = s->f[OFL_PRESSURE];
  for (size_t k = 1; k < s->nz - 1; ++k)
    for (size_t j = 1; j < s->ny - 1; ++j)
      for (size_t i = 1; i < s->nx - 1; ++i) {
        const size_t id = s->idx(i, j, k);
        const double pc = p[id];
        if (i > 1) u[id] -= (pc - p[s->idx(i - 1, j, k)]) * inv_h;
        if (j > 1) v[id] -= (pc - p[s->idx(i, j - 1, k)]) * inv_h;
        if (k > 1) w[id] -= (pc - p[s->idx(i, j, k - 1)]) * inv_h;
      }
  enforce_wall_bc(*s);
  return iters;
}

// src/fluid.rs:532-595
void ofl_inject_cyberpunk(ofl_solver *s, double time_sec, double dt) {
  const double cx = 0.5 * static_cast<double>(s->nx);
  const double cz = 0.5 * static_cast<double>(s->nz);
  const size_t base_j = std::min<size_t>(3, s->ny - 3);
  const double pulse = 0.65 + 0.35 * std::sin(time_sec * kTau * 0.55) +
                       0.25 * std::fmax(std::cos(time_sec * kTau * 1.35), 0.0);
  const double angle = time_sec * 1.85;
  const double orbit_r = static_cast<double>(s->nx) * 0.14;
  const double ca = std::cos(angle), sa = std::sin(angle);
  const double jets[2][6] = {
      {cx + orbit_r * ca, static_cast<double>(base_j) + 1.5, cz + orbit_r * sa,
       -2.6 * sa, 7.2 * pulse, 2.6 * ca},
      {cx - orbit_r * ca, static_cast<double>(base_j) + 2.0, cz - orbit_r * sa,
       2.6 * sa, 6.4 * pulse, -2.6 * ca},
  };
  const double r_cells = std::fmax(static_cast<double>(s->nx) * 0.105, 2.2);
  const double r2 = r_cells * r_cells;
  std::vector<double> &rho = s->f[OFL_DENSITY], &temp = s->f[OFL_TEMPERATURE];
  std::vector<double> &u = s->U(), &v = s->V(), &w = s->W();
  for (const auto &jet : jets) {
    const double jx = jet[0], jy = jet[1], jz = jet[2];
    const double vx = jet[3], vy = jet[4], vz = jet[5];
    size_t lo[3], hi[3];
    source_box(*s, jx, jy, jz, r_cells, lo, hi);
    for (size_t k = lo[2]; k <= hi[2]; ++k)
      for (size_t j = lo[1]; j <= hi[1]; ++j)
        for (size_t i = lo[0]; i <= hi[0]; ++i) {
          const double dx = static_cast<double>(i) - jx;
          const double dy = static_cast<double>(j) - jy;
          const double dz = static_cast<double>(k) - jz;
          const double d2 = dx * dx + dy * dy + dz * dz;
          if (d2 < r2) {
            const double wf = std::exp(-2.2 * d2 / r2);
            const size_t id = s->idx(i, j, k);
            rho[id] = std::fmin(rho[id] + dt * 9.5 * pulse * wf, 3.8);
            temp[id] = std::fmin(temp[id] + dt * 8.2 * pulse * wf, 4.5);
            u[id] += dt * vx * wf * 4.2;
            v[id] += dt * vy * wf * 4.2;
            w[id] += dt * vz * wf * 4.2;
          }
        }
  }
}

// Sphere source (extension): assignment of density/temperature inside the
// sphere, in the slot of step() where the reference injects its jets.
void ofl_inject_sphere(ofl_solver *s) {
  size_t lo[3], hi[3];
  source_box(*s, s->sph_c[0], s->sph_c[1], s->sph_c[2], s->sph_r, lo, hi);
  const double r2 = s->sph_r * s->sph_r;
  std::vector<double> &rho = s->f[OFL_DENSITY], &temp = s->f[OFL_TEMPERATURE];
  const bool amp = !s->sph_amp.empty();
  for (size_t k = lo[2]; k <= hi[2]; ++k)
    for (size_t j = lo[1]; j <= hi[1]; ++j)
      for (size_t i = lo[0]; i <= hi[0]; ++i) {
        const double dx = static_cast<double>(i) - s->sph_c[0];
        const double dy = static_cast<double>(j) - s->sph_c[1];
        const double dz = static_cast<double>(k) - s->sph_c[2];
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < r2) {
          const size_t id = s->idx(i, j, k);
          rho[id] = s->sph_rho;
          temp[id] = amp ? s->sph_temp * s->sph_amp[id] : s->sph_temp;
        }
      }
}

// src/fluid.rs:613-672
void ofl_compute_telemetry(const ofl_solver *s, double time_sec, double *out) {
  const double h = s->h;
  const double dv = h * h * h;
  const double inv_2h = 0.5 / h;
  const std::vector<double> &u = s->f[OFL_U], &v = s->f[OFL_V], &w = s->f[OFL_W];
  const std::vector<double> &rho = s->f[OFL_DENSITY];
  double ke = 0.0, ens = 0.0, peak = 0.0, mass = 0.0;
  double com[3] = {0.0, 0.0, 0.0};
  for (size_t k = 1; k < s->nz - 1; ++k)
    for (size_t j = 1; j < s->ny - 1; ++j)
      for (size_t i = 1; i < s->nx - 1; ++i) {
        const size_t id = s->idx(i, j, k);
        const double u2 = u[id] * u[id] + v[id] * v[id] + w[id] * w[id];
        ke += 0.5 * u2 * dv;
        const double dw_dy = (w[s->idx(i, j + 1, k)] - w[s->idx(i, j - 1, k)]) * inv_2h;
        const double dv_dz = (v[s->idx(i, j, k + 1)] - v[s->idx(i, j, k - 1)]) * inv_2h;
        const double du_dz = (u[s->idx(i, j, k + 1)] - u[s->idx(i, j, k - 1)]) * inv_2h;
        const double dw_dx = (w[s->idx(i + 1, j, k)] - w[s->idx(i - 1, j, k)]) * inv_2h;
        const double dv_dx = (v[s->idx(i + 1, j, k)] - v[s->idx(i - 1, j, k)]) * inv_2h;
        const double du_dy = (u[s->idx(i, j + 1, k)] - u[s->idx(i, j - 1, k)]) * inv_2h;
        const double ox = dw_dy - dv_dz;
        const double oy = du_dz - dw_dx;
        const double oz = dv_dx - du_dy;
        const double w2 = ox * ox + oy * oy + oz * oz;
        ens += 0.5 * w2 * dv;
        peak = std::fmax(peak, std::sqrt(w2));
        const double r = rho[id];
        if (r > 1e-8) {
          mass += r * dv;
          const double nxn = 2.0 * (static_cast<double>(i) / static_cast<double>(s->nx - 1)) - 1.0;
          const double nyn = 2.0 * (static_cast<double>(j) / static_cast<double>(s->ny - 1)) - 1.0;
          const double nzn = 2.0 * (static_cast<double>(k) / static_cast<double>(s->nz - 1)) - 1.0;
          const double wgt = r * dv;
          com[0] += nxn * wgt;
          com[1] += nyn * wgt;
          com[2] += nzn * wgt;
        }
      }
  if (mass > 1e-12) {
    const double inv = 1.0 / mass;  // Vec3 /= f64 multiplies by 1/rhs
    for (double &c : com) c = c * inv;
  }
  out[0] = time_sec;
  out[1] = ke;
  out[2] = ens;
  out[3] = peak;
  out[4] = mass;
  for (int a = 0; a < 3; ++a) out[5 + a] = rs_clamp(com[a], -1.0, 1.0);
}

// src/fluid.rs:598-611; the injection slot honours source_kind.
void ofl_step(ofl_solver *s, double dt, double time_sec, double *telemetry) {
  ofl_advect_maccormack(s, 0, dt, 0.996);
  ofl_advect_maccormack(s, 1, dt, 0.996);
  ofl_advect_maccormack(s, 2, dt, 0.996);
  if (s->source_kind == OFL_SOURCE_CYBERPUNK)
    ofl_inject_cyberpunk(s, time_sec, dt);
  else if (s->source_kind == OFL_SOURCE_SPHERE)
    ofl_inject_sphere(s);
  ofl_buoyancy_vorticity(s, dt);
  ofl_project(s);
  ofl_advect_maccormack(s, 3, dt, 0.996);
  ofl_advect_maccormack(s, 4, dt, 0.985);
  double tmp[8];
  ofl_compute_telemetry(s, time_sec, telemetry ? telemetry : tmp);
}

// src/fluid.rs:704-707
double ofl_max_density(const ofl_solver *s) {
  double m = 0.0;
  for (double d : s->f[OFL_DENSITY]) m = std::fmax(m, d);
  return m;
}

int ofl_last_cg_iters(const ofl_solver *s) { return s->last_cg_iters; }

long ofl_run(ofl_solver *s, int steps, double dt, double t0, double dt_time,
             double *telemetry) {
  long total = 0;
  for (int n = 0; n < steps; ++n) {
    ofl_step(s, dt, t0 + static_cast<double>(n) * dt_time,
             telemetry ? telemetry + 8 * static_cast<size_t>(n) : nullptr);
    if (s->last_cg_iters > 0) total += s->last_cg_iters;
  }
  return total;
}

void ofl_init_velocity_noise(ofl_solver *s, uint64_t seed, double lo, double hi) {
  Xoshiro rng(seed);
  for (int f = OFL_U; f <= OFL_W; ++f)
    for (double &x : s->f[f]) x = rng.range_f64(lo, hi);
  enforce_wall_bc(*s);
}

void ofl_rng_u64(uint64_t seed, size_t n, uint64_t *out) {
  Xoshiro rng(seed);
  for (size_t i = 0; i < n; ++i) out[i] = rng.next_u64();
}

void ofl_rng_f64(uint64_t seed, size_t n, double *out) {
  Xoshiro rng(seed);
  for (size_t i = 0; i < n; ++i) out[i] = rng.next_f64();
}

}  // extern "C"

// ---- FluidMedium (src/fluid.rs:687-874) --------------------------------------
namespace {

struct Medium {
  const double *dens, *temp;
  size_t nx, ny, nz;
  double bmin[3], bmax[3];
  double sigma_t_scale, majorant, max_density;
  size_t idx(size_t i, size_t j, size_t k) const { return (k * ny + j) * nx + i; }
};

Medium make_medium(const double *dens, const double *temp, size_t nx, size_t ny, size_t nz,
                   const double *bmin, const double *bmax, double sigma_t_scale) {
  Medium m{dens, temp, nx, ny, nz, {}, {}, sigma_t_scale, 0.0, 0.0};
  for (int a = 0; a < 3; ++a) {  // Aabb::new (src/math.rs:794-799): min_elem / max_elem
    m.bmin[a] = std::fmin(bmin[a], bmax[a]);
    m.bmax[a] = std::fmax(bmin[a], bmax[a]);
  }
  // FluidMedium::from_solver (src/fluid.rs:703-708)
  double mx = 0.0;
  for (size_t c = 0; c < nx * ny * nz; ++c) mx = std::fmax(mx, dens[c]);
  m.max_density = mx;
  m.majorant = std::fmax(mx * sigma_t_scale, 1e-4);
  return m;
}

// sample_density_and_temp (src/fluid.rs:739-786)
void med_sample(const Medium &m, const double p[3], double &rho, double &tmp) {
  if (p[0] < m.bmin[0] || p[0] > m.bmax[0] || p[1] < m.bmin[1] || p[1] > m.bmax[1] ||
      p[2] < m.bmin[2] || p[2] > m.bmax[2]) {
    rho = 0.0;
    tmp = 0.0;
    return;
  }
  double ext[3], uvw[3];
  for (int a = 0; a < 3; ++a) {
    ext[a] = std::fmax(m.bmax[a] - m.bmin[a], 0.0);  // Aabb::extent (src/math.rs:832-834)
    uvw[a] = (p[a] - m.bmin[a]) / std::fmax(ext[a], 1e-9);
  }
  const double ux = uvw[0], uy = uvw[1], uz = uvw[2];
  const double fx = rs_clamp(4.0 * ux * (1.0 - ux), 0.0, 1.0);
  const double fz = rs_clamp(4.0 * uz * (1.0 - uz), 0.0, 1.0);
  const double fy = rs_clamp(1.0 - (std::fmax(uy - 0.95, 0.0) / 0.05), 0.0, 1.0);
  const double feather = std::sqrt(fx * fz * fy);
  const double gx = rs_clamp(ux * static_cast<double>(m.nx - 1), 0.5,
                             static_cast<double>(m.nx) - 1.500001);
  const double gy = rs_clamp(uy * static_cast<double>(m.ny - 1), 0.5,
                             static_cast<double>(m.ny) - 1.500001);
  const double gz = rs_clamp(uz * static_cast<double>(m.nz - 1), 0.5,
                             static_cast<double>(m.nz) - 1.500001);
  const size_t i0 = rs_as_usize(std::floor(gx));
  const size_t j0 = rs_as_usize(std::floor(gy));
  const size_t k0 = rs_as_usize(std::floor(gz));
  const double tx = gx - static_cast<double>(i0);
  const double ty = gy - static_cast<double>(j0);
  const double tz = gz - static_cast<double>(k0);
  auto trilin = [&](const double *buf) {
    const double c000 = buf[m.idx(i0, j0, k0)];
    const double c100 = buf[m.idx(i0 + 1, j0, k0)];
    const double c010 = buf[m.idx(i0, j0 + 1, k0)];
    const double c110 = buf[m.idx(i0 + 1, j0 + 1, k0)];
    const double c001 = buf[m.idx(i0, j0, k0 + 1)];
    const double c101 = buf[m.idx(i0 + 1, j0, k0 + 1)];
    const double c011 = buf[m.idx(i0, j0 + 1, k0 + 1)];
    const double c111 = buf[m.idx(i0 + 1, j0 + 1, k0 + 1)];
    const double c00 = c000 * (1.0 - tx) + c100 * tx;
    const double c10 = c010 * (1.0 - tx) + c110 * tx;
    const double c01 = c001 * (1.0 - tx) + c101 * tx;
    const double c11 = c011 * (1.0 - tx) + c111 * tx;
    return (c00 * (1.0 - ty) + c10 * ty) * (1.0 - tz) + (c01 * (1.0 - ty) + c11 * ty) * tz;
  };
  rho = trilin(m.dens) * feather;
  tmp = trilin(m.temp) * feather;
}

// Ray::new (src/math.rs:763-774) with Vec3::normalize (src/math.rs:58-65); the
// length is dot(self, self).sqrt() with dot written as mul_add
// (src/math.rs:34-36).
struct Ray {
  double o[3], d[3], inv[3];
  double t_min, t_end;
  void at(double t, double p[3]) const {
    for (int a = 0; a < 3; ++a) p[a] = o[a] + d[a] * t;  // Ray::at (src/math.rs:776-779)
  }
};

Ray make_ray(const double *r8) {
  Ray r;
  for (int a = 0; a < 3; ++a) r.o[a] = r8[a];
  const double x = r8[3], y = r8[4], z = r8[5];
  const double len = std::sqrt(std::fma(x, x, std::fma(y, y, z * z)));
  if (len > 1e-18) {
    const double s = 1.0 / len;
    r.d[0] = x * s;
    r.d[1] = y * s;
    r.d[2] = z * s;
  } else {
    r.d[0] = 0.0;
    r.d[1] = 0.0;
    r.d[2] = 1.0;
  }
  for (int a = 0; a < 3; ++a) r.inv[a] = 1.0 / r.d[a];
  r.t_min = r8[6];
  r.t_end = r8[7];
  return r;
}

// Aabb::intersect (src/math.rs:859-890)
bool intersect(const Medium &m, const Ray &r, double t_min, double t_max, double &t0,
               double &t1) {
  for (int a = 0; a < 3; ++a) {
    const double ta = (m.bmin[a] - r.o[a]) * r.inv[a];
    const double tb = (m.bmax[a] - r.o[a]) * r.inv[a];
    t_min = std::fmax(t_min, std::fmin(ta, tb));
    t_max = std::fmin(t_max, std::fmax(ta, tb));
    if (a < 2 && t_max < t_min) return false;
  }
  if (!(t_max >= t_min)) return false;
  t0 = t_min;
  t1 = t_max;
  return true;
}

// transmittance (src/fluid.rs:840-874)
double transmittance(const Medium &m, const Ray &r, Xoshiro &rng) {
  if (m.max_density <= 1e-6) return 1.0;
  double t_enter, t_exit;
  if (!intersect(m, r, r.t_min, r.t_end, t_enter, t_exit)) return 1.0;
  double t = std::fmax(t_enter, r.t_min);
  const double limit = std::fmin(t_exit, r.t_end);
  if (t >= limit) return 1.0;
  double tr = 1.0;
  const double inv_maj = 1.0 / m.majorant;
  for (int s = 0; s < 256; ++s) {
    const double u = std::fmax(1.0 - rng.next_f64(), 1e-15);
    t -= std::log(u) * inv_maj;
    if (t >= limit) break;
    double p[3], rho, tmp;
    r.at(t, p);
    med_sample(m, p, rho, tmp);
    const double sigma_t = std::fmin(rho * m.sigma_t_scale, m.majorant);
    tr *= 1.0 - sigma_t * inv_maj;
    if (tr < 0.05) {
      const double q = std::fmin(1.0 - tr, 0.95);
      if (rng.next_f64() < q) return 0.0;
      tr /= 1.0 - q;
    }
  }
  return rs_clamp(tr, 0.0, 1.0);
}

// sample_interaction (src/fluid.rs:792-838)
bool interaction(const Medium &m, const Ray &r, Xoshiro &rng, double &t_hit, double &rho_hit,
                 double &tmp_hit) {
  if (m.max_density <= 1e-6) return false;
  double t_enter, t_exit;
  if (!intersect(m, r, r.t_min, r.t_end, t_enter, t_exit)) return false;
  double t = std::fmax(t_enter, r.t_min);
  const double limit = std::fmin(t_exit, r.t_end);
  if (t >= limit) return false;
  const double inv_maj = 1.0 / m.majorant;
  for (int s = 0; s < 256; ++s) {
    const double u = std::fmax(1.0 - rng.next_f64(), 1e-15);
    t -= std::log(u) * inv_maj;
    if (t >= limit) return false;
    double p[3], rho, tmp;
    r.at(t, p);
    med_sample(m, p, rho, tmp);
    const double sigma_t = rho * m.sigma_t_scale;
    if (rng.next_f64() * m.majorant < sigma_t) {
      t_hit = t;
      rho_hit = rho;
      tmp_hit = tmp;
      return true;
    }
  }
  return false;
}

}  // namespace

extern "C" {

void ofl_medium_sample(const double *dens, const double *temp, size_t nx, size_t ny, size_t nz,
                       const double *bmin, const double *bmax, const double *pts, size_t n,
                       double *rho, double *tmp) {
  const Medium m = make_medium(dens, temp, nx, ny, nz, bmin, bmax, 1.0);
  for (size_t c = 0; c < n; ++c) med_sample(m, pts + 3 * c, rho[c], tmp[c]);
}

void ofl_medium_transmittance(const double *dens, const double *temp, size_t nx, size_t ny,
                              size_t nz, const double *bmin, const double *bmax,
                              double sigma_t_scale, const double *rays, size_t n, uint64_t seed,
                              double *tr) {
  const Medium m = make_medium(dens, temp, nx, ny, nz, bmin, bmax, sigma_t_scale);
  for (size_t c = 0; c < n; ++c) {
    Xoshiro rng(seed + static_cast<uint64_t>(c));
    tr[c] = transmittance(m, make_ray(rays + 8 * c), rng);
  }
}

void ofl_medium_interaction(const double *dens, const double *temp, size_t nx, size_t ny,
                            size_t nz, const double *bmin, const double *bmax,
                            double sigma_t_scale, const double *rays, size_t n, uint64_t seed,
                            int32_t *hit, double *t, double *rho, double *tmp) {
  const Medium m = make_medium(dens, temp, nx, ny, nz, bmin, bmax, sigma_t_scale);
  for (size_t c = 0; c < n; ++c) {
    Xoshiro rng(seed + static_cast<uint64_t>(c));
    double th = 0.0, rh = 0.0, qh = 0.0;
    hit[c] = interaction(m, make_ray(rays + 8 * c), rng, th, rh, qh) ? 1 : 0;
    t[c] = th;
    rho[c] = rh;
    tmp[c] = qh;
  }
}
}  // extern "C"
