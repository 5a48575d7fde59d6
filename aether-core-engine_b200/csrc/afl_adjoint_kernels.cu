// afl_adjoint_kernels.cu -- vector-Jacobian products of the FP64 smoke step.
//
// No counterpart in the reference (which has no derivatives).  Each kernel is
// the adjoint of one forward stage of afl_stage.cuh, derived by hand:
//   * MacCormack advection: the recorded branch of every cell (near-wall
//     fallback / unclamped / clamped to the min or max corner of the 8-cell
//     stencil, and max(0) activity for scalars) selects the linear map that
//     the forward applied; trilinear samples scatter their adjoint to the 8
//     corners (atomics) and differentiate their weights with respect to the
//     sample position, i.e. to the velocity that moved it (zero where the
//     position was clamped).
//   * vorticity confinement: f = eps*h*(N x w), N = g/(|g| + 1e-10), g the
//     central gradient of |w|, w the central curl; adjoints of the cross
//     product, the normalisation, the gradient and the curl, in gather form.
//   * projection: u3 = BC(u2 - G p), A p = b = D u2, with the solve taken as
//     exact, so the adjoint is u2_bar = BC-masked u3_bar + D^T A^-1 (-G^T u3_bar);
//     A^-1 is applied with the same symmetric-operator CG as the forward.
// Built with -fmad=false, like the forward FP64 kernels, so the recording
// forward below reproduces the plain forward bit for bit.
#include "afl_stage.cuh"

namespace afl {

// ---- recording forward -----------------------------------------------------
// cell_advect_mc plus a mask byte per cell:
//   bit 0 near-wall fallback, bits 1-2 clamp (0 none, 1 to the min, 2 to the
//   max), bits 3-5 the clamping corner (dk<<2 | dj<<1 | di), bit 6 result > 0.
__global__ void __launch_bounds__(kTx *kTy)
    k_advect_mc_record(Dims g, const double *__restrict__ u, const double *__restrict__ v,
                       const double *__restrict__ w, const double *__restrict__ src,
                       const double *__restrict__ fwd, double *__restrict__ out, double scale_f,
                       double scale_b, double dissipation, int nonneg,
                       unsigned char *__restrict__ mask) {
  int i, j, k;
  if (!cell_of_thread(g, i, j, k)) return;
  const int c = (k * g.ny + j) * g.nx + i;
  double res = 0.0;
  unsigned char mk = 0;
  if (interior(g, i, j, k)) {
    const double uc = u[c], vc = v[c], wc = w[c];
    const double bx = double(i) - scale_f * uc;
    const double by = double(j) - scale_f * vc;
    const double bz = double(k) - scale_f * wc;
    const bool near_wall = bx < 1.5 || bx > double(g.nx) - 2.5 || by < 1.5 ||
                           by > double(g.ny) - 2.5 || bz < 1.5 || bz > double(g.nz) - 2.5;
    const double fc = fwd[c];
    double val;
    if (near_wall) {
      val = fc;
      mk = 1;
    } else {
      const double fx = double(i) - scale_b * uc;
      const double fy = double(j) - scale_b * vc;
      const double fz = double(k) - scale_b * wc;
      const double bwd = trilinear(fwd, g, footprint(g, fx, fy, fz));
      const double mc = fc + 0.5 * (src[c] - bwd);
      // the 8-cell extremes and where they sit (first corner in loop order)
      const int base = footprint(g, bx, by, bz).base;
      double lo = INFINITY, hi = -INFINITY;
      int clo = 0, chi = 0;
      for (int dk = 0; dk <= 1; ++dk)
        for (int dj = 0; dj <= 1; ++dj)
          for (int di = 0; di <= 1; ++di) {
            const double x = src[base + dk * g.nxy + dj * g.nx + di];
            const int corner = (dk << 2) | (dj << 1) | di;
            if (x < lo) { lo = x; clo = corner; }
            if (x > hi) { hi = x; chi = corner; }
          }
      val = mc;
      if (mc < lo) { val = lo; mk = static_cast<unsigned char>(2 | (clo << 3)); }
      if (val > hi) { val = hi; mk = static_cast<unsigned char>(4 | (chi << 3)); }
    }
    res = val * dissipation;
  }
  if (nonneg) res = fmax(res, 0.0);
  if (res > 0.0) mk |= 64;
  out[c] = res;
  mask[c] = mk;
}

// ---- trilinear pieces --------------------------------------------------------
struct TriW {
  int base;
  double tx, ty, tz;
  bool fx, fy, fz;  // position inside the clamp range along each axis
};

__device__ __forceinline__ TriW tri_at(const Dims &g, double x, double y, double z) {
  TriW t;
  const double xhi = double(g.nx) - 1.500001, yhi = double(g.ny) - 1.500001,
               zhi = double(g.nz) - 1.500001;
  t.fx = x > 0.5 && x < xhi;
  t.fy = y > 0.5 && y < yhi;
  t.fz = z > 0.5 && z < zhi;
  const Footprint<double> f = footprint(g, x, y, z);
  t.base = f.base;
  t.tx = f.tx;
  t.ty = f.ty;
  t.tz = f.tz;
  return t;
}

// Adds a * (weight of each corner) to dst at the 8 corners.
__device__ __forceinline__ void tri_scatter(const Dims &g, double *dst, const TriW &t, double a) {
  const double ox = 1.0 - t.tx, oy = 1.0 - t.ty, oz = 1.0 - t.tz;
  const int sy = g.nx, sz = g.nxy, b = t.base;
  atomicAdd(dst + b, a * ox * oy * oz);
  atomicAdd(dst + b + 1, a * t.tx * oy * oz);
  atomicAdd(dst + b + sy, a * ox * t.ty * oz);
  atomicAdd(dst + b + sy + 1, a * t.tx * t.ty * oz);
  atomicAdd(dst + b + sz, a * ox * oy * t.tz);
  atomicAdd(dst + b + sz + 1, a * t.tx * oy * t.tz);
  atomicAdd(dst + b + sz + sy, a * ox * t.ty * t.tz);
  atomicAdd(dst + b + sz + sy + 1, a * t.tx * t.ty * t.tz);
}

// Gradient of the trilinear sample of f with respect to the (unclamped)
// sample position.
__device__ __forceinline__ void tri_grad(const Dims &g, const double *f, const TriW &t,
                                         double &gx, double &gy, double &gz) {
  const int sy = g.nx, sz = g.nxy, b = t.base;
  const double c000 = f[b], c100 = f[b + 1], c010 = f[b + sy], c110 = f[b + sy + 1];
  const double c001 = f[b + sz], c101 = f[b + sz + 1], c011 = f[b + sz + sy],
               c111 = f[b + sz + sy + 1];
  const double ox = 1.0 - t.tx, oy = 1.0 - t.ty, oz = 1.0 - t.tz;
  const double c00 = c000 * ox + c100 * t.tx, c10 = c010 * ox + c110 * t.tx;
  const double c01 = c001 * ox + c101 * t.tx, c11 = c011 * ox + c111 * t.tx;
  gx = oz * (oy * (c100 - c000) + t.ty * (c110 - c010)) +
       t.tz * (oy * (c101 - c001) + t.ty * (c111 - c011));
  gy = oz * (c10 - c00) + t.tz * (c11 - c01);
  gz = (c01 * oy + c11 * t.ty) - (c00 * oy + c10 * t.ty);
  if (!t.fx) gx = 0.0;
  if (!t.fy) gy = 0.0;
  if (!t.fz) gz = 0.0;
}

// ---- MacCormack adjoint ---------------------------------------------------------
// Pass 1 (correction): from the output adjoint `ob` to the adjoints of fwd
// (scattered, `fb`), of src (`sb`) and of the velocity at each cell (`ub`, `vb`,
// `wb`, accumulated).
__global__ void __launch_bounds__(kTx *kTy)
    k_adv_mc_bwd(Dims g, const double *__restrict__ u, const double *__restrict__ v,
                 const double *__restrict__ w, const double *__restrict__ fwd,
                 const unsigned char *__restrict__ mask, double scale_b, double dissipation,
                 int nonneg, const double *__restrict__ ob, double *fb, double *sb, double *ub,
                 double *vb, double *wb) {
  int i, j, k;
  if (!cell_of_thread(g, i, j, k)) return;
  if (!interior(g, i, j, k)) return;
  const int c = (k * g.ny + j) * g.nx + i;
  const unsigned char mk = mask[c];
  if (nonneg && !(mk & 64)) return;
  const double gv = ob[c] * dissipation;
  if (gv == 0.0) return;
  if (mk & 1) {  // near-wall: out = fwd[c]
    atomicAdd(fb + c, gv);
    return;
  }
  const int clamp = (mk >> 1) & 3;
  if (clamp != 0) {  // out = src at the extreme corner
    const int corner = (mk >> 3) & 7;
    const int di = corner & 1, dj = (corner >> 1) & 1, dk = corner >> 2;
    // the corner belongs to the backtrace footprint (scale_f = -scale_b)
    const double sf = -scale_b;
    const Footprint<double> fp =
        footprint(g, double(i) - sf * u[c], double(j) - sf * v[c], double(k) - sf * w[c]);
    atomicAdd(sb + fp.base + dk * g.nxy + dj * g.nx + di, gv);
    return;
  }
  // out = fwd[c] + 0.5*(src[c] - bwd), bwd = trilinear(fwd, c + scale_f*vel)
  atomicAdd(fb + c, gv);
  atomicAdd(sb + c, 0.5 * gv);
  const double bb = -0.5 * gv;
  const double uc = u[c], vc = v[c], wc = w[c];
  const TriW t = tri_at(g, double(i) - scale_b * uc, double(j) - scale_b * vc,
                        double(k) - scale_b * wc);
  tri_scatter(g, fb, t, bb);
  double gx, gy, gz;
  tri_grad(g, fwd, t, gx, gy, gz);
  // position = idx - scale_b*vel; atomics: the velocity adjoint may be the
  // same array as the src adjoint that other cells scatter into
  atomicAdd(ub + c, bb * gx * (-scale_b));
  atomicAdd(vb + c, bb * gy * (-scale_b));
  atomicAdd(wb + c, bb * gz * (-scale_b));
}

// Pass 2 (semi-Lagrangian): fwd = trilinear(src, idx - scale_f*vel) on the
// interior; the adjoint of fwd goes to src (scattered) and to the velocity.
__global__ void __launch_bounds__(kTx *kTy)
    k_adv_sl_bwd(Dims g, const double *__restrict__ u, const double *__restrict__ v,
                 const double *__restrict__ w, const double *__restrict__ src, double scale_f,
                 const double *__restrict__ fb, double *sb, double *ub, double *vb, double *wb) {
  int i, j, k;
  if (!cell_of_thread(g, i, j, k)) return;
  if (!interior(g, i, j, k)) return;
  const int c = (k * g.ny + j) * g.nx + i;
  const double gv = fb[c];
  if (gv == 0.0) return;
  const TriW t = tri_at(g, double(i) - scale_f * u[c], double(j) - scale_f * v[c],
                        double(k) - scale_f * w[c]);
  tri_scatter(g, sb, t, gv);
  double gx, gy, gz;
  tri_grad(g, src, t, gx, gy, gz);
  atomicAdd(ub + c, gv * gx * (-scale_f));
  atomicAdd(vb + c, gv * gy * (-scale_f));
  atomicAdd(wb + c, gv * gz * (-scale_f));
}

// ---- sphere source adjoint ------------------------------------------------------
// rho = rho_val, temp = temp_val*amp inside the sphere: the incoming density and
// temperature have no influence there; the amplitude receives temp_val*temp_bar.
__global__ void __launch_bounds__(kTx *kTy)
    k_source_bwd(Dims g, int i0, int j0, int k0, int ni, int nj, double cx, double cy,
                 double cz, double r2, double temp_val, double *rhob, double *tempb,
                 double *ampb) {
  const int ii = blockIdx.x * kTx + threadIdx.x;
  const int jj = blockIdx.y * kTy + threadIdx.y;
  if (ii >= ni || jj >= nj) return;
  const int i = i0 + ii, j = j0 + jj, k = k0 + blockIdx.z;
  const double dx = double(i) - cx, dy = double(j) - cy, dz = double(k) - cz;
  if (!(dx * dx + dy * dy + dz * dz < r2)) return;
  const int c = (k * g.ny + j) * g.nx + i;
  if (ampb) ampb[c] += temp_val * tempb[c];
  rhob[c] = 0.0;
  tempb[c] = 0.0;
}

// ---- confinement + buoyancy adjoint ------------------------------------------
// Pass A (cells 2..n-3): from f_bar = dt*BC(u2_bar) to N_bar, the direct curl
// adjoint, and the adjoint of g = grad |w|.
__global__ void __launch_bounds__(kTx *kTy)
    k_conf_bwd_a(Dims g, const double *__restrict__ cx, const double *__restrict__ cy,
                 const double *__restrict__ cz, const double *__restrict__ cm,
                 const double *__restrict__ u2b, const double *__restrict__ v2b,
                 const double *__restrict__ w2b, double dt, double eps_h, double inv_2h,
                 double *gbx, double *gby, double *gbz, double *obx, double *oby, double *obz) {
  int i, j, k;
  if (!cell_of_thread(g, i, j, k)) return;
  const int c = (k * g.ny + j) * g.nx + i;
  double gxb = 0.0, gyb = 0.0, gzb = 0.0, oxb = 0.0, oyb = 0.0, ozb = 0.0;
  if (i >= 2 && i <= g.nx - 3 && j >= 2 && j <= g.ny - 3 && k >= 2 && k <= g.nz - 3) {
    const double fx = wall_u(g, i, j, k) ? 0.0 : dt * u2b[c];
    const double fy = wall_v(g, i, j, k) ? 0.0 : dt * v2b[c];
    const double fz = wall_w(g, i, j, k) ? 0.0 : dt * w2b[c];
    const int sy = g.nx, sz = g.nxy;
    const double gx = (cm[c + 1] - cm[c - 1]) * inv_2h;
    const double gy = (cm[c + sy] - cm[c - sy]) * inv_2h;
    const double gz = (cm[c + sz] - cm[c - sz]) * inv_2h;
    const double gn = sqrt(gx * gx + gy * gy + gz * gz);
    const double glen = gn + 1e-10;
    const double nx = gx / glen, ny = gy / glen, nz = gz / glen;
    const double ox = cx[c], oy = cy[c], oz = cz[c];
    // f = eps_h * (N x w):  N_bar = eps_h * (w x f_bar), w_bar = eps_h * (f_bar x N)
    const double nbx = eps_h * (oy * fz - oz * fy);
    const double nby = eps_h * (oz * fx - ox * fz);
    const double nbz = eps_h * (ox * fy - oy * fx);
    oxb = eps_h * (fy * nz - fz * ny);
    oyb = eps_h * (fz * nx - fx * nz);
    ozb = eps_h * (fx * ny - fy * nx);
    // N = g / (|g| + 1e-10)
    const double gdot = gx * nbx + gy * nby + gz * nbz;
    const double corr = gn > 0.0 ? gdot / (gn * glen * glen) : 0.0;
    gxb = nbx / glen - gx * corr;
    gyb = nby / glen - gy * corr;
    gzb = nbz / glen - gz * corr;
  }
  gbx[c] = gxb;
  gby[c] = gyb;
  gbz[c] = gzb;
  obx[c] = oxb;
  oby[c] = oyb;
  obz[c] = ozb;
}

// Pass B (interior cells): |w|_bar from the gradient adjoint (gather), added to
// the curl adjoint through |w| = sqrt(w.w).
__global__ void __launch_bounds__(kTx *kTy)
    k_conf_bwd_b(Dims g, const double *__restrict__ cx, const double *__restrict__ cy,
                 const double *__restrict__ cz, const double *__restrict__ cm,
                 const double *__restrict__ gbx, const double *__restrict__ gby,
                 const double *__restrict__ gbz, double inv_2h, double *obx, double *oby,
                 double *obz) {
  int i, j, k;
  if (!cell_of_thread(g, i, j, k)) return;
  if (!interior(g, i, j, k)) return;
  const int c = (k * g.ny + j) * g.nx + i;
  const int sy = g.nx, sz = g.nxy;
  // g_a(c') = (m(c'+e_a) - m(c'-e_a)) * inv_2h  =>  m_bar(c) = inv_2h * (g_bar_a(c-e_a) - g_bar_a(c+e_a))
  const double mb = inv_2h * ((gbx[c - 1] - gbx[c + 1]) + (gby[c - sy] - gby[c + sy]) +
                              (gbz[c - sz] - gbz[c + sz]));
  const double m = cm[c];
  if (m > 0.0 && mb != 0.0) {
    obx[c] += mb * cx[c] / m;
    oby[c] += mb * cy[c] / m;
    obz[c] += mb * cz[c] / m;
  }
}

// Pass C (every cell): velocity adjoint before confinement/buoyancy:
// identity (through the wall-BC mask) plus the curl adjoint in gather form;
// buoyancy sends dt*beta*v_bar to temperature and -dt*alpha*v_bar to density.
__global__ void __launch_bounds__(kTx *kTy)
    k_conf_bwd_c(Dims g, const double *__restrict__ u2b, const double *__restrict__ v2b,
                 const double *__restrict__ w2b, const double *__restrict__ obx,
                 const double *__restrict__ oby, const double *__restrict__ obz, double inv_2h,
                 double dt, double beta, double alpha, double *u1b, double *v1b, double *w1b,
                 double *rhob, double *tempb) {
  int i, j, k;
  if (!cell_of_thread(g, i, j, k)) return;
  const int c = (k * g.ny + j) * g.nx + i;
  const int sy = g.nx, sz = g.nxy;
  const double um = wall_u(g, i, j, k) ? 0.0 : u2b[c];
  const double vm = wall_v(g, i, j, k) ? 0.0 : v2b[c];
  const double wm = wall_w(g, i, j, k) ? 0.0 : w2b[c];
  // curl adjoint: a neighbour outside the grid contributes nothing (w_bar = 0 off the interior)
  auto at = [&](const double *a, int di, int dj, int dk) {
    const int ii = i + di, jj = j + dj, kk = k + dk;
    if (ii < 0 || ii >= g.nx || jj < 0 || jj >= g.ny || kk < 0 || kk >= g.nz) return 0.0;
    return a[c + di + dj * sy + dk * sz];
  };
  const double cu = inv_2h * ((at(oby, 0, 0, -1) - at(oby, 0, 0, 1)) -
                              (at(obz, 0, -1, 0) - at(obz, 0, 1, 0)));
  const double cv = inv_2h * ((at(obz, -1, 0, 0) - at(obz, 1, 0, 0)) -
                              (at(obx, 0, 0, -1) - at(obx, 0, 0, 1)));
  const double cw = inv_2h * ((at(obx, 0, -1, 0) - at(obx, 0, 1, 0)) -
                              (at(oby, -1, 0, 0) - at(oby, 1, 0, 0)));
  u1b[c] += um + cu;
  v1b[c] += vm + cv;
  w1b[c] += wm + cw;
  if (interior(g, i, j, k)) {
    tempb[c] += dt * beta * vm;
    rhob[c] -= dt * alpha * vm;
  }
}

// ---- projection adjoint -----------------------------------------------------------
// u3 = BC(u2 - G p): u3_bar is masked in place (then p_bar = -G^T u3_bar).
__global__ void __launch_bounds__(kTx *kTy)
    k_proj_bwd_a(Dims g, double *u3b, double *v3b, double *w3b) {
  int i, j, k;
  if (!cell_of_thread(g, i, j, k)) return;
  const int c = (k * g.ny + j) * g.nx + i;
  if (wall_u(g, i, j, k)) u3b[c] = 0.0;
  if (wall_v(g, i, j, k)) v3b[c] = 0.0;
  if (wall_w(g, i, j, k)) w3b[c] = 0.0;
}

__global__ void __launch_bounds__(kTx *kTy)
    k_proj_bwd_p(Dims g, const double *__restrict__ u3b, const double *__restrict__ v3b,
                 const double *__restrict__ w3b, double inv_h, double *pb) {
  int i, j, k;
  if (!cell_of_thread(g, i, j, k)) return;
  const int c = (k * g.ny + j) * g.nx + i;
  double acc = 0.0;
  if (interior(g, i, j, k)) {
    // (G p)_a(c) = (p(c) - p(c - e_a)) * inv_h for interior c with index_a > 1,
    // so -G^T u_bar at c = inv_h * (-u_bar_a(c) + u_bar_a(c + e_a)).
    if (i > 1) acc -= u3b[c];
    if (j > 1) acc -= v3b[c];
    if (k > 1) acc -= w3b[c];
    if (interior(g, i + 1, j, k)) acc += u3b[c + 1];
    if (interior(g, i, j + 1, k)) acc += v3b[c + g.nx];
    if (interior(g, i, j, k + 1)) acc += w3b[c + g.nxy];
  }
  pb[c] = acc * inv_h;
}

// u2_bar = u3_bar + D^T b_bar, b = -h*(u(c+x)-u(c) + ...) on the interior, then
// the mask of project's leading wall BC.
__global__ void __launch_bounds__(kTx *kTy)
    k_proj_bwd_b(Dims g, const double *__restrict__ u3b, const double *__restrict__ v3b,
                 const double *__restrict__ w3b, const double *__restrict__ bb, double h,
                 double *u2b, double *v2b, double *w2b) {
  int i, j, k;
  if (!cell_of_thread(g, i, j, k)) return;
  const int c = (k * g.ny + j) * g.nx + i;
  const double own = interior(g, i, j, k) ? bb[c] : 0.0;
  const double xm = (i >= 1 && interior(g, i - 1, j, k)) ? bb[c - 1] : 0.0;
  const double ym = (j >= 1 && interior(g, i, j - 1, k)) ? bb[c - g.nx] : 0.0;
  const double zm = (k >= 1 && interior(g, i, j, k - 1)) ? bb[c - g.nxy] : 0.0;
  const double ua = u3b[c] + (-h) * (xm - own);
  const double va = v3b[c] + (-h) * (ym - own);
  const double wa = w3b[c] + (-h) * (zm - own);
  u2b[c] = wall_u(g, i, j, k) ? 0.0 : ua;
  v2b[c] = wall_v(g, i, j, k) ? 0.0 : va;
  w2b[c] = wall_w(g, i, j, k) ? 0.0 : wa;
}

// ---- cyberpunk jets adjoint (inject_cyberpunk_sources, src/fluid.rs:573-593) --------
// Forward of one jet, k_inject_jet's arithmetic, recording in `mask` the cells
// whose density (bit 2*jet) or temperature (bit 2*jet+1) reached its cap:
// min(x, 3.8) and min(x, 4.5) pass x through below the cap and a constant at
// or above it.  The velocity increments do not depend on the state.
__global__ void __launch_bounds__(kTx *kTy)
    k_jet_record(Dims g, int jet, int i0, int j0, int k0, int ni, int nj, double *rho,
                 double *temp, double *u, double *v, double *w, double jx, double jy, double jz,
                 double vx, double vy, double vz, double r2, double dt, double pulse,
                 unsigned char *mask) {
  const int ii = blockIdx.x * kTx + threadIdx.x;
  const int jj = blockIdx.y * kTy + threadIdx.y;
  if (ii >= ni || jj >= nj) return;
  const int i = i0 + ii, j = j0 + jj, k = k0 + blockIdx.z;
  const double dx = double(i) - jx;
  const double dy = double(j) - jy;
  const double dz = double(k) - jz;
  const double d2 = dx * dx + dy * dy + dz * dz;
  if (!(d2 < r2)) return;
  const double wf = exp(-2.2 * d2 / r2);
  const int c = (k * g.ny + j) * g.nx + i;
  const double rn = rho[c] + dt * 9.5 * pulse * wf;
  const double tn = temp[c] + dt * 8.2 * pulse * wf;
  unsigned char m = mask[c];
  if (!(rn < 3.8)) m |= static_cast<unsigned char>(1u << (2 * jet));
  if (!(tn < 4.5)) m |= static_cast<unsigned char>(2u << (2 * jet));
  mask[c] = m;
  rho[c] = fmin(rn, 3.8);
  temp[c] = fmin(tn, 4.5);
  u[c] = u[c] + dt * vx * wf * 4.2;
  v[c] = v[c] + dt * vy * wf * 4.2;
  w[c] = w[c] + dt * vz * wf * 4.2;
}

// The jets' adjoint: the density/temperature adjoints pass through where no cap
// was reached (either jet), vanish where one was; velocity adjoints pass
// through unchanged.
__global__ void __launch_bounds__(kBlock)
    k_jet_bwd(int n, const unsigned char *__restrict__ mask, double *rhob, double *tempb) {
  for (int c = blockIdx.x * kBlock + threadIdx.x; c < n; c += gridDim.x * kBlock) {
    const unsigned m = mask[c];
    if (m & 0x5u) rhob[c] = 0.0;
    if (m & 0xAu) tempb[c] = 0.0;
  }
}

// ---- red-black SOR adjoint (solve_poisson_gauss_seidel, src/fluid.rs:397-442) --------
// A half-sweep of colour c sets, on the interior cells i of that colour,
// p_i <- (1 - w) p_i + w (b_i + sum of p over i's interior neighbours) / diag_i,
// a linear map of (p, b).  Its transpose: pass A lets every interior cell x of
// the other colour gather w pb_j / diag_j from its interior neighbours j (all
// of colour c; x is among j's neighbours exactly when both are interior), and
// colour-c cells add w pb_i / diag_i to bb_i; pass B scales pb_i by (1 - w) on
// colour c.  Pass A reads colour-c values only and pass B writes them only.
__device__ __forceinline__ double sor_diag(const Dims &g, int i, int j, int k) {
  return double(int(i > 1) + int(i + 2 < g.nx) + int(j > 1) + int(j + 2 < g.ny) + int(k > 1) +
                int(k + 2 < g.nz));
}

__global__ void __launch_bounds__(kTx *kTy)
    k_sor_bwd_a(Dims g, int color, double omega, double *pb, double *bb) {
  int i, j, k;
  if (!cell_of_thread(g, i, j, k)) return;
  if (!interior(g, i, j, k)) return;
  const int c = (k * g.ny + j) * g.nx + i;
  if (((i + j + k) & 1) == color) {
    bb[c] += omega * pb[c] / sor_diag(g, i, j, k);
    return;
  }
  double acc = 0.0;
  if (interior(g, i - 1, j, k)) acc += omega * pb[c - 1] / sor_diag(g, i - 1, j, k);
  if (interior(g, i + 1, j, k)) acc += omega * pb[c + 1] / sor_diag(g, i + 1, j, k);
  if (interior(g, i, j - 1, k)) acc += omega * pb[c - g.nx] / sor_diag(g, i, j - 1, k);
  if (interior(g, i, j + 1, k)) acc += omega * pb[c + g.nx] / sor_diag(g, i, j + 1, k);
  if (interior(g, i, j, k - 1)) acc += omega * pb[c - g.nxy] / sor_diag(g, i, j, k - 1);
  if (interior(g, i, j, k + 1)) acc += omega * pb[c + g.nxy] / sor_diag(g, i, j, k + 1);
  pb[c] += acc;
}

__global__ void __launch_bounds__(kTx *kTy)
    k_sor_bwd_b(Dims g, int color, double omega, double *pb) {
  int i, j, k;
  if (!cell_of_thread(g, i, j, k)) return;
  if (!interior(g, i, j, k) || ((i + j + k) & 1) != color) return;
  const int c = (k * g.ny + j) * g.nx + i;
  pb[c] = (1.0 - omega) * pb[c];
}

__global__ void __launch_bounds__(kBlock) k_add(int n, const double *__restrict__ x, double *y) {
  for (int c = blockIdx.x * kBlock + threadIdx.x; c < n; c += gridDim.x * kBlock) y[c] += x[c];
}

// ---- launchers -----------------------------------------------------------------
void adj_advect_mc_record(const Dims &g, const double *u, const double *v, const double *w,
                          const double *src, const double *fwd, double *out, double dt,
                          double diss, bool nonneg, unsigned char *mask, cudaStream_t st) {
  const double sf = dt / g.h, sb = (-dt) / g.h;
  k_advect_mc_record<<<plane_grid(g), dim3(kTx, kTy), 0, st>>>(g, u, v, w, src, fwd, out, sf, sb,
                                                               diss, nonneg ? 1 : 0, mask);
}

void adj_advect_bwd(const Dims &g, const double *u, const double *v, const double *w,
                    const double *src, const double *fwd, const unsigned char *mask, double dt,
                    double diss, bool nonneg, const double *ob, double *fb, double *sb,
                    double *ub, double *vb, double *wb, cudaStream_t st) {
  const double sf = dt / g.h, sbk = (-dt) / g.h;
  cudaMemsetAsync(fb, 0, sizeof(double) * static_cast<size_t>(g.n), st);
  k_adv_mc_bwd<<<plane_grid(g), dim3(kTx, kTy), 0, st>>>(g, u, v, w, fwd, mask, sbk, diss,
                                                         nonneg ? 1 : 0, ob, fb, sb, ub, vb, wb);
  k_adv_sl_bwd<<<plane_grid(g), dim3(kTx, kTy), 0, st>>>(g, u, v, w, src, sf, fb, sb, ub, vb, wb);
}

void adj_source_bwd(const Dims &g, const int lo[3], const int hi[3], const double c[3], double r2,
                    double temp_val, double *rhob, double *tempb, double *ampb, cudaStream_t st) {
  const int ni = hi[0] - lo[0] + 1, nj = hi[1] - lo[1] + 1, nk = hi[2] - lo[2] + 1;
  if (ni <= 0 || nj <= 0 || nk <= 0) return;
  dim3 grid((ni + kTx - 1) / kTx, (nj + kTy - 1) / kTy, nk);
  k_source_bwd<<<grid, dim3(kTx, kTy), 0, st>>>(g, lo[0], lo[1], lo[2], ni, nj, c[0], c[1], c[2],
                                               r2, temp_val, rhob, tempb, ampb);
}

void adj_confine_bwd(const Dims &g, const double *cx, const double *cy, const double *cz,
                     const double *cm, const double *u2b, const double *v2b, const double *w2b,
                     double dt, double eps, double beta, double alpha, double *gb[3],
                     double *ob[3], double *u1b, double *v1b, double *w1b, double *rhob,
                     double *tempb, cudaStream_t st) {
  const double inv_2h = 0.5 / g.h, eps_h = eps * g.h;
  k_conf_bwd_a<<<plane_grid(g), dim3(kTx, kTy), 0, st>>>(g, cx, cy, cz, cm, u2b, v2b, w2b, dt,
                                                         eps_h, inv_2h, gb[0], gb[1], gb[2], ob[0],
                                                         ob[1], ob[2]);
  k_conf_bwd_b<<<plane_grid(g), dim3(kTx, kTy), 0, st>>>(g, cx, cy, cz, cm, gb[0], gb[1], gb[2],
                                                         inv_2h, ob[0], ob[1], ob[2]);
  k_conf_bwd_c<<<plane_grid(g), dim3(kTx, kTy), 0, st>>>(g, u2b, v2b, w2b, ob[0], ob[1], ob[2],
                                                         inv_2h, dt, beta, alpha, u1b, v1b, w1b,
                                                         rhob, tempb);
}

void adj_project_bwd_p(const Dims &g, double *u3b, double *v3b, double *w3b, double *pb,
                       cudaStream_t st) {
  const double inv_h = 1.0 / g.h;
  k_proj_bwd_a<<<plane_grid(g), dim3(kTx, kTy), 0, st>>>(g, u3b, v3b, w3b);
  k_proj_bwd_p<<<plane_grid(g), dim3(kTx, kTy), 0, st>>>(g, u3b, v3b, w3b, inv_h, pb);
}

void adj_project_bwd_b(const Dims &g, const double *u3b, const double *v3b, const double *w3b,
                       const double *bb, double *u2b, double *v2b, double *w2b, cudaStream_t st) {
  k_proj_bwd_b<<<plane_grid(g), dim3(kTx, kTy), 0, st>>>(g, u3b, v3b, w3b, bb, g.h, u2b, v2b, w2b);
}

void adj_jet_record(const Dims &g, double time_sec, double dt, double *rho, double *temp,
                    double *u, double *v, double *w, unsigned char *mask, cudaStream_t st) {
  const JetPair jp = cyberpunk_jets(g, time_sec);
  for (int q = 0; q < 2; ++q) {
    const int ni = jp.hi[q][0] - jp.lo[q][0] + 1, nj = jp.hi[q][1] - jp.lo[q][1] + 1,
              nk = jp.hi[q][2] - jp.lo[q][2] + 1;
    if (ni <= 0 || nj <= 0 || nk <= 0) continue;
    dim3 grid((ni + kTx - 1) / kTx, (nj + kTy - 1) / kTy, nk);
    const double *J = jp.jet[q];
    k_jet_record<<<grid, dim3(kTx, kTy), 0, st>>>(g, q, jp.lo[q][0], jp.lo[q][1], jp.lo[q][2], ni,
                                                  nj, rho, temp, u, v, w, J[0], J[1], J[2], J[3],
                                                  J[4], J[5], jp.r2, dt, jp.pulse, mask);
  }
}

void adj_jet_bwd(const Dims &g, const unsigned char *mask, double *rhob, double *tempb,
                 cudaStream_t st) {
  k_jet_bwd<<<kReduceBlocks, kBlock, 0, st>>>(g.n, mask, rhob, tempb);
}

// y += x over the grid.
void adj_add(const Dims &g, const double *x, double *y, cudaStream_t st) {
  k_add<<<kReduceBlocks, kBlock, 0, st>>>(g.n, x, y);
}

// (pb, bb) <- the transpose of `sweeps` red-black sweeps applied to pb: on
// exit pb is the adjoint of the warm start and bb (zeroed here) that of the
// right-hand side.
void adj_sor_bwd(const Dims &g, int sweeps, double omega, double *pb, double *bb,
                 cudaStream_t st) {
  cudaMemsetAsync(bb, 0, sizeof(double) * static_cast<size_t>(g.n), st);
  for (int s = sweeps - 1; s >= 0; --s)
    for (int color = 1; color >= 0; --color) {
      k_sor_bwd_a<<<plane_grid(g), dim3(kTx, kTy), 0, st>>>(g, color, omega, pb, bb);
      k_sor_bwd_b<<<plane_grid(g), dim3(kTx, kTy), 0, st>>>(g, color, omega, pb);
    }
}

}  // namespace afl
