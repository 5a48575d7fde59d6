// afl_medium.cu -- FluidMedium's volume queries (src/fluid.rs:687-874) on the
// device: the renderer's per-ray medium calls (src/renderer.rs:236, 258, 306)
// as batched kernels over an f64 snapshot of the solver's density and
// temperature.
//
// One thread per ray (or point).  Each ray owns an Xoshiro256++ stream seeded
// Rng::from_seed(seed + ray index), consumed in the reference's order, so a
// ray's result depends only on its own inputs.  Built with -fmad=false: every
// product and sum rounds as in the reference's un-fused f64 expressions; the
// free-flight step calls the device `log`, which may differ from the host's
// libm in the last bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>

#include "../../include/aether_fluid.h"
#include "afl_launch.h"

namespace afl {
namespace {

constexpr int kMT = 128;            // threads per CTA
constexpr int kMaxSteps = 256;      // tracking steps per ray (src/fluid.rs:815, 859)

struct MediumDev {
  Dims g;
  const double *dens;
  const double *temp;
  double bmin[3], bmax[3];
  double sigma_t_scale;
  double majorant;
  double max_density;
};

struct V3 {
  double x, y, z;
};

// sample_density_and_temp (src/fluid.rs:739-786): zero outside the bounds; a
// feathered trilinear sample inside.
__device__ __forceinline__ void sample_dt(const MediumDev &m, V3 p, double &rho, double &tmp) {
  if (p.x < m.bmin[0] || p.x > m.bmax[0] || p.y < m.bmin[1] || p.y > m.bmax[1] ||
      p.z < m.bmin[2] || p.z > m.bmax[2]) {
    rho = 0.0;
    tmp = 0.0;
    return;
  }
  // Aabb::extent (src/math.rs:832-834): (max - min).max_elem(0)
  const double ex = fmax(m.bmax[0] - m.bmin[0], 0.0);
  const double ey = fmax(m.bmax[1] - m.bmin[1], 0.0);
  const double ez = fmax(m.bmax[2] - m.bmin[2], 0.0);
  const double ux = (p.x - m.bmin[0]) / fmax(ex, 1e-9);
  const double uy = (p.y - m.bmin[1]) / fmax(ey, 1e-9);
  const double uz = (p.z - m.bmin[2]) / fmax(ez, 1e-9);
  const double fx = rs_clamp(4.0 * ux * (1.0 - ux), 0.0, 1.0);
  const double fz = rs_clamp(4.0 * uz * (1.0 - uz), 0.0, 1.0);
  const double fy = rs_clamp(1.0 - (fmax(uy - 0.95, 0.0) / 0.05), 0.0, 1.0);
  const double feather = sqrt(fx * fz * fy);
  const double gx = rs_clamp(ux * double(m.g.nx - 1), 0.5, double(m.g.nx) - 1.500001);
  const double gy = rs_clamp(uy * double(m.g.ny - 1), 0.5, double(m.g.ny) - 1.500001);
  const double gz = rs_clamp(uz * double(m.g.nz - 1), 0.5, double(m.g.nz) - 1.500001);
  const int i0 = afl::floor_index(gx);
  const int j0 = afl::floor_index(gy);
  const int k0 = afl::floor_index(gz);
  const double tx = gx - double(i0), ty = gy - double(j0), tz = gz - double(k0);
  const int b = (k0 * m.g.ny + j0) * m.g.nx + i0, sy = m.g.nx, sz = m.g.nxy;
  auto trilin = [&](const double *f) {
    const double c000 = f[b], c100 = f[b + 1], c010 = f[b + sy], c110 = f[b + sy + 1];
    const double c001 = f[b + sz], c101 = f[b + sz + 1], c011 = f[b + sz + sy],
                 c111 = f[b + sz + sy + 1];
    const double c00 = c000 * (1.0 - tx) + c100 * tx;
    const double c10 = c010 * (1.0 - tx) + c110 * tx;
    const double c01 = c001 * (1.0 - tx) + c101 * tx;
    const double c11 = c011 * (1.0 - tx) + c111 * tx;
    return (c00 * (1.0 - ty) + c10 * ty) * (1.0 - tz) + (c01 * (1.0 - ty) + c11 * ty) * tz;
  };
  rho = trilin(m.dens) * feather;
  tmp = trilin(m.temp) * feather;
}

// Ray::new (src/math.rs:763-774): the direction normalised (Vec3::normalize,
// src/math.rs:58-65) and its componentwise inverse.
struct RayDev {
  V3 o, d, inv;
  double t_min, t_end;
};

__device__ __forceinline__ RayDev make_ray(const afl_ray &r) {
  RayDev out;
  out.o = {r.origin[0], r.origin[1], r.origin[2]};
  const double x = r.dir[0], y = r.dir[1], z = r.dir[2];
  // Vec3::length = dot(self, self).sqrt(), dot written with mul_add
  // (src/math.rs:34-36): fma(x, x, fma(y, y, z * z))
  const double len = sqrt(fma(x, x, fma(y, y, z * z)));
  if (len > 1e-18) {
    const double s = 1.0 / len;
    out.d = {x * s, y * s, z * s};
  } else {
    out.d = {0.0, 0.0, 1.0};
  }
  out.inv = {1.0 / out.d.x, 1.0 / out.d.y, 1.0 / out.d.z};
  out.t_min = r.t_min;
  out.t_end = r.t_end;
  return out;
}

__device__ __forceinline__ V3 ray_at(const RayDev &r, double t) {
  return {r.o.x + r.d.x * t, r.o.y + r.d.y * t, r.o.z + r.d.z * t};
}

// Aabb::intersect (src/math.rs:859-890), slab by slab.
__device__ __forceinline__ bool slab(const MediumDev &m, const RayDev &r, double t_min,
                                     double t_max, double &t_enter, double &t_exit) {
  const double o[3] = {r.o.x, r.o.y, r.o.z}, inv[3] = {r.inv.x, r.inv.y, r.inv.z};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double t0 = (m.bmin[a] - o[a]) * inv[a];
    const double t1 = (m.bmax[a] - o[a]) * inv[a];
    t_min = fmax(t_min, fmin(t0, t1));
    t_max = fmin(t_max, fmax(t0, t1));
    if (a < 2 && t_max < t_min) return false;
  }
  if (!(t_max >= t_min)) return false;
  t_enter = t_min;
  t_exit = t_max;
  return true;
}

__global__ void __launch_bounds__(kMT) k_medium_sample(MediumDev m, const double *__restrict__ pts,
                                                       int n, double *__restrict__ rho,
                                                       double *__restrict__ tmp) {
  const int t = blockIdx.x * kMT + threadIdx.x;
  if (t >= n) return;
  double r, q;
  sample_dt(m, {pts[3 * t], pts[3 * t + 1], pts[3 * t + 2]}, r, q);
  rho[t] = r;
  tmp[t] = q;
}

// transmittance (src/fluid.rs:840-874): ratio tracking with Russian roulette
// below 0.05.
__global__ void __launch_bounds__(kMT)
    k_medium_transmittance(MediumDev m, const afl_ray *__restrict__ rays, int n,
                           unsigned long long seed, double *__restrict__ out) {
  const int id = blockIdx.x * kMT + threadIdx.x;
  if (id >= n) return;
  double result = 1.0;
  if (m.max_density > 1e-6) {
    const RayDev r = make_ray(rays[id]);
    double t_enter, t_exit;
    if (slab(m, r, r.t_min, r.t_end, t_enter, t_exit)) {
      double t = fmax(t_enter, r.t_min);
      const double limit = fmin(t_exit, r.t_end);
      if (t < limit) {
        XoshiroRng rng(seed + static_cast<unsigned long long>(id));
        double tr = 1.0;
        const double inv_maj = 1.0 / m.majorant;
        bool zero = false;
        for (int s = 0; s < kMaxSteps; ++s) {
          const double u = fmax(1.0 - rng.next_f64(), 1e-15);
          t -= log(u) * inv_maj;
          if (t >= limit) break;
          double rho, tmp;
          sample_dt(m, ray_at(r, t), rho, tmp);
          const double sigma_t = fmin(rho * m.sigma_t_scale, m.majorant);
          tr *= 1.0 - sigma_t * inv_maj;
          if (tr < 0.05) {
            const double q = fmin(1.0 - tr, 0.95);
            if (rng.next_f64() < q) {
              zero = true;
              break;
            }
            tr /= 1.0 - q;
          }
        }
        result = zero ? 0.0 : rs_clamp(tr, 0.0, 1.0);
      }
    }
  }
  out[id] = result;
}

// sample_interaction (src/fluid.rs:792-838): Woodcock delta tracking.
__global__ void __launch_bounds__(kMT)
    k_medium_interaction(MediumDev m, const afl_ray *__restrict__ rays, int n,
                         unsigned long long seed, int32_t *__restrict__ hit,
                         double *__restrict__ out_t, double *__restrict__ out_rho,
                         double *__restrict__ out_tmp) {
  const int id = blockIdx.x * kMT + threadIdx.x;
  if (id >= n) return;
  int h = 0;
  double ht = 0.0, hr = 0.0, hq = 0.0;
  if (m.max_density > 1e-6) {
    const RayDev r = make_ray(rays[id]);
    double t_enter, t_exit;
    if (slab(m, r, r.t_min, r.t_end, t_enter, t_exit)) {
      double t = fmax(t_enter, r.t_min);
      const double limit = fmin(t_exit, r.t_end);
      if (t < limit) {
        XoshiroRng rng(seed + static_cast<unsigned long long>(id));
        const double inv_maj = 1.0 / m.majorant;
        for (int s = 0; s < kMaxSteps; ++s) {
          const double u = fmax(1.0 - rng.next_f64(), 1e-15);
          t -= log(u) * inv_maj;
          if (t >= limit) break;
          double rho, tmp;
          sample_dt(m, ray_at(r, t), rho, tmp);
          const double sigma_t = rho * m.sigma_t_scale;
          if (rng.next_f64() * m.majorant < sigma_t) {
            h = 1;
            ht = t;
            hr = rho;
            hq = tmp;
            break;
          }
        }
      }
    }
  }
  hit[id] = h;
  out_t[id] = ht;
  out_rho[id] = hr;
  out_tmp[id] = hq;
}

}  // namespace
}  // namespace afl

struct afl_medium {
  int device = 0;
  cudaStream_t stream = nullptr;
  afl::MediumDev dev{};
  double phase_g = 0.0;
  double *fields = nullptr;  // density, then temperature (n doubles each)
  void *in = nullptr, *out = nullptr;
  size_t in_cap = 0, out_cap = 0;
};

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

#define MED_CUDA(call)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)

struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceScope() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

constexpr size_t kMaxBatch = static_cast<size_t>(1) << 26;

afl_status grow(void **buf, size_t *cap, size_t bytes) {
  if (bytes <= *cap) return AFL_OK;
  if (*buf) cudaFree(*buf);
  *buf = nullptr;
  *cap = 0;
  MED_CUDA(cudaMalloc(buf, bytes));
  *cap = bytes;
  return AFL_OK;
}

afl_status finish(afl_medium *m) {
  MED_CUDA(cudaGetLastError());
  MED_CUDA(cudaStreamSynchronize(m->stream));
  return AFL_OK;
}

}  // namespace

extern "C" {

afl_status afl_medium_create(afl_solver *s, const double bounds_min[3],
                             const double bounds_max[3], double sigma_t_scale, double phase_g,
                             afl_medium **out) {
  if (!s || !bounds_min || !bounds_max || !out)
    return fail(AFL_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (!std::isfinite(sigma_t_scale) || !std::isfinite(phase_g))
    return fail(AFL_ERR_INVALID_ARGUMENT, "sigma_t_scale and phase_g must be finite");
  afl::SolverView v{};
  if (!afl::solver_view(s, &v)) return fail(AFL_ERR_INVALID_ARGUMENT, "bad solver handle");
  double max_density = 0.0;
  afl_status st = afl_max_density(s, &max_density);  // FluidMedium::from_solver's max loop
  if (st != AFL_OK) return st;
  DeviceScope scope(v.device);
  afl_medium *m = new afl_medium();
  m->device = v.device;
  auto bail = [&](afl_status code) {
    afl_medium_destroy(m);
    return code;
  };
  if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(AFL_ERR_CUDA, "cudaStreamCreate failed"));
  const size_t n = static_cast<size_t>(v.g.n);
  if (cudaMalloc(&m->fields, 2 * n * sizeof(double)) != cudaSuccess)
    return bail(fail(AFL_ERR_OUT_OF_MEMORY, "medium field copies"));
  // the copies follow the solver's stream, then the medium's
  if (v.f64) {
    cudaMemcpyAsync(m->fields, v.density, n * sizeof(double), cudaMemcpyDeviceToDevice, v.stream);
    cudaMemcpyAsync(m->fields + n, v.temperature, n * sizeof(double), cudaMemcpyDeviceToDevice,
                    v.stream);
  } else {
    afl::launch_convert_f32_to_f64(static_cast<const float *>(v.density), m->fields, v.g.n,
                                   v.stream);
    afl::launch_convert_f32_to_f64(static_cast<const float *>(v.temperature), m->fields + n,
                                   v.g.n, v.stream);
  }
  if (cudaStreamSynchronize(v.stream) != cudaSuccess || cudaGetLastError() != cudaSuccess)
    return bail(fail(AFL_ERR_CUDA, "copying the solver fields"));
  afl::MediumDev &d = m->dev;
  d.g = v.g;
  d.dens = m->fields;
  d.temp = m->fields + n;
  for (int a = 0; a < 3; ++a) {  // Aabb::new (src/math.rs:794-799)
    d.bmin[a] = std::fmin(bounds_min[a], bounds_max[a]);
    d.bmax[a] = std::fmax(bounds_min[a], bounds_max[a]);
  }
  d.sigma_t_scale = sigma_t_scale;
  d.max_density = max_density;
  d.majorant = std::fmax(max_density * sigma_t_scale, 1e-4);  // src/fluid.rs:708
  m->phase_g = phase_g < -0.9 ? -0.9 : (phase_g > 0.9 ? 0.9 : phase_g);
  *out = m;
  return AFL_OK;
}

afl_status afl_medium_destroy(afl_medium *m) {
  if (!m) return AFL_OK;
  DeviceScope scope(m->device);
  if (m->stream) cudaStreamSynchronize(m->stream);
  cudaFree(m->fields);
  cudaFree(m->in);
  cudaFree(m->out);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return AFL_OK;
}

afl_status afl_medium_info(const afl_medium *m, double out[4]) {
  if (!m || !out) return fail(AFL_ERR_INVALID_ARGUMENT, "null argument");
  out[0] = m->dev.max_density;
  out[1] = m->dev.majorant;
  out[2] = m->phase_g;
  out[3] = m->dev.sigma_t_scale;
  return AFL_OK;
}

afl_status afl_medium_sample_density_temp(afl_medium *m, const double *points, size_t n,
                                          double *density, double *temperature) {
  if (!m) return fail(AFL_ERR_INVALID_ARGUMENT, "null medium");
  if (n == 0) return AFL_OK;
  if (!points || !density || !temperature) return fail(AFL_ERR_INVALID_ARGUMENT, "null buffer");
  if (n > kMaxBatch) return fail(AFL_ERR_INVALID_ARGUMENT, "batch larger than 2^26");
  DeviceScope scope(m->device);
  afl_status st = grow(&m->in, &m->in_cap, 3 * n * sizeof(double));
  if (st == AFL_OK) st = grow(&m->out, &m->out_cap, 2 * n * sizeof(double));
  if (st != AFL_OK) return st;
  double *in = static_cast<double *>(m->in), *o = static_cast<double *>(m->out);
  MED_CUDA(cudaMemcpyAsync(in, points, 3 * n * sizeof(double), cudaMemcpyHostToDevice, m->stream));
  const int ni = static_cast<int>(n);
  afl::k_medium_sample<<<(ni + afl::kMT - 1) / afl::kMT, afl::kMT, 0, m->stream>>>(m->dev, in, ni,
                                                                                  o, o + n);
  MED_CUDA(cudaMemcpyAsync(density, o, n * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  MED_CUDA(cudaMemcpyAsync(temperature, o + n, n * sizeof(double), cudaMemcpyDeviceToHost,
                           m->stream));
  return finish(m);
}

afl_status afl_medium_transmittance(afl_medium *m, const afl_ray *rays, size_t n, uint64_t seed,
                                    double *transmittance) {
  if (!m) return fail(AFL_ERR_INVALID_ARGUMENT, "null medium");
  if (n == 0) return AFL_OK;
  if (!rays || !transmittance) return fail(AFL_ERR_INVALID_ARGUMENT, "null buffer");
  if (n > kMaxBatch) return fail(AFL_ERR_INVALID_ARGUMENT, "batch larger than 2^26");
  DeviceScope scope(m->device);
  afl_status st = grow(&m->in, &m->in_cap, n * sizeof(afl_ray));
  if (st == AFL_OK) st = grow(&m->out, &m->out_cap, n * sizeof(double));
  if (st != AFL_OK) return st;
  afl_ray *in = static_cast<afl_ray *>(m->in);
  double *o = static_cast<double *>(m->out);
  MED_CUDA(cudaMemcpyAsync(in, rays, n * sizeof(afl_ray), cudaMemcpyHostToDevice, m->stream));
  const int ni = static_cast<int>(n);
  afl::k_medium_transmittance<<<(ni + afl::kMT - 1) / afl::kMT, afl::kMT, 0, m->stream>>>(
      m->dev, in, ni, static_cast<unsigned long long>(seed), o);
  MED_CUDA(cudaMemcpyAsync(transmittance, o, n * sizeof(double), cudaMemcpyDeviceToHost,
                           m->stream));
  return finish(m);
}

afl_status afl_medium_sample_interaction(afl_medium *m, const afl_ray *rays, size_t n,
                                         uint64_t seed, int32_t *hit, double *t,
                                         double *density, double *temperature) {
  if (!m) return fail(AFL_ERR_INVALID_ARGUMENT, "null medium");
  if (n == 0) return AFL_OK;
  if (!rays || !hit) return fail(AFL_ERR_INVALID_ARGUMENT, "null buffer");
  if (n > kMaxBatch) return fail(AFL_ERR_INVALID_ARGUMENT, "batch larger than 2^26");
  DeviceScope scope(m->device);
  // outputs: t, density, temperature (doubles), then hit (int32)
  afl_status st = grow(&m->in, &m->in_cap, n * sizeof(afl_ray));
  if (st == AFL_OK) st = grow(&m->out, &m->out_cap, n * (3 * sizeof(double) + sizeof(int32_t)));
  if (st != AFL_OK) return st;
  afl_ray *in = static_cast<afl_ray *>(m->in);
  double *o = static_cast<double *>(m->out);
  int32_t *h = reinterpret_cast<int32_t *>(o + 3 * n);
  MED_CUDA(cudaMemcpyAsync(in, rays, n * sizeof(afl_ray), cudaMemcpyHostToDevice, m->stream));
  const int ni = static_cast<int>(n);
  afl::k_medium_interaction<<<(ni + afl::kMT - 1) / afl::kMT, afl::kMT, 0, m->stream>>>(
      m->dev, in, ni, static_cast<unsigned long long>(seed), h, o, o + n, o + 2 * n);
  MED_CUDA(cudaMemcpyAsync(hit, h, n * sizeof(int32_t), cudaMemcpyDeviceToHost, m->stream));
  if (t) MED_CUDA(cudaMemcpyAsync(t, o, n * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  if (density)
    MED_CUDA(cudaMemcpyAsync(density, o + n, n * sizeof(double), cudaMemcpyDeviceToHost,
                             m->stream));
  if (temperature)
    MED_CUDA(cudaMemcpyAsync(temperature, o + 2 * n, n * sizeof(double), cudaMemcpyDeviceToHost,
                             m->stream));
  return finish(m);
}

}  // extern "C"
