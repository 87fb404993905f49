// Device-side types and helpers shared by the kernels of the B200 kriging
// engine (sm_100a). Host code sees the same structs through btk_internal.h.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "btk_internal.h"
#include "btk_turn.cuh"

namespace btk {

// ---- exact-order FP64: no contraction into FMA, round to nearest ----------
// The neighbour search must rank samples exactly as the reference does, so
// projections and squared distances are evaluated with these intrinsics in
// the reference's order (nalgebra gemv: ((m0*x0 + m1*x1) + m2*x2);
// search/grid.rs:109-111: ((dx^2 + dy^2) + dz^2)).
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }

// y = M * x, M row-major 3x3, nalgebra column-accumulation order.
__device__ __forceinline__ void mulv_exact(const double* M, const double x[3], double y[3]) {
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    double s = xmul(M[3 * r + 0], x[0]);
    s = xadd(xmul(M[3 * r + 1], x[1]), s);
    s = xadd(xmul(M[3 * r + 2], x[2]), s);
    y[r] = s;
  }
}

__device__ __forceinline__ double d2_exact(double ax, double ay, double az, double bx, double by, double bz) {
  double dx = xsub(ax, bx), dy = xsub(ay, by), dz = xsub(az, bz);
  return xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
}

// Octant (or quadrant with planar data) of sample w around target t in the
// frame `axes` (search.rs:428-441): bit x<<2 | y<<1 | z of (axes*(w - t) >= 0).
__device__ __forceinline__ int sector_of(const double* axes, int planar, const double w[3], const double t[3]) {
  double v[3] = {xsub(w[0], t[0]), xsub(w[1], t[1]), xsub(w[2], t[2])}, d[3];
  mulv_exact(axes, v, d);
  int bx = d[0] >= 0.0, by = d[1] >= 0.0, bz = d[2] >= 0.0;
  return planar ? (bx << 1) | by : (bx << 2) | (by << 1) | bz;
}

// Sector of sample w around target t under a search's balancing
// (search.rs:428-441): plane sectors by the turn of the offset in the search
// frame (btk_turn.cuh: the reference's arithmetic, with a correctly rounded
// atan2 where the last bit could move the sample across a boundary), else
// the octant or quadrant.
__device__ __forceinline__ int search_sector(const SearchDev& sp, const double w[3], const double t[3]) {
  if (!sp.plane) return sector_of(sp.axes, sp.planar, w, t);
  const double v[3] = {xsub(w[0], t[0]), xsub(w[1], t[1]), xsub(w[2], t[2])};
  double d[3];
  mulv_exact(sp.axes, v, d);
  return turn::plane_sector(d[0], d[1], sp.plane);
}

// ---- variogram (crates/variogram/src/model.rs:76-126, composite.rs:69-85) ----
// Normalized shape g at t = h / range for the stationary models. Precision
// here is ordinary FP64 (the solve is compared to the oracle at 1e-10).
__device__ __forceinline__ double shape64(int model, double param, double t) {
  constexpr double kPi = 3.14159265358979323846;
  switch (model) {
    case BTK_SPHERICAL: return t >= 1.0 ? 1.0 : t * (1.5 - 0.5 * t * t);
    case BTK_EXPONENTIAL: return 1.0 - exp(-3.0 * t);
    case BTK_GAUSSIAN: return 1.0 - exp(-3.0 * t * t);
    case BTK_CUBIC: {
      if (t >= 1.0) return 1.0;
      double t2 = t * t, t3 = t2 * t, t5 = t3 * t2, t7 = t5 * t2;
      return 7.0 * t2 - 8.75 * t3 + 3.5 * t5 - 0.75 * t7;
    }
    case BTK_PENTASPHERICAL: {
      if (t >= 1.0) return 1.0;
      double t2 = t * t, t3 = t2 * t, t5 = t3 * t2;
      return 1.875 * t - 1.25 * t3 + 0.375 * t5;
    }
    case BTK_CIRCULAR:
      return t >= 1.0 ? 1.0 : 1.0 - (2.0 / kPi) * acos(t) + (2.0 * t / kPi) * sqrt(1.0 - t * t);
    case BTK_SINEHOLE: {
      double c = kPi * t;
      return 1.0 - sin(c) / c;
    }
    case BTK_MATERN: {
      int o = param < 1.0 ? 0 : (param < 2.0 ? 1 : 2);
      double k = o == 0 ? 3.0 : (o == 1 ? 3.0 * 1.7320508075688772 : 3.0 * 2.23606797749979);
      double delta = k * t, e = exp(-delta);
      if (o == 0) return 1.0 - e;
      if (o == 1) return 1.0 - (1.0 + delta) * e;
      return 1.0 - (1.0 + delta + delta * delta / 3.0) * e;
    }
    case BTK_POWER: return pow(t, param);  // unbounded (model.rs:124)
  }
  return 0.0;
}

// C(h) = C(0) - gamma(h); C(0) at h <= 0 (composite.rs:79-85).
__device__ __forceinline__ double cov64(const VgDev& vg, double h) {
  if (!(h > 0.0)) return vg.c0;
  double gam = 0.0;
  for (int s = 0; s < vg.nstruct; ++s) gam += vg.sill[s] * shape64(vg.model[s], vg.param[s], h * vg.inv_range[s]);
  return vg.c0 - (vg.nugget + gam);
}

// dC/dh at h > 0 (model.rs:181-312 via composite.rs:138-162), for the adjoint.
__device__ __forceinline__ double dshape64(int model, double param, double t) {
  constexpr double kPi = 3.14159265358979323846;
  switch (model) {
    case BTK_SPHERICAL: return t >= 1.0 ? 0.0 : 1.5 - 1.5 * t * t;
    case BTK_EXPONENTIAL: return 3.0 * exp(-3.0 * t);
    case BTK_GAUSSIAN: return 6.0 * t * exp(-3.0 * t * t);
    case BTK_CUBIC: {
      if (t >= 1.0) return 0.0;
      double t2 = t * t, t4 = t2 * t2, t6 = t4 * t2;
      return 14.0 * t - 26.25 * t2 + 17.5 * t4 - 5.25 * t6;
    }
    case BTK_PENTASPHERICAL: {
      if (t >= 1.0) return 0.0;
      double t2 = t * t;
      return 1.875 - 3.75 * t2 + 1.875 * t2 * t2;
    }
    case BTK_CIRCULAR: return t >= 1.0 ? 0.0 : (4.0 / kPi) * sqrt(fmax(1.0 - t * t, 0.0));
    case BTK_SINEHOLE: {
      double c = kPi * t;
      if (fabs(c) < 1e-4) return kPi * c / 3.0;
      return kPi * (sin(c) - c * cos(c)) / (c * c);
    }
    case BTK_MATERN: {
      int o = param < 1.0 ? 0 : (param < 2.0 ? 1 : 2);
      double k = o == 0 ? 3.0 : (o == 1 ? 3.0 * 1.7320508075688772 : 3.0 * 2.23606797749979);
      double delta = k * t, e = exp(-delta);
      if (o == 0) return k * e;
      if (o == 1) return k * delta * e;
      return k * (delta / 3.0) * (1.0 + delta) * e;
    }
  }
  return 0.0;
}

// FP32 lag-to-covariance (the mixed form's preconditioner only).
__device__ __forceinline__ float shape32(int model, float param, float t) {
  constexpr float kPi = 3.14159265f;
  switch (model) {
    case BTK_SPHERICAL: return t >= 1.f ? 1.f : t * (1.5f - 0.5f * t * t);
    case BTK_EXPONENTIAL: return 1.f - __expf(-3.f * t);
    case BTK_GAUSSIAN: return 1.f - __expf(-3.f * t * t);
    case BTK_CUBIC: {
      if (t >= 1.f) return 1.f;
      float t2 = t * t, t3 = t2 * t, t5 = t3 * t2, t7 = t5 * t2;
      return 7.f * t2 - 8.75f * t3 + 3.5f * t5 - 0.75f * t7;
    }
    case BTK_PENTASPHERICAL: {
      if (t >= 1.f) return 1.f;
      float t2 = t * t, t3 = t2 * t, t5 = t3 * t2;
      return 1.875f * t - 1.25f * t3 + 0.375f * t5;
    }
    case BTK_CIRCULAR:
      return t >= 1.f ? 1.f : 1.f - (2.f / kPi) * acosf(t) + (2.f * t / kPi) * sqrtf(1.f - t * t);
    case BTK_SINEHOLE: {
      float c = kPi * t;
      return 1.f - __sinf(c) / c;
    }
    case BTK_MATERN: {
      int o = param < 1.f ? 0 : (param < 2.f ? 1 : 2);
      float k = o == 0 ? 3.f : (o == 1 ? 5.19615242f : 6.70820393f);
      float delta = k * t, e = __expf(-delta);
      if (o == 0) return 1.f - e;
      if (o == 1) return 1.f - (1.f + delta) * e;
      return 1.f - (1.f + delta + delta * delta / 3.f) * e;
    }
  }
  return 0.f;
}

// ---- shared by the solve kernels (btk_solve.cu, btk_tile.cu) ----
// Lag |M (b - a)| between world points a and b, M the variogram frame
// (identity without anisotropy): the difference is taken in world
// coordinates, then rotated, with a fixed operation order, so the value
// depends on the pair alone (and is symmetric bit for bit) whichever kernel
// or tile evaluates it (kernel.rs:34-42 projects the same differences).
__device__ __forceinline__ double lag_world(const VgDev& vg, double ax, double ay, double az, double bx, double by,
                                            double bz) {
  double d0 = bx - ax, d1 = by - ay, d2 = bz - az;
  if (vg.has_frame) {
    const double* M = vg.frame;
    const double r0 = fma(M[2], d2, fma(M[1], d1, M[0] * d0));
    const double r1 = fma(M[5], d2, fma(M[4], d1, M[3] * d0));
    const double r2 = fma(M[8], d2, fma(M[7], d1, M[6] * d0));
    d0 = r0, d1 = r1, d2 = r2;
  }
  return sqrt(fma(d2, d2, fma(d1, d1, d0 * d0)));
}

__device__ __forceinline__ double kind_f(int kind, double kparam, double z) {
  return kind == BTK_SIMPLE ? z - kparam : (kind == BTK_INDICATOR ? (z <= kparam ? 1.0 : 0.0) : z);
}

__device__ __forceinline__ double lag64(const VgDev& vg, const double* a, const double* b) {
  double d[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  if (vg.has_frame) {
    double r[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) r[k] = vg.frame[3 * k] * d[0] + vg.frame[3 * k + 1] * d[1] + vg.frame[3 * k + 2] * d[2];
    d[0] = r[0], d[1] = r[1], d[2] = r[2];
  }
  return sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
}

__device__ __forceinline__ void tri_index(int e, int& i, int& j) {
  int r = int((1.0f + sqrtf(8.0f * float(e) + 1.0f)) * 0.5f);
  while (r * (r - 1) / 2 > e) --r;
  while ((r + 1) * r / 2 <= e) ++r;
  i = r, j = e - r * (r - 1) / 2;
}

__device__ __forceinline__ void write_fail(const SolveDev& a, int64_t ti, int8_t st, int n_used) {
  a.value[ti] = NAN;
  if (a.variance) a.variance[ti] = NAN;
  if (a.lagrange) a.lagrange[ti] = NAN;
  if (a.n_used) a.n_used[ti] = n_used;
  if (a.status) a.status[ti] = st;
}

// Estimate, variance and Lagrange multiplier from the five forms
// s[0] = 1'C^-1 c, s[1] = 1'C^-1 1, s[2] = f'C^-1 c, s[3] = f'C^-1 1,
// s[4] = c'C^-1 c (kernel.rs:86-122).
// Covariance of sample (sx, sy, sz) with the target (tx, ty, tz): point
// support, or, with block support, the mean over the block's discretization
// points of the point covariance with the nugget left out at zero lag (one
// point: point support) (crates/estimation/src/block.rs:101-116 with
// crates/variogram/src/composite.rs:108-115).
__device__ __forceinline__ double support_cov(const SolveDev& a, double tx, double ty, double tz, double sx,
                                              double sy, double sz) {
  if (a.sup_n <= 0) return cov64(a.vg, lag_world(a.vg, tx, ty, tz, sx, sy, sz));
  double sum = 0.0;
  for (int k = 0; k < a.sup_n; ++k) {
    const double h = lag_world(a.vg, tx + a.sup[3 * k], ty + a.sup[3 * k + 1], tz + a.sup[3 * k + 2], sx, sy, sz);
    sum += a.sup_n == 1 || h > 0.0 ? cov64(a.vg, h) : a.vg.c0 - a.vg.nugget;
  }
  return sum / double(a.sup_n);
}

__device__ __forceinline__ void epilogue(const SolveDev& a, int kind, int64_t ti, const double s[5], int n_used,
                                         int8_t flag) {
  // C(0) for point support; C(B,B) for a block (block.rs:186-187)
  const double c0 = a.sup_n > 0 ? *a.sup_cbb : a.vg.c0;
  double mu, value, swc;
  if (kind == BTK_SIMPLE) {
    mu = 0.0;
    value = a.kparam + s[2];
    swc = s[4];
  } else {
    mu = (s[0] - 1.0) / s[1];
    value = s[2] - mu * s[3];
    if (kind == BTK_INDICATOR) value = value < 0.0 ? 0.0 : (value > 1.0 ? 1.0 : value);
    swc = s[4] - mu * s[0];
  }
  a.value[ti] = value;
  if (a.variance) a.variance[ti] = fmax(c0 - swc - mu, 0.0);
  if (a.lagrange) a.lagrange[ti] = mu;
  if (a.n_used) a.n_used[ti] = n_used;
  if (a.status) a.status[ti] = int8_t(BTK_ST_OK | flag);
}

}  // namespace btk
