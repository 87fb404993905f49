// Device-side types and helpers shared by the kernels of the B200 kriging
// engine (sm_100a). Host code sees the same structs through btk_internal.h.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "btk_internal.h"

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

}  // namespace btk
