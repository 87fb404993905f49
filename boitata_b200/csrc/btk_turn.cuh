// Plane sectors of the search, bit for bit as the reference computes them
// (crates/estimation/src/search.rs:428-434):
//   turn = rem_euclid(atan2(-d.x, d.y), tau),
//   sector = min(floor(turn / tau * n), n - 1),
// with d the sample's offset in the search frame and atan2 the host libm's,
// which is correctly rounded but for very rare inputs. CUDA's atan2 may
// differ from it in the last bit, which moves a sample across a sector
// boundary only when turn / tau * n lies within a few ulps of an integer.
// So the sector is taken from CUDA's atan2 except in that band, where
// atan2 is recomputed correctly rounded: double-double arithmetic (Dekker's
// products and Knuth's sums), atan(t) = 2 atan(t / (1 + sqrt(1 + t^2)))
// three times to bring the argument below 0.1, then the Taylor series of
// atan to 18 terms (the error is far below the 2^-106 of the format), then
// the quadrant. The rest of the arithmetic is the reference's, operation for
// operation.
//
// Host and device: the host build is checked against the host libm's atan2
// on CPU (tests/test_sector_angles.py).
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define BTK_TURN_FN __host__ __device__ __forceinline__
#else
#define BTK_TURN_FN inline
#endif

namespace btk {
namespace turn {

struct DD {
  double hi, lo;
};

BTK_TURN_FN DD two_sum(double a, double b) {
  const double s = a + b;
  const double bb = s - a;
  return {s, (a - (s - bb)) + (b - bb)};
}

BTK_TURN_FN DD fast_two_sum(double a, double b) {  // |a| >= |b|
  const double s = a + b;
  return {s, b - (s - a)};
}

BTK_TURN_FN DD add(DD a, DD b) {
  DD s = two_sum(a.hi, b.hi);
  const DD t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return fast_two_sum(s.hi, s.lo);
}

BTK_TURN_FN DD neg(DD a) { return {-a.hi, -a.lo}; }

BTK_TURN_FN DD mul(DD a, DD b) {
  const double p = a.hi * b.hi;
  double e = fma(a.hi, b.hi, -p);
  e += a.hi * b.lo + a.lo * b.hi;
  return fast_two_sum(p, e);
}

BTK_TURN_FN DD div(DD a, DD b) {
  const double q1 = a.hi / b.hi;
  DD r = add(a, neg(mul(DD{q1, 0.0}, b)));
  const double q2 = r.hi / b.hi;
  r = add(r, neg(mul(DD{q2, 0.0}, b)));
  const double q3 = r.hi / b.hi;
  return add(fast_two_sum(q1, q2), DD{q3, 0.0});
}

BTK_TURN_FN DD sqrt_dd(DD a) {  // a > 0: one Newton step from the double root
  const double x = sqrt(a.hi);
  const DD x2 = mul(DD{x, 0.0}, DD{x, 0.0});
  const DD d = add(a, neg(x2));
  return fast_two_sum(x, d.hi / (2.0 * x));
}

// atan(t) for 0 <= t <= 1.
BTK_TURN_FN DD atan01(DD t) {
  const DD one{1.0, 0.0};
  for (int h = 0; h < 3; ++h) t = div(t, add(one, sqrt_dd(add(one, mul(t, t)))));
  const DD u2 = mul(t, t);
  constexpr int K = 18;
  DD s = div(one, DD{2.0 * K + 1.0, 0.0});
  for (int k = K - 1; k >= 0; --k) s = add(div(one, DD{2.0 * k + 1.0, 0.0}), neg(mul(u2, s)));
  const DD r = mul(t, s);
  return {8.0 * r.hi, 8.0 * r.lo};  // undo the three halvings (exact)
}

// atan2(y, x) correctly rounded (but for inputs within 2^-100 or so of a
// rounding midpoint), for finite nonzero x and y.
BTK_TURN_FN double atan2_rn(double y, double x) {
  const DD pi{3.141592653589793116, 1.2246467991473532e-16};
  const DD half_pi{1.5707963267948966, 6.123233995736766e-17};
  const double ax = fabs(x), ay = fabs(y);
  DD a = ay <= ax ? atan01(div(DD{ay, 0.0}, DD{ax, 0.0})) : add(half_pi, neg(atan01(div(DD{ax, 0.0}, DD{ay, 0.0}))));
  if (x < 0.0) a = add(pi, neg(a));
  if (y < 0.0) a = neg(a);
  return a.hi;
}

// The reference's sector arithmetic from a given atan2 value.
BTK_TURN_FN double turn_fraction(double at, int n) {
  constexpr double kTau = 6.283185307179586;
  double turn = fmod(at, kTau);  // rem_euclid
  if (turn < 0.0) turn += kTau;
  return turn / kTau * double(n);
}

BTK_TURN_FN int sector_from(double x, int n) {
  const int k = x > 0.0 ? int(x) : 0;  // `as usize`: NaN and negatives to 0
  return k < n - 1 ? k : n - 1;
}

// Plane sector (0 .. n - 1) of offset (dx, dy) in the search frame.
BTK_TURN_FN int plane_sector(double dx, double dy, int n) {
  const double y = -dx, x = dy;
  double f = turn_fraction(atan2(y, x), n);
  const double r = floor(f + 0.5);
  if (fabs(f - r) <= 1e-12 * fmax(1.0, f) && x != 0.0 && y != 0.0 && fabs(x) < 1e300 && fabs(y) < 1e300)
    f = turn_fraction(atan2_rn(y, x), n);  // within the band where a last-bit difference could move the sector
  return sector_from(f, n);
}

}  // namespace turn
}  // namespace btk
