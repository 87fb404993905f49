// ORACLE — test infrastructure only.
//
// A CPU restatement, in plain C++17, of boitatá's ordinary / simple /
// indicator kriging path (gstvschlz/boitata, workspace 0.7.1). The tests
// compare the CUDA engine in boitata_b200/ with it, and bench.py times it as
// the CPU baseline ("port"). Nothing in the product links, loads or calls it.
//
// Every function cites the reference file:line it follows. Floating-point
// evaluation order follows the reference wherever the result must be
// bit-identical (the search: projections, squared distances, octant signs);
// build with -ffp-contract=off so no FMA is formed (Rust forms none).
//
// Third-party arithmetic on the path: nalgebra 0.33 (Cargo.toml:32). Its
// Matrix3*Matrix3 and Matrix3*Vector3 go through gemm -> gemv, which adds
// columns in order: y = A[:,0]*x0; y = A[:,1]*x1 + y; y = A[:,2]*x2 + y
// (nalgebra src/base/blas.rs gemv/axcpy). mul3/mulv below restate that.
// Its 3-vector dot is (a0*b0 + a1*b1) + a2*b2 (blas.rs dotx fixed-size case).
// Its LU (src/linalg/lu.rs, gauss_step) scales the column by 1/diag and
// updates with axpy; krige_lu below restates it for the n > 64 cross-check.
//
// Pinned by tests/test_oracle_*.py against the reference's own known-answer
// and property tests (kernel.rs:182-278, krige.rs:218-388, coincident.rs:
// 114-256, lib.rs:111-137, grid.rs:421-537, search.rs:1121-1516,
// rotation.rs:45-90, model.rs:335-430) ported to Python.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <queue>
#include <utility>
#include <vector>
#include <thread>

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kTau = 6.28318530717958647692;

// ---------------------------------------------------------------- 3x3 math
struct M3 {
  double m[3][3];
};

M3 identity() {
  M3 r{};
  r.m[0][0] = r.m[1][1] = r.m[2][2] = 1.0;
  return r;
}

// nalgebra gemm via gemv, column by column (see header).
M3 mul3(const M3& a, const M3& b) {
  M3 r{};
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) {
      double y = a.m[i][0] * b.m[0][j];
      y = a.m[i][1] * b.m[1][j] + y;
      y = a.m[i][2] * b.m[2][j] + y;
      r.m[i][j] = y;
    }
  return r;
}

void mulv(const M3& a, const double x[3], double y[3]) {
  for (int i = 0; i < 3; ++i) {
    double s = a.m[i][0] * x[0];
    s = a.m[i][1] * x[1] + s;
    s = a.m[i][2] * x[2] + s;
    y[i] = s;
  }
}

M3 from_rows(double a00, double a01, double a02, double a10, double a11, double a12, double a20,
             double a21, double a22) {
  M3 r;
  r.m[0][0] = a00, r.m[0][1] = a01, r.m[0][2] = a02;
  r.m[1][0] = a10, r.m[1][1] = a11, r.m[1][2] = a12;
  r.m[2][0] = a20, r.m[2][1] = a21, r.m[2][2] = a22;
  return r;
}

double to_radians(double deg) { return deg * (kPi / 180.0); }  // f64::to_radians

// crates/core/src/rotation.rs:8-16
M3 rotation_matrix(double azimuth, double dip, double rake) {
  double sa = std::sin(to_radians(azimuth)), ca = std::cos(to_radians(azimuth));
  double sd = std::sin(to_radians(dip)), cd = std::cos(to_radians(dip));
  double sr = std::sin(to_radians(rake)), cr = std::cos(to_radians(rake));
  M3 r1 = from_rows(sa, ca, 0.0, -ca, sa, 0.0, 0.0, 0.0, 1.0);
  M3 r2 = from_rows(cd, 0.0, -sd, 0.0, 1.0, 0.0, sd, 0.0, cd);
  M3 r3 = from_rows(1.0, 0.0, 0.0, 0.0, cr, sr, 0.0, -sr, cr);
  return mul3(mul3(r3, r2), r1);
}

// crates/core/src/rotation.rs:40-43: rows (-r.row(1), r.row(0), r.row(2)).
M3 block_frame(double azimuth, double dip, double rake) {
  M3 r = rotation_matrix(azimuth, dip, rake);
  return from_rows(-r.m[1][0], -r.m[1][1], -r.m[1][2], r.m[0][0], r.m[0][1], r.m[0][2], r.m[2][0],
                   r.m[2][1], r.m[2][2]);
}

// ------------------------------------------------------------- anisotropy
struct Aniso {
  bool on = false;
  double azimuth = 0, dip = 0, rake = 0, major = 1, semi = 1, minor = 1;
  M3 rotation = identity();
};

Aniso make_aniso(double az, double dip, double rake, double major, double semi, double minor) {
  Aniso a;  // crates/variogram/src/aniso.rs:75-79
  a.on = true;
  a.azimuth = az, a.dip = dip, a.rake = rake, a.major = major, a.semi = semi, a.minor = minor;
  a.rotation = rotation_matrix(az, dip, rake);
  return a;
}

// aniso.rs:88-94: diag(1/major, 1/semi, 1/minor) * rotation
M3 aniso_matrix(const Aniso& a) {
  M3 d{};
  d.m[0][0] = 1.0 / a.major;
  d.m[1][1] = 1.0 / a.semi;
  d.m[2][2] = 1.0 / a.minor;
  return mul3(d, a.rotation);
}

double norm3(const double v[3]) { return std::sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]); }

// aniso.rs:101-110 and euclidean :114-119
double aniso_lag(const Aniso& a, const double p[3], const double q[3]) {
  double v[3] = {q[0] - p[0], q[1] - p[1], q[2] - p[2]};
  if (!a.on) return std::sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]);
  double r[3];
  mulv(a.rotation, v, r);
  double s[3] = {r[0] / a.major, r[1] / a.semi, r[2] / a.minor};
  return norm3(s);
}

// ---------------------------------------------------------------- models
enum Model { SPHERICAL = 0, EXPONENTIAL, GAUSSIAN, CUBIC, PENTASPHERICAL, CIRCULAR, SINEHOLE,
             MATERN, POWER };

double p2(double t) { return t * t; }                    // powi(2)
double p3(double t) { return t * (t * t); }              // powi(3): x * x^2
double p4(double t) { double s = t * t; return s * s; }  // powi(4)
double p5(double t) { double s = t * t; return t * (s * s); }
double p6(double t) { double s = t * t; return s * (s * s); }
double p7(double t) { double s = t * t; return (t * s) * (s * s); }

int matern_order(double order) { return order < 1.0 ? 0 : (order < 2.0 ? 1 : 2); }  // model.rs:138-146
double matern_nu(int o) { return o == 0 ? 0.5 : (o == 1 ? 1.5 : 2.5); }

// crates/variogram/src/model.rs:76-126 (and matern_shape :165-173)
double shape(int model, double param, double h, double range) {
  if (!std::isfinite(h)) return 0.0;
  if (h <= 0.0) return 0.0;
  double r = std::fmax(range, std::numeric_limits<double>::min());
  double t = h / r;
  switch (model) {
    case SPHERICAL: return t >= 1.0 ? 1.0 : 1.5 * t - 0.5 * p3(t);
    case EXPONENTIAL: return 1.0 - std::exp(-3.0 * t);
    case GAUSSIAN: return 1.0 - std::exp(-3.0 * t * t);
    case CUBIC:
      return t >= 1.0 ? 1.0
                      : 7.0 * p2(t) - (35.0 / 4.0) * p3(t) + (7.0 / 2.0) * p5(t) -
                            (3.0 / 4.0) * p7(t);
    case PENTASPHERICAL:
      return t >= 1.0 ? 1.0 : (15.0 / 8.0) * t - (5.0 / 4.0) * p3(t) + (3.0 / 8.0) * p5(t);
    case CIRCULAR:
      return t >= 1.0 ? 1.0
                      : 1.0 - (2.0 / kPi) * std::acos(t) + (2.0 * t / kPi) * std::sqrt(1.0 - t * t);
    case SINEHOLE: {
      double c = kPi * t;
      return 1.0 - std::sin(c) / c;
    }
    case MATERN: {
      int o = matern_order(param);
      double delta = (std::sqrt(2.0 * matern_nu(o)) * 3.0) * t;
      if (o == 0) return 1.0 - std::exp(-delta);
      if (o == 1) return 1.0 - (1.0 + delta) * std::exp(-delta);
      return 1.0 - (1.0 + delta + delta * delta / 3.0) * std::exp(-delta);
    }
    case POWER: return std::pow(t, param);
  }
  return 0.0;
}

// model.rs:207-312: (dG/dt, d2G/dt2)
void d_shape(int model, double param, double t, double* d1, double* d2) {
  switch (model) {
    case SPHERICAL:
      if (t >= 1.0) { *d1 = 0, *d2 = 0; } else { *d1 = 1.5 - 1.5 * t * t; *d2 = -3.0 * t; }
      return;
    case EXPONENTIAL: {
      double e = std::exp(-3.0 * t);
      *d1 = 3.0 * e, *d2 = -9.0 * e;
      return;
    }
    case GAUSSIAN: {
      double e = std::exp(-3.0 * t * t);
      *d1 = 6.0 * t * e, *d2 = (6.0 - 36.0 * t * t) * e;
      return;
    }
    case CUBIC:
      if (t >= 1.0) { *d1 = 0, *d2 = 0; return; }
      *d1 = 14.0 * t - (105.0 / 4.0) * p2(t) + (35.0 / 2.0) * p4(t) - (21.0 / 4.0) * p6(t);
      *d2 = 14.0 - (105.0 / 2.0) * t + 70.0 * p3(t) - (63.0 / 2.0) * p5(t);
      return;
    case PENTASPHERICAL:
      if (t >= 1.0) { *d1 = 0, *d2 = 0; return; }
      *d1 = 15.0 / 8.0 - (15.0 / 4.0) * t * t + (15.0 / 8.0) * p4(t);
      *d2 = -(15.0 / 2.0) * t + (15.0 / 2.0) * p3(t);
      return;
    case CIRCULAR: {
      if (t >= 1.0) { *d1 = 0, *d2 = 0; return; }
      double s = std::sqrt(std::fmax(1.0 - t * t, 0.0));
      *d1 = (4.0 / kPi) * s;
      *d2 = s > 0.0 ? -(4.0 / kPi) * t / s : -std::numeric_limits<double>::infinity();
      return;
    }
    case SINEHOLE: {
      double c = kPi * t;
      if (std::fabs(c) < 1e-4) { *d1 = kPi * c / 3.0; *d2 = kPi * kPi / 3.0; return; }
      double sn = std::sin(c), cs = std::cos(c);
      double u = (sn - c * cs) / (c * c);
      double du = (c * c * sn - 2.0 * sn + 2.0 * c * cs) / p3(c);
      *d1 = kPi * u, *d2 = kPi * kPi * du;
      return;
    }
    case MATERN: {  // model.rs:298-312
      int o = matern_order(param);
      double k = std::sqrt(2.0 * matern_nu(o)) * 3.0;
      double delta = k * t, e = std::exp(-delta);
      if (o == 0) { *d1 = k * e; *d2 = -k * k * e; }
      else if (o == 1) { *d1 = k * delta * e; *d2 = k * k * (1.0 - delta) * e; }
      else { *d1 = k * (delta / 3.0) * (1.0 + delta) * e; *d2 = k * k * (1.0 + delta - delta * delta) * e / 3.0; }
      return;
    }
    case POWER: {
      double e = param;
      if (t <= 0.0) {
        *d1 = e > 1.0 ? 0.0 : std::numeric_limits<double>::infinity();
        *d2 = e > 2.0 ? 0.0 : (e == 2.0 ? 2.0 : std::numeric_limits<double>::infinity());
      } else {
        *d1 = e * std::pow(t, e - 1.0);
        *d2 = e * (e - 1.0) * std::pow(t, e - 2.0);
      }
      return;
    }
  }
  *d1 = 0, *d2 = 0;
}

// model.rs:181-188
double shape_d1(int model, double param, double h, double range) {
  if (!std::isfinite(h) || h < 0.0) return 0.0;
  double r = std::fmax(range, std::numeric_limits<double>::min());
  double d1, d2;
  d_shape(model, param, h / r, &d1, &d2);
  return d1 / r;
}

// -------------------------------------------------------------- variogram
struct Structure { int model; double param, sill, range; };

struct Variogram {
  double nugget = 0;
  std::vector<Structure> s;
  Aniso aniso;

  // composite.rs:50-52 (Sum folds left to right)
  double total_sill() const {
    double sum = -0.0;
    for (auto& x : s) sum = sum + x.sill;
    return nugget + sum;
  }
  bool stationary() const {  // composite.rs:64-66
    for (auto& x : s) if (x.model == POWER) return false;
    return true;
  }
  // composite.rs:69-76
  double gamma(double h) const {
    double structural = -0.0;
    for (auto& x : s) structural = structural + x.sill * shape(x.model, x.param, h, x.range);
    return h > 0.0 ? nugget + structural : 0.0;
  }
  double cov(double h) const { return h <= 0.0 ? total_sill() : total_sill() - gamma(h); }  // :79-85
  double lag(const double p[3], const double q[3]) const { return aniso_lag(aniso, p, q); }  // :88-93
  double cov_points(const double p[3], const double q[3]) const { return cov(lag(p, q)); }  // :101-103
  // composite.rs:108-115: the nugget left out at zero lag (block support)
  double block_cov_points(const double p[3], const double q[3]) const {
    double h = lag(p, q);
    return h <= 0.0 ? total_sill() - nugget : cov(h);
  }
  // composite.rs:120-129
  double block_mean_cov(const std::vector<std::array<double, 3>>& pts) const {
    if (pts.size() == 1) return total_sill();
    double total = -0.0;
    for (auto& a : pts) {
      double row = -0.0;
      for (auto& b : pts) row = row + block_cov_points(a.data(), b.data());
      total = total + row;
    }
    return total / double(pts.size() * pts.size());
  }
};

// ------------------------------------------------------------------ kriging
enum Kind { ORDINARY = 0, SIMPLE = 1, INDICATOR = 2 };
enum Status { OK = 0, SEARCH_FAILED = 1, SINGULAR = 2, INSUFFICIENT = 3, INVALID = 4, NONE = -1 };

struct Sample { double loc[3]; double value; int64_t hole; double err; int64_t domain = -1; };

struct Estimate {
  double value = NAN, variance = NAN, lagrange = NAN, support = NAN;
  size_t n_used = 0;
  std::vector<double> weights;
};

// f64::clamp(0, 1): NaN stays NaN
double clamp01(double x) {
  if (x < 0.0) x = 0.0;
  if (x > 1.0) x = 1.0;
  return x;
}

// kernel.rs:11-17
constexpr size_t KMAX = 64;
constexpr double PIVOT = 1e-12;

// crates/estimation/src/kernel.rs:24-123. Returns NONE when the system is
// beyond the kernel (n == 0, n > 64, non-stationary variogram).
int kernel_krige(int kind, double kparam, const double t[3], const std::vector<Sample>& smp,
                 const Variogram& vg, Estimate& out) {
  size_t n = smp.size();
  if (n == 0 || n > KMAX || !vg.stationary()) return NONE;
  M3 frame = vg.aniso.on ? aniso_matrix(vg.aniso) : identity();
  static thread_local double p[KMAX][3];
  for (size_t i = 0; i < n; ++i) {
    double d[3] = {smp[i].loc[0] - t[0], smp[i].loc[1] - t[1], smp[i].loc[2] - t[2]};
    if (vg.aniso.on) mulv(frame, d, p[i]);
    else { p[i][0] = d[0], p[i][1] = d[1], p[i][2] = d[2]; }
  }
  auto norm = [](const double* a, const double* b) {
    return std::sqrt(p2(a[0] - b[0]) + p2(a[1] - b[1]) + p2(a[2] - b[2]));
  };
  double c0 = vg.total_sill();
  static thread_local double l[KMAX * (KMAX + 1) / 2];
  static thread_local double c[KMAX];
  const double zero[3] = {0, 0, 0};
  for (size_t i = 0; i < n; ++i) {
    size_t row = i * (i + 1) / 2;
    for (size_t j = 0; j < i; ++j) l[row + j] = vg.cov(norm(p[i], p[j]));
    l[row + i] = c0 + smp[i].err;
    c[i] = vg.cov(norm(p[i], zero));
  }
  auto dot = [](const double* a, const double* b, size_t len) {
    double s = -0.0;
    for (size_t k = 0; k < len; ++k) s = s + a[k] * b[k];
    return s;
  };
  for (size_t j = 0; j < n; ++j) {
    size_t rj = j * (j + 1) / 2;
    double d = l[rj + j] - dot(&l[rj], &l[rj], j);
    if (std::isnan(d) || d <= PIVOT * c0) return SINGULAR;
    d = std::sqrt(d);
    l[rj + j] = d;
    for (size_t i = j + 1; i < n; ++i) {
      size_t ri = i * (i + 1) / 2;
      l[ri + j] = (l[ri + j] - dot(&l[ri], &l[rj], j)) / d;
    }
  }
  auto solve = [&](double* v) {
    for (size_t i = 0; i < n; ++i) {
      size_t ri = i * (i + 1) / 2;
      v[i] = (v[i] - dot(&l[ri], v, i)) / l[ri + i];
    }
    for (size_t i = n; i-- > 0;) {
      double s = v[i];
      for (size_t k = i + 1; k < n; ++k) s -= l[k * (k + 1) / 2 + i] * v[k];
      v[i] = s / l[i * (i + 1) / 2 + i];
    }
  };
  double a[KMAX], b[KMAX];
  std::copy(c, c + n, a);
  solve(a);
  bool ordinary = kind != SIMPLE;
  double mu = 0.0;
  if (ordinary) {
    for (size_t i = 0; i < n; ++i) b[i] = 1.0;
    solve(b);
    double sa = -0.0, sb = -0.0;
    for (size_t i = 0; i < n; ++i) sa = sa + a[i];
    for (size_t i = 0; i < n; ++i) sb = sb + b[i];
    mu = (sa - 1.0) / sb;
  } else {
    for (size_t i = 0; i < n; ++i) b[i] = 0.0;
  }
  out.weights.resize(n);
  for (size_t i = 0; i < n; ++i) out.weights[i] = a[i] - mu * b[i];
  double value = -0.0;
  if (kind == SIMPLE) {
    for (size_t i = 0; i < n; ++i) value = value + out.weights[i] * (smp[i].value - kparam);
    value = kparam + value;
  } else if (kind == INDICATOR) {
    for (size_t i = 0; i < n; ++i) value = value + out.weights[i] * (smp[i].value <= kparam ? 1.0 : 0.0);
    value = clamp01(value);
  } else {
    for (size_t i = 0; i < n; ++i) value = value + out.weights[i] * smp[i].value;
  }
  double swc = -0.0;
  for (size_t i = 0; i < n; ++i) swc = swc + out.weights[i] * c[i];
  out.value = value;
  out.variance = std::fmax(c0 - swc - mu, 0.0);
  out.n_used = n;
  out.lagrange = mu;
  out.support = c0;
  return OK;
}

// nalgebra 0.33 LU with partial pivoting (lu.rs::new, gauss_step) and
// LU::solve (permute, unit-lower solve, upper solve), column oriented.
bool lu_solve(std::vector<double>& A, size_t dim, std::vector<double>& b) {
  std::vector<size_t> perm_a, perm_b;
  auto at = [&](size_t i, size_t j) -> double& { return A[i * dim + j]; };
  for (size_t i = 0; i < dim; ++i) {
    size_t piv = i;
    double best = std::fabs(at(i, i));
    for (size_t r = i + 1; r < dim; ++r)
      if (std::fabs(at(r, i)) > best) best = std::fabs(at(r, i)), piv = r;  // icamax: first max
    double diag = at(piv, i);
    if (diag == 0.0) continue;
    if (piv != i) {
      perm_a.push_back(i), perm_b.push_back(piv);
      for (size_t j = 0; j < dim; ++j) std::swap(at(i, j), at(piv, j));
    }
    double inv = 1.0 / diag;
    for (size_t r = i + 1; r < dim; ++r) at(r, i) *= inv;
    for (size_t k = i + 1; k < dim; ++k) {
      double pk = at(i, k);
      for (size_t r = i + 1; r < dim; ++r) at(r, k) = (-pk) * at(r, i) + at(r, k);
    }
  }
  for (size_t q = 0; q < perm_a.size(); ++q) std::swap(b[perm_a[q]], b[perm_b[q]]);
  for (size_t i = 0; i < dim; ++i) {
    double coeff = b[i];
    for (size_t r = i + 1; r < dim; ++r) b[r] = (-coeff) * at(r, i) + b[r];
  }
  for (size_t i = dim; i-- > 0;) {
    double diag = at(i, i);
    if (diag == 0.0) return false;
    double coeff = b[i] / diag;
    b[i] = coeff;
    for (size_t r = 0; r < i; ++r) b[r] = (-coeff) * at(r, i) + b[r];
  }
  return true;
}

// crates/estimation/src/krige.rs:127-201
int krige_lu(int kind, double kparam, const double t[3], const std::vector<Sample>& smp,
             const Variogram& vg, Estimate& out) {
  size_t n = smp.size();
  if (n == 0) return INSUFFICIENT;
  if (kind == SIMPLE && !vg.stationary()) return INVALID;
  std::vector<double> z(n);
  for (size_t i = 0; i < n; ++i)
    z[i] = kind == INDICATOR ? (smp[i].value <= kparam ? 1.0 : 0.0) : smp[i].value;
  double c0 = vg.total_sill();
  bool ordinary = kind != SIMPLE;
  size_t dim = ordinary ? n + 1 : n;
  std::vector<double> A(dim * dim, 0.0), b(dim, 0.0);
  for (size_t i = 0; i < n; ++i) {
    for (size_t j = 0; j < n; ++j) A[i * dim + j] = vg.cov_points(smp[i].loc, smp[j].loc);
    A[i * dim + i] += smp[i].err;
    b[i] = vg.cov_points(smp[i].loc, t);
  }
  std::vector<double> rhs = b;
  if (ordinary) {
    for (size_t i = 0; i < n; ++i) A[i * dim + n] = 1.0, A[n * dim + i] = 1.0;
    A[n * dim + n] = 0.0;
    rhs[n] = 1.0;
  }
  if (!lu_solve(A, dim, rhs)) return SINGULAR;
  out.weights.assign(rhs.begin(), rhs.begin() + n);
  double value = -0.0;
  if (kind == SIMPLE) {
    for (size_t i = 0; i < n; ++i) value = value + out.weights[i] * (z[i] - kparam);
    value = kparam + value;
  } else {
    for (size_t i = 0; i < n; ++i) value = value + out.weights[i] * z[i];
    if (kind == INDICATOR) value = clamp01(value);
  }
  double swc = -0.0;
  for (size_t i = 0; i < n; ++i) swc = swc + out.weights[i] * b[i];
  double mu = ordinary ? rhs[n] : 0.0;
  out.value = value;
  out.variance = std::fmax(c0 - swc - mu, 0.0);
  out.n_used = n;
  out.lagrange = mu;
  out.support = c0;
  return OK;
}

// crates/estimation/src/coincident.rs:11-15
constexpr double EPS = 1e-6;
bool close(const double* p, const double* q) {
  return p2(p[0] - q[0]) + p2(p[1] - q[1]) + p2(p[2] - q[2]) <= EPS * EPS;
}

// krige.rs:98-113
double kind_value(int kind, double kparam, const std::vector<double>& w, const std::vector<Sample>& s) {
  double sum = -0.0;
  for (size_t i = 0; i < w.size(); ++i) {
    double z = s[i].value;
    double f = kind == SIMPLE ? z - kparam : (kind == INDICATOR ? (z <= kparam ? 1.0 : 0.0) : z);
    sum = sum + w[i] * f;
  }
  if (kind == SIMPLE) return kparam + sum;
  if (kind == INDICATOR) return clamp01(sum);
  return sum;
}

// crates/estimation/src/krige.rs:83-95 with coincident.rs:27-111
int krige(int kind, double kparam, const double t[3], const std::vector<Sample>& smp,
          const Variogram& vg, Estimate& out) {
  size_t n = smp.size();
  bool any = false;
  for (size_t i = 0; i < n && !any; ++i)
    for (size_t j = 0; j < i; ++j)
      if (close(smp[i].loc, smp[j].loc)) { any = true; break; }
  if (any) {
    std::vector<size_t> of;
    std::vector<std::vector<size_t>> members;
    for (size_t i = 0; i < n; ++i) {
      size_t c = members.size();
      for (size_t m = 0; m < members.size(); ++m)
        if (close(smp[members[m][0]].loc, smp[i].loc)) { c = m; break; }
      if (c == members.size()) members.push_back({i});
      else members[c].push_back(i);
      of.push_back(c);
    }
    double c0 = vg.total_sill();
    std::vector<Sample> merged;
    for (auto& m : members) {
      Sample first = smp[m[0]];
      if (m.size() > 1) {
        double k = double(m.size());
        double var = 0.0;
        for (size_t i : m) {
          var += smp[i].err;
          for (size_t j : m) var += vg.cov_points(smp[i].loc, smp[j].loc);
        }
        double vs = -0.0;
        for (size_t i : m) vs = vs + smp[i].value;
        first.value = vs / k;
        first.err = var / (k * k) - c0;
      }
      merged.push_back(first);
    }
    Estimate e;
    int st = krige(kind, kparam, t, merged, vg, e);
    if (st != OK) return st;
    std::vector<double> w(n);
    for (size_t i = 0; i < n; ++i) w[i] = e.weights[of[i]] / double(members[of[i]].size());
    e.weights = w;
    e.value = kind_value(kind, kparam, w, smp);
    e.n_used = n;
    out = e;
    return OK;
  }
  int st = kernel_krige(kind, kparam, t, smp, vg, out);
  if (st != NONE) return st;
  return krige_lu(kind, kparam, t, smp, vg, out);
}

// ---------------------------------------------------------- block kriging
// crates/estimation/src/block.rs:40-57 (Discretization::points): i outer,
// k inner.
std::vector<std::array<double, 3>> disc_points(const double c[3], const double size[3], const int64_t nd[3]) {
  std::vector<std::array<double, 3>> pts;
  double dx = size[0] / double(nd[0]), dy = size[1] / double(nd[1]), dz = size[2] / double(nd[2]);
  double x0 = c[0] - size[0] / 2.0 + dx / 2.0, y0 = c[1] - size[1] / 2.0 + dy / 2.0, z0 = c[2] - size[2] / 2.0 + dz / 2.0;
  for (int64_t i = 0; i < nd[0]; ++i)
    for (int64_t j = 0; j < nd[1]; ++j)
      for (int64_t k = 0; k < nd[2]; ++k)
        pts.push_back({x0 + double(i) * dx, y0 + double(j) * dy, z0 + double(k) * dz});
  return pts;
}

// block.rs:61-72 (Discretization::offsets): block_frame(rotation)^T times the
// points of a block centred at the origin (nalgebra Matrix3 * Vector3).
std::vector<std::array<double, 3>> disc_offsets(const double size[3], const int64_t nd[3], const double rot[3]) {
  M3 f = block_frame(rot[0], rot[1], rot[2]);
  M3 ft;
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) ft.m[i][j] = f.m[j][i];
  const double zero[3] = {0.0, 0.0, 0.0};
  auto pts = disc_points(zero, size, nd);
  for (auto& p : pts) {
    double y[3];
    mulv(ft, p.data(), y);
    p = {y[0], y[1], y[2]};
  }
  return pts;
}

// block.rs:101-116 (block_covariances): the mean covariance of each sample
// with the discretization, point support for a single point.
void block_rhs(const std::vector<std::array<double, 3>>& pts, const std::vector<Sample>& smp, const Variogram& vg,
               std::vector<double>& rhs, double& cbb) {
  double np = double(pts.size());
  rhs.assign(smp.size(), 0.0);
  for (size_t i = 0; i < smp.size(); ++i) {
    double sum = -0.0;
    for (auto& p : pts)
      sum = sum + (pts.size() == 1 ? vg.cov_points(smp[i].loc, p.data()) : vg.block_cov_points(smp[i].loc, p.data()));
    rhs[i] = sum / np;
  }
  cbb = vg.block_mean_cov(pts);
}

// block.rs:120-198 (block_krige_points, Kind::Ordinary as Method::Block calls
// it, crates/py/src/estimation.rs:775-784), with the coincident guard of
// coincident.rs:27-111 as in krige().
int block_krige_points(const std::vector<std::array<double, 3>>& pts, const std::vector<Sample>& smp,
                       const Variogram& vg, Estimate& out) {
  size_t n = smp.size();
  if (n == 0) return INSUFFICIENT;
  if (pts.empty()) return INVALID;
  for (auto& p : pts)
    if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2])) return INVALID;
  bool any = false;
  for (size_t i = 0; i < n && !any; ++i)
    for (size_t j = 0; j < i; ++j)
      if (close(smp[i].loc, smp[j].loc)) { any = true; break; }
  if (any) {
    std::vector<size_t> of;
    std::vector<std::vector<size_t>> members;
    for (size_t i = 0; i < n; ++i) {
      size_t c = members.size();
      for (size_t m = 0; m < members.size(); ++m)
        if (close(smp[members[m][0]].loc, smp[i].loc)) { c = m; break; }
      if (c == members.size()) members.push_back({i});
      else members[c].push_back(i);
      of.push_back(c);
    }
    double c0 = vg.total_sill();
    std::vector<Sample> merged;
    for (auto& m : members) {
      Sample first = smp[m[0]];
      if (m.size() > 1) {
        double k = double(m.size());
        double var = 0.0;
        for (size_t i : m) {
          var += smp[i].err;
          for (size_t j : m) var += vg.cov_points(smp[i].loc, smp[j].loc);
        }
        double vs = -0.0;
        for (size_t i : m) vs = vs + smp[i].value;
        first.value = vs / k;
        first.err = var / (k * k) - c0;
      }
      merged.push_back(first);
    }
    Estimate e;
    int st = block_krige_points(pts, merged, vg, e);
    if (st != OK) return st;
    std::vector<double> w(n);
    for (size_t i = 0; i < n; ++i) w[i] = e.weights[of[i]] / double(members[of[i]].size());
    e.weights = w;
    e.value = kind_value(ORDINARY, 0.0, w, smp);
    e.n_used = n;
    out = e;
    return OK;
  }
  std::vector<double> rhs;
  double cbb;
  block_rhs(pts, smp, vg, rhs, cbb);
  size_t dim = n + 1;
  std::vector<double> A(dim * dim, 0.0), b(dim, 0.0);
  for (size_t i = 0; i < n; ++i) {
    for (size_t j = 0; j < n; ++j) A[i * dim + j] = vg.cov_points(smp[i].loc, smp[j].loc);
    A[i * dim + i] += smp[i].err;
    A[i * dim + n] = 1.0, A[n * dim + i] = 1.0;
    b[i] = rhs[i];
  }
  b[n] = 1.0;
  std::vector<double> x = b;
  if (!lu_solve(A, dim, x)) return SINGULAR;
  out.weights.assign(x.begin(), x.begin() + n);
  double value = -0.0;
  for (size_t i = 0; i < n; ++i) value = value + out.weights[i] * smp[i].value;
  double swc = -0.0;
  for (size_t i = 0; i < n; ++i) swc = swc + out.weights[i] * b[i];
  double mu = x[n];
  out.value = value;
  out.variance = std::fmax(cbb - swc - mu, 0.0);
  out.n_used = n;
  out.lagrange = mu;
  out.support = cbb;
  return OK;
}

// ---------------------------------------------------------------- search
struct SearchP {
  size_t min_samples = 4, max_samples = 16;
  double radius = INFINITY;
  int64_t max_per_hole = -1;  // -1 = None
  bool octant = false;
  int64_t sectors = 0, max_per_sector = 0;  // plane sectors; 0 = None
  Aniso aniso;
  int64_t max_per_octant = -1, min_sectors = -1, max_empty_sectors = -1, min_holes = -1;
  int calibration = 0;  // search.rs:94-100: 0 none, 1 Slope(target), 2 Efficiency(target)
  double target = 0.0;
  bool balances() const { return octant || sectors > 0; }
};

// crates/estimation/src/search.rs:214-264
bool check(const SearchP& p) {
  if (std::isnan(p.radius) || p.radius <= 0.0 || p.max_samples == 0 || p.min_samples > p.max_samples)
    return false;
  size_t count = 0, ring = 0;
  if (p.sectors > 0) {
    if (p.octant) return false;
    if (!(p.sectors >= 2 && p.sectors <= 360) || p.max_per_sector == 0) return false;
    count = ring = size_t(p.sectors);
  } else if (p.octant) count = 8, ring = 4;
  if (p.max_per_octant >= 0) {
    if (!p.octant) return false;
    if (p.max_per_octant == 0) return false;
  }
  bool rules = p.min_sectors >= 0 || p.max_empty_sectors >= 0;
  if (rules && !p.balances()) return false;
  if (p.min_sectors >= 0 &&
      (p.min_sectors == 0 || size_t(p.min_sectors) > count || size_t(p.min_sectors) > p.max_samples))
    return false;
  if (p.max_empty_sectors >= 0 && size_t(p.max_empty_sectors) >= ring) return false;
  if (p.min_holes >= 0 && (p.min_holes == 0 || size_t(p.min_holes) > p.max_samples)) return false;
  return true;
}

// grid.rs:109-111
double d2f(const double* p, const double* q) { return p2(p[0] - q[0]) + p2(p[1] - q[1]) + p2(p[2] - q[2]); }

uint64_t bits(double x) { uint64_t b; std::memcpy(&b, &x, 8); return b; }

int64_t f2i(double x) {  // Rust `as i64`: saturating, NaN -> 0
  if (std::isnan(x)) return 0;
  if (x >= 9.2233720368547758e18) return std::numeric_limits<int64_t>::max();
  if (x <= -9.2233720368547758e18) return std::numeric_limits<int64_t>::min();
  return int64_t(x);
}

// search.rs:704-745
struct Space {
  M3 frame = identity();
  bool has_origin = false;
  double origin[3] = {0, 0, 0};
  void project(const double p[3], double out[3]) const {
    double d[3] = {p[0] - origin[0], p[1] - origin[1], p[2] - origin[2]};
    mulv(frame, d, out);
  }
};

Space make_space(const Aniso* a, const std::vector<Sample>& s) {
  Space sp;
  sp.frame = a ? aniso_matrix(*a) : identity();
  for (auto& x : s)
    if (std::isfinite(x.loc[0]) && std::isfinite(x.loc[1]) && std::isfinite(x.loc[2])) {
      sp.has_origin = true;
      std::memcpy(sp.origin, x.loc, sizeof sp.origin);
      break;
    }
  return sp;
}

// search.rs:395-467
struct Sectors {
  M3 axes = identity();
  bool planar = false;
  int64_t plane = 0;
  size_t count() const { return plane > 0 ? size_t(plane) : (planar ? 4 : 8); }
  size_t of(const double t[3], const double s[3]) const {
    double v[3] = {s[0] - t[0], s[1] - t[1], s[2] - t[2]}, d[3];
    mulv(axes, v, d);
    if (plane > 0) {
      double turn = std::fmod(std::atan2(-d[0], d[1]), kTau);
      if (turn < 0.0) turn = turn + kTau;
      double x = turn / kTau * double(plane);
      size_t k = std::isnan(x) ? 0 : size_t(std::max(x, 0.0));
      return std::min(k, size_t(plane) - 1);
    }
    size_t bx = d[0] >= 0.0, by = d[1] >= 0.0, bz = d[2] >= 0.0;
    return planar ? (bx << 1) | by : (bx << 2) | (by << 1) | bz;
  }
  size_t longest_empty(const std::vector<size_t>& counts) const {
    std::vector<std::vector<size_t>> rings;
    if (plane > 0) {
      std::vector<size_t> r;
      for (int64_t i = 0; i < plane; ++i) r.push_back(size_t(i));
      rings.push_back(r);
    } else if (planar) rings = {{3, 1, 0, 2}};
    else rings = {{7, 3, 1, 5}, {6, 2, 0, 4}};
    size_t best = 0;
    for (auto& ring : rings) {
      bool all = true;
      for (size_t s : ring) all = all && counts[s] == 0;
      if (all) { best = std::max(best, ring.size()); continue; }
      size_t run = 0, longest = 0;
      for (int pass = 0; pass < 2; ++pass)
        for (size_t s : ring) { run = counts[s] == 0 ? run + 1 : 0; longest = std::max(longest, run); }
      best = std::max(best, longest);
    }
    return best;
  }
};

Sectors make_sectors(const Aniso* a, bool planar, const SearchP& p) {
  Sectors s;
  s.axes = a ? block_frame(a->azimuth, a->dip, a->rake) : identity();
  s.planar = planar;
  s.plane = p.sectors;
  return s;
}

// search.rs:476-577
struct Selector {
  const double* target;
  const SearchP* p;
  const Sectors* sec;
  std::vector<size_t> chosen;
  std::vector<std::pair<int64_t, size_t>> per_hole;
  size_t untagged = 0;
  std::vector<size_t> per_sector;
  size_t cap;
  Selector(const double* t, const SearchP& params, const Sectors& s) : target(t), p(&params), sec(&s) {
    per_sector.assign(params.balances() ? s.count() : 0, 0);
    if (params.sectors > 0) cap = size_t(params.max_per_sector);
    else if (params.octant)
      cap = params.max_per_octant >= 0 ? size_t(params.max_per_octant)
                                       : (params.max_samples + s.count() - 1) / s.count();
    else cap = std::numeric_limits<size_t>::max();
  }
  bool full() const { return chosen.size() >= p->max_samples; }
  bool offer(size_t idx, const double* loc, int64_t hole) {
    if (full()) return true;
    int64_t seen = -1;
    if (hole >= 0)
      for (size_t k = 0; k < per_hole.size(); ++k) if (per_hole[k].first == hole) { seen = int64_t(k); break; }
    if (p->max_per_hole >= 0 && seen >= 0 && per_hole[size_t(seen)].second >= size_t(p->max_per_hole)) return false;
    if (p->balances()) {
      size_t o = sec->of(target, loc);
      if (per_sector[o] >= cap) return false;
      per_sector[o] += 1;
    }
    if (hole >= 0 && seen >= 0) per_hole[size_t(seen)].second += 1;
    else if (hole >= 0) per_hole.push_back({hole, 1});
    else untagged += 1;
    chosen.push_back(idx);
    return full();
  }
  bool finish() const {
    if (chosen.size() < p->min_samples) return false;
    if (p->min_sectors >= 0) {
      size_t held = 0;
      for (size_t c : per_sector) held += c > 0;
      if (held < size_t(p->min_sectors)) return false;
    }
    if (p->max_empty_sectors >= 0 && sec->longest_empty(per_sector) > size_t(p->max_empty_sectors)) return false;
    if (p->min_holes >= 0 && per_hole.size() + untagged < size_t(p->min_holes)) return false;
    return true;
  }
};

bool planar_locs(const std::vector<Sample>& s) {  // search.rs:470-473
  if (s.empty()) return true;
  for (auto& x : s) if (!(x.loc[2] == s[0].loc[2])) return false;
  return true;
}

const Aniso* metric(const SearchP& p, const Variogram* vg) {  // search.rs:343-348
  if (p.aniso.on) return &p.aniso;
  if (vg && vg->aniso.on) return &vg->aniso;
  return nullptr;
}

// ---------------------------------------------------- grid (search/grid.rs)
constexpr int64_t REACH = 12;

struct Table { std::vector<std::array<int64_t, 3>> offsets; std::vector<std::pair<uint64_t, size_t>> shells; };

const Table& table() {  // grid.rs:39-64
  static Table t = [] {
    std::vector<std::pair<uint64_t, std::array<int64_t, 3>>> keyed;
    for (int64_t x = -REACH; x <= REACH; ++x)
      for (int64_t y = -REACH; y <= REACH; ++y)
        for (int64_t z = -REACH; z <= REACH; ++z) {
          std::array<int64_t, 3> o = {x, y, z};
          uint64_t m = 0;
          for (int64_t v : o) { uint64_t a = uint64_t(std::max<int64_t>(std::llabs(v) - 1, 0)); m += a * a; }
          keyed.push_back({m, o});
        }
    std::sort(keyed.begin(), keyed.end());
    Table tb;
    for (size_t k = 0; k < keyed.size(); ++k) {
      if (!tb.shells.empty() && tb.shells.back().first == keyed[k].first) tb.shells.back().second = k + 1;
      else tb.shells.push_back({keyed[k].first, k + 1});
      tb.offsets.push_back(keyed[k].second);
    }
    return tb;
  }();
  return t;
}

struct Entry { double p[3]; uint32_t i; };
using HeapItem = std::pair<uint64_t, uint32_t>;
using Heap = std::priority_queue<HeapItem, std::vector<HeapItem>, std::greater<HeapItem>>;

struct Grid {
  double lo[3], hi[3], h;
  int64_t dims[3];
  std::vector<uint32_t> start;
  std::vector<Entry> entries;

  static void bounds(const std::vector<std::array<double, 3>>& pts, double lo[3], double hi[3]) {  // :66-79
    for (int d = 0; d < 3; ++d) lo[d] = INFINITY, hi[d] = -INFINITY;
    for (auto& p : pts) {
      if (!(std::isfinite(p[0]) && std::isfinite(p[1]) && std::isfinite(p[2]))) continue;
      for (int d = 0; d < 3; ++d) { lo[d] = std::fmin(lo[d], p[d]); hi[d] = std::fmax(hi[d], p[d]); }
    }
    if (!(lo[0] <= hi[0])) for (int d = 0; d < 3; ++d) lo[d] = hi[d] = 0.0;
  }
  static double side(const double lo[3], const double hi[3], size_t n) {  // :83-106
    double ext[3];
    for (int d = 0; d < 3; ++d) ext[d] = hi[d] - lo[d];
    double longest = 0.0;
    for (double e : ext) longest = std::fmax(longest, e);
    if (longest <= 0.0) return 1.0;
    double prod = 1.0;
    int cnt = 0;
    for (double e : ext) if (e > longest * 1e-9) { prod = prod * e; cnt++; }
    double h = std::pow(prod / double(std::max<size_t>(n, 1)), 1.0 / double(cnt));
    auto cells = [&](double hh) {
      double c = 1.0;
      for (double e : ext) c = c * (std::floor(e / hh) + 1.0);
      return c;
    };
    while (cells(h) > 4.0 * double(n) + 64.0) h *= 2.0;
    return h;
  }
  void cell(const double p[3], int64_t c[3]) const {  // :196-200
    for (int d = 0; d < 3; ++d)
      c[d] = std::min(std::max(f2i(std::floor((p[d] - lo[d]) / h)), int64_t(0)), dims[d] - 1);
  }
  size_t id(const int64_t c[3]) const { return size_t(c[0] + dims[0] * (c[1] + dims[1] * c[2])); }

  void build(const std::vector<std::array<double, 3>>& pts) {  // :130-168
    bounds(pts, lo, hi);
    h = side(lo, hi, pts.size());
    for (int d = 0; d < 3; ++d) dims[d] = f2i(std::floor((hi[d] - lo[d]) / h)) + 1;
    size_t cells = size_t(dims[0] * dims[1] * dims[2]);
    std::vector<size_t> ids(pts.size());
    for (size_t i = 0; i < pts.size(); ++i) { int64_t c[3]; cell(pts[i].data(), c); ids[i] = id(c); }
    start.assign(cells + 1, 0);
    for (size_t c : ids) start[c + 1] += 1;
    for (size_t c = 0; c < cells; ++c) start[c + 1] += start[c];
    std::vector<uint32_t> fill(start);
    entries.assign(pts.size(), Entry{});
    for (size_t i = 0; i < pts.size(); ++i) {
      Entry e;
      std::memcpy(e.p, pts[i].data(), sizeof e.p);
      e.i = uint32_t(i);
      entries[fill[ids[i]]++] = e;
    }
  }
  void scan(const int64_t c[3], const double q[3], double radius2, Heap& heap) const {  // :367-380
    for (int d = 0; d < 3; ++d) if (c[d] < 0 || c[d] >= dims[d]) return;
    size_t k = id(c);
    for (uint32_t e = start[k]; e < start[k + 1]; ++e) {
      double dd = d2f(entries[e].p, q);
      if (dd <= radius2) heap.push({bits(dd), entries[e].i});
    }
  }
  void ring(const int64_t c[3], int64_t r, const double q[3], double radius2, Heap& heap) const {  // :348-365
    auto lo_ = [&](int d) { return std::max(-r, -c[d]); };
    auto hi_ = [&](int d) { return std::min(r, dims[d] - 1 - c[d]); };
    for (int64_t x = lo_(0); x <= hi_(0); ++x)
      for (int64_t y = lo_(1); y <= hi_(1); ++y) {
        std::vector<int64_t> zs;
        if (std::llabs(x) == r || std::llabs(y) == r) { for (int64_t z = lo_(2); z <= hi_(2); ++z) zs.push_back(z); }
        else { for (int64_t z : {-r, r}) if (z >= lo_(2) && z <= hi_(2)) zs.push_back(z); }
        for (int64_t z : zs) { int64_t cc[3] = {c[0] + x, c[1] + y, c[2] + z}; scan(cc, q, radius2, heap); }
      }
  }
  template <class F> static bool release(Heap& heap, double bound, F& visit) {  // :115-127
    while (!heap.empty()) {
      HeapItem top = heap.top();
      double dd;
      std::memcpy(&dd, &top.first, 8);
      if (dd >= bound) return false;
      heap.pop();
      if (visit(dd, size_t(top.second))) return true;
    }
    return false;
  }
  template <class F> void nearest(const double q[3], double radius2, F visit) const {  // :209-255
    const Table& tb = table();
    int64_t c[3];
    cell(q, c);
    double h2 = h * h;
    double beyond = h2 * double((REACH - 1) * (REACH - 1));
    Heap heap;
    size_t begin = 0;
    for (auto& sh : tb.shells) {
      double bound = std::fmin(h2 * double(sh.first), beyond) * (1.0 - 1e-9);
      if (bound > radius2) break;
      if (release(heap, bound, visit)) return;
      for (size_t k = begin; k < sh.second; ++k) {
        int64_t cc[3] = {c[0] + tb.offsets[k][0], c[1] + tb.offsets[k][1], c[2] + tb.offsets[k][2]};
        scan(cc, q, radius2, heap);
      }
      begin = sh.second;
    }
    int64_t far = 0;
    for (int d = 0; d < 3; ++d) far = std::max(far, std::max(c[d], dims[d] - 1 - c[d]));
    for (int64_t r = REACH + 1; r <= far; ++r) {
      double bound = p2(double(r - 1) * h) * (1.0 - 1e-9);
      if (bound > radius2) break;
      if (release(heap, bound, visit)) return;
      ring(c, r, q, radius2, heap);
    }
    release(heap, INFINITY, visit);
  }
};

// search.rs:692-776, 951-1005: the tree used by estimate_many
struct Tree {
  Grid grid;
  Space space;
  std::vector<std::array<double, 3>> points;
  const std::vector<Sample>* samples;
  SearchP params;
  Sectors sectors;

  Tree(const std::vector<Sample>& s, const SearchP& p, const Variogram* vg) : samples(&s), params(p) {
    const Aniso* a = metric(p, vg);
    space = make_space(a, s);
    sectors = make_sectors(a, planar_locs(s), p);
    points.resize(s.size());
    for (size_t i = 0; i < s.size(); ++i) space.project(s[i].loc, points[i].data());
    grid.build(points);
  }

  // search.rs:269-288 (Search::admits) with hard domain boundaries (no soft
  // distance) and no high-grade rule: a sample of another domain than the
  // target's never informs it; an untagged target or sample is admitted.
  static bool admits(int64_t tdomain, int64_t sdomain) { return tdomain < 0 || sdomain < 0 || tdomain == sdomain; }

  // search.rs:597-632 (one_per_location): samples at one location (the
  // coordinates' bits, -0 as 0) reduced to the first, replaced by the first
  // one of the target's domain if it is not; nothing changes without a
  // target domain.
  std::vector<size_t> one_per_location(const std::vector<size_t>& ordered, int64_t tdomain) const {
    if (tdomain < 0) return ordered;
    std::vector<size_t> out;
    std::vector<std::array<uint64_t, 3>> keys;
    for (size_t i : ordered) {
      std::array<uint64_t, 3> k;
      for (int a = 0; a < 3; ++a) {
        const double v = (*samples)[i].loc[a] + 0.0;
        std::memcpy(&k[a], &v, sizeof(double));
      }
      size_t at = keys.size();
      for (size_t j = 0; j < keys.size(); ++j)
        if (keys[j] == k) { at = j; break; }
      if (at == keys.size()) {
        keys.push_back(k);
        out.push_back(i);
      } else if ((*samples)[out[at]].domain != tdomain && (*samples)[i].domain == tdomain) {
        out[at] = i;
      }
    }
    return out;
  }

  // search.rs:951-1005 (neighbors_around): the (d2, index) stream of the grid
  // is offered in groups of equal d2, each reduced to the admitted samples
  // (without `left_out`) and one per location.
  bool neighbors(const double t[3], int64_t left_out, std::vector<size_t>& out, int64_t tdomain = -1) const {
    Selector sel(t, params, sectors);
    if (!samples->empty() && params.max_samples > 0) {
      double q[3];
      space.project(t, q);
      std::vector<size_t> group;
      double at = NAN;
      bool full = false;
      auto offer = [&]() {
        std::vector<size_t> admitted;
        for (size_t i : group)
          if (int64_t(i) != left_out && admits(tdomain, (*samples)[i].domain)) admitted.push_back(i);
        group.clear();
        for (size_t i : one_per_location(admitted, tdomain))
          if (sel.offer(i, (*samples)[i].loc, (*samples)[i].hole)) return true;
        return false;
      };
      grid.nearest(q, params.radius * params.radius, [&](double d2, size_t i) {
        if (d2 != at && !group.empty()) {
          full = offer();
          if (full) return true;
        }
        at = d2;
        group.push_back(i);
        return false;
      });
      if (!full) offer();
    }
    out = sel.chosen;
    return sel.finish();
  }
};

// search.rs:647-687: linear scan, the reference for the tree
bool scan_neighbors(const double t[3], const std::vector<Sample>& s, const SearchP& p, const Variogram* vg,
                    std::vector<size_t>& out) {
  const Aniso* a = metric(p, vg);
  Space sp = make_space(a, s);
  double q[3];
  sp.project(t, q);
  double radius2 = p.radius * p.radius;
  std::vector<std::pair<double, size_t>> cand;
  for (size_t i = 0; i < s.size(); ++i) {
    double pp[3];
    sp.project(s[i].loc, pp);
    double dd = d2f(pp, q);
    if (dd <= radius2) cand.push_back({dd, i});
  }
  std::stable_sort(cand.begin(), cand.end(), [](auto& x, auto& y) { return x.first < y.first; });
  Sectors sec = make_sectors(a, p.octant && planar_locs(s), p);
  Selector sel(t, p, sec);
  for (auto& c : cand) if (sel.offer(c.second, s[c.second].loc, s[c.second].hole)) break;
  out = sel.chosen;
  return sel.finish();
}

// crates/estimation/src/search.rs:913-936 (SearchTree::balanced): with a
// calibration and octants or sectors, the chosen samples go round-robin over
// the sectors, each sector in selection order: a stable sort by the rank of
// each sample within its sector.
std::vector<size_t> balanced(const Tree& tree, const double t[3], const std::vector<size_t>& chosen) {
  if (!tree.params.balances() || tree.params.calibration == 0) return chosen;
  std::vector<size_t> seen(tree.sectors.count(), 0);
  std::vector<std::pair<size_t, size_t>> ranked;
  for (size_t i : chosen) {
    size_t o = tree.sectors.of(t, (*tree.samples)[i].loc);
    seen[o] += 1;
    ranked.push_back({seen[o], i});
  }
  std::stable_sort(ranked.begin(), ranked.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
  std::vector<size_t> out;
  for (auto& r : ranked) out.push_back(r.second);
  return out;
}

// crates/estimation/src/kriging_algebra.rs:336-395 (prefix_quality) for the
// drifts of ordinary kriging (one column of ones, x0 = 1) and simple kriging
// (none). nalgebra's Cholesky (column j from the columns before it by axpy,
// then sqrt of a positive diagonal and a division) of the covariance matrix
// serves every leading part; its lower solves are column sweeps. Entry k is
// the slope and efficiency from the first k + 1 samples; ok[k] = 0 for None.
void prefix_quality(const std::vector<Sample>& smp, const Variogram& vg, const std::vector<double>& rhs,
                    bool ordinary, double support, std::vector<double>& slope, std::vector<double>& eff,
                    std::vector<int>& ok) {
  const size_t n = smp.size();
  slope.assign(n, NAN), eff.assign(n, NAN), ok.assign(n, 0);
  std::vector<double> L(n * n, 0.0);  // column-major, as nalgebra stores it
  auto at = [&](size_t i, size_t j) -> double& { return L[j * n + i]; };
  for (size_t j = 0; j < n; ++j)
    for (size_t i = 0; i < n; ++i) at(i, j) = vg.cov_points(smp[i].loc, smp[j].loc) + (i == j ? smp[i].err : 0.0);
  for (size_t j = 0; j < n; ++j) {
    for (size_t k = 0; k < j; ++k) {
      const double factor = -at(j, k);
      for (size_t i = j; i < n; ++i) at(i, j) = factor * at(i, k) + at(i, j);
    }
    const double diag = at(j, j);
    if (!(diag > 0.0)) return;  // not positive definite: every entry None
    const double denom = std::sqrt(diag);
    at(j, j) = denom;
    for (size_t i = j + 1; i < n; ++i) at(i, j) = at(i, j) / denom;
  }
  std::vector<double> y = rhs, z(n, 1.0);
  for (size_t i = 0; i < n; ++i) {  // solve_lower_triangular, column by column
    const double cy = y[i] / at(i, i), cz = z[i] / at(i, i);
    y[i] = cy, z[i] = cz;
    for (size_t r = i + 1; r < n; ++r) y[r] = (-cy) * at(r, i) + y[r], z[r] = (-cz) * at(r, i) + z[r];
  }
  double sy = 0.0, a = 0.0, b = 0.0;
  for (size_t k = 0; k < n; ++k) {
    sy += y[k] * y[k];
    double cov = sy, mu = 0.0;
    if (ordinary) {
      a = a + z[k] * z[k];
      b = b + z[k] * y[k];
      if (!(a > 0.0)) continue;
      const double l = std::sqrt(a);  // the 1 x 1 Cholesky factor and its solve
      const double m = ((b - 1.0) / l) / l;
      cov = sy - m * b;
      mu = m * 1.0;
    }
    slope[k] = cov / (cov - mu);
    eff[k] = (cov + mu) / support;
    ok[k] = 1;
  }
}

// kriging_algebra.rs:397-412 (calibrated_count): the fewest leading samples,
// from min_samples, whose quality meets the calibration (met = 1), or all.
size_t calibrated_count(const SearchP& p, const std::vector<double>& slope, const std::vector<double>& eff,
                        const std::vector<int>& ok, int* met) {
  const size_t from = std::max<size_t>(p.min_samples, 1);
  for (size_t k = from - 1; k < ok.size(); ++k) {
    if (!ok[k]) continue;
    const bool meets = p.calibration == 1 ? slope[k] >= p.target : eff[k] >= p.target;
    if (meets) { *met = 1; return k + 1; }
  }
  *met = 0;
  return ok.size();
}

// crates/py/src/estimation.rs:846-895 (Method::calibrated) for the kriging
// kinds and block kriging: the samples a calibrated search keeps, in place.
// `rhs` holds each sample's covariance with the target's support.
int calibrate(const SearchP& p, const Variogram& vg, int kind, const std::vector<double>& rhs, double support,
              std::vector<Sample>& sel) {
  if (p.calibration == 0) return -1;
  std::vector<double> slope, eff;
  std::vector<int> ok;
  prefix_quality(sel, vg, rhs, kind != SIMPLE, support, slope, eff, ok);
  int met = 0;
  sel.resize(calibrated_count(p, slope, eff, ok, &met));
  return met;
}

}  // namespace

// ===================================================================== C ABI
extern "C" {

struct orc_structure { int32_t model; double param, sill, range; };
struct orc_aniso { int32_t on; double azimuth, dip, rake, major, semi, minor; };
struct orc_variogram { double nugget; int32_t nstruct; orc_structure s[4]; orc_aniso aniso; };
struct orc_search {
  int64_t min_samples, max_samples;
  double radius;
  int64_t max_per_hole, octant, sectors, max_per_sector, max_per_octant, min_sectors,
      max_empty_sectors, min_holes;
  orc_aniso aniso;
  int64_t calibration;  // 0 none, 1 slope, 2 efficiency
  double calibration_target;
};
struct orc_result { double value, variance, lagrange, support; int64_t n_used; int32_t status; };

static Aniso conv_aniso(const orc_aniso& a) {
  if (!a.on) return Aniso{};
  return make_aniso(a.azimuth, a.dip, a.rake, a.major, a.semi, a.minor);
}
static Variogram conv_vg(const orc_variogram* v) {
  Variogram g;
  g.nugget = v->nugget;
  for (int k = 0; k < v->nstruct; ++k) g.s.push_back({v->s[k].model, v->s[k].param, v->s[k].sill, v->s[k].range});
  g.aniso = conv_aniso(v->aniso);
  return g;
}
static SearchP conv_search(const orc_search* s) {
  SearchP p;
  p.min_samples = size_t(s->min_samples);
  p.max_samples = size_t(s->max_samples);
  p.radius = s->radius;
  p.max_per_hole = s->max_per_hole;
  p.octant = s->octant != 0;
  p.sectors = s->sectors;
  p.max_per_sector = s->max_per_sector;
  p.max_per_octant = s->max_per_octant;
  p.min_sectors = s->min_sectors;
  p.max_empty_sectors = s->max_empty_sectors;
  p.min_holes = s->min_holes;
  p.aniso = conv_aniso(s->aniso);
  p.calibration = int(s->calibration);
  p.target = s->calibration_target;
  return p;
}
static std::vector<Sample> conv_samples(int64_t n, const double* xyz, const double* v, const double* err,
                                        const int64_t* hole) {
  std::vector<Sample> s(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) {
    s[i].loc[0] = xyz[3 * i], s[i].loc[1] = xyz[3 * i + 1], s[i].loc[2] = xyz[3 * i + 2];
    s[i].value = v ? v[i] : 0.0;
    s[i].err = err ? err[i] : 0.0;
    s[i].hole = hole ? hole[i] : -1;
  }
  return s;
}
static void put(const Estimate& e, int st, orc_result* r) {
  r->status = st;
  if (st == OK) {
    r->value = e.value, r->variance = e.variance, r->lagrange = e.lagrange, r->support = e.support;
    r->n_used = int64_t(e.n_used);
  } else {
    r->value = r->variance = r->lagrange = r->support = NAN;
    r->n_used = 0;
  }
}

int orc_num_threads(void) { return int(std::max(1u, std::thread::hardware_concurrency())); }

void orc_rotation_matrix(double az, double dip, double rake, double* out9) {
  M3 r = rotation_matrix(az, dip, rake);
  for (int i = 0; i < 9; ++i) out9[i] = r.m[i / 3][i % 3];
}
void orc_block_frame(double az, double dip, double rake, double* out9) {
  M3 r = block_frame(az, dip, rake);
  for (int i = 0; i < 9; ++i) out9[i] = r.m[i / 3][i % 3];
}
void orc_aniso_matrix(const orc_aniso* a, double* out9) {
  M3 r = aniso_matrix(conv_aniso(*a));
  for (int i = 0; i < 9; ++i) out9[i] = r.m[i / 3][i % 3];
}
double orc_shape(int32_t model, double param, double h, double range) { return shape(model, param, h, range); }
double orc_shape_d1(int32_t model, double param, double h, double range) { return shape_d1(model, param, h, range); }
double orc_cov(const orc_variogram* v, double h) { return conv_vg(v).cov(h); }
double orc_cov_points(const orc_variogram* v, const double* p, const double* q) { return conv_vg(v).cov_points(p, q); }
int32_t orc_check_search(const orc_search* s) { return check(conv_search(s)) ? 1 : 0; }

// which: 0 = krige (guard + kernel + LU), 1 = kernel only (-1 when beyond it), 2 = LU only
int32_t orc_krige(int32_t which, int32_t kind, double kparam, const double* t, int64_t n, const double* xyz,
                  const double* v, const double* err, const orc_variogram* vgp, orc_result* res, double* weights) {
  Variogram vg = conv_vg(vgp);
  std::vector<Sample> s = conv_samples(n, xyz, v, err, nullptr);
  Estimate e;
  int st = which == 0 ? krige(kind, kparam, t, s, vg, e)
                      : (which == 1 ? kernel_krige(kind, kparam, t, s, vg, e) : krige_lu(kind, kparam, t, s, vg, e));
  put(e, st, res);
  if (st == OK && weights) std::copy(e.weights.begin(), e.weights.end(), weights);
  return st;
}

// prefix_quality (kriging_algebra.rs:336-395) of n samples around t with the
// ordinary (1) or simple (0) drift and support variance `support`: slope,
// efficiency and ok (0 for None) per leading part.
void orc_prefix_quality(int64_t n, const double* xyz, const double* err, const double* t, const orc_variogram* vgp,
                        int32_t ordinary, double support, double* slope, double* eff, int32_t* ok) {
  Variogram vg = conv_vg(vgp);
  std::vector<Sample> s = conv_samples(n, xyz, nullptr, err, nullptr);
  std::vector<double> rhs, sl, ef;
  for (auto& x : s) rhs.push_back(vg.cov_points(x.loc, t));
  std::vector<int> k;
  prefix_quality(s, vg, rhs, ordinary != 0, support, sl, ef, k);
  for (int64_t i = 0; i < n; ++i) slope[i] = sl[i], eff[i] = ef[i], ok[i] = k[i];
}

// Brute-force (d2 bits, index) stream of the grid, for the grid tests:
// writes every index within radius2 of q in visit order; returns the count.
int64_t orc_grid_visit(int64_t n, const double* pts, const double* q, double radius2, int64_t* out_idx,
                       uint64_t* out_bits, int64_t stop_after) {
  std::vector<std::array<double, 3>> p(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) p[i] = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
  Grid g;
  g.build(p);
  int64_t k = 0;
  g.nearest(q, radius2, [&](double dd, size_t i) {
    out_idx[k] = int64_t(i);
    out_bits[k] = bits(dd);
    ++k;
    return stop_after > 0 && k >= stop_after;
  });
  return k;
}

void* orc_tree_new(int64_t n, const double* xyz, const int64_t* hole, const orc_search* sp, const orc_variogram* vgp) {
  auto* s = new std::vector<Sample>(conv_samples(n, xyz, nullptr, nullptr, hole));
  Variogram* vg = vgp ? new Variogram(conv_vg(vgp)) : nullptr;
  Tree* t = new Tree(*s, conv_search(sp), vg);
  delete vg;
  struct Box { std::vector<Sample>* s; Tree* t; };
  return new Box{s, t};
}
void orc_tree_free(void* h) {
  struct Box { std::vector<Sample>* s; Tree* t; };
  auto* b = static_cast<Box*>(h);
  delete b->t;
  delete b->s;
  delete b;
}
// Returns 1 when the search succeeds, 0 when it fails; `out` gets the chosen
// indices in selection order either way (count in *nout).
int32_t orc_tree_neighbors(void* h, const double* t, int64_t left_out, int64_t* out, int64_t* nout) {
  struct Box { std::vector<Sample>* s; Tree* t; };
  auto* b = static_cast<Box*>(h);
  std::vector<size_t> c;
  bool ok = b->t->neighbors(t, left_out, c);
  for (size_t k = 0; k < c.size(); ++k) out[k] = int64_t(c[k]);
  *nout = int64_t(c.size());
  return ok ? 1 : 0;
}
int32_t orc_scan_neighbors(int64_t n, const double* xyz, const int64_t* hole, const orc_search* sp,
                           const orc_variogram* vgp, const double* t, int64_t* out, int64_t* nout) {
  std::vector<Sample> s = conv_samples(n, xyz, nullptr, nullptr, hole);
  Variogram vg;
  if (vgp) vg = conv_vg(vgp);
  std::vector<size_t> c;
  bool ok = scan_neighbors(t, s, conv_search(sp), vgp ? &vg : nullptr, c);
  for (size_t k = 0; k < c.size(); ++k) out[k] = int64_t(c[k]);
  *nout = int64_t(c.size());
  return ok ? 1 : 0;
}

// The per-target columns of the diagnostics table (crates/py/src/estimation.rs:
// 1046-1105) that need the samples used or the weights. neighborhood_stats
// (crates/estimation/src/neighborhood.rs:66-98), called with k = the samples
// used, radius = inf and no anisotropy (estimation.rs:1041): Euclidean
// distances (aniso.rs:114-119) sorted ascending (a stable sort), n_within,
// n_holes (a hole counted once, an untagged sample once each) and their mean;
// Estimate::negative_weight_sum (krige.rs:70-75). out[4] = {negative weight
// sum, mean distance, n_holes, n_within}.
static void diag_of(const double t[3], const std::vector<Sample>& sel, const Estimate& e, double* out) {
  std::vector<std::pair<double, int64_t>> d;
  d.reserve(sel.size());
  for (auto& x : sel) {
    double dx = x.loc[0] - t[0], dy = x.loc[1] - t[1], dz = x.loc[2] - t[2];
    d.push_back({std::sqrt(dx * dx + dy * dy + dz * dz), x.hole});
  }
  std::stable_sort(d.begin(), d.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
  const double radius = std::numeric_limits<double>::infinity();
  double within = 0.0, holes = 0.0, sum = 0.0;
  std::vector<int64_t> seen;
  for (auto& x : d) {
    if (!(x.first <= radius)) continue;
    within += 1.0;
    if (x.second < 0) {
      holes += 1.0;
    } else if (std::find(seen.begin(), seen.end(), x.second) == seen.end()) {
      seen.push_back(x.second);
      holes += 1.0;
    }
  }
  for (auto& x : d) sum += x.first;
  double neg = e.weights.empty() ? NAN : -0.0;
  for (double w : e.weights)
    if (w < 0.0) neg = neg + w;
  out[0] = neg;
  out[1] = d.empty() ? NAN : sum / double(d.size());
  out[2] = holes;
  out[3] = within;
}

// crates/estimation/src/batch.rs:15-38 (estimate_many) and :165-190
// (leave_one_out_at, when `loo` is set: targets are the samples themselves,
// each searched without itself). One result per target; `nbr` (optional,
// m x max_samples) receives the chosen indices, -1 padded; `diag` (optional,
// m x 5) the diagnostics columns of diag_of and target_met (1, 0; NaN without
// a calibration), NaN where a target is not estimated. A calibrated search
// orders the chosen samples with balanced and keeps the calibrated count. Threads take static chunks of targets, like rayon's per-target
// independence.
// With `sdomain` (the samples' domain codes, or null) each target krigs from
// its own domain, tdomain[k] (batch.rs:15-38 `domains`; the left-out
// sample's own with `loo`); a target code < 0 is a domain without samples,
// which the reference leaves unestimated (crates/py/src/estimation.rs:1655-
// 1657), here SEARCH_FAILED.
int32_t orc_estimate_many(int64_t m, const double* targets, int32_t loo, int64_t n, const double* xyz,
                          const double* v, const double* err, const int64_t* hole, const orc_search* sp,
                          const orc_variogram* vgp, int32_t kind, double kparam, int32_t nthreads,
                          orc_result* res, int64_t* nbr, double* diag, const int64_t* sdomain,
                          const int64_t* tdomain) {
  std::vector<Sample> s = conv_samples(n, xyz, v, err, hole);
  if (sdomain)
    for (int64_t i = 0; i < n; ++i) s[size_t(i)].domain = sdomain[i];
  SearchP p = conv_search(sp);
  if (!check(p)) return -1;
  Variogram vg = conv_vg(vgp);
  Tree tree(s, p, &vg);
  int64_t cnt = loo ? n : m;
  size_t maxs = p.max_samples;
  auto work = [&](int64_t k0, int64_t k1) {
    for (int64_t k = k0; k < k1; ++k) {
      const double* t = loo ? s[size_t(k)].loc : &targets[3 * k];
      const int64_t dom = !sdomain ? -1 : (loo ? sdomain[k] : tdomain[k]);
      std::vector<size_t> chosen;
      bool ok = sdomain && dom < 0 ? false : tree.neighbors(t, loo ? k : -1, chosen, dom);
      if (nbr) {
        for (size_t j = 0; j < maxs; ++j) nbr[size_t(k) * maxs + j] = j < chosen.size() ? int64_t(chosen[j]) : -1;
      }
      if (diag) for (int c = 0; c < 5; ++c) diag[5 * k + c] = NAN;
      if (!ok || (loo && chosen.empty())) { Estimate e; put(e, SEARCH_FAILED, &res[k]); continue; }
      std::vector<Sample> sel;
      sel.reserve(chosen.size());
      for (size_t i : balanced(tree, t, chosen)) sel.push_back(s[i]);
      int met = -1;
      if (p.calibration) {
        std::vector<double> rhs;
        for (auto& x : sel) rhs.push_back(vg.cov_points(x.loc, t));
        met = calibrate(p, vg, kind, rhs, vg.total_sill(), sel);
      }
      Estimate e;
      int st = krige(kind, kparam, t, sel, vg, e);
      put(e, st, &res[k]);
      if (diag && st == OK) {
        diag_of(t, sel, e, diag + 5 * k);
        diag[5 * k + 4] = met < 0 ? NAN : double(met);
      }
    }
  };
  int nt = nthreads > 0 ? nthreads : orc_num_threads();
  std::vector<std::thread> pool;
  int64_t chunk = (cnt + nt - 1) / nt;
  for (int w = 0; w < nt; ++w) {
    int64_t k0 = int64_t(w) * chunk, k1 = std::min(cnt, k0 + chunk);
    if (k0 < k1) pool.emplace_back(work, k0, k1);
  }
  for (auto& th : pool) th.join();
  return 0;
}

// crates/estimation/src/batch.rs:197-243 (k_fold_at over every sample): the
// j-th of the sorted hole ids goes to fold j % k and an untagged sample i to
// fold i % k; each fold's samples are kriged, each in its own domain, from a
// tree over the samples outside the fold (a new space, so a new origin).
int32_t orc_k_fold(int64_t k, int64_t n, const double* xyz, const double* v, const double* err, const int64_t* hole,
                   const int64_t* sdomain, const orc_search* sp, const orc_variogram* vgp, int32_t kind,
                   double kparam, orc_result* res) {
  if (k < 2) return -2;
  std::vector<Sample> s = conv_samples(n, xyz, v, err, hole);
  if (sdomain)
    for (int64_t i = 0; i < n; ++i) s[size_t(i)].domain = sdomain[i];
  SearchP p = conv_search(sp);
  if (!check(p)) return -1;
  Variogram vg = conv_vg(vgp);
  std::vector<int64_t> ids;
  for (auto& x : s)
    if (x.hole >= 0) ids.push_back(x.hole);
  std::sort(ids.begin(), ids.end());
  ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
  std::vector<int64_t> fold(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) {
    const int64_t h = s[size_t(i)].hole;
    const int64_t r = h < 0 ? i : int64_t(std::lower_bound(ids.begin(), ids.end(), h) - ids.begin());
    fold[size_t(i)] = r % k;
  }
  for (int64_t f = 0; f < k; ++f) {
    std::vector<Sample> train;
    for (int64_t i = 0; i < n; ++i)
      if (fold[size_t(i)] != f) train.push_back(s[size_t(i)]);
    Tree tree(train, p, &vg);
    for (int64_t i = 0; i < n; ++i) {
      if (fold[size_t(i)] != f) continue;
      const double* t = s[size_t(i)].loc;
      std::vector<size_t> chosen;
      Estimate e;
      if (!tree.neighbors(t, -1, chosen, sdomain ? s[size_t(i)].domain : -1) || chosen.empty()) {
        put(e, SEARCH_FAILED, &res[i]);
        continue;
      }
      std::vector<Sample> sel;
      for (size_t c : balanced(tree, t, chosen)) sel.push_back(train[c]);
      if (p.calibration) {
        std::vector<double> rhs;
        for (auto& x : sel) rhs.push_back(vg.cov_points(x.loc, t));
        calibrate(p, vg, kind, rhs, vg.total_sill(), sel);
      }
      put(e, krige(kind, kparam, t, sel, vg, e), &res[i]);
    }
  }
  return 0;
}

// crates/simulation/src/sgs.rs:586-760 (`sequential`), one node at a time:
// node j (in simulation order) is searched among the data and the nodes
// before it (a linear scan, which selects as the tree does, search.rs:647-
// 687), simple-kriged with mean 0 from their scores, and draws
// mean + sqrt(variance) * z[j]; a failed search draws z[j]. The node then
// joins the conditioning set as sample n_data + j, with no hole. how[j] = 1
// kriged, 2 marginal. Returns -1 - j when kriging node j fails.
int64_t orc_sgs(int64_t n_data, const double* xyz, const double* scores, const int64_t* hole, int64_t m,
                const double* nodes, const double* z, const orc_search* sp, const orc_variogram* vgp, double* out,
                int8_t* how) {
  std::vector<Sample> s = conv_samples(n_data, xyz, scores, nullptr, hole);
  SearchP p = conv_search(sp);
  Variogram vg = conv_vg(vgp);
  s.reserve(size_t(n_data + m));
  for (int64_t j = 0; j < m; ++j) {
    const double* t = &nodes[3 * j];
    std::vector<size_t> chosen;
    const bool ok = scan_neighbors(t, s, p, &vg, chosen);
    double score;
    if (!ok || chosen.empty()) {
      score = z[j];
      how[j] = 2;
    } else {
      std::vector<Sample> sel;
      for (size_t i : chosen) sel.push_back(s[i]);
      Estimate e;
      if (krige(SIMPLE, 0.0, t, sel, vg, e) != OK) return -1 - j;
      score = e.value + std::sqrt(std::fmax(e.variance, 0.0)) * z[j];
      how[j] = 1;
    }
    out[j] = score;
    Sample node;
    node.loc[0] = t[0], node.loc[1] = t[1], node.loc[2] = t[2];
    node.value = score, node.err = 0.0, node.hole = -1;
    s.push_back(node);
  }
  return 0;
}

// krige (krige.rs:83-95) of m targets from given neighbour lists (m x k,
// -1 padded): frozen neighbourhoods for the leave-one-out gradient checks.
// With skip_coincident, a system holding two samples within 1e-6 m gets
// status 5 and no estimate.
int32_t orc_krige_lists(int64_t m, const double* targets, int64_t n, const double* xyz, const double* v,
                        const double* err, const int64_t* nbr, int64_t k, const orc_variogram* vgp, int32_t kind,
                        double kparam, int32_t skip_coincident, orc_result* res) {
  std::vector<Sample> s = conv_samples(n, xyz, v, err, nullptr);
  Variogram vg = conv_vg(vgp);
  for (int64_t t = 0; t < m; ++t) {
    std::vector<Sample> sel;
    for (int64_t j = 0; j < k; ++j)
      if (nbr[t * k + j] >= 0) sel.push_back(s[size_t(nbr[t * k + j])]);
    Estimate e;
    if (sel.empty()) { put(e, SEARCH_FAILED, &res[t]); continue; }
    bool twins = false;
    for (size_t i = 0; i < sel.size() && !twins; ++i)
      for (size_t j = 0; j < i; ++j)
        if (close(sel[i].loc, sel[j].loc)) { twins = true; break; }
    if (skip_coincident && twins) { put(e, 5, &res[t]); continue; }
    int st = krige(kind, kparam, &targets[3 * t], sel, vg, e);
    put(e, st, &res[t]);
  }
  return 0;
}

// Discretization offsets (nd0 nd1 nd2 x 3) of a block of `size` turned by
// `rotation` (block.rs:61-72).
void orc_block_offsets(const double* size, const int64_t* nd, const double* rotation, double* out) {
  auto o = disc_offsets(size, nd, rotation);
  for (size_t k = 0; k < o.size(); ++k) out[3 * k] = o[k][0], out[3 * k + 1] = o[k][1], out[3 * k + 2] = o[k][2];
}

// block_krige_points of one block centred at t from the given samples (for
// the block.rs tests): the points are t + offsets (np x 3).
int32_t orc_block_krige(const double* t, int64_t np, const double* offsets, int64_t n, const double* xyz,
                        const double* v, const double* err, const orc_variogram* vgp, orc_result* res,
                        double* weights) {
  Variogram vg = conv_vg(vgp);
  std::vector<Sample> s = conv_samples(n, xyz, v, err, nullptr);
  std::vector<std::array<double, 3>> pts(static_cast<size_t>(np));
  for (int64_t k = 0; k < np; ++k) pts[k] = {t[0] + offsets[3 * k], t[1] + offsets[3 * k + 1], t[2] + offsets[3 * k + 2]};
  Estimate e;
  int st = block_krige_points(pts, s, vg, e);
  put(e, st, res);
  if (st == OK && weights) std::copy(e.weights.begin(), e.weights.end(), weights);
  return st;
}

// Block kriging of m block centres (crates/py/src/estimation.rs:775-784 via
// estimate_many, batch.rs:15-38): the search at the centre, then
// block_krige_points over centre + offsets (np x 3).
int32_t orc_estimate_block(int64_t m, const double* targets, int64_t n, const double* xyz, const double* v,
                           const double* err, const int64_t* hole, const orc_search* sp, const orc_variogram* vgp,
                           int64_t np, const double* offsets, int32_t nthreads, orc_result* res) {
  std::vector<Sample> s = conv_samples(n, xyz, v, err, hole);
  SearchP p = conv_search(sp);
  if (!check(p)) return -1;
  Variogram vg = conv_vg(vgp);
  Tree tree(s, p, &vg);
  auto work = [&](int64_t k0, int64_t k1) {
    for (int64_t k = k0; k < k1; ++k) {
      const double* t = &targets[3 * k];
      std::vector<size_t> chosen;
      bool ok = tree.neighbors(t, -1, chosen);
      if (!ok) { Estimate e; put(e, SEARCH_FAILED, &res[k]); continue; }
      std::vector<Sample> sel;
      for (size_t i : balanced(tree, t, chosen)) sel.push_back(s[i]);
      std::vector<std::array<double, 3>> pts(static_cast<size_t>(np));
      for (int64_t q = 0; q < np; ++q)
        pts[q] = {t[0] + offsets[3 * q], t[1] + offsets[3 * q + 1], t[2] + offsets[3 * q + 2]};
      if (p.calibration) {  // block.rs block_covariances: the block's rhs and C(B,B)
        std::vector<double> rhs;
        double cbb = 0.0;
        block_rhs(pts, sel, vg, rhs, cbb);
        calibrate(p, vg, ORDINARY, rhs, cbb, sel);
      }
      Estimate e;
      int st = block_krige_points(pts, sel, vg, e);
      put(e, st, &res[k]);
    }
  };
  int nt = nthreads > 0 ? nthreads : orc_num_threads();
  std::vector<std::thread> pool;
  int64_t chunk = (m + nt - 1) / nt;
  for (int w = 0; w < nt; ++w) {
    int64_t k0 = int64_t(w) * chunk, k1 = std::min(m, k0 + chunk);
    if (k0 < k1) pool.emplace_back(work, k0, k1);
  }
  for (auto& th : pool) th.join();
  return 0;
}

// crates/core/src/block_model.rs:62-86: centroid of cell `index`, x fastest.
void orc_centroids(const double* origin, const double* size, const int64_t* count, const double* rotation,
                   int64_t first, int64_t m, double* out) {
  M3 f = block_frame(rotation[0], rotation[1], rotation[2]);
  M3 ft;
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) ft.m[i][j] = f.m[j][i];
  uint64_t nx = uint64_t(count[0]), ny = uint64_t(count[1]);
  for (int64_t k = 0; k < m; ++k) {
    uint64_t index = uint64_t(first + k);
    uint64_t ijk[3] = {index % nx, index / nx % ny, index / (nx * ny)};
    double local[3], world[3];
    for (int a = 0; a < 3; ++a) local[a] = (double(ijk[a]) + 0.5) * size[a];
    mulv(ft, local, world);
    for (int a = 0; a < 3; ++a) out[3 * k + a] = origin[a] + world[a];
  }
}

}  // extern "C"
