// Per-system kriging solve (K2 assembly, K3 factor-and-solve, K4 epilogue),
// one system per warp (n <= 32) or per warp pair (n <= 64).
//
// Reference: crates/estimation/src/kernel.rs:24-123 (and the coincident
// guard of crates/estimation/src/coincident.rs:27-111 via krige.rs:83-95).
// The reference factors C = L L^T (packed Cholesky), solves C a = c and
// C b = 1, and forms mu = (sum a - 1) / sum b, w = a - mu b, value = w . z,
// sigma^2 = max(C0 - w . c - mu, 0), with a singular system where a pivot is
// NaN or <= 1e-12 C0.
//
// B200 form: the estimate, variance and Lagrange multiplier only need the
// quadratic forms u^T C^-1 v for u, v in {c, 1, f(z)}. With C = L D L^T (L
// unit lower) and y_v = L^-1 v they are sum_i y_u,i y_v,i / D_i, so one
// right-looking LDL^T pass, with the three forward substitutions fused into
// it, replaces the factorisation and both triangular solves: no back
// substitution and no square roots. D_k is the Schur-complement pivot, the
// same quantity the reference tests against 1e-12 C0.
//
// Layout: row i of the lower triangle lives in registers of lane i (A[R],
// compile-time indexed); step k broadcasts the unscaled column k and the
// three y_k through a double-buffered shared-memory line, one group barrier
// per step. Assembly is balanced: the n(n-1)/2 covariances are spread over
// all lanes into a packed shared-memory triangle, then each lane loads its
// row (conflict-free: row offsets i(i-1)/2 cover every bank pair twice).
//
// Mixed form: the same assembly (FP64), an FP32 LDL^T with fused forward
// substitution and an FP32 back substitution give approximate solutions
// x_v; FP64 residuals r_v = v - C x_v (C from the FP64 triangle) drive up to
// three steps of iterative refinement (x_v += C~^-1 r_v with the stored FP32
// factors) until the corrected forms u^T x_v + x_u^T r_v, whose error is
// second order in the residuals, are good to about 1e-8 C0. The Lagrange
// multiplier and the variance are then formed in FP64. A system whose FP32
// factorisation breaks down (a pivot NaN or not positive) or whose
// refinement does not converge goes to an FP64 re-solve list (status flag
// BTK_ST_FP64_FALLBACK), which also takes the singular decision.
#include <cstddef>

#include "btk_device.cuh"
#include "btk_group.cuh"

namespace btk {
namespace {

// 16-byte aligned, with a size a multiple of 16, so every group's column line
// takes 16-byte (double2) loads.
template <int NW>
struct alignas(16) SolveSmem {
  static constexpr int R = 32 * NW;
  double P[R][3];
  double T[R * (R - 1) / 2];
  alignas(16) double col[2][R + 2];  // column below the pivot (0 .. R-2), the pivot (R), a sink (R+1)
  double rhs[2][4];
  double red[NW][8];
  int ired[NW];
  double mz[R], me[R];
  int cof[R], cfirst[R], csize[R];
};

static_assert(sizeof(SolveSmem<1>) % 16 == 0 && sizeof(SolveSmem<2>) % 16 == 0, "group stride");
static_assert(offsetof(SolveSmem<1>, col) % 16 == 0 && offsetof(SolveSmem<2>, col) % 16 == 0, "column line");
static_assert((sizeof(double) * (32 + 2)) % 16 == 0 && (sizeof(double) * (64 + 2)) % 16 == 0, "line stride");
static_assert((sizeof(float) * (32 + 4)) % 16 == 0 && (sizeof(float) * (64 + 4)) % 16 == 0, "FP32 line stride");

template <int NW>
struct MixedSmem {
  static constexpr int R = 32 * NW;
  SolveSmem<NW> base;
  alignas(16) float colf[2][R + 4];  // column below the pivot (0 .. R-2), the pivot (R), a sink (R+1)
  float rhsf[2][4];
  float L[R][R + 1];
  double xs[3][R];
};

// Coincident guard on one lane (coincident.rs:27-82): samples within 1e-6 m
// of a cluster's first member join it; each cluster becomes one datum at the
// first member with the mean of f(z) (the value the spread weights give,
// krige.rs:89-92) and error variance sum_ij C / k^2 - C0 + sum err / k^2.
// World coordinates in P, errors in me, f(z) in mz; rewritten in place.
template <int NW>
__device__ void merge_clusters(SolveSmem<NW>& S, int n, const VgDev& vg, int* nn_out) {
  const double eps2 = kEps * kEps;
  int* of = S.cof;
  int* first = S.cfirst;
  int* size = S.csize;
  int nc = 0;
  for (int i = 0; i < n; ++i) {
    int c = -1;
    for (int q = 0; q < nc && c < 0; ++q) {
      const double* a = S.P[first[q]];
      if (d2_exact(a[0], a[1], a[2], S.P[i][0], S.P[i][1], S.P[i][2]) <= eps2) c = q;
    }
    if (c < 0) c = nc, first[nc] = i, size[nc] = 0, ++nc;
    of[i] = c;
    size[c] += 1;
  }
  // Cluster c is written to slot c <= first[c]; every sample it reads has an
  // index >= first[c], and no later cluster reads a slot below its own first
  // member, so the rewrite can run in place in cluster order.
  for (int c = 0; c < nc; ++c) {
    const int f = first[c];
    double loc0 = S.P[f][0], loc1 = S.P[f][1], loc2 = S.P[f][2], err = S.me[f], zb = S.mz[f];
    if (size[c] > 1) {
      const double k = double(size[c]);
      double var = 0.0, zs = 0.0;
      for (int i = f; i < n; ++i) {
        if (of[i] != c) continue;
        var += S.me[i];
        zs += S.mz[i];
        for (int j = f; j < n; ++j)
          if (of[j] == c) var += cov64(vg, lag64(vg, S.P[i], S.P[j]));
      }
      err = var / (k * k) - vg.c0;
      zb = zs / k;
    }
    S.P[c][0] = loc0, S.P[c][1] = loc1, S.P[c][2] = loc2;
    S.me[c] = err, S.mz[c] = zb;
  }
  *nn_out = nc;
}

// Everything up to the packed covariance triangle: loads the system of
// target ti, applies the coincident guard, projects into the variogram
// frame, assembles T (strictly lower, packed) and returns this row's data.
// Returns false (outputs written) when there is nothing to solve.
// kPairs: no fit-time twin flags; the system's own sample pairs are tested.
template <int NW, bool kPairs = false>
__device__ __forceinline__ bool assemble(const SolveDev& a, SolveSmem<NW>& S, int gid, int wig, int row, int64_t ti,
                                         int& n, int& nn, bool& have, double& c, double& err, double& zf,
                                         int& kind) {
  constexpr int R = 32 * NW;
  kind = a.kinds ? int(a.kinds[ti]) : a.kind;
  n = a.count[ti];
  const int8_t st = a.sstatus[ti];
  if (st == BTK_ST_OK && n > R && a.lu) {  // beyond this kernel: the dense LU takes it
    if (row == 0) a.lu[atomicAdd(reinterpret_cast<unsigned long long*>(a.lu_len), 1ull)] = ti;
    return false;
  }
  if (st != BTK_ST_OK || n <= 0 || n > R) {
    if (row == 0) write_fail(a, ti, st != BTK_ST_OK ? st : (n > R ? BTK_ST_UNSUPPORTED : BTK_ST_SEARCH_FAILED), 0);
    return false;
  }
  // A caller's list longer than its row: nothing of it is read.
  if (kPairs && a.nsamples > 0 && n > a.max_samples) {
    if (row == 0) write_fail(a, ti, BTK_ST_INVALID, 0);
    return false;
  }
  const double t[3] = {a.tx[ti], a.ty[ti], a.tz[ti]};
  have = row < n;
  double w[3] = {0, 0, 0};
  double z = 0.0;
  err = 0.0;
  int tw = 0;
  bool bad = false;
  if (have) {
    const uint32_t j = a.nbr[ti * a.max_samples + row];
    bad = kPairs && a.nsamples > 0 && int64_t(j) >= a.nsamples;
    if (!bad) {
      w[0] = a.sx[j], w[1] = a.sy[j], w[2] = a.sz[j];
      z = a.sv[j];
      if (a.se) err = a.se[j];
      if (!kPairs) tw = a.twin[j];
    }
  }
  if (kPairs && a.nsamples > 0 && group_any<NW>(S, gid, wig, bad)) {  // an index past the caller's samples
    if (row == 0) write_fail(a, ti, BTK_ST_INVALID, 0);
    return false;
  }
  zf = kind_f(kind, a.kparam, z);
  nn = n;
  if (kPairs) {  // coincident.rs:27-31 on this system's samples
    if (have) S.P[row][0] = w[0], S.P[row][1] = w[1], S.P[row][2] = w[2];
    gsync<NW>(gid);
    if (have)
      for (int q = 0; q < row; ++q)
        if (d2_exact(S.P[q][0], S.P[q][1], S.P[q][2], w[0], w[1], w[2]) <= kEps * kEps) {
          tw = 1;
          break;
        }
    gsync<NW>(gid);
  }
  if (group_any<NW>(S, gid, wig, tw != 0)) {
    if (have) S.P[row][0] = w[0], S.P[row][1] = w[1], S.P[row][2] = w[2], S.me[row] = err, S.mz[row] = zf;
    gsync<NW>(gid);
    if (row == 0) merge_clusters<NW>(S, n, a.vg, &S.ired[0]);
    gsync<NW>(gid);
    nn = S.ired[0];
    have = row < nn;
    if (have) w[0] = S.P[row][0], w[1] = S.P[row][1], w[2] = S.P[row][2], err = S.me[row], zf = S.mz[row];
    gsync<NW>(gid);
  }
  // World coordinates; every lag is taken by lag_world (kernel.rs:34-42).
  if (have) S.P[row][0] = w[0], S.P[row][1] = w[1], S.P[row][2] = w[2];
  gsync<NW>(gid);
  const int E = nn * (nn - 1) / 2;
  for (int e = row; e < E; e += R) {
    int i, j;
    tri_index(e, i, j);
    S.T[e] = cov64(a.vg, lag_world(a.vg, S.P[j][0], S.P[j][1], S.P[j][2], S.P[i][0], S.P[i][1], S.P[i][2]));
  }
  c = have ? support_cov(a, t[0], t[1], t[2], w[0], w[1], w[2]) : 0.0;
  gsync<NW>(gid);
  return true;
}


template <int NW, bool kPairs = false>
__global__ void __launch_bounds__(128) k_solve64(SolveDev a, int8_t flag) {
  constexpr int R = 32 * NW;
  constexpr int GROUPS = 128 / R;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int gid = threadIdx.x / R, row = threadIdx.x % R, wig = row >> 5;
  SolveSmem<NW>& S = reinterpret_cast<SolveSmem<NW>*>(smem_raw)[gid];
  const int64_t nitems = a.list ? *a.list_len : a.m;
  const double c0 = a.vg.c0;
  for (int64_t item = int64_t(blockIdx.x) * GROUPS + gid; item < nitems; item += int64_t(gridDim.x) * GROUPS) {
    const int64_t ti = a.list ? a.list[item] : item;
    gsync<NW>(gid);
    int n, nn, kind;
    bool have;
    double c, err, zf;
    if (!assemble<NW, kPairs>(a, S, gid, wig, row, ti, n, nn, have, c, err, zf, kind)) continue;

    double A[R];
    const int tri = row * (row - 1) / 2;
#pragma unroll
    for (int q = 0; q < R; ++q)
      A[q] = q < row ? (have ? S.T[tri + q] : 0.0) : (q == row ? (have ? c0 + err : 1.0) : 0.0);
    double y0 = have ? c : 0.0, y1 = have ? 1.0 : 0.0, y2 = have ? zf : 0.0;
    double dme = 1.0;
    bool sing = false;
    const double thr = kPivot * c0;
    eliminate_staged<NW>(A, nn, row, wig, S, gid, y0, y1, y2, dme, sing, thr);
    if (sing) {
      if (row == 0) write_fail(a, ti, BTK_ST_SINGULAR, 0);
      continue;
    }
    const double wt = have ? 1.0 / dme : 0.0;
    double s[5] = {y1 * y0 * wt, y1 * y1 * wt, y2 * y0 * wt, y2 * y1 * wt, y0 * y0 * wt};
    group_sum5<NW>(S, gid, wig, s);
    if (row == 0) epilogue(a, kind, ti, s, n, flag);
  }
}



// Iterative refinement: at most this many FP32 corrections after the first
// solve; each takes its residual in FP64 from the FP64 triangle.
constexpr int kRefineSteps = 3;

// Four CTAs an SM: shared memory allows no more for either group size, and
// given only the block size the compiler held the one-warp form to 96
// registers and spilled about 100 bytes a thread.
template <int NW, bool kPairs = false>
__global__ void __launch_bounds__(128, 4) k_solve_mixed(SolveDev a, int64_t* redo, int64_t* redo_len) {
  constexpr int R = 32 * NW;
  constexpr int GROUPS = 128 / R;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int gid = threadIdx.x / R, row = threadIdx.x % R, wig = row >> 5;
  MixedSmem<NW>& X = reinterpret_cast<MixedSmem<NW>*>(smem_raw)[gid];
  SolveSmem<NW>& S = X.base;
  const int64_t nitems = a.list ? *a.list_len : a.m;
  const double c0 = a.vg.c0;
  for (int64_t item = int64_t(blockIdx.x) * GROUPS + gid; item < nitems; item += int64_t(gridDim.x) * GROUPS) {
    const int64_t ti = a.list ? a.list[item] : item;
    gsync<NW>(gid);
    int n, nn, kind;
    bool have;
    double c, err, zf;
    if (!assemble<NW, kPairs>(a, S, gid, wig, row, ti, n, nn, have, c, err, zf, kind)) continue;

    // FP32 LDL^T with the forward substitution of (c, 1, f) fused in.
    float A[R];
    const int tri = row * (row - 1) / 2;
    const double diag = have ? c0 + err : 1.0;
#pragma unroll
    for (int q = 0; q < R; ++q)
      A[q] = q < row ? (have ? float(S.T[tri + q]) : 0.f) : (q == row ? float(diag) : 0.f);
    float y0 = have ? float(c) : 0.f, y1 = have ? 1.f : 0.f, y2 = have ? float(zf) : 0.f;
    float dme = 1.f;
    bool weak = false;
    constexpr int Q = R / 4;
    const int n1 = min(nn, Q), n2 = min(nn, 2 * Q), n3 = min(nn, 3 * Q);
    // An FP32 pivot at most nn ulp(C0) is not resolved from the rounding of
    // its row, so it leaves no factorisation to refine with (nor a trustworthy
    // smallest pivot for the error test below): the FP64 form takes the
    // system, and with it the singular decision (a pivot at most 1e-12 C0,
    // kernel.rs:61). The FP32 form never declares a system singular.
    const float thr = float(nn) * 1.1920929e-7f * float(c0);
    eliminate_rows_f32<NW, R>(A, 0, n1, row, X, gid, y0, y1, y2, dme, weak, thr);
    if (!weak) eliminate_rows_f32<NW, 3 * Q>(A, n1, n2, row, X, gid, y0, y1, y2, dme, weak, thr);
    if (!weak) eliminate_rows_f32<NW, 2 * Q>(A, n2, n3, row, X, gid, y0, y1, y2, dme, weak, thr);
    if (!weak) eliminate_rows_f32<NW, Q>(A, n3, nn, row, X, gid, y0, y1, y2, dme, weak, thr);
    if (weak) {
      if (row == 0) redo[atomicAdd(reinterpret_cast<unsigned long long*>(redo_len), 1ull)] = ti;
      continue;
    }
    // First solve x = C~^-1 v (y is already L^-1 v).
    float u0 = y0, u1 = y1, u2 = y2;
    sweep_f32<NW>(X, gid, row, nn, dme, false, u0, u1, u2);
    double x0 = have ? double(u0) : 0.0, x1 = have ? double(u1) : 0.0, x2 = have ? double(u2) : 0.0;
    const double cmax = group_max<NW>(S, gid, wig, have ? fabs(c) : 0.0);
    const double zmax = group_max<NW>(S, gid, wig, have ? fabs(zf) : 0.0);
    const double dmin = -group_max<NW>(S, gid, wig, have ? -double(dme) : -1e300);
    double r0 = 0.0, r1 = 0.0, r2 = 0.0, rho = 0.0;
    for (int it = 0;; ++it) {
      // FP64 residuals r_v = v - C x_v with C from the FP64 triangle.
      X.xs[0][row] = x0, X.xs[1][row] = x1, X.xs[2][row] = x2;
      gsync<NW>(gid);
      r0 = r1 = r2 = 0.0;
      if (have) {
        double a0 = diag * x0, a1 = diag * x1, a2 = diag * x2;
        for (int j = 0; j < nn; ++j) {
          if (j == row) continue;
          const double cij = j < row ? S.T[tri + j] : S.T[j * (j - 1) / 2 + row];
          a0 = fma(cij, X.xs[0][j], a0);
          a1 = fma(cij, X.xs[1][j], a1);
          a2 = fma(cij, X.xs[2][j], a2);
        }
        r0 = c - a0, r1 = 1.0 - a1, r2 = zf - a2;
      }
      // The corrected forms below err by about rho^2 C0 / D_min (rho the
      // relative residual, D_min the smallest FP32 pivot): refine until that
      // is at most 1e-8, or give the system to the FP64 form.
      const double prev = rho;
      rho = group_max<NW>(S, gid, wig, have ? fmax(fmax(fabs(r0) / fmax(cmax, 1e-300), fabs(r1)),
                                                   fabs(r2) / fmax(zmax, 1e-300)) : 0.0);
      if (rho * rho * c0 / dmin <= 1e-8) break;
      // Out of steps, no factorisation worth the name (rho >= 1), or a step
      // that did not halve the residual: refinement will not converge.
      if (it == kRefineSteps || !(rho < 1.0) || (it > 0 && !(rho < 0.5 * prev))) break;
      u0 = float(r0), u1 = float(r1), u2 = float(r2);
      sweep_f32<NW>(X, gid, row, nn, dme, true, u0, u1, u2);
      if (have) x0 += double(u0), x1 += double(u1), x2 += double(u2);
      gsync<NW>(gid);  // every row has read xs
    }
    // Corrected forms u'x_v + x_u'r_v (error second order in the residuals).
    double s[5] = {x0 + x1 * r0, x1 + x1 * r1, zf * x0 + x2 * r0, zf * x1 + x2 * r1, c * x0 + x0 * r0};
    if (!have) s[0] = s[1] = s[2] = s[3] = s[4] = 0.0;
    group_sum5<NW>(S, gid, wig, s);
    if (!(rho * rho * c0 / dmin <= 1e-8) || !(s[1] > 0.0) || !(fabs(s[0]) < 1e30)) {
      if (row == 0) redo[atomicAdd(reinterpret_cast<unsigned long long*>(redo_len), 1ull)] = ti;
      continue;
    }
    if (row == 0) epilogue(a, kind, ti, s, n, 0);
  }
}

__global__ void k_bucket(int64_t m, const int32_t* count, const int8_t* sstatus, int64_t* small, int64_t* large,
                         int64_t* lens) {
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < m; t += int64_t(gridDim.x) * blockDim.x) {
    const bool big = sstatus[t] == BTK_ST_OK && count[t] > 32;
    unsigned long long* len = reinterpret_cast<unsigned long long*>(lens + (big ? 1 : 0));
    (big ? large : small)[atomicAdd(len, 1ull)] = t;
  }
}

template <class K>
int blocks_for(const Launch& L, K kern, size_t smem) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, smem) != cudaSuccess || per_sm < 1) per_sm = 1;
  if (L.tuning.solve_blocks_per_sm > 0 && L.tuning.solve_blocks_per_sm < per_sm) per_sm = L.tuning.solve_blocks_per_sm;
  return L.sm_count * per_sm;
}

template <int NW, bool kPairs = false>
cudaError_t run_fp64(const Launch& L, const SolveDev& a, int8_t flag) {
  const size_t smem = sizeof(SolveSmem<NW>) * (128 / (32 * NW));
  auto kern = k_solve64<NW, kPairs>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  kern<<<blocks_for(L, kern, smem), 128, smem, L.stream>>>(a, flag);
  ++*L.counter;
  return cudaGetLastError();
}

template <int NW, bool kPairs = false>
cudaError_t run_mixed(const Launch& L, const SolveDev& a, int64_t* redo, int64_t* redo_len) {
  const size_t smem = sizeof(MixedSmem<NW>) * (128 / (32 * NW));
  auto kern = k_solve_mixed<NW, kPairs>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  kern<<<blocks_for(L, kern, smem), 128, smem, L.stream>>>(a, redo, redo_len);
  ++*L.counter;
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_bucket(const Launch& L, int64_t m, const int32_t* count, const int8_t* sstatus, int64_t* lists,
                          int64_t* lens) {
  cudaError_t e = cudaMemsetAsync(lens, 0, 2 * sizeof(int64_t), L.stream);
  if (e != cudaSuccess) return e;
  int64_t b = (m + 255) / 256;
  if (b > int64_t(L.sm_count) * 8) b = int64_t(L.sm_count) * 8;
  if (b < 1) b = 1;
  k_bucket<<<int(b), 256, 0, L.stream>>>(m, count, sstatus, lists, lists + m, lens);
  ++*L.counter;
  return cudaGetLastError();
}

// rows: 32 (one warp per system) or 64 (a warp pair).
cudaError_t launch_solve(const Launch& L, const SolveDev& a, int rows) {
  return rows > 32 ? run_fp64<2>(L, a, 0) : run_fp64<1>(L, a, 0);
}

cudaError_t launch_solve_mixed(const Launch& L, const SolveDev& a, int rows, int64_t* redo, int64_t* redo_len) {
  return rows > 32 ? run_mixed<2>(L, a, redo, redo_len) : run_mixed<1>(L, a, redo, redo_len);
}

cudaError_t launch_solve_redo(const Launch& L, const SolveDev& a, int rows) {
  return rows > 32 ? run_fp64<2>(L, a, BTK_ST_FP64_FALLBACK) : run_fp64<1>(L, a, BTK_ST_FP64_FALLBACK);
}

// The same two kernels for systems of at most 32 samples without fit-time
// twin flags (a.twin unused): each system tests its own sample pairs.
cudaError_t launch_solve_mixed_pairs(const Launch& L, const SolveDev& a, int64_t* redo, int64_t* redo_len) {
  return run_mixed<1, true>(L, a, redo, redo_len);
}

cudaError_t launch_solve_redo_pairs(const Launch& L, const SolveDev& a) {
  return run_fp64<1, true>(L, a, BTK_ST_FP64_FALLBACK);
}

}  // namespace btk
