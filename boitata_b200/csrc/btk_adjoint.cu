// A kriging objective and its gradient with respect to the variogram (K5),
// over frozen neighbourhoods: the leave-one-out loss or the mean estimate of
// a block model.
//
// Objectives (ordinary kriging, crates/estimation/src/kernel.rs:24-123):
//   - leave-one-out: L = (1/N) sum_i (z*_i - z_i)^2 over the samples whose
//     leave-one-out estimate z*_i (crates/estimation/src/batch.rs:165-190)
//     exists, each from the list the leave-one-out search gave at fit;
//   - block-model mean: J = (1/N) sum_t z*_t over the targets t whose
//     estimate exists, each from the list the search gave when frozen.
// Systems holding coincident samples (the reference merges them, coincident.rs)
// are left out of both. Parameters theta: nugget, each structure's sill, each
// structure's major range, the semi/major and minor/major ratios and the
// azimuth, dip and rake (degrees) of the shared anisotropy
// (crates/variogram/src/{composite,aniso}.rs).
//
// For one system with bordered matrix K = [C 1; 1' 0], K [w; mu] = [c; 1]
// and z* = z'w, the adjoint K [lambda; nu] = [z; 0] gives
//   dz*/dtheta = lambda' dc/dtheta - lambda' dC/dtheta w,
// so with a = 2 (z* - z_i) lambda (leave-one-out) or a = lambda (mean) the
// system adds sum_j a_j dc_j/dtheta - sum_jk a_j w_k dC_jk/dtheta to the
// gradient sum. w and lambda come from x_v = C^-1 v for v = c, 1, z:
// mu = (1'x_c - 1) / 1'x_1, w = x_c - mu x_1, nu = 1'x_z / 1'x_1 and
// lambda = x_z - nu x_1. The covariance derivatives are recomputed pair by
// pair, never stored: C(h) = sum_s sill_s (1 - g_s(h / r_s)) for h > 0 and
// C(0) = C0, so dC/dsill_s = 1 - g_s, dC/dr_s = sill_s g_s'(t) h / r_s^2,
// dC/dh = -sum_s sill_s g_s'(t) / r_s and dh/dphi = (M d)'(dM/dphi d) / h for
// the lag h = |M d| of world offset d, M = diag(1, 1/semi, 1/minor) R, with
// the shape derivatives of crates/variogram/src/model.rs:181-312.
//
// One group of NW warps per system (n <= 32 NW), lane = row. Every lag is
// lag_world's (with the frame M when the variogram has an anisotropy, else
// the plain Euclidean norm, M being orthogonal then), as in the prediction
// kernels, so the FP64 objective is the prediction path's estimate to the bit. Two forms:
//   - FP64: the shifted, windowed right-looking LDL^T of the prediction
//     kernels with the forward substitutions fused in, the multipliers kept
//     in place of the covariance triangle, and one backward sweep for x;
//   - mixed: the FP32 LDL^T with its multipliers in shared memory, then FP64
//     iterative refinement (residuals from the FP64 triangle, corrections
//     from the FP32 factors) until x is good to about 1e-8 relative; the
//     systems it does not converge on are redone by the FP64 form.
// Gradient terms are accumulated in FP64. Per-system partial sums go to a
// buffer that is reduced in a fixed order, so results are deterministic.
#include <type_traits>

#include "btk_device.cuh"
#include "btk_group.cuh"

namespace btk {
namespace {

constexpr int kMaxTheta = 1 + 2 * BTK_MAX_STRUCT + 5;
constexpr int kRefine = 4;  // most FP64 refinement steps of the mixed form

template <int NW>
struct alignas(16) GradSmem {
  static constexpr int R = 32 * NW;
  double W[R][3];             // world coordinates of the samples
  double T[R * (R - 1) / 2];  // covariances, strictly lower, packed; the FP64 form's multipliers after the load
  alignas(16) double col[2][R + 2];
  double rhs[2][4];
  double red[NW][8];
  int ired[NW];
  double w[R], adj[R];
  double xs[3][R];
};

template <int NW>
struct alignas(16) GradSmemMixed {
  static constexpr int R = 32 * NW;
  GradSmem<NW> base;
  alignas(16) float colf[2][R + 4];
  float rhsf[2][4];
  float L[R][R + 1];
};

template <int NW>
__device__ __forceinline__ GradSmem<NW>& base_of(GradSmem<NW>& s) {
  return s;
}
template <int NW>
__device__ __forceinline__ GradSmem<NW>& base_of(GradSmemMixed<NW>& s) {
  return s.base;
}

// M d for the lag frame M (row-major), in lag_world's operation order.
__device__ __forceinline__ void frame_apply(const VgDev& vg, const double d[3], double md[3]) {
  const double* M = vg.frame;
  md[0] = fma(M[2], d[2], fma(M[1], d[1], M[0] * d[0]));
  md[1] = fma(M[5], d[2], fma(M[4], d[1], M[3] * d[0]));
  md[2] = fma(M[8], d[2], fma(M[7], d[1], M[6] * d[0]));
}

__device__ __forceinline__ double norm3(const double v[3]) { return sqrt(fma(v[2], v[2], fma(v[1], v[1], v[0] * v[0]))); }

// Adds coef * dC(h)/dtheta for a lag h > 0 with projected offset Md and world
// offset d to g (theta order: nugget, sills, ranges, semi, minor, az, dip, rake).
__device__ __forceinline__ void add_lag_terms(const GradDev& a, double coef, double h, const double Md[3],
                                              const double d[3], double* g) {
  const int S = a.vg.nstruct;
  double dcdh = 0.0;
  for (int s = 0; s < S; ++s) {
    const double ir = a.vg.inv_range[s];
    const double t = h * ir;
    const double gs = shape64(a.vg.model[s], a.vg.param[s], t);
    const double gp = dshape64(a.vg.model[s], a.vg.param[s], t);
    g[1 + s] += coef * (1.0 - gs);
    g[1 + S + s] += coef * a.vg.sill[s] * gp * h * ir * ir;
    dcdh -= a.vg.sill[s] * gp * ir;
  }
  const double f = coef * dcdh / h;
#pragma unroll
  for (int p = 0; p < 5; ++p) {
    const double* dM = a.dM[p];
    const double e0 = dM[0] * d[0] + dM[1] * d[1] + dM[2] * d[2];
    const double e1 = dM[3] * d[0] + dM[4] * d[1] + dM[5] * d[2];
    const double e2 = dM[6] * d[0] + dM[7] * d[1] + dM[8] * d[2];
    g[1 + 2 * S + p] += f * (Md[0] * e0 + Md[1] * e1 + Md[2] * e2);
  }
}

// FP64 backward sweep x = L^-T D^-1 y with the multipliers L[k][row] packed
// at T[k (k - 1) / 2 + row].
template <int NW>
__device__ __forceinline__ void sweep_back64(GradSmem<NW>& S, int gid, int row, int nn, double dme, double& u0,
                                             double& u1, double& u2) {
  u0 /= dme, u1 /= dme, u2 /= dme;
  gsync<NW>(gid);
  for (int k = nn - 1; k >= 0; --k) {
    const int b = k & 1;
    if (row == k) S.rhs[b][0] = u0, S.rhs[b][1] = u1, S.rhs[b][2] = u2;
    gsync<NW>(gid);
    if (row < k) {
      const double l = S.T[k * (k - 1) / 2 + row];
      u0 = fma(-l, S.rhs[b][0], u0);
      u1 = fma(-l, S.rhs[b][1], u1);
      u2 = fma(-l, S.rhs[b][2], u2);
    }
  }
}

// Resident CTAs an SM: the FP64 form with two-warp groups held to 168
// registers, three CTAs instead of two at 244 (the c5 mean gradient went from
// 1.32 to 1.13 s, results bit-identical); the mixed one-warp form five (the
// c4 mixed gradient), the others four.
template <int NW, bool MIXED>
__global__ void __launch_bounds__(128, MIXED ? (NW == 1 ? 5 : 4) : (NW == 1 ? 4 : 3)) k_grad(GradDev a) {
  constexpr int R = 32 * NW;
  constexpr int GROUPS = 128 / R;
  constexpr int Q = R / 4;
  using Sx = typename std::conditional<MIXED, GradSmemMixed<NW>, GradSmem<NW>>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int gid = threadIdx.x / R, row = threadIdx.x % R, wig = row >> 5;
  Sx& X = reinterpret_cast<Sx*>(smem_raw)[gid];
  GradSmem<NW>& S = base_of<NW>(X);
  const int ns = a.vg.nstruct;
  const int ntheta = 1 + 2 * ns + 5;
  const double c0 = a.vg.c0;
  const bool mean = a.tx != nullptr;
  const int64_t nitems = a.list ? *a.list_len : a.n;
  for (int64_t item = int64_t(blockIdx.x) * GROUPS + gid; item < nitems; item += int64_t(gridDim.x) * GROUPS) {
    const int64_t i = a.list ? a.list[item] : item;
    const int64_t si = a.first + i;  // the left-out sample, or the target
    double* out = a.part + i * a.stride;
    gsync<NW>(gid);
    const int n = a.count[si];
    const bool solvable = a.sstatus[si] == BTK_ST_OK && n > 0 && n <= R;
    const bool have = solvable && row < n;
    const double t[3] = {mean ? a.tx[si] : a.sx[si], mean ? a.ty[si] : a.sy[si], mean ? a.tz[si] : a.sz[si]};
    double w[3] = {0.0, 0.0, 0.0}, z = 0.0, err = 0.0;
    int tw = 0;
    if (have) {
      const uint32_t j = a.nbr[si * a.max_samples + row];
      w[0] = a.sx[j], w[1] = a.sy[j], w[2] = a.sz[j], z = a.sv[j];
      if (a.se) err = a.se[j];
      tw = a.twin ? a.twin[j] : 0;
    }
    // uniform over the group: `solvable` depends on the system alone
    if (!solvable || group_any<NW>(S, gid, wig, tw != 0)) {
      if (row == 0) {
        for (int k = 0; k < a.stride; ++k) out[k] = 0.0;
        if (a.value) a.value[si] = NAN;
      }
      continue;
    }
    if (have) S.W[row][0] = w[0], S.W[row][1] = w[1], S.W[row][2] = w[2];
    gsync<NW>(gid);
    const int E = n * (n - 1) / 2;
    for (int e = row; e < E; e += R) {
      int p, q;
      tri_index(e, p, q);
      S.T[e] = cov64(a.vg, lag_world(a.vg, S.W[q][0], S.W[q][1], S.W[q][2], S.W[p][0], S.W[p][1], S.W[p][2]));
    }
    const double dt[3] = {w[0] - t[0], w[1] - t[1], w[2] - t[2]};  // lag_world(t, w)'s offset
    double pt[3];
    frame_apply(a.vg, dt, pt);
    const double hc = a.vg.has_frame ? norm3(pt) : norm3(dt);  // lag_world's h, frame or not
    const double c = have ? cov64(a.vg, hc) : 0.0;
    const double diag = have ? c0 + err : 1.0;
    const int tri = row * (row - 1) / 2;
    gsync<NW>(gid);

    double x0 = 0.0, x1 = 0.0, x2 = 0.0;
    double estimate = 0.0;  // the FP64 form's, from the same forms as the prediction epilogue
    bool redo = false;
    const int n1 = min(n, Q), n2 = min(n, 2 * Q), n3 = min(n, 3 * Q);
    if constexpr (MIXED) {
      float A[R];
#pragma unroll
      for (int q = 0; q < R; ++q)
        A[q] = q < row ? (have ? float(S.T[tri + q]) : 0.f) : (q == row ? float(diag) : 0.f);
      float y0 = have ? float(c) : 0.f, y1 = have ? 1.f : 0.f, y2 = have ? float(z) : 0.f;
      float dme = 1.f;
      bool weak = false;
      // A pivot at most n ulp(C0) is not resolved in FP32: the FP64 form takes the system.
      const float thr = float(n) * 1.1920929e-7f * float(c0);
      eliminate_rows_f32<NW, R>(A, 0, n1, row, X, gid, y0, y1, y2, dme, weak, thr);
      if (!weak) eliminate_rows_f32<NW, 3 * Q>(A, n1, n2, row, X, gid, y0, y1, y2, dme, weak, thr);
      if (!weak) eliminate_rows_f32<NW, 2 * Q>(A, n2, n3, row, X, gid, y0, y1, y2, dme, weak, thr);
      if (!weak) eliminate_rows_f32<NW, Q>(A, n3, n, row, X, gid, y0, y1, y2, dme, weak, thr);
      redo = weak;
      if (!weak) {
        float u0 = y0, u1 = y1, u2 = y2;
        sweep_f32<NW>(X, gid, row, n, dme, false, u0, u1, u2);
        x0 = have ? double(u0) : 0.0, x1 = have ? double(u1) : 0.0, x2 = have ? double(u2) : 0.0;
        const double cmax = fmax(group_max<NW>(S, gid, wig, have ? fabs(c) : 0.0), 1e-300);
        const double zmax = fmax(group_max<NW>(S, gid, wig, have ? fabs(z) : 0.0), 1e-300);
        const double dmin = -group_max<NW>(S, gid, wig, have ? -double(dme) : -1e300);
        // x errs by about rho C0 / D_min (rho the relative residual): refine
        // until that is at most 1e-8, as long as each step halves rho.
        double rho = 0.0;
        for (int it = 0;; ++it) {
          S.xs[0][row] = x0, S.xs[1][row] = x1, S.xs[2][row] = x2;
          gsync<NW>(gid);
          double r0 = 0.0, r1 = 0.0, r2 = 0.0;
          if (have) {
            double a0 = diag * x0, a1 = diag * x1, a2 = diag * x2;
            for (int j = 0; j < n; ++j) {
              if (j == row) continue;
              const double cij = j < row ? S.T[tri + j] : S.T[j * (j - 1) / 2 + row];
              a0 = fma(cij, S.xs[0][j], a0);
              a1 = fma(cij, S.xs[1][j], a1);
              a2 = fma(cij, S.xs[2][j], a2);
            }
            r0 = c - a0, r1 = 1.0 - a1, r2 = z - a2;
          }
          const double prev = rho;
          rho = group_max<NW>(S, gid, wig, have ? fmax(fmax(fabs(r0) / cmax, fabs(r1)), fabs(r2) / zmax) : 0.0);
          if (rho * c0 / dmin <= 1e-8) break;
          if (it == kRefine || !(rho < 1.0) || (it > 0 && !(rho < 0.5 * prev))) {
            redo = true;
            break;
          }
          float v0 = float(r0), v1 = float(r1), v2 = float(r2);
          sweep_f32<NW>(X, gid, row, n, dme, true, v0, v1, v2);
          if (have) x0 += double(v0), x1 += double(v1), x2 += double(v2);
          gsync<NW>(gid);  // every row has read xs
        }
      }
      if (redo) {  // uniform over the group
        if (row == 0) a.redo[atomicAdd(reinterpret_cast<unsigned long long*>(a.redo_len), 1ull)] = i;
        continue;
      }
    } else {
      double A[R];
#pragma unroll
      for (int q = 0; q < R; ++q) A[q] = q < row ? (have ? S.T[tri + q] : 0.0) : (q == row ? diag : 0.0);
      double y0 = have ? c : 0.0, y1 = have ? 1.0 : 0.0, y2 = have ? z : 0.0, dme = 1.0;
      bool sing = false;
      const double thr = kPivot * c0;
      gsync<NW>(gid);  // every row has its covariances: the triangle now takes the multipliers
      double* Lrow = S.T + tri;
      // Uniform windows for both warps: warp 0's own (eliminate_staged) made the
      // objective faster but the objective with its gradient slower (c5: 1.155
      // against 1.129 s), the kernel's code being larger.
      eliminate_rows<NW, R, true>(A, 0, n1, row, S, gid, y0, y1, y2, dme, sing, thr, Lrow);
      if (!sing) eliminate_rows<NW, 3 * Q, true>(A, n1, n2, row, S, gid, y0, y1, y2, dme, sing, thr, Lrow);
      if (!sing) eliminate_rows<NW, 2 * Q, true>(A, n2, n3, row, S, gid, y0, y1, y2, dme, sing, thr, Lrow);
      if (!sing) eliminate_rows<NW, Q, true>(A, n3, n, row, S, gid, y0, y1, y2, dme, sing, thr, Lrow);
      if (sing) {  // a pivot at most 1e-12 C0 (kernel.rs:61): no estimate
        if (row == 0) {
          for (int k = 0; k < a.stride; ++k) out[k] = 0.0;
          if (a.value) a.value[si] = NAN;
        }
        continue;
      }
      // The estimate as the prediction kernels form it (u'C^-1 v = sum y_u y_v / D),
      // so the objective is their value to the bit.
      const double wt = have ? 1.0 / dme : 0.0;
      double f5[5] = {y1 * y0 * wt, y1 * y1 * wt, y2 * y0 * wt, y2 * y1 * wt, y0 * y0 * wt};
      group_sum5<NW>(S, gid, wig, f5);
      const double mu5 = (f5[0] - 1.0) / f5[1];
      estimate = f5[2] - mu5 * f5[3];
      double u0 = y0, u1 = y1, u2 = y2;
      sweep_back64<NW>(S, gid, row, n, dme, u0, u1, u2);
      x0 = have ? u0 : 0.0, x1 = have ? u1 : 0.0, x2 = have ? u2 : 0.0;
    }
    double sums[3] = {x0, x1, x2};
    group_sum<NW, 3>(S, gid, wig, sums);
    const double mu = (sums[0] - 1.0) / sums[1];  // kernel.rs:93
    const double wl = x0 - mu * x1;               // weights
    const double nu = sums[2] / sums[1];
    const double lam = x2 - nu * x1;              // adjoint weights
    double est[1] = {have ? wl * z : 0.0};
    if (MIXED)
      group_sum<NW, 1>(S, gid, wig, est);
    else
      est[0] = estimate;
    const double resid = est[0] - (mean ? 0.0 : a.sv[si]);
    const double adj = have ? (mean ? lam : 2.0 * resid * lam) : 0.0;
    if (row == 0) {
      out[0] = mean ? est[0] : resid * resid;
      out[1] = 1.0;
      if (a.value) a.value[si] = est[0];
    }
    if (!a.want_grad) continue;
    S.w[row] = have ? wl : 0.0, S.adj[row] = adj;
    gsync<NW>(gid);
    double g[kMaxTheta];
#pragma unroll
    for (int k = 0; k < kMaxTheta; ++k) g[k] = 0.0;
    if (have) {
      // Diagonal: C_jj = nugget + sum sill + err.
      const double f = -adj * wl;
      g[0] += f;
      for (int s = 0; s < ns; ++s) g[1 + s] += f;
      // Right-hand side c_j = C(|M (s_j - t)|).
      if (hc > 0.0) {
        add_lag_terms(a, adj, hc, pt, dt, g);
      } else {
        g[0] += adj;
        for (int s = 0; s < ns; ++s) g[1 + s] += adj;
      }
    }
    for (int e = row; e < E; e += R) {  // sample pairs (p > q)
      int p, q;
      tri_index(e, p, q);
      const double coef = -(S.adj[p] * S.w[q] + S.adj[q] * S.w[p]);
      const double d[3] = {S.W[p][0] - S.W[q][0], S.W[p][1] - S.W[q][1], S.W[p][2] - S.W[q][2]};
      double md[3];
      frame_apply(a.vg, d, md);
      const double h = a.vg.has_frame ? norm3(md) : norm3(d);
      if (h > 0.0) add_lag_terms(a, coef, h, md, d, g);
    }
    group_sum<NW, 8>(S, gid, wig, g);
    group_sum<NW, kMaxTheta - 8>(S, gid, wig, g + 8);
    if (row == 0)
      for (int k = 0; k < ntheta; ++k) out[2 + k] = g[k];
  }
}

// Column sums of part[n][stride] in a fixed order: one block per column.
__global__ void k_col_sums(int64_t n, int stride, const double* part, double* sums) {
  __shared__ double s[256];
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) acc += part[i * stride + blockIdx.x];
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[blockIdx.x] = s[0];
}

template <int NW, bool MIXED>
cudaError_t run_grad(const Launch& L, const GradDev& a) {
  using Sx = typename std::conditional<MIXED, GradSmemMixed<NW>, GradSmem<NW>>::type;
  const size_t smem = sizeof(Sx) * (128 / (32 * NW));
  auto kern = k_grad<NW, MIXED>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, smem);
  if (e != cudaSuccess) return e;
  int64_t blocks = int64_t(L.sm_count) * (per_sm > 0 ? per_sm : 1);
  const int64_t need = (a.n + (128 / (32 * NW)) - 1) / (128 / (32 * NW));
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
  kern<<<int(blocks), 128, smem, L.stream>>>(a);
  ++*L.counter;
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_grad(const Launch& L, const GradDev& a0, double* sums, int rows, bool mixed) {
  if (a0.n <= 0) return cudaSuccess;
  GradDev a = a0;
  a.list = nullptr, a.list_len = nullptr;
  cudaError_t e = cudaSuccess;
  if (mixed) {
    e = cudaMemsetAsync(a.redo_len, 0, sizeof(int64_t), L.stream);
    if (e == cudaSuccess) e = rows > 32 ? run_grad<2, true>(L, a) : run_grad<1, true>(L, a);
    a.list = a.redo, a.list_len = a.redo_len;  // what the mixed pass left, in FP64
  }
  if (e == cudaSuccess) e = rows > 32 ? run_grad<2, false>(L, a) : run_grad<1, false>(L, a);
  if (e != cudaSuccess) return e;
  k_col_sums<<<a.stride, 256, 0, L.stream>>>(a.n, a.stride, a.part, sums);
  ++*L.counter;
  return cudaGetLastError();
}

}  // namespace btk
