// Leave-one-out loss and its gradient with respect to the variogram (K5).
//
// Loss: L = (1/N) sum_i (z*_i - z_i)^2 over the samples whose leave-one-out
// ordinary-kriging estimate z*_i (crates/estimation/src/batch.rs:165-190 with
// kernel.rs:24-123) exists, with each sample's neighbourhood frozen (the
// lists the leave-one-out search gave at fit). Parameters theta: nugget,
// each structure's sill, each structure's major range, the semi/major and
// minor/major ratios and the azimuth, dip and rake (degrees) of the shared
// anisotropy (crates/variogram/src/{composite,aniso}.rs).
//
// For one system with bordered matrix K = [C 1; 1' 0], K [w; mu] = [c; 1]
// and z* = z'w, the adjoint K [lambda; nu] = [z; 0] gives
//   dz*/dtheta = lambda' dc/dtheta - lambda' dC/dtheta w,
// so with a = 2 (z* - z_i) lambda the system adds
//   sum_j a_j dc_j/dtheta - sum_jk a_j w_k dC_jk/dtheta
// to the gradient. C = L D L' is factored once (the forward's
// factorisation); w and lambda come from three solves (c, 1, z) on it. The
// covariance derivatives are recomputed pair by pair, never stored:
// C(h) = sum_s sill_s (1 - g_s(h / r_s)) for h > 0 and C(0) = C0, so
//   dC/dsill_s = 1 - g_s,  dC/dr_s = sill_s g_s'(t) h / r_s^2,
//   dC/dh = -sum_s sill_s g_s'(t) / r_s,  dh/dphi = (M d)' (dM/dphi d) / h
// for the lag h = |M d| of world offset d, M = diag(1, 1/semi, 1/minor) R.
//
// One warp per system (n <= 32), FP64 throughout, per-system partial sums
// written to a buffer and reduced in a fixed order (deterministic).
#include "btk_device.cuh"

namespace btk {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int R = 32;
constexpr int kMaxTheta = 1 + 2 * BTK_MAX_STRUCT + 5;

struct AdjSmem {
  double W[R][3];  // world coordinates of the samples
  double P[R][3];  // M (s - t)
  double T[R * (R - 1) / 2];
  double L[R][R + 1];
  double col[2][R];
  double rhs[2][4];
  double w[R], adj[R];
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ void tri_ij(int e, int& i, int& j) {
  int r = int((1.0f + sqrtf(8.0f * float(e) + 1.0f)) * 0.5f);
  while (r * (r - 1) / 2 > e) --r;
  while ((r + 1) * r / 2 <= e) ++r;
  i = r, j = e - r * (r - 1) / 2;
}

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

__global__ void __launch_bounds__(128) k_loo_grad(GradDev a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  AdjSmem& S = reinterpret_cast<AdjSmem*>(smem_raw)[threadIdx.x >> 5];
  const int ns = a.vg.nstruct;
  const int ntheta = 1 + 2 * ns + 5;
  const double c0 = a.vg.c0;
  const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
  for (int64_t i = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); i < a.n; i += warps) {
    __syncwarp();
    double* out = a.part + i * a.stride;
    const int64_t si = a.first + i;  // the left-out sample
    const int n = a.count[si];
    bool skip = a.sstatus[si] != BTK_ST_OK || n <= 0 || n > R;
    const bool have = !skip && lane < n;
    const double t[3] = {a.sx[si], a.sy[si], a.sz[si]};
    double w0 = 0, w1 = 0, w2 = 0, z = 0, err = 0;
    int tw = 0;
    if (have) {
      const uint32_t j = a.nbr[si * a.max_samples + lane];
      w0 = a.sx[j], w1 = a.sy[j], w2 = a.sz[j], z = a.sv[j];
      if (a.se) err = a.se[j];
      tw = a.twin[j];
    }
    // Systems holding coincident samples (merged by the reference's guard)
    // are left out of the loss and the gradient.
    skip = skip || __any_sync(kFull, tw != 0);
    if (skip) {
      if (lane == 0) {
        for (int k = 0; k < a.stride; ++k) out[k] = 0.0;
        if (a.value) a.value[si] = NAN;
      }
      continue;
    }
    double p[3] = {w0 - t[0], w1 - t[1], w2 - t[2]};
    {
      const double* M = a.vg.frame;
      const double r0 = M[0] * p[0] + M[1] * p[1] + M[2] * p[2];
      const double r1 = M[3] * p[0] + M[4] * p[1] + M[5] * p[2];
      const double r2 = M[6] * p[0] + M[7] * p[1] + M[8] * p[2];
      p[0] = r0, p[1] = r1, p[2] = r2;
    }
    if (have) {
      S.P[lane][0] = p[0], S.P[lane][1] = p[1], S.P[lane][2] = p[2];
      S.W[lane][0] = w0, S.W[lane][1] = w1, S.W[lane][2] = w2;
    }
    __syncwarp();
    const int E = n * (n - 1) / 2;
    for (int e = lane; e < E; e += R) {
      int r, q;
      tri_ij(e, r, q);
      const double dx = S.P[r][0] - S.P[q][0], dy = S.P[r][1] - S.P[q][1], dz = S.P[r][2] - S.P[q][2];
      S.T[e] = cov64(a.vg, sqrt(dx * dx + dy * dy + dz * dz));
    }
    const double hc = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    const double c = have ? cov64(a.vg, hc) : 0.0;
    __syncwarp();

    // LDL' with the forward substitutions of c, 1 and z fused in.
    double A[R];
    const int tri = lane * (lane - 1) / 2;
#pragma unroll
    for (int q = 0; q < R; ++q) A[q] = q < lane ? (have ? S.T[tri + q] : 0.0) : (q == lane ? (have ? c0 + err : 1.0) : 0.0);
    double y0 = have ? c : 0.0, y1 = have ? 1.0 : 0.0, y2 = have ? z : 0.0, dme = 1.0;
    bool sing = false;
#pragma unroll
    for (int k = 0; k < R; ++k) {
      if (k >= n) break;
      const int b = k & 1;
      S.col[b][lane] = A[k];
      if (lane == k) S.rhs[b][0] = y0, S.rhs[b][1] = y1, S.rhs[b][2] = y2;
      __syncwarp();
      const double dk = S.col[b][k];
      if (!(dk > kPivot * c0)) {
        sing = true;
        break;
      }
      if (lane == k) dme = dk;
      if (lane > k) {
        const double f = A[k] * (1.0 / dk);
#pragma unroll
        for (int q = k + 1; q < R; ++q) A[q] = fma(-f, S.col[b][q], A[q]);
        y0 = fma(-f, S.rhs[b][0], y0);
        y1 = fma(-f, S.rhs[b][1], y1);
        y2 = fma(-f, S.rhs[b][2], y2);
        A[k] = f;
      }
    }
    if (sing) {
      if (lane == 0) {
        for (int k = 0; k < a.stride; ++k) out[k] = 0.0;
        if (a.value) a.value[si] = NAN;
      }
      continue;
    }
    // Back substitution L' x = D^-1 y: x_c = C^-1 c, x_1 = C^-1 1, x_z = C^-1 z.
#pragma unroll
    for (int q = 0; q < R; ++q) S.L[lane][q] = A[q];
    double u0 = y0 / dme, u1 = y1 / dme, u2 = y2 / dme;
    __syncwarp();
    for (int k = n - 1; k >= 0; --k) {
      const int b = k & 1;
      if (lane == k) S.rhs[b][0] = u0, S.rhs[b][1] = u1, S.rhs[b][2] = u2;
      __syncwarp();
      if (lane < k) {
        const double l = S.L[k][lane];
        u0 = fma(-l, S.rhs[b][0], u0);
        u1 = fma(-l, S.rhs[b][1], u1);
        u2 = fma(-l, S.rhs[b][2], u2);
      }
    }
    if (!have) u0 = u1 = u2 = 0.0;
    const double sa = warp_sum(u0), sb = warp_sum(u1), se = warp_sum(u2);
    const double mu = (sa - 1.0) / sb;  // kernel.rs:93
    const double wl = u0 - mu * u1;     // weights
    const double est = warp_sum(have ? wl * z : 0.0);
    const double nu = se / sb;
    const double lam = u2 - nu * u1;  // adjoint weights
    const double resid = est - a.sv[si];
    const double adj = have ? 2.0 * resid * lam : 0.0;
    if (lane == 0) {
      out[0] = resid * resid;
      out[1] = 1.0;
      if (a.value) a.value[si] = est;
    }
    if (!a.want_grad) continue;
    S.w[lane] = have ? wl : 0.0, S.adj[lane] = adj;
    __syncwarp();
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
        const double d[3] = {w0 - t[0], w1 - t[1], w2 - t[2]};
        add_lag_terms(a, adj, hc, p, d, g);
      } else {
        g[0] += adj;
        for (int s = 0; s < ns; ++s) g[1 + s] += adj;
      }
    }
    for (int e = lane; e < E; e += R) {  // sample pairs (r > q)
      int r, q;
      tri_ij(e, r, q);
      const double coef = -(S.adj[r] * S.w[q] + S.adj[q] * S.w[r]);
      const double Md[3] = {S.P[r][0] - S.P[q][0], S.P[r][1] - S.P[q][1], S.P[r][2] - S.P[q][2]};
      const double d[3] = {S.W[r][0] - S.W[q][0], S.W[r][1] - S.W[q][1], S.W[r][2] - S.W[q][2]};
      const double h = sqrt(Md[0] * Md[0] + Md[1] * Md[1] + Md[2] * Md[2]);
      if (h > 0.0) add_lag_terms(a, coef, h, Md, d, g);
    }
    for (int k = 0; k < ntheta; ++k) {
      const double v = warp_sum(g[k]);
      if (lane == 0) out[2 + k] = v;
    }
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

}  // namespace

cudaError_t launch_loo_grad(const Launch& L, const GradDev& a, double* sums) {
  const size_t smem = sizeof(AdjSmem) * 4;
  cudaError_t e = cudaFuncSetAttribute(k_loo_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_loo_grad, 128, smem);
  if (e != cudaSuccess) return e;
  int64_t blocks = int64_t(L.sm_count) * (per_sm > 0 ? per_sm : 1);
  const int64_t need = (a.n + 3) / 4;
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
  k_loo_grad<<<int(blocks), 128, smem, L.stream>>>(a);
  k_col_sums<<<a.stride, 256, 0, L.stream>>>(a.n, a.stride, a.part, sums);
  *L.counter += 2;
  return cudaGetLastError();
}

}  // namespace btk
