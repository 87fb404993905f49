// Search calibration on the device: crates/py/src/estimation.rs:846-895
// (Method::calibrated) with crates/estimation/src/kriging_algebra.rs:336-412
// (prefix_quality, calibrated_count) and search.rs:913-936 (balanced).
//
// Between the search and the solve, each target's neighbour list is, with
// octants or sectors, reordered round-robin over the sectors, each sector in
// selection order; then one Cholesky factorisation of its covariance matrix
// gives the slope of regression and kriging efficiency of every leading part,
// and the count is cut to the fewest leading samples, from min_samples, that
// reach the target (all of them where none does). The solve kernels then
// krige the cut lists as they krige any other.
//
// One CTA of 128 threads per target, the matrix in shared memory (right-
// looking Cholesky, one barrier per column), the forward solves of the
// right-hand side and of the ones column by column sweeps, the prefix scan by
// one thread.
#include "btk_device.cuh"

namespace btk {
namespace {

constexpr int kThreads = 128;
constexpr int kMaxSectors = 360;

struct CalHead {
  int64_t ti;
  int n, kind, fail;
  double t[3];
  int rank[kMaxLU];
  uint32_t idx[kMaxLU];
  int count[kMaxSectors];
};

struct CalLayout {
  size_t p, e, y, z, yo, zo, c, total;
  int stride;
};

__host__ __device__ inline size_t cal_align(size_t v) { return (v + 15) & ~size_t(15); }

__host__ __device__ inline CalLayout cal_layout(int kmax) {
  CalLayout l;
  l.stride = kmax | 1;
  l.p = cal_align(sizeof(CalHead));
  l.e = l.p + sizeof(double) * 3 * kmax;
  l.y = l.e + sizeof(double) * kmax;
  l.z = l.y + sizeof(double) * kmax;
  l.yo = l.z + sizeof(double) * kmax;
  l.zo = l.yo + sizeof(double) * kmax;
  l.c = cal_align(l.zo + sizeof(double) * kmax);
  l.total = l.c + sizeof(double) * size_t(kmax) * l.stride;
  return l;
}

__global__ void __launch_bounds__(kThreads) k_calibrate(SolveDev a, SearchDev sp, CalDev c, int kmax) {
  extern __shared__ __align__(16) unsigned char smem[];
  const CalLayout lay = cal_layout(kmax);
  CalHead& H = *reinterpret_cast<CalHead*>(smem);
  double* P = reinterpret_cast<double*>(smem + lay.p);  // [3][kmax], world
  double* E = reinterpret_cast<double*>(smem + lay.e);
  double* Y = reinterpret_cast<double*>(smem + lay.y);    // right-hand side, swept in place
  double* Z = reinterpret_cast<double*>(smem + lay.z);    // ones, swept in place
  double* YO = reinterpret_cast<double*>(smem + lay.yo);  // L^-1 rhs
  double* ZO = reinterpret_cast<double*>(smem + lay.zo);  // L^-1 1
  double* C = reinterpret_cast<double*>(smem + lay.c);    // lower triangle, row-major
  const int S = lay.stride;
  const int tid = threadIdx.x;
  const int64_t nitems = a.perm ? a.nwork : a.m;
  const VgDev& vg = a.vg;
  for (int64_t item = blockIdx.x; item < nitems; item += gridDim.x) {
    __syncthreads();
    if (tid == 0) {
      const int64_t ti = a.perm ? a.perm[item] : item;
      H.ti = -1;
      if (ti >= 0) {
        const int n = c.count[ti];
        c.met[ti] = -1;
        if (a.sstatus[ti] == BTK_ST_OK && n > 0 && n <= kmax) {
          H.ti = ti, H.n = n, H.fail = 0;
          H.kind = a.kinds ? int(a.kinds[ti]) : a.kind;
          H.t[0] = a.tx[ti], H.t[1] = a.ty[ti], H.t[2] = a.tz[ti];
        }
      }
    }
    __syncthreads();
    const int64_t ti = H.ti;
    if (ti < 0) continue;
    const int n = H.n;
    uint32_t* row = c.nbr + ti * a.max_samples;
    if (c.balance) {  // search.rs:913-936: a stable sort by the rank within the sector
      if (tid == 0) {
        const int nsec = sp.plane ? sp.plane : (sp.planar ? 4 : 8);
        for (int q = 0; q < nsec; ++q) H.count[q] = 0;
        int top = 0;
        for (int i = 0; i < n; ++i) {
          const uint32_t j = row[i];
          const double w[3] = {a.sx[j], a.sy[j], a.sz[j]};
          const int o = search_sector(sp, w, H.t);
          H.idx[i] = j;
          H.rank[i] = ++H.count[o];
          top = H.rank[i] > top ? H.rank[i] : top;
        }
        int out = 0;
        for (int r = 1; r <= top; ++r)
          for (int i = 0; i < n; ++i)
            if (H.rank[i] == r) row[out++] = H.idx[i];
      }
      __syncthreads();
    }
    for (int r = tid; r < n; r += kThreads) {
      const uint32_t j = row[r];
      P[r] = a.sx[j], P[kmax + r] = a.sy[j], P[2 * kmax + r] = a.sz[j];
      E[r] = a.se ? a.se[j] : 0.0;
    }
    __syncthreads();
    // Covariance matrix (error variances on the diagonal) and right-hand side.
    for (int e = tid; e < n * n; e += kThreads) {
      const int i = e / n, j = e % n;
      if (j > i) continue;
      C[i * S + j] = i == j ? vg.c0 + E[i]
                            : cov64(vg, lag_world(vg, P[j], P[kmax + j], P[2 * kmax + j], P[i], P[kmax + i],
                                                  P[2 * kmax + i]));
    }
    for (int i = tid; i < n; i += kThreads) {
      Y[i] = support_cov(a, H.t[0], H.t[1], H.t[2], P[i], P[kmax + i], P[2 * kmax + i]);
      Z[i] = 1.0;
    }
    __syncthreads();
    // Cholesky, right-looking; not positive definite makes every part None.
    for (int k = 0; k < n; ++k) {
      const double piv = C[k * S + k];
      if (!(piv > 0.0)) {  // uniform: every thread read the same pivot
        if (tid == 0) H.fail = 1;
        break;
      }
      const double lkk = sqrt(piv);
      __syncthreads();
      if (tid == 0) C[k * S + k] = lkk;
      for (int i = k + 1 + tid; i < n; i += kThreads) C[i * S + k] = C[i * S + k] / lkk;
      __syncthreads();
      const int rest = n - k - 1;
      for (int e = tid; e < rest * rest; e += kThreads) {
        const int i = k + 1 + e / rest, j = k + 1 + e % rest;
        if (j <= i) C[i * S + j] -= C[i * S + k] * C[j * S + k];
      }
      __syncthreads();
    }
    __syncthreads();
    if (H.fail) {
      if (tid == 0) c.met[ti] = 0;  // every part None: all the samples, not met
      continue;
    }
    // Forward solves L yo = rhs, L zo = 1, column by column.
    for (int i = 0; i < n; ++i) {
      const double cy = Y[i] / C[i * S + i], cz = Z[i] / C[i * S + i];
      for (int r = i + 1 + tid; r < n; r += kThreads) {
        Y[r] -= cy * C[r * S + i];
        Z[r] -= cz * C[r * S + i];
      }
      if (tid == 0) YO[i] = cy, ZO[i] = cz;
      __syncthreads();
    }
    if (tid == 0) {  // prefix_quality's scan and calibrated_count
      const bool ordinary = H.kind != BTK_SIMPLE;
      const double sv = a.sup_n > 0 ? *a.sup_cbb : vg.c0;
      const int from = c.min_samples > 1 ? c.min_samples : 1;
      double sy = 0.0, qa = 0.0, qb = 0.0;
      int keep = n, met = 0;
      for (int k = 0; k < n; ++k) {
        sy += YO[k] * YO[k];
        double cov = sy, mu = 0.0;
        bool some = true;
        if (ordinary) {
          qa += ZO[k] * ZO[k];
          qb += ZO[k] * YO[k];
          if (qa > 0.0) {
            const double l = sqrt(qa);  // the 1 x 1 Cholesky factor of Z^T C^-1 Z and its solve
            const double m = ((qb - 1.0) / l) / l;
            cov = sy - m * qb;
            mu = m;
          } else {
            some = false;
          }
        }
        if (!some || k + 1 < from) continue;
        const double q = c.calibration == 1 ? cov / (cov - mu) : (cov + mu) / sv;
        if (q >= c.target) {
          keep = k + 1, met = 1;
          break;
        }
      }
      c.count[ti] = keep;
      c.met[ti] = int8_t(met);
    }
  }
}

}  // namespace

cudaError_t launch_calibrate(const Launch& L, const SolveDev& a, const SearchDev& sp, const CalDev& c, int kmax) {
  if (kmax < 1 || kmax > kMaxLU || (c.calibration != 1 && c.calibration != 2)) return cudaErrorInvalidValue;
  if (sp.plane > kMaxSectors) return cudaErrorInvalidValue;
  const size_t smem = cal_layout(kmax).total;
  cudaError_t e = cudaFuncSetAttribute(k_calibrate, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_calibrate, kThreads, smem);
  if (e != cudaSuccess) return e;
  int64_t blocks = int64_t(L.sm_count) * (per_sm > 0 ? per_sm : 1);
  const int64_t items = a.perm ? a.nwork : a.m;
  if (blocks > items) blocks = items;
  if (blocks < 1) return cudaSuccess;
  k_calibrate<<<int(blocks), kThreads, smem, L.stream>>>(a, sp, c, kmax);
  ++*L.counter;
  return cudaGetLastError();
}

}  // namespace btk
