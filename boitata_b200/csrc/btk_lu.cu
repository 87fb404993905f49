// Dense LU solve of the bordered kriging system, FP64, one CTA per system:
// crates/estimation/src/krige.rs:127-201 (krige_lu), the reference's path
// beyond kernel.rs (kernel.rs:11): systems of more than 64 samples, and
// variograms that are not stationary (a power structure, composite.rs:64-66),
// whose bordered matrix is not positive definite.
//
// The system and its LU live in shared memory up to 128 samples; beyond, the
// matrix lives in a per-CTA slice of a global scratch buffer (one CTA per
// SM), the rest of the system in shared memory. The factorisation follows
// nalgebra 0.33's LU (lu.rs: partial pivoting on the first largest |a_ri| of
// the column, a zero pivot column skipped, the column scaled by 1 / pivot,
// the trailing block updated); solve applies the row swaps in order, then the
// unit-lower and upper substitutions, and a zero U diagonal makes the system
// singular, as LU::solve returning None does. The coincident guard
// (coincident.rs:27-111) and block support apply as in the other solve paths.
//
// The diagnostics form (DIAG) takes every system the solve estimated (status
// OK) and writes only the table columns that need the samples or weights
// (crates/py/src/estimation.rs:1046-1105): the negative weight sum of the
// weights spread over coincident samples as coincident.rs:98-104 spreads them,
// the mean Euclidean distance to the samples used, and their distinct holes.
#include "btk_device.cuh"

namespace btk {
namespace {

constexpr unsigned kFull = 0xffffffffu;

struct LuHead {
  int64_t ti;
  double t[3];
  int n, nn, dim, kind, twin, sing, nperm;
  int piv[2];        // pivot row of the column, double-buffered by column parity
  double pv[2];      // and its value
  // Look-ahead: each warp's first largest |a_r,k+1| over its rows after column
  // k's update (value, signed value, row), double-buffered by column parity.
  double wabs[2][16], wval[2][16];
  int wrow[2][16];
};

struct LuLayout {
  size_t head, p, e, f, b, x, perm, clus, a, total;
  int stride;
};

__host__ __device__ inline size_t align16(size_t v) { return (v + 15) & ~size_t(15); }

// Shared-memory layout of one system of at most kmax samples. With `global`
// the bordered matrix lives in the CTA's slice of a global scratch buffer
// instead (systems beyond kMaxLU samples, whose matrix does not fit).
__host__ __device__ inline LuLayout lu_layout(int kmax, bool global = false) {
  LuLayout l;
  const int dmax = kmax + 1;
  l.stride = dmax | 1;
  l.head = 0;
  l.p = align16(sizeof(LuHead));
  l.e = l.p + sizeof(double) * 3 * kmax;
  l.f = l.e + sizeof(double) * kmax;
  l.b = l.f + sizeof(double) * kmax;
  l.x = l.b + sizeof(double) * dmax;
  l.perm = l.x + sizeof(double) * dmax;
  l.clus = l.perm + sizeof(int) * 2 * dmax;  // cluster of each sample, first member and size of each cluster
  l.a = align16(l.clus + sizeof(int) * 3 * kmax);
  l.total = global ? l.a : l.a + sizeof(double) * size_t(dmax) * l.stride;
  return l;
}

// Doubles of one system's matrix in the global scratch (GA form).
__host__ __device__ inline size_t lu_matrix_doubles(int kmax) {
  const int dmax = kmax + 1;
  return size_t(dmax) * size_t(dmax | 1);
}

// NT threads per system: 128 up to 64 samples, 512 beyond (one system per SM
// then, its matrix filling most of the shared memory). GA: the matrix in the
// CTA's slice of a.lu_scratch (beyond kMaxLU samples).
// Launch bounds: given only the block size, the compiler held the 512-thread
// form to 64 registers and spilled; a minimum of one CTA an SM (its matrix
// fills the shared memory) leaves it about 100, without spills. The
// 128-thread form (at most 65 columns) keeps the compiler's own choice (no
// minimum): 64 registers, no spills.
template <bool DIAG, int NT, bool GA = false>
__global__ void __launch_bounds__(NT, NT > 128 ? 1 : 0) k_solve_lu(SolveDev a, int kmax) {
  constexpr int kThreads = NT, kWarps = NT / 32;
  extern __shared__ __align__(16) unsigned char smem[];
  const LuLayout lay = lu_layout(kmax, GA);
  LuHead& H = *reinterpret_cast<LuHead*>(smem + lay.head);
  int* cof = reinterpret_cast<int*>(smem + lay.clus);
  int* cfirst = cof + kmax;
  int* csize = cfirst + kmax;
  double* P = reinterpret_cast<double*>(smem + lay.p);  // [3][kmax], world
  double* E = reinterpret_cast<double*>(smem + lay.e);
  double* F = reinterpret_cast<double*>(smem + lay.f);  // f(z)
  double* B = reinterpret_cast<double*>(smem + lay.b);
  double* X = reinterpret_cast<double*>(smem + lay.x);
  int* pa = reinterpret_cast<int*>(smem + lay.perm);
  int* pb = pa + kmax + 1;
  double* A = GA ? a.lu_scratch + size_t(blockIdx.x) * lu_matrix_doubles(kmax)
                 : reinterpret_cast<double*>(smem + lay.a);
  const int S = lay.stride;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t nitems = a.list ? *a.list_len : (a.perm ? a.nwork : a.m);
  const VgDev& vg = a.vg;
  for (int64_t item = blockIdx.x; item < nitems; item += gridDim.x) {
    __syncthreads();
    if (tid == 0) {
      int64_t ti = a.list ? a.list[item] : (a.perm ? a.perm[item] : item);
      H.ti = ti, H.n = 0, H.twin = 0, H.sing = 0, H.nperm = 0;
      if (ti >= 0) {
        const int n = a.count[ti];
        const int8_t st = DIAG ? int8_t(a.status[ti] & 0x0F) : a.sstatus[ti];
        H.kind = a.kinds ? int(a.kinds[ti]) : a.kind;
        H.t[0] = a.tx[ti], H.t[1] = a.ty[ti], H.t[2] = a.tz[ti];
        if (DIAG) {
          if (a.negw) a.negw[ti] = NAN;
          if (a.mdist) a.mdist[ti] = NAN;
          if (a.nholes) a.nholes[ti] = 0;
          if (st != BTK_ST_OK || n <= 0 || n > kmax) H.ti = -1;
          else H.n = n;
        } else if (st != BTK_ST_OK) {
          write_fail(a, ti, st, 0);
          H.ti = -1;
        } else if (n <= 0) {
          write_fail(a, ti, BTK_ST_SEARCH_FAILED, 0);
          H.ti = -1;
        } else if (n > kmax) {
          write_fail(a, ti, BTK_ST_UNSUPPORTED, 0);
          H.ti = -1;
        } else if (H.kind == BTK_SIMPLE && !vg.stationary) {  // check_simple (krige.rs:117-124)
          write_fail(a, ti, BTK_ST_INVALID, 0);
          H.ti = -1;
        } else {
          H.n = n;
        }
      }
    }
    __syncthreads();
    const int64_t ti = H.ti;
    if (ti < 0) continue;
    const int n = H.n;
    for (int r = tid; r < n; r += kThreads) {
      const uint32_t j = a.nbr[ti * a.max_samples + r];
      P[r] = a.sx[j], P[kmax + r] = a.sy[j], P[2 * kmax + r] = a.sz[j];
      E[r] = a.se ? a.se[j] : 0.0;
      F[r] = kind_f(H.kind, a.kparam, a.sv[j]);
      if (a.twin && a.twin[j]) H.twin = 1;
    }
    __syncthreads();
    if (tid == 0) {
      if (DIAG) {  // neighborhood_stats over the samples used (neighborhood.rs:76-98)
        for (int i = 0; i < n; ++i) {  // distances, insertion-sorted ascending (a stable sort)
          const double dx = P[i] - H.t[0], dy = P[kmax + i] - H.t[1], dz = P[2 * kmax + i] - H.t[2];
          const double d = sqrt(dx * dx + dy * dy + dz * dz);
          int q = i;
          while (q > 0 && B[q - 1] > d) B[q] = B[q - 1], --q;
          B[q] = d;
        }
        double sum = 0.0;
        for (int i = 0; i < n; ++i) sum += B[i];
        if (a.mdist) a.mdist[ti] = sum / double(n);
        int holes = n;
        if (a.hole) {
          holes = 0;
          for (int i = 0; i < n; ++i) {
            const uint32_t h = a.hole[a.nbr[ti * a.max_samples + i]];
            bool seen = false;
            for (int q = 0; q < i && !seen; ++q) seen = a.hole[a.nbr[ti * a.max_samples + q]] == h;
            holes += seen ? 0 : 1;
          }
        }
        if (a.nholes) a.nholes[ti] = holes;
      }
      int nn = n;
      if (H.twin) {  // coincident guard, as merge_clusters in btk_solve.cu
        const double eps2 = kEps * kEps;
        int nc = 0;
        for (int i = 0; i < n; ++i) {
          int c = -1;
          for (int q = 0; q < nc && c < 0; ++q) {
            const int f = cfirst[q];
            if (d2_exact(P[f], P[kmax + f], P[2 * kmax + f], P[i], P[kmax + i], P[2 * kmax + i]) <= eps2) c = q;
          }
          if (c < 0) c = nc, cfirst[nc] = i, csize[nc] = 0, ++nc;
          cof[i] = c;
          csize[c] += 1;
        }
        for (int c = 0; c < nc; ++c) {
          const int f = cfirst[c];
          double x0 = P[f], x1 = P[kmax + f], x2 = P[2 * kmax + f], err = E[f], zb = F[f];
          if (csize[c] > 1) {
            const double k = double(csize[c]);
            double var = 0.0, zs = 0.0;
            for (int i = f; i < n; ++i) {
              if (cof[i] != c) continue;
              var += E[i];
              zs += F[i];
              for (int j = f; j < n; ++j)
                if (cof[j] == c)
                  var += cov64(vg, lag_world(vg, P[i], P[kmax + i], P[2 * kmax + i], P[j], P[kmax + j],
                                             P[2 * kmax + j]));
            }
            err = var / (k * k) - vg.c0;
            zb = zs / k;
          }
          P[c] = x0, P[kmax + c] = x1, P[2 * kmax + c] = x2, E[c] = err, F[c] = zb;
        }
        nn = nc;
      }
      H.nn = nn;
      H.dim = H.kind == BTK_SIMPLE ? nn : nn + 1;
    }
    __syncthreads();
    const int nn = H.nn, dim = H.dim;
    const double t0 = H.t[0], t1 = H.t[1], t2 = H.t[2];
    // The bordered system (krige.rs:150-166) and its right-hand side: the
    // lower triangle and the diagonal, each entry written to both halves
    // (lag_world is symmetric to the bit).
    for (int e = tid; e < dim * (dim + 1) / 2; e += kThreads) {
      int i, j;
      tri_index(e, i, j);  // (i + 1, j): the strict lower triangle of dim + 1 rows
      i -= 1;
      double v;
      if (i < nn && j < nn)
        v = i == j ? vg.c0 + E[i]
                   : cov64(vg, lag_world(vg, P[j], P[kmax + j], P[2 * kmax + j], P[i], P[kmax + i], P[2 * kmax + i]));
      else
        v = (i == nn && j == nn) ? 0.0 : 1.0;
      A[i * S + j] = v;
      A[j * S + i] = v;
    }
    for (int i = tid; i < dim; i += kThreads) {
      const double v = i < nn ? support_cov(a, t0, t1, t2, P[i], P[kmax + i], P[2 * kmax + i]) : 1.0;
      B[i] = v, X[i] = v;
    }
    __syncthreads();
    if constexpr (NT > 128) {
    // LU with partial pivoting (nalgebra lu.rs), the 512-thread form: per column k the first largest
    // |a_rk| (r >= k) is the pivot; rows k and the pivot swap; each warp scales
    // and updates its rows below k (row k is only read meanwhile). Column k's
    // pivot comes from column k - 1's update (look-ahead): lane 0 of each warp
    // keeps the first largest |a_r,k| over the warp's rows (ascending) as it
    // writes them, and after the column's barrier every thread reduces the
    // warps' candidates, larger value first and the lower row on a tie, which
    // is the first largest over all rows. Column 0, and a column after a
    // skipped one, take warp 0's search instead. Each lane keeps the pivot
    // row's entries of its columns in registers for all of its warp's rows.
    // Columns a lane caches: all of them while dim - k - 1 <= 32 kCache (dim up to 161).
    constexpr int kCache = 5;
    bool ahead = false;        // uniform: piv and diag hold column k's pivot
    int piv = 0;
    double diag = 0.0;
    for (int k = 0; k < dim; ++k) {
      const int b = k & 1;
      if (!ahead) {
        if (warp == 0) {
          double bv = -1.0;
          int bi = k;
          for (int r = k + lane; r < dim; r += 32) {
            const double v = fabs(A[r * S + k]);
            if (v > bv) bv = v, bi = r;
          }
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            const double v2 = __shfl_xor_sync(kFull, bv, o);
            const int i2 = __shfl_xor_sync(kFull, bi, o);
            if (v2 > bv || (v2 == bv && i2 < bi)) bv = v2, bi = i2;
          }
          if (lane == 0) H.piv[b] = bi, H.pv[b] = A[bi * S + k];
        }
        __syncthreads();
        piv = H.piv[b], diag = H.pv[b];
      }
      ahead = false;
      if (diag == 0.0) continue;  // uniform: a zero column is skipped
      if (piv != k) {
        for (int j = tid; j < dim; j += kThreads) {
          const double tmp = A[k * S + j];
          A[k * S + j] = A[piv * S + j];
          A[piv * S + j] = tmp;
        }
        if (tid == 0) pa[H.nperm] = k, pb[H.nperm] = piv, ++H.nperm;
        __syncthreads();
      }
      const double inv = 1.0 / diag;
      double prow[kCache];
#pragma unroll
      for (int q = 0; q < kCache; ++q) {
        const int c = k + 1 + lane + 32 * q;
        prow[q] = c < dim ? A[k * S + c] : 0.0;
      }
      double bv = -1.0, sv = 0.0;
      int bi = k + 1;
      for (int r = k + 1 + warp; r < dim; r += kWarps) {
        const double l = A[r * S + k] * inv;
        __syncwarp();
        if (lane == 0) A[r * S + k] = l;
#pragma unroll
        for (int q = 0; q < kCache; ++q) {
          const int c = k + 1 + lane + 32 * q;
          if (c < dim) {
            const double v = fma(-prow[q], l, A[r * S + c]);
            A[r * S + c] = v;
            if (q == 0 && lane == 0 && fabs(v) > bv) bv = fabs(v), sv = v, bi = r;
          }
        }
        for (int c = k + 1 + lane + 32 * kCache; c < dim; c += 32) A[r * S + c] = fma(-A[k * S + c], l, A[r * S + c]);
      }
      if (lane == 0) H.wabs[b][warp] = bv, H.wval[b][warp] = sv, H.wrow[b][warp] = bi;
      __syncthreads();
      if (k + 1 < dim) {
        double best = -1.0, val = 0.0;
        int row = k + 1;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
          const double v = H.wabs[b][w];
          const int i = H.wrow[b][w];
          if (v > best || (v == best && i < row)) best = v, val = H.wval[b][w], row = i;
        }
        // No row's |a| exceeded -1 (all NaN): row k + 1 with its own value, as the search gives.
        piv = row, diag = best < 0.0 ? A[(k + 1) * S + k + 1] : val;
        ahead = true;
      }
    }
    } else {
    // LU with partial pivoting (nalgebra lu.rs), the 128-thread form (at most
    // 65 columns): per column, warp 0 finds the first largest |a_rk| (r >= k);
    // rows k and the pivot swap; each warp scales and updates its rows below k
    // (row k is only read meanwhile). The look-ahead of the 512-thread form
    // costs more than it saves at this size (32-sample power models: 9.3
    // against 10.6 M systems/s).
    for (int k = 0; k < dim; ++k) {
      const int b = k & 1;
      if (warp == 0) {
        double bv = -1.0;
        int bi = k;
        for (int r = k + lane; r < dim; r += 32) {
          const double v = fabs(A[r * S + k]);
          if (v > bv) bv = v, bi = r;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const double v2 = __shfl_xor_sync(kFull, bv, o);
          const int i2 = __shfl_xor_sync(kFull, bi, o);
          if (v2 > bv || (v2 == bv && i2 < bi)) bv = v2, bi = i2;
        }
        if (lane == 0) H.piv[b] = bi, H.pv[b] = A[bi * S + k];
      }
      __syncthreads();
      const int piv = H.piv[b];
      const double diag = H.pv[b];
      if (diag == 0.0) continue;  // uniform: a zero column is skipped
      if (piv != k) {
        for (int j = tid; j < dim; j += kThreads) {
          const double tmp = A[k * S + j];
          A[k * S + j] = A[piv * S + j];
          A[piv * S + j] = tmp;
        }
        if (tid == 0) pa[H.nperm] = k, pb[H.nperm] = piv, ++H.nperm;
        __syncthreads();
      }
      const double inv = 1.0 / diag;
      for (int r = k + 1 + warp; r < dim; r += kWarps) {
        const double l = A[r * S + k] * inv;
        __syncwarp();
        if (lane == 0) A[r * S + k] = l;
        for (int c = k + 1 + lane; c < dim; c += 32) A[r * S + c] = fma(-A[k * S + c], l, A[r * S + c]);
      }
      __syncthreads();
    }
    }
    // LU::solve: row swaps, then L (unit lower) and U substitutions.
    if constexpr (NT > 128) {
      // Blocked by 32 rows: warp 0 solves the diagonal block with the block's
      // unknowns in registers (lane = row), then every thread applies the
      // block's solved entries to one row beyond it. Each row still takes its
      // updates one column at a time in the serial order (ascending for L,
      // descending for U) with the same FMAs, so X is the serial solve's to
      // the bit; the block's other warps no longer wait on warp 0.
      if (tid == 0)
        for (int q = 0; q < H.nperm; ++q) {
          const double tmp = X[pa[q]];
          X[pa[q]] = X[pb[q]];
          X[pb[q]] = tmp;
        }
      __syncthreads();
      const int nblk = (dim + 31) / 32;
      for (int j = 0; j < nblk; ++j) {
        const int j0 = 32 * j, j1 = min(dim, j0 + 32);
        if (warp == 0) {
          const int r = j0 + lane;
          double x = r < j1 ? X[r] : 0.0;
          for (int i = j0; i < j1; ++i) {
            const double coeff = __shfl_sync(kFull, x, i - j0);
            if (r > i && r < j1) x = fma(-coeff, A[r * S + i], x);
          }
          if (r < j1) X[r] = x;
        }
        __syncthreads();
        for (int r = j1 + tid; r < dim; r += kThreads) {
          double x = X[r];
          for (int i = j0; i < j1; ++i) x = fma(-X[i], A[r * S + i], x);
          X[r] = x;
        }
        __syncthreads();
      }
      for (int j = nblk - 1; j >= 0; --j) {
        const int j0 = 32 * j, j1 = min(dim, j0 + 32);
        if (warp == 0) {
          const int r = j0 + lane;
          double x = r < j1 ? X[r] : 0.0;
          bool sing = false;
          for (int i = j1 - 1; i >= j0; --i) {
            const double d = A[i * S + i];
            if (d == 0.0) {  // uniform over the warp
              sing = true;
              break;
            }
            const double coeff = __shfl_sync(kFull, x / d, i - j0);
            if (r == i) x = coeff;
            else if (r < i && r >= j0) x = fma(-coeff, A[r * S + i], x);
          }
          if (r < j1) X[r] = x;
          if (lane == 0 && sing) H.sing = 1;
        }
        __syncthreads();
        if (H.sing) break;  // uniform: every thread read it after the barrier
        for (int r = tid; r < j0; r += kThreads) {
          double x = X[r];
          for (int i = j1 - 1; i >= j0; --i) x = fma(-X[i], A[r * S + i], x);
          X[r] = x;
        }
        __syncthreads();
      }
    } else if (warp == 0) {
      if (lane == 0)
        for (int q = 0; q < H.nperm; ++q) {
          const double tmp = X[pa[q]];
          X[pa[q]] = X[pb[q]];
          X[pb[q]] = tmp;
        }
      __syncwarp();
      for (int i = 0; i < dim; ++i) {
        const double coeff = X[i];
        for (int r = i + 1 + lane; r < dim; r += 32) X[r] = fma(-coeff, A[r * S + i], X[r]);
        __syncwarp();
      }
      for (int i = dim - 1; i >= 0; --i) {
        const double d = A[i * S + i];
        if (d == 0.0) {  // uniform over the warp
          if (lane == 0) H.sing = 1;
          break;
        }
        const double coeff = X[i] / d;
        __syncwarp();
        if (lane == 0) X[i] = coeff;
        for (int r = lane; r < i; r += 32) X[r] = fma(-coeff, A[r * S + i], X[r]);
        __syncwarp();
      }
    }
    __syncthreads();
    if (DIAG) {
      if (tid == 0 && !H.sing && a.negw) {  // krige.rs:70-75 over the spread weights
        double neg = -0.0;
        for (int i = 0; i < n; ++i) {
          const double w = H.twin ? X[cof[i]] / double(csize[cof[i]]) : X[i];
          if (w < 0.0) neg += w;
        }
        a.negw[ti] = neg;
      }
      if (!H.sing && a.wout)  // Estimate::weights, one per sample of the list (batch.rs:76-95)
        for (int i = tid; i < n; i += NT)
          a.wout[ti * a.max_samples + i] = H.twin ? X[cof[i]] / double(csize[cof[i]]) : X[i];
      continue;
    }
    if (tid == 0) {
      if (H.sing) {
        write_fail(a, ti, BTK_ST_SINGULAR, 0);
      } else {  // krige.rs:177-200
        double value = 0.0, swc = 0.0;
        for (int i = 0; i < nn; ++i) value += X[i] * F[i], swc += X[i] * B[i];
        const int kind = H.kind;
        if (kind == BTK_SIMPLE) value = a.kparam + value;
        if (kind == BTK_INDICATOR) value = value < 0.0 ? 0.0 : (value > 1.0 ? 1.0 : value);
        const double mu = kind == BTK_SIMPLE ? 0.0 : X[nn];
        const double cb = a.sup_n > 0 ? *a.sup_cbb : vg.c0;
        a.value[ti] = value;
        if (a.variance) a.variance[ti] = fmax(cb - swc - mu, 0.0);
        if (a.lagrange) a.lagrange[ti] = mu;
        if (a.n_used) a.n_used[ti] = n;
        if (a.status) a.status[ti] = BTK_ST_OK;
      }
    }
  }
}

}  // namespace

size_t lu_scratch_doubles(int sm_count, int kmax) {
  return kmax > kMaxLU ? size_t(sm_count) * lu_matrix_doubles(kmax) : 0;
}

cudaError_t launch_solve_lu(const Launch& L, const SolveDev& a, int kmax, bool diag) {
  if (kmax < 1 || kmax > kMaxLUGlobal) return cudaErrorInvalidValue;
  if (diag && !a.status) return cudaErrorInvalidValue;
  const bool global = kmax > kMaxLU;
  if (global && !a.lu_scratch) return cudaErrorInvalidValue;
  const size_t smem = lu_layout(kmax, global).total;
  const bool wide = kmax > 64;
  const int threads = wide ? 512 : 128;
  auto kern = global ? (diag ? k_solve_lu<true, 512, true> : k_solve_lu<false, 512, true>)
                     : diag ? (wide ? k_solve_lu<true, 512> : k_solve_lu<true, 128>)
                            : (wide ? k_solve_lu<false, 512> : k_solve_lu<false, 128>);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  if (e != cudaSuccess) return e;
  // The global form: one CTA per SM, each with its own slice of the scratch.
  int64_t blocks = int64_t(L.sm_count) * (global ? 1 : (per_sm > 0 ? per_sm : 1));
  const int64_t items = a.perm ? a.nwork : a.m;
  if (!a.list && blocks > items) blocks = items;
  if (blocks < 1) blocks = 1;
  kern<<<int(blocks), threads, smem, L.stream>>>(a, kmax);
  ++*L.counter;
  return cudaGetLastError();
}

}  // namespace btk
