// Groups of NW warps (32 NW threads) that work on one system together: the
// barrier, and the reductions over the group through a small shared-memory
// scratch (any struct with `double red[NW][8]` and `int ired[NW]`). With
// NW = 1 they are warp shuffles and __syncwarp; with NW = 2 a named barrier
// (one per group, ids 1..) joins the two warps.
#pragma once

#include <cuda_runtime.h>

namespace btk {

constexpr unsigned kFull = 0xffffffffu;

template <int NW>
__device__ __forceinline__ void gsync(int gid) {
  if (NW == 1)
    __syncwarp();
  else
    asm volatile("bar.sync %0, %1;" ::"r"(gid + 1), "r"(NW * 32) : "memory");
}

template <int NW, class Sm>
__device__ __forceinline__ bool group_any(Sm& S, int gid, int wig, bool pred) {
  int v = __any_sync(kFull, pred);
  if (NW == 1) return v != 0;
  if ((threadIdx.x & 31) == 0) S.ired[wig] = v;
  gsync<NW>(gid);
  int all = 0;
#pragma unroll
  for (int w = 0; w < NW; ++w) all |= S.ired[w];
  gsync<NW>(gid);
  return all != 0;
}

// Sums of K <= 8 values over the group, returned on every lane.
template <int NW, int K, class Sm>
__device__ __forceinline__ void group_sum(Sm& S, int gid, int wig, double v[K]) {
#pragma unroll
  for (int q = 0; q < K; ++q)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(kFull, v[q], o);
  if (NW == 1) return;
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int q = 0; q < K; ++q) S.red[wig][q] = v[q];
  gsync<NW>(gid);
#pragma unroll
  for (int q = 0; q < K; ++q) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < NW; ++w) s += S.red[w][q];
    v[q] = s;
  }
  gsync<NW>(gid);
}

template <int NW, class Sm>
__device__ __forceinline__ void group_sum5(Sm& S, int gid, int wig, double v[5]) {
  group_sum<NW, 5>(S, gid, wig, v);
}

// Maximum of one value over the group, on every lane.
template <int NW, class Sm>
__device__ __forceinline__ double group_max(Sm& S, int gid, int wig, double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
  if (NW == 1) return v;
  if ((threadIdx.x & 31) == 0) S.red[wig][7] = v;
  gsync<NW>(gid);
  double m = S.red[0][7];
#pragma unroll
  for (int w = 1; w < NW; ++w) m = fmax(m, S.red[w][7]);
  gsync<NW>(gid);
  return m;
}

// Pivots k0 .. k1-1 of the FP64 right-looking LDL^T with the forward
// substitution of y fused in, the row kept shifted so that slot 0 holds the
// current pivot column: a step writes it to the group's line, then
// A[q] <- A[q+1] - f col[q] over the W slots that can still hold live
// columns. The loop body is the same for every k, so it is a runtime loop
// and A stays in registers. With kStoreL the multiplier L[row][k] goes to
// Lrow[k] (the row's packed strictly lower part) for later substitutions.
template <int NW, int W, bool kStoreL = false, class Sm>
__device__ __forceinline__ void eliminate_rows(double (&A)[32 * NW], int k0, int k1, int row, Sm& S,
                                               int gid, double& y0, double& y1, double& y2, double& dme, bool& sing,
                                               double thr, double* Lrow = nullptr) {
  constexpr int R = 32 * NW;
  for (int k = k0; k < k1; ++k) {
    const int b = k & 1;
    S.col[b][row > k ? row - k - 1 : (row == k ? R : R + 1)] = A[0];
    if (row == k) S.rhs[b][0] = y0, S.rhs[b][1] = y1, S.rhs[b][2] = y2;
    gsync<NW>(gid);
    const double d = S.col[b][R];
    if (!(d > thr)) {  // NaN or at most 1e-12 C0 (kernel.rs:61); uniform over the group
      sing = true;
      return;
    }
    if (row == k) dme = d;
    const double f = row > k ? A[0] * (1.0 / d) : 0.0;
    if (kStoreL && row > k) Lrow[k] = f;
#pragma unroll
    for (int q = 0; q < W; q += 2) {
      const double2 cv = *reinterpret_cast<const double2*>(&S.col[b][q]);
      A[q] = fma(-f, cv.x, A[q + 1]);
      A[q + 1] = q + 2 < R ? fma(-f, cv.y, A[q + 2]) : 0.0;
    }
    y0 = fma(-f, S.rhs[b][0], y0);
    y1 = fma(-f, S.rhs[b][1], y1);
    y2 = fma(-f, S.rhs[b][2], y2);
  }
}

// The pivots 0 .. nn-1 in four stages of R/4 with windows of R, 3R/4, R/2 and
// R/4 slots (the columns a step can still change in row R - 1). In a group of
// two warps, warp 0's rows (0 .. 31) hold at most 31 - k live slots at pivot
// k: it takes windows of 32 and 16 slots in the first two stages and none
// after (it still meets every barrier), so it skips the updates of columns its
// rows do not have. The live slots take the same operations either way.
template <int NW, bool kStoreL = false, class Sm>
__device__ __forceinline__ void eliminate_staged(double (&A)[32 * NW], int nn, int row, int wig, Sm& S, int gid,
                                                 double& y0, double& y1, double& y2, double& dme, bool& sing,
                                                 double thr, double* Lrow = nullptr) {
  constexpr int R = 32 * NW, Q = R / 4;
  const int n1 = min(nn, Q), n2 = min(nn, 2 * Q), n3 = min(nn, 3 * Q);
  if (NW == 2 && wig == 0) {
    eliminate_rows<NW, 32, kStoreL>(A, 0, n1, row, S, gid, y0, y1, y2, dme, sing, thr, Lrow);
    if (!sing) eliminate_rows<NW, 16, kStoreL>(A, n1, n2, row, S, gid, y0, y1, y2, dme, sing, thr, Lrow);
    if (!sing) eliminate_rows<NW, 0, kStoreL>(A, n2, n3, row, S, gid, y0, y1, y2, dme, sing, thr, Lrow);
    if (!sing) eliminate_rows<NW, 0, kStoreL>(A, n3, nn, row, S, gid, y0, y1, y2, dme, sing, thr, Lrow);
  } else {
    eliminate_rows<NW, R, kStoreL>(A, 0, n1, row, S, gid, y0, y1, y2, dme, sing, thr, Lrow);
    if (!sing) eliminate_rows<NW, 3 * Q, kStoreL>(A, n1, n2, row, S, gid, y0, y1, y2, dme, sing, thr, Lrow);
    if (!sing) eliminate_rows<NW, 2 * Q, kStoreL>(A, n2, n3, row, S, gid, y0, y1, y2, dme, sing, thr, Lrow);
    if (!sing) eliminate_rows<NW, Q, kStoreL>(A, n3, nn, row, S, gid, y0, y1, y2, dme, sing, thr, Lrow);
  }
}

// The FP32 form of eliminate_rows: the multiplier of row i at step k goes to
// L[i][k] for the substitutions, and a pivot at most thr or NaN leaves the
// system to the FP64 form.
template <int NW, int W, class Sm>
__device__ __forceinline__ void eliminate_rows_f32(float (&A)[32 * NW], int k0, int k1, int row, Sm& X,
                                                   int gid, float& y0, float& y1, float& y2, float& dme, bool& weak,
                                                   float thr) {
  constexpr int R = 32 * NW;
  for (int k = k0; k < k1; ++k) {
    const int b = k & 1;
    X.colf[b][row > k ? row - k - 1 : (row == k ? R : R + 1)] = A[0];
    if (row == k) X.rhsf[b][0] = y0, X.rhsf[b][1] = y1, X.rhsf[b][2] = y2;
    gsync<NW>(gid);
    const float d = X.colf[b][R];
    if (!(d > thr)) {  // uniform over the group
      weak = true;
      return;
    }
    if (row == k) dme = d;
    const float f = row > k ? A[0] * __frcp_rn(d) : 0.f;
    if (row > k) X.L[row][k] = f;
#pragma unroll
    for (int q = 0; q < W; q += 4) {
      const float4 cv = *reinterpret_cast<const float4*>(&X.colf[b][q]);
      A[q] = fmaf(-f, cv.x, A[q + 1]);
      A[q + 1] = fmaf(-f, cv.y, A[q + 2]);
      A[q + 2] = fmaf(-f, cv.z, A[q + 3]);
      A[q + 3] = q + 4 < R ? fmaf(-f, cv.w, A[q + 4]) : 0.f;
    }
    y0 = fmaf(-f, X.rhsf[b][0], y0);
    y1 = fmaf(-f, X.rhsf[b][1], y1);
    y2 = fmaf(-f, X.rhsf[b][2], y2);
  }
}

// x <- C~^-1 x for the FP32 factors C~ = L D L^T of eliminate_rows_f32 on
// three right-hand sides at once, one entry per row: the forward sweep with
// L (skipped when `forward` is false, for a y already forward-substituted
// during the elimination), the scale by 1 / D, and the backward sweep with
// L^T, column by column through the group's broadcast line.
template <int NW, class Sm>
__device__ __forceinline__ void sweep_f32(Sm& X, int gid, int row, int nn, float dme, bool forward,
                                          float& u0, float& u1, float& u2) {
  if (forward) {
    gsync<NW>(gid);
    for (int k = 0; k < nn; ++k) {
      const int b = k & 1;
      if (row == k) X.rhsf[b][0] = u0, X.rhsf[b][1] = u1, X.rhsf[b][2] = u2;
      gsync<NW>(gid);
      if (row > k) {
        const float l = X.L[row][k];
        u0 = fmaf(-l, X.rhsf[b][0], u0);
        u1 = fmaf(-l, X.rhsf[b][1], u1);
        u2 = fmaf(-l, X.rhsf[b][2], u2);
      }
    }
  }
  u0 /= dme, u1 /= dme, u2 /= dme;
  gsync<NW>(gid);
  for (int k = nn - 1; k >= 0; --k) {
    const int b = k & 1;
    if (row == k) X.rhsf[b][0] = u0, X.rhsf[b][1] = u1, X.rhsf[b][2] = u2;
    gsync<NW>(gid);
    if (row < k) {
      const float l = X.L[k][row];
      u0 = fmaf(-l, X.rhsf[b][0], u0);
      u1 = fmaf(-l, X.rhsf[b][1], u1);
      u2 = fmaf(-l, X.rhsf[b][2], u2);
    }
  }
}

}  // namespace btk
