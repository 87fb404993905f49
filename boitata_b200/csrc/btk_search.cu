// Neighbour search (K1): the samples a target is kriged from, identical,
// index for index and in order, to the reference's SearchTree for plain and
// octant (or quadrant) searches.
//
// What the reference computes (crates/estimation/src/search.rs:476-577,
// 951-1005 and search/grid.rs:209-255): the samples within `radius` of the
// target in the search frame, ranked by (squared distance bits, index), are
// offered in that order to a greedy selector that keeps at most `cap` per
// sector and stops at `max_samples`. Since a sector's acceptance depends only
// on earlier samples of the same sector, the selection equals: per sector,
// its `cap` smallest (d2, index) candidates; merged by (d2, index); the first
// `max_samples`. That is what this kernel keeps.
//
// B200 mapping: one warp serves a tile of 32 targets, one per lane (block-
// model tiles are 4 x 4 x 2 cells). The warp walks grid cells outward from
// the tile's bounding box shell by shell; each shell's candidate ranges are
// contiguous in the cell-sorted sample arrays, staged 32 at a time through
// shared memory (coalesced loads, broadcast reads), and every lane tests
// every candidate against its own target with exact-order FP64. Each lane
// keeps one max-heap per sector in shared memory ([slot][lane] layout, free
// of bank conflicts). A lane is done once the distance from its target to
// the unvisited cells exceeds its current threshold (radius^2, or the
// largest sector root once every sector is full); the tile ends when all
// lanes are done or the grid is exhausted.
#include <climits>

#include "btk_device.cuh"

namespace btk {
namespace {

constexpr unsigned kFull = 0xffffffffu;

template <int SLOTS, bool OCT>
struct WarpSmem {
  double hd[SLOTS][32];    // heap keys: squared distance
  uint32_t hi[SLOTS][32];  // heap keys: sample index
  int cnt[OCT ? 8 : 1][32];
  double cp[3][32];  // staged candidates, projected
  double cw[3][32];  // staged candidates, world (octant signs)
  uint32_t ci[32];
};

__device__ __forceinline__ bool key_less(double da, uint32_t ia, double db, uint32_t ib) {
  return da < db || (da == db && ia < ib);
}

// Squared lower bound on the distance from q to any point of the cells
// [x0..x1] x [y0..y1] x [z0..z1], less the grid's rounding slack.
__device__ __forceinline__ double box_lb2(const GridDev& g, const double q[3], int x0, int x1, int y0, int y1,
                                          int z0, int z1) {
  int a[3] = {x0, y0, z0}, b[3] = {x1, y1, z1};
  double s = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double lo = g.lo[d] + a[d] * g.h, hi = g.lo[d] + (b[d] + 1) * g.h;
    double gap = fmax(fmax(lo - q[d], q[d] - hi), 0.0);
    gap = fmax(gap - g.slack, 0.0);
    s += gap * gap;
  }
  return s * (1.0 - 1e-12);
}

// Squared lower bound on the distance from q to any cell outside the box
// [c0..c1] (clipped to the grid): the nearest face with cells beyond it.
__device__ __forceinline__ double outside_lb2(const GridDev& g, const double q[3], const int c0[3], const int c1[3]) {
  double lb = INFINITY;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (c0[d] > 0) lb = fmin(lb, fmax(q[d] - (g.lo[d] + c0[d] * g.h), 0.0));
    if (c1[d] < g.dims[d] - 1) lb = fmin(lb, fmax((g.lo[d] + (c1[d] + 1) * g.h) - q[d], 0.0));
  }
  if (lb == INFINITY) return INFINITY;
  lb = fmax(lb - g.slack, 0.0);
  return lb * lb * (1.0 - 1e-12);
}

template <int SLOTS, bool OCT>
__device__ __forceinline__ double max_root(const WarpSmem<SLOTS, OCT>& S, int lane, int nsec, int cap) {
  double m = S.hd[0][lane];
  for (int s = 1; s < nsec; ++s) m = fmax(m, S.hd[s * cap][lane]);
  return m;
}

// Offers candidate (d2, idx) of sector `sec` to this lane's lists.
template <int SLOTS, bool OCT>
__device__ __forceinline__ void consider(WarpSmem<SLOTS, OCT>& S, int lane, int nsec, int cap, int sec, double d2,
                                         uint32_t idx, double& thr, int& nfull) {
  const int base = sec * cap;
  int c = S.cnt[sec][lane];
  if (c < cap) {  // heap not full: sift up
    int pos = c;
    while (pos > 0) {
      int par = (pos - 1) >> 1;
      double pd = S.hd[base + par][lane];
      uint32_t pi = S.hi[base + par][lane];
      if (!key_less(pd, pi, d2, idx)) break;
      S.hd[base + pos][lane] = pd;
      S.hi[base + pos][lane] = pi;
      pos = par;
    }
    S.hd[base + pos][lane] = d2;
    S.hi[base + pos][lane] = idx;
    S.cnt[sec][lane] = c + 1;
    if (c + 1 == cap && ++nfull == nsec) thr = max_root(S, lane, nsec, cap);
    return;
  }
  if (!key_less(d2, idx, S.hd[base][lane], S.hi[base][lane])) return;
  int pos = 0;  // replace the root (the largest kept) and sift down
  while (true) {
    int ch = 2 * pos + 1;
    if (ch >= cap) break;
    double cd = S.hd[base + ch][lane];
    uint32_t cix = S.hi[base + ch][lane];
    if (ch + 1 < cap) {
      double rd = S.hd[base + ch + 1][lane];
      uint32_t ri = S.hi[base + ch + 1][lane];
      if (key_less(cd, cix, rd, ri)) ch = ch + 1, cd = rd, cix = ri;
    }
    if (!key_less(d2, idx, cd, cix)) break;
    S.hd[base + pos][lane] = cd;
    S.hi[base + pos][lane] = cix;
    pos = ch;
  }
  S.hd[base + pos][lane] = d2;
  S.hi[base + pos][lane] = idx;
  if (nfull == nsec) thr = max_root(S, lane, nsec, cap);
}

template <int SLOTS, bool OCT>
__device__ __forceinline__ void sift_down(WarpSmem<SLOTS, OCT>& S, int lane, int pos, int len) {
  double d = S.hd[pos][lane];
  uint32_t i = S.hi[pos][lane];
  while (true) {
    int ch = 2 * pos + 1;
    if (ch >= len) break;
    double cd = S.hd[ch][lane];
    uint32_t cix = S.hi[ch][lane];
    if (ch + 1 < len) {
      double rd = S.hd[ch + 1][lane];
      uint32_t ri = S.hi[ch + 1][lane];
      if (key_less(cd, cix, rd, ri)) ch = ch + 1, cd = rd, cix = ri;
    }
    if (!key_less(d, i, cd, cix)) break;
    S.hd[pos][lane] = cd;
    S.hi[pos][lane] = cix;
    pos = ch;
  }
  S.hd[pos][lane] = d;
  S.hi[pos][lane] = i;
}

template <int SLOTS, bool OCT>
__global__ void k_search(SearchDev sp, GridDev g, const double* __restrict__ tx, const double* __restrict__ ty,
                         const double* __restrict__ tz, const int64_t* __restrict__ perm, int64_t m, int loo,
                         uint32_t* __restrict__ nbr, int32_t* __restrict__ count, int8_t* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  WarpSmem<SLOTS, OCT>& S = reinterpret_cast<WarpSmem<SLOTS, OCT>*>(smem_raw)[wib];
  const int nsec = OCT ? sp.nsec : 1;
  const int cap = sp.cap;
  const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);

  for (int64_t tile = int64_t(blockIdx.x) * (blockDim.x >> 5) + wib; tile * 32 < m; tile += warps) {
    const int64_t k = tile * 32 + lane;
    int64_t ti = -1;
    if (k < m) ti = perm ? perm[k] : k;
    const bool active = ti >= 0;
    double t[3] = {0, 0, 0}, q[3] = {0, 0, 0};
    int cq[3] = {INT_MAX, INT_MAX, INT_MAX}, cqh[3] = {INT_MIN, INT_MIN, INT_MIN};
    if (active) {
      t[0] = tx[ti], t[1] = ty[ti], t[2] = tz[ti];
      double d[3] = {xsub(t[0], sp.origin[0]), xsub(t[1], sp.origin[1]), xsub(t[2], sp.origin[2])};
      mulv_exact(sp.frame, d, q);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        double u = fmin(fmax(floor((q[a] - g.lo[a]) / g.h), 0.0), double(g.dims[a] - 1));
        cq[a] = cqh[a] = int(u);
      }
    }
    int b0[3], b1[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      int lo = cq[a], hi = cqh[a];
      for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(kFull, lo, o));
        hi = max(hi, __shfl_xor_sync(kFull, hi, o));
      }
      b0[a] = lo, b1[a] = hi;
    }
    if (b0[0] == INT_MAX) continue;  // no target in this tile

    for (int s = 0; s < nsec; ++s) S.cnt[s][lane] = 0;
    double thr = active ? sp.radius2 : -1.0;
    int nfull = 0;
    bool done = !active;
    const uint32_t left = (loo && active) ? uint32_t(ti) : 0xffffffffu;

    for (int r = 0;; ++r) {
      int c0[3], c1[3], p0[3], p1[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        c0[a] = max(b0[a] - r, 0), c1[a] = min(b1[a] + r, g.dims[a] - 1);
        p0[a] = max(b0[a] - r + 1, 0), p1[a] = min(b1[a] + r - 1, g.dims[a] - 1);
      }
      if (r > 0 && c0[0] == p0[0] && c1[0] == p1[0] && c0[1] == p0[1] && c1[1] == p1[1] && c0[2] == p0[2] &&
          c1[2] == p1[2])
        break;  // the grid is exhausted
      const int ny = c1[1] - c0[1] + 1;
      const int64_t nrows = int64_t(ny) * (c1[2] - c0[2] + 1);
      for (int64_t rb = 0; rb < nrows; rb += 32) {
        const int64_t row = rb + lane;
        uint32_t a1 = 0, e1 = 0, a2 = 0, e2 = 0;
        int y = 0, z = 0, xa1 = 0, xb1 = -1, xa2 = 0, xb2 = -1;
        if (row < nrows) {
          y = c0[1] + int(row % ny), z = c0[2] + int(row / ny);
          const bool inner = r > 0 && y >= p0[1] && y <= p1[1] && z >= p0[2] && z <= p1[2];
          const int64_t base = int64_t(g.dims[0]) * (y + int64_t(g.dims[1]) * z);
          if (!inner) {
            xa1 = c0[0], xb1 = c1[0];
          } else {
            if (p0[0] > c0[0]) xa1 = c0[0], xb1 = p0[0] - 1;
            if (p1[0] < c1[0]) xa2 = p1[0] + 1, xb2 = c1[0];
          }
          if (xb1 >= xa1) a1 = g.start[base + xa1], e1 = g.start[base + xb1 + 1];
          if (xb2 >= xa2) a2 = g.start[base + xa2], e2 = g.start[base + xb2 + 1];
        }
        unsigned pending = __ballot_sync(kFull, e1 > a1 || e2 > a2);
        while (pending) {
          const int j = __ffs(pending) - 1;
          pending &= pending - 1;
          const int yj = __shfl_sync(kFull, y, j), zj = __shfl_sync(kFull, z, j);
#pragma unroll
          for (int seg = 0; seg < 2; ++seg) {
            const uint32_t a = __shfl_sync(kFull, seg ? a2 : a1, j), e = __shfl_sync(kFull, seg ? e2 : e1, j);
            if (a >= e) continue;
            const int xa = __shfl_sync(kFull, seg ? xa2 : xa1, j), xb = __shfl_sync(kFull, seg ? xb2 : xb1, j);
            const bool need = !done && box_lb2(g, q, xa, xb, yj, yj, zj, zj) <= thr;
            if (!__any_sync(kFull, need)) continue;
            for (uint32_t base = a; base < e; base += 32) {
              const int nc = int(min(32u, e - base));
              if (lane < nc) {
                const uint32_t src = base + lane;
                S.cp[0][lane] = g.px[src], S.cp[1][lane] = g.py[src], S.cp[2][lane] = g.pz[src];
                S.ci[lane] = g.idx[src];
                if (OCT) S.cw[0][lane] = g.wx[src], S.cw[1][lane] = g.wy[src], S.cw[2][lane] = g.wz[src];
              }
              __syncwarp();
              if (need) {
                for (int c = 0; c < nc; ++c) {
                  const double d2 = d2_exact(S.cp[0][c], S.cp[1][c], S.cp[2][c], q[0], q[1], q[2]);
                  if (d2 <= thr) {
                    const uint32_t idx = S.ci[c];
                    if (idx == left) continue;
                    int sec = 0;
                    if (OCT) {
                      const double w[3] = {S.cw[0][c], S.cw[1][c], S.cw[2][c]};
                      sec = sector_of(sp.axes, sp.planar, w, t);
                    }
                    consider(S, lane, nsec, cap, sec, d2, idx, thr, nfull);
                  }
                }
              }
              __syncwarp();
            }
          }
        }
      }
      done = done || outside_lb2(g, q, c0, c1) > thr;
      if (__all_sync(kFull, done)) break;
    }

    // Gather every kept entry, sort by (d2, index), keep max_samples.
    int total = 0;
    for (int s = 0; s < nsec; ++s) {
      const int cs = S.cnt[s][lane];
      for (int e = 0; e < cs; ++e) {
        S.hd[total + e][lane] = S.hd[s * cap + e][lane];
        S.hi[total + e][lane] = S.hi[s * cap + e][lane];
      }
      total += cs;
    }
    for (int pos = total / 2 - 1; pos >= 0; --pos) sift_down(S, lane, pos, total);
    for (int end = total - 1; end > 0; --end) {
      double d = S.hd[0][lane];
      uint32_t i = S.hi[0][lane];
      S.hd[0][lane] = S.hd[end][lane], S.hi[0][lane] = S.hi[end][lane];
      S.hd[end][lane] = d, S.hi[end][lane] = i;
      sift_down(S, lane, 0, end);
    }
    const int nout = min(total, sp.max_samples);
    if (active) {
      const bool ok = nout >= sp.min_samples && !(loo && nout == 0);
      count[ti] = nout;
      status[ti] = ok ? BTK_ST_OK : BTK_ST_SEARCH_FAILED;
    }
    __syncwarp();
    // Rows of the neighbour table, one target at a time (coalesced).
    for (int l = 0; l < 32; ++l) {
      const int64_t tl = __shfl_sync(kFull, ti, l);
      const int nl = __shfl_sync(kFull, nout, l);
      if (tl < 0) continue;
      for (int j = lane; j < sp.max_samples; j += 32)
        nbr[tl * sp.max_samples + j] = j < nl ? S.hi[j][l] : 0xffffffffu;
    }
    __syncwarp();
  }
}

template <int SLOTS, bool OCT>
cudaError_t run(const Launch& L, const SearchDev& sp, const GridDev& g, const double* tx, const double* ty,
                const double* tz, const int64_t* perm, int64_t m, int loo, uint32_t* nbr, int32_t* count,
                int8_t* status) {
  constexpr int kWarps = SLOTS > 32 ? 2 : 4;
  const size_t smem = sizeof(WarpSmem<SLOTS, OCT>) * kWarps;
  auto kern = k_search<SLOTS, OCT>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kWarps * 32, smem);
  if (e != cudaSuccess) return e;
  const int64_t tiles = (m + 31) / 32;
  int64_t blocks = int64_t(L.sm_count) * (per_sm > 0 ? per_sm : 1);
  const int64_t need = (tiles + kWarps - 1) / kWarps;
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
  kern<<<int(blocks), kWarps * 32, smem, L.stream>>>(sp, g, tx, ty, tz, perm, m, loo, nbr, count, status);
  ++*L.counter;
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_search(const Launch& L, const SearchDev& sp, const GridDev& g, const double* tx,
                          const double* ty, const double* tz, const int64_t* perm, int64_t m, int loo,
                          uint32_t* nbr, int32_t* count, int8_t* status) {
  const int slots = sp.nsec * sp.cap;
  const bool oct = sp.nsec > 1;
  if (slots > kMaxSlots) return cudaErrorInvalidValue;
  if (slots <= 32)
    return oct ? run<32, true>(L, sp, g, tx, ty, tz, perm, m, loo, nbr, count, status)
               : run<32, false>(L, sp, g, tx, ty, tz, perm, m, loo, nbr, count, status);
  return oct ? run<64, true>(L, sp, g, tx, ty, tz, perm, m, loo, nbr, count, status)
             : run<64, false>(L, sp, g, tx, ty, tz, perm, m, loo, nbr, count, status);
}

}  // namespace btk
