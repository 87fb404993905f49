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
// model tiles are 4 x 4 x 2 cells). The warp grows a box of grid cells from
// the tile's own cells; each new slab of the box is a set of cell rows, each
// row a contiguous range of the cell-sorted sample arrays, staged 32 samples
// at a time through shared memory (coalesced loads, broadcast reads). Every
// lane tests every staged candidate against its own target with exact-order
// FP64 and keeps one max-heap per sector in shared memory ([slot][lane]
// layout, free of bank conflicts).
//
// Sectors are orthants of the grid axes in the search frame (SearchDev
// bit_axis / bit_sign), so a row is scanned only if, for some lane, it can
// hold a sample of a sector that is still open (fewer than `cap` kept) within
// the radius, or of a full sector closer than that sector's largest kept
// distance. The box grows only across faces beyond which some lane still
// needs cells by the same test, and the tile ends when no face is needed.
// A target whose empty octant points out of the data therefore stops as soon
// as the cells in that orthant run out, not at the search radius.
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

// Squared lower bound on the distance from q to the box [lo, hi], less the
// grid's rounding slack.
__device__ __forceinline__ double lb2(const GridDev& g, const double q[3], const double lo[3], const double hi[3]) {
  double s = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double gap = fmax(fmax(lo[d] - q[d], q[d] - hi[d]), 0.0);
    gap = fmax(gap - g.slack, 0.0);
    s += gap * gap;
  }
  return s * (1.0 - 1e-12);
}

// Sectors a sample in the box [lo, hi] may fall in, seen from q.
__device__ __forceinline__ unsigned box_sectors(const SearchDev& sp, const GridDev& g, const double q[3],
                                                const double lo[3], const double hi[3], unsigned all) {
  unsigned mask = all;
  const double d0l = lo[0] - q[0], d1l = lo[1] - q[1], d2l = lo[2] - q[2];
  const double d0h = hi[0] - q[0], d1h = hi[1] - q[1], d2h = hi[2] - q[2];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (k >= sp.nbits) break;
    const int a = sp.bit_axis[k];  // selected, not indexed: keeps lo/hi in registers
    const double dlo = a == 0 ? d0l : (a == 1 ? d1l : d2l), dhi = a == 0 ? d0h : (a == 1 ? d1h : d2h);
    const bool up = sp.bit_sign[k] > 0 ? dhi >= -g.slack : dlo <= g.slack;  // bit 1 possible
    const bool dn = sp.bit_sign[k] > 0 ? dlo <= g.slack : dhi >= -g.slack;  // bit 0 possible
    mask &= (up ? sp.bit_mask[k] : 0u) | (dn ? ~sp.bit_mask[k] : 0u);
  }
  return mask & all;
}

__device__ __forceinline__ void cell_box(const GridDev& g, int x0, int x1, int y0, int y1, int z0, int z1,
                                         double lo[3], double hi[3]) {
  lo[0] = g.lo[0] + x0 * g.h, hi[0] = g.lo[0] + (x1 + 1) * g.h;
  lo[1] = g.lo[1] + y0 * g.h, hi[1] = g.lo[1] + (y1 + 1) * g.h;
  lo[2] = g.lo[2] + z0 * g.h, hi[2] = g.lo[2] + (z1 + 1) * g.h;
}

// Per-lane state of the sector lists used to decide what is still needed.
struct Need {
  double radius2;
  unsigned open;   // sectors with fewer than `cap` kept
  double root[8];  // largest kept (d2) of each full sector
  __device__ __forceinline__ bool wants(unsigned mask, double l2) const {
    if (mask & open) return l2 <= radius2;
    double m = -1.0;
#pragma unroll
    for (int s = 0; s < 8; ++s)
      if ((mask >> s) & 1u) m = fmax(m, root[s]);
    return l2 <= m;
  }
};

template <int SLOTS, bool OCT>
__device__ __forceinline__ double max_root(const WarpSmem<SLOTS, OCT>& S, int lane, int nsec, int cap) {
  double m = S.hd[0][lane];
  for (int s = 1; s < nsec; ++s) m = fmax(m, S.hd[s * cap][lane]);
  return m;
}

__device__ __forceinline__ void set_root(Need& nd, int sec, double v) {
#pragma unroll
  for (int s = 0; s < 8; ++s)
    if (s == sec) nd.root[s] = v;
}

// Inserts (d2, idx) into sector list `base` holding c entries (a max-heap
// on (d2, index) in this lane's column): sift up while the list is filling,
// else replace the root and sift down. Returns the new root's d2. Kept out
// of line: it runs for a small share of the candidates, and the candidate
// loop around it runs faster when its code stays small.
template <int SLOTS, bool OCT>
__device__ __noinline__ double heap_insert(WarpSmem<SLOTS, OCT>& S, int lane, int base, int cap, int c, double d2,
                                           uint32_t idx) {
  if (c < cap) {
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
    return S.hd[base][lane];
  }
  int pos = 0;
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
  return S.hd[base][lane];
}

// Offers candidate (d2, idx) of sector `sec` to this lane's lists.
template <int SLOTS, bool OCT>
__device__ __forceinline__ void consider(WarpSmem<SLOTS, OCT>& S, int lane, int nsec, int cap, int sec, double d2,
                                         uint32_t idx, double& thr, Need& nd) {
  const int base = sec * cap;
  const int c = S.cnt[sec][lane];
  if (c >= cap && !key_less(d2, idx, S.hd[base][lane], S.hi[base][lane])) return;
  const double root = heap_insert(S, lane, base, cap, c, d2, idx);
  if (c < cap) S.cnt[sec][lane] = c + 1;
  if (c + 1 >= cap) {  // full (now or before): the root bounds what the sector still takes
    nd.open &= ~(1u << sec);
    set_root(nd, sec, root);
    if (nd.open == 0) thr = max_root(S, lane, nsec, cap);
  }
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
  const unsigned all = (1u << nsec) - 1u;
  const int cap = sp.cap;
  const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
  const double glo[3] = {g.lo[0], g.lo[1], g.lo[2]};
  const double ghi[3] = {g.lo[0] + g.dims[0] * g.h, g.lo[1] + g.dims[1] * g.h, g.lo[2] + g.dims[2] * g.h};

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
    int b0[3], b1[3];  // current box of cells (inclusive)
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
    Need nd;
    nd.radius2 = active ? sp.radius2 : -1.0;
    nd.open = active ? all : 0u;
#pragma unroll
    for (int s = 0; s < 8; ++s) nd.root[s] = -1.0;
    const uint32_t left = (loo && active) ? uint32_t(ti) : 0xffffffffu;
    int p0[3] = {1, 1, 1}, p1[3] = {0, 0, 0};  // previous box: empty at first

    while (true) {
      // Rows of the new slab: (y, z) over the box; x segments outside the previous box.
      const int ny = b1[1] - b0[1] + 1;
      const int64_t nrows = int64_t(ny) * (b1[2] - b0[2] + 1);
      for (int64_t rb = 0; rb < nrows; rb += 32) {
        const int64_t row = rb + lane;
        uint32_t a1 = 0, e1 = 0, a2 = 0, e2 = 0;
        int y = 0, z = 0, xa1 = 0, xb1 = -1, xa2 = 0, xb2 = -1;
        if (row < nrows) {
          y = b0[1] + int(row % ny), z = b0[2] + int(row / ny);
          const bool inner = y >= p0[1] && y <= p1[1] && z >= p0[2] && z <= p1[2];
          const int64_t base = int64_t(g.dims[0]) * (y + int64_t(g.dims[1]) * z);
          if (!inner) {
            xa1 = b0[0], xb1 = b1[0];
          } else {
            if (p0[0] > b0[0]) xa1 = b0[0], xb1 = p0[0] - 1;
            if (p1[0] < b1[0]) xa2 = p1[0] + 1, xb2 = b1[0];
          }
          if (xb1 >= xa1) a1 = g.start[base + xa1], e1 = g.start[base + xb1 + 1];
          if (xb2 >= xa2) a2 = g.start[base + xa2], e2 = g.start[base + xb2 + 1];
        }
        unsigned pending = __ballot_sync(kFull, e1 > a1 || e2 > a2);
        while (pending) {
          const int j = __ffs(pending) - 1;
          pending &= pending - 1;
          const int yj = __shfl_sync(kFull, y, j), zj = __shfl_sync(kFull, z, j);
#pragma unroll 1  // one copy of the candidate loop: the kernel is instruction-fetch bound
          for (int seg = 0; seg < 2; ++seg) {
            const uint32_t a = __shfl_sync(kFull, seg ? a2 : a1, j), e = __shfl_sync(kFull, seg ? e2 : e1, j);
            if (a >= e) continue;
            const int xa = __shfl_sync(kFull, seg ? xa2 : xa1, j), xb = __shfl_sync(kFull, seg ? xb2 : xb1, j);
            double lo[3], hi[3];
            cell_box(g, xa, xb, yj, yj, zj, zj, lo, hi);
            const bool need = active && nd.wants(box_sectors(sp, g, q, lo, hi, all), lb2(g, q, lo, hi));
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
#pragma unroll 1
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
                    consider(S, lane, nsec, cap, sec, d2, idx, thr, nd);
                  }
                }
              }
              __syncwarp();
            }
          }
        }
      }
      // Grow the box across each face some lane still needs cells beyond.
#pragma unroll
      for (int a = 0; a < 3; ++a) p0[a] = b0[a], p1[a] = b1[a];
      bool grew = false;
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        const int a = f >> 1;
        const bool high = f & 1;
        if (high ? b1[a] >= g.dims[a] - 1 : b0[a] <= 0) continue;
        double lo[3] = {glo[0], glo[1], glo[2]}, hi[3] = {ghi[0], ghi[1], ghi[2]};
        if (high)
          lo[a] = g.lo[a] + (b1[a] + 1) * g.h;
        else
          hi[a] = g.lo[a] + b0[a] * g.h;
        const bool need = active && nd.wants(box_sectors(sp, g, q, lo, hi, all), lb2(g, q, lo, hi));
        if (__any_sync(kFull, need)) {
          if (high)
            b1[a] += 1;
          else
            b0[a] -= 1;
          grew = true;
        }
      }
      if (!grew) break;
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
  const int kWarps = L.tuning.search_warps > 0 ? L.tuning.search_warps : (SLOTS > 32 ? 2 : 4);
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
