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
  uint8_t cnt[OCT ? 8 : 1][32];  // at most 64 kept per sector
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

__device__ __forceinline__ void set_root(Need& nd, int sec, double v) {
#pragma unroll
  for (int s = 0; s < 8; ++s)
    if (s == sec) nd.root[s] = v;
}

// Inserts (d2, idx) into sector list `base` holding c entries (a max-heap
// on (d2, index) in this lane's column): sift up while the list is filling,
// else replace the root and sift down. Returns the new root's d2.
template <int SLOTS, bool OCT>
__device__ __forceinline__ double heap_insert(WarpSmem<SLOTS, OCT>& S, int lane, int base, int cap, int c,
                                              double d2, uint32_t idx) {
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

// The same, out of line. The 64-slot search (at most 8 warps an SM, bound by
// shared memory) runs faster with the call: its candidate loop stays small.
// The 32-slot search (16 warps, 128 registers) runs faster with it inline:
// 11.4 against 11.0 ms at 3.2M blocks.
template <int SLOTS, bool OCT>
__device__ __noinline__ double heap_insert_call(WarpSmem<SLOTS, OCT>& S, int lane, int base, int cap, int c,
                                                double d2, uint32_t idx) {
  return heap_insert(S, lane, base, cap, c, d2, idx);
}

// Offers candidate (d2, idx) of sector `sec` to this lane's lists.
template <int SLOTS, bool OCT>
__device__ __forceinline__ void consider(WarpSmem<SLOTS, OCT>& S, int lane, int nsec, int cap, int sec, double d2,
                                         uint32_t idx, double& thr, Need& nd) {
  const int base = sec * cap;
  const int c = S.cnt[sec][lane];
  if (c >= cap && !key_less(d2, idx, S.hd[base][lane], S.hi[base][lane])) return;
  double root;
  if constexpr (SLOTS <= 32)
    root = heap_insert(S, lane, base, cap, c, d2, idx);
  else
    root = heap_insert_call(S, lane, base, cap, c, d2, idx);
  if (c < cap) S.cnt[sec][lane] = c + 1;
  if (c + 1 >= cap) {  // full (now or before): the root bounds what the sector still takes
    nd.open &= ~(1u << sec);
    set_root(nd, sec, root);
    if (nd.open == 0) {  // every sector full: the largest root, from the register copies
      double m = nd.root[0];
#pragma unroll
      for (int s = 1; s < 8; ++s) m = fmax(m, nd.root[s]);
      thr = m;
    }
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

// At most 32 slots, the kernel is held to 128 registers a thread (no spills),
// and a 4-warp CTA's 56.8 KB of shared memory fits four times in the SM:
// 16 warps resident instead of 12 (150 registers), and the c2 search went
// from 13.3 to 11.8 ms at 3.2M blocks. A 64-slot warp needs 26.6 KB, so
// shared memory bounds those CTAs first and their registers stay free.
template <int SLOTS, bool OCT>
__global__ void __launch_bounds__(256, SLOTS > 32 ? 1 : 2) k_search(SearchDev sp, GridDev g, const double* __restrict__ tx, const double* __restrict__ ty,
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
                // The next candidate's coordinates and index load while this
                // one is offered (the heaps' stores never touch the staged
                // arrays).
                double nx = S.cp[0][0], ny = S.cp[1][0], nz = S.cp[2][0];
                uint32_t ni = S.ci[0];
#pragma unroll 1
                for (int c = 0; c < nc; ++c) {
                  const double cx = nx, cy = ny, cz = nz;
                  const uint32_t idx = ni;
                  if (c + 1 < nc) nx = S.cp[0][c + 1], ny = S.cp[1][c + 1], nz = S.cp[2][c + 1], ni = S.ci[c + 1];
                  const double d2 = d2_exact(cx, cy, cz, q[0], q[1], q[2]);
                  if (d2 <= thr) {
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

// ---- searches with hole and sector rules ----------------------------------
// search.rs:476-577: per-hole caps, plane sectors, min_sectors,
// max_empty_sectors and min_holes make a sample's acceptance depend on
// earlier samples of other sectors, so the per-sector lists above no longer
// give the selection. Here one warp serves one target: it grows a box of
// cells from the target's cell, keeps every candidate within the threshold
// (the radius, then the K-th nearest once more than 2K - 32 were seen: a
// bitonic sort keeps the K nearest), sorts them by (d2, index), computes
// their sectors in parallel, and lane 0 runs the reference's greedy selector
// (Selector::offer / finish) over them. When the selection is not full and
// candidates within the radius were cut, further rounds rescan for the
// candidates beyond the last one offered that could still be accepted (open
// sectors, holes below their cap; cells pruned by octant), until the
// selection is full, no sector is open or the radius is exhausted: the
// result is the reference's for any number of candidates.
constexpr int kRulesK = BTK_RULES_CANDIDATES;
// A simulation's plain or octant search of at most 64 samples keeps fewer
// candidates per round: its candidate set grows with every simulated node,
// and the K-nearest cut, not the selection, dominates the search.
constexpr int kSgsK = 128, kSgsK32 = 64;  // at most 64 / at most 32 samples
// Slots of the accepted-hole table: at least the most samples a list holds
// (each accepted sample adds at most one hole), so a lookup always ends.
constexpr int kHoleHash = 128;        // lists of at most 128 samples
constexpr int kHoleHashBig = 2048;    // up to kMaxLUGlobal samples
constexpr uint32_t kNoHole = 0xffffffffu;

template <int K, int HH = kHoleHash>
struct RulesSmem {
  static constexpr int kHash = HH;
  double cd[2 * K];
  uint32_t ci[2 * K];
  uint16_t sec[2 * K];
  uint32_t hkey[HH];
  int hcnt[HH];
  int per_sector[360];
};

// Ascending bitonic sort of (d2, index) keys 0 .. n-1 by one warp, padded to a
// power of two with +inf keys.
__device__ void warp_sort(double* d, uint32_t* ix, int n, int lane) {
  int n2 = 1;
  while (n2 < n) n2 <<= 1;
  for (int j = n + lane; j < n2; j += 32) d[j] = INFINITY, ix[j] = 0xffffffffu;
  __syncwarp();
  for (int size = 2; size <= n2; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = lane; t < n2 / 2; t += 32) {
        const int lo = 2 * t - (t & (stride - 1)), hi = lo + stride;
        const bool up = (lo & size) == 0;
        const bool sw = up ? key_less(d[hi], ix[hi], d[lo], ix[lo]) : key_less(d[lo], ix[lo], d[hi], ix[hi]);
        if (sw) {
          const double td = d[lo];
          const uint32_t ti = ix[lo];
          d[lo] = d[hi], ix[lo] = ix[hi];
          d[hi] = td, ix[hi] = ti;
        }
      }
      __syncwarp();
    }
}

// Sectors::of (search.rs:427-441): plane sectors by angle in the major /
// semi-major plane, else octants / quadrants.

// Sectors::longest_empty (search.rs:445-467).
__device__ int longest_empty(const SearchDev& sp, const int* counts) {
  auto ring_run = [&](const int* ring, int len) {
    bool all = true;
    for (int i = 0; i < len; ++i) all = all && counts[ring[i]] == 0;
    if (all) return len;
    int run = 0, longest = 0;
    for (int i = 0; i < 2 * len; ++i) {
      run = counts[ring[i % len]] == 0 ? run + 1 : 0;
      longest = max(longest, run);
    }
    return longest;
  };
  if (sp.plane) {
    bool all = true;
    for (int i = 0; i < sp.plane; ++i) all = all && counts[i] == 0;
    if (all) return sp.plane;
    int run = 0, longest = 0;
    for (int i = 0; i < 2 * sp.plane; ++i) {
      run = counts[i % sp.plane] == 0 ? run + 1 : 0;
      longest = max(longest, run);
    }
    return longest;
  }
  if (sp.planar) {
    const int ring[4] = {3, 1, 0, 2};
    return ring_run(ring, 4);
  }
  const int up[4] = {7, 3, 1, 5}, down[4] = {6, 2, 0, 4};
  return max(ring_run(up, 4), ring_run(down, 4));
}

// Hole slot of h in the warp's table of accepted holes (the free slot where
// it would go when absent).
template <class Sm>
__device__ __forceinline__ int hole_slot(const Sm& S, uint32_t h) {
  constexpr int HH = Sm::kHash;
  int k = int((h * 2654435761u) >> (HH == kHoleHash ? 25 : 21)) & (HH - 1);  // 7 or 11 bits
  for (int probe = 0; probe < HH; ++probe) {
    if (S.hkey[k] == h || S.hkey[k] == kNoHole) break;
    k = (k + 1) & (HH - 1);
  }
  return k;
}

// One pass over the cells around target q: every candidate with key above
// (after_d, after_i), d2 within the threshold, and, once `filter` is set, in
// an open sector (per_sector below the cap) from a hole below its cap, goes
// into the warp's buffer; above 2K - 32 candidates the buffer keeps its K
// nearest. Returns the count; *dropped tells whether candidates were cut.
template <int K, int HH>
__device__ int rules_scan(const SearchDev& sp, const GridDev& g, RulesSmem<K, HH>& S, const double q[3], const double t[3],
                          uint32_t left, double after_d, uint32_t after_i, bool filter, unsigned openmask,
                          bool& dropped, int lane, uint32_t my, double& d2u, int32_t dom) {
  const double glo[3] = {g.lo[0], g.lo[1], g.lo[2]};
  const double ghi[3] = {g.lo[0] + g.dims[0] * g.h, g.lo[1] + g.dims[1] * g.h, g.lo[2] + g.dims[2] * g.h};
  const unsigned all = sp.nsec > 1 ? (1u << sp.nsec) - 1u : 1u;
  const bool prune = filter && sp.balances && !sp.plane;  // orthant pruning of rows and faces
  int b0[3], b1[3], p0[3] = {1, 1, 1}, p1[3] = {0, 0, 0};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double u = fmin(fmax(floor((q[a] - g.lo[a]) / g.h), 0.0), double(g.dims[a] - 1));
    b0[a] = b1[a] = int(u);
  }
  int n = 0;
  double thr = sp.radius2;
  dropped = false;
  while (true) {
    const int ny = b1[1] - b0[1] + 1;
    const int64_t nrows = int64_t(ny) * (b1[2] - b0[2] + 1);
    for (int64_t rb = 0; rb < nrows; rb += 32) {
      const int64_t row = rb + lane;
      uint32_t a1 = 0, e1 = 0, a2 = 0, e2 = 0;
      if (row < nrows) {
        const int y = b0[1] + int(row % ny), z = b0[2] + int(row / ny);
        const bool inner = y >= p0[1] && y <= p1[1] && z >= p0[2] && z <= p1[2];
        const int64_t base = int64_t(g.dims[0]) * (y + int64_t(g.dims[1]) * z);
        int xa1 = 0, xb1 = -1, xa2 = 0, xb2 = -1;
        if (!inner) {
          xa1 = b0[0], xb1 = b1[0];
        } else {
          if (p0[0] > b0[0]) xa1 = b0[0], xb1 = p0[0] - 1;
          if (p1[0] < b1[0]) xa2 = p1[0] + 1, xb2 = b1[0];
        }
        double lo[3], hi[3];
        if (xb1 >= xa1) {
          cell_box(g, xa1, xb1, y, y, z, z, lo, hi);
          if (lb2(g, q, lo, hi) <= thr && (!prune || (box_sectors(sp, g, q, lo, hi, all) & openmask)))
            a1 = g.start[base + xa1], e1 = g.start[base + xb1 + 1];
        }
        if (xb2 >= xa2) {
          cell_box(g, xa2, xb2, y, y, z, z, lo, hi);
          if (lb2(g, q, lo, hi) <= thr && (!prune || (box_sectors(sp, g, q, lo, hi, all) & openmask)))
            a2 = g.start[base + xa2], e2 = g.start[base + xb2 + 1];
        }
      }
      unsigned pending = __ballot_sync(kFull, e1 > a1 || e2 > a2);
      while (pending) {
        const int j = __ffs(pending) - 1;
        pending &= pending - 1;
#pragma unroll 1
        for (int seg = 0; seg < 2; ++seg) {
          const uint32_t a = __shfl_sync(kFull, seg ? a2 : a1, j), e = __shfl_sync(kFull, seg ? e2 : e1, j);
          for (uint32_t base = a; base < e; base += 32) {
            const uint32_t c = base + lane;
            bool keep = false;
            double d2 = 0.0;
            uint32_t idx = 0;
            if (c < e) {
              d2 = d2_exact(g.px[c], g.py[c], g.pz[c], q[0], q[1], q[2]);
              idx = g.idx[c];
              keep = d2 <= thr && idx != left && key_less(after_d, after_i, d2, idx);
              if (sp.sdom) keep = keep && sp.sdom[idx] == dom;  // samples of the target's domain only
              if (sp.sgs && d2 <= thr && idx >= sp.sgs_node0) {  // a grid node of a simulation
                if (idx < my && !sp.sgs_done[idx]) d2u = fmin(d2u, d2);
                keep = keep && idx < my && sp.sgs_done[idx];
              }
              if (keep && filter) {
                if (sp.balances) {
                  const double wv[3] = {sp.sx[idx], sp.sy[idx], sp.sz[idx]};
                  keep = S.per_sector[search_sector(sp, wv, t)] < sp.rcap;
                }
                if (keep && sp.max_per_hole >= 0 && sp.hole) {
                  const uint32_t h = sp.hole[idx];
                  const int k = hole_slot(S, h);
                  keep = !(S.hkey[k] == h && S.hcnt[k] >= sp.max_per_hole);
                }
              }
            }
            const unsigned bal = __ballot_sync(kFull, keep);
            if (keep) {
              const int pos = n + __popc(bal & ((1u << lane) - 1u));
              S.cd[pos] = d2, S.ci[pos] = idx;
            }
            n += __popc(bal);
            if (n > 2 * K - 32) {  // keep the K nearest
              __syncwarp();
              warp_sort(S.cd, S.ci, n, lane);
              n = K;
              thr = S.cd[K - 1];
              dropped = true;
            }
            __syncwarp();
          }
        }
      }
    }
    // Grow the box across each face beyond which cells may hold a candidate.
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
      if (lb2(g, q, lo, hi) <= thr && (!prune || (box_sectors(sp, g, q, lo, hi, all) & openmask))) {
        if (high)
          b1[a] += 1;
        else
          b0[a] -= 1;
        grew = true;
      }
    }
    if (!grew) break;
  }
  __syncwarp();
  if (n > 0) warp_sort(S.cd, S.ci, n, lane);
  return n;
}

// With the 512-candidate buffers (16.5 KB a warp) shared memory holds an SM to
// three CTAs, so up to 170 registers cost no occupancy; given only the block
// size the compiler kept 128 and spilled about 210 bytes a thread. The SGS
// forms (small buffers, four CTAs by registers) keep 128.
template <int K, int HH = kHoleHash>
__global__ void __launch_bounds__(128, K >= 512 ? 3 : 4) k_search_rules(SearchDev sp, GridDev g, const double* __restrict__ tx,
                                                      const double* __restrict__ ty, const double* __restrict__ tz,
                                                      const int64_t* __restrict__ perm, int64_t m, int loo,
                                                      uint32_t* __restrict__ nbr, int32_t* __restrict__ count,
                                                      int8_t* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  RulesSmem<K, HH>& S = reinterpret_cast<RulesSmem<K, HH>*>(smem_raw)[threadIdx.x >> 5];
  const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
  for (int64_t w = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); w < m; w += warps) {
    const int64_t ti = perm ? perm[w] : w;
    if (ti < 0) continue;
    const double t[3] = {tx[ti], ty[ti], tz[ti]};
    double q[3];
    {
      const double d[3] = {xsub(t[0], sp.origin[0]), xsub(t[1], sp.origin[1]), xsub(t[2], sp.origin[2])};
      mulv_exact(sp.frame, d, q);
    }
    const uint32_t left = loo ? uint32_t(ti) : 0xffffffffu;
    const uint32_t my = sp.sgs ? sp.sgs_node0 + uint32_t(ti) : 0xffffffffu;
    const int32_t dom = sp.sdom ? sp.tdom[ti] : 0;  // the target's domain (hard boundaries)
    double d2u = INFINITY, far = 0.0;  // nearest unsimulated earlier node; farthest accepted
    for (int i = lane; i < HH; i += 32) S.hkey[i] = kNoHole, S.hcnt[i] = 0;
    for (int i = lane; i < 360; i += 32) S.per_sector[i] = 0;
    __syncwarp();
    // Selector state (lane 0's copy is the one that counts)
    int nchosen = 0, untagged = 0, nholes = 0;
    double after_d = -1.0;
    uint32_t after_i = 0u;
    bool filter = false;
    unsigned openmask = 0xffffffffu;
    bool dropped = false;
    // Each round offers the next candidates in (d2, index) order; a round
    // after the first takes only candidates that could still be accepted.
    for (int round = 0; round < 1 << 20; ++round) {
      // After a cut, only the K nearest are an exact prefix of the (d2, index)
      // order: entries kept since then can skip cut ones of equal d2.
      const int nscan =
          rules_scan(sp, g, S, q, t, left, after_d, after_i, filter, openmask, dropped, lane, my, d2u, dom);
      const int n = dropped ? K : nscan;
      if (sp.balances)
        for (int i = lane; i < n; i += 32) {
          const uint32_t idx = S.ci[i];
          const double wv[3] = {sp.sx[idx], sp.sy[idx], sp.sz[idx]};
          S.sec[i] = uint16_t(search_sector(sp, wv, t));
        }
      __syncwarp();
      if (lane == 0)  // Selector::offer (search.rs:535-559)
        for (int i = 0; i < n && nchosen < sp.max_samples; ++i) {
          const uint32_t idx = S.ci[i];
          const uint32_t h = sp.hole ? sp.hole[idx] : kNoHole;
          int slot = -1;
          if (h != kNoHole) {
            slot = hole_slot(S, h);
            if (sp.max_per_hole >= 0 && S.hkey[slot] == h && S.hcnt[slot] >= sp.max_per_hole) continue;
          }
          if (sp.balances) {
            const int o = S.sec[i];
            if (S.per_sector[o] >= sp.rcap) continue;
            S.per_sector[o] += 1;
          }
          if (h != kNoHole) {
            if (S.hkey[slot] != h) S.hkey[slot] = h, ++nholes;
            S.hcnt[slot] += 1;
          } else {
            ++untagged;
          }
          far = S.cd[i];
          nbr[ti * sp.max_samples + nchosen++] = idx;  // the list goes straight to its row
        }
      nchosen = __shfl_sync(kFull, nchosen, 0);
      __syncwarp();
      if (nchosen >= sp.max_samples || !dropped || n == 0) break;
      // Candidates beyond the last one offered may still be taken: those in
      // sectors below their cap, from holes below theirs.
      after_d = S.cd[n - 1], after_i = S.ci[n - 1];
      filter = true;
      openmask = 0u;
      if (sp.balances) {
        bool any_open = false;
        for (int o = 0; o < sp.rsec; ++o) {
          const bool open = S.per_sector[o] < sp.rcap;
          any_open = any_open || open;
          if (open && o < 32) openmask |= 1u << o;
        }
        if (!any_open) break;
        if (sp.plane) openmask = 0xffffffffu;
      } else {
        openmask = 0xffffffffu;
      }
      __syncwarp();
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d2u = fmin(d2u, __shfl_xor_sync(kFull, d2u, o));
    if (lane == 0) {  // Selector::finish (search.rs:561-590)
      int8_t st = BTK_ST_OK;
      if (nchosen < sp.min_samples || (loo && nchosen == 0)) {
        st = BTK_ST_SEARCH_FAILED;
      } else if (sp.min_sectors >= 0) {
        int held = 0;
        for (int o = 0; o < sp.rsec; ++o) held += S.per_sector[o] > 0;
        if (held < sp.min_sectors) st = BTK_ST_SEARCH_FAILED;
      }
      if (st == BTK_ST_OK && sp.max_empty_sectors >= 0 && longest_empty(sp, S.per_sector) > sp.max_empty_sectors)
        st = BTK_ST_SEARCH_FAILED;
      if (st == BTK_ST_OK && sp.min_holes >= 0 && nholes + untagged < sp.min_holes) st = BTK_ST_SEARCH_FAILED;
      if (sp.sgs) {  // crates/simulation/src/sgs.rs:600-625: reach of the search, with a margin
        const double reach2 = (st == BTK_ST_OK && nchosen >= sp.max_samples) ? far : sp.radius2;
        if (d2u < INFINITY && d2u <= reach2 * (1.0 + 1e-8)) st = kStStale;  // an unsimulated node was seen
      }
      count[ti] = nchosen;
      status[ti] = st;
    }
    __syncwarp();
    for (int j = nchosen + lane; j < sp.max_samples; j += 32) nbr[ti * sp.max_samples + j] = 0xffffffffu;
    __syncwarp();
  }
}

}  // namespace

cudaError_t launch_search(const Launch& L, const SearchDev& sp, const GridDev& g, const double* tx,
                          const double* ty, const double* tz, const int64_t* perm, int64_t m, int loo,
                          uint32_t* nbr, int32_t* count, int8_t* status) {
  if (sp.rules) {
    constexpr int kWarps = 4;
    const bool small = sp.sgs && sp.max_samples <= 64 && sp.max_per_hole < 0 && !sp.plane && sp.min_sectors < 0 &&
                       sp.max_empty_sectors < 0 && sp.min_holes < 0;
    const bool tiny = small && sp.max_samples <= 32;
    const bool big = sp.max_samples > kMaxLU;  // more accepted holes than the small table holds
    const size_t smem = (big    ? sizeof(RulesSmem<kRulesK, kHoleHashBig>)
                         : tiny ? sizeof(RulesSmem<kSgsK32>)
                         : small ? sizeof(RulesSmem<kSgsK>)
                                 : sizeof(RulesSmem<kRulesK>)) *
                        kWarps;
    auto kern = big    ? k_search_rules<kRulesK, kHoleHashBig>
                : tiny ? k_search_rules<kSgsK32>
                : small ? k_search_rules<kSgsK>
                        : k_search_rules<kRulesK>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kWarps * 32, smem);
    if (e != cudaSuccess) return e;
    int64_t blocks = int64_t(L.sm_count) * (per_sm > 0 ? per_sm : 1);
    const int64_t need = (m + kWarps - 1) / kWarps;
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    kern<<<int(blocks), kWarps * 32, smem, L.stream>>>(sp, g, tx, ty, tz, perm, m, loo, nbr, count, status);
    ++*L.counter;
    return cudaGetLastError();
  }
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
