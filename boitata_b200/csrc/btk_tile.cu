// Tile-shared kriging solve: the systems of kTileTargets consecutive work
// slots (half of a 32-target search tile, so a compact patch of blocks)
// share one covariance table over the union of their samples.
//
// Reference: crates/estimation/src/kernel.rs:24-123 (per-system assembly,
// factorisation, estimate and variance); the quantities are the same as in
// btk_solve.cu, only the assembly is shared. Neighbouring blocks of a block
// model draw on nearly the same samples (a 4 x 4 block patch of the 3.2M-block
// drill-hole model needs about 52 distinct samples for its 16 x 32 system
// rows), so evaluating C(s_u, s_v) once per tile instead of once per system
// cuts the covariance evaluations per target from n(n-1)/2 = 496 to about 85.
// A system then gathers its rows from the table by union index.
//
// Per tile (one CTA of 128 threads):
//   1. the union of the tile's neighbour lists through a shared-memory hash
//      (open addressing, 1024 slots for at most 16 x 32 keys), its samples
//      numbered in order of first appearance (target by target, each list
//      nearest first), so that a system's rows sit at nearby indices and
//      their gathers spread over the shared-memory banks;
//   2. the union's world coordinates and the table C[u][v] (FP64, full
//      square, diagonal C0 + the sample's error variance), every lag from
//      lag_world, so an entry is bit for bit the one the per-system kernels
//      assemble and results do not depend on the tiling;
//   3. the systems: FP64 form one per warp, lane = row, the right-looking
//      LDL^T of btk_solve.cu with the row kept shifted (slot 0 = the pivot
//      column) and windows of 32, 24, 16 and 8 slots; mixed form two per
//      warp, lane = row of both as a float2 (system a in .x, b in .y), the
//      same elimination with packed FP32 FMA (__ffma2_rn) writing each pivot
//      column to a packed per-warp triangle in shared memory, a
//      column-oriented backward sweep over that triangle for x = C^-1 v, FP64
//      residuals r = v - C x from the FP64 table and the corrected forms
//      u'x_v + x_u'r_v, as in btk_solve.cu's mixed kernel. The tensor form
//      of the mixed solve (tuning tile_tensor) factors the same two systems
//      blocked instead: the lower triangles in place in the packed triangle,
//      8-column panels on the CUDA cores, the trailing updates as split-TF32
//      mma.sync tiles (factor_tc); the sweep and the FP64 tail are shared.
//
// Systems the tile does not take: a failed search (outputs written here),
// n > 32 (appended to `large`) and a sample flagged coincident at fit time
// (appended to `small`). A tile whose union exceeds the table, but not twice
// the table, is retried as two halves of 8 targets, each with a union of its
// own; what still does not fit goes to `small`. In the mixed form, a system
// whose FP32 factorisation breaks down goes to `redo` (FP64), and one whose
// corrected forms fail the residual test goes to `small`, where the
// per-system mixed kernel refines it iteratively (and hands it to `redo` if
// that does not converge). The per-system kernels of btk_solve.cu take
// those lists. The table entries do not depend on the order in which
// samples enter the union or on the tile (each is a function of its sample
// pair alone), so the FP64 form gives bit for bit the per-system kernel's
// results.
#include "btk_device.cuh"

namespace btk {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kT = kTileTargets;
constexpr int kHash = 1024;
constexpr uint32_t kEmpty = 0xffffffffu;
constexpr int kThreads = 128;

struct TileHead {
  int64_t ti[kT];
  int n[kT];
  int kind[kT];
  int twin[kT];
  int go[kT];
  int nu;
  int any;
  int wsum[kThreads / 32];
  uint8_t map[kT][32];
  uint16_t slot[kT][32];
};

struct WarpFp64 {
  double col[2][36];  // [buffer]: column below the pivot (0..30), pivot (32), sink (33)
  double rhs[2][4];
};

// Mixed form: two systems per warp, a float2 (system a, system b) per slot.
// Column k of the elimination (D_k L[j][k] for j > k, both systems) goes to
// lt[kLtPad + col_off(k) + j - k - 1]; a column starts on an even index and
// its length is rounded up to even, so it can be read in 16-byte lines. The
// pads keep the reads past a column's end, and the backward sweep's reads
// for rows that no longer need them, inside the warp's own area.
constexpr int kLtPad = 32;
constexpr int kLtLen = 512;  // sum over k of (31 - k) rounded up to even
struct WarpMixed {
  union {
    float2 lt[kLtPad + kLtLen + kLtPad];
    double xs[32][6];  // after the backward sweep: x of row j (a: c, 1, f; b: c, 1, f)
  };
  float2 prhs[2][4];  // [buffer]: pivot, y_c, y_1, y_f of the pivot row
};

// Start of column k in the packed triangle (see WarpMixed).
__device__ __forceinline__ int col_off(int k) {
  const int m = k >> 1;
  return 64 * m - 2 * m * m + ((k & 1) ? 32 - 2 * m : 0);
}

__host__ __device__ constexpr size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

struct Layout {
  size_t head, ukey, p, z, e, table, warp, total;
};

__host__ __device__ inline Layout layout(int umax, int stride, bool mixed) {
  Layout l;
  l.head = 0;
  l.ukey = align16(sizeof(TileHead));
  l.p = align16(l.ukey + sizeof(uint32_t) * umax);
  l.z = l.p + sizeof(double) * 3 * umax;
  l.e = l.z + sizeof(double) * umax;
  l.table = align16(l.e + sizeof(double) * umax);
  size_t tb = sizeof(double) * size_t(umax) * stride;
  const size_t hash = sizeof(uint32_t) * 2 * kHash + sizeof(uint8_t) * kHash;  // keys, first entries, uidx
  if (tb < hash) tb = hash;
  l.warp = align16(l.table + tb);
  l.total = l.warp + (kThreads / 32) * (mixed ? sizeof(WarpMixed) : sizeof(WarpFp64));
  return l;
}

__device__ __forceinline__ float rcp_approx(float d) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d));
  return r;
}

enum TileBuild { kTileEmpty = 0, kTileReady = 1, kTileOverflow = 2 };

// The union and covariance table of the tile's targets lo .. hi-1. The first
// pass (lo = 0, hi = kT) also reads the tile's targets and routes failed
// searches and n > 32; if its union exceeds the table it returns
// kTileOverflow and the caller retries the two halves, each with a union of
// its own, before a half that still does not fit goes to the per-system
// kernels. kTileEmpty: nothing left for the solve phase. Ends with the block
// synchronised.
__device__ int build_tile(const TileDev& a, int64_t tile, unsigned char* smem, const Layout& lay, int lo, int hi) {
  const SolveDev& s = a.s;
  TileHead& H = *reinterpret_cast<TileHead*>(smem + lay.head);
  uint32_t* ukey = reinterpret_cast<uint32_t*>(smem + lay.ukey);
  double* P = reinterpret_cast<double*>(smem + lay.p);
  double* Z = reinterpret_cast<double*>(smem + lay.z);
  double* E = reinterpret_cast<double*>(smem + lay.e);
  double* UU = reinterpret_cast<double*>(smem + lay.table);
  uint32_t* keys = reinterpret_cast<uint32_t*>(smem + lay.table);  // phase 1 only
  uint32_t* lowest = keys + kHash;  // per slot: the lowest entry t * 32 + r holding its key
  uint8_t* uidx = reinterpret_cast<uint8_t*>(lowest + kHash);
  const int tid = threadIdx.x;
  const int umax = a.umax, S = a.stride;
  const bool first = lo == 0 && hi == kT;

  if (first && tid < kT) {
    const int64_t w = tile * kT + tid;
    int64_t ti = w < a.nwork ? (a.perm ? a.perm[w] : w) : -1;
    int n = 0, kd = s.kind;
    if (ti >= 0) {
      n = s.count[ti];
      const int8_t st = s.sstatus[ti];
      if (s.kinds) kd = s.kinds[ti];
      if (st != BTK_ST_OK) {
        write_fail(s, ti, st, 0);
        ti = -1;
      } else if (n <= 0) {
        write_fail(s, ti, BTK_ST_SEARCH_FAILED, 0);
        ti = -1;
      } else if (n > 32) {
        a.large[atomicAdd(reinterpret_cast<unsigned long long*>(a.large_len), 1ull)] = ti;
        ti = -1;
      }
    }
    H.ti[tid] = ti;
    H.n[tid] = ti >= 0 ? n : 0;
    H.kind[tid] = kd;
  }
  if (tid < kT) H.twin[tid] = 0;
  if (tid == 0) H.nu = 0;
  for (int i = tid; i < kHash; i += kThreads) keys[i] = kEmpty, lowest[i] = kEmpty;
  __syncthreads();

  // 1. Union of the neighbour lists.
  for (int e = tid; e < kT * 32; e += kThreads) {
    const int t = e >> 5, r = e & 31;
    const int64_t ti = H.ti[t];
    if (ti < 0 || r >= H.n[t] || t < lo || t >= hi) continue;
    const uint32_t key = s.nbr[ti * s.max_samples + r];
    if (s.twin && s.twin[key]) H.twin[t] = 1;
    uint32_t h = (key * 2654435761u) >> 22;  // multiplicative hash, 10 bits
    for (int probe = 0; probe < kHash; ++probe) {  // at most kT * 32 < kHash keys: a free slot exists
      const uint32_t old = atomicCAS(&keys[h], kEmpty, key);
      if (old == kEmpty || old == key) break;
      h = (h + 1) & (kHash - 1);
    }
    H.slot[t][r] = uint16_t(h);
    atomicMin(&lowest[h], uint32_t(e));
  }
  __syncthreads();
  // Union indices in order of first appearance, target by target and each
  // target's list in (d2, index) order: a system's rows then take nearby
  // indices, which spread its row gathers over the shared-memory banks (the
  // table's values do not depend on the indices). Thread tid takes entries
  // 4 tid .. 4 tid + 3; a block scan of their first-appearance counts gives
  // each new sample its index.
  {
    uint32_t fl = 0;  // bit j: entry 4 tid + j is its key's first
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int e = 4 * tid + j, t = e >> 5, r = e & 31;
      if (H.ti[t] >= 0 && r < H.n[t] && t >= lo && t < hi && lowest[H.slot[t][r]] == uint32_t(e)) fl |= 1u << j;
    }
    const int cnt = __popc(fl);
    const int lane = tid & 31, warp = tid >> 5;
    int inc = cnt;  // inclusive warp scan
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(kFull, inc, o);
      if (lane >= o) inc += v;
    }
    if (lane == 31) H.wsum[warp] = inc;
    __syncthreads();
    int base = inc - cnt;
    for (int w = 0; w < warp; ++w) base += H.wsum[w];
    if (tid == kThreads - 1) H.nu = base + cnt;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (!((fl >> j) & 1u)) continue;
      const int e = 4 * tid + j, t = e >> 5, r = e & 31;
      const int h = H.slot[t][r];
      uidx[h] = uint8_t(base < 255 ? base : 255);
      if (base < umax) ukey[base] = keys[h];
      ++base;
    }
  }
  __syncthreads();
  const int nu = H.nu;
  if (nu > umax) {  // the table would not hold these targets: halves, then per-system kernels
    // Halves only when both could fit: above 2 umax one of them holds more
    // than umax samples (scattered targets, a simulation's path order).
    if (first && nu <= 2 * umax) return kTileOverflow;  // uniform: every thread read the same H.nu
    if (tid >= lo && tid < hi && H.ti[tid] >= 0)
      a.small[atomicAdd(reinterpret_cast<unsigned long long*>(a.small_len), 1ull)] = H.ti[tid];
    __syncthreads();
    return kTileEmpty;
  }
  for (int e = tid; e < kT * 32; e += kThreads) {
    const int t = e >> 5, r = e & 31;
    // 0 outside lo .. hi: a map entry always indexes this pass's table
    H.map[t][r] = (H.ti[t] >= 0 && r < H.n[t] && t >= lo && t < hi) ? uidx[H.slot[t][r]] : uint8_t(0);
  }
  if (tid < kT) {
    const int64_t ti = H.ti[tid];
    const bool in = ti >= 0 && tid >= lo && tid < hi;
    const bool go = in && !H.twin[tid];
    if (in && !go) a.small[atomicAdd(reinterpret_cast<unsigned long long*>(a.small_len), 1ull)] = ti;
    H.go[tid] = go;
  }
  if (tid == 0) {
    int any = 0;
    for (int t = lo; t < hi; ++t) any |= H.ti[t] >= 0 && !H.twin[t];
    H.any = any;
  }
  __syncthreads();
  if (!H.any) return kTileEmpty;  // uniform: every thread read the same H.any

  // 2. Union coordinates (world) and the covariance table.
  for (int u = tid; u < nu; u += kThreads) {
    const uint32_t k = ukey[u];
    P[u] = s.sx[k], P[umax + u] = s.sy[k], P[2 * umax + u] = s.sz[k];
    Z[u] = s.sv[k];
    E[u] = s.se ? s.se[k] : 0.0;
  }
  __syncthreads();  // the hash is dead from here: its space becomes the table
  const int npairs = nu * (nu - 1) / 2;
  for (int e = tid; e < npairs; e += kThreads) {
    int i, j;
    tri_index(e, i, j);
    const double c = cov64(s.vg, lag_world(s.vg, P[j], P[umax + j], P[2 * umax + j], P[i], P[umax + i], P[2 * umax + i]));
    UU[i * S + j] = c;
    UU[j * S + i] = c;
  }
  for (int u = tid; u < nu; u += kThreads) UU[u * S + u] = s.vg.c0 + E[u];
  __syncthreads();
  return kTileReady;
}

// C(target, union sample u).
__device__ __forceinline__ double cov_to(const SolveDev& s, const double* P, int umax, int u, const double t[3]) {
  return support_cov(s, t[0], t[1], t[2], P[u], P[umax + u], P[2 * umax + u]);
}

// Pivots k0 .. k1-1 of the FP64 right-looking LDL^T with the forward
// substitution of y fused in. The row is kept shifted so that slot 0 holds
// the current pivot column: a step writes it to the warp's line, then
// A[q] <- A[q+1] - f col[q] over the W slots that still hold live columns
// (the shift makes the loop body the same for every k, so it is a runtime
// loop and the code stays small). Same operations, in the same order, as
// the unrolled per-system kernel.
template <int W>
__device__ __forceinline__ void eliminate(double (&A)[32], int k0, int k1, int lane, WarpFp64& Ws, double (&y)[3],
                                          double& dme, bool& sing, double thr) {
  for (int k = k0; k < k1; ++k) {
    const int b = k & 1;
    Ws.col[b][lane > k ? lane - k - 1 : (lane == k ? 32 : 33)] = A[0];
    if (lane == k) Ws.rhs[b][0] = y[0], Ws.rhs[b][1] = y[1], Ws.rhs[b][2] = y[2];
    __syncwarp();
    const double d = Ws.col[b][32];
    if (!(d > thr)) {  // NaN or at most 1e-12 C0 (kernel.rs:61)
      sing = true;
      return;
    }
    if (lane == k) dme = d;
    const double f = lane > k ? A[0] * (1.0 / d) : 0.0;
#pragma unroll
    for (int q = 0; q < W; q += 2) {
      const double2 cv = *reinterpret_cast<const double2*>(&Ws.col[b][q]);
      A[q] = fma(-f, cv.x, A[q + 1]);
      A[q + 1] = q + 2 < 32 ? fma(-f, cv.y, A[q + 2]) : 0.0;
    }
    const double2 r01 = *reinterpret_cast<const double2*>(&Ws.rhs[b][0]);
    y[0] = fma(-f, r01.x, y[0]);
    y[1] = fma(-f, r01.y, y[1]);
    y[2] = fma(-f, Ws.rhs[b][2], y[2]);
  }
}

// FP64 form: system t of the tile on one warp.
__device__ void solve_fp64(const TileDev& a, const TileHead& H, const double* P, const double* Z, const double* UU,
                           int umax, int S, WarpFp64& W, int t) {
  const SolveDev& s = a.s;
  const int lane = threadIdx.x & 31;
  const int64_t ti = H.ti[t];
  const int n = H.n[t], kind = H.kind[t];
  const double c0 = s.vg.c0;
  const bool have = lane < n;
  const int ma = H.map[t][lane];
  const double pt[3] = {s.tx[ti], s.ty[ti], s.tz[ti]};
  const double c = have ? cov_to(s, P, umax, ma, pt) : 0.0;
  const double zf = have ? kind_f(kind, s.kparam, Z[ma]) : 0.0;
  const double* Ur = UU + ma * S;
  double A[32];
#pragma unroll
  for (int q = 0; q < 32; ++q) A[q] = (have && q < n) ? Ur[H.map[t][q]] : (q == lane ? 1.0 : 0.0);
  double y[3] = {have ? c : 0.0, have ? 1.0 : 0.0, have ? zf : 0.0};
  double dme = 1.0;
  bool sing = false;
  const double thr = kPivot * c0;
  // Four stages of eight pivots over windows of 32, 24, 16 and 8 slots (the
  // columns a step can still change), each a runtime loop.
  const int n1 = min(n, 8), n2 = min(n, 16), n3 = min(n, 24);
  eliminate<32>(A, 0, n1, lane, W, y, dme, sing, thr);
  if (!sing) eliminate<24>(A, n1, n2, lane, W, y, dme, sing, thr);
  if (!sing) eliminate<16>(A, n2, n3, lane, W, y, dme, sing, thr);
  if (!sing) eliminate<8>(A, n3, n, lane, W, y, dme, sing, thr);
  __syncwarp();
  if (sing) {
    if (lane == 0) write_fail(s, ti, BTK_ST_SINGULAR, 0);
    return;
  }
  const double y0 = y[0], y1 = y[1], y2 = y[2];
  const double wt = have ? 1.0 / dme : 0.0;
  double v[5] = {y1 * y0 * wt, y1 * y1 * wt, y2 * y0 * wt, y2 * y1 * wt, y0 * y0 * wt};
#pragma unroll
  for (int q = 0; q < 5; ++q)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(kFull, v[q], o);
  if (lane == 0) epilogue(s, kind, ti, v, n, 0);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ float warp_maxf(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

__device__ __forceinline__ float2 rcp2(float2 d) { return make_float2(rcp_approx(d.x), rcp_approx(d.y)); }

// Entry (i, c), i > c, of the packed lower triangle (see WarpMixed); the
// tensor form keeps the diagonal in the front pad, lt[c].
__device__ __forceinline__ int tri(int i, int c) { return kLtPad + col_off(c) + i - c - 1; }

// x = hi + lo with hi and lo in TF32 (round to nearest): a product of two
// such splits, hi*hi + hi*lo + lo*hi, carries about FP32's precision.
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(x));
  const float r = x - __uint_as_float(hi);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(r));
}

// d += a b for a 16x8 (row) by 8x8 (col) TF32 tile, FP32 accumulation.
// Fragments (PTX ISA, mma.m16n8k8 .tf32), g = lane / 4, t = lane % 4:
// a0 (g, t), a1 (g + 8, t), a2 (g, t + 4), a3 (g + 8, t + 4);
// b0 (k = t, n = g), b1 (k = t + 4, n = g);
// d0 (g, 2t), d1 (g, 2t + 1), d2 (g + 8, 2t), d3 (g + 8, 2t + 1).
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// The FP32 LDL^T of two systems (float2: a in .x, b in .y) in blocked form
// with the trailing updates on the tensor pipe. The lower triangles sit in
// place in the warp's packed triangle (padded rows and columns: the
// identity); each panel of 8 columns is factored row per lane on the CUDA
// cores, with the forward substitution of y fused in, writing its columns
// D_k L[i][k] back in place; the trailing lower triangle then takes
// -W L^T (W = L D, the panel's columns) as 16x8 tiles of split-TF32 mma,
// three per tile and system (lo*hi, hi*lo, hi*hi). On return the triangle
// holds what the unblocked form writes, so the backward sweep is shared.
__device__ __forceinline__ void factor_tc(const TileHead& H, const double* Ua, const double* Ub, WarpMixed& Ws,
                                          int ta, int tb, int na, int nb, int nmax, int lane, float2 (&y)[3],
                                          float2& dme) {
  float2* lt = Ws.lt;
  // The columns that take pivots, every row below the diagonal; columns
  // past nmax are never read for a system's results.
  for (int c = 0; c < nmax; ++c) {
    if (lane >= c) {
      const int mca = H.map[ta][c], mcb = H.map[tb][c];
      const float vx = (lane < na && c < na) ? float(Ua[mca]) : (lane == c ? 1.f : 0.f);
      const float vy = (lane < nb && c < nb) ? float(Ub[mcb]) : (lane == c ? 1.f : 0.f);
      lt[lane == c ? c : tri(lane, c)] = make_float2(vx, vy);
    }
  }
  __syncwarp();
  const int g = lane >> 2, t = lane & 3;
  const int np = (nmax + 7) >> 3;
  for (int p = 0; p < np; ++p) {
    const int kb = 8 * p;
    float2 pa[8];  // this lane's row in the panel's columns
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int c = kb + m;
      pa[m] = lane > c ? lt[tri(lane, c)] : (lane == c ? lt[c] : make_float2(0.f, 0.f));
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int k = kb + j;
      if (k >= nmax) break;
      const int b = k & 1;
      if (lane > k) lt[tri(lane, k)] = pa[j];
      if (lane == k) {  // pivot and right-hand side, two 16-byte stores
        reinterpret_cast<float4*>(Ws.prhs[b])[0] = make_float4(pa[j].x, pa[j].y, y[0].x, y[0].y);
        reinterpret_cast<float4*>(Ws.prhs[b])[1] = make_float4(y[1].x, y[1].y, y[2].x, y[2].y);
      }
      __syncwarp();
      const float4 p0 = reinterpret_cast<const float4*>(Ws.prhs[b])[0];
      const float4 p1 = reinterpret_cast<const float4*>(Ws.prhs[b])[1];
      if (lane == k) dme = make_float2(p0.x, p0.y);
      const float2 nrd = make_float2(rcp_approx(-p0.x), rcp_approx(-p0.y));
      const float2 nf = lane > k ? __fmul2_rn(pa[j], nrd) : make_float2(0.f, 0.f);  // -L[lane][k]
      // The panel's later columns: column k at rows kb + m, entries m - j - 1.
      const float2* col = lt + kLtPad + col_off(k);
#pragma unroll
      for (int m = j + 1; m < 8; m += 2) {
        const float4 c4 = *reinterpret_cast<const float4*>(&col[m - j - 1]);
        pa[m] = __ffma2_rn(nf, make_float2(c4.x, c4.y), pa[m]);
        if (m + 1 < 8) pa[m + 1] = __ffma2_rn(nf, make_float2(c4.z, c4.w), pa[m + 1]);
      }
      y[0] = __ffma2_rn(nf, make_float2(p0.z, p0.w), y[0]);
      y[1] = __ffma2_rn(nf, make_float2(p1.x, p1.y), y[1]);
      y[2] = __ffma2_rn(nf, make_float2(p1.z, p1.w), y[2]);
    }
    if (p + 1 >= np) break;
    // A full panel (8 (p + 1) < nmax): the trailing update on the tensor pipe.
    __syncwarp();
    const float2 d0 = make_float2(__shfl_sync(kFull, dme.x, kb + t), __shfl_sync(kFull, dme.y, kb + t));
    const float2 d1 = make_float2(__shfl_sync(kFull, dme.x, kb + t + 4), __shfl_sync(kFull, dme.y, kb + t + 4));
    const float2 rd[2] = {rcp2(d0), rcp2(d1)};
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      if (16 * mt + 15 < kb + 8) continue;  // every row of the m-tile already pivoted
      uint32_t ah[2][4], al[2][4];          // [system][fragment]: -W[r][kb + t + 4 (e / 2)]
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int r = 16 * mt + g + 8 * (e & 1), kk = kb + t + 4 * (e >> 1);
        const float2 w = r > kk ? lt[tri(r, kk)] : make_float2(0.f, 0.f);
        split_tf32(-w.x, ah[0][e], al[0][e]);
        split_tf32(-w.y, ah[1][e], al[1][e]);
      }
      for (int nt = p + 1; nt < np; ++nt) {
        if (16 * mt + 15 < 8 * nt) continue;  // above the diagonal
        uint32_t bh[2][2], bl[2][2];          // [system][fragment]: L[8 nt + g][kb + t + 4 q]
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int c = 8 * nt + g, kk = kb + t + 4 * q;
          const float2 w = lt[tri(c, kk)];
          split_tf32(w.x * rd[q].x, bh[0][q], bl[0][q]);
          split_tf32(w.y * rd[q].y, bh[1][q], bl[1][q]);
        }
        float cx[4], cy[4];
        int at[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int r = 16 * mt + g + 8 * (e >> 1), c = 8 * nt + 2 * t + (e & 1);
          at[e] = r > c ? tri(r, c) : (r == c ? c : -1);
          const float2 v = at[e] >= 0 ? lt[at[e]] : make_float2(0.f, 0.f);
          cx[e] = v.x, cy[e] = v.y;
        }
        mma_tf32(cx, al[0], bh[0]);
        mma_tf32(cx, ah[0], bl[0]);
        mma_tf32(cx, ah[0], bh[0]);
        mma_tf32(cy, al[1], bh[1]);
        mma_tf32(cy, ah[1], bl[1]);
        mma_tf32(cy, ah[1], bh[1]);
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (at[e] >= 0) lt[at[e]] = make_float2(cx[e], cy[e]);
      }
    }
    __syncwarp();
  }
}

// Pivots k0 .. k1-1 of the FP32 LDL^T of two systems at once (float2 lanes:
// system a in .x, b in .y), forward substitution of y fused in; the row is
// kept shifted (slot 0 = the current pivot column) and a step updates the W
// slots that can still hold live columns, as in the FP64 eliminate().
template <int W>
__device__ __forceinline__ void eliminate2(float2 (&A)[32], int k0, int k1, int lane, WarpMixed& Ws,
                                           float2 (&y)[3], float2& dme) {
  float2* col = Ws.lt + kLtPad + col_off(k0);
  for (int k = k0; k < k1; ++k) {
    const int b = k & 1;
    if (lane > k) col[lane - k - 1] = A[0];
    if (lane == k) {  // pivot and right-hand side, two 16-byte stores
      reinterpret_cast<float4*>(Ws.prhs[b])[0] = make_float4(A[0].x, A[0].y, y[0].x, y[0].y);
      reinterpret_cast<float4*>(Ws.prhs[b])[1] = make_float4(y[1].x, y[1].y, y[2].x, y[2].y);
    }
    __syncwarp();
    const float4 p0 = reinterpret_cast<const float4*>(Ws.prhs[b])[0];
    const float4 p1 = reinterpret_cast<const float4*>(Ws.prhs[b])[1];
    if (lane == k) dme = make_float2(p0.x, p0.y);
    const float2 nrd = make_float2(rcp_approx(-p0.x), rcp_approx(-p0.y));
    const float2 nf = lane > k ? __fmul2_rn(A[0], nrd) : make_float2(0.f, 0.f);  // -L[lane][k]
#pragma unroll
    for (int q = 0; q < W; q += 2) {
      const float4 c4 = *reinterpret_cast<const float4*>(&col[q]);
      A[q] = __ffma2_rn(nf, make_float2(c4.x, c4.y), A[q + 1]);
      A[q + 1] = q + 2 < 32 ? __ffma2_rn(nf, make_float2(c4.z, c4.w), A[q + 2]) : make_float2(0.f, 0.f);
    }
    y[0] = __ffma2_rn(nf, make_float2(p0.z, p0.w), y[0]);
    y[1] = __ffma2_rn(nf, make_float2(p1.x, p1.y), y[1]);
    y[2] = __ffma2_rn(nf, make_float2(p1.z, p1.w), y[2]);
    col += (32 - k) & ~1;  // the next column: this one's length rounded up to even
  }
}

// Mixed form: systems 2p (a) and 2p + 1 (b) of the tile on one warp, lane = row;
// TC: the blocked factorisation with tensor-pipe trailing updates.
template <bool TC>
__device__ void solve_mixed(const TileDev& a, const TileHead& H, const double* P, const double* Z, const double* UU,
                            int umax, int S, WarpMixed& W, int p) {
  const SolveDev& s = a.s;
  const int lane = threadIdx.x & 31;
  const int ta = 2 * p, tb = 2 * p + 1;
  const bool go_a = H.go[ta] != 0, go_b = H.go[tb] != 0;
  const int na = go_a ? H.n[ta] : 0, nb = go_b ? H.n[tb] : 0;
  const int nmax = max(na, nb);
  const double c0 = s.vg.c0;
  const bool ha = lane < na, hb = lane < nb;
  const int ma = H.map[ta][lane], mb = H.map[tb][lane];
  double ca = 0.0, cb = 0.0, za = 0.0, zb = 0.0;
  if (ha) {
    const int64_t ti = H.ti[ta];
    const double pt[3] = {s.tx[ti], s.ty[ti], s.tz[ti]};
    ca = cov_to(s, P, umax, ma, pt);
    za = kind_f(H.kind[ta], s.kparam, Z[ma]);
  }
  if (hb) {
    const int64_t ti = H.ti[tb];
    const double pt[3] = {s.tx[ti], s.ty[ti], s.tz[ti]};
    cb = cov_to(s, P, umax, mb, pt);
    zb = kind_f(H.kind[tb], s.kparam, Z[mb]);
  }
  const double* Ua = UU + ma * S;
  const double* Ub = UU + mb * S;
  float2 y[3] = {make_float2(float(ca), float(cb)), make_float2(ha ? 1.f : 0.f, hb ? 1.f : 0.f),
                 make_float2(float(za), float(zb))};
  float2 dme = make_float2(1.f, 1.f);
  if constexpr (TC) {
    factor_tc(H, Ua, Ub, W, ta, tb, na, nb, nmax, lane, y, dme);
  } else {
    float2 A[32];
#pragma unroll
    for (int q = 0; q < 32; ++q) {
      A[q].x = (ha && q < na) ? float(Ua[H.map[ta][q]]) : (q == lane ? 1.f : 0.f);
      A[q].y = (hb && q < nb) ? float(Ub[H.map[tb][q]]) : (q == lane ? 1.f : 0.f);
    }
    const int n1 = min(nmax, 8), n2 = min(nmax, 16), n3 = min(nmax, 24);
    eliminate2<32>(A, 0, n1, lane, W, y, dme);
    eliminate2<24>(A, n1, n2, lane, W, y, dme);
    eliminate2<16>(A, n2, n3, lane, W, y, dme);
    eliminate2<8>(A, n3, nmax, lane, W, y, dme);
  }
  // An FP32 pivot that is NaN or at most n ulp(C0) is not resolved from the
  // rounding of its row: the FP64 form takes the system (and with it the
  // singular decision, kernel.rs:61). Lane k holds pivot k; the padded rows'
  // unit pivots of the smaller system take no part.
  const bool weak_a = __any_sync(kFull, ha && !(dme.x > float(na) * 1.1920929e-7f * float(c0)));
  const bool weak_b = __any_sync(kFull, hb && !(dme.y > float(nb) * 1.1920929e-7f * float(c0)));
  __syncwarp();
  // Backward sweep L^T x = D^-1 y, column-oriented: once x_k is known every
  // row i < k takes D_i L[k][i] x_k (column i of the triangle) into acc_i,
  // and x_i = y_i / D_i - acc_i / D_i: y / D is taken once, so a step costs
  // one packed FMA per right-hand side.
  const float2 rdme = rcp2(dme), nrd = make_float2(-rdme.x, -rdme.y);
  const float2 yd[3] = {__fmul2_rn(y[0], rdme), __fmul2_rn(y[1], rdme), __fmul2_rn(y[2], rdme)};
  float2 acc[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
  float2 x[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
  const float2* my_col = W.lt + kLtPad + col_off(lane) - lane - 1;  // + k: D_i L[k][i]
  for (int k = nmax - 1; k >= 0; --k) {
    float2 z[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const float2 w = __ffma2_rn(acc[v], nrd, yd[v]);
      z[v].x = __shfl_sync(kFull, w.x, k);
      z[v].y = __shfl_sync(kFull, w.y, k);
    }
    if (lane == k) x[0] = z[0], x[1] = z[1], x[2] = z[2];
    // Rows below k take no more terms: their lanes skip the load, which
    // would only add bank conflicts (the columns' starts fall on few banks).
    const float2 l = lane < k ? my_col[k] : make_float2(0.f, 0.f);
#pragma unroll
    for (int v = 0; v < 3; ++v) acc[v] = __ffma2_rn(l, z[v], acc[v]);
  }
  __syncwarp();  // the triangle is dead: its space holds x for the residuals
  const double xa[3] = {ha ? double(x[0].x) : 0.0, ha ? double(x[1].x) : 0.0, ha ? double(x[2].x) : 0.0};
  const double xb[3] = {hb ? double(x[0].y) : 0.0, hb ? double(x[1].y) : 0.0, hb ? double(x[2].y) : 0.0};
  W.xs[lane][0] = xa[0], W.xs[lane][1] = xa[1], W.xs[lane][2] = xa[2];
  W.xs[lane][3] = xb[0], W.xs[lane][4] = xb[1], W.xs[lane][5] = xb[2];
  __syncwarp();
  // FP64 residuals r_v = v - C x_v from the FP64 table (rows past n have x = 0).
  double aa[3] = {0.0, 0.0, 0.0}, ab[3] = {0.0, 0.0, 0.0};
  for (int j = 0; j < nmax; ++j) {
    const double2 x01 = *reinterpret_cast<const double2*>(&W.xs[j][0]);
    const double2 x23 = *reinterpret_cast<const double2*>(&W.xs[j][2]);
    const double2 x45 = *reinterpret_cast<const double2*>(&W.xs[j][4]);
    const double cja = Ua[H.map[ta][j]], cjb = Ub[H.map[tb][j]];
    aa[0] = fma(cja, x01.x, aa[0]), aa[1] = fma(cja, x01.y, aa[1]), aa[2] = fma(cja, x23.x, aa[2]);
    ab[0] = fma(cjb, x23.y, ab[0]), ab[1] = fma(cjb, x45.x, ab[1]), ab[2] = fma(cjb, x45.y, ab[2]);
  }
  __syncwarp();
  double ra[3] = {0.0, 0.0, 0.0}, rb[3] = {0.0, 0.0, 0.0};
  if (ha) ra[0] = ca - aa[0], ra[1] = 1.0 - aa[1], ra[2] = za - aa[2];
  if (hb) rb[0] = cb - ab[0], rb[1] = 1.0 - ab[1], rb[2] = zb - ab[2];
  // Refinement tests, as in the per-system mixed kernel: the corrected forms
  // err by about rho^2 C0 / D_min (rho the relative residual).
  const float cmax_a = warp_maxf(ha ? float(fabs(ca)) : 0.f), cmax_b = warp_maxf(hb ? float(fabs(cb)) : 0.f);
  const float zmax_a = warp_maxf(ha ? float(fabs(za)) : 0.f), zmax_b = warp_maxf(hb ? float(fabs(zb)) : 0.f);
  const double ica = 1.0 / fmax(double(cmax_a), 1e-300), iza = 1.0 / fmax(double(zmax_a), 1e-300);
  const double icb = 1.0 / fmax(double(cmax_b), 1e-300), izb = 1.0 / fmax(double(zmax_b), 1e-300);
  const float rho_a = warp_maxf(float(fmax(fmax(fabs(ra[0]) * ica, fabs(ra[1])), fabs(ra[2]) * iza)));
  const float rho_b = warp_maxf(float(fmax(fmax(fabs(rb[0]) * icb, fabs(rb[1])), fabs(rb[2]) * izb)));
  const float dmin_a = -warp_maxf(ha ? -dme.x : -3.0e38f), dmin_b = -warp_maxf(hb ? -dme.y : -3.0e38f);
  double va[5] = {xa[0] + xa[1] * ra[0], xa[1] + xa[1] * ra[1], za * xa[0] + xa[2] * ra[0], za * xa[1] + xa[2] * ra[1],
                  ca * xa[0] + xa[0] * ra[0]};
  double vb[5] = {xb[0] + xb[1] * rb[0], xb[1] + xb[1] * rb[1], zb * xb[0] + xb[2] * rb[0], zb * xb[1] + xb[2] * rb[1],
                  cb * xb[0] + xb[0] * rb[0]};
#pragma unroll
  for (int q = 0; q < 5; ++q) va[q] = warp_sum(va[q]), vb[q] = warp_sum(vb[q]);
  if (lane < 2) {
    const bool is_a = lane == 0;
    const bool go = is_a ? go_a : go_b;
    if (go) {
      const int64_t ti = H.ti[is_a ? ta : tb];
      const double* v = is_a ? va : vb;
      const double rho = is_a ? rho_a : rho_b, dmin = is_a ? dmin_a : dmin_b;
      const bool weak = is_a ? weak_a : weak_b;
      if (weak)
        a.redo[atomicAdd(reinterpret_cast<unsigned long long*>(a.redo_len), 1ull)] = ti;
      else if (!(rho * rho * c0 / dmin <= 1e-8) || !(v[1] > 0.0) || !(fabs(v[0]) < 1e30))
        a.small[atomicAdd(reinterpret_cast<unsigned long long*>(a.small_len), 1ull)] = ti;  // refined there
      else
        epilogue(s, H.kind[is_a ? ta : tb], ti, v, is_a ? na : nb, 0);
    }
  }
  __syncwarp();
}

// Four CTAs per SM in both forms: 128 registers a thread (the mixed form's
// two float2 rows fit without spills), and with a 64-sample table both
// forms' shared memory fits four times in the SM's 228 KB. The mixed form
// at three CTAs (168 registers) took 20.1 ms at 3.2M blocks, at four 18.1.
template <int FORM>  // 0: FP64; 1: mixed; 2: mixed with the tensor-pipe factorisation
__global__ void __launch_bounds__(kThreads, 4) k_tile(TileDev a) {
  constexpr bool MIXED = FORM != 0;
  extern __shared__ __align__(16) unsigned char smem[];
  const Layout lay = layout(a.umax, a.stride, MIXED);
  const TileHead& H = *reinterpret_cast<const TileHead*>(smem + lay.head);
  const double* P = reinterpret_cast<const double*>(smem + lay.p);
  const double* Z = reinterpret_cast<const double*>(smem + lay.z);
  const double* UU = reinterpret_cast<const double*>(smem + lay.table);
  const int warp = threadIdx.x >> 5;
  const int64_t ntiles = (a.nwork + kT - 1) / kT;
  // Systems whose go flag is set; a half tile (an even number of targets)
  // leaves the other half's flags clear, so the mixed form's pairs stay whole.
  auto solve_all = [&]() {
    if (MIXED) {
      WarpMixed& W = reinterpret_cast<WarpMixed*>(smem + lay.warp)[warp];
      for (int p = warp; p < kT / 2; p += kThreads / 32)
        if (H.go[2 * p] || H.go[2 * p + 1]) solve_mixed<FORM == 2>(a, H, P, Z, UU, a.umax, a.stride, W, p);
    } else {
      WarpFp64& W = reinterpret_cast<WarpFp64*>(smem + lay.warp)[warp];
      for (int t = warp; t < kT; t += kThreads / 32)
        if (H.go[t]) solve_fp64(a, H, P, Z, UU, a.umax, a.stride, W, t);
    }
  };
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    __syncthreads();  // the previous tile's systems are done with the table
    const int built = build_tile(a, tile, smem, lay, 0, kT);
    if (built == kTileReady) {
      solve_all();
    } else if (built == kTileOverflow) {
      for (int h = 0; h < 2; ++h) {
        __syncthreads();  // the previous half is done with the table and the head
        if (build_tile(a, tile, smem, lay, h * (kT / 2), (h + 1) * (kT / 2)) == kTileReady) solve_all();
      }
    }
  }
}

}  // namespace

namespace {

template <int FORM>
cudaError_t launch_form(const Launch& L, const TileDev& a) {
  const size_t smem = layout(a.umax, a.stride, FORM != 0).total;
  int per_sm = 0;
  cudaError_t e = cudaFuncSetAttribute(k_tile<FORM>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tile<FORM>, kThreads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  if (L.tuning.solve_blocks_per_sm > 0 && L.tuning.solve_blocks_per_sm < per_sm) per_sm = L.tuning.solve_blocks_per_sm;
  const int64_t ntiles = (a.nwork + kT - 1) / kT;
  int64_t blocks = int64_t(L.sm_count) * per_sm;
  if (blocks > ntiles) blocks = ntiles;
  if (blocks < 1) blocks = 1;
  k_tile<FORM><<<int(blocks), kThreads, smem, L.stream>>>(a);
  ++*L.counter;
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_tile(const Launch& L, const TileDev& a0, bool mixed) {
  TileDev a = a0;
  if (a.umax < 2 || a.umax > 255) return cudaErrorInvalidValue;
  a.stride = a.umax | 1;  // odd row stride
  if (!mixed) return launch_form<0>(L, a);
  return L.tuning.tile_tensor ? launch_form<2>(L, a) : launch_form<1>(L, a);
}

}  // namespace btk
