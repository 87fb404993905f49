// Fit-time kernels: projection of the samples into the search frame, their
// bounding box, the uniform grid (counting sort by cell), the coincident-
// sample flags, and block-model centroids.
//
// The projection p = frame * (s - origin) with the origin at the first
// sample follows crates/estimation/src/search.rs:704-745 bit for bit
// (exact-order FP64, no FMA), since the search ranks samples by distances
// between these points. The grid itself is this engine's own: any grid
// gives the same (d2, index)-ordered candidates as search/grid.rs.
#include <cfloat>

#include <cub/device/device_radix_sort.cuh>

#include "btk_device.cuh"

namespace btk {
namespace {

__global__ void k_project(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                          const double* __restrict__ z, const double* __restrict__ frame,
                          const double* __restrict__ origin, double* px, double* py, double* pz) {
  double M[9], o[3];
#pragma unroll
  for (int k = 0; k < 9; ++k) M[k] = frame[k];
  o[0] = origin[0], o[1] = origin[1], o[2] = origin[2];
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    double d[3] = {xsub(x[i], o[0]), xsub(y[i], o[1]), xsub(z[i], o[2])}, p[3];
    mulv_exact(M, d, p);
    px[i] = p[0], py[i] = p[1], pz[i] = p[2];
  }
}

// Per-block min/max of the three coordinates, then one block folds them.
__global__ void k_bounds_partial(int64_t n, const double* px, const double* py, const double* pz, double* partial) {
  __shared__ double s[6][256];
  double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    double p[3] = {px[i], py[i], pz[i]};
#pragma unroll
    for (int d = 0; d < 3; ++d) lo[d] = fmin(lo[d], p[d]), hi[d] = fmax(hi[d], p[d]);
  }
  for (int d = 0; d < 3; ++d) s[d][threadIdx.x] = lo[d], s[3 + d][threadIdx.x] = hi[d];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int d = 0; d < 3; ++d) {
        s[d][threadIdx.x] = fmin(s[d][threadIdx.x], s[d][threadIdx.x + w]);
        s[3 + d][threadIdx.x] = fmax(s[3 + d][threadIdx.x], s[3 + d][threadIdx.x + w]);
      }
    __syncthreads();
  }
  if (threadIdx.x < 6) partial[blockIdx.x * 6 + threadIdx.x] = s[threadIdx.x][0];
}

__global__ void k_bounds_final(int nblocks, const double* partial, double* out6) {
  if (threadIdx.x != 0) return;
  double r[6] = {DBL_MAX, DBL_MAX, DBL_MAX, -DBL_MAX, -DBL_MAX, -DBL_MAX};
  for (int b = 0; b < nblocks; ++b)
    for (int d = 0; d < 3; ++d) r[d] = fmin(r[d], partial[6 * b + d]), r[3 + d] = fmax(r[3 + d], partial[6 * b + 3 + d]);
  for (int k = 0; k < 6; ++k) out6[k] = r[k];
}

__device__ __forceinline__ int cell_axis(double p, double lo, double h, int dim) {
  double u = floor((p - lo) / h);
  u = fmin(fmax(u, 0.0), double(dim - 1));  // fmax maps NaN to 0
  return int(u);
}

__global__ void k_cell_count(int64_t n, const double* px, const double* py, const double* pz, GridDev g,
                             uint32_t* count, uint32_t* cell_of) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    int cx = cell_axis(px[i], g.lo[0], g.h, g.dims[0]);
    int cy = cell_axis(py[i], g.lo[1], g.h, g.dims[1]);
    int cz = cell_axis(pz[i], g.lo[2], g.h, g.dims[2]);
    int64_t id = cx + int64_t(g.dims[0]) * (cy + int64_t(g.dims[1]) * cz);
    cell_of[i] = uint32_t(id);
    atomicAdd(&count[id], 1u);
  }
}

// Exclusive scan of `count` into `start` (ncells + 1 entries) by one block:
// each thread sums a contiguous chunk, the block scans the chunk sums.
__global__ void k_scan(int64_t ncells, const uint32_t* count, uint32_t* start) {
  __shared__ uint32_t sums[1024];
  int64_t chunk = (ncells + blockDim.x - 1) / blockDim.x;
  int64_t a = threadIdx.x * chunk, b = min(ncells, a + chunk);
  uint32_t s = 0;
  for (int64_t c = a; c < b; ++c) s += count[c];
  sums[threadIdx.x] = s;
  __syncthreads();
  for (int w = 1; w < blockDim.x; w <<= 1) {
    uint32_t v = threadIdx.x >= w ? sums[threadIdx.x - w] : 0;
    __syncthreads();
    sums[threadIdx.x] += v;
    __syncthreads();
  }
  uint32_t run = sums[threadIdx.x] - s;
  for (int64_t c = a; c < b; ++c) {
    start[c] = run;
    run += count[c];
  }
  if (threadIdx.x == blockDim.x - 1) start[ncells] = sums[threadIdx.x];
}

__global__ void k_iota(int64_t n, uint32_t* v) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    v[i] = uint32_t(i);
}

// Samples in cell order, each cell in sample-index order (`order` is the
// stable sort of the indices by cell), so the layout, and the leave-one-out
// walk that follows it, are the same on every run.
__global__ void k_gather(int64_t n, const double* x, const double* y, const double* z, const double* px,
                         const double* py, const double* pz, const uint32_t* order, double* spx, double* spy,
                         double* spz, double* swx, double* swy, double* swz, uint32_t* sidx) {
  for (int64_t pos = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; pos < n;
       pos += int64_t(gridDim.x) * blockDim.x) {
    const uint32_t i = order[pos];
    spx[pos] = px[i], spy[pos] = py[i], spz[pos] = pz[i];
    swx[pos] = x[i], swy[pos] = y[i], swz[pos] = z[i];
    sidx[pos] = i;
  }
}

int cell_bits(int64_t ncells) {
  int b = 1;
  while (b < 32 && (int64_t(1) << b) < ncells) ++b;
  return b;
}

// twin[i] = 1 when another sample lies within 1e-6 m of sample i, by the
// test of crates/estimation/src/coincident.rs:13-15 (exact order). Pairs
// that close are in the same or adjacent cells (`reach` covers the frame's
// stretch); a system needs the coincident guard only if it holds a twin.
__global__ void k_twins(int64_t n, GridDev g, int reach, const double* x, const double* y, const double* z,
                        uint8_t* twin) {
  const double eps2 = kEps * kEps;
  for (int64_t s = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; s < n; s += int64_t(gridDim.x) * blockDim.x) {
    int c[3] = {cell_axis(g.px[s], g.lo[0], g.h, g.dims[0]), cell_axis(g.py[s], g.lo[1], g.h, g.dims[1]),
                cell_axis(g.pz[s], g.lo[2], g.h, g.dims[2])};
    uint32_t me = g.idx[s];
    double w[3] = {g.wx[s], g.wy[s], g.wz[s]};
    bool found = false;
    for (int dz = -reach; dz <= reach && !found; ++dz)
      for (int dy = -reach; dy <= reach && !found; ++dy) {
        int cy = c[1] + dy, cz = c[2] + dz;
        if (cy < 0 || cy >= g.dims[1] || cz < 0 || cz >= g.dims[2]) continue;
        int x0 = max(c[0] - reach, 0), x1 = min(c[0] + reach, g.dims[0] - 1);
        int64_t row = int64_t(g.dims[0]) * (cy + int64_t(g.dims[1]) * cz);
        for (uint32_t e = g.start[row + x0]; e < g.start[row + x1 + 1]; ++e) {
          if (g.idx[e] == me) continue;
          if (d2_exact(w[0], w[1], w[2], g.wx[e], g.wy[e], g.wz[e]) <= eps2) { found = true; break; }
        }
      }
    twin[me] = found ? 1 : 0;
  }
}

// Centroids of block-model cells (crates/core/src/block_model.rs:76-86):
// origin + block_frame^T * ((ijk + 0.5) * size), exact order. With
// `perm_tiles` the work items are tiles of tw[0] x tw[1] x tw[2] = 32 cells
// (one per search lane) and perm_tiles[k] is the cell of work item k, or -1.
__global__ void k_centroids(btk_geometry geo, Frame9 ft, int tx0, int ty0, int tz0, int64_t first, int64_t m,
                            double* tx, double* ty, double* tz, int64_t* perm_tiles) {
  double F[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) F[k] = ft.m[k];
  const int64_t nx = geo.count[0], ny = geo.count[1], nz = geo.count[2];
  const int64_t tx_n = (nx + tx0 - 1) / tx0, ty_n = (ny + ty0 - 1) / ty0;
  for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < m; k += int64_t(gridDim.x) * blockDim.x) {
    int64_t i, j, l, cell;
    if (perm_tiles) {
      int64_t tile = k >> 5, lane = k & 31;
      int64_t a = tile % tx_n, b = tile / tx_n % ty_n, c = tile / (tx_n * ty_n);
      i = tx0 * a + lane % tx0, j = ty0 * b + lane / tx0 % ty0, l = tz0 * c + lane / (tx0 * ty0);
      if (i >= nx || j >= ny || l >= nz) {
        perm_tiles[k] = -1;
        continue;
      }
      cell = i + nx * (j + ny * l);
      perm_tiles[k] = cell;
    } else {
      cell = first + k;
      i = cell % nx, j = cell / nx % ny, l = cell / (nx * ny);
    }
    double local[3] = {xmul(xadd(double(i), 0.5), geo.size[0]), xmul(xadd(double(j), 0.5), geo.size[1]),
                       xmul(xadd(double(l), 0.5), geo.size[2])};
    double w[3];
    mulv_exact(F, local, w);
    int64_t out = perm_tiles ? cell : k;
    tx[out] = xadd(geo.origin[0], w[0]);
    ty[out] = xadd(geo.origin[1], w[1]);
    tz[out] = xadd(geo.origin[2], w[2]);
  }
}

int grid_blocks(const Launch& L, int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  int64_t cap = int64_t(L.sm_count) * 8;
  return int(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

cudaError_t launch_project(const Launch& L, int64_t n, const double* x, const double* y, const double* z,
                           const double* frame, const double* origin, double* px, double* py, double* pz) {
  k_project<<<grid_blocks(L, n, 256), 256, 0, L.stream>>>(n, x, y, z, frame, origin, px, py, pz);
  ++*L.counter;
  return cudaGetLastError();
}

cudaError_t launch_bounds(const Launch& L, int64_t n, const double* px, const double* py, const double* pz,
                          double* partial, double* out6) {
  int nb = grid_blocks(L, n, 256);
  if (nb > 1024) nb = 1024;
  k_bounds_partial<<<nb, 256, 0, L.stream>>>(n, px, py, pz, partial);
  k_bounds_final<<<1, 32, 0, L.stream>>>(nb, partial, out6);
  *L.counter += 2;
  return cudaGetLastError();
}

size_t grid_sort_temp_bytes(int64_t n, int64_t ncells) {
  size_t bytes = 0;
  cub::DoubleBuffer<uint32_t> k(nullptr, nullptr), v(nullptr, nullptr);
  if (cub::DeviceRadixSort::SortPairs(nullptr, bytes, k, v, int(n), 0, cell_bits(ncells)) != cudaSuccess) return 0;
  return bytes;
}

cudaError_t launch_grid_build(const Launch& L, int64_t n, const double* x, const double* y, const double* z,
                              const double* px, const double* py, const double* pz, GridDev g, uint32_t* count,
                              uint32_t* start, uint32_t* cell_of, double* spx, double* spy, double* spz,
                              double* swx, double* swy, double* swz, uint32_t* sidx, uint32_t* sort_keys,
                              uint32_t* sort_vals, void* temp, size_t temp_bytes) {
  cudaError_t e = cudaMemsetAsync(count, 0, sizeof(uint32_t) * size_t(g.ncells), L.stream);
  if (e != cudaSuccess) return e;
  int nb = grid_blocks(L, n, 256);
  k_cell_count<<<nb, 256, 0, L.stream>>>(n, px, py, pz, g, count, cell_of);
  k_scan<<<1, 1024, 0, L.stream>>>(g.ncells, count, start);
  k_iota<<<nb, 256, 0, L.stream>>>(n, sort_vals);
  e = cudaMemcpyAsync(sort_keys, cell_of, sizeof(uint32_t) * size_t(n), cudaMemcpyDeviceToDevice, L.stream);
  if (e != cudaSuccess) return e;
  cub::DoubleBuffer<uint32_t> k(sort_keys, sort_keys + n), v(sort_vals, sort_vals + n);
  e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, k, v, int(n), 0, cell_bits(g.ncells), L.stream);
  if (e != cudaSuccess) return e;
  k_gather<<<nb, 256, 0, L.stream>>>(n, x, y, z, px, py, pz, v.Current(), spx, spy, spz, swx, swy, swz, sidx);
  *L.counter += 5;
  return cudaGetLastError();
}

cudaError_t launch_twins(const Launch& L, int64_t n, GridDev g, int reach, const double* x, const double* y,
                         const double* z, uint8_t* twin) {
  k_twins<<<grid_blocks(L, n, 128), 128, 0, L.stream>>>(n, g, reach, x, y, z, twin);
  ++*L.counter;
  return cudaGetLastError();
}

cudaError_t launch_centroids(const Launch& L, btk_geometry g, Frame9 frame_t, int64_t first, int64_t m,
                             double* tx, double* ty, double* tz, int64_t* perm_tiles) {
  const int* t = L.tuning.tile;
  k_centroids<<<grid_blocks(L, m, 256), 256, 0, L.stream>>>(g, frame_t, t[0], t[1], t[2], first, m, tx, ty, tz,
                                                            perm_tiles);
  ++*L.counter;
  return cudaGetLastError();
}

}  // namespace btk
