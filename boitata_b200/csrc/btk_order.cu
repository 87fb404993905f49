// Spatial order of caller-supplied targets. The reference krigs targets in
// the caller's order on CPU threads (crates/estimation/src/batch.rs:15-38);
// here a search warp serves 32 consecutive work slots and a solve tile 16, so
// targets that arrive in row-major order (a block model flattened x fastest)
// would put 80 m strips into one warp. A Hilbert key (21 bits per axis) over
// the targets' bounding box, each axis weighted by the caller's w[d] with one
// scale for all three, is sorted on the device with CUB's radix sort, and the
// sorted indices are the work-slot permutation. Consecutive Hilbert keys are
// neighbouring cells, so a run of 32 targets is one compact region; a Morton
// key's runs can straddle far-apart octants (on the 3.2M-block model the
// Hilbert order searched and solved 2.3 ms faster). Results are written by
// target index, so the order is invisible to the caller.
//
// Targets that form an axis-aligned lattice (a block model's centroids passed
// as coordinates, in any order) take the order the block-model path gives
// them instead: tiles of the tuned 32-cell shape, the tiles in Hilbert order,
// the cells of a tile x fastest. A Hilbert run of 32 lattice points is a
// 4 x 4 x 2 slab of varying orientation, while the tuned tile has the shape
// the search ellipsoid favours (on the 3.2M-block model the call took 32.8
// instead of 34.9 ms). The lattice is found on the device: per axis the
// smallest positive step between consecutive targets, then every coordinate
// within 1e-6 steps of a whole number of steps from the low edge.
#include <cub/device/device_radix_sort.cuh>

#include "btk_device.cuh"

namespace btk {
namespace {

// The low 21 bits of v spread to every third bit (bit i -> bit 3i).
__device__ __forceinline__ uint64_t spread3(uint32_t v) {
  uint64_t x = v & 0x1fffffu;
  x = (x | x << 32) & 0x1f00000000ffffull;
  x = (x | x << 16) & 0x1f0000ff0000ffull;
  x = (x | x << 8) & 0x100f00f00f00f00full;
  x = (x | x << 4) & 0x10c30c30c30c30c3ull;
  x = (x | x << 2) & 0x1249249249249249ull;
  return x;
}

constexpr unsigned kFull = 0xffffffffu;
constexpr double kLatticeMax = 524288.0;  // steps per axis: tile coordinates keep 19 bits

// Transposed Hilbert index of (X0, X1, X2), 21 bits each (J. Skilling,
// "Programming the Hilbert curve", AIP Conf. Proc. 707, 2004): undo the
// excess work of each level from the top, Gray-encode, then interleave with
// axis 0 most significant in each group of three bits. Points whose
// coordinates are all below 2^b take the first 2^(3b) indices.
__device__ __forceinline__ uint64_t hilbert3(uint32_t X0, uint32_t X1, uint32_t X2) {
  uint32_t X[3] = {X0, X1, X2};
  for (uint32_t Q = 1u << 20; Q > 1; Q >>= 1) {
    const uint32_t P = Q - 1;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (X[d] & Q) {
        X[0] ^= P;
      } else {
        const uint32_t t = (X[0] ^ X[d]) & P;
        X[0] ^= t, X[d] ^= t;
      }
    }
  }
  X[1] ^= X[0], X[2] ^= X[1];
  uint32_t t = 0;
  for (uint32_t Q = 1u << 20; Q > 1; Q >>= 1)
    if (X[2] & Q) t ^= Q - 1;
  X[0] ^= t, X[1] ^= t, X[2] ^= t;
  return spread3(X[2]) | (spread3(X[1]) << 1) | (spread3(X[0]) << 2);
}

// lat[a] <- the bits of the smallest positive |c[i+1] - c[i]| along axis a
// (positive doubles order as their bits; lat[a] starts all ones: none yet).
__global__ void k_lattice_steps(int64_t m, const double* __restrict__ x, const double* __restrict__ y,
                                const double* __restrict__ z, unsigned long long* __restrict__ lat) {
  unsigned long long best[3] = {~0ull, ~0ull, ~0ull};
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i + 1 < m;
       i += int64_t(gridDim.x) * blockDim.x) {
    const double d[3] = {fabs(x[i + 1] - x[i]), fabs(y[i + 1] - y[i]), fabs(z[i + 1] - z[i])};
#pragma unroll
    for (int a = 0; a < 3; ++a)
      if (d[a] > 0.0 && d[a] <= 1.7e308)
        best[a] = min(best[a], static_cast<unsigned long long>(__double_as_longlong(d[a])));
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best[a] = min(best[a], __shfl_xor_sync(kFull, best[a], o));
    if ((threadIdx.x & 31) == 0 && best[a] != ~0ull) atomicMin(lat + a, best[a]);
  }
}

// Step along axis a; 0 when no two consecutive targets differ along it.
__device__ __forceinline__ double lattice_step(const unsigned long long* lat, int a) {
  return lat[a] == ~0ull ? 0.0 : __longlong_as_double(static_cast<long long>(lat[a]));
}

// lat[3] <- 1 when some coordinate is not within 1e-6 steps of a whole number
// of steps from the low edge b6[a], that number is kLatticeMax or more, or it
// differs from the edge along an axis without a step (NaN included).
__global__ void k_lattice_check(int64_t m, const double* __restrict__ x, const double* __restrict__ y,
                                const double* __restrict__ z, const double* __restrict__ b6,
                                unsigned long long* __restrict__ lat) {
  const double s[3] = {lattice_step(lat, 0), lattice_step(lat, 1), lattice_step(lat, 2)};
  bool off = false;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x) {
    const double c[3] = {x[i], y[i], z[i]};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (s[a] == 0.0) {
        off = off || !(c[a] == b6[a]);
      } else {
        const double u = (c[a] - b6[a]) / s[a], r = rint(u);
        off = off || !(fabs(u - r) <= 1e-6 && r < kLatticeMax);
      }
    }
  }
  if (__any_sync(kFull, off) && (threadIdx.x & 31) == 0) atomicOr(lat + 3, 1ull);
}

// Sort keys of targets 0 .. m-1. A lattice (lat[3] clear): the target's tile
// of tile.x x tile.y x tile.z cells in Hilbert order, then its cell in the
// tile, x fastest. Otherwise the Hilbert key of the bounding box, each axis
// weighted by w.
__global__ void k_order_keys(int64_t m, const double* __restrict__ x, const double* __restrict__ y,
                             const double* __restrict__ z, Frame9 w, const double* __restrict__ b6,
                             const unsigned long long* __restrict__ lat, int3 tile, uint64_t* __restrict__ key,
                             int64_t* __restrict__ idx) {
  if (lat[3] == 0) {  // uniform: the lattice order
    const double s[3] = {lattice_step(lat, 0), lattice_step(lat, 1), lattice_step(lat, 2)};
    const uint32_t tx = uint32_t(tile.x), ty = uint32_t(tile.y), tz = uint32_t(tile.z);
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x) {
      const double c[3] = {x[i], y[i], z[i]};
      uint32_t g[3];  // below kLatticeMax: checked
#pragma unroll
      for (int a = 0; a < 3; ++a) g[a] = s[a] == 0.0 ? 0u : uint32_t(rint((c[a] - b6[a]) / s[a]));
      const uint64_t cell = g[0] % tx + tx * (g[1] % ty + ty * (g[2] % tz));  // < 32
      key[i] = (hilbert3(g[0] / tx, g[1] / ty, g[2] / tz) << 5) | cell;
      idx[i] = i;
    }
    return;
  }
  const double ext = fmax(fmax((b6[3] - b6[0]) * w.m[0], (b6[4] - b6[1]) * w.m[1]), (b6[5] - b6[2]) * w.m[2]);
  const double sc = ext > 0.0 ? 2097151.0 / ext : 0.0;
  const double sx = sc * w.m[0], sy = sc * w.m[1], sz = sc * w.m[2];
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x) {
    // fmax maps NaN to the low edge; clamping keeps every key in 63 bits
    const uint32_t qx = uint32_t(fmin(fmax((x[i] - b6[0]) * sx, 0.0), 2097151.0));
    const uint32_t qy = uint32_t(fmin(fmax((y[i] - b6[1]) * sy, 0.0), 2097151.0));
    const uint32_t qz = uint32_t(fmin(fmax((z[i] - b6[2]) * sz, 0.0), 2097151.0));
    key[i] = hilbert3(qx, qy, qz);
    idx[i] = i;
  }
}

}  // namespace

size_t morton_temp_bytes(int64_t m) {
  size_t bytes = 0;
  cub::DoubleBuffer<uint64_t> k(nullptr, nullptr);
  cub::DoubleBuffer<int64_t> v(nullptr, nullptr);
  if (cub::DeviceRadixSort::SortPairs(nullptr, bytes, k, v, int(m), 0, 63) != cudaSuccess) return 0;
  return bytes;
}

cudaError_t launch_morton_order(const Launch& L, int64_t m, const double* x, const double* y, const double* z,
                                const double w[3], double* partial, double* b6, unsigned long long* lat,
                                uint64_t* keys, int64_t* vals, void* temp, size_t temp_bytes, const int64_t** perm) {
  Frame9 wk{};
  for (int d = 0; d < 3; ++d) wk.m[d] = w[d] > 0.0 ? w[d] : 1.0;
  const int* tw = L.tuning.tile;
  if (tw[0] < 1 || tw[1] < 1 || tw[2] < 1 || tw[0] * tw[1] * tw[2] != 32) return cudaErrorInvalidValue;
  cudaError_t e = launch_bounds(L, m, x, y, z, partial, b6);
  if (e != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(lat, 0xFF, 3 * sizeof(unsigned long long), L.stream)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(lat + 3, 0, sizeof(unsigned long long), L.stream)) != cudaSuccess) return e;
  int64_t b = (m + 255) / 256;
  if (b > int64_t(L.sm_count) * 8) b = int64_t(L.sm_count) * 8;
  if (b < 1) b = 1;
  k_lattice_steps<<<int(b), 256, 0, L.stream>>>(m, x, y, z, lat);
  k_lattice_check<<<int(b), 256, 0, L.stream>>>(m, x, y, z, b6, lat);
  k_order_keys<<<int(b), 256, 0, L.stream>>>(m, x, y, z, wk, b6, lat, make_int3(tw[0], tw[1], tw[2]), keys, vals);
  *L.counter += 3;
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  cub::DoubleBuffer<uint64_t> k(keys, keys + m);
  cub::DoubleBuffer<int64_t> v(vals, vals + m);
  e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, k, v, int(m), 0, 63, L.stream);
  if (e != cudaSuccess) return e;
  *L.counter += 4;  // the sort's passes (histogram and scatter kernels)
  *perm = v.Current();
  return cudaSuccess;
}

}  // namespace btk
