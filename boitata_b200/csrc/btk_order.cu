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

__global__ void k_order_keys(int64_t m, const double* __restrict__ x, const double* __restrict__ y,
                         const double* __restrict__ z, Frame9 w, const double* __restrict__ b6,
                         uint64_t* __restrict__ key, int64_t* __restrict__ idx) {
  const double ext = fmax(fmax((b6[3] - b6[0]) * w.m[0], (b6[4] - b6[1]) * w.m[1]), (b6[5] - b6[2]) * w.m[2]);
  const double s = ext > 0.0 ? 2097151.0 / ext : 0.0;
  const double sx = s * w.m[0], sy = s * w.m[1], sz = s * w.m[2];
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x) {
    // fmax maps NaN to the low edge; clamping keeps every key in 63 bits
    const uint32_t qx = uint32_t(fmin(fmax((x[i] - b6[0]) * sx, 0.0), 2097151.0));
    const uint32_t qy = uint32_t(fmin(fmax((y[i] - b6[1]) * sy, 0.0), 2097151.0));
    const uint32_t qz = uint32_t(fmin(fmax((z[i] - b6[2]) * sz, 0.0), 2097151.0));
    // Axes to the transposed Hilbert index (J. Skilling, "Programming the
    // Hilbert curve", AIP Conf. Proc. 707, 2004): undo the excess work of
    // each level from the top, Gray-encode, then interleave with axis 0 most
    // significant in each group of three bits.
    uint32_t X[3] = {qx, qy, qz};
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
    key[i] = spread3(X[2]) | (spread3(X[1]) << 1) | (spread3(X[0]) << 2);
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
                                const double w[3], double* partial, double* b6, uint64_t* keys, int64_t* vals,
                                void* temp, size_t temp_bytes, const int64_t** perm) {
  Frame9 wk{};
  for (int d = 0; d < 3; ++d) wk.m[d] = w[d] > 0.0 ? w[d] : 1.0;
  cudaError_t e = launch_bounds(L, m, x, y, z, partial, b6);
  if (e != cudaSuccess) return e;
  int64_t b = (m + 255) / 256;
  if (b > int64_t(L.sm_count) * 8) b = int64_t(L.sm_count) * 8;
  if (b < 1) b = 1;
  k_order_keys<<<int(b), 256, 0, L.stream>>>(m, x, y, z, wk, b6, keys, vals);
  ++*L.counter;
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
