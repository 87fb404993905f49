// Block support: the mean covariance C(B,B) of a discretized block
// (crates/variogram/src/composite.rs:120-129, block_mean_cov): the mean over
// all pairs of discretization points of the point covariance with the nugget
// left out at zero lag (composite.rs:108-115); one point is point support,
// C(0) with the nugget. The lags come from the offsets alone, so C(B,B) is the
// same for every block of a model and is computed once per call.
#include "btk_device.cuh"

namespace btk {
namespace {

__global__ void k_support_cbb(VgDev vg, const double* __restrict__ off, int nd, double* cbb) {
  __shared__ double part[256];
  double acc = 0.0;
  const int64_t pairs = int64_t(nd) * nd;
  for (int64_t e = threadIdx.x; e < pairs; e += blockDim.x) {
    const int i = int(e / nd), j = int(e % nd);
    const double h = lag_world(vg, off[3 * i], off[3 * i + 1], off[3 * i + 2], off[3 * j], off[3 * j + 1],
                               off[3 * j + 2]);
    acc += h > 0.0 ? cov64(vg, h) : vg.c0 - vg.nugget;
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *cbb = nd == 1 ? vg.c0 : part[0] / double(pairs);
}

}  // namespace

cudaError_t launch_support_cbb(const Launch& L, const VgDev& vg, const double* off, int nd, double* cbb) {
  k_support_cbb<<<1, 256, 0, L.stream>>>(vg, off, nd, cbb);
  ++*L.counter;
  return cudaGetLastError();
}

}  // namespace btk
