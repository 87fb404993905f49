// Sequential Gaussian simulation on the device: the conditioning loop of
// crates/simulation/src/sgs.rs:586-760 (`sequential`), run as the reference
// runs it, in batches whose stale nodes are redone, so the realization is the
// sequential one.
//
// The context holds the data and then the grid nodes in simulation order as
// one sample set (one grid, built once): node j is sample node0 + j, and its
// search sees the data and the nodes before it that are already simulated
// (SearchDev::sgs). A window of the path is searched and simple-kriged in
// parallel; a node whose reach holds an earlier node not yet simulated is
// stale and waits for the next round of the window. These kernels commit the
// kriged nodes (score = mean + sqrt(variance) z, or z where the search found
// too few samples) into the sample values, and list the window's nodes still
// to do, in path order.
#include <cub/block/block_scan.cuh>

#include "btk_device.cuh"

namespace btk {
namespace {

constexpr int kCompactThreads = 1024;

// Nodes first .. last - 1 not yet simulated, in order, by one block.
__global__ void __launch_bounds__(kCompactThreads)
    k_sgs_pending(int64_t first, int64_t last, uint32_t node0, const uint8_t* __restrict__ done,
                  int64_t* __restrict__ list, int64_t* __restrict__ len) {
  using Scan = cub::BlockScan<int, kCompactThreads>;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ int64_t base;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  for (int64_t c = first; c < last; c += kCompactThreads) {
    const int64_t j = c + threadIdx.x;
    const int flag = j < last && !done[node0 + j] ? 1 : 0;
    int pos = 0, total = 0;
    Scan(tmp).ExclusiveSum(flag, pos, total);
    if (flag) list[base + pos] = j;
    __syncthreads();
    if (threadIdx.x == 0) base += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) *len = base;
}

// sgs.rs:702-745: a kriged node draws from its simple-kriging mean and
// variance, a node whose search failed from the standard normal (the
// marginal of the scores); either joins the conditioning set.
__global__ void k_sgs_commit(int64_t nwork, const int64_t* __restrict__ list, const double* __restrict__ mean,
                             const double* __restrict__ var, const int8_t* __restrict__ status,
                             const double* __restrict__ z, uint32_t node0, double* __restrict__ sv,
                             uint8_t* __restrict__ done, double* __restrict__ score, int8_t* __restrict__ how,
                             int64_t* __restrict__ failed) {
  for (int64_t w = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; w < nwork; w += int64_t(gridDim.x) * blockDim.x) {
    const int64_t j = list[w];
    const int st = status[j] & 0x0F;
    if (st == kStStale) continue;
    double s;
    int8_t h;
    if (st == BTK_ST_OK) {
      s = __dadd_rn(mean[j], __dmul_rn(sqrt(var[j]), z[j]));
      h = 1;
    } else if (st == BTK_ST_SEARCH_FAILED) {
      s = z[j];
      h = 2;
    } else {  // the reference's krige error ends the simulation
      atomicMin(reinterpret_cast<unsigned long long*>(failed), static_cast<unsigned long long>(j));
      continue;
    }
    sv[node0 + j] = s;
    score[j] = s;
    how[j] = h;
    __threadfence();
    done[node0 + j] = 1;
  }
}

}  // namespace

cudaError_t launch_sgs_pending(const Launch& L, int64_t first, int64_t last, uint32_t node0, const uint8_t* done,
                               int64_t* list, int64_t* len) {
  k_sgs_pending<<<1, kCompactThreads, 0, L.stream>>>(first, last, node0, done, list, len);
  ++*L.counter;
  return cudaGetLastError();
}

cudaError_t launch_sgs_commit(const Launch& L, int64_t nwork, const int64_t* list, const double* mean,
                              const double* var, const int8_t* status, const double* z, uint32_t node0, double* sv,
                              uint8_t* done, double* score, int8_t* how, int64_t* failed) {
  if (nwork <= 0) return cudaSuccess;
  int64_t blocks = (nwork + 255) / 256;
  if (blocks > int64_t(L.sm_count) * 8) blocks = int64_t(L.sm_count) * 8;
  k_sgs_commit<<<int(blocks), 256, 0, L.stream>>>(nwork, list, mean, var, status, z, node0, sv, done, score, how,
                                                  failed);
  ++*L.counter;
  return cudaGetLastError();
}

}  // namespace btk
