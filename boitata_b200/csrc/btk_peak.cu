// Diagnostics: a CUDA-core FMA throughput probe (the roofline denominator for
// the solve kernels, which are FP64/FP32 CUDA-core bound, not tensor or HBM
// bound) and per-phase event timing of the last prediction.
#include "btk_internal.h"

namespace btk {
namespace {

// Independent FMA chains per thread; the result is stored so nothing is
// optimised away. 8 chains x `iters` x 2 flops per thread.
template <class T>
__global__ void k_fma(int iters, T a, T b, T* out) {
  T x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = T(threadIdx.x + k);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = x[k] * a + b;
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  if (s == T(-1.2345)) out[0] = s;
}

}  // namespace

double measure_fma_flops(cudaStream_t s, int sm_count, int fp64, int64_t* counter) {
  const int threads = 512, blocks = sm_count * 8, iters = 4096;
  void* out = nullptr;
  if (cudaMalloc(&out, 64) != cudaSuccess) return -1.0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 6; ++rep) {
    cudaEventRecord(e0, s);
    if (fp64)
      k_fma<double><<<blocks, threads, 0, s>>>(iters, 0.999999, 1e-9, static_cast<double*>(out));
    else
      k_fma<float><<<blocks, threads, 0, s>>>(iters, 0.999999f, 1e-9f, static_cast<float*>(out));
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;  // first launch is warm-up
    ++*counter;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (cudaGetLastError() != cudaSuccess) return -1.0;
  const double flops = 2.0 * 8.0 * double(iters) * double(threads) * double(blocks);
  return flops / (double(best) * 1e-3);
}

}  // namespace btk
