// Kriging that allocates nothing, for callers that cannot call cudaMalloc:
// a host that owns every device allocation itself (an arena or memory-pool
// allocator it must account for, a plugin running inside another program's
// CUDA context, a process whose device memory budget is fixed up front).
// The caller passes its own device buffers for every input and output; the
// one piece of scratch the solve needs, the list of systems the FP32
// factorisation leaves to FP64 and its count, lives in the static device
// array below instead of a cudaMalloc'd buffer.
#include <cstdio>
#include <string>

#include "btk_internal.h"

namespace {

using btk::Launch;
using btk::SolveDev;
using btk::VgDev;

// g_redo[0] is the count, g_redo[1..] the target indices to re-solve in FP64.
// 8 * (BTK_NOALLOC_MAX_SYSTEMS + 1) bytes (2 MiB) on every GPU that loads the
// library, held until the process exits; every call shares it.
static __device__ __align__(256) int64_t g_redo[BTK_NOALLOC_MAX_SYSTEMS + 1];

// Device address of g_redo in the current context. In host code g_redo names
// a host-side stand-in, not device memory, so the kernels only ever receive
// the address cudaGetSymbolAddress gives. The address belongs to one CUDA
// context (one load of this module), so it is looked up on every call rather
// than cached: a call from another context on the same device, or after a
// cudaDeviceReset, gets that context's own array. The lookup is cheap once
// the module is loaded; the first one in a context loads it, which is why the
// first call there should come before any stream capture.
cudaError_t scratch_here(int64_t** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_redo);
  if (e == cudaSuccess) *out = static_cast<int64_t*>(p);
  return e;
}

int say(char* err, size_t errlen, int code, const std::string& msg) {
  if (err && errlen) std::snprintf(err, errlen, "%s", msg.c_str());
  return code;
}

}  // namespace

extern "C" int btk_solve_noalloc(int device, const btk_variogram* vg, int32_t kind, double kparam,
                                 const double* d_x, const double* d_y, const double* d_z, const double* d_values,
                                 const double* d_err, int64_t n_samples, int64_t m, const double* d_tx,
                                 const double* d_ty, const double* d_tz, const uint32_t* d_nbr, int32_t max_samples,
                                 const int32_t* d_count, const int8_t* d_status, const btk_outputs* d_out,
                                 void* stream, char* err, size_t errlen) {
  if (m < 0 || m > BTK_NOALLOC_MAX_SYSTEMS)
    return say(err, errlen, BTK_EINVAL,
               "btk_solve_noalloc takes at most " + std::to_string(BTK_NOALLOC_MAX_SYSTEMS) +
                   " systems per call, got " + std::to_string(m) + "; split the targets into several calls");
  if (max_samples < 1 || max_samples > 32)
    return say(err, errlen, BTK_EUNSUPPORTED, "btk_solve_noalloc takes at most 32 samples per system");
  if (kind < BTK_ORDINARY || kind > BTK_INDICATOR) return say(err, errlen, BTK_EINVAL, "unknown kriging kind");
  if (!d_x || !d_y || !d_z || !d_values || !d_nbr || !d_count || !d_status || !d_out || !d_out->value ||
      (m > 0 && (!d_tx || !d_ty || !d_tz)))
    return say(err, errlen, BTK_EINVAL, "every input and the value output must be device pointers");
  if (n_samples < 1 || n_samples > int64_t(UINT32_MAX))
    return say(err, errlen, BTK_EINVAL,
               "n_samples must be the number of samples behind d_x .. d_values (1 .. 2^32 - 1)");
  if (device < 0) return say(err, errlen, BTK_EINVAL, "device index out of range");
  VgDev vgd{};
  std::string why;
  int rc = btk::prepare_variogram(vg, &vgd, &why);
  if (rc != BTK_OK) return say(err, errlen, rc, why);
  if (!vgd.stationary)
    return say(err, errlen, BTK_EUNSUPPORTED, "btk_solve_noalloc takes stationary variograms (no power structure)");
  if (m == 0) return BTK_OK;

  int before = 0;
  cudaError_t e = cudaGetDevice(&before);
  if (e == cudaSuccess && before != device) e = cudaSetDevice(device);
  int64_t* scratch = nullptr;
  if (e == cudaSuccess) e = scratch_here(&scratch);
  int sm = 0;
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, device);
  int64_t launches = 0;
  Launch L{static_cast<cudaStream_t>(stream), sm, &launches};
  SolveDev a{};
  a.vg = vgd;
  a.kind = kind;
  a.kparam = kparam;
  a.max_samples = max_samples;
  a.sx = d_x, a.sy = d_y, a.sz = d_z, a.sv = d_values, a.se = d_err;
  a.twin = nullptr;  // the pair-testing kernels check each system themselves
  a.tx = d_tx, a.ty = d_ty, a.tz = d_tz;
  a.nbr = d_nbr, a.count = d_count, a.sstatus = d_status;
  a.nsamples = n_samples;  // every index and count is checked against the caller's buffers
  a.m = m;
  a.value = d_out->value, a.variance = d_out->variance, a.lagrange = d_out->lagrange;
  a.n_used = d_out->n_used, a.status = d_out->status;
  // The count starts at zero on every call; the list needs no clearing.
  if (e == cudaSuccess) e = cudaMemsetAsync(scratch, 0, sizeof(int64_t), L.stream);
  if (e == cudaSuccess) e = btk::launch_solve_mixed_pairs(L, a, scratch + 1, scratch);
  if (e == cudaSuccess) {
    SolveDev r = a;
    r.list = scratch + 1, r.list_len = scratch;
    e = btk::launch_solve_redo_pairs(L, r);
  }
  if (before != device) cudaSetDevice(before);
  if (e != cudaSuccess) return say(err, errlen, BTK_ECUDA, std::string("btk_solve_noalloc: ") + cudaGetErrorString(e));
  return BTK_OK;
}
