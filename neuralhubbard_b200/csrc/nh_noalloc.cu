// nh_slogpf_noalloc: the batched log-Pfaffian with FP64 refinement, using a fixed static device
// buffer for its scratch instead of a caller-provided workspace.
//
// Some callers cannot allocate device memory: a plugin that is handed only its input and output
// buffers by a host runtime that owns all device memory (and offers no workspace), or code on a
// path where cudaMalloc is not acceptable because it can synchronise the device.  nh_slogpf needs
// scratch for the list of matrices it re-factorises in FP64; this variant keeps that list in
// g_slogpf_scratch below, a file-scope __device__ array of kNoAllocMaxBatch + 64 int32 words
// (256.25 KiB) that every GPU loading the library holds until the process exits.
//
// The first call on a device looks up the array's device address with cudaGetSymbolAddress (the
// array's name in host code is only a host-side stand-in) and caches it; make that first call
// before any stream capture.  All calls share the array and overwrite it (the count word is
// written by each call before it is read), so calls whose kernels overlap on the GPU, e.g. on
// two streams at once, race and must be serialised by the caller.
#include <mutex>

#include "nh_common.cuh"

namespace nh {
namespace {

constexpr int kNoAllocMaxBatch = NH_SLOGPF_NOALLOC_MAX_BATCH;
constexpr int kMaxDevices = 64;

// [0, kNoAllocMaxBatch): list of matrices to re-factorise; [kNoAllocMaxBatch]: their count.
__device__ __align__(256) int32_t g_slogpf_scratch[kNoAllocMaxBatch + 64];

std::mutex g_noalloc_mu;
int32_t* g_noalloc_ptr[kMaxDevices] = {};

// Device address of g_slogpf_scratch on the current device (looked up once per device).
int scratch_address(int32_t** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return check_cuda(e, "slogpf_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices)
    return fail(NH_ERR_UNSUPPORTED, "slogpf_noalloc: device ordinal %d >= %d", dev, kMaxDevices);
  std::lock_guard<std::mutex> g(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_slogpf_scratch);
    if (e != cudaSuccess) return check_cuda(e, "slogpf_noalloc: cudaGetSymbolAddress");
    g_noalloc_ptr[dev] = static_cast<int32_t*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return NH_OK;
}

}  // namespace
}  // namespace nh

using namespace nh;

extern "C" int nh_slogpf_noalloc(const float* F, int n, int batch, double cond_tau, float* sign,
                                 double* logabs, int32_t* flags, void* stream) {
  if (!F || !sign || !logabs || batch < 0)
    return fail(NH_ERR_INVALID, "slogpf_noalloc: bad arguments");
  if (batch > kNoAllocMaxBatch)
    return fail(NH_ERR_UNSUPPORTED, "slogpf_noalloc: batch %d exceeds the static scratch limit %d",
                batch, kNoAllocMaxBatch);
  if (n <= 0 || n % 2 || n > kNumThreads)
    return fail(NH_ERR_UNSUPPORTED,
                "slogpf_noalloc: n=%d must be even and <= %d (beyond, nh_slogpf with a workspace)",
                n, kNumThreads);
  const bool refine = cond_tau > 0.0;
  if (refine && !flags) return fail(NH_ERR_INVALID, "slogpf_noalloc: refinement needs flags");
  if (batch == 0) return NH_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int32_t* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc) return rc;
  rc = launch_pfaffian_from_F(F, n, batch, nullptr, nullptr, false, cond_tau, 0, sign, logabs,
                              flags, nullptr, st);
  if (rc || !refine || !pfaffian64_fits(n)) return rc;
  int32_t* list = scratch;
  int32_t* count = scratch + kNoAllocMaxBatch;  // written by the listing kernel on every call
  if ((rc = launch_flagged(flags, batch, nullptr, 1, list, count, st))) return rc;
  return launch_pfaffian_from_F(F, n, batch, list, count, true, 0.0,
                                NH_FLAG_GROWTH | NH_FLAG_REFINED, sign, logabs, flags, nullptr, st);
}
