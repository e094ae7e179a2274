// lm_dpotrf_noalloc: the Cholesky factorisation with all of its device
// scratch in one file-scope array of this library, for callers that cannot
// allocate device memory at call time — code running where cudaMalloc is
// unavailable or forbidden (inside a memory-pool-managed runtime that owns
// every allocation, a real-time loop with a no-allocation rule, a plugin
// host that hands out only pre-registered buffers).
//
// Scratch: the 128 x 128 inverse of the current diagonal block plus a copy of
// the panel below it, (128 + kNoAllocMaxN) x 128 doubles, and two status words
// — about 4.3 MB per device.  CUDA loads a library's device code lazily by
// default, so the array is reserved on a device when the first call there
// looks up its address (a call with n = 0 does only that); from then on the
// device holds it until the process exits.
#include <mutex>

#include "common.cuh"
#include "internal.h"

namespace {

constexpr int kNoAllocMaxN = 4096;  // largest n this entry point accepts
constexpr int kPanel = 128;
constexpr size_t kScratchDoubles = (size_t)(kPanel + kNoAllocMaxN) * kPanel;

// [0, 2): status words (error, info); the scratch starts 256 bytes in.
static __device__ __align__(256) double g_noalloc_scratch[32 + kScratchDoubles];

std::mutex g_setup_mu;
double* g_scratch_dev[lm::kMaxDevices] = {};  // device address of the array, per device
int g_num_sms[lm::kMaxDevices] = {};

// Once per device, with that device current: the array's device address.
// (In host code `g_noalloc_scratch` names a host-side stand-in, not device
// memory, so it must never be passed to a kernel directly.)
int setup(int dev) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (g_scratch_dev[dev]) return LM_OK;
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    lm::set_last_error(std::string("cudaGetSymbolAddress(g_noalloc_scratch) failed: ") + cudaGetErrorString(e));
    return LM_ERR_CUDA;
  }
  int sms = 0;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) {
    lm::set_last_error(std::string("cudaDeviceGetAttribute failed: ") + cudaGetErrorString(e));
    return LM_ERR_CUDA;
  }
  g_num_sms[dev] = sms;
  g_scratch_dev[dev] = static_cast<double*>(p);
  return LM_OK;
}

}  // namespace

extern "C" int lm_dpotrf_noalloc(void* stream, int n, double* A, int lda, int* info) {
  if (n < 0 || (n > 0 && (!A || lda < n))) return LM_ERR_ARG;
  if (n > kNoAllocMaxN) {
    lm::set_last_error("lm_dpotrf_noalloc: n = " + std::to_string(n) + " exceeds its scratch limit of " +
                       std::to_string(kNoAllocMaxN));
    return LM_ERR_ARG;
  }
  if (n > 0 && ((reinterpret_cast<uintptr_t>(A) & 15) || (lda & 1))) {
    lm::set_last_error("lm_dpotrf_noalloc: A must be 16-byte aligned with an even leading dimension");
    return LM_ERR_UNSUPPORTED;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= lm::kMaxDevices) return LM_ERR_CUDA;
  LM_TRY(setup(dev));  // also for n = 0: the warm-up call that reserves the array
  if (n == 0) {
    if (info) *info = 0;
    return LM_OK;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* base = g_scratch_dev[dev];
  int* status = reinterpret_cast<int*>(base);  // error word, info word
  // the status words must start at zero; the scratch is overwritten before use
  LM_CUDA_TRY(cudaMemsetAsync(status, 0, 2 * sizeof(int), st));
  LM_TRY(lm::dpotrf_borrowed(dev, g_num_sms[dev], st, n, A, lda, status, base + 32, kScratchDoubles * sizeof(double)));
  int h[2] = {0, 0};
  LM_CUDA_TRY(cudaMemcpyAsync(h, status, sizeof h, cudaMemcpyDeviceToHost, st));
  LM_CUDA_TRY(cudaStreamSynchronize(st));
  if (h[0] != 0) {
    lm::set_last_error("lm_dpotrf_noalloc: a bounded device-side wait timed out");
    return LM_ERR_TIMEOUT;
  }
  if (info) *info = h[1];
  return h[1];
}
