// Shared device/host helpers for the sm_100a dense-solve library.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "lm_b200.h"

namespace lm {

// Device-side status words live in lm_ctx::d_status:
//   [0] device error code (0 = none; LM_DEVERR_* below)
//   [1] LAPACK-style info of the last factorisation (0 = ok, k+1 = first bad pivot)
//   [2] scratch counter (ticket dispenser for persistent kernels)
enum : int {
  LM_DEVERR_NONE = 0,
  LM_DEVERR_TIMEOUT = 1,   // a bounded wait gave up
  LM_DEVERR_BOUNDS = 2,    // a self-check found an out-of-range index
};

// Every spin-wait in this library gives up after this many polls, records
// LM_DEVERR_TIMEOUT and returns.  With the hardware's own suspend inside
// mbarrier.try_wait this bounds a wait to well under a few seconds.
constexpr uint32_t kSpinLimit = 1u << 24;

struct Ctx;  // defined in api.cu

#define LM_CUDA_TRY(expr)                                                        \
  do {                                                                           \
    cudaError_t e__ = (expr);                                                    \
    if (e__ != cudaSuccess) {                                                    \
      lm::set_last_error(std::string(#expr) + ": " + cudaGetErrorString(e__));   \
      return LM_ERR_CUDA;                                                        \
    }                                                                            \
  } while (0)

#define LM_TRY(expr)            \
  do {                          \
    int s__ = (expr);           \
    if (s__ != LM_OK) return s__; \
  } while (0)

void set_last_error(const std::string& msg);

__host__ __device__ inline int cdiv(int a, int b) { return (a + b - 1) / b; }
__host__ __device__ inline long long cdivll(long long a, long long b) { return (a + b - 1) / b; }

// ---------------------------------------------------------------------------
// PTX wrappers: shared-memory addresses, mbarriers, TMA, cluster barriers.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on an mbarrier phase.  Returns false (and records a timeout in
// the device status) if the phase never completes.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* status) {
  for (uint32_t it = 0; it < kSpinLimit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  atomicCAS(status, 0, LM_DEVERR_TIMEOUT);
  return false;
}

// Non-suspending variant for latency-critical waits: polls with
// mbarrier.test_wait (never parks the warp), still bounded by kSpinLimit.
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_spin(uint64_t* bar, uint32_t parity, int* status) {
  for (uint32_t it = 0; it < 4 * kSpinLimit; ++it)
    if (mbar_test(bar, parity)) return true;
  atomicCAS(status, 0, LM_DEVERR_TIMEOUT);
  return false;
}

// 2D tiled TMA load (no multicast) into this CTA's shared memory, completing
// on an mbarrier of this CTA.
__device__ __forceinline__ void tma_load_2d(void* smem_dst, const CUtensorMap* tmap, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap* tmap) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tmap)) : "memory");
}

// Cluster-wide barrier (all threads of all CTAs in the cluster).
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::
                   : "memory");
}

__device__ __forceinline__ uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

__device__ __forceinline__ uint32_t cluster_nctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}

// Map a shared-memory address of this CTA to the same offset in CTA `rank`
// of the cluster (distributed shared memory), as a shared::cluster address.
__device__ __forceinline__ uint32_t dsmem_map(const void* p, uint32_t rank) {
  uint32_t out;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(smem_u32(p)), "r"(rank));
  return out;
}

__device__ __forceinline__ double dsmem_ld_f64(uint32_t addr) {
  double v;
  asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(addr) : "memory");
  return v;
}
__device__ __forceinline__ float dsmem_ld_f32(uint32_t addr) {
  float v;
  asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(addr) : "memory");
  return v;
}
__device__ __forceinline__ int dsmem_ld_s32(uint32_t addr) {
  int v;
  asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
  return v;
}
template <typename T>
__device__ __forceinline__ T dsmem_ld(uint32_t addr);
template <>
__device__ __forceinline__ double dsmem_ld<double>(uint32_t a) { return dsmem_ld_f64(a); }
template <>
__device__ __forceinline__ float dsmem_ld<float>(uint32_t a) { return dsmem_ld_f32(a); }

// Asynchronous 16-byte store into (possibly another CTA's) shared memory that
// completes tx bytes on the destination CTA's mbarrier (both addresses are
// shared::cluster addresses from dsmem_map).
__device__ __forceinline__ void st_async_16(uint32_t dst, uint32_t remote_bar, uint32_t a, uint32_t b, uint32_t c,
                                            uint32_t d) {
  asm volatile(
      "st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, [%5];" ::"r"(dst),
      "r"(a), "r"(b), "r"(c), "r"(d), "r"(remote_bar)
      : "memory");
}

// FP64 tensor-core MMA, m16n8k4 (row.col): D = A*B + D.
__device__ __forceinline__ void dmma_16x8x4(double (&d)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

}  // namespace lm
