// Low-precision GEMM on the 5th-generation tensor cores (tcgen05), the
// trailing-matrix contraction of the factorisation used by iterative
// refinement:  C = alpha * A * Bt^T + beta * C,  C FP32 row-major, A m x k and
// Bt n x k (both K-major), accumulation in FP32.  Operand modes:
//   kTf32    FP32 storage, one kind::tf32 product;
//   kTf32x3  FP32 high parts + FP32 remainders, three kind::tf32 products
//            (hi*hi + hi*lo + lo*hi: close to FP32 accuracy);
//   kBf16    BF16 storage, one kind::f16 product with BF16 operands.
//
// One CTA per SM, persistent over 128 x 128 output tiles:
//   warp 0      TMA producer: A / Bt k-slices (one 128-byte swizzle row: 32
//               FP32 or 64 BF16 elements) into the stage ring, and an L2
//               prefetch of each tile's C block as the tile starts;
//   warp 1      MMA issuer (one thread): 4 x tcgen05.mma (32 bytes of K) per slice
//               into a TMEM accumulator (two 128-column buffers, so the next
//               tile's MMAs overlap this tile's epilogue); tcgen05.commit
//               releases smem stages and hands accumulators to the epilogue;
//   warps 2..5  epilogue: tcgen05.ld of their 32 TMEM lanes, C read from the
//               TMA-loaded swizzled block, result written back in place and
//               stored by one TMA bulk tensor store.
// Every wait is bounded; on a timeout the kernel records the error, skips the
// remaining work, and still frees its TMEM before exiting.  No multicast.
#include "common.cuh"
#include "internal.h"

namespace lm {

namespace {

enum : int { kTf32 = 0, kTf32x3 = 1, kBf16 = 2 };

constexpr int TBM = 128, TBN = 128;        // tile M, N; a k-slice is one 128-byte swizzle row
constexpr int T_A_BYTES = TBM * 128;       // 16 KB
constexpr int T_B_BYTES = TBN * 128;       // 16 KB
constexpr int T_C_BYTES = TBM * TBN * 4;   // 64 KB (4 boxes of 32 columns)
constexpr int T_THREADS = 6 * 32;

// Per mode: elements per 128-byte k-slice (TBK), whether the operands come
// as high parts + remainders (SPLIT: each k-step issues hi*hi + hi*lo + lo*hi),
// and the operand stages (2 for split, 4 otherwise).  Every MMA reads 32
// bytes of K (8 TF32 or 16 BF16 elements), four per slice.
template <int MODE>
struct TcCfg {
  static constexpr bool SPLIT = MODE == kTf32x3;
  static constexpr int TBK = MODE == kBf16 ? 64 : 32;
  static constexpr int STAGES = SPLIT ? 2 : 4;
  static constexpr int STAGE_BYTES = (T_A_BYTES + T_B_BYTES) * (SPLIT ? 2 : 1);
  static constexpr int SMEM = STAGES * STAGE_BYTES + T_C_BYTES + 1024 + 256;
};
constexpr uint32_t T_TMEM_COLS = 256;      // 2 accumulators x 128 fp32 columns

struct SgemmArgs {
  int m, n, k;
  float alpha, beta;
  int tiles_m, tiles_n, num_tiles;
  int* status;
  const int* gate;  // when set and *gate == 0 the launch does nothing
};

// ---- tcgen05 / bulk-copy wrappers -------------------------------------------
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_mma_tf32(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void tc_mma_f16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                           uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrive on an mbarrier of this CTA when all previously issued tcgen05.mma of
// this thread have completed.
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// 32 lanes x 32 consecutive fp32 columns of TMEM into 32 registers per thread.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tma_prefetch_l2_2d(const CUtensorMap* tmap, int x, int y) {
  asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];" ::"l"(
                   reinterpret_cast<uint64_t>(tmap)),
               "r"(x), "r"(y)
               : "memory");
}
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* tmap, const void* smem_src, int x, int y) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                   reinterpret_cast<uint64_t>(tmap)),
               "r"(x), "r"(y), "r"(smem_u32(smem_src))
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void named_bar(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// K-major operand, 128-byte swizzle: 8-row core groups 1024 B apart.
__device__ __forceinline__ uint64_t sw128_kmajor_desc(uint32_t smem_addr) {
  return (uint64_t)((smem_addr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptors: D f32 (bits 4-5 = 1), A and B format (bits 7-9,
// 10-12: 2 = TF32 for kind::tf32, 1 = BF16 for kind::f16), both K-major,
// N >> 3 (bits 17-22), M >> 4 (bits 24-28).
constexpr uint32_t kIdescTF32 = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TBN >> 3) << 17) |
                                ((uint32_t)(TBM >> 4) << 24);
constexpr uint32_t kIdescBF16 = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TBN >> 3) << 17) |
                                ((uint32_t)(TBM >> 4) << 24);

// byte offset of element (r, c) in a [128 rows][32 floats] 128B-swizzled box
__device__ __forceinline__ uint32_t cbox_off(int r, int c) {
  return (uint32_t)(r * 128 + ((((c >> 2) ^ (r & 7))) << 4) + ((c & 3) << 2));
}

template <int MODE>
__global__ void __launch_bounds__(T_THREADS, 1)
    sgemm_tf32_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      const __grid_constant__ CUtensorMap tmC, const __grid_constant__ CUtensorMap tmAl,
                      const __grid_constant__ CUtensorMap tmBl, SgemmArgs g) {
  constexpr bool SPLIT = TcCfg<MODE>::SPLIT;
  constexpr int TBK = TcCfg<MODE>::TBK;
  constexpr int TSTAGES = TcCfg<MODE>::STAGES;
  constexpr int T_STAGE_BYTES = TcCfg<MODE>::STAGE_BYTES;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  // stage s: [A | B | A_lo | B_lo] (the last two only when SPLIT)
  unsigned char* sA = smem;
  unsigned char* sC = smem + TSTAGES * T_STAGE_BYTES;
  uint64_t* full = reinterpret_cast<uint64_t*>(sC + T_C_BYTES);
  uint64_t* empty = full + TSTAGES;
  uint64_t* acc_full = empty + TSTAGES;   // [2]
  uint64_t* acc_empty = acc_full + 2;     // [2]
  uint64_t* c_full = acc_empty + 2;       // [1]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(c_full + 1);

  if (g.gate != nullptr && *g.gate == 0) return;  // uniform over the grid, before any barrier or TMEM
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int KT = (g.k + TBK - 1) / TBK;
  const bool use_beta = g.beta != 0.0f;

  if (threadIdx.x == 0) {
    for (int s = 0; s < TSTAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 4);
    }
    mbar_init(c_full, 1);
    fence_barrier_init();
  }
  if (warp == 1) tmem_alloc(tmem_slot, T_TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tmem_slot;
  bool ok = true;

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      tma_prefetch_desc(&tmA);
      tma_prefetch_desc(&tmB);
      int it = 0;
      for (int t = blockIdx.x; t < g.num_tiles && ok; t += gridDim.x) {
        const int tm = t % g.tiles_m, tn = t / g.tiles_m;
        // this tile's C block towards L2 while its operands stream in, so
        // that the epilogue's C load does not wait on DRAM
        if (use_beta) {
#pragma unroll
          for (int q = 0; q < TBN / 32; ++q) tma_prefetch_l2_2d(&tmC, tn * TBN + q * 32, tm * TBM);
        }
        for (int kb = 0; kb < KT && ok; ++kb, ++it) {
          const int s = it % TSTAGES;
          const uint32_t ph = (uint32_t)((it / TSTAGES) & 1) ^ 1u;
          if (!mbar_wait(&empty[s], ph, g.status)) { ok = false; break; }
          mbar_arrive_expect_tx(&full[s], T_STAGE_BYTES);
          unsigned char* st0 = sA + s * T_STAGE_BYTES;
          tma_load_2d(st0, &tmA, kb * TBK, tm * TBM, &full[s]);
          tma_load_2d(st0 + T_A_BYTES, &tmB, kb * TBK, tn * TBN, &full[s]);
          if (SPLIT) {
            tma_load_2d(st0 + T_A_BYTES + T_B_BYTES, &tmAl, kb * TBK, tm * TBM, &full[s]);
            tma_load_2d(st0 + 2 * T_A_BYTES + T_B_BYTES, &tmBl, kb * TBK, tn * TBN, &full[s]);
          }
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      int it = 0, lt = 0;
      for (int t = blockIdx.x; t < g.num_tiles && ok; t += gridDim.x, ++lt) {
        const int b = lt & 1;
        const uint32_t dt = tbase + (uint32_t)(b * TBN);
        if (!mbar_wait(&acc_empty[b], (uint32_t)(((lt >> 1) & 1) ^ 1), g.status)) { ok = false; break; }
        tc_fence_after();
        for (int kb = 0; kb < KT; ++kb, ++it) {
          const int s = it % TSTAGES;
          if (!mbar_wait(&full[s], (uint32_t)((it / TSTAGES) & 1), g.status)) { ok = false; break; }
          tc_fence_after();
          const uint32_t a0 = smem_u32(sA + s * T_STAGE_BYTES);
          const uint32_t b0 = a0 + T_A_BYTES;
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {  // four MMAs of 32 bytes of K per slice
            if (MODE == kBf16)
              tc_mma_f16(dt, sw128_kmajor_desc(a0 + kk * 32), sw128_kmajor_desc(b0 + kk * 32), kIdescBF16,
                         (kb > 0 || kk > 0) ? 1u : 0u);
            else
              tc_mma_tf32(dt, sw128_kmajor_desc(a0 + kk * 32), sw128_kmajor_desc(b0 + kk * 32), kIdescTF32,
                          (kb > 0 || kk > 0) ? 1u : 0u);
            if (SPLIT) {
              const uint32_t al = b0 + T_B_BYTES, bl = al + T_A_BYTES;
              tc_mma_tf32(dt, sw128_kmajor_desc(a0 + kk * 32), sw128_kmajor_desc(bl + kk * 32), kIdescTF32, 1u);
              tc_mma_tf32(dt, sw128_kmajor_desc(al + kk * 32), sw128_kmajor_desc(b0 + kk * 32), kIdescTF32, 1u);
            }
          }
          tc_commit(&empty[s]);  // smem stage free once these MMAs have read it
        }
        if (!ok) break;
        tc_commit(&acc_full[b]);  // accumulator complete
      }
    }
  } else {
    // ---------------- epilogue (warps 2..5, TMEM lane quarter = warp % 4) ----------------
    const int quarter = warp & 3;
    const int row_in_tile = quarter * 32 + lane;
    const bool leader = (warp == 2 && lane == 0);
    int lt = 0;
    for (int t = blockIdx.x; t < g.num_tiles; t += gridDim.x, ++lt) {
      const int tm = t % g.tiles_m, tn = t / g.tiles_m;
      const int b = lt & 1;
      if (ok && use_beta && leader) {
        bulk_wait_read0();  // the previous tile's store has finished reading sC
        mbar_arrive_expect_tx(c_full, T_C_BYTES);
#pragma unroll
        for (int q = 0; q < TBN / 32; ++q) tma_load_2d(sC + q * (TBM * 128), &tmC, tn * TBN + q * 32, tm * TBM, c_full);
      }
      if (ok && !mbar_wait(&acc_full[b], (uint32_t)((lt >> 1) & 1), g.status)) ok = false;
      if (ok && use_beta && !mbar_wait(c_full, (uint32_t)(lt & 1), g.status)) ok = false;
      if (!use_beta && leader) bulk_wait_read0();
      named_bar(1, 128);  // C block present (or free) for all epilogue warps
      __syncwarp();       // converged for the warp-wide tcgen05.ld (.sync.aligned)
      tc_fence_after();
      if (ok) {
#pragma unroll 1
        for (int q = 0; q < TBN / 32; ++q) {
          float acc[32];
          tmem_ld32(tbase + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * TBN + q * 32), acc);
          unsigned char* box = sC + q * (TBM * 128);
#pragma unroll
          for (int c4 = 0; c4 < 8; ++c4) {
            float4* p = reinterpret_cast<float4*>(box + cbox_off(row_in_tile, c4 * 4));
            float4 o = use_beta ? *p : make_float4(0.f, 0.f, 0.f, 0.f);
            o.x = fmaf(g.alpha, acc[c4 * 4 + 0], use_beta ? g.beta * o.x : 0.f);
            o.y = fmaf(g.alpha, acc[c4 * 4 + 1], use_beta ? g.beta * o.y : 0.f);
            o.z = fmaf(g.alpha, acc[c4 * 4 + 2], use_beta ? g.beta * o.z : 0.f);
            o.w = fmaf(g.alpha, acc[c4 * 4 + 3], use_beta ? g.beta * o.w : 0.f);
            *p = o;
          }
        }
      }
      tc_fence_before();
      if (lane == 0) mbar_arrive(&acc_empty[b]);  // TMEM buffer may be overwritten
      fence_proxy_async_smem();                  // smem writes visible to the TMA store
      named_bar(1, 128);
      if (ok && leader) {
#pragma unroll
        for (int q = 0; q < TBN / 32; ++q) tma_store_2d(&tmC, sC + q * (TBM * 128), tn * TBN + q * 32, tm * TBM);
        bulk_commit();
      }
    }
    if (leader) bulk_wait0();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tbase, T_TMEM_COLS);
  }
}

}  // namespace

void count_launch(int n);

namespace {

template <int MODE>
int sgemm_launch(Ctx& ctx, int m, int n, int k, float alpha, const void* A, long long lda, const void* Bt,
                 long long ldb, float beta, float* C, long long ldc, cudaStream_t st, const void* Alo,
                 const void* Btlo, int max_ctas, const int* gate) {
  constexpr int TBK = TcCfg<MODE>::TBK;
  constexpr int ES = MODE == kBf16 ? 2 : 4;  // operand element bytes
  const CUtensorMapDataType dt = MODE == kBf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(Bt) | reinterpret_cast<uintptr_t>(C) |
       reinterpret_cast<uintptr_t>(Alo) | reinterpret_cast<uintptr_t>(Btlo)) & 15)
    return LM_ERR_UNSUPPORTED;
  if (((lda * ES) | (ldb * ES) | (ldc * 4)) & 15) return LM_ERR_UNSUPPORTED;  // 16-byte row strides for TMA
  static bool attr_set[kMaxDevices] = {};
  const int dev = ctx_device(ctx);
  if (!attr_set[dev]) {
    LM_CUDA_TRY(cudaFuncSetAttribute(sgemm_tf32_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     TcCfg<MODE>::SMEM));
    attr_set[dev] = true;
  }
  CUtensorMap tA, tB, tC, tAl, tBl;
  LM_TRY(make_tmap_2d(&tA, dt, ES, A, k, m, lda, TBK, TBM, CU_TENSOR_MAP_SWIZZLE_128B));
  LM_TRY(make_tmap_2d(&tB, dt, ES, Bt, k, n, ldb, TBK, TBN, CU_TENSOR_MAP_SWIZZLE_128B));
  LM_TRY(make_tmap_2d(&tC, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, C, n, m, ldc, 32, TBM, CU_TENSOR_MAP_SWIZZLE_128B));
  if (TcCfg<MODE>::SPLIT) {
    LM_TRY(make_tmap_2d(&tAl, dt, ES, Alo, k, m, lda, TBK, TBM, CU_TENSOR_MAP_SWIZZLE_128B));
    LM_TRY(make_tmap_2d(&tBl, dt, ES, Btlo, k, n, ldb, TBK, TBN, CU_TENSOR_MAP_SWIZZLE_128B));
  } else {
    tAl = tA;
    tBl = tB;
  }
  SgemmArgs g;
  g.m = m; g.n = n; g.k = k; g.alpha = alpha; g.beta = beta;
  g.tiles_m = cdiv(m, TBM);
  g.tiles_n = cdiv(n, TBN);
  g.num_tiles = g.tiles_m * g.tiles_n;
  g.status = ctx_status(ctx);
  g.gate = gate;
  const int grid = std::min(g.num_tiles, max_ctas > 0 ? std::min(max_ctas, ctx_num_sms(ctx)) : ctx_num_sms(ctx));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid, 1, 1);
  cfg.blockDim = dim3(T_THREADS, 1, 1);
  cfg.dynamicSmemBytes = TcCfg<MODE>::SMEM;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;  // explicit 1-CTA clusters for the shared::cluster forms
  attr[0].val.clusterDim.x = 1;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  {
    const int products = TcCfg<MODE>::SPLIT ? 3 : 1;
    Prof prof(ctx, kPhaseGemm, 2.0 * m * n * k * products,
              (double)ES * ((double)m * k + (double)n * k) * (TcCfg<MODE>::SPLIT ? 2 : 1) + 8.0 * m * n, st);
    LM_CUDA_TRY(cudaLaunchKernelEx(&cfg, sgemm_tf32_kernel<MODE>, tA, tB, tC, tAl, tBl, g));
  }
  count_launch(1);
  return LM_OK;
}

}  // namespace

int sgemm_tf32(Ctx& ctx, int m, int n, int k, float alpha, const float* A, long long lda, const float* Bt,
               long long ldb, float beta, float* C, long long ldc, cudaStream_t st, const float* Alo,
               const float* Btlo, int max_ctas, const int* gate) {
  if (m <= 0 || n <= 0) return LM_OK;
  if (k <= 0) return LM_ERR_ARG;
  if (Alo != nullptr && Btlo != nullptr)
    return sgemm_launch<kTf32x3>(ctx, m, n, k, alpha, A, lda, Bt, ldb, beta, C, ldc, st, Alo, Btlo, max_ctas, gate);
  return sgemm_launch<kTf32>(ctx, m, n, k, alpha, A, lda, Bt, ldb, beta, C, ldc, st, nullptr, nullptr, max_ctas,
                             gate);
}

int sgemm_bf16(Ctx& ctx, int m, int n, int k, float alpha, const void* A, long long lda, const void* Bt,
               long long ldb, float beta, float* C, long long ldc, cudaStream_t st, int max_ctas) {
  if (m <= 0 || n <= 0) return LM_OK;
  if (k <= 0) return LM_ERR_ARG;
  return sgemm_launch<kBf16>(ctx, m, n, k, alpha, A, lda, Bt, ldb, beta, C, ldc, st, nullptr, nullptr, max_ctas,
                             nullptr);
}

}  // namespace lm
