// FP64 GEMM on the sm_100a FP64 tensor cores (DMMA, mma.sync m16n8k4 f64).
//
// Replaces linear-massiv's rawGemmKernel family (Internal/Kernel.hs:145-806:
// the 4x8 AVX2 register-blocked micro-kernel over 64^3 cache blocks, with
// B-panel packing above min dimension 96).  On B200 the "cache blocking" is a
// 128 x 128 (or 128 x 64) CTA tile, the "packing" is a TMA tile load into
// 128-byte-swizzled shared memory, and the "micro-kernel" is a warp tile of
// 64 x 32 FP64 accumulators fed by DMMA.
//
// Structure (one CTA per SM, persistent over output tiles):
//   warp NC       : TMA producer (one elected lane) filling a STAGES-deep ring
//                   of A/B k-slices (16 doubles = 128 B deep), mbarrier-tracked;
//   warps 0..NC-1 : consumers, each a 64 x 32 warp tile of m16n8k4 DMMAs,
//                   then a fused epilogue C = alpha*acc + beta*C (in place),
//                   optionally restricted to the lower triangle (SYRK tiles).
// No cluster multicast is used anywhere.
#include "common.cuh"
#include "internal.h"

namespace lm {
namespace {

constexpr int kBK = 16;  // doubles per k-slice: one 128-byte swizzle row

__device__ __forceinline__ uint32_t swz128(int r, int c) {
  // byte offset of element (r, c) in a [rows][16] double tile stored with the
  // TMA 128-byte swizzle (16-byte chunk index XOR row mod 8)
  return (uint32_t)(r * 128 + ((((c >> 1) ^ (r & 7))) << 4) + ((c & 1) << 3));
}

__device__ __forceinline__ double lds_f64(uint32_t addr) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(addr));
  return v;
}

struct GemmArgs {
  int m, n, k;
  double alpha, beta;
  double* C;
  long long ldc;
  int lower_only;
  int tiles_m, tiles_n, num_tiles;
  int* status;
};

template <int BM, int BN>
struct GemmCfg {
  static constexpr int NC = (BM / 64) * (BN / 32);  // consumer warps
  static constexpr int THREADS = (NC + 1) * 32;
  static constexpr int A_BYTES = BM * kBK * 8;
  static constexpr int B_BYTES = BN * kBK * 8;
  static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  static constexpr int STAGES = (200 * 1024) / STAGE_BYTES > 8 ? 8 : (200 * 1024) / STAGE_BYTES;
  static constexpr int SMEM = STAGES * STAGE_BYTES + 2 * STAGES * 8 + 1024;  // + alignment slack
};

__device__ __forceinline__ void tile_coords(const GemmArgs& g, int t, int& tm, int& tn) {
  if (g.lower_only) {
    // tiles (tm, tn) with tn <= tm, enumerated row by row
    int r = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((long long)(r + 1) * (r + 2) / 2 <= t) ++r;
    while ((long long)r * (r + 1) / 2 > t) --r;
    tm = r;
    tn = t - r * (r + 1) / 2;
  } else {
    const int GROUP = 8;
    const int per_group = GROUP * g.tiles_n;
    const int gid = t / per_group;
    const int first_m = gid * GROUP;
    const int gsz = min(g.tiles_m - first_m, GROUP);
    const int in = t % per_group;
    tm = first_m + in % gsz;
    tn = in / gsz;
  }
}

template <int BM, int BN, bool AT, bool BT>
__global__ void __launch_bounds__(GemmCfg<BM, BN>::THREADS, 1)
    dgemm_dmma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      GemmArgs g) {
  using Cfg = GemmCfg<BM, BN>;
  constexpr int STAGES = Cfg::STAGES;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* sA = smem;
  unsigned char* sB = smem + STAGES * Cfg::A_BYTES;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * Cfg::STAGE_BYTES);
  uint64_t* empty = full + STAGES;

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int KT = (g.k + kBK - 1) / kBK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], Cfg::NC);
    }
    fence_barrier_init();
  }
  __syncthreads();

  if (warp == Cfg::NC) {
    // ---------------- producer ----------------
    if (lane == 0) {
      tma_prefetch_desc(&tmA);
      tma_prefetch_desc(&tmB);
      int it = 0;
      for (int t = blockIdx.x; t < g.num_tiles; t += gridDim.x) {
        int tm, tn;
        tile_coords(g, t, tm, tn);
        for (int kb = 0; kb < KT; ++kb, ++it) {
          const int s = it % STAGES;
          const uint32_t ph = (uint32_t)((it / STAGES) & 1) ^ 1u;
          if (!mbar_wait(&empty[s], ph, g.status)) return;
          mbar_arrive_expect_tx(&full[s], Cfg::STAGE_BYTES);
          if (AT) {
#pragma unroll
            for (int j = 0; j < BM / 16; ++j)
              tma_load_2d(sA + s * Cfg::A_BYTES + j * 2048, &tmA, tm * BM + j * 16, kb * kBK, &full[s]);
          } else {
            tma_load_2d(sA + s * Cfg::A_BYTES, &tmA, kb * kBK, tm * BM, &full[s]);
          }
          if (BT) {
            tma_load_2d(sB + s * Cfg::B_BYTES, &tmB, kb * kBK, tn * BN, &full[s]);
          } else {
#pragma unroll
            for (int j = 0; j < BN / 16; ++j)
              tma_load_2d(sB + s * Cfg::B_BYTES + j * 2048, &tmB, tn * BN + j * 16, kb * kBK, &full[s]);
          }
        }
      }
    }
    return;
  }

  // ---------------- consumers ----------------
  const int wm = warp / (BN / 32);
  const int wn = warp % (BN / 32);
  const int gq = lane >> 2;  // groupID
  const int tq = lane & 3;   // threadID_in_group
  const uint32_t sA32 = smem_u32(sA);
  const uint32_t sB32 = smem_u32(sB);

  int it = 0;
  for (int t = blockIdx.x; t < g.num_tiles; t += gridDim.x) {
    int tm, tn;
    tile_coords(g, t, tm, tn);
    double acc[4][4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0;

    for (int kb = 0; kb < KT; ++kb, ++it) {
      const int s = it % STAGES;
      const uint32_t ph = (uint32_t)((it / STAGES) & 1);
      if (!mbar_wait(&full[s], ph, g.status)) return;
      const uint32_t aBase = sA32 + s * Cfg::A_BYTES;
      const uint32_t bBase = sB32 + s * Cfg::B_BYTES;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        double af[4][2], bf[4];
        const int kc = kk * 4 + tq;
#pragma unroll
        for (int mi = 0; mi < 4; ++mi) {
          const int r = wm * 64 + mi * 16 + gq;
          if (AT) {
            af[mi][0] = lds_f64(aBase + (r >> 4) * 2048 + swz128(kc, r & 15));
            af[mi][1] = lds_f64(aBase + ((r + 8) >> 4) * 2048 + swz128(kc, (r + 8) & 15));
          } else {
            af[mi][0] = lds_f64(aBase + swz128(r, kc));
            af[mi][1] = lds_f64(aBase + swz128(r + 8, kc));
          }
        }
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
          const int nl = wn * 32 + ni * 8 + gq;
          if (BT)
            bf[ni] = lds_f64(bBase + swz128(nl, kc));
          else
            bf[ni] = lds_f64(bBase + (nl >> 4) * 2048 + swz128(kc, nl & 15));
        }
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
          for (int ni = 0; ni < 4; ++ni) dmma_16x8x4(acc[mi][ni], af[mi][0], af[mi][1], bf[ni]);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }

    // ---------------- epilogue: C = alpha*acc + beta*C ----------------
    const bool vec_ok = ((g.ldc & 1) == 0) && ((reinterpret_cast<uintptr_t>(g.C) & 15) == 0);
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int row = tm * BM + wm * 64 + mi * 16 + gq + h * 8;
        if (row >= g.m) continue;
        double* crow = g.C + (long long)row * g.ldc;
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
          const int col = tn * BN + wn * 32 + ni * 8 + 2 * tq;
          const double v0 = acc[mi][ni][2 * h], v1 = acc[mi][ni][2 * h + 1];
          const bool in0 = col < g.n && (!g.lower_only || col <= row);
          const bool in1 = col + 1 < g.n && (!g.lower_only || col + 1 <= row);
          if (in0 && in1 && vec_ok) {
            double2* p = reinterpret_cast<double2*>(crow + col);
            double2 o = make_double2(0.0, 0.0);
            if (g.beta != 0.0) o = *p;
            o.x = fma(g.alpha, v0, g.beta != 0.0 ? g.beta * o.x : 0.0);
            o.y = fma(g.alpha, v1, g.beta != 0.0 ? g.beta * o.y : 0.0);
            *p = o;
          } else {
            if (in0) {
              const double old = (g.beta != 0.0) ? g.beta * crow[col] : 0.0;
              crow[col] = fma(g.alpha, v0, old);
            }
            if (in1) {
              const double old = (g.beta != 0.0) ? g.beta * crow[col + 1] : 0.0;
              crow[col + 1] = fma(g.alpha, v1, old);
            }
          }
        }
      }
    }
  }
}

__global__ void scale_kernel(double* C, long long ldc, int m, int n, double beta, int lower_only) {
  const long long total = (long long)m * n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / n), c = (int)(i % n);
    if (lower_only && c > r) continue;
    double* p = C + (long long)r * ldc + c;
    *p = (beta == 0.0) ? 0.0 : beta * *p;
  }
}

template <int BM, int BN, bool AT, bool BT>
int launch_dmma(Ctx& ctx, const GemmDesc& d, cudaStream_t st) {
  using Cfg = GemmCfg<BM, BN>;
  static bool attr_set[kMaxDevices] = {};  // per instantiation and device, set under the API lock
  auto kern = dgemm_dmma_kernel<BM, BN, AT, BT>;
  const int dev = ctx_device(ctx);
  if (!attr_set[dev]) {
    LM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM));
    attr_set[dev] = true;
  }
  CUtensorMap tmA, tmB;
  if (AT)
    LM_TRY(make_tmap_2d(&tmA, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, d.A, d.m, d.k, d.lda, 16, kBK,
                        CU_TENSOR_MAP_SWIZZLE_128B));
  else
    LM_TRY(make_tmap_2d(&tmA, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, d.A, d.k, d.m, d.lda, kBK, BM,
                        CU_TENSOR_MAP_SWIZZLE_128B));
  if (BT)
    LM_TRY(make_tmap_2d(&tmB, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, d.B, d.k, d.n, d.ldb, kBK, BN,
                        CU_TENSOR_MAP_SWIZZLE_128B));
  else
    LM_TRY(make_tmap_2d(&tmB, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, d.B, d.n, d.k, d.ldb, 16, kBK,
                        CU_TENSOR_MAP_SWIZZLE_128B));
  GemmArgs g;
  g.m = d.m; g.n = d.n; g.k = d.k;
  g.alpha = d.alpha; g.beta = d.beta;
  g.C = d.C; g.ldc = d.ldc;
  g.lower_only = d.lower_only ? 1 : 0;
  g.tiles_m = cdiv(d.m, BM);
  g.tiles_n = cdiv(d.n, BN);
  g.num_tiles = d.lower_only ? g.tiles_m * (g.tiles_m + 1) / 2 : g.tiles_m * g.tiles_n;
  g.status = ctx_status(ctx);
  int grid = std::min(g.num_tiles, d.max_ctas > 0 ? d.max_ctas : ctx_num_sms(ctx));
  kern<<<grid, Cfg::THREADS, Cfg::SMEM, st>>>(tmA, tmB, g);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

}  // namespace

int dgemm(Ctx& ctx, const GemmDesc& d, cudaStream_t st) {
  if (d.m < 0 || d.n < 0 || d.k < 0) return LM_ERR_ARG;
  if (d.m == 0 || d.n == 0) return LM_OK;
  if (d.lower_only && d.m != d.n) return LM_ERR_ARG;
  if (d.k == 0 || d.alpha == 0.0) {
    if (d.beta == 1.0) return LM_OK;
    const long long total = (long long)d.m * d.n;
    const int grid = (int)std::min<long long>(cdivll(total, 256), 4LL * ctx_num_sms(ctx));
    scale_kernel<<<grid, 256, 0, st>>>(d.C, d.ldc, d.m, d.n, d.beta, d.lower_only ? 1 : 0);
    count_launch(1);
    LM_CUDA_TRY(cudaGetLastError());
    return LM_OK;
  }
  // TMA needs 16-byte aligned bases and row strides.
  if ((reinterpret_cast<uintptr_t>(d.A) & 15) || (reinterpret_cast<uintptr_t>(d.B) & 15) ||
      (d.lda & 1) || (d.ldb & 1))
    return LM_ERR_UNSUPPORTED;
  if (d.a_trans && d.b_trans) return LM_ERR_UNSUPPORTED;
  const bool narrow = d.n <= 64 && !d.lower_only;
  if (d.a_trans)
    return narrow ? launch_dmma<128, 64, true, false>(ctx, d, st)
                  : launch_dmma<128, 128, true, false>(ctx, d, st);
  if (d.b_trans)
    return narrow ? launch_dmma<128, 64, false, true>(ctx, d, st)
                  : launch_dmma<128, 128, false, true>(ctx, d, st);
  return narrow ? launch_dmma<128, 64, false, false>(ctx, d, st)
                : launch_dmma<128, 128, false, false>(ctx, d, st);
}

}  // namespace lm
