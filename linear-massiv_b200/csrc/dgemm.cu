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
// Short-k updates with beta != 0 (the factorisations' trailing updates) stage
// each C tile in shared memory: the producer TMA-loads it while the tile's
// main loop runs, so the epilogue reads C on chip instead of waiting on
// L2/HBM (at k = 128 those waits were about a third of the time).
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
  int prefetch_c;  // TMA-prefetch each C tile into L2 when its main loop starts
  int tiles_m, tiles_n, num_tiles;
  int* status;
};

__device__ __forceinline__ void tma_prefetch_l2_2d(const CUtensorMap* tmap, int x, int y) {
  asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];" ::"l"(
                   reinterpret_cast<uint64_t>(tmap)),
               "r"(x), "r"(y)
               : "memory");
}

// MINB CTAs share an SM: with two, one CTA's epilogue (C read-modify-write)
// overlaps the other's DMMA main loop, which matters for the short-k
// trailing updates of the factorisations.
template <int BM, int BN, int MINB, bool CSM = false>
struct GemmCfg {
  static constexpr int NC = (BM / 64) * (BN / 32);  // consumer warps
  // Short-k update (CSM): the producer is a whole warpgroup so that
  // setmaxnreg can move its registers to the consumers (a lone producer warp
  // puts three warps on one SM sub-partition, which caps every thread at 168
  // registers and spills the 64 x 32 FP64 accumulator tile in the main loop;
  // at k = 128 that cost 17%, while the long-k kernel measured the same
  // either way)
  static constexpr bool SPLIT_REGS = CSM && NC == 8 && MINB == 1;
  static constexpr int PRODUCER_WARPS = SPLIT_REGS ? 4 : 1;
  static constexpr int THREADS = (NC + PRODUCER_WARPS) * 32;
  static constexpr int LAUNCH_REGS = 168;  // 65536 / 384, rounded down to 8
  static constexpr int CONSUMER_REGS = 232, PRODUCER_REGS = 40;
  static_assert(!SPLIT_REGS || NC * 32 * CONSUMER_REGS + PRODUCER_WARPS * 32 * PRODUCER_REGS <=
                                     THREADS * LAUNCH_REGS,
                "register split must fit in what the CTA is launched with");
  static constexpr int A_BYTES = BM * kBK * 8;
  static constexpr int B_BYTES = BN * kBK * 8;
  static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  // C staged in smem as BN / 16 boxes of BM x 16 doubles (128-byte swizzle)
  static constexpr int C_BYTES = CSM ? BM * BN * 8 : 0;
  static constexpr int BUDGET = CSM ? 227 * 1024 - C_BYTES - 2048 : (200 * 1024) / MINB;
  static constexpr int STAGES = BUDGET / STAGE_BYTES > 8 ? 8 : BUDGET / STAGE_BYTES;
  static constexpr int SMEM = STAGES * STAGE_BYTES + C_BYTES + 2 * STAGES * 8 + 16 + 1024;  // + alignment slack
  static_assert(SMEM <= 227 * 1024, "shared memory per CTA");
  static_assert(STAGES >= 2, "operand ring depth");
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

// CSM: C staged in shared memory (tmC then maps 16-double x BM boxes with the
// 128-byte swizzle); requires beta != 0.
template <int BM, int BN, bool AT, bool BT, int MINB, bool CSM>
__global__ void __launch_bounds__(GemmCfg<BM, BN, MINB, CSM>::THREADS, MINB)
    dgemm_dmma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      const __grid_constant__ CUtensorMap tmC, GemmArgs g) {
  using Cfg = GemmCfg<BM, BN, MINB, CSM>;
  constexpr int STAGES = Cfg::STAGES;
  constexpr int C_BOX = BM * 16 * 8;  // bytes of one staged C box
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* sA = smem;
  unsigned char* sB = smem + STAGES * Cfg::A_BYTES;
  unsigned char* sC = smem + STAGES * Cfg::STAGE_BYTES;  // 1024-aligned: stage sizes are multiples of 2 KB
  uint64_t* full = reinterpret_cast<uint64_t*>(sC + Cfg::C_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* cfull = empty + STAGES;  // C tile landed
  uint64_t* cempty = cfull + 1;      // every consumer warp has read it

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int KT = (g.k + kBK - 1) / kBK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], Cfg::NC);
    }
    mbar_init(cfull, 1);
    mbar_init(cempty, Cfg::NC);
    fence_barrier_init();
  }
  __syncthreads();

  if (warp >= Cfg::NC) {
    // ---------------- producer ----------------
    if constexpr (Cfg::SPLIT_REGS)
      asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(Cfg::PRODUCER_REGS) : "memory");
    if (warp == Cfg::NC && lane == 0) {
      tma_prefetch_desc(&tmA);
      tma_prefetch_desc(&tmB);
      if (CSM) tma_prefetch_desc(&tmC);
      int it = 0, cj = 0;
      for (int t = blockIdx.x; t < g.num_tiles; t += gridDim.x, ++cj) {
        int tm, tn;
        tile_coords(g, t, tm, tn);
        if (!CSM && g.prefetch_c) tma_prefetch_l2_2d(&tmC, tn * BN, tm * BM);
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
          if (CSM && kb == min(STAGES, KT) - 1) {
            // this tile's C, once the previous tile's epilogue has read the
            // buffer; issued after the first ring slots so that the main
            // loop never waits on it
            if (!mbar_wait(cempty, (uint32_t)(cj & 1) ^ 1u, g.status)) return;
            mbar_arrive_expect_tx(cfull, Cfg::C_BYTES);
#pragma unroll
            for (int j = 0; j < BN / 16; ++j) tma_load_2d(sC + j * C_BOX, &tmC, tn * BN + j * 16, tm * BM, cfull);
          }
        }
      }
    }
    return;
  }

  // ---------------- consumers ----------------
  if constexpr (Cfg::SPLIT_REGS)
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(Cfg::CONSUMER_REGS) : "memory");
  const int wm = warp / (BN / 32);
  const int wn = warp % (BN / 32);
  const int gq = lane >> 2;  // groupID
  const int tq = lane & 3;   // threadID_in_group
  const uint32_t sA32 = smem_u32(sA);
  const uint32_t sB32 = smem_u32(sB);

  int it = 0, cj = 0;
  for (int t = blockIdx.x; t < g.num_tiles; t += gridDim.x, ++cj) {
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
      // lanes leave the poll independently: reconverge before the warp-wide
      // mma.sync of this slice
      __syncwarp();
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
    // Per 16-row slice: issue all of its C loads first, then the FMAs and stores.
    const bool vec_ok = ((g.ldc & 1) == 0) && ((reinterpret_cast<uintptr_t>(g.C) & 15) == 0);
    const bool use_beta = g.beta != 0.0;
    if constexpr (CSM) {
      if (!mbar_wait(cfull, (uint32_t)(cj & 1), g.status)) return;
      __syncwarp();
      const uint32_t sC32 = smem_u32(sC);
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int rl = wm * 64 + mi * 16 + gq + h * 8;  // row within the tile
          const int row = tm * BM + rl;
#pragma unroll
          for (int ni = 0; ni < 4; ++ni) {
            const int cl = wn * 32 + ni * 8 + 2 * tq;  // column within the tile (even)
            double2 o;
            asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];"
                         : "=d"(o.x), "=d"(o.y)
                         : "r"(sC32 + (cl >> 4) * C_BOX + swz128(rl, cl & 15)));
            if (row >= g.m) continue;
            const int col = tn * BN + cl;
            const bool in0 = col < g.n && (!g.lower_only || col <= row);
            const bool in1 = col + 1 < g.n && (!g.lower_only || col + 1 <= row);
            const double r0 = fma(g.alpha, acc[mi][ni][2 * h], g.beta * o.x);
            const double r1 = fma(g.alpha, acc[mi][ni][2 * h + 1], g.beta * o.y);
            double* crow = g.C + (long long)row * g.ldc;
            if (in0 && in1 && vec_ok) {
              *reinterpret_cast<double2*>(crow + col) = make_double2(r0, r1);
            } else {
              if (in0) crow[col] = r0;
              if (in1) crow[col + 1] = r1;
            }
          }
        }
      __syncwarp();
      if (lane == 0) mbar_arrive(cempty);
    } else {
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) {
        double old[2][4][2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int row = tm * BM + wm * 64 + mi * 16 + gq + h * 8;
          const double* crow = g.C + (long long)row * g.ldc;
#pragma unroll
          for (int ni = 0; ni < 4; ++ni) {
            const int col = tn * BN + wn * 32 + ni * 8 + 2 * tq;
            old[h][ni][0] = 0.0;
            old[h][ni][1] = 0.0;
            if (use_beta && row < g.m) {
              const bool in0 = col < g.n && (!g.lower_only || col <= row);
              const bool in1 = col + 1 < g.n && (!g.lower_only || col + 1 <= row);
              if (in0 && in1 && vec_ok) {
                const double2 o = *reinterpret_cast<const double2*>(crow + col);
                old[h][ni][0] = o.x;
                old[h][ni][1] = o.y;
              } else {
                if (in0) old[h][ni][0] = crow[col];
                if (in1) old[h][ni][1] = crow[col + 1];
              }
            }
          }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int row = tm * BM + wm * 64 + mi * 16 + gq + h * 8;
          if (row >= g.m) continue;
          double* crow = g.C + (long long)row * g.ldc;
#pragma unroll
          for (int ni = 0; ni < 4; ++ni) {
            const int col = tn * BN + wn * 32 + ni * 8 + 2 * tq;
            const bool in0 = col < g.n && (!g.lower_only || col <= row);
            const bool in1 = col + 1 < g.n && (!g.lower_only || col + 1 <= row);
            const double r0 = fma(g.alpha, acc[mi][ni][2 * h], use_beta ? g.beta * old[h][ni][0] : 0.0);
            const double r1 = fma(g.alpha, acc[mi][ni][2 * h + 1], use_beta ? g.beta * old[h][ni][1] : 0.0);
            if (in0 && in1 && vec_ok) {
              *reinterpret_cast<double2*>(crow + col) = make_double2(r0, r1);
            } else {
              if (in0) crow[col] = r0;
              if (in1) crow[col + 1] = r1;
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

template <int BM, int BN, bool AT, bool BT, int MINB, bool CSM = false>
int launch_dmma(Ctx& ctx, const GemmDesc& d, cudaStream_t st) {
  using Cfg = GemmCfg<BM, BN, MINB, CSM>;
  static bool attr_set[kMaxDevices] = {};  // per instantiation and device, set under the API lock
  auto kern = dgemm_dmma_kernel<BM, BN, AT, BT, MINB, CSM>;
  const int dev = ctx_device(ctx);
  if (!attr_set[dev]) {
    LM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM));
    if (Cfg::SPLIT_REGS) {
      // the setmaxnreg split assumes the CTA is launched with LAUNCH_REGS per
      // thread; with fewer the consumers' increase could never be granted,
      // so the caller falls back to another kernel
      cudaFuncAttributes fa;
      LM_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
      if (fa.numRegs < Cfg::LAUNCH_REGS) return LM_ERR_UNSUPPORTED;
    }
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
  CUtensorMap tmC;
  const bool c_ok = d.beta != 0.0 && !(reinterpret_cast<uintptr_t>(d.C) & 15) && !(d.ldc & 1);
  if (CSM && !c_ok) return LM_ERR_ARG;
  if (CSM)
    LM_TRY(make_tmap_2d(&tmC, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, d.C, d.n, d.m, d.ldc, 16, BM,
                        CU_TENSOR_MAP_SWIZZLE_128B));
  else if (c_ok)
    LM_TRY(make_tmap_2d(&tmC, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, d.C, d.n, d.m, d.ldc, BN, BM,
                        CU_TENSOR_MAP_SWIZZLE_NONE));
  else
    tmC = tmA;  // unused
  GemmArgs g;
  g.prefetch_c = c_ok ? 1 : 0;
  g.m = d.m; g.n = d.n; g.k = d.k;
  g.alpha = d.alpha; g.beta = d.beta;
  g.C = d.C; g.ldc = d.ldc;
  g.lower_only = d.lower_only ? 1 : 0;
  g.tiles_m = cdiv(d.m, BM);
  g.tiles_n = cdiv(d.n, BN);
  g.num_tiles = d.lower_only ? g.tiles_m * (g.tiles_m + 1) / 2 : g.tiles_m * g.tiles_n;
  g.status = ctx_status(ctx);
  const int sms = d.max_sms > 0 ? std::min(d.max_sms, ctx_num_sms(ctx)) : ctx_num_sms(ctx);
  int grid = std::min(g.num_tiles, MINB * sms);
  kern<<<grid, Cfg::THREADS, Cfg::SMEM, st>>>(tmA, tmB, tmC, g);
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
  // Short k with beta != 0 (the factorisations' trailing updates): 128 x 128
  // tiles with C staged in shared memory.  Other short-k or narrow products:
  // 128 x 64 tiles, two CTAs per SM.  Long k: 128 x 128 tiles, one CTA per
  // SM, deeper pipeline.
  const double flops = d.lower_only ? (double)d.m * (d.m + 1) * d.k : 2.0 * d.m * d.n * d.k;
  const double bytes = 8.0 * ((double)d.m * d.k + (double)d.k * d.n +
                              (d.beta != 0.0 ? 2.0 : 1.0) * (d.lower_only ? 0.5 : 1.0) * d.m * d.n);
  Prof prof(ctx, kPhaseGemm, flops, bytes, st);
  const bool narrow = (d.n <= 64 || d.k <= 256) && !d.lower_only;
  const bool c_tma = d.beta != 0.0 && !(reinterpret_cast<uintptr_t>(d.C) & 15) && !(d.ldc & 1);
  if (d.k <= 256 && d.n > 64 && c_tma) {
    int rc;
    if (d.a_trans)
      rc = launch_dmma<128, 128, true, false, 1, true>(ctx, d, st);
    else if (d.b_trans)
      rc = launch_dmma<128, 128, false, true, 1, true>(ctx, d, st);
    else
      rc = launch_dmma<128, 128, false, false, 1, true>(ctx, d, st);
    // LM_ERR_UNSUPPORTED before any launch: compiled with fewer registers
    // than the register split needs; the kernels below take the update
    if (rc != LM_ERR_UNSUPPORTED) return rc;
  }
  if (d.a_trans)
    return narrow ? launch_dmma<128, 64, true, false, 2>(ctx, d, st)
                  : launch_dmma<128, 128, true, false, 1>(ctx, d, st);
  if (d.b_trans)
    return narrow ? launch_dmma<128, 64, false, true, 2>(ctx, d, st)
                  : launch_dmma<128, 128, false, true, 1>(ctx, d, st);
  return narrow ? launch_dmma<128, 64, false, false, 2>(ctx, d, st)
                : launch_dmma<128, 128, false, false, 1>(ctx, d, st);
}

}  // namespace lm
