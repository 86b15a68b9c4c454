// Cosine preweight + Shepp-Logan ramp filter as a split-BF16 Toeplitz GEMM on
// the 5th-generation tensor cores (tcgen05, TMEM accumulators, TMA-fed).
//
// Reference math: src/filtering.cu:187-207 (preweight) and :15-25, :57-175
// (f[j] = sum_m p[m] h[j-m], |j-m| <= YL-1, h[n] = -2/(pi^2 (4n^2-1))/dYL).
// Written as a matrix product over all detector rows r:
//
//   F[r][n] = sum_k P[r][k] T[n][k],   T[n][k] = h[n-k]  (n, k < YL; 0 beyond)
//
// Both operands are split into three BF16 parts (x = x0 + x1 + x2, each part
// the BF16 rounding of what the previous ones leave) and the product is
// accumulated in FP32 from the six terms P0T0 + P0T1 + P1T0 + P0T2 + P1T1 +
// P2T0, i.e. with ~24 significant bits per operand. The ramp kernel cancels
// heavily on projection data (sum |p h| >> |sum p h|): a two-part (hi+lo)
// split leaves a systematic 6e-4 relative error on real rows, the three-part
// split 6e-7, below an FP32 direct sum (4e-6). The result is written as the
// fast backprojection's BF16 channel pairs (word j = (F[j], F[j+1])).
//
// Stages:
//   1. prep kernel: rebinned (or row-layout) FP32 -> preweighted, split,
//      K-major BF16 rows A0/A1/A2 [rows][KP] (KP = YL rounded up to 64).
//   2. GEMM kernel, persistent (one CTA of 6 warps per SM walking the
//      (128-row, 112-column) output tiles): warp 0 lane 0 issues TMA loads of
//      A0..A2 (128 x 64) and T0..T2 (128 x 64; 16 extra columns give every
//      pair its right neighbour) into a 2-stage ring of 128B-swizzled
//      shared-memory tiles, across tile boundaries; warp 1 lane 0 issues 24
//      tcgen05.mma (M=128, N=128, K=16) per 64-wide K block into one of two
//      TMEM accumulators of 128 FP32 columns (alternating by tile) and
//      commits each stage back to the producer and each finished tile to the
//      epilogue; warps 2-5 read their 32 TMEM lanes each (tcgen05.ld 32x32b),
//      store BF16 pairs and release the accumulator, so that a tile's
//      epilogue runs under the next tile's MMAs.
// Every mbarrier wait is bounded: on timeout the kernel records an error in a
// device flag, stops issuing, lets committed work drain, frees its TMEM and
// returns; hr_filter_tc_check reports the flag.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "hr_internal.h"

namespace {

constexpr int kBM = 128;      // output rows per CTA (TMEM lanes)
constexpr int kBNOut = 112;   // output columns per CTA
constexpr int kBN = 128;      // MMA N: kBNOut + 16 neighbour columns
constexpr int kBK = 64;       // K block: 64 BF16 = one 128-byte swizzle row
constexpr int kStages = 2;
constexpr int kTileA = kBM * kBK * 2;          // 16 KiB
constexpr int kTileB = kBN * kBK * 2;          // 16 KiB
constexpr int kParts = 3;                      // BF16 parts per operand
constexpr int kStageBytes = kParts * kTileA + kParts * kTileB;
constexpr int kEpiWarps = 4;                   // epilogue warps (one per TMEM lane quarter)
constexpr int kTmemCols = 2 * kBN;             // two accumulators
constexpr int kThreads = 32 * (2 + kEpiWarps); // producer warp, MMA warp, epilogue warps
constexpr uint32_t kWaitLimit = 1u << 20;      // try_wait rounds before a wait is declared hung

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// Bounded wait on an mbarrier phase. Returns false (after setting the error
// flag and the CTA's abort flag) if the phase does not complete within
// `limit` polls, or if another role of the CTA has already aborted.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, int* err, volatile int* abort_flag,
                                          uint32_t limit) {
  const uint32_t addr = smem_u32(bar);
  for (uint32_t i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(phase)
        : "memory");
    if (done) return true;
    if (*abort_flag) return false;
  }
  atomicExch(err, 1);
  *abort_flag = 1;
  return false;
}

// Bounded wait for the completion of a phase whose TMA copies were issued,
// ignoring the abort flag: a CTA that aborts still lets its own copies land
// in its shared memory before it exits.
__device__ __forceinline__ void mbar_drain(uint64_t* bar, uint32_t phase, int* err, uint32_t limit) {
  const uint32_t addr = smem_u32(bar);
  for (uint32_t i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(phase)
        : "memory");
    if (done) return;
  }
  atomicExch(err, 2);
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// UMMA shared-memory descriptor of a K-major, 128B-swizzled tile whose 8-row
// groups are 1024 bytes apart (LBO = 16 B, SBO = 1024 B, version 1).
__device__ __forceinline__ uint64_t umma_desc_sw128(const void* tile) {
  const uint64_t addr = smem_u32(tile);
  return ((addr & 0x3FFFF) >> 4) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor: BF16 x BF16 -> F32, both K-major, M = 128, N = kBN.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kBN >> 3) << 17) |
                            ((uint32_t)(kBM >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a_desc, uint64_t b_desc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(a_desc), "l"(b_desc), "r"(kIdesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const uint32_t a = __bfloat16_as_ushort(__float2bfloat16_rn(lo));
  const uint32_t b = __bfloat16_as_ushort(__float2bfloat16_rn(hi));
  return a | (b << 16);
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Persistent: one CTA per SM walks the output tiles blockIdx.x, + gridDim.x, ...
// (column tiles of a row tile consecutive). Warp 0 streams the tiles' K blocks
// through the shared-memory ring; warp 1 accumulates each tile into one of two
// TMEM accumulators, alternately, and commits it to tfull; warps 2-5 (each
// reading its own quarter of the TMEM lanes) store a finished accumulator as
// BF16 channel pairs and hand it back through tempty, so a tile's epilogue runs
// under the next tile's MMAs. Per output element the products are accumulated
// in the same order as before, so the values are the same.
__global__ void __launch_bounds__(kThreads, 1)
    toeplitz_tc_kernel(const __grid_constant__ CUtensorMap tmA0, const __grid_constant__ CUtensorMap tmA1,
                       const __grid_constant__ CUtensorMap tmA2, const __grid_constant__ CUtensorMap tmT0,
                       const __grid_constant__ CUtensorMap tmT1, const __grid_constant__ CUtensorMap tmT2,
                       uint32_t* __restrict__ out, long long rows, int YL, int n_tiles, int k_blocks,
                       long long n_work, int* __restrict__ err, int stall_kb, uint32_t wait_limit) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* tfull = empty + kStages;  // [2] accumulator b holds a finished tile
  uint64_t* tempty = tfull + 2;       // [2] accumulator b has been read out
  uint64_t* drained = tempty + 2;     // the MMA issuer's own operations have completed (abort path)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drained + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], kEpiWarps);
    }
    mbar_init(drained, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---- producer: TMA loads of every K block of every tile -----------------
    long long last_g[kStages];
    for (int s = 0; s < kStages; ++s) last_g[s] = -1;
    long long g = 0;  // K blocks issued over the CTA's tiles
    bool ok = true;
    for (long long t = blockIdx.x; t < n_work && ok; t += gridDim.x) {
      const int m0 = (int)(t / n_tiles) * kBM, n0 = (int)(t % n_tiles) * kBNOut;
      for (int kb = 0; kb < k_blocks; ++kb, ++g) {
        const int s = (int)(g % kStages);
        if (g >= kStages && !mbar_wait(&empty[s], (uint32_t)((g / kStages) - 1) & 1, err, abort_flag, wait_limit)) {
          ok = false;
          break;
        }
        if (kb == stall_kb) continue;  // test hook: this block's stage is never filled
        last_g[s] = g;
        uint8_t* st = smem + s * kStageBytes;
        mbar_expect_tx(&full[s], kStageBytes);
        tma_load_2d(st, &tmA0, &full[s], kb * kBK, m0);
        tma_load_2d(st + kTileA, &tmA1, &full[s], kb * kBK, m0);
        tma_load_2d(st + 2 * kTileA, &tmA2, &full[s], kb * kBK, m0);
        tma_load_2d(st + 3 * kTileA, &tmT0, &full[s], kb * kBK, n0);
        tma_load_2d(st + 3 * kTileA + kTileB, &tmT1, &full[s], kb * kBK, n0);
        tma_load_2d(st + 3 * kTileA + 2 * kTileB, &tmT2, &full[s], kb * kBK, n0);
      }
    }
    // every issued copy has landed before the CTA can exit (after an abort nobody consumes them)
    for (int s = 0; s < kStages; ++s)
      if (last_g[s] >= 0) mbar_drain(&full[s], (uint32_t)(last_g[s] / kStages) & 1, err, wait_limit);
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer ----------------------------------------------------------
    long long g = 0;
    bool ok = true, issued = false;
    int i = 0;  // tiles of this CTA
    for (long long t = blockIdx.x; t < n_work && ok; t += gridDim.x, ++i) {
      const int b = i & 1;
      if (i >= 2 && !mbar_wait(&tempty[b], (uint32_t)((i >> 1) - 1) & 1, err, abort_flag, wait_limit)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t acc = tmem + (uint32_t)(b * kBN);
      for (int kb = 0; kb < k_blocks; ++kb, ++g) {
        const int s = (int)(g % kStages);
        if (!mbar_wait(&full[s], (uint32_t)(g / kStages) & 1, err, abort_flag, wait_limit)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint8_t* st = smem + s * kStageBytes;
        const uint64_t a0 = umma_desc_sw128(st), a1 = umma_desc_sw128(st + kTileA),
                       a2 = umma_desc_sw128(st + 2 * kTileA);
        const uint64_t t0 = umma_desc_sw128(st + 3 * kTileA), t1 = umma_desc_sw128(st + 3 * kTileA + kTileB),
                       t2 = umma_desc_sw128(st + 3 * kTileA + 2 * kTileB);
#pragma unroll
        for (int kk = 0; kk < kBK / 16; ++kk) {
          const uint64_t step = (uint64_t)(kk * 32) >> 4;  // 16 BF16 = 32 bytes along K
          // smallest terms first, so that they are not absorbed by the large ones
          umma_bf16(acc, a2 + step, t0 + step, (kb | kk) ? 1u : 0u);
          umma_bf16(acc, a1 + step, t1 + step, 1u);
          umma_bf16(acc, a0 + step, t2 + step, 1u);
          umma_bf16(acc, a1 + step, t0 + step, 1u);
          umma_bf16(acc, a0 + step, t1 + step, 1u);
          umma_bf16(acc, a0 + step, t0 + step, 1u);
        }
        umma_commit(&empty[s]);
        issued = true;
      }
      if (ok) umma_commit(&tfull[b]);  // arrives when every MMA of the tile has completed
    }
    // after an abort, the tensor core finishes what was issued before the TMEM is freed
    if (!ok && issued) {
      umma_commit(drained);
      mbar_drain(drained, 0, err, wait_limit);
    }
  } else if (warp >= 2) {
    // ---- epilogue: TMEM -> BF16 channel pairs, tile after tile -----------------
    const int q = warp & 3;  // the TMEM lane quarter this warp may read
    int i = 0;
    for (long long t = blockIdx.x; t < n_work; t += gridDim.x, ++i) {
      const int b = i & 1;
      const bool waited = mbar_wait(&tfull[b], (uint32_t)(i >> 1) & 1, err, abort_flag, wait_limit);
      // tcgen05.ld is warp-collective: the whole warp reads TMEM or none of it does
      if (!__all_sync(0xffffffffu, waited && !*abort_flag)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const long long m0 = (t / n_tiles) * kBM;
      const int n0 = (int)(t % n_tiles) * kBNOut;
      const long long row = m0 + q * 32 + lane;
      const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * kBN);
      float cur[8], nxt[8];
      tmem_ld8(taddr, cur);
      uint32_t* orow = out + row * (long long)YL;
#pragma unroll 1
      for (int c = 0; c < kBNOut / 8; ++c) {
        tmem_ld8(taddr + (uint32_t)((c + 1) * 8), nxt);
        const int j0 = n0 + c * 8;
        if (row < rows) {
          uint32_t w[8];
#pragma unroll
          for (int k = 0; k < 7; ++k) w[k] = pack_bf16x2(cur[k], cur[k + 1]);
          w[7] = pack_bf16x2(cur[7], nxt[0]);
          if (j0 + 8 <= YL && (YL & 3) == 0) {  // row starts are 16-byte aligned only if YL % 4 == 0
            reinterpret_cast<uint4*>(orow + j0)[0] = make_uint4(w[0], w[1], w[2], w[3]);
            reinterpret_cast<uint4*>(orow + j0)[1] = make_uint4(w[4], w[5], w[6], w[7]);
          } else {
            for (int k = 0; k < 8 && j0 + k < YL; ++k) orow[j0 + k] = w[k];
          }
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) cur[k] = nxt[k];
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[b]);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// Preweight + split into K-major BF16 rows. Tile of 64 channels x 32 rows k
// of one view, transposed through shared memory: reads are contiguous along
// k (rebin layout) or j (row layout); each thread writes two adjacent
// channels of a row as one 32-bit word per part (128 bytes per warp). The
// CTA strides over the views (grid z may be smaller than the view count).
template <int IN_LAYOUT>
__global__ void __launch_bounds__(256) prep_split_kernel(__nv_bfloat162* __restrict__ a0,
                                                         __nv_bfloat162* __restrict__ a1,
                                                         __nv_bfloat162* __restrict__ a2,
                                                         const float* __restrict__ in,
                                                         const float2* __restrict__ wt, int YL, int ZL, int KP,
                                                         int nviews, int view0) {
  __shared__ float tile[64][33];  // [j][k]
  const int j0 = blockIdx.x * 64, k0 = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  for (long long v = blockIdx.z; v < nviews; v += gridDim.z) {  // uniform over the CTA
    if (v != blockIdx.z) __syncthreads();                        // the previous view's tile has been read
    if (IN_LAYOUT == HR_LAYOUT_REBIN) {
      for (int yy = ty; yy < 64; yy += 8) {
        const int j = j0 + yy, k = k0 + tx;
        tile[yy][tx] = (j < YL && k < ZL) ? in[((size_t)(view0 + v) * YL + j) * ZL + k] : 0.0f;
      }
    } else {
      for (int yy = ty; yy < 32; yy += 8) {
        const int k = k0 + yy;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int j = j0 + tx + 32 * h;
          tile[tx + 32 * h][yy] = (j < YL && k < ZL) ? in[((size_t)(view0 + v) * ZL + k) * YL + j] : 0.0f;
        }
      }
    }
    __syncthreads();
    for (int yy = ty; yy < 32; yy += 8) {
      const int k = k0 + yy, j = j0 + 2 * tx;
      if (k >= ZL || j >= KP) continue;  // KP is a multiple of 64: j + 1 < KP too
      const float2 w = __ldg(wt + (((size_t)k * KP + j) >> 1));  // the preweights of channels j, j+1 (0 beyond YL)
      float x[2] = {tile[2 * tx][yy] * w.x, tile[2 * tx + 1][yy] * w.y};
      __nv_bfloat16 p0[2], p1[2], p2[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        p0[h] = __float2bfloat16_rn(x[h]);
        const float r1 = x[h] - __bfloat162float(p0[h]);
        p1[h] = __float2bfloat16_rn(r1);
        p2[h] = __float2bfloat16_rn(r1 - __bfloat162float(p1[h]));
      }
      const size_t o = (((size_t)v * ZL + k) * KP + j) >> 1;
      a0[o] = __halves2bfloat162(p0[0], p0[1]);
      a1[o] = __halves2bfloat162(p1[0], p1[1]);
      a2[o] = __halves2bfloat162(p2[0], p2[1]);
    }
  }
}

uint16_t f2bf_host(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

float bf2f_host(uint16_t b) {
  const uint32_t u = (uint32_t)b << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int get_encoder(EncodeTiledFn* fn) {
  static EncodeTiledFn cached = nullptr;
  if (!cached) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    HR_CUDA_TRY(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || p == nullptr)
      return hr::fail(HR_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled is not available");
    cached = reinterpret_cast<EncodeTiledFn>(p);
  }
  *fn = cached;
  return HR_OK;
}

// 2D BF16 tensor [outer][inner] (inner contiguous), box [box_outer][64], 128B swizzle.
int make_map(CUtensorMap* map, const void* base, uint64_t inner, uint64_t outer, uint32_t box_outer) {
  EncodeTiledFn enc;
  HR_TRY(get_encoder(&enc));
  const cuuint64_t dims[2] = {inner, outer};
  const cuuint64_t strides[1] = {inner * 2};
  const cuuint32_t box[2] = {(cuuint32_t)kBK, box_outer};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return hr::fail(HR_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return HR_OK;
}

}  // namespace

struct hr_filter_tc_plan {
  int YL, ZL, ViewN, KP, n_tiles, TR;  // TR: rows of the Toeplitz operand
  float PLC, ZLC, dYL, dZL, SO;
  long long rows;
  __nv_bfloat16* d_a[kParts];
  __nv_bfloat16* d_t[kParts];
  float* d_wt;  // cosine preweights [ZL][KP] (0 for channels >= YL), the reference's float expression
  int* d_err;
  CUtensorMap m_a[kParts], m_t[kParts];
  size_t bytes;
  bool owns_a;  // false: the split parts live in a caller's scratch
  int stall_kb;          // test hook (hr_filter_tc_test_stall): K block never loaded, -1 normally
  uint32_t wait_limit;   // polls before a pipeline wait gives up
};

static void tc_destroy(hr_filter_tc_plan* p) {
  if (!p) return;
  for (int i = 0; i < kParts; ++i) {
    if (p->owns_a) cudaFree(p->d_a[i]);
    cudaFree(p->d_t[i]);
  }
  cudaFree(p->d_wt);
  cudaFree(p->d_err);
  delete p;
}

// ext: three scratch buffers of at least filter_tc_scratch_bytes(YL, ZL, ViewN)
// bytes each for the split parts (shared between plans that run one after the
// other), or nullptr to allocate them in the plan.
static int tc_create(hr_filter_tc_plan** plan, int YL, int ZL, int ViewN, float PLC, float ZLC, float dYL, float dZL,
                     float SO, void* const* ext) {
  HR_REQUIRE(plan != nullptr, "hr_filter_tc_plan_create: plan is NULL");
  *plan = nullptr;
  HR_REQUIRE(YL > 1 && ZL > 0 && ViewN > 0, "tensor-core filter: invalid sizes (YL=%d ZL=%d ViewN=%d)", YL, ZL,
             ViewN);
  HR_REQUIRE(YL <= 4096, "tensor-core filter: YL=%d exceeds 4096", YL);
  HR_REQUIRE(dYL != 0.0f && SO > 0.0f, "tensor-core filter: dYL must be non-zero and SO > 0");
  const long long rows = (long long)ZL * ViewN;
  HR_REQUIRE(rows + kBM < (1LL << 31), "tensor-core filter: %lld rows exceed the TMA coordinate range", rows);
  HR_TRY(hr::require_device());
  int dev = 0, major = 0;
  HR_CUDA_TRY(cudaGetDevice(&dev));
  HR_CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
  HR_REQUIRE(major == 10, "tensor-core filter: needs an sm_100 device (found compute capability %d.x)", major);

  hr_filter_tc_plan* p = new hr_filter_tc_plan{};
  p->YL = YL; p->ZL = ZL; p->ViewN = ViewN; p->PLC = PLC; p->ZLC = ZLC; p->dYL = dYL; p->dZL = dZL; p->SO = SO;
  p->rows = rows;
  p->owns_a = ext == nullptr;
  p->stall_kb = -1;
  p->wait_limit = kWaitLimit;
  p->KP = (YL + kBK - 1) / kBK * kBK;
  p->n_tiles = (YL + kBNOut - 1) / kBNOut;
  p->TR = p->n_tiles * kBNOut + (kBN - kBNOut);
  // Toeplitz operand T[n][k] = h[n-k], n, k < YL, in double, split in three BF16 parts.
  std::vector<uint16_t> tp[kParts];
  for (int i = 0; i < kParts; ++i) tp[i].assign((size_t)p->TR * p->KP, 0);
  const double pi2 = M_PI * M_PI;
  for (int n = 0; n < YL; ++n)
    for (int k = 0; k < YL; ++k) {
      const int d = n - k;
      double r = -2.0 / (pi2 * (4.0 * d * d - 1.0)) / (double)dYL;
      for (int i = 0; i < kParts; ++i) {
        const uint16_t b = f2bf_host((float)r);
        tp[i][(size_t)n * p->KP + k] = b;
        r -= (double)bf2f_host(b);
      }
    }
  const size_t abytes = (size_t)rows * p->KP * 2, tbytes = (size_t)p->TR * p->KP * 2;
  // preweights (src/filtering.cu:187-207, in float as there)
  std::vector<float> wt((size_t)ZL * p->KP, 0.0f);
  const float SO2 = SO * SO;
  for (int k = 0; k < ZL; ++k) {
    const float b = ((float)k - ZLC) * dZL;
    for (int j = 0; j < YL; ++j) {
      const float t = ((float)j - PLC) * dYL;
      wt[(size_t)k * p->KP + j] = SO2 / std::sqrt(SO2 * (SO2 + b * b) - b * t * b * t);
    }
  }
  int st = HR_OK;
  cudaError_t e = cudaMalloc(&p->d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&p->d_wt, sizeof(float) * wt.size());
  if (e == cudaSuccess) e = cudaMemcpy(p->d_wt, wt.data(), sizeof(float) * wt.size(), cudaMemcpyHostToDevice);
  for (int i = 0; i < kParts && e == cudaSuccess; ++i) {
    if (ext)
      p->d_a[i] = static_cast<__nv_bfloat16*>(ext[i]);
    else
      e = cudaMalloc(&p->d_a[i], abytes);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_t[i], tbytes);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_t[i], tp[i].data(), tbytes, cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMemset(p->d_err, 0, sizeof(int));
  if (e != cudaSuccess)
    st = hr::fail(e == cudaErrorMemoryAllocation ? HR_ERR_OUT_OF_MEMORY : HR_ERR_CUDA, "tensor-core filter plan: %s",
                  cudaGetErrorString(e));
  for (int i = 0; i < kParts && st == HR_OK; ++i) {
    st = make_map(&p->m_a[i], p->d_a[i], p->KP, rows, kBM);
    if (st == HR_OK) st = make_map(&p->m_t[i], p->d_t[i], p->KP, p->TR, kBN);
  }
  if (st != HR_OK) {
    tc_destroy(p);
    return st;
  }
  p->bytes = kParts * ((ext ? 0 : abytes) + tbytes) + sizeof(int) + sizeof(float) * wt.size();
  *plan = p;
  return HR_OK;
}

size_t hr::filter_tc_scratch_bytes(int YL, int ZL, int ViewN) {
  return (size_t)ZL * ViewN * ((YL + kBK - 1) / kBK * kBK) * 2;
}

int hr::filter_tc_create_shared(hr_filter_tc_plan** plan, int YL, int ZL, int ViewN, float PLC, float ZLC, float dYL,
                                float dZL, float SO, void* const scratch[3]) {
  HR_REQUIRE(scratch && scratch[0] && scratch[1] && scratch[2], "tensor-core filter: NULL scratch");
  return tc_create(plan, YL, ZL, ViewN, PLC, ZLC, dYL, dZL, SO, scratch);
}

void hr::filter_tc_scratch(const hr_filter_tc_plan* p, void* scratch[3]) {
  for (int i = 0; i < kParts; ++i) scratch[i] = p->d_a[i];
}

extern "C" int hr_filter_tc_plan_create(hr_filter_tc_plan** plan, int YL, int ZL, int ViewN, float PLC, float ZLC,
                                        float dYL, float dZL, float SO) {
  hr::clear_error();
  return tc_create(plan, YL, ZL, ViewN, PLC, ZLC, dYL, dZL, SO, nullptr);
}

int hr::filter_tc_execute_limited(const hr_filter_tc_plan* p, uint32_t* d_pairs, const float* d_in, int in_layout,
                                  int view0, int max_prep_ctas, cudaStream_t s) {
  HR_REQUIRE(p != nullptr && d_pairs != nullptr && d_in != nullptr, "hr_filter_tc_execute: NULL argument");
  HR_REQUIRE(view0 >= 0, "hr_filter_tc_execute: view0 < 0");
  HR_REQUIRE(in_layout == HR_LAYOUT_ROWS || in_layout == HR_LAYOUT_REBIN, "hr_filter_tc_execute: unknown layout %d",
             in_layout);
  HR_REQUIRE(((uintptr_t)d_pairs & 15) == 0, "hr_filter_tc_execute: output must be 16-byte aligned");
  HR_REQUIRE(p->ViewN <= 65535, "hr_filter_tc_execute: %d views exceed one launch (65535)", p->ViewN);
  const int gxy = (p->KP / 64) * ((p->ZL + 31) / 32);
  int gz = p->ViewN;  // the prep kernel strides over the views
  if (max_prep_ctas > 0) gz = std::max(1, std::min(gz, max_prep_ctas / gxy));
  const dim3 pgrid(p->KP / 64, (p->ZL + 31) / 32, gz);
  auto* a0 = reinterpret_cast<__nv_bfloat162*>(p->d_a[0]);
  auto* a1 = reinterpret_cast<__nv_bfloat162*>(p->d_a[1]);
  auto* a2 = reinterpret_cast<__nv_bfloat162*>(p->d_a[2]);
  if (in_layout == HR_LAYOUT_REBIN)
    prep_split_kernel<HR_LAYOUT_REBIN><<<pgrid, 256, 0, s>>>(a0, a1, a2, d_in, reinterpret_cast<const float2*>(p->d_wt),
                                                             p->YL, p->ZL, p->KP, p->ViewN, view0);
  else
    prep_split_kernel<HR_LAYOUT_ROWS><<<pgrid, 256, 0, s>>>(a0, a1, a2, d_in, reinterpret_cast<const float2*>(p->d_wt),
                                                            p->YL, p->ZL, p->KP, p->ViewN, view0);
  HR_CUDA_TRY(cudaGetLastError());
  const size_t smem = (size_t)kStages * kStageBytes + 1024 + 128;
  HR_CUDA_TRY(cudaFuncSetAttribute(toeplitz_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long m_tiles = (p->rows + kBM - 1) / kBM;
  const long long work = m_tiles * p->n_tiles;
  const int grid = (int)std::min<long long>(work, hr::sm_count());  // persistent: one CTA per SM
  toeplitz_tc_kernel<<<grid, kThreads, smem, s>>>(p->m_a[0], p->m_a[1], p->m_a[2], p->m_t[0], p->m_t[1], p->m_t[2],
                                                  d_pairs, p->rows, p->YL, p->n_tiles, p->KP / kBK, work, p->d_err,
                                                  p->stall_kb, p->wait_limit);
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}

extern "C" int hr_filter_tc_execute(const hr_filter_tc_plan* p, uint32_t* d_pairs, const float* d_in, int in_layout,
                                    int view0, void* stream) {
  return hr::filter_tc_execute_limited(p, d_pairs, d_in, in_layout, view0, 0, hr::as_stream(stream));
}

extern "C" int hr_filter_tc_check(const hr_filter_tc_plan* p) {
  HR_REQUIRE(p != nullptr, "hr_filter_tc_check: NULL plan");
  int err = 0;
  HR_CUDA_TRY(cudaMemcpy(&err, p->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    HR_CUDA_TRY(cudaMemset(p->d_err, 0, sizeof(int)));
    return hr::fail(HR_ERR_CUDA, "tensor-core filter: a pipeline wait timed out (kernel aborted its tile)");
  }
  return HR_OK;
}

extern "C" int hr_filter_tc_test_stall(hr_filter_tc_plan* p, int k_block, unsigned int wait_polls) {
  HR_REQUIRE(p != nullptr, "hr_filter_tc_test_stall: NULL plan");
  HR_REQUIRE(k_block < 0 || wait_polls > 0, "hr_filter_tc_test_stall: wait_polls must be positive");
  p->stall_kb = k_block < 0 ? -1 : k_block;
  p->wait_limit = k_block < 0 ? kWaitLimit : (uint32_t)wait_polls;
  return HR_OK;
}

extern "C" size_t hr_filter_tc_device_bytes(const hr_filter_tc_plan* p) { return p ? p->bytes : 0; }

extern "C" void hr_filter_tc_plan_destroy(hr_filter_tc_plan* p) { tc_destroy(p); }
