// Learned artifact correction: a 2.5D residual CNN on reconstructed slices,
// with its own BF16 training and inference kernels.
//
// Network (8 conv layers, 3x3, zero padding, stride 1):
//   input  : 5 adjacent slices of a half-view reconstruction, u = mu / mu_w - 1,
//            NHWC BF16 with the 5 channels padded to 16
//   L1     : 16 -> 32, ReLU;   L2..L7: 32 -> 32, ReLU;   L8: 32 -> 16 (channel 0 used)
//   output : centre slice (FP32, not rounded) + mu_w * L8 channel 0
//
// Convolutions run as implicit GEMMs on the 5th-generation tensor cores: one
// tile is 128 output pixels of one image row (M = 128, TMEM lanes) by COUT
// channels (N), K = 9 taps x CIN channels. A 3 x 130-pixel halo of the input
// is staged in shared memory in the K-major no-swizzle layout (one plane of
// 16-byte pixel chunks per 8-channel group; each plane is one TMA box of 8
// channels x 130 pixels, zero-filled outside the image), so the A operand of
// tap (dy, dx) is the same buffer seen from another 16-byte-aligned start
// address: every input pixel is loaded once per tile and nine descriptor
// offsets replace an im2col copy. The weights (B operand) stay in shared
// memory for the CTA's life. Persistent, warp-specialised CTAs: warp 0 issues
// the TMA loads into a 3-stage halo ring, warp 1 issues the 9*CIN/16
// tcgen05.mma of a tile into one of two TMEM accumulators, warps 2-5 read the
// other accumulator and run the epilogue (bias + ReLU + BF16 store; gradient
// masking by the forward activation; fused residual + loss + output
// gradient), so loads, MMAs and stores of consecutive tiles overlap. Every
// mbarrier wait is bounded and sets an error flag when it gives up. The
// backward data pass is the same kernel with the weights transposed and
// flipped. Weight gradients are a register-tiled FP32 reduction on the CUDA
// cores.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "hr_internal.h"

namespace {

constexpr int kTileM = 128;                  // output pixels per tile (one row segment)
constexpr int kHalo = kTileM + 2;            // halo pixels per row
constexpr int kBox = kHalo * 16;             // bytes of one TMA box: 8 channels x 130 pixels
constexpr int kPlane = 17 * 128;             // plane stride: one box, 128-byte aligned
constexpr int kRing = 6;                     // halo ring: input rows in flight
constexpr int kThreads = 192;                // warp 0 TMA, warp 1 MMA, warps 2-5 epilogue
constexpr int kTmemCols = 64;                // two 32-column accumulators
constexpr uint32_t kWaitLimit = 1u << 22;    // try_wait rounds before a wait is declared hung
constexpr int kLayers = 8;
constexpr int kCin[kLayers] = {16, 32, 32, 32, 32, 32, 32, 32};
constexpr int kCout[kLayers] = {32, 32, 32, 32, 32, 32, 32, 16};

enum Epi { EPI_RELU = 0, EPI_MASK = 1, EPI_LOSS = 2, EPI_RESID = 3 };

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// K-major, no-swizzle UMMA shared-memory descriptor: core matrices of 8 rows x
// 16 bytes (128 contiguous bytes); lbo = bytes between core matrices along K,
// sbo = bytes between 8-row groups along M/N; version 1, layout 0 (none).
__device__ __forceinline__ uint64_t desc_noswz(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr & 0x3FFFF) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
         (1ull << 46);
}

// BF16 x BF16 -> F32, both K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTileM >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

// Bounded wait on an mbarrier phase; gives up (returning false) when another
// role of the CTA has aborted, or after `limit` rounds (then records the
// error and aborts the CTA).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, volatile int* abort_flag, int* err,
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

// Bounded wait for a phase the thread itself started (issued TMA copies, or
// the completion of its own tensor-core operations), ignoring the abort flag:
// an aborting CTA still lets them finish before it frees TMEM and exits.
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

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// 4D tiled TMA load (no multicast): box {8 channels, 130 pixels, 1 row, 1 image}.
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, uint64_t* bar, int c, int x, int y,
                                            int b) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], "
      "[%2];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c), "r"(x), "r"(y), "r"(b)
      : "memory");
}

__device__ __forceinline__ float bf_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf_hi(uint32_t w) { return __uint_as_float(w & 0xffff0000u); }
__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(lo)) |
         ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(hi)) << 16);
}

template <int N>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, float (&v)[N]);

template <>
__device__ __forceinline__ void tmem_ld<16>(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

template <>
__device__ __forceinline__ void tmem_ld<32>(uint32_t taddr, float (&v)[32]) {
  float a[16], b[16];
  tmem_ld<16>(taddr, a);
  tmem_ld<16>(taddr + 16, b);
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    v[i] = a[i];
    v[16 + i] = b[i];
  }
}

struct ConvArgs {
  CUtensorMap in_map;    // the input as a 4D tensor {CIN, W, H, B} of BF16, box {8, 130, 1, 1}
  const uint16_t* in;    // NHWC BF16 [B][H][W][CIN]
  const uint16_t* wimg;  // B operand image [9*CIN/8][COUT][8] BF16
  const float* bias;     // [COUT] (EPI_RELU, EPI_LOSS, EPI_RESID)
  uint16_t* out;         // NHWC BF16 [B][H][W][COUT] (EPI_RELU, EPI_MASK); output gradient (EPI_LOSS)
  const uint16_t* mask;  // NHWC BF16 [B][H][W][COUT]: forward activation whose > 0 passes the gradient (EPI_MASK)
  // residual epilogues: element (b, y, x) of base/target/pred at b*sb + (y*W + x)*sp
  const float* base;
  const float* target;   // EPI_LOSS
  float* pred;           // EPI_RESID output (EPI_LOSS: optional)
  long long sb, sp;
  float scale;           // mu_w: pred = base + scale * r
  float grad_scale;      // EPI_LOSS: d loss / d r = grad_scale * (pred - target) / scale
  float* loss;           // EPI_LOSS: accumulates sum ((pred - target) / scale)^2
  int B, H, W;
  int rows_per_unit;     // output rows a CTA computes down one 128-pixel column strip
  int* err;
  int stall_row;         // test hook: the CTA's input row of this index is never loaded (-1: none)
  uint32_t wait_limit;   // polls before a pipeline wait gives up
};

// Epilogue of one output row segment: the thread's pixel (b, y, x) with its COUT accumulator values.
template <int COUT, int EPI>
__device__ __forceinline__ void conv_epilogue(const ConvArgs& a, const float (&v)[COUT], const float* bias_s, int b,
                                              int y, int x, int lane) {
  const bool valid = x < a.W;
  const size_t pix = ((size_t)b * a.H + y) * a.W + x;
  if constexpr (EPI == EPI_RELU) {
    if (valid) {
      uint4* o = reinterpret_cast<uint4*>(a.out + pix * COUT);
#pragma unroll
      for (int c = 0; c < COUT / 8; ++c) {
        float u[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) u[j] = fmaxf(v[8 * c + j] + bias_s[8 * c + j], 0.0f);
        o[c] = make_uint4(pack2(u[0], u[1]), pack2(u[2], u[3]), pack2(u[4], u[5]), pack2(u[6], u[7]));
      }
    }
  } else if constexpr (EPI == EPI_MASK) {
    if (valid) {
      const uint4* m = reinterpret_cast<const uint4*>(a.mask + pix * COUT);
      uint4* o = reinterpret_cast<uint4*>(a.out + pix * COUT);
#pragma unroll
      for (int c = 0; c < COUT / 8; ++c) {
        const uint4 mv = __ldg(m + c);
        const uint32_t mw[4] = {mv.x, mv.y, mv.z, mv.w};
        float u[8];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          u[2 * j] = bf_lo(mw[j]) > 0.0f ? v[8 * c + 2 * j] : 0.0f;
          u[2 * j + 1] = bf_hi(mw[j]) > 0.0f ? v[8 * c + 2 * j + 1] : 0.0f;
        }
        o[c] = make_uint4(pack2(u[0], u[1]), pack2(u[2], u[3]), pack2(u[4], u[5]), pack2(u[6], u[7]));
      }
    }
  } else {
    const float r = v[0] + bias_s[0];
    float e2 = 0.0f;
    if (valid) {
      const size_t off = (size_t)b * a.sb + ((size_t)y * a.W + x) * a.sp;
      const float pr = a.base[off] + a.scale * r;
      if constexpr (EPI == EPI_RESID) {
        a.pred[off] = pr;
      } else {
        if (a.pred) a.pred[off] = pr;
        const float e = (pr - a.target[off]) / a.scale;
        e2 = e * e;
        uint4* o = reinterpret_cast<uint4*>(a.out + pix * COUT);
        o[0] = make_uint4(pack2(a.grad_scale * e, 0.0f), 0u, 0u, 0u);
#pragma unroll
        for (int c = 1; c < COUT / 8; ++c) o[c] = make_uint4(0u, 0u, 0u, 0u);
      }
    }
    if constexpr (EPI == EPI_LOSS) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) e2 += __shfl_xor_sync(0xffffffffu, e2, o);
      if (lane == 0 && e2 != 0.0f) atomicAdd(a.loss, e2);
    }
  }
}

template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(kThreads) conv_tc_kernel(const __grid_constant__ ConvArgs a) {
  constexpr int G = CIN / 8;                 // 8-channel groups (TMA boxes per input row)
  constexpr int kRow = G * kPlane;           // bytes of one input row (130 pixels)
  constexpr int kWBytes = 9 * CIN * COUT * 2;
  constexpr int kKSteps = 9 * CIN / 16;
  constexpr uint32_t kIdesc = idesc_bf16(COUT);
  constexpr uint32_t kTxBytes = G * kBox;
  static_assert(CIN % 16 == 0 && (COUT == 16 || COUT == 32), "unsupported channel counts");
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  uint8_t* wsm = smem + kRing * kRow;  // weights
  uint64_t* full = reinterpret_cast<uint64_t*>(wsm + kWBytes);
  uint64_t* empty = full + kRing;
  uint64_t* tfull = empty + kRing;
  uint64_t* tempty = tfull + 2;
  uint64_t* mdone = tempty + 2;  // the MMA issuer's last commit (one spare slot keeps 16-byte alignment)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mdone + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  float* bias_s = reinterpret_cast<float*>(tmem_slot + 4);  // 16-byte aligned, COUT floats

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < kWBytes / 16; i += kThreads)
    reinterpret_cast<uint4*>(wsm)[i] = __ldg(reinterpret_cast<const uint4*>(a.wimg) + i);
  if (tid < COUT) bias_s[tid] = a.bias ? __ldg(a.bias + tid) : 0.0f;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (tid == 0) {
    for (int s = 0; s < kRing; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int s = 0; s < 2; ++s) {
      mbar_init(&tfull[s], 1);
      mbar_init(&tempty[s], 128);
    }
    mbar_init(mdone, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t smem_a = smem_u32(smem), w_a = smem_u32(wsm);

  // Work units: (image b, 128-pixel column strip seg, chunk of rows_per_unit output rows). Down a
  // strip each input row is loaded once into the ring and serves three consecutive output rows;
  // a unit of n output rows loads n + 2 input rows (zero rows above and below the image).
  const int nseg = (a.W + kTileM - 1) / kTileM;
  const int rpu = a.rows_per_unit;
  const int nchunk = (a.H + rpu - 1) / rpu;
  const long long units = (long long)a.B * nseg * nchunk;
  if (warp == 0) {
    // ---- producer: input rows of each unit into the ring, G boxes per row --------------------
    if (lane == 0) {
      int h = 0;  // input rows loaded by this CTA
      int last_h[kRing];
      for (int s = 0; s < kRing; ++s) last_h[s] = -1;
      bool ok = true;
      for (long long un = blockIdx.x; un < units && ok; un += gridDim.x) {
        const int seg = (int)(un % nseg), chunk = (int)((un / nseg) % nchunk);
        const int b = (int)(un / ((long long)nseg * nchunk));
        const int y0 = chunk * rpu, ny = min(rpu, a.H - y0);
        for (int j = 0; j < ny + 2; ++j, ++h) {
          const int s = h % kRing;
          if (h >= kRing && !mbar_wait(&empty[s], ((h / kRing) - 1) & 1, abort_flag, a.err, a.wait_limit)) {
            ok = false;
            break;
          }
          if (h == a.stall_row) continue;  // test hook: this row's slot is never filled
          last_h[s] = h;
          mbar_expect_tx(&full[s], kTxBytes);
          for (int g = 0; g < G; ++g)
            tma_load_4d(smem_a + s * kRow + g * kPlane, &a.in_map, &full[s], g * 8, seg * kTileM - 1, y0 - 1 + j, b);
        }
      }
      // every issued copy lands before the CTA exits (after an abort nobody consumes them)
      for (int s = 0; s < kRing; ++s)
        if (last_h[s] >= 0) mbar_drain(&full[s], (last_h[s] / kRing) & 1, a.err, a.wait_limit);
    }
  } else if (warp == 1) {
    // ---- MMA issuer: output row i of a unit reads input rows i, i+1, i+2 of the unit ---------
    if (lane == 0) {
      int hbase = 0, o = 0;
      bool ok = true;
      for (long long un = blockIdx.x; un < units && ok; un += gridDim.x) {
        const int chunk = (int)((un / nseg) % nchunk);
        const int ny = min(rpu, a.H - chunk * rpu);
        for (int i = 0; i < ny && ok; ++i, ++o) {
          for (int j = (i == 0 ? 0 : 2); j < 3 && ok; ++j) {
            const int hh = hbase + i + j;
            ok = mbar_wait(&full[hh % kRing], (hh / kRing) & 1, abort_flag, a.err, a.wait_limit);
          }
          const int acc = o & 1;
          if (ok && o >= 2) ok = mbar_wait(&tempty[acc], ((o >> 1) - 1) & 1, abort_flag, a.err, a.wait_limit);
          if (!ok) break;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
          for (int k = 0; k < kKSteps; ++k) {
            const int k0 = k * 16;
            const int tap = k0 / CIN, c0 = k0 - tap * CIN;
            const int dy = tap / 3, dx = tap - dy * 3;  // input row and pixel offset
            const uint32_t row = smem_a + ((hbase + i + dy) % kRing) * kRow;
            const uint64_t ad = desc_noswz(row + (c0 / 8) * kPlane + dx * 16, kPlane, 128);
            const uint64_t bd = desc_noswz(w_a + (k0 / 8) * (COUT * 16), COUT * 16, 128);
            umma(tmem + acc * 32, ad, bd, kIdesc, k > 0 ? 1u : 0u);
          }
          umma_commit(&tfull[acc]);                       // the accumulator is ready
          umma_commit(&empty[(hbase + i) % kRing]);        // input row i serves no later output row
          if (i == ny - 1) {
            umma_commit(&empty[(hbase + i + 1) % kRing]);  // the unit's last two input rows
            umma_commit(&empty[(hbase + i + 2) % kRing]);
          }
        }
        hbase += ny + 2;
      }
      // every tensor-core operation issued above completes before TMEM is freed
      umma_commit(mdone);
      mbar_drain(mdone, 0, a.err, a.wait_limit);
    }
  } else {
    // ---- epilogue: warps 2-5, TMEM lane quarter warp % 4 --------------------------------------
    const int q = warp & 3;
    int it = 0;
    bool ok = true;
    for (long long un = blockIdx.x; un < units && ok; un += gridDim.x) {
      const int seg = (int)(un % nseg), chunk = (int)((un / nseg) % nchunk);
      const int b = (int)(un / ((long long)nseg * nchunk));
      const int y0 = chunk * rpu, ny = min(rpu, a.H - y0);
      for (int i = 0; i < ny; ++i, ++it) {
        const int acc = it & 1;
        if (!mbar_wait(&tfull[acc], (it >> 1) & 1, abort_flag, a.err, a.wait_limit)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        float v[COUT];
        tmem_ld<COUT>(tmem + acc * 32 + ((uint32_t)(q * 32) << 16), v);
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        mbar_arrive(&tempty[acc]);  // the registers hold the tile: the accumulator may be reused
        conv_epilogue<COUT, EPI>(a, v, bias_s, b, y0 + i, seg * kTileM + q * 32 + lane, lane);
      }
    }
  }
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
}

// Weight gradients on the CUDA cores: dW[co][tap][ci] += sum_p G[p][co] X[p + tap][ci],
// db[co] += sum_p G[p][co]. Thread (cq, ci) owns 4 output channels x 9 taps of one
// input channel (36 accumulators): per pixel 9 + 4 shared-memory reads for 36 FMAs.
template <int CIN, int COUT>
__global__ void __launch_bounds__((COUT / 4) * CIN) wgrad_kernel(const uint16_t* __restrict__ X,
                                                                 const uint16_t* __restrict__ Gr, int B, int H,
                                                                 int W, float* __restrict__ dW,
                                                                 float* __restrict__ db) {
  constexpr int NT = (COUT / 4) * CIN;
  extern __shared__ float wg_smem[];
  float (*xs)[kHalo][CIN] = reinterpret_cast<float (*)[kHalo][CIN]>(wg_smem);          // [3][kHalo][CIN]
  float (*gs)[COUT] = reinterpret_cast<float (*)[COUT]>(wg_smem + 3 * kHalo * CIN);    // [kTileM][COUT]
  const int tid = threadIdx.x;
  const int ci = tid % CIN, cq = tid / CIN;
  float acc[4][9];
  float bacc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 9; ++j) acc[i][j] = 0.0f;
  const int nseg = (W + kTileM - 1) / kTileM;
  const long long tiles = (long long)B * H * nseg;
  for (long long t = blockIdx.x; t < tiles; t += gridDim.x) {
    const int seg = (int)(t % nseg);
    const long long by = t / nseg;
    const int y = (int)(by % H), b = (int)(by / H);
    const int x0 = seg * kTileM;
    __syncthreads();
    for (int i = tid; i < 3 * kHalo * (CIN / 2); i += NT) {
      const int r = i / (kHalo * (CIN / 2)), rem = i - r * (kHalo * (CIN / 2));
      const int pix = rem / (CIN / 2), c2 = rem - pix * (CIN / 2);
      const int yy = y + r - 1, xx = x0 + pix - 1;
      uint32_t w = 0u;
      if (yy >= 0 && yy < H && xx >= 0 && xx < W)
        w = __ldg(reinterpret_cast<const uint32_t*>(X + (((size_t)b * H + yy) * W + xx) * CIN) + c2);
      xs[r][pix][2 * c2] = bf_lo(w);
      xs[r][pix][2 * c2 + 1] = bf_hi(w);
    }
    for (int i = tid; i < kTileM * (COUT / 2); i += NT) {
      const int p = i / (COUT / 2), c2 = i - p * (COUT / 2);
      const int xx = x0 + p;
      uint32_t w = 0u;
      if (xx < W) w = __ldg(reinterpret_cast<const uint32_t*>(Gr + (((size_t)b * H + y) * W + xx) * COUT) + c2);
      gs[p][2 * c2] = bf_lo(w);
      gs[p][2 * c2 + 1] = bf_hi(w);
    }
    __syncthreads();
    for (int p = 0; p < kTileM; ++p) {
      float g[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) g[i] = gs[p][4 * cq + i];
#pragma unroll
      for (int tap = 0; tap < 9; ++tap) {
        const float xv = xs[tap / 3][p + tap % 3][ci];
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[i][tap] = fmaf(g[i], xv, acc[i][tap]);
      }
      if (ci == 0) {
#pragma unroll
        for (int i = 0; i < 4; ++i) bacc[i] += g[i];
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int co = 4 * cq + i;
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) atomicAdd(dW + ((size_t)co * 9 + tap) * CIN + ci, acc[i][tap]);
    if (ci == 0) atomicAdd(db + co, bacc[i]);
  }
}

// Master FP32 weights W[co][tap][ci] -> BF16 operand images:
//   forward  B[n = co][k = tap*CIN + ci]             at [(k/8)][co][k%8]
//   backward B[n = ci][k = tap'*COUT + co] = W[co][8 - tap'][ci]  at [(k/8)][ci][k%8]
__global__ void weight_images_kernel(const float* __restrict__ w, uint16_t* __restrict__ fwd,
                                     uint16_t* __restrict__ bwd, int CIN, int COUT) {
  const int n = 9 * CIN * COUT;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int ci = i % CIN, tap = (i / CIN) % 9, co = i / (9 * CIN);
    const uint16_t v = __bfloat16_as_ushort(__float2bfloat16_rn(w[i]));
    const int kf = tap * CIN + ci;
    fwd[((size_t)(kf / 8) * COUT + co) * 8 + kf % 8] = v;
    if (bwd) {
      const int kb = (8 - tap) * COUT + co;
      bwd[((size_t)(kb / 8) * CIN + ci) * 8 + kb % 8] = v;
    }
  }
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters.
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// Input of the network from a volume [YN][XN][ZN] (z fastest): sample s is
// slice z = z0 + s, channels = slices z-2..z+2 (clamped to the volume), as
// u = mu / mu_w - 1 in BF16, padded to 16 channels.
__global__ void pack_input_kernel(uint16_t* __restrict__ out, const float* __restrict__ vol, int XN, int YN,
                                  int ZN, int z0, int nz, float inv_mu) {
  const long long total = (long long)nz * YN * XN;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long px = i % ((long long)YN * XN);
    const int s = (int)(i / ((long long)YN * XN));
    const int z = z0 + s;
    const float* col = vol + px * ZN;
    uint32_t w[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      float lo = 0.f, hi = 0.f;
      if (2 * c < 5) lo = col[min(max(z + 2 * c - 2, 0), ZN - 1)] * inv_mu - 1.0f;
      if (2 * c + 1 < 5) hi = col[min(max(z + 2 * c - 1, 0), ZN - 1)] * inv_mu - 1.0f;
      w[c] = pack2(lo, hi);
    }
    uint4* o = reinterpret_cast<uint4*>(out + i * 16);
    o[0] = make_uint4(w[0], w[1], w[2], w[3]);
    o[1] = make_uint4(w[4], w[5], w[6], w[7]);
  }
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

// The NHWC BF16 activation [B][H][W][C] as a 4D TMA tensor {C, W, H, B}; box
// {8, 130, 1, 1}; out-of-range elements read as zero (the conv padding).
int make_act_map(CUtensorMap* map, const void* base, int C, int B, int H, int W) {
  EncodeTiledFn enc;
  HR_TRY(get_encoder(&enc));
  HR_REQUIRE(((uintptr_t)base & 15) == 0, "conv: activation must be 16-byte aligned");
  const cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
  const cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
  const cuuint32_t box[4] = {8, (cuuint32_t)kHalo, 1, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return hr::fail(HR_ERR_CUDA, "cuTensorMapEncodeTiled (activation) failed (%d)", (int)r);
  return HR_OK;
}

// Dynamic shared memory of a conv CTA: input-row ring + weights + barriers + alignment slack.
template <int CIN, int COUT>
constexpr size_t conv_smem() {
  return (size_t)kRing * (CIN / 8) * kPlane + 9 * CIN * COUT * 2 + 256 + COUT * 4 + 128;  // barriers fit in 256
}

template <int CIN, int COUT, int EPI>
int launch_conv(ConvArgs& a, cudaStream_t s) {
  const size_t smem = conv_smem<CIN, COUT>();
  HR_TRY(make_act_map(&a.in_map, a.in, CIN, a.B, a.H, a.W));
  HR_CUDA_TRY(cudaFuncSetAttribute(conv_tc_kernel<CIN, COUT, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
  // the largest shared-memory carveout, so that several CTAs (input-row rings) fit on an SM
  HR_CUDA_TRY(cudaFuncSetAttribute(conv_tc_kernel<CIN, COUT, EPI>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   (int)cudaSharedmemCarveoutMaxShared));
  // resident CTAs per SM from the kernel's resources: shared memory (1 KiB reserved per CTA), TMEM
  // columns, registers and threads. CTAs never wait on one another, so a grid larger than what is
  // resident is only queued.
  cudaFuncAttributes fa;
  HR_CUDA_TRY(cudaFuncGetAttributes(&fa, conv_tc_kernel<CIN, COUT, EPI>));
  int dev = 0, smem_sm = 0;
  HR_CUDA_TRY(cudaGetDevice(&dev));
  HR_CUDA_TRY(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
  const int by_smem = smem_sm / (int)(smem + fa.sharedSizeBytes + 1024);
  const int by_tmem = 512 / kTmemCols;
  const int by_regs = 65536 / std::max(1, fa.numRegs * kThreads);
  const int per_sm = std::max(1, std::min({by_smem, by_tmem, by_regs, 2048 / kThreads}));
  const long long ctas = (long long)per_sm * hr::sm_count();
  // rows per unit: about four units per resident CTA (balance), at least 4 rows (each unit reloads 2 rows)
  const long long strips = (long long)a.B * ((a.W + kTileM - 1) / kTileM);
  a.rows_per_unit = (int)std::min<long long>(64, std::max<long long>(4, strips * a.H / (4 * ctas)));
  const long long units = strips * ((a.H + a.rows_per_unit - 1) / a.rows_per_unit);
  const long long grid = std::min<long long>(units, ctas);
  if (grid <= 0) return HR_OK;
  conv_tc_kernel<CIN, COUT, EPI><<<(unsigned)grid, kThreads, smem, s>>>(a);
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}

template <int CIN, int COUT>
int launch_wgrad(const uint16_t* X, const uint16_t* Gr, int B, int H, int W, float* dW, float* db, cudaStream_t s) {
  const long long tiles = (long long)B * H * ((W + kTileM - 1) / kTileM);
  const long long grid = std::min<long long>(tiles, 2LL * hr::sm_count());
  if (grid <= 0) return HR_OK;
  const size_t smem = sizeof(float) * (3 * kHalo * CIN + kTileM * COUT);
  HR_CUDA_TRY(cudaFuncSetAttribute(wgrad_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  HR_CUDA_TRY(cudaFuncSetAttribute(wgrad_kernel<CIN, COUT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   (int)cudaSharedmemCarveoutMaxShared));
  wgrad_kernel<CIN, COUT><<<(unsigned)grid, (COUT / 4) * CIN, smem, s>>>(X, Gr, B, H, W, dW, db);
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}

}  // namespace

struct hr_cnn {
  // parameters: per layer W[co][tap][ci] then b[co], concatenated (FP32 master)
  size_t woff[kLayers], boff[kLayers], nparam = 0;
  float *d_p = nullptr, *d_g = nullptr, *d_m = nullptr, *d_v = nullptr;
  uint16_t *d_wf[kLayers] = {}, *d_wb[kLayers] = {};  // BF16 operand images (forward, backward)
  // activations / gradients for up to cap_pix pixels (B*H*W)
  long long cap_pix = 0;
  uint16_t* d_act[kLayers] = {};  // [0]: input (16 ch), [k]: output of layer k (32 ch), k = 1..7
  uint16_t *d_g0 = nullptr, *d_g1 = nullptr;  // ping-pong gradients (32 ch)
  float* d_loss = nullptr;
  int* d_err = nullptr;
  long long step = 0;
  size_t bytes = 0;
  int stall_row = -1;               // test hook (hr_cnn_test_stall)
  uint32_t wait_limit = kWaitLimit;
};

namespace {

void cnn_free_acts(hr_cnn* n) {
  for (auto& p : n->d_act) {
    cudaFree(p);
    p = nullptr;
  }
  cudaFree(n->d_g0);
  cudaFree(n->d_g1);
  n->d_g0 = n->d_g1 = nullptr;
  n->cap_pix = 0;
}

void cnn_destroy(hr_cnn* n) {
  if (!n) return;
  cnn_free_acts(n);
  cudaFree(n->d_p);
  cudaFree(n->d_g);
  cudaFree(n->d_m);
  cudaFree(n->d_v);
  for (int l = 0; l < kLayers; ++l) {
    cudaFree(n->d_wf[l]);
    cudaFree(n->d_wb[l]);
  }
  cudaFree(n->d_loss);
  cudaFree(n->d_err);
  delete n;
}

int ensure_acts(hr_cnn* n, long long pix) {
  if (pix <= n->cap_pix) return HR_OK;
  cnn_free_acts(n);
  HR_CUDA_TRY(cudaMalloc(&n->d_act[0], (size_t)pix * 16 * 2));
  for (int l = 1; l < kLayers; ++l) HR_CUDA_TRY(cudaMalloc(&n->d_act[l], (size_t)pix * 32 * 2));
  HR_CUDA_TRY(cudaMalloc(&n->d_g0, (size_t)pix * 32 * 2));
  HR_CUDA_TRY(cudaMalloc(&n->d_g1, (size_t)pix * 32 * 2));
  n->cap_pix = pix;
  return HR_OK;
}

int refresh_images(hr_cnn* n, cudaStream_t s) {
  for (int l = 0; l < kLayers; ++l) {
    weight_images_kernel<<<64, 256, 0, s>>>(n->d_p + n->woff[l], n->d_wf[l], n->d_wb[l], kCin[l], kCout[l]);
    HR_CUDA_TRY(cudaGetLastError());
  }
  return HR_OK;
}

ConvArgs base_args(const hr_cnn* n, int B, int H, int W) {
  ConvArgs a{};
  a.B = B;
  a.H = H;
  a.W = W;
  a.err = n->d_err;
  a.stall_row = n->stall_row;
  a.wait_limit = n->wait_limit;
  return a;
}

// Layers 1..7 (ReLU) from d_act[0] into d_act[1..7].
int forward_trunk(hr_cnn* n, int B, int H, int W, cudaStream_t s) {
  for (int l = 0; l < kLayers - 1; ++l) {
    ConvArgs a = base_args(n, B, H, W);
    a.in = n->d_act[l];
    a.wimg = n->d_wf[l];
    a.bias = n->d_p + n->boff[l];
    a.out = n->d_act[l + 1];
    if (l == 0)
      HR_TRY((launch_conv<16, 32, EPI_RELU>(a, s)));
    else
      HR_TRY((launch_conv<32, 32, EPI_RELU>(a, s)));
  }
  return HR_OK;
}

}  // namespace

extern "C" size_t hr_cnn_param_count(void) {
  size_t n = 0;
  for (int l = 0; l < kLayers; ++l) n += (size_t)9 * kCin[l] * kCout[l] + kCout[l];
  return n;
}

extern "C" int hr_cnn_create(hr_cnn** net, const float* h_params) {
  hr::clear_error();
  HR_REQUIRE(net != nullptr && h_params != nullptr, "hr_cnn_create: NULL argument");
  *net = nullptr;
  HR_TRY(hr::require_device());
  int dev = 0, major = 0;
  HR_CUDA_TRY(cudaGetDevice(&dev));
  HR_CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
  HR_REQUIRE(major == 10, "learned correction: needs an sm_100 device (found compute capability %d.x)", major);
  hr_cnn* n = new hr_cnn;
  size_t off = 0;
  for (int l = 0; l < kLayers; ++l) {
    n->woff[l] = off;
    off += (size_t)9 * kCin[l] * kCout[l];
    n->boff[l] = off;
    off += kCout[l];
  }
  n->nparam = off;
  cudaError_t e = cudaSuccess;
  for (float** p : {&n->d_p, &n->d_g, &n->d_m, &n->d_v})
    if (e == cudaSuccess) e = cudaMalloc(p, off * sizeof(float));
  for (int l = 0; l < kLayers && e == cudaSuccess; ++l) {
    e = cudaMalloc(&n->d_wf[l], (size_t)9 * kCin[l] * kCout[l] * 2);
    if (e == cudaSuccess) e = cudaMalloc(&n->d_wb[l], (size_t)9 * kCin[l] * kCout[l] * 2);
  }
  if (e == cudaSuccess) e = cudaMalloc(&n->d_loss, sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&n->d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpy(n->d_p, h_params, off * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(n->d_m, 0, off * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(n->d_v, 0, off * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(n->d_err, 0, sizeof(int));
  int st = e == cudaSuccess ? HR_OK
                            : hr::fail(e == cudaErrorMemoryAllocation ? HR_ERR_OUT_OF_MEMORY : HR_ERR_CUDA,
                                       "hr_cnn_create: %s", cudaGetErrorString(e));
  if (st == HR_OK) st = refresh_images(n, nullptr);
  if (st == HR_OK && cudaStreamSynchronize(nullptr) != cudaSuccess)
    st = hr::fail(HR_ERR_CUDA, "hr_cnn_create: weight preparation failed");
  if (st != HR_OK) {
    cnn_destroy(n);
    return st;
  }
  *net = n;
  return HR_OK;
}

extern "C" int hr_cnn_get_params(const hr_cnn* n, float* h_params) {
  HR_REQUIRE(n != nullptr && h_params != nullptr, "hr_cnn_get_params: NULL argument");
  HR_CUDA_TRY(cudaMemcpy(h_params, n->d_p, n->nparam * sizeof(float), cudaMemcpyDeviceToHost));
  return HR_OK;
}

extern "C" int hr_cnn_get_grads(const hr_cnn* n, float* h_grads) {
  HR_REQUIRE(n != nullptr && h_grads != nullptr, "hr_cnn_get_grads: NULL argument");
  HR_CUDA_TRY(cudaMemcpy(h_grads, n->d_g, n->nparam * sizeof(float), cudaMemcpyDeviceToHost));
  return HR_OK;
}

// Forward + loss + backward (parameter gradients into the plan's gradient
// buffer); lr > 0 then applies one Adam step. d_x: network input NHWC16 BF16
// [B][H][W][16]; d_base/d_target: FP32 [B][H][W] centre slice and reference.
extern "C" int hr_cnn_train_step(hr_cnn* n, const uint16_t* d_x, const float* d_base, const float* d_target, int B,
                                 int H, int W, float mu_w, float lr, float* loss_out, void* stream) {
  HR_REQUIRE(n != nullptr && d_x != nullptr && d_base != nullptr && d_target != nullptr,
             "hr_cnn_train_step: NULL argument");
  HR_REQUIRE(B > 0 && H > 0 && W > 0 && mu_w > 0.0f, "hr_cnn_train_step: invalid sizes");
  HR_REQUIRE(((uintptr_t)d_x & 15) == 0, "hr_cnn_train_step: input must be 16-byte aligned");
  cudaStream_t s = hr::as_stream(stream);
  const long long pix = (long long)B * H * W;
  HR_TRY(ensure_acts(n, pix));
  HR_CUDA_TRY(cudaMemcpyAsync(n->d_act[0], d_x, (size_t)pix * 16 * 2, cudaMemcpyDeviceToDevice, s));
  HR_CUDA_TRY(cudaMemsetAsync(n->d_loss, 0, sizeof(float), s));
  HR_CUDA_TRY(cudaMemsetAsync(n->d_g, 0, n->nparam * sizeof(float), s));
  HR_TRY(forward_trunk(n, B, H, W, s));
  // L8 with the fused residual, loss and output gradient (16 channels, channel 0 used)
  ConvArgs a = base_args(n, B, H, W);
  a.in = n->d_act[7];
  a.wimg = n->d_wf[7];
  a.bias = n->d_p + n->boff[7];
  a.out = n->d_g0;
  a.base = d_base;
  a.target = d_target;
  a.sb = (long long)H * W;
  a.sp = 1;
  a.scale = mu_w;
  a.grad_scale = 2.0f / (float)pix;
  a.loss = n->d_loss;
  HR_TRY((launch_conv<32, 16, EPI_LOSS>(a, s)));
  // backward: G_k (gradient at layer k's output) -> dW_k, and G_{k-1} masked by act_{k-1} > 0
  uint16_t* g = n->d_g0;
  uint16_t* gn = n->d_g1;
  for (int l = kLayers - 1; l >= 0; --l) {
    const int ci = kCin[l], co = kCout[l];
    float* dW = n->d_g + n->woff[l];
    float* db = n->d_g + n->boff[l];
    if (ci == 16)
      HR_TRY((launch_wgrad<16, 32>(n->d_act[l], g, B, H, W, dW, db, s)));
    else if (co == 16)
      HR_TRY((launch_wgrad<32, 16>(n->d_act[l], g, B, H, W, dW, db, s)));
    else
      HR_TRY((launch_wgrad<32, 32>(n->d_act[l], g, B, H, W, dW, db, s)));
    if (l == 0) break;
    ConvArgs b = base_args(n, B, H, W);
    b.in = g;
    b.wimg = n->d_wb[l];
    b.out = gn;
    b.mask = n->d_act[l];
    if (co == 16)
      HR_TRY((launch_conv<16, 32, EPI_MASK>(b, s)));
    else
      HR_TRY((launch_conv<32, 32, EPI_MASK>(b, s)));
    std::swap(g, gn);
  }
  if (lr > 0.0f) {
    ++n->step;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, (float)n->step), c2 = 1.0f - std::pow(b2, (float)n->step);
    adam_kernel<<<128, 256, 0, s>>>(n->d_p, n->d_g, n->d_m, n->d_v, (int)n->nparam, lr, b1, b2, 1e-8f, c1, c2);
    HR_CUDA_TRY(cudaGetLastError());
    HR_TRY(refresh_images(n, s));
  }
  if (loss_out) {
    float l = 0.f;
    HR_CUDA_TRY(cudaMemcpyAsync(&l, n->d_loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    HR_CUDA_TRY(cudaStreamSynchronize(s));
    *loss_out = l / (float)pix;
  }
  return HR_OK;
}

// Inference: out[b][y][x] = base + mu_w * net(x) for a batch of network inputs
// (the same layouts as hr_cnn_train_step; base and out may use any strides).
extern "C" int hr_cnn_forward(hr_cnn* n, float* d_out, const uint16_t* d_x, const float* d_base, long long sb,
                              long long sp, int B, int H, int W, float mu_w, void* stream) {
  HR_REQUIRE(n != nullptr && d_out != nullptr && d_x != nullptr && d_base != nullptr, "hr_cnn_forward: NULL argument");
  HR_REQUIRE(B > 0 && H > 0 && W > 0 && mu_w > 0.0f, "hr_cnn_forward: invalid sizes");
  cudaStream_t s = hr::as_stream(stream);
  const long long pix = (long long)B * H * W;
  HR_TRY(ensure_acts(n, pix));
  if (d_x != n->d_act[0])
    HR_CUDA_TRY(cudaMemcpyAsync(n->d_act[0], d_x, (size_t)pix * 16 * 2, cudaMemcpyDeviceToDevice, s));
  HR_TRY(forward_trunk(n, B, H, W, s));
  ConvArgs a = base_args(n, B, H, W);
  a.in = n->d_act[7];
  a.wimg = n->d_wf[7];
  a.bias = n->d_p + n->boff[7];
  a.base = d_base;
  a.pred = d_out;
  a.sb = sb;
  a.sp = sp;
  a.scale = mu_w;
  return launch_conv<32, 16, EPI_RESID>(a, s);
}

// Corrects a whole reconstructed volume [YN][XN][ZN] (z fastest): every slice
// with its two neighbours on each side (clamped at the ends), chunk slices at
// a time. d_out must not alias d_vol.
extern "C" int hr_cnn_apply_volume(hr_cnn* n, float* d_out, const float* d_vol, int XN, int YN, int ZN, float mu_w,
                                   int chunk, void* stream) {
  HR_REQUIRE(n != nullptr && d_out != nullptr && d_vol != nullptr, "hr_cnn_apply_volume: NULL argument");
  HR_REQUIRE((const void*)d_out != (const void*)d_vol, "hr_cnn_apply_volume: in-place correction is not supported");
  HR_REQUIRE(XN > 0 && YN > 0 && ZN > 0 && chunk > 0 && mu_w > 0.0f, "hr_cnn_apply_volume: invalid sizes");
  cudaStream_t s = hr::as_stream(stream);
  HR_TRY(ensure_acts(n, (long long)std::min(chunk, ZN) * XN * YN));
  for (int z0 = 0; z0 < ZN; z0 += chunk) {
    const int nz = std::min(chunk, ZN - z0);
    pack_input_kernel<<<8 * hr::sm_count(), 256, 0, s>>>(n->d_act[0], d_vol, XN, YN, ZN, z0, nz, 1.0f / mu_w);
    HR_CUDA_TRY(cudaGetLastError());
    HR_TRY(hr_cnn_forward(n, d_out + z0, n->d_act[0], d_vol + z0, 1, ZN, nz, YN, XN, mu_w, stream));
  }
  return HR_OK;
}

// The network input for slices [z0, z0 + nz) of a volume (for training data).
extern "C" int hr_cnn_pack_input(uint16_t* d_x, const float* d_vol, int XN, int YN, int ZN, int z0, int nz, float mu_w,
                                 void* stream) {
  HR_REQUIRE(d_x != nullptr && d_vol != nullptr, "hr_cnn_pack_input: NULL argument");
  HR_REQUIRE(XN > 0 && YN > 0 && ZN > 0 && nz > 0 && z0 >= 0 && z0 + nz <= ZN && mu_w > 0.0f,
             "hr_cnn_pack_input: invalid sizes");
  pack_input_kernel<<<8 * hr::sm_count(), 256, 0, hr::as_stream(stream)>>>(d_x, d_vol, XN, YN, ZN, z0, nz,
                                                                          1.0f / mu_w);
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}

extern "C" int hr_cnn_check(const hr_cnn* n) {
  HR_REQUIRE(n != nullptr, "hr_cnn_check: NULL network");
  int err = 0;
  HR_CUDA_TRY(cudaMemcpy(&err, n->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    HR_CUDA_TRY(cudaMemset(n->d_err, 0, sizeof(int)));
    return hr::fail(HR_ERR_CUDA, "learned correction: a tensor-core wait timed out (kernel aborted)");
  }
  return HR_OK;
}

extern "C" int hr_cnn_test_stall(hr_cnn* n, int row, unsigned int wait_polls) {
  HR_REQUIRE(n != nullptr, "hr_cnn_test_stall: NULL network");
  HR_REQUIRE(row < 0 || wait_polls > 0, "hr_cnn_test_stall: wait_polls must be positive");
  n->stall_row = row < 0 ? -1 : row;
  n->wait_limit = row < 0 ? kWaitLimit : (uint32_t)wait_polls;
  return HR_OK;
}

extern "C" void hr_cnn_destroy(hr_cnn* n) { cnn_destroy(n); }
