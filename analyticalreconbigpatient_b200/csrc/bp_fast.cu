// 3D-weighted helical backprojection, fast form (BF16 filtered data).
//
// Same algorithm as the plain form (src/Parallel_FDK_Helical_3DWeighting.cpp:
// 42-113, views s1..s2), rearranged so that a voxel-view update costs one FMA
// for the detector row, two 32-bit gathers, one FMA and one SFU reciprocal
// for the weight:
//
//   weight = w1 Gc^k1 / (w2 G^k1 + w1 Gc^k1) = 1 / (1 + 2^Q 2^C)
//   Q(view, slice) = k1 (log2|t2| - log2|t2 -/+ 0.5|) + log2(w2/w1)
//   C(column, view) = k1 log2((temp1 - UU)/(temp1 + UU))
//
// with t2 = z - h View/2pi. t2 and 2^Q depend only on (view, slice): they are
// evaluated once per plan in FP64 (the helical source position accumulates
// over ~1e4-1e5 views) and stored per z block as a float2 table (2^Q is 0 or
// +inf where a view weight w is 0, which gives the weights 1 and 0); a CTA covers
// one z block, so every thread of a CTA reads the same table entry (broadcast)
// and a per-(block, view) bit mask tells which of its slices have the view in
// their [s1, s2] window. Everything per (column, view) -- UU, Yr,
// temp1 = sqrt(SO^2 - Yr^2), the projection slope K = SO SD/(temp1 (temp1+UU)
// dZL), 2^C, the channel -- is FP32, computed once and reused for the NZ slices.
//
// Filtered data are BF16 "pairs": word u of a detector row holds the values of
// channels u (low half) and u+1 (high half), so one 32-bit load gives both
// horizontal taps of a row. The bilinear tap uses floor instead of the
// reference's ceil; both give the same interpolated value away from exact
// integers, where the blend is continuous. The texture variants (further
// down) copy the pairs' low halves into layered FP16 or FP32 textures and let
// the texture units do the bilinear tap.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "hr_internal.h"
#include "bp_fast.h"

namespace {

constexpr int kBx = 8, kBy = 32;  // CTA tile (x, y): 8 warps of 8 x 4 columns
constexpr double kTwoPiTrunc = 2.0 * 3.14159265358979;
constexpr double kInvTwoPi = 1.0 / (2.0 * 3.141592653589793);
constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23: adding it rounds to an integer
constexpr float kFarT2 = 1e30f;         // table t2 of a slice that does not have the view

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float lg2_approx(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// floor(x) for |x| < 2^22 without a conversion instruction: returns the
// integer and writes the float value.
__device__ __forceinline__ int floor_magic(float x, float& fl) {
  const float r = (x - 0.49999997f) + kMagic;  // round-to-nearest of x - 1/2
  fl = r - kMagic;
  return __float_as_int(r) - 0x4B400000;
}

struct FastParams {
  int XN, YN, ZN, YL, ZL, PN;
  float XNC, YNC, dx, dy, SO2, SOSDdZL, invdYL, YLC0, ZLC0, k1, DeltaFai;
};

// ---- packed FP32x2 arithmetic (sm_100: one instruction for two lanes) ----
__device__ __forceinline__ uint64_t pk2(float a, float b) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void up2(uint64_t r, float& a, float& b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r));
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

// Per (column, view) quantities shared by the slices of a thread.
struct ColView {
  float K, E, fu;  // E = 2^C
  int u0;
  uint64_t fu2;    // (fu, fu) for packed row blends
};

template <class PT>
__device__ __forceinline__ bool col_view(const PT& P, float x, float y, float2 cs, ColView& cv) {
  const float UU = -x * cs.x - y * cs.y;
  const float Yr = -x * cs.y + y * cs.x;
  const float t1sq = P.SO2 - Yr * Yr;
  const float temp1 = t1sq * rsqrtf(t1sq);
  const float A = temp1 + UU, B = temp1 - UU;
  cv.K = P.SOSDdZL * rcp_approx(temp1 * A);
  cv.E = ex2_approx(P.k1 * lg2_approx(B * rcp_approx(A)));
  const float u1 = fmaf(Yr, P.invdYL, P.YLC0);
  float u0f;
  cv.u0 = floor_magic(u1, u0f);
  cv.fu = u1 - u0f;
  cv.fu2 = pk2(cv.fu, cv.fu);
  return (unsigned)cv.u0 <= (unsigned)(P.YL - 2);
}

// Bilinear tap from two BF16 channel pairs (rows V0 and V0+1): the two row
// blends run as one packed FP32x2 FMA (lane-wise the same roundings as two
// scalar FMAs).
__device__ __forceinline__ float blend(uint32_t w0, uint32_t w1, uint64_t fu2, float fz) {
  const uint64_t lo = pk2(__uint_as_float(w0 << 16), __uint_as_float(w1 << 16));                  // taps u
  const uint64_t hi = pk2(__uint_as_float(w0 & 0xffff0000u), __uint_as_float(w1 & 0xffff0000u));  // taps u+1
  float ra, rb;
  up2(fma2(fu2, sub2(hi, lo), lo), ra, rb);
  return fmaf(fz, rb - ra, ra);
}

// NZ slices per thread; CH == 0: slices one after the other (branch per
// slice); CH > 0: chunks of CH slices whose row positions are computed first,
// whose 2*CH gathers are then issued together (addresses clamped into the
// detector, out-of-detector or out-of-window slices weighted by 0), and only
// then consumed -- more loads in flight per warp at the cost of registers.
// Per-scan table pointers of the fast backprojection.
struct ZTabs {
  const float2* trig;     // per view: {cos, sin}
  const float2* ztab;     // per z block and view of its window: NZ x {t2, 2^Q}
  const uint32_t* zmask;  // per z block and view: slices whose window holds the view
  const int2* zblock;     // per z block: {first view, number of views}
  const int* zoff;        // per z block: table row of its first view
  const int4* seg;        // per z block: view segments of the segmented texture variants
};

template <int NZ, int CH, class PT>
__device__ __forceinline__ void fast_column(float* __restrict__ vol, const uint32_t* __restrict__ fpb,
                                            const ZTabs& T, const PT& P, int xi, int yi, int b) {
  const float2* __restrict__ trig = T.trig;
  const float2* __restrict__ ztab = T.ztab;
  const uint32_t* __restrict__ zmask = T.zmask;
  const int z0 = b * NZ;
  const int2 blk = T.zblock[b];  // {first view, number of views} of the block's union window
  const int off = T.zoff[b];     // row of the block's first view in the table
  const float x = ((float)xi - P.XNC) * P.dx;
  const float y = ((float)yi - P.YNC) * P.dy;
  float res[NZ];
#pragma unroll
  for (int m = 0; m < NZ; ++m) res[m] = 0.0f;
  const int pYL = P.YL, pZL = P.ZL;  // per-update constants, kept in registers
  const float pZLC0 = P.ZLC0;
  const size_t plane = (size_t)pZL * pYL;
  const float2* btab = ztab + (size_t)off * NZ;
  const uint32_t* bmask = zmask + off;
  for (int q = 0; q < blk.y; ++q) {
    const uint32_t mask = __ldg(bmask + q);
    if (mask == 0u) continue;
    const int p = blk.x + q;
    ColView cv;
    if (!col_view(P, x, y, __ldg(trig + p), cv)) continue;
    const uint32_t* col = fpb + (size_t)p * plane + cv.u0;
    const float2* e = btab + (size_t)q * NZ;
    if constexpr (CH == 0) {
#pragma unroll
      for (int m = 0; m < NZ; ++m) {
        if (!(mask & (1u << m))) continue;
        const float2 tq = __ldg(e + m);  // {t2, 2^Q}
        float v0f;
        const float v1 = fmaf(tq.x, cv.K, pZLC0);
        const int v0 = floor_magic(v1, v0f);
        if ((unsigned)v0 > (unsigned)(pZL - 2)) continue;
        const uint32_t w0 = __ldg(col + (size_t)v0 * pYL);
        const uint32_t w1 = __ldg(col + (size_t)(v0 + 1) * pYL);
        const float wgt = rcp_approx(fmaf(tq.y, cv.E, 1.0f));
        res[m] = fmaf(wgt, blend(w0, w1, cv.fu2, v1 - v0f), res[m]);
      }
    } else {
      const float4* e4 = reinterpret_cast<const float4*>(e);
#pragma unroll
      for (int c = 0; c < NZ / CH; ++c) {
        const uint32_t cm = (mask >> (c * CH)) & ((1u << CH) - 1u);
        if (cm == 0u) continue;  // uniform over the CTA
        float t2[CH], qv[CH], fz[CH];
        int vrow[CH];
        bool ok[CH];
#pragma unroll
        for (int i = 0; i < CH; i += 2) {
          const float4 t = __ldg(e4 + (c * CH + i) / 2);  // {t2, 2^Q} of two slices
          t2[i] = t.x; qv[i] = t.y; t2[i + 1] = t.z; qv[i + 1] = t.w;
        }
#pragma unroll
        for (int i = 0; i < CH; ++i) {
          float v0f;
          const float v1 = fmaf(t2[i], cv.K, pZLC0);
          const int v0 = floor_magic(v1, v0f);
          ok[i] = ((cm >> i) & 1u) && (unsigned)v0 <= (unsigned)(pZL - 2);
          vrow[i] = ok[i] ? v0 : 0;
          fz[i] = v1 - v0f;
        }
        uint32_t w0[CH], w1[CH];
#pragma unroll
        for (int i = 0; i < CH; ++i) {
          w0[i] = __ldg(col + (size_t)vrow[i] * pYL);
          w1[i] = __ldg(col + (size_t)(vrow[i] + 1) * pYL);
        }
#pragma unroll
        for (int i = 0; i < CH; ++i) {
          const float wgt = ok[i] ? rcp_approx(fmaf(qv[i], cv.E, 1.0f)) : 0.0f;
          res[c * CH + i] = fmaf(wgt, blend(w0[i], w1[i], cv.fu2, fz[i]), res[c * CH + i]);
        }
      }
    }
  }
  float* out = vol + ((size_t)yi * P.XN + xi) * P.ZN + z0;
#pragma unroll
  for (int m = 0; m < NZ; ++m)
    if (z0 + m < P.ZN) out[m] = res[m] * P.DeltaFai;
}


// Two slices per instruction: slices (2c, 2c+1) of the thread share packed
// registers through the row position, the bilinear blend, the weight and the
// accumulation; the two table entries come in one 128-bit load and the
// window test is one uniform branch per pair. Same operations per (voxel,
// view) as bp_fast_kernel, in the same view order.
template <int NZ, class PT>
__device__ __forceinline__ void fast_column_pairs(float* __restrict__ vol, const uint32_t* __restrict__ fpb,
                                                  const ZTabs& T, const PT& P, int xi, int yi, int b) {
  static_assert(NZ % 2 == 0, "slices are processed in pairs");
  const float2* __restrict__ trig = T.trig;
  const float2* __restrict__ ztab = T.ztab;
  const uint32_t* __restrict__ zmask = T.zmask;
  const int z0 = b * NZ;
  const int2 blk = T.zblock[b];
  const int off = T.zoff[b];
  const float x = ((float)xi - P.XNC) * P.dx;
  const float y = ((float)yi - P.YNC) * P.dy;
  uint64_t res[NZ / 2];
#pragma unroll
  for (int c = 0; c < NZ / 2; ++c) res[c] = 0ull;
  const int pYL = P.YL;
  const size_t plane = (size_t)P.ZL * pYL;
  const float4* btab = reinterpret_cast<const float4*>(ztab + (size_t)off * NZ);
  const uint32_t* bmask = zmask + off;
  const uint64_t half2 = pk2(-0.49999997f, -0.49999997f), magic2 = pk2(kMagic, kMagic);
  const uint64_t one2 = pk2(1.0f, 1.0f);
  const uint64_t zlc2 = pk2(P.ZLC0, P.ZLC0);
  const unsigned vmax = (unsigned)(P.ZL - 2);
  for (int q = 0; q < blk.y; ++q) {
    const uint32_t mask = __ldg(bmask + q);
    if (mask == 0u) continue;
    const int p = blk.x + q;
    ColView cv;
    if (!col_view(P, x, y, __ldg(trig + p), cv)) continue;
    const uint32_t* col = fpb + (size_t)p * plane + cv.u0;
    const float4* e = btab + (size_t)q * (NZ / 2);
    const uint64_t k2 = pk2(cv.K, cv.K), e2 = pk2(cv.E, cv.E), fu2 = pk2(cv.fu, cv.fu);
#pragma unroll
    for (int c = 0; c < NZ / 2; ++c) {
      const uint32_t pm = (mask >> (2 * c)) & 3u;
      if (pm == 0u) continue;  // uniform over the CTA
      const float4 t = __ldg(e + c);  // {t2, 2^Q} of slices 2c and 2c+1
      const uint64_t v1 = fma2(pk2(t.x, t.z), k2, zlc2);
      const uint64_t r = add2(add2(v1, half2), magic2);  // round(v1 - 1/2) in the low mantissa bits
      const uint64_t v0f = sub2(r, magic2);
      const uint64_t fz = sub2(v1, v0f);
      float ra_, rb_;
      up2(r, ra_, rb_);
      const int va = __float_as_int(ra_) - 0x4B400000, vb = __float_as_int(rb_) - 0x4B400000;
      const bool oka = (pm & 1u) && (unsigned)va <= vmax;
      const bool okb = (pm & 2u) && (unsigned)vb <= vmax;
      const uint32_t* ca = col + (size_t)(oka ? va : 0) * pYL;
      const uint32_t* cb = col + (size_t)(okb ? vb : 0) * pYL;
      const uint32_t wa0 = __ldg(ca), wa1 = __ldg(ca + pYL);
      const uint32_t wb0 = __ldg(cb), wb1 = __ldg(cb + pYL);
      // (slice a, slice b) lanes: row V0 taps u, u+1 and row V0+1 taps u, u+1
      const uint64_t r0u0 = pk2(__uint_as_float(wa0 << 16), __uint_as_float(wb0 << 16));
      const uint64_t r0u1 = pk2(__uint_as_float(wa0 & 0xffff0000u), __uint_as_float(wb0 & 0xffff0000u));
      const uint64_t r1u0 = pk2(__uint_as_float(wa1 << 16), __uint_as_float(wb1 << 16));
      const uint64_t r1u1 = pk2(__uint_as_float(wa1 & 0xffff0000u), __uint_as_float(wb1 & 0xffff0000u));
      const uint64_t ra = fma2(fu2, sub2(r0u1, r0u0), r0u0);
      const uint64_t rb = fma2(fu2, sub2(r1u1, r1u0), r1u0);
      const uint64_t tap = fma2(fz, sub2(rb, ra), ra);
      float sa, sb;
      up2(fma2(pk2(t.y, t.w), e2, one2), sa, sb);
      const uint64_t wgt = pk2(oka ? rcp_approx(sa) : 0.0f, okb ? rcp_approx(sb) : 0.0f);
      res[c] = fma2(wgt, tap, res[c]);
    }
  }
  float* out = vol + ((size_t)yi * P.XN + xi) * P.ZN + z0;
#pragma unroll
  for (int c = 0; c < NZ / 2; ++c) {
    float a, bb;
    up2(res[c], a, bb);
    if (z0 + 2 * c < P.ZN) out[2 * c] = a * P.DeltaFai;
    if (z0 + 2 * c + 1 < P.ZN) out[2 * c + 1] = bb * P.DeltaFai;
  }
}

// CH >= 0: fast_column<NZ, CH>; CH < 0: slice pairs in packed FP32x2.
template <int NZ, int CH, class PT = FastParams>
__device__ __forceinline__ void column(float* vol, const uint32_t* fpb, const ZTabs& T, const PT& P, int xi, int yi,
                                       int b) {
  if constexpr (CH < 0)
    fast_column_pairs<NZ, PT>(vol, fpb, T, P, xi, yi, b);
  else
    fast_column<NZ, CH, PT>(vol, fpb, T, P, xi, yi, b);
}

// One CTA per (8 x 16 column tile, z block); grid z covers z blocks
// [b_first, b_first + gridDim.z).
template <int NZ, int CH>
__global__ void __launch_bounds__(kBx* kBy) bp_fast_kernel(float* __restrict__ vol, const uint32_t* __restrict__ fpb,
                                                          const ZTabs T, const FastParams P, int b_first) {
  const int xi = blockIdx.x * kBx + threadIdx.x;
  const int yi = blockIdx.y * kBy + threadIdx.y;
  if (xi >= P.XN || yi >= P.YN) return;
  column<NZ, CH>(vol, fpb, T, P, xi, yi, b_first + blockIdx.z);
}

// Several scans of uneven size in one persistent launch. Work items are
// (scan, z block, column tile), numbered scan by scan with the column tile
// fastest; each CTA claims the next item from a global counter when it
// finishes one, so the items in flight stay a narrow window of the order (a
// few z blocks, whose views stay in L2), as under the hardware block
// scheduler; a static round robin lets CTAs drift apart and spreads the
// window over many z blocks. Each scan keeps the slices per thread its own
// geometry favours (16, 8 or 4: a uniform branch per item).
// Per-scan texture handles of the texture variants.
struct TexRef {
  const unsigned long long* texs;  // texture object of each array of 2^lsh views
  const float* scale;              // {1 / FP16 scale, ...}
  int lsh;
};

struct BatchScan {
  FastParams P;
  ZTabs T;
  TexRef X;
  float* vol;
  const uint32_t* fpb;
  int tiles_x, tiles_y, item0, nz;
};
struct BatchParams {
  BatchScan s[hr::kBatchMaxScans];
  int n;
  int begin, count;  // items [begin, begin + count)
  int grid;          // CTAs launched
  int* counter;      // zero at launch
};

// MB: CTAs per SM the register allocation must allow (1: no constraint);
// CH: gathers of CH slices issued together (0: one slice at a time).
template <int MB, int CH>
__global__ void __launch_bounds__(kBx* kBy, MB) bp_fast_batch_kernel(const __grid_constant__ BatchParams B) {
  __shared__ int s_item;
  const bool leader = threadIdx.x == 0 && threadIdx.y == 0;
  for (;;) {
    if (leader) s_item = atomicAdd(B.counter, 1);
    __syncthreads();
    const int k = s_item;
    __syncthreads();
    if (k >= B.count) break;
    const int item = B.begin + k;
    int sc = 0;
    while (sc + 1 < B.n && item >= B.s[sc + 1].item0) ++sc;
    const BatchScan& S = B.s[sc];
    const int local = item - S.item0;
    const int t = local / S.tiles_x;
    const int xi = (local - t * S.tiles_x) * kBx + threadIdx.x;
    const int yi = (t % S.tiles_y) * kBy + threadIdx.y;
    const int b = t / S.tiles_y;
    if (xi < S.P.XN && yi < S.P.YN) {
      if (S.nz == 16)
        column<16, CH>(S.vol, S.fpb, S.T, S.P, xi, yi, b);
      else if (S.nz == 8)
        column<8, CH>(S.vol, S.fpb, S.T, S.P, xi, yi, b);
      else
        column<4, CH>(S.vol, S.fpb, S.T, S.P, xi, yi, b);
    }
  }
}

// ---- texture variants ----
// The filtered data as layered 2D textures (one layer per view), sampled with
// the texture units' bilinear filtering at (u1 + 1/2, V + 1/2): one TEX per
// update replaces the two gathers, the BF16 unpacking and the three blends.
// The hardware blends with 1.8 fixed-point weights, so a tap differs from the
// FP32 blend by up to 1/256 of the neighbour difference (the fast form's
// accuracy budget covers it). Taps come from the low halves of the BF16 pairs:
// the same sample values as the gather variants wherever FP16 holds the BF16
// value exactly. The scale puts the largest |value| in [2^14, 2^15), and FP16
// (subnormals included) represents a BF16 value exactly down to 2^-17, i.e.
// over 2^31 below the largest |value|; smaller values are rounded to FP16's
// 2^-24 step (an absolute error of at most 2^-39 of the largest |value|).

// Largest |value| of the filtered data (bits of a non-negative float order
// like unsigned integers), for the FP16 scale.
__global__ void tex_absmax_kernel(float* __restrict__ scale, const uint32_t* __restrict__ fpb, long long n) {
  unsigned m = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    m = max(m, (__ldg(fpb + i) << 16) & 0x7fffffffu);
  m = __reduce_max_sync(0xffffffffu, m);
  if ((threadIdx.x & 31) == 0 && m) atomicMax(reinterpret_cast<unsigned*>(scale + 1), m);
}

// BF16 pairs [views][ZL][YL] -> the layered arrays, rows [r0, r1) (rows =
// views x ZL; one CTA row at a time). FP16 (MODE 0): scaled by 2^k with the
// largest |value| in [2^14, 2^15); scale[0] = 2^-k, which the backprojection
// folds into its output. Views filled range by range while the fan data is
// still arriving (a streamed execution) cannot know the largest |value| of the
// scan: the first range (MODE 1) puts its own largest |value| in [2^10, 2^11)
// and keeps the factor in scale[2]; later ranges (MODE 2) reuse it, and
// scale[3] = 1 records that the running largest |value| (scale[1]) no longer
// fits below FP16's largest finite value, or that the first range was all
// zeros, so that the caller refills the whole copy with MODE 0. Any power of
// two that keeps the values in FP16's normal range gives the same samples up
// to that power.
constexpr int kStreamHeadroom = 4;  // binades between the first range's largest |value| and MODE 0's range
template <bool HALF, int MODE>
__global__ void tex_fill_kernel(float* __restrict__ scale, const unsigned long long* __restrict__ surfs,
                                const uint32_t* __restrict__ fpb, long long r0, long long r1, int ZL, int YL,
                                int lsh) {
  float sc = 1.0f;
  if constexpr (HALF && MODE == 2) {
    sc = scale[2];
    if (blockIdx.x == 0 && threadIdx.x == 0 && !(scale[1] * sc < 65504.0f)) scale[3] = 1.0f;
  } else if constexpr (HALF) {
    const int e = (int)(__float_as_uint(scale[1]) >> 23) - 127;  // max |value| < 2^(e+1)
    const int k = min(max(127 + 14 - (MODE == 1 ? kStreamHeadroom : 0) - e, 1), 253);  // biased exponent of the factor
    sc = __int_as_float(k << 23);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      scale[0] = __int_as_float((254 - k) << 23);
      if (MODE == 1) {
        scale[2] = sc;
        scale[3] = scale[1] == 0.0f ? 1.0f : 0.0f;
      }
    }
  } else {
    if (blockIdx.x == 0 && threadIdx.x == 0) scale[0] = 1.0f;
  }
  const int lmask = (1 << lsh) - 1;
  if (HALF && (YL & 3) == 0 && (reinterpret_cast<uintptr_t>(fpb) & 15) == 0) {
    // four channels per thread: one 16-byte load of their pairs (rows start 16-byte aligned), one 8-byte
    // (four-texel) surface store
    const int G = YL >> 2;
    const long long n = (r1 - r0) * G;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
      const long long r = r0 + i / G;
      const int g = (int)(i - (r - r0) * G);
      const int p = (int)(r / ZL), v = (int)(r - (long long)p * ZL);
      const uint4 w = __ldg(reinterpret_cast<const uint4*>(fpb + r * YL) + g);
      const __half2 h01 = __floats2half2_rn(__uint_as_float(w.x << 16) * sc, __uint_as_float(w.y << 16) * sc);
      const __half2 h23 = __floats2half2_rn(__uint_as_float(w.z << 16) * sc, __uint_as_float(w.w << 16) * sc);
      const uint2 out = make_uint2(*reinterpret_cast<const uint32_t*>(&h01), *reinterpret_cast<const uint32_t*>(&h23));
      surf2DLayeredwrite(out, surfs[p >> lsh], g * 8, v, p & lmask, cudaBoundaryModeZero);
    }
    return;
  }
  for (long long r = r0 + blockIdx.x; r < r1; r += gridDim.x) {
    const int p = (int)(r / ZL), v = (int)(r - (long long)p * ZL);
    const cudaSurfaceObject_t so = surfs[p >> lsh];
    const uint32_t* row = fpb + r * YL;
    for (int u = threadIdx.x; u < YL; u += blockDim.x) {
      const float val = __uint_as_float(__ldg(row + u) << 16);
      if constexpr (HALF)
        surf2DLayeredwrite(__half_as_ushort(__float2half_rn(val * sc)), so, u * 2, v, p & lmask, cudaBoundaryModeZero);
      else
        surf2DLayeredwrite(val, so, u * 4, v, p & lmask, cudaBoundaryModeZero);
    }
  }
}

// Same tables, window masks and weight as fast_column; the tap is a texture
// sample. The NZ samples of a (column, view) are issued before any is used.
template <int NZ>
__device__ __forceinline__ void tex_column(float* __restrict__ vol, const TexRef& X, const ZTabs& T,
                                           const FastParams& P, int xi, int yi, int b) {
  static_assert(NZ % 2 == 0, "table entries are read two slices at a time");
  const unsigned long long* __restrict__ texs = X.texs;
  const int lsh = X.lsh;
  const int z0 = b * NZ;
  const int2 blk = T.zblock[b];
  const int off = T.zoff[b];
  const float x = ((float)xi - P.XNC) * P.dx;
  const float y = ((float)yi - P.YNC) * P.dy;
  float res[NZ];
#pragma unroll
  for (int m = 0; m < NZ; ++m) res[m] = 0.0f;
  const float4* btab = reinterpret_cast<const float4*>(T.ztab + (size_t)off * NZ);
  const uint32_t* bmask = T.zmask + off;
  const float utop = (float)(P.YL - 1), vtop = (float)P.ZL - 0.5f;
  const float zlch = P.ZLC0 + 0.5f;
  const int lmask = (1 << lsh) - 1;
  for (int q = 0; q < blk.y; ++q) {
    const uint32_t mask = __ldg(bmask + q);
    if (mask == 0u) continue;
    const int p = blk.x + q;
    const float2 cs = __ldg(T.trig + p);
    const float UU = -x * cs.x - y * cs.y;
    const float Yr = -x * cs.y + y * cs.x;
    const float u1 = fmaf(Yr, P.invdYL, P.YLC0);
    if (!(u1 >= 0.0f && u1 < utop)) continue;  // floor(u1) in [0, YL-2]
    const float t1sq = P.SO2 - Yr * Yr;
    const float temp1 = t1sq * rsqrtf(t1sq);
    const float A = temp1 + UU, B = temp1 - UU;
    const float K = P.SOSDdZL * rcp_approx(temp1 * A);
    const float E = ex2_approx(P.k1 * lg2_approx(B * rcp_approx(A)));
    const cudaTextureObject_t tx = __ldg(texs + (p >> lsh));
    const int layer = p & lmask;
    const float xt = u1 + 0.5f;
    const float4* e = btab + (size_t)q * (NZ / 2);
    float tap[NZ], qv[NZ];
#pragma unroll
    for (int c = 0; c < NZ / 2; ++c) {
      const float4 t = __ldg(e + c);  // {t2, 2^Q} of slices 2c and 2c+1
      qv[2 * c] = t.y;
      qv[2 * c + 1] = t.w;
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int m = 2 * c + i;
        const float vh = fmaf(i ? t.z : t.x, K, zlch);  // row position + 1/2
        const bool ok = vh >= 0.5f && vh < vtop;  // floor in [0, ZL-2]; false for slices without the view
        tap[m] = ok ? tex2DLayered<float>(tx, xt, vh, layer) : 0.0f;
      }
    }
#pragma unroll
    for (int m = 0; m < NZ; ++m) res[m] = fmaf(rcp_approx(fmaf(qv[m], E, 1.0f)), tap[m], res[m]);
  }
  const float outs = P.DeltaFai * __ldg(X.scale);
  float* out = vol + ((size_t)yi * P.XN + xi) * P.ZN + z0;
#pragma unroll
  for (int m = 0; m < NZ; ++m)
    if (z0 + m < P.ZN) out[m] = res[m] * outs;
}

template <int NZ>
__global__ void __launch_bounds__(kBx* kBy) bp_tex_kernel(float* __restrict__ vol, const TexRef X, const ZTabs T,
                                                         const FastParams P, int b_first) {
  const int xi = blockIdx.x * kBx + threadIdx.x;
  const int yi = blockIdx.y * kBy + threadIdx.y;
  if (xi >= P.XN || yi >= P.YN) return;
  tex_column<NZ>(vol, X, T, P, xi, yi, b_first + blockIdx.z);
}

// ---- segmented texture variants ----
// A z block's union window, cut into segments over which the slices holding
// the view are a fixed range [MA, MB] (the table's view masks, built on the
// host): slices entering at the start of the window and leaving at its end
// cost nothing outside their own windows. Per slice the views are visited in
// the same order with the same operations as tex_column (a slice without the
// view added exactly 0 there), so both give the same bits.
struct SegCtx {
  const float2* trig;
  const float4* btab;  // the block's first table row, two slices per float4
  const unsigned long long* texs;
  float x, y, utop, vtop, zlch;
  int blk0, lsh, lmask;
};

template <int NZ, int MA, int MB>
__device__ __forceinline__ void tex_range(float (&res)[NZ], const SegCtx& c, const FastParams& P, int q0, int q1) {
#pragma unroll 1
  for (int q = q0; q < q1; ++q) {
    const int p = c.blk0 + q;
    const float2 cs = __ldg(c.trig + p);
    const float UU = -c.x * cs.x - c.y * cs.y;
    const float Yr = -c.x * cs.y + c.y * cs.x;
    const float u1 = fmaf(Yr, P.invdYL, P.YLC0);
    if (!(u1 >= 0.0f && u1 < c.utop)) continue;  // floor(u1) in [0, YL-2]
    const float t1sq = P.SO2 - Yr * Yr;
    const float temp1 = t1sq * rsqrtf(t1sq);
    const float A = temp1 + UU, B = temp1 - UU;
    const float K = P.SOSDdZL * rcp_approx(temp1 * A);
    const float E = ex2_approx(P.k1 * lg2_approx(B * rcp_approx(A)));
    const cudaTextureObject_t tx = __ldg(c.texs + (p >> c.lsh));
    const int layer = p & c.lmask;
    const float xt = u1 + 0.5f;
    const float4* e = c.btab + (size_t)q * (NZ / 2);
    float tap[NZ], qv[NZ];
#pragma unroll
    for (int cc = MA / 2; cc <= MB / 2; ++cc) {
      const float4 t = __ldg(e + cc);  // {t2, 2^Q} of slices 2cc and 2cc+1
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int m = 2 * cc + i;
        if (m < MA || m > MB) continue;
        qv[m] = i ? t.w : t.y;
        const float vh = fmaf(i ? t.z : t.x, K, c.zlch);  // row position + 1/2
        const bool ok = vh >= 0.5f && vh < c.vtop;
        tap[m] = ok ? tex2DLayered<float>(tx, xt, vh, layer) : 0.0f;
      }
    }
#pragma unroll
    for (int m = MA; m <= MB; ++m) res[m] = fmaf(rcp_approx(fmaf(qv[m], E, 1.0f)), tap[m], res[m]);
  }
}

// Two views per iteration. With thick slices few slices share a view, and one
// view's few taps in flight per warp leave the texture units waiting on
// latency; here both views' taps are issued before either is used. Each
// slice still accumulates view q before view q+1 with the same operations as
// tex_range, so the bits are the same. A view whose column misses the
// detector is skipped as there (its per-view values are not used).
template <int NZ, int MA, int MB>
__device__ __forceinline__ void tex_range2(float (&res)[NZ], const SegCtx& c, const FastParams& P, int q0, int q1) {
  int q = q0;
#pragma unroll 1
  for (; q + 1 < q1; q += 2) {
    float tap[2][NZ], qv[2][NZ], E[2];
    bool onv[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int p = c.blk0 + q + h;
      const float2 cs = __ldg(c.trig + p);
      const float UU = -c.x * cs.x - c.y * cs.y;
      const float Yr = -c.x * cs.y + c.y * cs.x;
      const float u1 = fmaf(Yr, P.invdYL, P.YLC0);
      onv[h] = u1 >= 0.0f && u1 < c.utop;  // floor(u1) in [0, YL-2]
      const float t1sq = P.SO2 - Yr * Yr;
      const float temp1 = t1sq * rsqrtf(t1sq);
      const float A = temp1 + UU, B = temp1 - UU;
      const float K = P.SOSDdZL * rcp_approx(temp1 * A);
      E[h] = ex2_approx(P.k1 * lg2_approx(B * rcp_approx(A)));
      const cudaTextureObject_t tx = __ldg(c.texs + (p >> c.lsh));
      const int layer = p & c.lmask;
      const float xt = u1 + 0.5f;
      const float4* e = c.btab + (size_t)(q + h) * (NZ / 2);
#pragma unroll
      for (int cc = MA / 2; cc <= MB / 2; ++cc) {
        const float4 t = __ldg(e + cc);
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int m = 2 * cc + i;
          if (m < MA || m > MB) continue;
          qv[h][m] = i ? t.w : t.y;
          const float vh = fmaf(i ? t.z : t.x, K, c.zlch);
          const bool ok = onv[h] && vh >= 0.5f && vh < c.vtop;
          tap[h][m] = ok ? tex2DLayered<float>(tx, xt, vh, layer) : 0.0f;
        }
      }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h)
      if (onv[h]) {
#pragma unroll
        for (int m = MA; m <= MB; ++m) res[m] = fmaf(rcp_approx(fmaf(qv[h][m], E[h], 1.0f)), tap[h][m], res[m]);
      }
  }
  if (q < q1) tex_range<NZ, MA, MB>(res, c, P, q, q1);  // an odd last view
}

// Widest slice range the two-view loop runs (wider ranges: one view at a
// time, whose taps already fill the texture pipe).
constexpr int kTwoViewMaxRange = 4;

// Runs segment sg = {q0, q1, ma, mb} with the code specialised for its range
// (V = 2: two views per iteration for ranges of at most kTwoViewMaxRange slices).
template <int NZ, int V, int MA, int MB>
__device__ __forceinline__ void tex_dispatch(float (&res)[NZ], const SegCtx& c, const FastParams& P, int4 sg) {
  if (sg.z == MA && sg.w == MB) {
    if constexpr (V == 2 && MB - MA + 1 <= kTwoViewMaxRange)
      tex_range2<NZ, MA, MB>(res, c, P, sg.x, sg.y);
    else
      tex_range<NZ, MA, MB>(res, c, P, sg.x, sg.y);
    return;
  }
  if constexpr (MB + 1 < NZ)
    tex_dispatch<NZ, V, MA, MB + 1>(res, c, P, sg);
  else if constexpr (MA + 1 < NZ)
    tex_dispatch<NZ, V, MA + 1, MA + 1>(res, c, P, sg);
}

// One column of z block b with the segmented view loop (segments in T.seg).
template <int NZ, int V = 1>
__device__ __forceinline__ void tex_seg_column(float* __restrict__ vol, const TexRef& X, const ZTabs& T,
                                               const FastParams& P, int xi, int yi, int b) {
  static_assert(NZ % 2 == 0, "table entries are read two slices at a time");
  const int z0 = b * NZ;
  SegCtx c;
  c.trig = T.trig;
  c.btab = reinterpret_cast<const float4*>(T.ztab + (size_t)T.zoff[b] * NZ);
  c.texs = X.texs;
  c.x = ((float)xi - P.XNC) * P.dx;
  c.y = ((float)yi - P.YNC) * P.dy;
  c.utop = (float)(P.YL - 1);
  c.vtop = (float)P.ZL - 0.5f;
  c.zlch = P.ZLC0 + 0.5f;
  c.blk0 = T.zblock[b].x;
  c.lsh = X.lsh;
  c.lmask = (1 << X.lsh) - 1;
  float res[NZ];
#pragma unroll
  for (int m = 0; m < NZ; ++m) res[m] = 0.0f;
  const int4* sb = T.seg + (size_t)b * (hr::kSegPerNz * NZ);
#pragma unroll 1
  for (int sgi = 0; sgi < hr::kSegPerNz * NZ; ++sgi) {
    const int4 sg = __ldg(sb + sgi);
    if (sg.x >= sg.y) continue;  // unused entry (uniform over the CTA)
    tex_dispatch<NZ, V, 0, 0>(res, c, P, sg);
  }
  const float outs = P.DeltaFai * __ldg(X.scale);
  float* out = vol + ((size_t)yi * P.XN + xi) * P.ZN + z0;
#pragma unroll
  for (int m = 0; m < NZ; ++m)
    if (z0 + m < P.ZN) out[m] = res[m] * outs;
}

template <int NZ, int V>
__global__ void __launch_bounds__(kBx* kBy) bp_tex_seg_kernel(float* __restrict__ vol, const TexRef X, const ZTabs T,
                                                             const FastParams P, int b_first) {
  const int xi = blockIdx.x * kBx + threadIdx.x;
  const int yi = blockIdx.y * kBy + threadIdx.y;
  if (xi >= P.XN || yi >= P.YN) return;
  tex_seg_column<NZ, V>(vol, X, T, P, xi, yi, b_first + blockIdx.z);
}

// The same column code with registers bounded for 6 CTAs of 256 threads per
// SM (40 registers instead of 48: one CTA more per SM to hide the texture
// latency).
template <int NZ, int V>
__global__ void __launch_bounds__(kBx* kBy, 6) bp_tex_seg6_kernel(float* __restrict__ vol, const TexRef X,
                                                                 const ZTabs T, const FastParams P, int b_first) {
  const int xi = blockIdx.x * kBx + threadIdx.x;
  const int yi = blockIdx.y * kBy + threadIdx.y;
  if (xi >= P.XN || yi >= P.YN) return;
  tex_seg_column<NZ, V>(vol, X, T, P, xi, yi, b_first + blockIdx.z);
}

// The persistent multi-scan launch with texture taps: the work items and
// their claiming as in bp_fast_batch_kernel; each scan samples its own arrays
// with 8 or 4 slices per thread (NZF = 0: the scan's own choice) or 4 for all
// scans (NZF = 4: the smaller body leaves registers for the scan parameters,
// which a dynamic scan index keeps out of the constant-operand path).
template <int MB, int NZF>
__global__ void __launch_bounds__(kBx* kBy, MB) bp_tex_batch_kernel(const __grid_constant__ BatchParams B) {
  __shared__ int s_item;
  const bool leader = threadIdx.x == 0 && threadIdx.y == 0;
  for (;;) {
    if (leader) s_item = atomicAdd(B.counter, 1);
    __syncthreads();
    const int k = s_item;
    __syncthreads();
    if (k >= B.count) break;
    const int item = B.begin + k;
    int sc = 0;
    while (sc + 1 < B.n && item >= B.s[sc + 1].item0) ++sc;
    const BatchScan& S = B.s[sc];
    const int local = item - S.item0;
    const int t = local / S.tiles_x;
    const int xi = (local - t * S.tiles_x) * kBx + threadIdx.x;
    const int yi = (t % S.tiles_y) * kBy + threadIdx.y;
    const int b = t / S.tiles_y;
    if (xi < S.P.XN && yi < S.P.YN) {
      if (NZF == 0 && S.nz == 8)
        tex_column<8>(S.vol, S.X, S.T, S.P, xi, yi, b);
      else
        tex_column<4>(S.vol, S.X, S.T, S.P, xi, yi, b);
    }
  }
}

// The persistent multi-scan launch with texture taps and code specialised per
// scan: the work item's scan index selects, by a chain of uniform branches,
// a copy of the column code that reads scan K's descriptor at a constant
// index, so its constants stay constant-bank operands as in the single-scan
// kernel instead of occupying registers for the whole launch.
template <int NZF, int K>
__device__ __forceinline__ void tex_item_spec(const BatchParams& B, int sc, int local) {
  if (sc == K) {
    const BatchScan& S = B.s[K];
    const int t = local / S.tiles_x;
    const int xi = (local - t * S.tiles_x) * kBx + threadIdx.x;
    const int yi = (t % S.tiles_y) * kBy + threadIdx.y;
    const int b = t / S.tiles_y;
    if (xi < S.P.XN && yi < S.P.YN) {
      if (NZF == 0 && S.nz == 8)
        tex_column<8>(S.vol, S.X, S.T, S.P, xi, yi, b);
      else
        tex_column<NZF == 0 ? 4 : NZF>(S.vol, S.X, S.T, S.P, xi, yi, b);
    }
    return;
  }
  if constexpr (K + 1 < hr::kBatchMaxScans) tex_item_spec<NZF, K + 1>(B, sc, local);
}

template <int MB, int NZF>
__global__ void __launch_bounds__(kBx* kBy, MB) bp_tex_batch_spec_kernel(const __grid_constant__ BatchParams B) {
  __shared__ int s_item;
  const bool leader = threadIdx.x == 0 && threadIdx.y == 0;
  for (;;) {
    if (leader) s_item = atomicAdd(B.counter, 1);
    __syncthreads();
    const int k = s_item;
    __syncthreads();
    if (k >= B.count) break;
    const int item = B.begin + k;
    int sc = 0;
    while (sc + 1 < B.n && item >= B.s[sc + 1].item0) ++sc;
    tex_item_spec<NZF, 0>(B, sc, item - B.s[sc].item0);
  }
}

// The persistent multi-scan launch with the segmented texture column code:
// work items and their claiming as in bp_tex_batch_kernel; each scan runs the
// segmented loop over its own view segments with its own slices per thread
// (8 or 4).
template <int MB>
__global__ void __launch_bounds__(kBx* kBy, MB) bp_tex_seg_batch_kernel(const __grid_constant__ BatchParams B) {
  __shared__ int s_item;
  const bool leader = threadIdx.x == 0 && threadIdx.y == 0;
  for (;;) {
    if (leader) s_item = atomicAdd(B.counter, 1);
    __syncthreads();
    const int k = s_item;
    __syncthreads();
    if (k >= B.count) break;
    const int item = B.begin + k;
    int sc = 0;
    while (sc + 1 < B.n && item >= B.s[sc + 1].item0) ++sc;
    const BatchScan& S = B.s[sc];
    const int local = item - S.item0;
    const int t = local / S.tiles_x;
    const int xi = (local - t * S.tiles_x) * kBx + threadIdx.x;
    const int yi = (t % S.tiles_y) * kBy + threadIdx.y;
    const int b = t / S.tiles_y;
    if (xi < S.P.XN && yi < S.P.YN) {
      if (S.nz == 8)
        tex_seg_column<8>(S.vol, S.X, S.T, S.P, xi, yi, b);
      else
        tex_seg_column<4>(S.vol, S.X, S.T, S.P, xi, yi, b);
    }
  }
}

// fp32 [n][YL] rows -> BF16 pairs (u, u+1), round to nearest even.
__global__ void pack_pairs_kernel(uint32_t* __restrict__ out, const float* __restrict__ in, long long rows, int YL) {
  const long long total = rows * YL;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long r = i / YL;
    const int u = (int)(i - r * YL);
    const float a = in[i];
    const float b = u + 1 < YL ? in[i + 1] : 0.0f;
    const uint32_t lo = __bfloat16_as_ushort(__float2bfloat16_rn(a));
    const uint32_t hi = __bfloat16_as_ushort(__float2bfloat16_rn(b));
    out[i] = lo | (hi << 16);
  }
}

}  // namespace

namespace hr {

// Host-side table build for NZ slices per thread, FP64 (the reference's view
// angle, source height and window rules, ..._3DWeighting.cpp:61-75, 79, 95-102).
static int build_host(BpFastHostSet* t, int NZ, const BpFastGeom& g, const double* w) {
  const int nblocks = (g.ZN + NZ - 1) / NZ;
  std::vector<int> s0(g.ZN), lo(g.ZN), hi(g.ZN);
  std::vector<double> zc(g.ZN);
  for (int zi = 0; zi < g.ZN; ++zi) {
    const double z = (zi - g.ZNC) * g.dz;
    zc[zi] = z;
    const double beta0 = kTwoPiTrunc * z / g.h;
    s0[zi] = (int)std::ceil((beta0 - g.BetaS) / g.DeltaFai - 0.5);
    const int s1 = s0[zi] - g.half, s2 = s0[zi] + g.half;
    if (zi < g.ZN_valid && s1 < g.PN && s2 > 0) {
      lo[zi] = s1 < 0 ? 0 : s1;
      hi[zi] = s2 > g.PN - 1 ? g.PN - 1 : s2;
    } else {
      lo[zi] = 1;
      hi[zi] = 0;
    }
  }
  t->nz = NZ;
  t->nblocks = nblocks;
  t->zb.assign(3 * nblocks, 0);
  size_t total = 0;
  for (int b = 0; b < nblocks; ++b) {
    int a = 0x7fffffff, e = -1;
    for (int m = 0; m < NZ; ++m) {
      const int zi = b * NZ + m;
      if (zi < g.ZN && lo[zi] <= hi[zi]) {
        a = std::min(a, lo[zi]);
        e = std::max(e, hi[zi]);
      }
    }
    if (e < a) {
      a = 0;
      e = -1;
    }
    t->zb[2 * b] = a;                    // first view of the block's union window
    t->zb[2 * b + 1] = e - a + 1;        // its number of views
    t->zb[2 * nblocks + b] = (int)total;  // table row of its first view
    total += (size_t)(e - a + 1);
  }
  HR_REQUIRE(total < (1ull << 31) / NZ, "fast backprojection: z-block table too large");
  // slices without the view: t2 far outside any detector (the texture variants'
  // row test rejects them without the mask; finite, so masked-out blends of the
  // gather variants stay finite before their zero weight)
  t->tab.assign(total * NZ, make_float2(kFarT2, 0.f));
  t->mask.assign(total, 0u);
  for (int b = 0; b < nblocks; ++b) {
    for (int q = 0; q < t->zb[2 * b + 1]; ++q) {
      const int p = t->zb[2 * b] + q;
      const double View = g.BetaS + p * g.DeltaFai;
      const double hv = g.h * View * kInvTwoPi;
      uint32_t mk = 0;
      const size_t row = (size_t)t->zb[2 * nblocks + b] + q;
      for (int m = 0; m < NZ; ++m) {
        const int zi = b * NZ + m;
        if (zi >= g.ZN || p < lo[zi] || p > hi[zi]) continue;
        const double t2 = zc[zi] - hv;
        const int d1 = (int)(g.N_pi - (double)(s0[zi] - p));
        const int d2 = p < s0[zi] ? (int)(d1 + g.N_pi) : (int)(d1 - g.N_pi);
        const double tc = p < s0[zi] ? t2 - 0.5 : t2 + 0.5;
        double Q = g.k1 * (std::log2(std::fabs(t2)) - std::log2(std::fabs(tc)));
        Q += std::log2(w[d2]) - std::log2(w[d1]);
        t->tab[row * NZ + m] = make_float2((float)t2, (float)std::exp2(Q));
        mk |= 1u << m;
      }
      t->mask[row] = mk;
    }
  }
  // view segments of each block for the segmented variants: runs of views
  // with the same active range [lowest, highest slice of the mask]; views no
  // slice needs are dropped; a block whose runs exceed the capacity keeps one
  // segment over its whole window (slices without a view sample nothing)
  const int cap = kSegPerNz * NZ;
  t->seg.assign((size_t)nblocks * cap, make_int4(0, 0, 0, 0));
  std::vector<int4> sv;
  for (int b = 0; b < nblocks; ++b) {
    sv.clear();
    const size_t r0 = (size_t)t->zb[2 * nblocks + b];
    for (int q = 0; q < t->zb[2 * b + 1]; ++q) {
      const uint32_t mk = t->mask[r0 + q];
      if (mk == 0u) continue;
      const int ma = __builtin_ctz(mk), mb = 31 - __builtin_clz(mk);
      if (!sv.empty() && sv.back().y == q && sv.back().z == ma && sv.back().w == mb)
        sv.back().y = q + 1;
      else
        sv.push_back(make_int4(q, q + 1, ma, mb));
    }
    if ((int)sv.size() > cap) {
      int4 all = make_int4(sv.front().x, sv.back().y, NZ, -1);
      for (const int4& g : sv) {
        all.z = std::min(all.z, g.z);
        all.w = std::max(all.w, g.w);
      }
      sv.assign(1, all);
    }
    std::copy(sv.begin(), sv.end(), t->seg.begin() + (size_t)b * cap);
  }
  return HR_OK;
}

int bp_fast_host_tables(BpFastHost* h, const BpFastGeom& g, const double* w) {
  for (int i = 0; i < kFastTableSets; ++i) HR_TRY(build_host(&h->set[i], kFastNz[i], g, w));
  h->trig.resize(g.PN);
  for (int p = 0; p < g.PN; ++p) {
    const double View = g.BetaS + p * g.DeltaFai;
    h->trig[p] = make_float2((float)std::cos(View), (float)std::sin(View));
  }
  return HR_OK;
}

int bp_fast_reserve(BpFast* f, const size_t rows[kFastTableSets], const int nblocks[kFastTableSets], int PN) {
  f->bytes = 0;
  for (int i = 0; i < kFastTableSets; ++i) {
    BpFastTables& t = f->t[i];
    t.nz = kFastNz[i];
    t.nblocks = nblocks[i];
    t.cap_rows = std::max<size_t>(rows[i], 1);
    HR_CUDA_TRY(cudaMalloc(&t.d_tab, sizeof(float2) * t.cap_rows * t.nz));
    HR_CUDA_TRY(cudaMalloc(&t.d_mask, sizeof(uint32_t) * t.cap_rows));
    HR_CUDA_TRY(cudaMalloc(&t.d_zblock, sizeof(int) * 3 * (size_t)t.nblocks));
    HR_CUDA_TRY(cudaMalloc(&t.d_seg, sizeof(int4) * kSegPerNz * t.nz * (size_t)t.nblocks));
    t.bytes = (sizeof(float2) * t.nz + sizeof(uint32_t)) * t.cap_rows + sizeof(int) * 3 * (size_t)t.nblocks +
              sizeof(int4) * kSegPerNz * t.nz * (size_t)t.nblocks;
    f->bytes += t.bytes;
  }
  f->cap_views = PN;
  HR_CUDA_TRY(cudaMalloc(&f->d_trig, sizeof(float2) * (size_t)PN));
  f->bytes += sizeof(float2) * (size_t)PN;
  return HR_OK;
}

int bp_fast_upload(BpFast* f, const BpFastHost& h, cudaStream_t s) {
  for (int i = 0; i < kFastTableSets; ++i) {
    BpFastTables& t = f->t[i];
    const BpFastHostSet& ht = h.set[i];
    HR_REQUIRE(ht.nblocks == t.nblocks && ht.mask.size() <= t.cap_rows,
               "fast backprojection: tables exceed the reserved capacity");
    HR_CUDA_TRY(cudaMemcpyAsync(t.d_tab, ht.tab.data(), sizeof(float2) * ht.tab.size(), cudaMemcpyHostToDevice, s));
    HR_CUDA_TRY(cudaMemcpyAsync(t.d_mask, ht.mask.data(), sizeof(uint32_t) * ht.mask.size(), cudaMemcpyHostToDevice,
                                s));
    HR_CUDA_TRY(cudaMemcpyAsync(t.d_zblock, ht.zb.data(), sizeof(int) * ht.zb.size(), cudaMemcpyHostToDevice, s));
    HR_CUDA_TRY(cudaMemcpyAsync(t.d_seg, ht.seg.data(), sizeof(int4) * ht.seg.size(), cudaMemcpyHostToDevice, s));
    t.h_zb.assign(ht.zb.begin(), ht.zb.begin() + 2 * (size_t)ht.nblocks);
  }
  HR_REQUIRE(h.trig.size() <= (size_t)f->cap_views, "fast backprojection: more views than reserved");
  HR_CUDA_TRY(cudaMemcpyAsync(f->d_trig, h.trig.data(), sizeof(float2) * h.trig.size(), cudaMemcpyHostToDevice, s));
  return HR_OK;
}

int bp_fast_create(BpFast* f, const BpFastGeom& g, const double* w) {
  BpFastHost h;
  HR_TRY(bp_fast_host_tables(&h, g, w));
  size_t rows[kFastTableSets];
  int nb[kFastTableSets];
  for (int i = 0; i < kFastTableSets; ++i) {
    rows[i] = h.set[i].mask.size();
    nb[i] = h.set[i].nblocks;
  }
  HR_TRY(bp_fast_reserve(f, rows, nb, g.PN));
  HR_TRY(bp_fast_upload(f, h, nullptr));
  HR_CUDA_TRY(cudaStreamSynchronize(nullptr));
  f->variant = kFastDefaultVariant;
  return HR_OK;
}

static void tex_free(BpFastTex* t) {
  for (unsigned long long o : t->tex) cudaDestroyTextureObject(o);
  for (unsigned long long o : t->surf) cudaDestroySurfaceObject(o);
  for (cudaArray_t a : t->arr) cudaFreeArray(a);
  cudaFree(t->d_obj);
  cudaFree(t->d_scale);
  *t = BpFastTex{};
}

static int tex_alloc_arrays(BpFastTex* t, int kind, int YL, int ZL, int views) {
  int dev = 0, mw = 0, mh = 0, ml = 0;
  HR_CUDA_TRY(cudaGetDevice(&dev));
  HR_CUDA_TRY(cudaDeviceGetAttribute(&mw, cudaDevAttrMaxSurface2DLayeredWidth, dev));
  HR_CUDA_TRY(cudaDeviceGetAttribute(&mh, cudaDevAttrMaxSurface2DLayeredHeight, dev));
  HR_CUDA_TRY(cudaDeviceGetAttribute(&ml, cudaDevAttrMaxSurface2DLayeredLayers, dev));
  int tw = 0, th = 0, tl = 0;
  HR_CUDA_TRY(cudaDeviceGetAttribute(&tw, cudaDevAttrMaxTexture2DLayeredWidth, dev));
  HR_CUDA_TRY(cudaDeviceGetAttribute(&th, cudaDevAttrMaxTexture2DLayeredHeight, dev));
  HR_CUDA_TRY(cudaDeviceGetAttribute(&tl, cudaDevAttrMaxTexture2DLayeredLayers, dev));
  const int esz = kind == kTexHalf ? 2 : 4;
  HR_REQUIRE(YL * esz <= mw && YL <= tw && ZL <= std::min(mh, th) && std::min(ml, tl) >= 2,
             "fast backprojection: %d x %d detector rows exceed the layered texture limits", ZL, YL);
  t->kind = kind;
  t->YL = YL;
  t->ZL = ZL;
  t->views = views;
  t->lsh = 0;
  while ((2 << t->lsh) <= std::min(std::min(ml, tl), 2048)) ++t->lsh;
  const int L = 1 << t->lsh;
  t->n = (views + L - 1) / L;
  const cudaChannelFormatDesc desc = kind == kTexHalf ? cudaCreateChannelDescHalf() : cudaCreateChannelDesc<float>();
  for (int i = 0; i < t->n; ++i) {
    const int layers = std::min(L, views - i * L);
    cudaArray_t a = nullptr;
    HR_CUDA_TRY(cudaMalloc3DArray(&a, &desc, make_cudaExtent(YL, ZL, layers),
                                  cudaArrayLayered | cudaArraySurfaceLoadStore));
    t->arr.push_back(a);
    cudaResourceDesc rd{};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = a;
    cudaTextureDesc td{};
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    cudaTextureObject_t to = 0;
    HR_CUDA_TRY(cudaCreateTextureObject(&to, &rd, &td, nullptr));
    t->tex.push_back(to);
    cudaSurfaceObject_t so = 0;
    HR_CUDA_TRY(cudaCreateSurfaceObject(&so, &rd));
    t->surf.push_back(so);
  }
  std::vector<unsigned long long> obj(t->tex);
  obj.insert(obj.end(), t->surf.begin(), t->surf.end());
  HR_CUDA_TRY(cudaMalloc(&t->d_obj, sizeof(unsigned long long) * obj.size()));
  HR_CUDA_TRY(cudaMemcpy(t->d_obj, obj.data(), sizeof(unsigned long long) * obj.size(), cudaMemcpyHostToDevice));
  HR_CUDA_TRY(cudaMalloc(&t->d_scale, 4 * sizeof(float)));
  t->bytes = (size_t)views * YL * ZL * esz;
  return HR_OK;
}

// Arrays of the given kind for `views` views (kept when they already fit).
static int tex_alloc(BpFastTex* t, int kind, int YL, int ZL, int views) {
  if (t->kind == kind && (kind == 0 || (t->YL == YL && t->ZL == ZL && t->views >= views))) return HR_OK;
  tex_free(t);
  if (kind == 0) return HR_OK;
  const int st = tex_alloc_arrays(t, kind, YL, ZL, views);
  if (st != HR_OK) tex_free(t);
  return st;
}

int bp_fast_tex_prepare(BpFast* f, const BpFastGeom& g) {
  return tex_alloc(&f->tex, kFastVariants[f->variant].tex, g.YL, g.ZL, std::max(f->cap_views, g.PN));
}

// BF16 pairs of the geometry's views -> the plan's layered arrays.
int bp_fast_tex_fill(const BpFast& f, const BpFastGeom& g, const uint32_t* fpb, cudaStream_t s) {
  return bp_fast_tex_fill_range(f, g, fpb, 0, g.PN, 0, s);
}

int bp_fast_tex_fill_range(const BpFast& f, const BpFastGeom& g, const uint32_t* fpb, int p0, int p1, int mode,
                           cudaStream_t s) {
  const BpFastTex& t = f.tex;
  HR_REQUIRE(t.kind != 0 && t.views >= g.PN && t.YL == g.YL && t.ZL == g.ZL,
             "fast backprojection: the textures of variant %d are not prepared", f.variant);
  HR_REQUIRE(0 <= p0 && p0 <= p1 && p1 <= g.PN && mode >= 0 && mode <= 2, "fast backprojection: fill of views "
             "[%d, %d) (mode %d) outside [0, %d)", p0, p1, mode, g.PN);
  const long long r0 = (long long)p0 * g.ZL, r1 = (long long)p1 * g.ZL;
  const int grid = (int)std::max(1LL, std::min<long long>(r1 - r0, 16LL * sm_count()));
  if (t.kind == kTexHalf) {
    if (mode != 2) HR_CUDA_TRY(cudaMemsetAsync(t.d_scale + 1, 0, sizeof(float), s));
    if (r1 > r0) tex_absmax_kernel<<<4 * sm_count(), 256, 0, s>>>(t.d_scale, fpb + r0 * g.YL, (r1 - r0) * g.YL);
    if (mode == 0)
      tex_fill_kernel<true, 0><<<grid, 256, 0, s>>>(t.d_scale, t.d_obj + t.n, fpb, r0, r1, g.ZL, g.YL, t.lsh);
    else if (mode == 1)
      tex_fill_kernel<true, 1><<<grid, 256, 0, s>>>(t.d_scale, t.d_obj + t.n, fpb, r0, r1, g.ZL, g.YL, t.lsh);
    else
      tex_fill_kernel<true, 2><<<grid, 256, 0, s>>>(t.d_scale, t.d_obj + t.n, fpb, r0, r1, g.ZL, g.YL, t.lsh);
  } else {
    if (mode == 1) HR_CUDA_TRY(cudaMemsetAsync(t.d_scale + 3, 0, sizeof(float), s));
    tex_fill_kernel<false, 0><<<grid, 256, 0, s>>>(t.d_scale, t.d_obj + t.n, fpb, r0, r1, g.ZL, g.YL, t.lsh);
  }
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}

int bp_fast_tex_refill_needed(const BpFast& f, bool* needed) {
  *needed = false;
  if (f.tex.kind != kTexHalf) return HR_OK;
  float flag = 0.f;
  HR_CUDA_TRY(cudaMemcpy(&flag, f.tex.d_scale + 3, sizeof(float), cudaMemcpyDeviceToHost));
  *needed = flag != 0.f;
  return HR_OK;
}

void bp_fast_destroy(BpFast* f) {
  tex_free(&f->tex);
  for (int i = 0; i < kFastTableSets; ++i) {
    cudaFree(f->t[i].d_tab);
    cudaFree(f->t[i].d_mask);
    cudaFree(f->t[i].d_zblock);
    cudaFree(f->t[i].d_seg);
  }
  cudaFree(f->d_trig);
  *f = BpFast{};
}

static FastParams make_params(const BpFastGeom& g) {
  FastParams P;
  P.XN = g.XN; P.YN = g.YN; P.ZN = g.ZN; P.YL = g.YL; P.ZL = g.ZL; P.PN = g.PN;
  P.XNC = (float)g.XNC; P.YNC = (float)g.YNC; P.dx = (float)g.dx; P.dy = (float)g.dy;
  P.SO2 = (float)(g.SO * g.SO);
  P.SOSDdZL = (float)(g.SO * g.SD / g.dZL);
  P.invdYL = (float)(1.0 / g.dYL);
  P.YLC0 = (float)g.YLC;
  P.ZLC0 = (float)g.ZLC;
  P.k1 = (float)g.k1;
  P.DeltaFai = (float)g.DeltaFai;
  return P;
}

static TexRef texref(const BpFast& f) { return TexRef{f.tex.d_obj, f.tex.d_scale, f.tex.lsh}; }

static ZTabs ztabs(const BpFastTables& t, const BpFast& f) {
  return ZTabs{f.d_trig, t.d_tab, t.d_mask, reinterpret_cast<const int2*>(t.d_zblock), t.d_zblock + 2 * t.nblocks,
               t.d_seg};
}

template <int NZ, int CH>
static void launch_variant(const BpFastTables& t, const BpFast& f, const FastParams& P, float* vol,
                           const uint32_t* fpb, int b_first, int b_count, cudaStream_t s) {
  dim3 grid((P.XN + kBx - 1) / kBx, (P.YN + kBy - 1) / kBy, b_count);
  bp_fast_kernel<NZ, CH><<<grid, dim3(kBx, kBy), 0, s>>>(vol, fpb, ztabs(t, f), P, b_first);
}

template <int NZ>
static void launch_tex(const BpFastTables& t, const BpFast& f, const FastParams& P, float* vol, int b_first,
                       int b_count, cudaStream_t s) {
  dim3 grid((P.XN + kBx - 1) / kBx, (P.YN + kBy - 1) / kBy, b_count);
  bp_tex_kernel<NZ><<<grid, dim3(kBx, kBy), 0, s>>>(vol, texref(f), ztabs(t, f), P, b_first);
}

template <int NZ, int V>
static void launch_tex_seg(const BpFastTables& t, const BpFast& f, const FastParams& P, float* vol, int b_first,
                           int b_count, bool occ6, cudaStream_t s) {
  dim3 grid((P.XN + kBx - 1) / kBx, (P.YN + kBy - 1) / kBy, b_count);
  if (occ6)
    bp_tex_seg6_kernel<NZ, V><<<grid, dim3(kBx, kBy), 0, s>>>(vol, texref(f), ztabs(t, f), P, b_first);
  else
    bp_tex_seg_kernel<NZ, V><<<grid, dim3(kBx, kBy), 0, s>>>(vol, texref(f), ztabs(t, f), P, b_first);
}

// Launches variant v over z blocks [b_first, b_first + b_count) (count < 0: all).
static int run_variant(const BpFast& f, const BpFastGeom& g, int v, float* vol, const uint32_t* fpb, int b_first,
                       int b_count, cudaStream_t s) {
  const FastVariant& fv = kFastVariants[v];
  const BpFastTables& t = f.t[fv.table];
  if (b_count < 0) b_count = t.nblocks;
  HR_REQUIRE((g.YN + kBy - 1) / kBy <= 65535 && b_count <= 65535, "fast backprojection: grid too large");
  if (b_count == 0) return HR_OK;
  const FastParams P = make_params(g);
  if (fv.tex) {
    HR_REQUIRE(f.tex.kind == fv.tex && f.tex.views >= g.PN, "fast backprojection: the textures of variant %d are "
               "not prepared", v);
    if (fv.seg) {
      const bool two = fv.seg == 2, occ6 = fv.occ == 6;
      if (kFastNz[fv.table] == 8)
        two ? launch_tex_seg<8, 2>(t, f, P, vol, b_first, b_count, occ6, s)
            : launch_tex_seg<8, 1>(t, f, P, vol, b_first, b_count, occ6, s);
      else
        two ? launch_tex_seg<4, 2>(t, f, P, vol, b_first, b_count, occ6, s)
            : launch_tex_seg<4, 1>(t, f, P, vol, b_first, b_count, occ6, s);
    } else {
      switch (kFastNz[fv.table]) {
        case 16: launch_tex<16>(t, f, P, vol, b_first, b_count, s); break;
        case 8: launch_tex<8>(t, f, P, vol, b_first, b_count, s); break;
        default: launch_tex<4>(t, f, P, vol, b_first, b_count, s); break;
      }
    }
    HR_CUDA_TRY(cudaGetLastError());
    return HR_OK;
  }
  switch (v) {
    case 0: launch_variant<16, 0>(t, f, P, vol, fpb, b_first, b_count, s); break;
    case 1: launch_variant<16, 4>(t, f, P, vol, fpb, b_first, b_count, s); break;
    case 2: launch_variant<16, 8>(t, f, P, vol, fpb, b_first, b_count, s); break;
    case 3: launch_variant<8, 0>(t, f, P, vol, fpb, b_first, b_count, s); break;
    case 4: launch_variant<8, 4>(t, f, P, vol, fpb, b_first, b_count, s); break;
    case 5: launch_variant<8, 8>(t, f, P, vol, fpb, b_first, b_count, s); break;
    case 6: launch_variant<16, -1>(t, f, P, vol, fpb, b_first, b_count, s); break;
    case 7: launch_variant<8, -1>(t, f, P, vol, fpb, b_first, b_count, s); break;
    case 8: launch_variant<4, 0>(t, f, P, vol, fpb, b_first, b_count, s); break;
    case 9: launch_variant<4, -1>(t, f, P, vol, fpb, b_first, b_count, s); break;
    case 10: launch_variant<4, 4>(t, f, P, vol, fpb, b_first, b_count, s); break;
    default: return hr::fail(HR_ERR_INVALID_ARGUMENT, "fast backprojection: unknown variant %d", v);
  }
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}

static int table_of_nz(int nz) {
  for (int i = 0; i < kFastTableSets; ++i)
    if (kFastNz[i] == nz) return i;
  return -1;
}

long long bp_fast_batch_items(const BpFastBatchScan* scans, int n) {
  long long total = 0;
  for (int i = 0; i < n; ++i) {
    const BpFastGeom& g = *scans[i].g;
    const int ts = table_of_nz(scans[i].nz);
    if (ts < 0) return -1;
    total += (long long)((g.XN + kBx - 1) / kBx) * ((g.YN + kBy - 1) / kBy) * scans[i].f->t[ts].nblocks;
  }
  return total;
}

template <int MB, int CH>
static int batch_launch(const BatchParams* B, int* ctas, cudaStream_t s) {
  if (ctas) {
    int per_sm = 0;
    HR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bp_fast_batch_kernel<MB, CH>, kBx * kBy, 0));
    *ctas = std::max(per_sm, 1) * sm_count();
    return HR_OK;
  }
  bp_fast_batch_kernel<MB, CH><<<B->grid, dim3(kBx, kBy), 0, s>>>(*B);
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}

template <int MB, int NZF>
static int batch_launch_tex(const BatchParams* B, int* ctas, cudaStream_t s) {
  if (ctas) {
    int per_sm = 0;
    HR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bp_tex_batch_kernel<MB, NZF>, kBx * kBy, 0));
    *ctas = std::max(per_sm, 1) * sm_count();
    return HR_OK;
  }
  bp_tex_batch_kernel<MB, NZF><<<B->grid, dim3(kBx, kBy), 0, s>>>(*B);
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}

template <int MB, int NZF>
static int batch_launch_spec(const BatchParams* B, int* ctas, cudaStream_t s) {
  if (ctas) {
    int per_sm = 0;
    HR_CUDA_TRY(
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bp_tex_batch_spec_kernel<MB, NZF>, kBx * kBy, 0));
    *ctas = std::max(per_sm, 1) * sm_count();
    return HR_OK;
  }
  bp_tex_batch_spec_kernel<MB, NZF><<<B->grid, dim3(kBx, kBy), 0, s>>>(*B);
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}

template <int MB>
static int batch_launch_seg(const BatchParams* B, int* ctas, cudaStream_t s) {
  if (ctas) {
    int per_sm = 0;
    HR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bp_tex_seg_batch_kernel<MB>, kBx * kBy, 0));
    *ctas = std::max(per_sm, 1) * sm_count();
    return HR_OK;
  }
  bp_tex_seg_batch_kernel<MB><<<B->grid, dim3(kBx, kBy), 0, s>>>(*B);
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}

// ctas != nullptr: report the resident CTAs of batch variant bv; else launch *B.
static int batch_dispatch(int bv, const BatchParams* B, int* ctas, cudaStream_t s) {
  switch (bv) {
    case 0: return batch_launch<1, 0>(B, ctas, s);
    case 1: return batch_launch<5, 0>(B, ctas, s);
    case 2: return batch_launch<6, 0>(B, ctas, s);
    case 3: return batch_launch<1, 4>(B, ctas, s);
    case 4: return batch_launch<5, 4>(B, ctas, s);
    case 5: return batch_launch<6, 4>(B, ctas, s);
    case 6: return batch_launch_tex<1, 0>(B, ctas, s);
    case 7: return batch_launch_tex<4, 0>(B, ctas, s);
    case 8: return batch_launch_tex<4, 4>(B, ctas, s);
    case 9: return batch_launch_tex<5, 4>(B, ctas, s);
    case 10: return batch_launch_tex<6, 4>(B, ctas, s);
    case 12: return batch_launch_spec<1, 0>(B, ctas, s);
    case 13: return batch_launch_spec<1, 4>(B, ctas, s);
    case 14: return batch_launch_spec<5, 4>(B, ctas, s);
    case 15: return batch_launch_seg<1>(B, ctas, s);
    case 16: return batch_launch_seg<4>(B, ctas, s);
    case 11:  // per-scan launches: no persistent grid
      if (ctas) {
        *ctas = 0;
        return HR_OK;
      }
      return hr::fail(HR_ERR_INVALID_ARGUMENT, "batch backprojection: variant 11 is not a persistent launch");
    default: return hr::fail(HR_ERR_INVALID_ARGUMENT, "batch backprojection: unknown variant %d", bv);
  }
}

int bp_fast_batch_grid(int bv, int* ctas) { return batch_dispatch(bv, nullptr, ctas, nullptr); }

int bp_fast_batch_execute(const BpFastBatchScan* scans, int n, int bv, int begin, int count, int ctas,
                          int* d_counter, cudaStream_t s) {
  HR_REQUIRE(n >= 1 && n <= kBatchMaxScans, "batch backprojection: %d scans (1..%d per launch)", n, kBatchMaxScans);
  HR_REQUIRE(d_counter != nullptr, "batch backprojection: no work counter");
  HR_REQUIRE(bv >= 0 && bv < kBatchVariants_n, "batch backprojection: unknown variant %d", bv);
  HR_REQUIRE(ctas >= 1, "batch backprojection: no CTAs");
  BatchParams B{};
  long long item0 = 0;
  for (int i = 0; i < n; ++i) {
    const BpFastGeom& g = *scans[i].g;
    const int ts = table_of_nz(scans[i].nz);
    HR_REQUIRE(ts >= 0, "batch backprojection: scan %d: %d slices per thread is not a table set", i, scans[i].nz);
    const BpFastTables& t = scans[i].f->t[ts];
    BatchScan& S = B.s[i];
    S.P = make_params(g);
    S.T = ztabs(t, *scans[i].f);
    S.vol = scans[i].vol;
    S.fpb = scans[i].fpb;
    S.X = texref(*scans[i].f);
    HR_REQUIRE(!kBatchVariants[bv].tex || (scans[i].f->tex.kind == kTexHalf && scans[i].f->tex.views >= g.PN &&
                                           (scans[i].nz == 8 || scans[i].nz == 4)),
               "batch backprojection: scan %d has no FP16 texture copy for variant %d", i, bv);
    HR_REQUIRE(!kBatchVariants[bv].tex || kBatchVariants[bv].chunk == 0 || scans[i].nz == kBatchVariants[bv].chunk,
               "batch backprojection: variant %d runs %d slices per thread", bv, kBatchVariants[bv].chunk);
    S.tiles_x = (g.XN + kBx - 1) / kBx;
    S.tiles_y = (g.YN + kBy - 1) / kBy;
    S.item0 = (int)item0;
    S.nz = scans[i].nz;
    item0 += (long long)S.tiles_x * S.tiles_y * t.nblocks;
  }
  HR_REQUIRE(item0 < (1ll << 31), "batch backprojection: too many work items");
  HR_REQUIRE(begin >= 0 && count >= 0 && (long long)begin + count <= item0,
             "batch backprojection: items [%d, %d) outside [0, %lld)", begin, begin + count, item0);
  B.n = n;
  B.begin = begin;
  B.count = count;
  B.grid = std::min(ctas, std::max(count, 1));
  B.counter = d_counter;
  if (count == 0) return HR_OK;
  HR_CUDA_TRY(cudaMemsetAsync(d_counter, 0, sizeof(int), s));
  return batch_dispatch(bv, &B, nullptr, s);
}

int bp_fast_best_tex_variant(const BpFast& f) {
  // FP16 texture variants with 8 (11) and 4 (13) slices per thread
  return f.tuned == 1 && f.tuned_ms[13] < f.tuned_ms[11] ? 13 : 11;
}

int bp_fast_variant_nz(int v) { return v >= 0 && v < kFastVariants_n ? kFastNz[kFastVariants[v].table] : 0; }

int bp_fast_best_per_slice_nz(const BpFast& f) {
  // per-slice variants of each table set: 0 (16), 3 (8), 8 (4)
  const int cand[3] = {0, 3, 8};
  int best = 3;
  for (int v : cand)
    if (f.tuned == 1 && f.tuned_ms[v] < f.tuned_ms[best]) best = v;
  return kFastNz[kFastVariants[best].table];
}

int bp_fast_execute(const BpFast& f, const BpFastGeom& g, float* vol, const uint32_t* fpb, cudaStream_t s) {
  if (kFastVariants[f.variant].tex) HR_TRY(bp_fast_tex_fill(f, g, fpb, s));
  return run_variant(f, g, f.variant, vol, fpb, 0, -1, s);
}

int bp_fast_execute_blocks(const BpFast& f, const BpFastGeom& g, float* vol, const uint32_t* fpb, int b_first,
                           int b_count, cudaStream_t s) {
  const BpFastTables& t = f.t[kFastVariants[f.variant].table];
  HR_REQUIRE(b_first >= 0 && b_count >= 0 && b_first + b_count <= t.nblocks,
             "fast backprojection: z blocks [%d, %d) outside [0, %d)", b_first, b_first + b_count, t.nblocks);
  return run_variant(f, g, f.variant, vol, fpb, b_first, b_count, s);
}

const BpFastTables& bp_fast_variant_tables(const BpFast& f) { return f.t[kFastVariants[f.variant].table]; }

// HELIXRECON_BP_VARIANT=<index> pins the variant and skips the timing (for
// profiling runs, whose serialised launches would skew the choice, and for
// reproducible benchmarks).
static int pinned_variant() {
  const char* e = std::getenv("HELIXRECON_BP_VARIANT");
  if (!e || !*e) return -1;
  char* end = nullptr;
  const long v = std::strtol(e, &end, 10);
  if (*end != '\0' || v < 0 || v >= kFastVariants_n) return -2;
  return (int)v;
}

// Times every variant on the same middle band of 32 slices (all columns) and
// keeps the fastest. The band is written into vol; synchronises the stream.
int bp_fast_autotune(BpFast* f, const BpFastGeom& g, float* vol, const uint32_t* fpb, cudaStream_t s) {
  const int pin = pinned_variant();
  HR_REQUIRE(pin != -2, "HELIXRECON_BP_VARIANT must be an integer in [0, %d)", kFastVariants_n);
  if (pin >= 0) {
    f->variant = pin;
    f->tuned = 2;
    return bp_fast_tex_prepare(f, g);
  }
  cudaEvent_t e0, e1;
  HR_CUDA_TRY(cudaEventCreate(&e0));
  HR_CUDA_TRY(cudaEventCreate(&e1));
  const int band = 32;
  const int z_first = std::max(0, g.ZN / 2 - band / 2);
  float best = 1e30f;
  int best_v = f->variant;
  int st = HR_OK;
  float fill_ms = 0.f;  // texture variants: filling the arrays, per slice of the volume
  for (int v = 0; v < kFastVariants_n && st == HR_OK; ++v) {
    const int nz = kFastNz[kFastVariants[v].table];
    const int b0 = z_first / nz;
    const int bc = std::min((band + nz - 1) / nz, f->t[kFastVariants[v].table].nblocks - b0);
    if (kFastVariants[v].tex && f->tex.kind != kFastVariants[v].tex) {
      f->variant = v;
      st = bp_fast_tex_prepare(f, g);
      for (int rep = 0; rep < 2 && st == HR_OK; ++rep) {
        cudaEventRecord(e0, s);
        st = bp_fast_tex_fill(*f, g, fpb, s);
        cudaEventRecord(e1, s);
        if (st == HR_OK && cudaEventSynchronize(e1) != cudaSuccess)
          st = hr::fail(HR_ERR_CUDA, "fast backprojection autotune failed");
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        fill_ms = t / (float)std::max(g.ZN_valid, 1);
      }
    }
    float ms = 1e30f;
    for (int rep = 0; rep < 3 && st == HR_OK; ++rep) {
      cudaEventRecord(e0, s);
      st = run_variant(*f, g, v, vol, fpb, b0, bc, s);
      cudaEventRecord(e1, s);
      if (cudaEventSynchronize(e1) != cudaSuccess) st = hr::fail(HR_ERR_CUDA, "fast backprojection autotune failed");
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      if (rep > 0) ms = std::min(ms, t / (float)(bc * nz) + (kFastVariants[v].tex ? fill_ms : 0.f));  // per slice
    }
    f->tuned_ms[v] = ms;
    if (ms < best) {
      best = ms;
      best_v = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  f->variant = best_v;
  if (st != HR_OK) {
    f->variant = kFastDefaultVariant;
    tex_free(&f->tex);
    return st;
  }
  f->tuned = 1;
  return bp_fast_tex_prepare(f, g);
}

int bp_fast_describe(const BpFast& f, char* buf, int len) {
  if (!buf || len <= 0) return HR_OK;
  const FastVariant& fv = kFastVariants[f.variant];
  int n = snprintf(buf, (size_t)len, "slices_per_thread=%d gathers=%s tile=%dx%d %s", kFastNz[fv.table],
                   fv.tex == kTexHalf ? (fv.seg == 2 ? (fv.occ ? "texture-fp16-segmented-two-views-6ctas"
                                                               : "texture-fp16-segmented-two-views")
                                        : fv.seg ? (fv.occ ? "texture-fp16-segmented-6ctas" : "texture-fp16-segmented")
                                        : "texture-fp16")
                   : fv.tex == kTexFloat ? "texture-fp32"
                   : fv.chunk < 0 ? "paired-f32x2" : fv.chunk == 0 ? "per-slice" : fv.chunk == 4 ? "chunk4" : "chunk8",
                   kBx, kBy, f.tuned == 2 ? "(pinned by HELIXRECON_BP_VARIANT)"
                   : f.tuned ? "(autotuned; ms/slice:" : "(default)");
  if (f.tuned == 1) {
    for (int v = 0; v < kFastVariants_n && n > 0 && n < len; ++v)
      n += snprintf(buf + n, (size_t)(len - n), " v%d=%.4f", v, f.tuned_ms[v]);
    if (n > 0 && n < len) snprintf(buf + n, (size_t)(len - n), ")");
  }
  return HR_OK;
}

int pack_pairs(uint32_t* out, const float* in, long long rows, int YL, cudaStream_t s) {
  pack_pairs_kernel<<<8 * sm_count(), 256, 0, s>>>(out, in, rows, YL);
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}

}  // namespace hr

extern "C" int hr_pack_bf16_pairs(uint32_t* d_out, const float* d_in, long long rows, int YL, void* stream) {
  HR_REQUIRE(d_out != nullptr && d_in != nullptr && rows >= 0 && YL > 0, "hr_pack_bf16_pairs: invalid argument");
  HR_REQUIRE((const void*)d_out != (const void*)d_in, "hr_pack_bf16_pairs: in-place packing is not supported");
  return hr::pack_pairs(d_out, d_in, rows, YL, hr::as_stream(stream));
}
