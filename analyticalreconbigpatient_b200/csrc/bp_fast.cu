// 3D-weighted helical backprojection, fast form (BF16 filtered data).
//
// Same algorithm as the plain form (src/Parallel_FDK_Helical_3DWeighting.cpp:
// 42-113, views s1..s2), rearranged so that a voxel-view update costs one FMA
// for the detector row, two 32-bit gathers and two SFU operations:
//
//   weight = w1 Gc^k1 / (w2 G^k1 + w1 Gc^k1) = 1 / (1 + 2^(Q + C))
//   Q(view, slice) = k1 (log2|t2| - log2|t2 -/+ 0.5|) + log2(w2/w1)
//   C(column, view) = k1 log2((temp1 - UU)/(temp1 + UU))
//
// with t2 = z - h View/2pi. t2 and Q depend only on (view, slice): they are
// evaluated once per plan in FP64 (the helical source position accumulates
// over ~1e4-1e5 views) and stored per z block as a float2 table; a CTA covers
// one z block, so every thread of a CTA reads the same table entry (broadcast)
// and a per-(block, view) bit mask tells which of its slices have the view in
// their [s1, s2] window. Everything per (column, view) -- UU, Yr,
// temp1 = sqrt(SO^2 - Yr^2), the projection slope K = SO SD/(temp1 (temp1+UU)
// dZL), C, the channel -- is FP32, computed once and reused for the NZ slices.
//
// Filtered data are BF16 "pairs": word u of a detector row holds the values of
// channels u (low half) and u+1 (high half), so one 32-bit load gives both
// horizontal taps of a row. The bilinear tap uses floor instead of the
// reference's ceil; both give the same interpolated value away from exact
// integers, where the blend is continuous.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "hr_internal.h"
#include "bp_fast.h"

namespace {

constexpr int kBx = 8, kBy = 16;  // CTA tile (x, y): 4 warps of 8 x 4 columns
constexpr double kTwoPiTrunc = 2.0 * 3.14159265358979;
constexpr double kInvTwoPi = 1.0 / (2.0 * 3.141592653589793);
constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23: adding it rounds to an integer

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

template <int NZ>
__global__ void __launch_bounds__(kBx* kBy) bp_fast_kernel(float* __restrict__ vol, const uint32_t* __restrict__ fpb,
                                                          const float2* __restrict__ trig,
                                                          const float2* __restrict__ ztab,
                                                          const uint32_t* __restrict__ zmask,
                                                          const int2* __restrict__ zblock,
                                                          const int* __restrict__ zoff, FastParams P) {
  const int xi = blockIdx.x * kBx + threadIdx.x;
  const int yi = blockIdx.y * kBy + threadIdx.y;
  const int b = blockIdx.z;
  const int z0 = b * NZ;
  if (xi >= P.XN || yi >= P.YN) return;
  const int2 blk = zblock[b];  // {first view, number of views} of the block's union window
  const int off = zoff[b];     // row of the block's first view in the table
  const float x = ((float)xi - P.XNC) * P.dx;
  const float y = ((float)yi - P.YNC) * P.dy;
  float res[NZ];
#pragma unroll
  for (int m = 0; m < NZ; ++m) res[m] = 0.0f;
  const size_t plane = (size_t)P.ZL * P.YL;
  const float2* btab = ztab + (size_t)off * NZ;
  const uint32_t* bmask = zmask + off;
  for (int q = 0; q < blk.y; ++q) {
    const uint32_t mask = __ldg(bmask + q);
    if (mask == 0u) continue;
    const int p = blk.x + q;
    const float2 cs = __ldg(trig + p);
    const float UU = -x * cs.x - y * cs.y;
    const float Yr = -x * cs.y + y * cs.x;
    const float t1sq = P.SO2 - Yr * Yr;
    const float temp1 = t1sq * rsqrtf(t1sq);
    const float A = temp1 + UU, B = temp1 - UU;
    const float K = P.SOSDdZL * rcp_approx(temp1 * A);
    const float C = P.k1 * lg2_approx(B * rcp_approx(A));
    float u0f;
    const int u0 = floor_magic(fmaf(Yr, P.invdYL, P.YLC0), u0f);
    if ((unsigned)u0 > (unsigned)(P.YL - 2)) continue;
    const float fu = fmaf(Yr, P.invdYL, P.YLC0) - u0f;
    const uint32_t* col = fpb + (size_t)p * plane + u0;
    const float2* e = btab + (size_t)q * NZ;
#pragma unroll
    for (int m = 0; m < NZ; ++m) {
      if (!(mask & (1u << m))) continue;
      const float2 tq = __ldg(e + m);  // {t2, Q}
      float v0f;
      const float v1 = fmaf(tq.x, K, P.ZLC0);
      const int v0 = floor_magic(v1, v0f);
      if ((unsigned)v0 > (unsigned)(P.ZL - 2)) continue;
      const float fz = v1 - v0f;
      const uint32_t w0 = __ldg(col + (size_t)v0 * P.YL);
      const uint32_t w1 = __ldg(col + (size_t)(v0 + 1) * P.YL);
      const float a0 = __uint_as_float(w0 << 16), a1 = __uint_as_float(w0 & 0xffff0000u);
      const float b0 = __uint_as_float(w1 << 16), b1 = __uint_as_float(w1 & 0xffff0000u);
      const float ra = fmaf(fu, a1 - a0, a0);
      const float rb = fmaf(fu, b1 - b0, b0);
      const float tap = fmaf(fz, rb - ra, ra);
      const float wgt = rcp_approx(1.0f + ex2_approx(tq.y + C));
      res[m] = fmaf(wgt, tap, res[m]);
    }
  }
  float* out = vol + ((size_t)yi * P.XN + xi) * P.ZN + z0;
#pragma unroll
  for (int m = 0; m < NZ; ++m)
    if (z0 + m < P.ZN) out[m] = res[m] * P.DeltaFai;
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

// Host-side table build, FP64 (the reference's view angle, source height and
// window rules, ..._3DWeighting.cpp:61-75, 79, 95-102).
int bp_fast_create(BpFast* f, const BpFastGeom& g, const double* w) {
  constexpr int NZ = kBpFastNz;
  const int nblocks = (g.ZN + NZ - 1) / NZ;
  std::vector<int> s0(g.ZN), lo(g.ZN), hi(g.ZN);
  std::vector<double> zc(g.ZN);
  for (int zi = 0; zi < g.ZN; ++zi) {
    const double z = (zi - g.ZNC) * g.dz;
    zc[zi] = z;
    const double beta0 = kTwoPiTrunc * z / g.h;
    s0[zi] = (int)std::ceil((beta0 - g.BetaS) / g.DeltaFai - 0.5);
    const int s1 = s0[zi] - g.half, s2 = s0[zi] + g.half;
    if (s1 < g.PN && s2 > 0) {
      lo[zi] = s1 < 0 ? 0 : s1;
      hi[zi] = s2 > g.PN - 1 ? g.PN - 1 : s2;
    } else {
      lo[zi] = 1;
      hi[zi] = 0;
    }
  }
  std::vector<int> first(nblocks), count(nblocks), off(nblocks);
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
    first[b] = a;
    count[b] = e - a + 1;
    off[b] = (int)total;
    total += (size_t)count[b];
  }
  HR_REQUIRE(total < (1ull << 31) / NZ, "fast backprojection: z-block table too large");
  std::vector<float2> tab(total * NZ, make_float2(0.f, 0.f));
  std::vector<uint32_t> mask(total, 0u);
  for (int b = 0; b < nblocks; ++b) {
    for (int q = 0; q < count[b]; ++q) {
      const int p = first[b] + q;
      const double View = g.BetaS + p * g.DeltaFai;
      const double hv = g.h * View * kInvTwoPi;
      uint32_t mk = 0;
      for (int m = 0; m < NZ; ++m) {
        const int zi = b * NZ + m;
        if (zi >= g.ZN || p < lo[zi] || p > hi[zi]) continue;
        const double t2 = zc[zi] - hv;
        const int d1 = (int)(g.N_pi - (double)(s0[zi] - p));
        const int d2 = p < s0[zi] ? (int)(d1 + g.N_pi) : (int)(d1 - g.N_pi);
        const double w1 = w[d1], w2 = w[d2];
        const double tc = p < s0[zi] ? t2 - 0.5 : t2 + 0.5;
        double Q = g.k1 * (std::log2(std::fabs(t2)) - std::log2(std::fabs(tc)));
        Q += std::log2(w2) - std::log2(w1);
        tab[(size_t)(off[b] + q) * NZ + m] = make_float2((float)t2, (float)Q);
        mk |= 1u << m;
      }
      mask[off[b] + q] = mk;
    }
  }
  std::vector<float2> trig(g.PN);
  for (int p = 0; p < g.PN; ++p) {
    const double View = g.BetaS + p * g.DeltaFai;
    trig[p] = make_float2((float)std::cos(View), (float)std::sin(View));
  }
  // zblock records: [nblocks] int2 {first, count}, then [nblocks] int offsets
  std::vector<int> zb(3 * nblocks);
  for (int b = 0; b < nblocks; ++b) {
    zb[2 * b] = first[b];
    zb[2 * b + 1] = count[b];
    zb[2 * nblocks + b] = off[b];
  }
  f->nblocks = nblocks;
  HR_CUDA_TRY(cudaMalloc(&f->d_tab, sizeof(float2) * tab.size()));
  HR_CUDA_TRY(cudaMalloc(&f->d_mask, sizeof(uint32_t) * (mask.size() + 1)));
  HR_CUDA_TRY(cudaMalloc(&f->d_trig, sizeof(float2) * trig.size()));
  HR_CUDA_TRY(cudaMalloc(&f->d_zblock, sizeof(int) * zb.size()));
  HR_CUDA_TRY(cudaMemcpy(f->d_tab, tab.data(), sizeof(float2) * tab.size(), cudaMemcpyHostToDevice));
  HR_CUDA_TRY(cudaMemcpy(f->d_mask, mask.data(), sizeof(uint32_t) * mask.size(), cudaMemcpyHostToDevice));
  HR_CUDA_TRY(cudaMemcpy(f->d_trig, trig.data(), sizeof(float2) * trig.size(), cudaMemcpyHostToDevice));
  HR_CUDA_TRY(cudaMemcpy(f->d_zblock, zb.data(), sizeof(int) * zb.size(), cudaMemcpyHostToDevice));
  f->bytes = sizeof(float2) * tab.size() + sizeof(uint32_t) * mask.size() + sizeof(float2) * trig.size() +
             sizeof(int) * zb.size();
  return HR_OK;
}

void bp_fast_destroy(BpFast* f) {
  cudaFree(f->d_tab);
  cudaFree(f->d_mask);
  cudaFree(f->d_trig);
  cudaFree(f->d_zblock);
  *f = BpFast{};
}

int bp_fast_execute(const BpFast& f, const BpFastGeom& g, float* vol, const uint32_t* fpb, cudaStream_t s) {
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
  dim3 grid((g.XN + kBx - 1) / kBx, (g.YN + kBy - 1) / kBy, f.nblocks);
  HR_REQUIRE(grid.y <= 65535 && grid.z <= 65535, "fast backprojection: grid too large");
  bp_fast_kernel<kBpFastNz><<<grid, dim3(kBx, kBy), 0, s>>>(
      vol, fpb, f.d_trig, f.d_tab, f.d_mask, reinterpret_cast<const int2*>(f.d_zblock), f.d_zblock + 2 * f.nblocks, P);
  HR_CUDA_TRY(cudaGetLastError());
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
