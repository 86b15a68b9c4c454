// Curved-detector fan -> parallel rebinning.
//
// Reference: src/ParallelRebinningCBCurve.cpp:22-97 (CPU template, the parity
// target) and src/ParallelRebinningCBCurveGPU.cu:6-104 (GPU kernel).
//
// For output sample (view i, channel j, row k):
//   Theta = i*DeltaTheta, t = (j-PLC)*DeltaT, Fai = Theta + asin(t/SO),
//   a = atan(t/sqrt(SO^2-t^2)), FaiIndex = Fai/DeltaFai, UIndex = a/dYA + YLC,
//   FI = ceil(FaiIndex), UI = ceil(UIndex), bilinear in (FI-1, FI) x (UI-1, UI)
//   with the CPU clamp rule (index > N-1 clamps; the reference GPU uses >=).
//
// Everything that depends only on the channel j (Beta, UIndex, UI, coeYB,
// coeYU) is computed once per plan on the host, in the reference CPU's own
// arithmetic (float operands, the C double asin/atan/sqrt the reference binds
// to, rounded to float on assignment), so the per-channel values are the same
// bits. The device then does, per (i, j), the float multiply/add/divide and
// ceil the reference does -- with __fmul_rn/__fadd_rn/__fdiv_rn so that no FMA
// contraction changes a rounding -- and per row k the 4-tap blend in the
// reference's operation order. The result is bit-identical to the CPU path.
//
// Layout [ViewN][YL][ZL], ZL fastest: the ZL rows of one (view, channel) are
// contiguous, so a thread moves 4 rows at once (16-byte loads/stores) and the
// four taps of a warp are contiguous runs. Grid: x over (channel, row quad),
// y over the output views [i0, i1) (grid-stride beyond 65535); the clamp is
// always against the whole scan's ViewN, so a range of views has the bits of
// the same views of a whole-scan launch.
#include <algorithm>
#include <cmath>
#include <vector>

#include "hr_internal.h"

struct ChanInfo {
  float beta;  // asin(t/SO) rounded to float
  float cyb;   // coeYB = UI - UIndex
  float cyu;   // coeYU = (float)(1.0 - coeYB)
  int ybyu;    // IndexYB | IndexYU << 16
};

struct hr_rebin_plan {
  int YL, ZL, ViewN;
  float DeltaTheta, DeltaFai;
  ChanInfo* d_chan;
  float beta_lo, beta_hi;  // smallest and largest per-channel angle offset (for hr::rebin_fan_views)
};

namespace {

template <int VEC>
struct VecT;
template <>
struct VecT<4> {
  using T = float4;
};
template <>
struct VecT<1> {
  using T = float;
};

__device__ __forceinline__ float blend4(float wbb, float wub, float wbu, float wuu, float a, float b, float c,
                                        float d) {
  float acc = __fmul_rn(wbb, a);
  acc = __fadd_rn(acc, __fmul_rn(wub, b));
  acc = __fadd_rn(acc, __fmul_rn(wbu, c));
  acc = __fadd_rn(acc, __fmul_rn(wuu, d));
  return acc;
}

template <int VEC>
__global__ void __launch_bounds__(256) rebin_kernel(float* __restrict__ out, const float* __restrict__ proj,
                                                    const ChanInfo* __restrict__ chan, int YL, int ZL, int ViewN,
                                                    float DeltaTheta, float DeltaFai, int i0, int i1) {
  using V = typename VecT<VEC>::T;
  const int nkq = ZL / VEC;
  const int jk = blockIdx.x * blockDim.x + threadIdx.x;
  if (jk >= YL * nkq) return;
  const int j = jk / nkq;
  const int k = (jk - j * nkq) * VEC;
  const ChanInfo c = chan[j];
  const int YB = c.ybyu & 0xffff, YU = c.ybyu >> 16;
  for (int i = i0 + (int)blockIdx.y; i < i1; i += gridDim.y) {
    const float Theta = __fmul_rn((float)i, DeltaTheta);
    const float Fai = __fadd_rn(Theta, c.beta);
    const float FaiIndex = __fdiv_rn(Fai, DeltaFai);
    const int FI = (int)ceilf(FaiIndex);
    const float cxb = __fsub_rn((float)FI, FaiIndex);
    const float cxu = __double2float_rn(__dsub_rn(1.0, (double)cxb));
    int XU, XB;
    if (FI <= 0) {
      XU = 0;
      XB = 0;
    } else if (FI > ViewN - 1) {
      XU = ViewN - 1;
      XB = ViewN - 1;
    } else {
      XU = FI;
      XB = FI - 1;
    }
    const float wbb = __fmul_rn(cxb, c.cyb), wub = __fmul_rn(cxu, c.cyb);
    const float wbu = __fmul_rn(cxb, c.cyu), wuu = __fmul_rn(cxu, c.cyu);
    const size_t zl = (size_t)ZL;
    const V a = *reinterpret_cast<const V*>(proj + ((size_t)XB * YL + YB) * zl + k);
    const V b = *reinterpret_cast<const V*>(proj + ((size_t)XU * YL + YB) * zl + k);
    const V cc = *reinterpret_cast<const V*>(proj + ((size_t)XB * YL + YU) * zl + k);
    const V d = *reinterpret_cast<const V*>(proj + ((size_t)XU * YL + YU) * zl + k);
    V r;
    if constexpr (VEC == 4) {
      r.x = blend4(wbb, wub, wbu, wuu, a.x, b.x, cc.x, d.x);
      r.y = blend4(wbb, wub, wbu, wuu, a.y, b.y, cc.y, d.y);
      r.z = blend4(wbb, wub, wbu, wuu, a.z, b.z, cc.z, d.z);
      r.w = blend4(wbb, wub, wbu, wuu, a.w, b.w, cc.w, d.w);
    } else {
      r = blend4(wbb, wub, wbu, wuu, a, b, cc, d);
    }
    *reinterpret_cast<V*>(out + ((size_t)i * YL + j) * zl + k) = r;
  }
}

// rebin_kernel's arithmetic with NQ 16-byte quads of rows per thread: 4 NQ
// rows share one (view, channel) index computation, and every row is blended
// with the same scalar non-contracting operations, so the bits are the same.
// (Packed FP32x2 multiplies and adds were tried for the blends and measured
// 1-2 ulp away from the reference on a quarter of the samples: they do not
// round like the scalar mul.rn / add.rn sequence.)
template <int NQ>
__global__ void __launch_bounds__(256) rebin_rows_kernel(float* __restrict__ out, const float* __restrict__ proj,
                                                       const ChanInfo* __restrict__ chan, int YL, int ZL, int ViewN,
                                                       float DeltaTheta, float DeltaFai, int i0, int i1) {
  const int nkq = ZL / (4 * NQ);
  const int jk = blockIdx.x * blockDim.x + threadIdx.x;
  if (jk >= YL * nkq) return;
  const int j = jk / nkq;
  const int k = (jk - j * nkq) * 4 * NQ;
  const ChanInfo c = chan[j];
  const int YB = c.ybyu & 0xffff, YU = c.ybyu >> 16;
  const size_t zl = (size_t)ZL;
  for (int i = i0 + (int)blockIdx.y; i < i1; i += gridDim.y) {
    const float Theta = __fmul_rn((float)i, DeltaTheta);
    const float Fai = __fadd_rn(Theta, c.beta);
    const float FaiIndex = __fdiv_rn(Fai, DeltaFai);
    const int FI = (int)ceilf(FaiIndex);
    const float cxb = __fsub_rn((float)FI, FaiIndex);
    const float cxu = __double2float_rn(__dsub_rn(1.0, (double)cxb));
    int XU, XB;
    if (FI <= 0) {
      XU = 0;
      XB = 0;
    } else if (FI > ViewN - 1) {
      XU = ViewN - 1;
      XB = ViewN - 1;
    } else {
      XU = FI;
      XB = FI - 1;
    }
    const float wbb = __fmul_rn(cxb, c.cyb), wub = __fmul_rn(cxu, c.cyb);
    const float wbu = __fmul_rn(cxb, c.cyu), wuu = __fmul_rn(cxu, c.cyu);
    const float4* pa = reinterpret_cast<const float4*>(proj + ((size_t)XB * YL + YB) * zl + k);
    const float4* pb = reinterpret_cast<const float4*>(proj + ((size_t)XU * YL + YB) * zl + k);
    const float4* pc = reinterpret_cast<const float4*>(proj + ((size_t)XB * YL + YU) * zl + k);
    const float4* pd = reinterpret_cast<const float4*>(proj + ((size_t)XU * YL + YU) * zl + k);
    float4 a[NQ], b[NQ], cc[NQ], d[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      a[q] = pa[q];
      b[q] = pb[q];
      cc[q] = pc[q];
      d[q] = pd[q];
    }
    float4* po = reinterpret_cast<float4*>(out + ((size_t)i * YL + j) * zl + k);
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      float4 r;
      r.x = blend4(wbb, wub, wbu, wuu, a[q].x, b[q].x, cc[q].x, d[q].x);
      r.y = blend4(wbb, wub, wbu, wuu, a[q].y, b[q].y, cc[q].y, d[q].y);
      r.z = blend4(wbb, wub, wbu, wuu, a[q].z, b[q].z, cc[q].z, d[q].z);
      r.w = blend4(wbb, wub, wbu, wuu, a[q].w, b[q].w, cc[q].w, d[q].w);
      po[q] = r;
    }
  }
}

// Per-channel values in the reference CPU's arithmetic
// (ParallelRebinningCBCurve.cpp:37-48, 71-85 with T = float).
void channel_table(std::vector<ChanInfo>& tab, int YL, float YLC, float dYA, float PLC, float DeltaT, float SO) {
  tab.resize(YL);
  for (int j = 0; j < YL; ++j) {
    const float t = ((float)j - PLC) * DeltaT;
    const float Beta = (float)std::asin((double)(t / SO));
    const float a = (float)std::atan((double)t / std::sqrt((double)(SO * SO - t * t)));
    const float UIndex = a / dYA + YLC;
    const int UI = (int)std::ceil((double)UIndex);
    const float coeYB = (float)UI - UIndex;
    const float coeYU = (float)(1.0 - (double)coeYB);
    int YU, YB;
    if (UI <= 0) {
      YU = 0;
      YB = 0;
    } else if (UI > YL - 1) {
      YU = YL - 1;
      YB = YL - 1;
    } else {
      YU = UI;
      YB = UI - 1;
    }
    tab[j] = ChanInfo{Beta, coeYB, coeYU, YB | (YU << 16)};
  }
}

}  // namespace

extern "C" int hr_rebin_plan_create(hr_rebin_plan** plan, int YL, int ZL, int ViewN, float YLC, float dYA,
                                    float DeltaTheta, float PLC, float DeltaT, float DeltaFai, float SO) {
  hr::clear_error();
  HR_REQUIRE(plan != nullptr, "hr_rebin_plan_create: plan is NULL");
  *plan = nullptr;
  HR_REQUIRE(YL > 0 && ZL > 0 && ViewN > 0, "rebin: sizes must be positive (YL=%d ZL=%d ViewN=%d)", YL, ZL, ViewN);
  HR_REQUIRE(YL < 32768, "rebin: YL=%d exceeds 32767", YL);
  HR_REQUIRE(DeltaFai != 0.0f && SO > 0.0f && dYA != 0.0f, "rebin: DeltaFai, dYA must be non-zero and SO > 0");
  HR_REQUIRE((size_t)YL * ZL < (size_t)1 << 31, "rebin: YL*ZL too large");
  HR_TRY(hr::require_device());
  std::vector<ChanInfo> tab;
  channel_table(tab, YL, YLC, dYA, PLC, DeltaT, SO);
  hr_rebin_plan* p = new hr_rebin_plan{YL, ZL, ViewN, DeltaTheta, DeltaFai, nullptr, tab[0].beta, tab[0].beta};
  for (const ChanInfo& c : tab) {
    p->beta_lo = std::min(p->beta_lo, c.beta);
    p->beta_hi = std::max(p->beta_hi, c.beta);
  }
  cudaError_t e = cudaMalloc(&p->d_chan, sizeof(ChanInfo) * YL);
  if (e == cudaSuccess) e = cudaMemcpy(p->d_chan, tab.data(), sizeof(ChanInfo) * YL, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(p->d_chan);
    delete p;
    return hr::fail(e == cudaErrorMemoryAllocation ? HR_ERR_OUT_OF_MEMORY : HR_ERR_CUDA, "rebin plan: %s",
                    cudaGetErrorString(e));
  }
  *plan = p;
  return HR_OK;
}

int hr::rebin_execute_range(const hr_rebin_plan* p, float* d_out, const float* d_proj, int i0, int i1, int max_ctas,
                            cudaStream_t s) {
  HR_REQUIRE(p != nullptr && d_out != nullptr && d_proj != nullptr, "hr_rebin_execute: NULL argument");
  HR_REQUIRE(d_out != d_proj, "hr_rebin_execute: in-place rebinning is not supported");
  HR_REQUIRE(0 <= i0 && i0 <= i1 && i1 <= p->ViewN, "hr_rebin_execute: views [%d, %d) outside [0, %d)", i0, i1,
             p->ViewN);
  if (i1 == i0) return HR_OK;
  const bool al16 = ((uintptr_t)d_out % 16 == 0) && ((uintptr_t)d_proj % 16 == 0);
  const int nq = !al16 ? 0 : p->ZL % 8 == 0 ? 2 : p->ZL % 4 == 0 ? 1 : 0;  // 16-byte quads per thread
  const int nkq = nq ? p->ZL / (4 * nq) : p->ZL;
  const int threads = 256;
  const int gx = (p->YL * nkq + threads - 1) / threads;
  int gy = std::min(i1 - i0, 65535);  // the kernels stride over the views
  if (max_ctas > 0) gy = std::max(1, std::min(gy, max_ctas / gx));
  const dim3 grid(gx, gy);
  if (nq == 2)
    rebin_rows_kernel<2><<<grid, threads, 0, s>>>(d_out, d_proj, p->d_chan, p->YL, p->ZL, p->ViewN, p->DeltaTheta,
                                               p->DeltaFai, i0, i1);
  else if (nq == 1)
    rebin_rows_kernel<1><<<grid, threads, 0, s>>>(d_out, d_proj, p->d_chan, p->YL, p->ZL, p->ViewN, p->DeltaTheta,
                                               p->DeltaFai, i0, i1);
  else
    rebin_kernel<1><<<grid, threads, 0, s>>>(d_out, d_proj, p->d_chan, p->YL, p->ZL, p->ViewN, p->DeltaTheta,
                                            p->DeltaFai, i0, i1);
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}

int hr::rebin_execute_limited(const hr_rebin_plan* p, float* d_out, const float* d_proj, int max_ctas,
                              cudaStream_t s) {
  HR_REQUIRE(p != nullptr, "hr_rebin_execute: NULL argument");
  return rebin_execute_range(p, d_out, d_proj, 0, p->ViewN, max_ctas, s);
}

// Output view i reads the fan views FI - 1 and FI with FI = ceil((i DeltaTheta + beta_j) / DeltaFai) over the
// channels j (clamped to the scan). Bounded here in double with one view of slack on each side for the float
// rounding of the kernel's arithmetic.
static void fan_view_bounds(double dt, double df, float beta_lo, float beta_hi, int ViewN, int i0, int i1, int* f0,
                            int* f1) {
  double a = 1e300, b = -1e300;  // FaiIndex is monotone in i and in beta: its extremes are at the corners
  for (const int i : {i0, i1 - 1})
    for (const float beta : {beta_lo, beta_hi}) {
      const double x = (i * dt + beta) / df;
      a = std::min(a, x);
      b = std::max(b, x);
    }
  const double lo = std::floor(a) - 2.0, hi = std::ceil(b) + 1.0;
  *f0 = (int)std::max(0.0, std::min(lo, (double)(ViewN - 1)));
  *f1 = (int)std::max(0.0, std::min(hi, (double)(ViewN - 1)));
}

void hr::rebin_fan_views(const hr_rebin_plan* p, int i0, int i1, int* f0, int* f1) {
  fan_view_bounds(p->DeltaTheta, p->DeltaFai, p->beta_lo, p->beta_hi, p->ViewN, i0, i1, f0, f1);
}

extern "C" int hr_rebin_fan_views(int YL, int ViewN, float YLC, float dYA, float DeltaTheta, float PLC, float DeltaT,
                                  float DeltaFai, float SO, int i0, int i1, int* f0, int* f1) {
  hr::clear_error();
  HR_REQUIRE(f0 != nullptr && f1 != nullptr, "hr_rebin_fan_views: NULL argument");
  HR_REQUIRE(YL > 0 && ViewN > 0 && DeltaFai != 0.0f && SO > 0.0f && dYA != 0.0f,
             "hr_rebin_fan_views: invalid geometry");
  HR_REQUIRE(0 <= i0 && i0 < i1 && i1 <= ViewN, "hr_rebin_fan_views: views [%d, %d) outside [0, %d)", i0, i1, ViewN);
  std::vector<ChanInfo> tab;
  channel_table(tab, YL, YLC, dYA, PLC, DeltaT, SO);
  float lo = tab[0].beta, hi = tab[0].beta;
  for (const ChanInfo& c : tab) {
    lo = std::min(lo, c.beta);
    hi = std::max(hi, c.beta);
  }
  fan_view_bounds(DeltaTheta, DeltaFai, lo, hi, ViewN, i0, i1, f0, f1);
  return HR_OK;
}

extern "C" int hr_rebin_execute(const hr_rebin_plan* p, float* d_out, const float* d_proj, void* stream) {
  return hr::rebin_execute_limited(p, d_out, d_proj, 0, hr::as_stream(stream));
}

extern "C" void hr_rebin_plan_destroy(hr_rebin_plan* p) {
  if (!p) return;
  cudaFree(p->d_chan);
  delete p;
}
