// 3D-weighted helical parallel-cone backprojection (plain FP32 and FP64 forms).
//
// Reference: src/Parallel_FDK_Helical_3DWeighting.cpp:42-113 (CPU, the parity
// target) and src/ParallelFDKHelical3DWeightingGPU.cu:14-87 (GPU). For voxel
// (x, y, z): s0 = ceil((2 pi z/h - BetaS)/DeltaFai - 0.5), views
// s0 -/+ ceil(N_pi HSCoef) clamped to [0, PN-1] (the CPU loop; the reference
// GPU loop starts at view 0 and reads w[] out of bounds for far views), and
// per view: UU, Yr, temp1 = sqrt(SO^2 - Yr^2), temp2 = z - h View/2pi,
// Zr = temp2 SO SD/(UU temp1 + SO^2 - Yr^2), U = ceil(Yr/dYL + YLC),
// V = ceil(Zr/dZL + ZLC), bilinear tap if 0 < U < YL and 0 < V < ZL, and the
// 3D weight w[d1] Gama_C^k1 / (w[d2] Gama^k1 + w[d1] Gama_C^k1).
//
// Index selection is bit-exact to the CPU path: x, y, z, s0, UU, Yr, temp1,
// U1 and temp2 are evaluated in double with the reference's operation order
// through non-contracting __d*_rn intrinsics, from per-view cos/sin/h*View/2pi
// tables that the plan computes on the host with the same C library calls. V
// is first located with one FMA from a per-(column, view) slope; only when
// that estimate lies within 1e-9 of an integer (the estimate's error is below
// 1e-12) is Zr/dZL + ZLC recomputed exactly, so ceil() never disagrees.
//
// Work decomposition: a thread owns NZ consecutive voxels of one (x, y)
// column. Everything that does not depend on z (the trig, UU, Yr, temp1, U,
// Dey, the projection slope, 1/(temp1 +- UU)) is computed once per column and
// view and reused for the NZ voxels; the NZ windows [s1, s2] are uniform over
// the CTA (all its threads share the z block), so the per-voxel window test
// is a uniform branch. A warp is an 8 x 4 (x, y) tile, which keeps its 32
// detector taps within a few cache lines of one or two rows.
#include <cmath>
#include <vector>

#include "hr_internal.h"
#include "bp_fast.h"

namespace {

constexpr int kBx = 8, kBy = 16;  // CTA tile (x, y); warps are 8 x 4
constexpr double kTwoPiTrunc = 2.0 * 3.14159265358979;         // ..._3DWeighting.cpp:16,62
constexpr double kInvTwoPi = 1.0 / (2.0 * 3.141592653589793);  // :51,79

struct ViewTab {
  double c, s, hv;  // cos(View), sin(View), h*View*invPI
};

struct BpParams {
  int XN, YN, ZN, YL, ZL, PN, N_2pi, half;
  int qcap;  // longest union view window of a z block of the plain kernel (its weight table rows)
  double XNC, YNC, ZNC, dx, dy, dz, YLC, ZLC, dYL, dZL, h, BetaS, DeltaFai, N_pi, SO, SD, k1;
  double SO2, SOSD, SOSDdZL;
  float k1f, DeltaFaif;
};

}  // namespace

struct hr_bp_plan {
  BpParams prm;
  int form;
  ViewTab* d_views;
  float* d_w;
  double* d_wd;
  hr::BpFastGeom fg;
  hr::BpFast fast;
};

namespace {

// Voxel centre and central view, exactly as the CPU reference.
struct ZInfo {
  double z;
  int s0, lo, hi;
};

__device__ __forceinline__ ZInfo z_info(const BpParams& P, int zi) {
  ZInfo r;
  r.z = __dmul_rn(__dsub_rn((double)zi, P.ZNC), P.dz);
  const double beta0 = __ddiv_rn(__dmul_rn(kTwoPiTrunc, r.z), P.h);
  const double sarg = __dsub_rn(__ddiv_rn(__dsub_rn(beta0, P.BetaS), P.DeltaFai), 0.5);
  r.s0 = (int)ceil(sarg);
  const int s1 = r.s0 - P.half, s2 = r.s0 + P.half;
  if (zi < P.ZN && s1 < P.PN && s2 > 0) {
    r.lo = s1 < 0 ? 0 : s1;
    r.hi = s2 > P.PN - 1 ? P.PN - 1 : s2;
  } else {
    r.lo = 0x7fffffff;
    r.hi = -0x7fffffff;
  }
  return r;
}

// Per (column, view) quantities.
struct ColView {
  int U;          // channel of the upper tap
  double U1;      // Yr/dYL + YLC
  double denom;   // UU*temp1 + SO^2 - Yr^2
  double A, B;    // temp1 + UU, temp1 - UU
  double slope;   // SO SD / dZL / denom
};

__device__ __forceinline__ ColView col_view(const BpParams& P, double x, double y, const ViewTab& v) {
  ColView r;
  const double UU = __dsub_rn(__dmul_rn(-x, v.c), __dmul_rn(y, v.s));
  const double Yr = __dadd_rn(__dmul_rn(-x, v.s), __dmul_rn(y, v.c));
  const double Yr2 = __dmul_rn(Yr, Yr);
  const double temp1 = __dsqrt_rn(__dsub_rn(P.SO2, Yr2));
  r.denom = __dsub_rn(__dadd_rn(__dmul_rn(UU, temp1), P.SO2), Yr2);
  r.U1 = __dadd_rn(__ddiv_rn(Yr, P.dYL), P.YLC);
  r.U = (int)ceil(r.U1);
  r.A = __dadd_rn(temp1, UU);
  r.B = __dsub_rn(temp1, UU);
  r.slope = P.SOSDdZL / r.denom;
  return r;
}

// Row index V and its fraction Dez = V - V1, bit-exact to the reference.
__device__ __forceinline__ int row_index(const BpParams& P, const ColView& cv, double temp2, double& dez) {
  const double v1a = fma(temp2, cv.slope, P.ZLC);
  int V = (int)ceil(v1a);
  double d = (double)V - v1a;
  if (d < 1e-9 || d > 1.0 - 1e-9) {
    const double Zr = __ddiv_rn(__dmul_rn(temp2, P.SOSD), cv.denom);
    const double V1 = __dadd_rn(__ddiv_rn(Zr, P.dZL), P.ZLC);
    V = (int)ceil(V1);
    d = __dsub_rn((double)V, V1);
  }
  dez = d;
  return V;
}

// ---------------------------------------------------------------------------
// Plain form: FP32 filtered data, FP32 weights and accumulation.
// ---------------------------------------------------------------------------
template <int NZ>
__global__ void __launch_bounds__(kBx* kBy) bp_plain_kernel(float* __restrict__ vol, const float* __restrict__ fp,
                                                           const ViewTab* __restrict__ views,
                                                           const float* __restrict__ gw, BpParams P) {
  extern __shared__ float w_s[];  // [N_2pi]
  for (int t = threadIdx.y * kBx + threadIdx.x; t < P.N_2pi; t += kBx * kBy) w_s[t] = gw[t];
  __syncthreads();
  const int xi = blockIdx.x * kBx + threadIdx.x;
  const int yi = blockIdx.y * kBy + threadIdx.y;
  const int z0 = blockIdx.z * NZ;
  if (xi >= P.XN || yi >= P.YN) return;
  const double x = __dmul_rn(__dsub_rn((double)xi, P.XNC), P.dx);
  const double y = __dmul_rn(__dsub_rn((double)yi, P.YNC), P.dy);
  ZInfo zin[NZ];
  float res[NZ];
  int pstart = 0x7fffffff, pend = -0x7fffffff;
#pragma unroll
  for (int m = 0; m < NZ; ++m) {
    zin[m] = z_info(P, z0 + m);
    res[m] = 0.0f;
    pstart = min(pstart, zin[m].lo);
    pend = max(pend, zin[m].hi);
  }
  const size_t plane = (size_t)P.ZL * P.YL;
  for (int p = pstart; p <= pend; ++p) {
    const ViewTab v = views[p];
    const ColView cv = col_view(P, x, y, v);
    if (cv.U <= 0 || cv.U >= P.YL) continue;
    const float dey = (float)((double)cv.U - cv.U1);
    const float invA = 1.0f / (float)cv.A, invB = 1.0f / (float)cv.B;
    const float* col = fp + (size_t)p * plane + (cv.U - 1);
#pragma unroll
    for (int m = 0; m < NZ; ++m) {
      if (p < zin[m].lo || p > zin[m].hi) continue;
      const double temp2 = __dsub_rn(zin[m].z, v.hv);
      double dezd;
      const int V = row_index(P, cv, temp2, dezd);
      if (V <= 0 || V >= P.ZL) continue;
      const float dez = (float)dezd;
      const float* r0 = col + (size_t)(V - 1) * P.YL;
      const float* r1 = r0 + P.YL;
      const float ra = dey * __ldg(r0) + (1.0f - dey) * __ldg(r0 + 1);
      const float rb = dey * __ldg(r1) + (1.0f - dey) * __ldg(r1 + 1);
      const float touying = dez * ra + (1.0f - dez) * rb;
      const int before = p < zin[m].s0;
      const int d1 = (int)(P.N_pi - (double)(zin[m].s0 - p));
      const int d2 = before ? (int)(d1 + P.N_pi) : (int)(d1 - P.N_pi);
      const float w1 = w_s[d1], w2 = w_s[d2];
      const float t2 = (float)temp2;
      const float gama = fabsf(t2) * invA;
      const float gamac = fabsf(before ? t2 - 0.5f : t2 + 0.5f) * invB;
      const float e = exp2f(P.k1f * (log2f(gama) - log2f(gamac)));
      const float weight = w1 / (w1 + w2 * fminf(e, 3.0e38f));
      res[m] += weight * touying;
    }
  }
  float* out = vol + ((size_t)yi * P.XN + xi) * P.ZN + z0;
#pragma unroll
  for (int m = 0; m < NZ; ++m)
    if (z0 + m < P.ZN) out[m] = res[m] * P.DeltaFaif;
}

__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Plain form with the 3D weight factored (the same split as the fast form):
//   weight = w1 Gc^k1 / (w2 G^k1 + w1 Gc^k1) = 1 / (1 + Q2(view, slice) E(column, view))
//   Q2 = (w2 / w1) (|t2| / |t2 -/+ 0.5|)^k1,   E = ((temp1 - UU) / (temp1 + UU))^k1.
// Each CTA (one z block of NZ slices) first tabulates Q2 for its union view
// window in shared memory (FP64, -1 where the view is outside the slice's
// window), so an update costs one table read, one FMA and one reciprocal for
// its weight instead of two logarithms, an exponential and a division. Index
// selection (s0, windows, U, V) is unchanged: bit-exact to the reference.
template <int NZ>
__global__ void __launch_bounds__(kBx* kBy) bp_plain_q_kernel(float* __restrict__ vol, const float* __restrict__ fp,
                                                             const ViewTab* __restrict__ views,
                                                             const float* __restrict__ gw, BpParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* z_s = reinterpret_cast<double*>(smem_raw);        // [NZ] voxel z of the block's slices
  int* s0_s = reinterpret_cast<int*>(z_s + NZ);             // [NZ] central view
  int* lo_s = s0_s + NZ;                                     // [NZ] clamped window [lo, hi]
  int* hi_s = lo_s + NZ;                                     // [NZ]
  float* w_s = reinterpret_cast<float*>(hi_s + NZ);         // [N_2pi]
  float* q_s = w_s + P.N_2pi;                                // [qcap][NZ]
  const int tid = threadIdx.y * kBx + threadIdx.x;
  const int z0 = blockIdx.z * NZ;
  for (int t = tid; t < P.N_2pi; t += kBx * kBy) w_s[t] = gw[t];
  // the block's union window (uniform over the CTA; every thread evaluates it)
  int pstart = 0x7fffffff, pend = -0x7fffffff;
#pragma unroll
  for (int m = 0; m < NZ; ++m) {
    const ZInfo zi = z_info(P, z0 + m);
    if (tid == 0) {
      z_s[m] = zi.z;
      s0_s[m] = zi.s0;
      lo_s[m] = zi.lo;
      hi_s[m] = zi.hi;
    }
    pstart = min(pstart, zi.lo);
    pend = max(pend, zi.hi);
  }
  // views of the union window; 0 for a block whose slices all lie outside the
  // scan (pstart > pend: compared before subtracting, which would overflow).
  // The host sizes qcap from the same expressions; the clamp only keeps the
  // table in bounds.
  int len = pend >= pstart ? pend - pstart + 1 : 0;
  if (len > P.qcap) len = P.qcap;
  __syncthreads();  // w_s and the slice data
  for (int e = tid; e < len * NZ; e += kBx * kBy) {
    const int q = e / NZ, m = e - q * NZ;
    const int p = pstart + q;
    float qv = -1.0f;
    if (p >= lo_s[m] && p <= hi_s[m]) {
      const int before = p < s0_s[m];
      const int d1 = (int)(P.N_pi - (double)(s0_s[m] - p));
      const int d2 = before ? (int)(d1 + P.N_pi) : (int)(d1 - P.N_pi);
      const double w1 = w_s[d1], w2 = w_s[d2];
      const double t2 = __dsub_rn(z_s[m], views[p].hv);
      const double tc = before ? t2 - 0.5 : t2 + 0.5;
      qv = w2 == 0.0 ? 0.0f : (float)(w2 / w1 * pow(fabs(t2) / fabs(tc), P.k1));
    }
    q_s[e] = qv;
  }
  __syncthreads();
  const int xi = blockIdx.x * kBx + threadIdx.x;
  const int yi = blockIdx.y * kBy + threadIdx.y;
  if (xi >= P.XN || yi >= P.YN) return;
  const double x = __dmul_rn(__dsub_rn((double)xi, P.XNC), P.dx);
  const double y = __dmul_rn(__dsub_rn((double)yi, P.YNC), P.dy);
  float res[NZ];
#pragma unroll
  for (int m = 0; m < NZ; ++m) res[m] = 0.0f;
  const size_t plane = (size_t)P.ZL * P.YL;
  for (int q = 0; q < len; ++q) {
    const int p = pstart + q;
    const ViewTab v = views[p];
    const ColView cv = col_view(P, x, y, v);
    if (cv.U <= 0 || cv.U >= P.YL) continue;
    const float dey = (float)((double)cv.U - cv.U1);
    const float E = fminf(exp2f(P.k1f * log2f((float)cv.B / (float)cv.A)), 3.0e38f);
    const float* col = fp + (size_t)p * plane + (cv.U - 1);
    const float* qrow = q_s + q * NZ;
#pragma unroll
    for (int m = 0; m < NZ; ++m) {
      const float q2 = qrow[m];
      if (q2 < 0.0f) continue;  // view outside slice m's window (uniform over the CTA)
      const double temp2 = __dsub_rn(z_s[m], v.hv);
      double dezd;
      const int V = row_index(P, cv, temp2, dezd);
      if (V <= 0 || V >= P.ZL) continue;
      const float dez = (float)dezd;
      const float* r0 = col + (size_t)(V - 1) * P.YL;
      const float* r1 = r0 + P.YL;
      const float ra = dey * __ldg(r0) + (1.0f - dey) * __ldg(r0 + 1);
      const float rb = dey * __ldg(r1) + (1.0f - dey) * __ldg(r1 + 1);
      const float touying = dez * ra + (1.0f - dez) * rb;
      res[m] += rcp_approx(fmaf(q2, E, 1.0f)) * touying;
    }
  }
  float* out = vol + ((size_t)yi * P.XN + xi) * P.ZN + z0;
#pragma unroll
  for (int m = 0; m < NZ; ++m)
    if (z0 + m < P.ZN) out[m] = res[m] * P.DeltaFaif;
}

// ---------------------------------------------------------------------------
// FP64 form: the reference CPU's data path in double on the GPU.
// ---------------------------------------------------------------------------
template <int NZ>
__global__ void __launch_bounds__(kBx* kBy) bp_fp64_kernel(double* __restrict__ vol, const double* __restrict__ fp,
                                                          const ViewTab* __restrict__ views,
                                                          const double* __restrict__ gw, BpParams P) {
  extern __shared__ double wd_s[];  // [N_2pi]
  for (int t = threadIdx.y * kBx + threadIdx.x; t < P.N_2pi; t += kBx * kBy) wd_s[t] = gw[t];
  __syncthreads();
  const int xi = blockIdx.x * kBx + threadIdx.x;
  const int yi = blockIdx.y * kBy + threadIdx.y;
  const int z0 = blockIdx.z * NZ;
  if (xi >= P.XN || yi >= P.YN) return;
  const double x = __dmul_rn(__dsub_rn((double)xi, P.XNC), P.dx);
  const double y = __dmul_rn(__dsub_rn((double)yi, P.YNC), P.dy);
  ZInfo zin[NZ];
  double res[NZ];
  int pstart = 0x7fffffff, pend = -0x7fffffff;
#pragma unroll
  for (int m = 0; m < NZ; ++m) {
    zin[m] = z_info(P, z0 + m);
    res[m] = 0.0;
    pstart = min(pstart, zin[m].lo);
    pend = max(pend, zin[m].hi);
  }
  const size_t plane = (size_t)P.ZL * P.YL;
  for (int p = pstart; p <= pend; ++p) {
    const ViewTab v = views[p];
    const ColView cv = col_view(P, x, y, v);
    if (cv.U <= 0 || cv.U >= P.YL) continue;
    const double dey = __dsub_rn((double)cv.U, cv.U1);
    const double* col = fp + (size_t)p * plane + (cv.U - 1);
#pragma unroll
    for (int m = 0; m < NZ; ++m) {
      if (p < zin[m].lo || p > zin[m].hi) continue;
      const double temp2 = __dsub_rn(zin[m].z, v.hv);
      const double Zr = __ddiv_rn(__dmul_rn(temp2, P.SOSD), cv.denom);
      const double V1 = __dadd_rn(__ddiv_rn(Zr, P.dZL), P.ZLC);
      const int V = (int)ceil(V1);
      if (V <= 0 || V >= P.ZL) continue;
      const double dez = __dsub_rn((double)V, V1);
      const double* r0 = col + (size_t)(V - 1) * P.YL;
      const double* r1 = r0 + P.YL;
      const double touying = dey * dez * r0[0] + dey * (1.0 - dez) * r1[0] + (1.0 - dey) * dez * r0[1] +
                             (1.0 - dey) * (1.0 - dez) * r1[1];
      const int before = p < zin[m].s0;
      const int d1 = (int)(P.N_pi - (double)(zin[m].s0 - p));
      const int d2 = before ? (int)(d1 + P.N_pi) : (int)(d1 - P.N_pi);
      const double w1 = wd_s[d1], w2 = wd_s[d2];
      const double gama = fabs(temp2 / cv.A);
      const double gamac = before ? fabs((temp2 - 0.5) / cv.B) : fabs((temp2 + 0.5) / cv.B);
      const double m1 = pow(gama, P.k1);
      const double m2 = pow(gamac, P.k1);
      const double weight = (w1 * m2) / (w2 * m1 + w1 * m2);
      res[m] += weight * touying * P.DeltaFai;
    }
  }
  double* out = vol + ((size_t)yi * P.XN + xi) * P.ZN + z0;
#pragma unroll
  for (int m = 0; m < NZ; ++m)
    if (z0 + m < P.ZN) out[m] = res[m];
}

constexpr int kNzPlain = 8;
constexpr int kNzFp64 = 4;

// Checks a backprojection geometry and fills the kernels' parameter block. Every
// entry that backprojects (the plans and the allocation-free entry) goes through
// it, so they accept exactly the same geometries.
// The geometry checks of every backprojection entry (host only); *half: the window's half width.
int geom_checks(const hr_bp_geom* g, const char* who, int* half_out) {
  HR_REQUIRE(g->XN > 0 && g->YN > 0 && g->ZN > 0 && g->YL > 1 && g->ZL > 1 && g->PN > 0 && g->N_2pi > 1,
             "%s: invalid sizes", who);
  HR_REQUIRE(g->h != 0.0 && g->DeltaFai != 0.0 && g->dYL != 0.0 && g->dZL != 0.0 && g->SO > 0.0,
             "%s: h, DeltaFai, dYL, dZL must be non-zero and SO > 0", who);
  HR_REQUIRE((long long)g->XN * g->YN * g->ZN < (1LL << 40), "%s: volume too large", who);
  HR_REQUIRE(g->N_2pi <= 8192, "%s: N_2pi=%d exceeds 8192", who, g->N_2pi);
  // For views in [s0-half, s0+half] the weight indices are d1 = N_pi-(s0-p)
  // and d1 +/- N_pi; they stay inside [0, N_2pi) iff half <= N_pi and
  // N_pi + half <= N_2pi - 1 (the reference GPU kernel reads outside it).
  const int half = (int)std::ceil(g->N_pi * g->HSCoef);
  HR_REQUIRE(half >= 0 && (double)half <= g->N_pi && g->N_pi + half <= g->N_2pi - 1 &&
                 2.0 * g->N_pi <= g->N_2pi + 1e-9,
             "%s: HSCoef=%g, N_pi=%g give a view window outside the weight table", who, g->HSCoef, g->N_pi);
  *half_out = half;
  return HR_OK;
}

int bp_params_from_geom(const hr_bp_geom* g, const char* who, BpParams* out) {
  int half = 0;
  HR_TRY(geom_checks(g, who, &half));
  HR_TRY(hr::require_device());
  BpParams P{};
  P.XN = g->XN; P.YN = g->YN; P.ZN = g->ZN; P.YL = g->YL; P.ZL = g->ZL; P.PN = g->PN; P.N_2pi = g->N_2pi;
  P.half = half;
  P.XNC = g->XNC; P.YNC = g->YNC; P.ZNC = g->ZNC; P.dx = g->dx; P.dy = g->dy; P.dz = g->dz;
  P.YLC = g->YLC; P.ZLC = g->ZLC; P.dYL = g->dYL; P.dZL = g->dZL; P.h = g->h; P.BetaS = g->BetaS;
  P.DeltaFai = g->DeltaFai; P.N_pi = g->N_pi; P.SO = g->SO; P.SD = g->SD; P.k1 = g->k1;
  P.SO2 = g->SO * g->SO;
  P.SOSD = g->SO * g->SD;
  P.SOSDdZL = P.SOSD / g->dZL;
  P.k1f = (float)g->k1;
  P.DeltaFaif = (float)g->DeltaFai;
  // longest union view window of a z block of kNzPlain slices, with the
  // device's expressions for the central view and the clamped window
  P.qcap = 0;
  for (int z0 = 0; z0 < g->ZN; z0 += kNzPlain) {
    int a = 0x7fffffff, e = -0x7fffffff;
    for (int zi = z0; zi < z0 + kNzPlain && zi < g->ZN; ++zi) {
      const double z = (zi - g->ZNC) * g->dz;
      const double beta0 = kTwoPiTrunc * z / g->h;
      const int s0 = (int)std::ceil((beta0 - g->BetaS) / g->DeltaFai - 0.5);
      const int s1 = s0 - half, s2 = s0 + half;
      if (s1 < g->PN && s2 > 0) {
        a = std::min(a, s1 < 0 ? 0 : s1);
        e = std::max(e, s2 > g->PN - 1 ? g->PN - 1 : s2);
      }
    }
    if (e >= a) P.qcap = std::max(P.qcap, e - a + 1);
  }
  *out = P;
  return HR_OK;
}

// Dynamic shared memory of bp_plain_q_kernel.
size_t plain_q_smem(const BpParams& P) {
  return sizeof(double) * kNzPlain + 3 * sizeof(int) * kNzPlain + sizeof(float) * P.N_2pi +
         sizeof(float) * (size_t)P.qcap * kNzPlain;
}
// Above this the per-CTA weight table would cost too much occupancy (very
// thick slices: long union windows); the per-update weight kernel runs instead.
constexpr size_t kPlainQSmemMax = 96 * 1024;

// The plain-form launch of both the plan and the allocation-free entry (the
// same kernel for the same geometry, so their results are identical).
int launch_plain(const BpParams& P, float* vol, const float* fp, const ViewTab* views, const float* w,
                 cudaStream_t s) {
  dim3 grid((P.XN + kBx - 1) / kBx, (P.YN + kBy - 1) / kBy, (P.ZN + kNzPlain - 1) / kNzPlain);
  HR_REQUIRE(grid.z <= 65535 && grid.y <= 65535, "backprojection: grid too large");
  const size_t qsmem = plain_q_smem(P);
  if (P.qcap > 0 && qsmem <= kPlainQSmemMax) {
    HR_CUDA_TRY(cudaFuncSetAttribute(bp_plain_q_kernel<kNzPlain>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)qsmem));
    bp_plain_q_kernel<kNzPlain><<<grid, dim3(kBx, kBy), qsmem, s>>>(vol, fp, views, w, P);
  } else {
    bp_plain_kernel<kNzPlain><<<grid, dim3(kBx, kBy), sizeof(float) * P.N_2pi, s>>>(vol, fp, views, w, P);
  }
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}

// Per-view tables in the reference's own arithmetic
// (src/Parallel_FDK_Helical_3DWeighting.cpp:73, :76-79): the host C library's
// cos/sin, which the bit-exact index selection depends on.
void fill_view_table(ViewTab* tab, int PN, double BetaS, double DeltaFai, double h) {
  for (int p = 0; p < PN; ++p) {
    const double View = BetaS + p * DeltaFai;
    tab[p] = ViewTab{std::cos(View), std::sin(View), h * View * kInvTwoPi};
  }
}

}  // namespace

void hr::fast_geom_fill(const hr_bp_geom& g, int half, BpFastGeom* f) {
  f->XN = g.XN; f->YN = g.YN; f->ZN = g.ZN; f->YL = g.YL; f->ZL = g.ZL; f->PN = g.PN; f->half = half;
  f->XNC = g.XNC; f->YNC = g.YNC; f->ZNC = g.ZNC; f->dx = g.dx; f->dy = g.dy; f->dz = g.dz;
  f->YLC = g.YLC; f->ZLC = g.ZLC; f->dYL = g.dYL; f->dZL = g.dZL; f->h = g.h; f->BetaS = g.BetaS;
  f->DeltaFai = g.DeltaFai; f->N_pi = g.N_pi; f->SO = g.SO; f->SD = g.SD; f->k1 = g.k1;
  f->ZN_valid = g.ZN;
}

int hr::fast_geom_of(const hr_bp_geom& g, BpFastGeom* f) {
  int half = 0;
  HR_TRY(geom_checks(&g, "backprojection", &half));
  fast_geom_fill(g, half, f);
  return HR_OK;
}

extern "C" int hr_bp_plan_create(hr_bp_plan** plan, const hr_bp_geom* g, const double* w, int form) {
  hr::clear_error();
  HR_REQUIRE(plan != nullptr && g != nullptr && w != nullptr, "hr_bp_plan_create: NULL argument");
  *plan = nullptr;
  HR_REQUIRE(form == HR_FORM_PLAIN || form == HR_FORM_FP64 || form == HR_FORM_FAST,
             "hr_bp_plan_create: unknown form %d", form);
  BpParams P{};
  HR_TRY(bp_params_from_geom(g, "backprojection", &P));
  const int half = P.half;

  std::vector<ViewTab> tab(g->PN);
  fill_view_table(tab.data(), g->PN, g->BetaS, g->DeltaFai, g->h);
  std::vector<float> wf(g->N_2pi);
  for (int i = 0; i < g->N_2pi; ++i) wf[i] = (float)w[i];

  hr_bp_plan* pl = new hr_bp_plan{P, form, nullptr, nullptr, nullptr, hr::BpFastGeom{}, hr::BpFast{}};
  if (form == HR_FORM_FAST) {
    hr::fast_geom_fill(*g, half, &pl->fg);
    const int st = hr::bp_fast_create(&pl->fast, pl->fg, w);
    if (st != HR_OK) {
      hr::bp_fast_destroy(&pl->fast);
      delete pl;
      return st;
    }
    *plan = pl;
    return HR_OK;
  }
  cudaError_t e = cudaMalloc(&pl->d_views, sizeof(ViewTab) * g->PN);
  if (e == cudaSuccess) e = cudaMalloc(&pl->d_w, sizeof(float) * g->N_2pi);
  if (e == cudaSuccess) e = cudaMalloc(&pl->d_wd, sizeof(double) * g->N_2pi);
  if (e == cudaSuccess) e = cudaMemcpy(pl->d_views, tab.data(), sizeof(ViewTab) * g->PN, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(pl->d_w, wf.data(), sizeof(float) * g->N_2pi, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(pl->d_wd, w, sizeof(double) * g->N_2pi, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(pl->d_views);
    cudaFree(pl->d_w);
    cudaFree(pl->d_wd);
    delete pl;
    return hr::fail(e == cudaErrorMemoryAllocation ? HR_ERR_OUT_OF_MEMORY : HR_ERR_CUDA, "bp plan: %s",
                    cudaGetErrorString(e));
  }
  *plan = pl;
  return HR_OK;
}

extern "C" int hr_bp_execute(const hr_bp_plan* pl, void* d_vol, const void* d_fp, void* stream) {
  HR_REQUIRE(pl != nullptr && d_vol != nullptr && d_fp != nullptr, "hr_bp_execute: NULL argument");
  const BpParams& P = pl->prm;
  cudaStream_t s = hr::as_stream(stream);
  if (pl->form == HR_FORM_FAST)
    return hr::bp_fast_execute(pl->fast, pl->fg, static_cast<float*>(d_vol), static_cast<const uint32_t*>(d_fp), s);
  if (pl->form == HR_FORM_PLAIN)
    return launch_plain(P, static_cast<float*>(d_vol), static_cast<const float*>(d_fp), pl->d_views, pl->d_w, s);
  {
    dim3 grid((P.XN + kBx - 1) / kBx, (P.YN + kBy - 1) / kBy, (P.ZN + kNzFp64 - 1) / kNzFp64);
    HR_REQUIRE(grid.z <= 65535 && grid.y <= 65535, "backprojection: grid too large");
    bp_fp64_kernel<kNzFp64><<<grid, dim3(kBx, kBy), sizeof(double) * P.N_2pi, s>>>(
        static_cast<double*>(d_vol), static_cast<const double*>(d_fp), pl->d_views, pl->d_wd, P);
  }
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}

int hr::bp_plan_fast_parts(const hr_bp_plan* pl, const BpFastGeom** g, const BpFast** f) {
  HR_REQUIRE(pl != nullptr && pl->form == HR_FORM_FAST, "backprojection plan is not of the fast form");
  *g = &pl->fg;
  *f = &pl->fast;
  return HR_OK;
}

extern "C" int hr_bp_autotune(hr_bp_plan* pl, void* d_vol, const void* d_fp, void* stream) {
  HR_REQUIRE(pl != nullptr && d_vol != nullptr && d_fp != nullptr, "hr_bp_autotune: NULL argument");
  if (pl->form != HR_FORM_FAST) return HR_OK;
  return hr::bp_fast_autotune(&pl->fast, pl->fg, static_cast<float*>(d_vol), static_cast<const uint32_t*>(d_fp),
                              hr::as_stream(stream));
}

extern "C" int hr_bp_select(hr_bp_plan* pl, int variant) {
  HR_REQUIRE(pl != nullptr, "hr_bp_select: NULL plan");
  if (pl->form != HR_FORM_FAST) return variant == 0 ? HR_OK : hr::fail(HR_ERR_INVALID_ARGUMENT, "hr_bp_select: "
                                                                        "only the fast form has variants");
  HR_REQUIRE(variant >= 0 && variant < hr::kFastVariants_n, "hr_bp_select: variant %d out of range [0, %d)",
             variant, hr::kFastVariants_n);
  pl->fast.variant = variant;
  return hr::bp_fast_tex_prepare(&pl->fast, pl->fg);
}

extern "C" int hr_bp_describe(const hr_bp_plan* pl, char* buf, int len) {
  HR_REQUIRE(pl != nullptr, "hr_bp_describe: NULL plan");
  if (pl->form == HR_FORM_FAST) return hr::bp_fast_describe(pl->fast, buf, len);
  if (buf && len > 0)
    snprintf(buf, (size_t)len, "%s slices_per_thread=%d tile=%dx%d%s", pl->form == HR_FORM_FP64 ? "fp64" : "plain",
             pl->form == HR_FORM_FP64 ? kNzFp64 : kNzPlain, kBx, kBy,
             pl->form == HR_FORM_FP64 ? ""
             : pl->prm.qcap > 0 && plain_q_smem(pl->prm) <= kPlainQSmemMax ? " weights=per-block table"
                                                                            : " weights=per update");
  return HR_OK;
}

extern "C" void hr_bp_plan_destroy(hr_bp_plan* pl) {
  if (!pl) return;
  hr::bp_fast_destroy(&pl->fast);
  cudaFree(pl->d_views);
  cudaFree(pl->d_w);
  cudaFree(pl->d_wd);
  delete pl;
}

// ---------------------------------------------------------------------------
// Plain-form backprojection that allocates nothing.
//
// Some callers cannot call cudaMalloc: streaming pipelines that must not
// allocate once they run, because cudaMalloc and cudaFree synchronise the whole
// device and would stall the other streams; hosts whose pooling allocator owns
// all device memory (a MATLAB session, a framework's caching allocator), where
// a second allocator fragments or exhausts the pool; and services that run
// under a fixed device-memory budget. This entry keeps its only scratch -- the
// per-view cos/sin/source-height table -- in a file-scope device array of
// kNoAllocMaxViews entries (768 KiB, held by every GPU that loads the library
// until the process exits) and takes everything else (filtered data, weight
// table, volume) from the caller.
//
// The table is computed on the host with the same C library calls as the plan
// (fill_view_table) and copied into the array, so both entries select the same
// view/row/channel indices and give bit-identical volumes.
// ---------------------------------------------------------------------------
#include <mutex>

namespace {
constexpr int kNoAllocMaxViews = 32768;
constexpr int kNoAllocMaxDevices = 64;
}  // namespace

static __device__ __align__(256) ViewTab g_noalloc_views[kNoAllocMaxViews];

namespace {

std::mutex g_noalloc_mutex;
ViewTab* g_noalloc_ptr[kNoAllocMaxDevices] = {};
// Host staging of the table (pageable, file scope: filled and copied under
// g_noalloc_mutex).
ViewTab g_noalloc_host[kNoAllocMaxViews];

// Device address of g_noalloc_views on the current device, looked up once per
// device (with that device current). In host code the array's name is only a
// host-side stand-in, never a device address. Called with g_noalloc_mutex held.
int noalloc_views(ViewTab** out) {
  int dev = 0;
  HR_CUDA_TRY(cudaGetDevice(&dev));
  HR_REQUIRE(dev >= 0 && dev < kNoAllocMaxDevices, "hr_bp_plain_noalloc: device %d out of range", dev);
  if (g_noalloc_ptr[dev] == nullptr) {
    void* p = nullptr;
    HR_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_views));
    g_noalloc_ptr[dev] = static_cast<ViewTab*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return HR_OK;
}

}  // namespace

extern "C" int hr_bp_plain_noalloc(float* d_vol, const float* d_fp, const float* d_w, const hr_bp_geom* g,
                                   void* stream) {
  hr::clear_error();
  HR_REQUIRE(d_vol != nullptr && d_fp != nullptr && d_w != nullptr && g != nullptr,
             "hr_bp_plain_noalloc: NULL argument");
  HR_REQUIRE(g->PN <= kNoAllocMaxViews,
             "hr_bp_plain_noalloc: PN=%d views exceed the fixed scratch table of %d views (use hr_bp_plan_create)",
             g->PN, kNoAllocMaxViews);
  BpParams P{};
  HR_TRY(bp_params_from_geom(g, "hr_bp_plain_noalloc", &P));
  cudaStream_t s = hr::as_stream(stream);
  ViewTab* views = nullptr;
  {
    // A copy from pageable host memory returns once the data are staged, so
    // the host buffer may be refilled by the next call as soon as it returns.
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    HR_TRY(noalloc_views(&views));
    fill_view_table(g_noalloc_host, P.PN, P.BetaS, P.DeltaFai, P.h);
    HR_CUDA_TRY(cudaMemcpyAsync(views, g_noalloc_host, sizeof(ViewTab) * P.PN, cudaMemcpyHostToDevice, s));
  }
  return launch_plain(P, d_vol, d_fp, views, d_w, s);
}
