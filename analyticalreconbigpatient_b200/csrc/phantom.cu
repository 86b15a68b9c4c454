// Analytic FP64 projector of ellipsoid / elliptic-cylinder phantoms onto the
// helical curved-detector fan geometry (synthetic data source; the reference
// ships no data). One thread per detector sample (view i, channel j, row k),
// k fastest so that a warp writes contiguous rows.
//
// Fan view i: source angle beta = BetaS + i dBeta at S = (SO cos beta,
// SO sin beta, h beta / 2pi). Channel j: fan angle gamma = (j - YLC0) dYA; the
// ray's in-plane direction is -(cos(beta - gamma), sin(beta - gamma)), i.e.
// parallel view angle beta - gamma, which is the relation the rebinning
// inverts (Fai = Theta + asin(t/SO), src/ParallelRebinningCBCurve.cpp:37-39).
// Row k: the ray rises (k - ZLC0) dZL over the in-plane distance SD.
#include <algorithm>
#include <cmath>

#include "hr_internal.h"

namespace {

constexpr int kObjStride = 17;

__device__ double chord(const double* o, const double S[3], const double D[3], double Dn) {
  const double p0[3] = {S[0] - o[1], S[1] - o[2], S[2] - o[3]};
  const double* R = o + 7;
  double q0[3], q1[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    q0[i] = R[0 * 3 + i] * p0[0] + R[1 * 3 + i] * p0[1] + R[2 * 3 + i] * p0[2];
    q1[i] = R[0 * 3 + i] * D[0] + R[1 * 3 + i] * D[1] + R[2 * 3 + i] * D[2];
  }
  const int type = (int)o[0];
  const int nd = type == 1 ? 2 : 3;
  double A = 0.0, B = 0.0, C = -1.0;
  for (int i = 0; i < nd; ++i) {
    const double u0 = q0[i] / o[4 + i], u1 = q1[i] / o[4 + i];
    A += u1 * u1;
    B += u0 * u1;
    C += u0 * u0;
  }
  if (A <= 0.0) return 0.0;
  const double disc = B * B - A * C;
  if (disc <= 0.0) return 0.0;
  const double sq = sqrt(disc);
  double lo = (-B - sq) / A, hi = (-B + sq) / A;
  if (type == 1) {
    const double zlo = o[3] - o[6], zhi = o[3] + o[6];
    if (D[2] == 0.0) {
      if (S[2] < zlo || S[2] > zhi) return 0.0;
    } else {
      double t0 = (zlo - S[2]) / D[2], t1 = (zhi - S[2]) / D[2];
      if (t0 > t1) {
        const double tt = t0;
        t0 = t1;
        t1 = tt;
      }
      lo = fmax(lo, t0);
      hi = fmin(hi, t1);
    }
    if (hi <= lo) return 0.0;
  }
  return (hi - lo) * Dn;
}

__global__ void __launch_bounds__(256) project_kernel(float* __restrict__ proj, int YL, int ZL, int ViewN, double SO,
                                                      double SD, double dYA, double YLC0, double dZL, double ZLC0,
                                                      double BetaS, double dBeta, double h,
                                                      const double* __restrict__ gobj, int nobj) {
  extern __shared__ double obj[];
  for (int t = threadIdx.x; t < nobj * kObjStride; t += blockDim.x) obj[t] = gobj[t];
  __syncthreads();
  const int jk = blockIdx.x * blockDim.x + threadIdx.x;
  if (jk >= YL * ZL) return;
  const int j = jk / ZL, k = jk - j * ZL;
  const double gam = (j - YLC0) * dYA;
  const double slope = (k - ZLC0) * dZL / SD;
  const double Dn = sqrt(1.0 + slope * slope);
  for (int i = blockIdx.y; i < ViewN; i += gridDim.y) {
    const double beta = BetaS + i * dBeta;
    double sb, cb, st, ct;
    sincos(beta, &sb, &cb);
    sincos(beta - gam, &st, &ct);
    const double S[3] = {SO * cb, SO * sb, h * beta / (2.0 * M_PI)};
    const double D[3] = {-ct, -st, slope};
    double acc = 0.0;
    for (int e = 0; e < nobj; ++e) acc += obj[e * kObjStride + 16] * chord(obj + e * kObjStride, S, D, Dn);
    proj[((size_t)i * YL + j) * ZL + k] = (float)acc;
  }
}

// ---- Poisson photon noise ---------------------------------------------------
// Counter-based stream: draw j of sample i is splitmix64 of a per-sample state,
// so the result does not depend on the launch shape.
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long& x) {
  unsigned long long z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ double uniform01(unsigned long long& st) {
  return (double)(splitmix64(st) >> 11) * 0x1.0p-53;  // [0, 1)
}

// Poisson(lam). lam < 10: multiplication of uniforms (Knuth); otherwise the
// transformed rejection method with squeeze, PTRS (W. Hoermann, "The
// transformed rejection method for generating Poisson random variables",
// Insurance: Mathematics and Economics 12, 1993). Both loops are bounded; their
// expected iteration counts are lam + 1 < 11 and about 1.1.
__device__ double poisson(double lam, unsigned long long& st) {
  if (!(lam > 0.0)) return 0.0;
  if (lam < 10.0) {
    const double L = exp(-lam);
    double prod = uniform01(st);
    int k = 0;
    while (prod > L && k < 1000) {
      prod *= uniform01(st);
      ++k;
    }
    return (double)k;
  }
  const double slam = sqrt(lam), loglam = log(lam);
  const double b = 0.931 + 2.53 * slam;
  const double a = -0.059 + 0.02483 * b;
  const double inv_alpha = 1.1239 + 1.1328 / (b - 3.4);
  const double vr = 0.9277 - 3.6224 / (b - 2.0);
  for (int it = 0; it < 1000; ++it) {
    const double U = uniform01(st) - 0.5;
    const double V = uniform01(st);
    const double us = 0.5 - fabs(U);
    const double k = floor((2.0 * a / us + b) * U + lam + 0.43);
    if (us >= 0.07 && V <= vr) return k;
    if (k < 0.0 || (us < 0.013 && V > us)) continue;
    if (log(V) + log(inv_alpha) - log(a / (us * us) + b) <= -lam + k * loglam - lgamma(k + 1.0)) return k;
  }
  return floor(lam + 0.5);  // not reached in practice (acceptance > 0.9 per draw)
}

// p -> -log(max(N, 1) / I0) with N ~ Poisson(I0 exp(-p)): line integrals with
// the photon noise of a transmission measurement at I0 photons per ray.
__global__ void poisson_noise_kernel(float* __restrict__ proj, long long n, double I0, unsigned long long seed) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    unsigned long long st = seed ^ (0xD1B54A32D192ED03ull * (unsigned long long)(i + 1));
    splitmix64(st);
    const double N = poisson(I0 * exp(-(double)proj[i]), st);
    proj[i] = (float)-log(fmax(N, 1.0) / I0);
  }
}

}  // namespace

extern "C" int hr_project_ellipsoids(float* d_proj, int YL, int ZL, int ViewN, double SO, double SD, double dYA,
                                     double YLC0, double dZL, double ZLC0, double BetaS, double dBeta, double h,
                                     const double* d_obj, int nobj, void* stream) {
  hr::clear_error();
  HR_REQUIRE(d_proj != nullptr && (d_obj != nullptr || nobj == 0), "hr_project_ellipsoids: NULL argument");
  HR_REQUIRE(YL > 0 && ZL > 0 && ViewN > 0 && nobj >= 0, "hr_project_ellipsoids: invalid sizes");
  HR_REQUIRE((long long)YL * ZL < (1LL << 31), "hr_project_ellipsoids: YL*ZL too large");
  const size_t smem = sizeof(double) * kObjStride * (size_t)nobj;
  HR_REQUIRE(smem <= 200 * 1024, "hr_project_ellipsoids: %d objects exceed the shared-memory table", nobj);
  if (smem > 48 * 1024)
    HR_CUDA_TRY(cudaFuncSetAttribute(project_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid((YL * ZL + 255) / 256, ViewN < 65535 ? ViewN : 65535);
  project_kernel<<<grid, 256, smem, hr::as_stream(stream)>>>(d_proj, YL, ZL, ViewN, SO, SD, dYA, YLC0, dZL, ZLC0,
                                                             BetaS, dBeta, h, d_obj, nobj);
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}

extern "C" int hr_add_poisson_noise(float* d_proj, long long n, double I0, unsigned long long seed, void* stream) {
  hr::clear_error();
  HR_REQUIRE(d_proj != nullptr || n == 0, "hr_add_poisson_noise: NULL data");
  HR_REQUIRE(n >= 0 && I0 >= 1.0, "hr_add_poisson_noise: need n >= 0 and I0 >= 1");
  if (n == 0) return HR_OK;
  const long long blocks = std::min<long long>((n + 255) / 256, 8LL * hr::sm_count());
  poisson_noise_kernel<<<(unsigned)blocks, 256, 0, hr::as_stream(stream)>>>(d_proj, n, I0, seed);
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}
