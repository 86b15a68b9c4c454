// Cosine preweight + Shepp-Logan ramp filter, FP32, cuFFT-free.
//
// Reference: src/filtering.cu:187-207 (preweight), :15-25 and :57-84 (kernel
// h[n] = -2/(pi^2 (4n^2-1))/dYL, n = -YL..YL, wrapped into NN = 2^ceil(log2 3YL)
// and transformed), :86-175 (zero-pad, C2C FFT, multiply, inverse, keep the
// first YL samples / NN); CPU spec src/analyticalReconBigPatient.m:107-134.
//
// The reference computes a linear convolution f[j] = sum_m p[m] h[j-m] with
// |j-m| <= YL-1 through a length-NN circular one. Any circular length
// N >= 2 YL - 1 gives the same linear convolution, so this filter uses
// N = 2^ceil(log2(2 YL - 1)) (2048 for YL = 888, the reference pads to 4096).
// h is even, so its transform H is real; two real rows a, b are filtered at
// once as one complex signal a + i b:  ifft(H fft(a + i b)) = (h*a) + i (h*b).
// The inverse transform is done with the forward one: ifft(Z) =
// conj(fft(conj(Z)))/N, with 1/N folded into H.
//
// Kernel shape: persistent CTAs (256 threads) keep the twiddle and H tables
// in shared memory and loop over tiles of 2*RP rows. A tile is loaded with the
// preweight applied, transformed in shared memory by a Stockham radix-4 (+ one
// radix-2) FFT that ping-pongs between two buffers, filtered, transformed
// again and stored. The input may be in the reference's row
// layout [v][ZL][YL] or in the rebinning's layout [v][YL][ZL]; for the latter
// the 4 rows of a tile are 16 contiguous bytes per channel.
#include <cmath>
#include <vector>

#include "hr_internal.h"

struct hr_filter_plan {
  int YL, ZL, ViewN, log2N;
  float PLC, ZLC, dYL, dZL, SO;
  float* d_H;    // real spectrum of the wrapped kernel, divided by N
  float2* d_tw;  // exp(-2 pi i t / N), t in [0, N)
};

namespace {

constexpr int kThreads = 256;
constexpr int kRowPairs = 2;  // row pairs per tile

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// One Stockham stage of radix R over `pairs` transforms of length N stored
// back to back. Butterfly jb of a transform reads src[jb + r N/R], applies
// twiddles W_{Ns R}^{r k} (k = jb mod Ns), does a length-R DFT and writes
// dst[(jb/Ns) Ns R + k + r Ns]. src and dst are distinct shared buffers.
template <int N, int R>
__device__ __forceinline__ void stockham_stage(const float2* __restrict__ src, float2* __restrict__ dst,
                                               const float2* __restrict__ tw, int Ns, int pairs) {
  constexpr int NB = N / R;  // butterflies per transform
  const int total = pairs * NB;
  const int stride = N / (Ns * R);
  for (int u = threadIdx.x; u < total; u += kThreads) {
    const int p = u / NB, jb = u - p * NB;
    const int k = jb % Ns;
    const float2* s = src + p * N + jb;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      float2 x = s[r * NB];
      if (r > 0) x = cmul(x, tw[r * k * stride]);
      v[r] = x;
    }
    if constexpr (R == 4) {
      const float2 a0 = make_float2(v[0].x + v[2].x, v[0].y + v[2].y);
      const float2 a1 = make_float2(v[0].x - v[2].x, v[0].y - v[2].y);
      const float2 a2 = make_float2(v[1].x + v[3].x, v[1].y + v[3].y);
      const float2 a3 = make_float2(v[1].y - v[3].y, -(v[1].x - v[3].x));  // (v1 - v3) * (-i)
      v[0] = make_float2(a0.x + a2.x, a0.y + a2.y);
      v[1] = make_float2(a1.x + a3.x, a1.y + a3.y);
      v[2] = make_float2(a0.x - a2.x, a0.y - a2.y);
      v[3] = make_float2(a1.x - a3.x, a1.y - a3.y);
    } else {
      const float2 a0 = v[0], a1 = v[1];
      v[0] = make_float2(a0.x + a1.x, a0.y + a1.y);
      v[1] = make_float2(a0.x - a1.x, a0.y - a1.y);
    }
    float2* d = dst + p * N + (jb / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) d[r * Ns] = v[r];
  }
  __syncthreads();
}

// Forward FFT of `pairs` transforms held in X; Y is scratch of the same size.
// Returns the buffer that holds the result.
template <int LOG2N>
__device__ __forceinline__ float2* fft_forward(float2* X, float2* Y, const float2* tw, int pairs) {
  constexpr int N = 1 << LOG2N;
  int Ns = 1;
#pragma unroll
  for (int s = 0; s < LOG2N / 2; ++s) {
    stockham_stage<N, 4>(X, Y, tw, Ns, pairs);
    float2* t = X;
    X = Y;
    Y = t;
    Ns *= 4;
  }
  if constexpr (LOG2N % 2 == 1) {
    stockham_stage<N, 2>(X, Y, tw, Ns, pairs);
    X = Y;
  }
  return X;
}

template <int LOG2N, int IN_LAYOUT>
__global__ void __launch_bounds__(kThreads) filter_fft_kernel(float* __restrict__ out, const float* __restrict__ in,
                                                              const float* __restrict__ gH,
                                                              const float2* __restrict__ gtw, int YL, int ZL,
                                                              int ViewN, int view0, float PLC, float ZLC, float dYL,
                                                              float dZL, float SO) {
  constexpr int N = 1 << LOG2N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* X0 = reinterpret_cast<float2*>(smem_raw);  // [kRowPairs][N]
  float2* X1 = X0 + kRowPairs * N;                   // [kRowPairs][N] ping-pong partner
  float2* tw = X1 + kRowPairs * N;                   // [N]
  float* H = reinterpret_cast<float*>(tw + N);      // [N]
  for (int t = threadIdx.x; t < N; t += kThreads) {
    tw[t] = gtw[t];
    H[t] = gH[t];
  }
  const long long rows = (long long)ZL * ViewN;
  const long long tiles = (rows + 2 * kRowPairs - 1) / (2 * kRowPairs);
  const float SO2 = SO * SO;
  for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const long long r0 = tile * 2 * kRowPairs;
    const int nrows = (int)((rows - r0) < 2 * kRowPairs ? (rows - r0) : 2 * kRowPairs);
    const int pairs = (nrows + 1) / 2;
    float2* X = X0;
    __syncthreads();  // previous tile's stores have read the buffers
    // ---- load + preweight -------------------------------------------------
    if constexpr (IN_LAYOUT == HR_LAYOUT_ROWS) {
      for (int q = 0; q < 2 * kRowPairs; ++q) {
        const long long r = r0 + q;
        const int k = (int)(r % ZL);
        const long long v = r / ZL;
        const float b = ((float)k - ZLC) * dZL;
        const float* src = in + ((size_t)(view0 + v) * ZL + k) * YL;
        float* dstc = reinterpret_cast<float*>(X + (q >> 1) * N) + (q & 1);
        for (int j = threadIdx.x; j < N; j += kThreads) {
          float val = 0.0f;
          if (q < nrows && j < YL) {
            const float t = ((float)j - PLC) * dYL;
            const float wei = SO2 / sqrtf(SO2 * (SO2 + b * b) - b * t * b * t);
            val = src[j] * wei;
          }
          dstc[2 * j] = val;
        }
      }
    } else {
      // [v][YL][ZL]: 2*kRowPairs consecutive rows k of one channel are contiguous.
      for (int e = threadIdx.x; e < N * 2 * kRowPairs; e += kThreads) {
        const int q = e % (2 * kRowPairs);
        const int j = e / (2 * kRowPairs);
        float val = 0.0f;
        if (q < nrows && j < YL) {
          const long long r = r0 + q;
          const int k = (int)(r % ZL);
          const long long v = r / ZL;
          const float b = ((float)k - ZLC) * dZL;
          const float t = ((float)j - PLC) * dYL;
          const float wei = SO2 / sqrtf(SO2 * (SO2 + b * b) - b * t * b * t);
          val = in[((size_t)(view0 + v) * YL + j) * ZL + k] * wei;
        }
        reinterpret_cast<float*>(X + (q >> 1) * N)[2 * j + (q & 1)] = val;
      }
    }
    __syncthreads();
    X = fft_forward<LOG2N>(X, X == X0 ? X1 : X0, tw, pairs);
    // Z = H/N * conj(X)
    for (int e = threadIdx.x; e < pairs * N; e += kThreads) {
      const float hk = H[e & (N - 1)];
      const float2 x = X[e];
      X[e] = make_float2(hk * x.x, -hk * x.y);
    }
    __syncthreads();
    X = fft_forward<LOG2N>(X, X == X0 ? X1 : X0, tw, pairs);
    // result = conj(fft(Z)): row a = Re, row b = -Im
    for (int q = 0; q < nrows; ++q) {
      const long long r = r0 + q;
      float* dst = out + (size_t)r * YL;
      const float* srcc = reinterpret_cast<const float*>(X + (q >> 1) * N) + (q & 1);
      const float sign = (q & 1) ? -1.0f : 1.0f;
      for (int j = threadIdx.x; j < YL; j += kThreads) dst[j] = sign * srcc[2 * j];
    }
  }
}

size_t smem_bytes(int log2N) {
  const size_t N = (size_t)1 << log2N;
  return 2 * kRowPairs * N * sizeof(float2) + N * sizeof(float2) + N * sizeof(float);
}

template <int LOG2N, int IN_LAYOUT>
int launch_t(const hr_filter_plan* p, float* out, const float* in, int view0, cudaStream_t s) {
  auto kern = filter_fft_kernel<LOG2N, IN_LAYOUT>;
  const size_t smem = smem_bytes(LOG2N);
  HR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long rows = (long long)p->ZL * p->ViewN;
  const long long tiles = (rows + 2 * kRowPairs - 1) / (2 * kRowPairs);
  int per_sm = 0;
  HR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem));
  if (per_sm < 1) per_sm = 1;
  const long long want = (long long)per_sm * hr::sm_count();
  const int grid = (int)(tiles < want ? tiles : want);
  kern<<<grid, kThreads, smem, s>>>(out, in, p->d_H, p->d_tw, p->YL, p->ZL, p->ViewN, view0, p->PLC, p->ZLC, p->dYL,
                                    p->dZL, p->SO);
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}

template <int IN_LAYOUT>
int launch_layout(const hr_filter_plan* p, float* out, const float* in, int view0, cudaStream_t s) {
  switch (p->log2N) {
    case 3: return launch_t<3, IN_LAYOUT>(p, out, in, view0, s);
    case 4: return launch_t<4, IN_LAYOUT>(p, out, in, view0, s);
    case 5: return launch_t<5, IN_LAYOUT>(p, out, in, view0, s);
    case 6: return launch_t<6, IN_LAYOUT>(p, out, in, view0, s);
    case 7: return launch_t<7, IN_LAYOUT>(p, out, in, view0, s);
    case 8: return launch_t<8, IN_LAYOUT>(p, out, in, view0, s);
    case 9: return launch_t<9, IN_LAYOUT>(p, out, in, view0, s);
    case 10: return launch_t<10, IN_LAYOUT>(p, out, in, view0, s);
    case 11: return launch_t<11, IN_LAYOUT>(p, out, in, view0, s);
    case 12: return launch_t<12, IN_LAYOUT>(p, out, in, view0, s);
    default: return hr::fail(HR_ERR_UNSUPPORTED, "filter: transform length 2^%d unsupported", p->log2N);
  }
}

}  // namespace

extern "C" int hr_filter_plan_create(hr_filter_plan** plan, int YL, int ZL, int ViewN, float PLC, float ZLC,
                                     float dYL, float dZL, float SO) {
  hr::clear_error();
  HR_REQUIRE(plan != nullptr, "hr_filter_plan_create: plan is NULL");
  *plan = nullptr;
  HR_REQUIRE(YL > 1 && ZL > 0 && ViewN > 0, "filter: invalid sizes (YL=%d ZL=%d ViewN=%d)", YL, ZL, ViewN);
  HR_REQUIRE(YL <= 2048, "filter: YL=%d exceeds 2048", YL);
  HR_REQUIRE(dYL != 0.0f && SO > 0.0f, "filter: dYL must be non-zero and SO > 0");
  HR_TRY(hr::require_device());
  int log2N = 3;
  while ((1 << log2N) < 2 * YL - 1) ++log2N;
  const int N = 1 << log2N;
  // Wrapped kernel and its (real) spectrum, in double.
  std::vector<double> hs(N, 0.0);
  const double pi2 = M_PI * M_PI;
  for (int n = 0; n < YL; ++n) {
    const double hn = -2.0 / (pi2 * (4.0 * n * n - 1.0)) / (double)dYL;
    hs[n] = hn;
    if (n > 0) hs[N - n] = hn;
  }
  std::vector<double> ct(N);
  for (int t = 0; t < N; ++t) ct[t] = std::cos(2.0 * M_PI * t / N);
  std::vector<float> H(N);
  for (int k = 0; k < N; ++k) {
    double acc = 0.0;
    for (int n = 0; n < N; ++n)
      if (hs[n] != 0.0) acc += hs[n] * ct[(size_t)k * n % N];
    H[k] = (float)(acc / N);
  }
  std::vector<float2> tw(N);
  for (int t = 0; t < N; ++t)
    tw[t] = make_float2((float)std::cos(2.0 * M_PI * t / N), (float)-std::sin(2.0 * M_PI * t / N));
  hr_filter_plan* p = new hr_filter_plan{YL, ZL, ViewN, log2N, PLC, ZLC, dYL, dZL, SO, nullptr, nullptr};
  cudaError_t e = cudaMalloc(&p->d_H, sizeof(float) * N);
  if (e == cudaSuccess) e = cudaMalloc(&p->d_tw, sizeof(float2) * N);
  if (e == cudaSuccess) e = cudaMemcpy(p->d_H, H.data(), sizeof(float) * N, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(p->d_tw, tw.data(), sizeof(float2) * N, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(p->d_H);
    cudaFree(p->d_tw);
    delete p;
    return hr::fail(e == cudaErrorMemoryAllocation ? HR_ERR_OUT_OF_MEMORY : HR_ERR_CUDA, "filter plan: %s",
                    cudaGetErrorString(e));
  }
  *plan = p;
  return HR_OK;
}

extern "C" int hr_filter_execute(const hr_filter_plan* p, float* d_out, const float* d_in, int in_layout, int view0,
                                 void* stream) {
  HR_REQUIRE(p != nullptr && d_out != nullptr && d_in != nullptr, "hr_filter_execute: NULL argument");
  HR_REQUIRE(view0 >= 0, "hr_filter_execute: view0 < 0");
  HR_REQUIRE(in_layout == HR_LAYOUT_ROWS || in_layout == HR_LAYOUT_REBIN, "hr_filter_execute: unknown layout %d",
             in_layout);
  // The kernel reads its input through the non-coherent read-only path
  // (__restrict__), so input and output must not overlap.
  const size_t in_views = (size_t)view0 + p->ViewN;
  const char* ib = reinterpret_cast<const char*>(d_in);
  const char* ie = ib + in_views * p->ZL * p->YL * sizeof(float);
  const char* ob = reinterpret_cast<const char*>(d_out);
  const char* oe = ob + (size_t)p->ViewN * p->ZL * p->YL * sizeof(float);
  HR_REQUIRE(oe <= ib || ie <= ob, "hr_filter_execute: input and output overlap (in-place filtering is not supported)");
  cudaStream_t s = hr::as_stream(stream);
  if (in_layout == HR_LAYOUT_ROWS) return launch_layout<HR_LAYOUT_ROWS>(p, d_out, d_in, view0, s);
  return launch_layout<HR_LAYOUT_REBIN>(p, d_out, d_in, view0, s);
}

extern "C" void hr_filter_plan_destroy(hr_filter_plan* p) {
  if (!p) return;
  cudaFree(p->d_H);
  cudaFree(p->d_tw);
  delete p;
}
