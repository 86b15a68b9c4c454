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
//
// N = 2048 (YL in (512, 1024], the scanners' 888 channels) runs a register-
// resident kernel instead: one warp per pair of rows, 64 points per lane
// (N = 64 x 32). Forward: each lane j transforms x[j + 32 m] over m with a
// 64-point DFT (8 x 8, in registers), multiplies by W_2048^(j c), and the
// warp exchanges through shared memory so that lane t holds columns c = t,
// t+32 for all j; a 32-point DFT over j (4 x 8) gives frequencies c + 64 q,
// which are multiplied by H. The inverse runs the same steps backwards: a
// 32-point inverse DFT over q, the conjugate twiddle, an exchange back, and
// a 64-point inverse DFT per lane gives y[j + 32 n] in registers, stored
// straight to the output rows. Two shared-memory exchanges per pair of rows,
// no block-wide barrier after set-up.
#include <cmath>
#include <cstdlib>
#include <vector>

#include "hr_internal.h"

struct hr_filter_plan {
  int YL, ZL, ViewN, log2N;
  float PLC, ZLC, dYL, dZL, SO;
  float* d_H;    // real spectrum of the wrapped kernel, divided by N
  float2* d_tw;  // exp(-2 pi i t / N), t in [0, N)
  float* d_wt;   // N = 2048: preweight of every (row k, channel j), [ZL][YL]
  float2* d_tw2; // N = 2048: W_2048^(j c) as [c][j], c in [0, 64), j in [0, 32)
  float2* d_tw3; // N = 2048, two warps per row pair: W_2048^(j k1) as [k1][j], k1 in [0, 32), j in [0, 64)
  float2* d_G;   // N = 2048, two warps per row pair: {H[k1 + 32 k] + H[k1 + 32 k + 1024], difference} at [k][k1]
  float* d_wt8;  // N = 2048, ZL % 8 == 0: d_wt as [ZL / 8][YL][8] (the staged rebinning-layout path)
  int kernel2048;  // 0: two warps per row pair; 1: one warp per row pair (HELIXRECON_FILTER2048=1)
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

// ---------------------------------------------------------------------------
// N = 2048: register-resident transforms, one warp per row pair.
// ---------------------------------------------------------------------------
namespace fft2k {

constexpr int kN = 2048;
constexpr int kWarps = 4;      // row pairs in flight per CTA
constexpr int kStride = 66;    // exchange row stride in float2 (64 + 2: 16-byte lanes hit distinct banks)

// W_64^x (forward), x in [0, 64); W_32^x = W_64^(2x).
__constant__ float2 c_w64[64];

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// a * w (INV: a * conj(w))
template <bool INV>
__device__ __forceinline__ float2 cmulw(float2 a, float2 w) {
  return INV ? make_float2(a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y)
             : make_float2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
}
// a * (-i) forward, a * (+i) inverse
template <bool INV>
__device__ __forceinline__ float2 rot(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}
// a * W_8 (forward (1 - i)/sqrt 2, inverse (1 + i)/sqrt 2)
template <bool INV>
__device__ __forceinline__ float2 w8(float2 a) {
  const float r = 0.70710678118654752f;
  return INV ? make_float2((a.x - a.y) * r, (a.x + a.y) * r) : make_float2((a.x + a.y) * r, (a.y - a.x) * r);
}

// Complex add / subtract as one packed FP32x2 instruction (sm_100): each lane
// is an IEEE round-to-nearest add, the same bits as two scalar adds.
__device__ __forceinline__ unsigned long long f2u(float2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ float2 u2f(unsigned long long r) {
  float2 a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
__device__ __forceinline__ float2 padd(float2 a, float2 b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2u(a)), "l"(f2u(b)));
  return u2f(d);
}
__device__ __forceinline__ float2 psub(float2 a, float2 b) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2u(a)), "l"(f2u(b)));
  return u2f(d);
}

// 4-point DFT of v[O], v[O+S], v[O+2S], v[O+3S], in place, natural order.
template <bool INV, int O, int S, int L>
__device__ __forceinline__ void dft4(float2 (&v)[L]) {
  const float2 t0 = padd(v[O], v[O + 2 * S]), t1 = psub(v[O], v[O + 2 * S]);
  const float2 t2 = padd(v[O + S], v[O + 3 * S]), t3 = rot<INV>(psub(v[O + S], v[O + 3 * S]));
  v[O] = padd(t0, t2);
  v[O + 2 * S] = psub(t0, t2);
  v[O + S] = cadd(t1, t3);
  v[O + 3 * S] = csub(t1, t3);
}

// 8-point DFT of v[O + S i], i in [0, 8), in place, natural order (even/odd split).
template <bool INV, int O, int S, int L>
__device__ __forceinline__ void dft8(float2 (&v)[L]) {
  dft4<INV, O, 2 * S>(v);      // E[k] at v[O + 2S k]
  dft4<INV, O + S, 2 * S>(v);  // O[k] at v[O + S + 2S k]
  const float2 e0 = v[O], e1 = v[O + 2 * S], e2 = v[O + 4 * S], e3 = v[O + 6 * S];
  const float2 o0 = v[O + S], o1 = w8<INV>(v[O + 3 * S]), o2 = rot<INV>(v[O + 5 * S]);
  const float2 o3 = rot<INV>(w8<INV>(v[O + 7 * S]));
  v[O] = padd(e0, o0);
  v[O + 4 * S] = psub(e0, o0);
  v[O + S] = padd(e1, o1);
  v[O + 5 * S] = psub(e1, o1);
  v[O + 2 * S] = cadd(e2, o2);
  v[O + 6 * S] = csub(e2, o2);
  v[O + 3 * S] = padd(e3, o3);
  v[O + 7 * S] = psub(e3, o3);
}

template <bool INV, int M2>
__device__ __forceinline__ void dft64_cols(float2 (&v)[64]) {
  dft8<INV, M2, 8>(v);
  if constexpr (M2 + 1 < 8) dft64_cols<INV, M2 + 1>(v);
}
template <bool INV, int K1>
__device__ __forceinline__ void dft64_rows(float2 (&v)[64]) {
  dft8<INV, 8 * K1, 1>(v);
  if constexpr (K1 + 1 < 8) dft64_rows<INV, K1 + 1>(v);
}
// 64-point DFT of v (natural order in); position 8 k1 + k2 ends up holding
// frequency k1 + 8 k2.
template <bool INV>
__device__ __forceinline__ void dft64(float2 (&v)[64]) {
  dft64_cols<INV, 0>(v);  // over m1 for each m2: position m2 + 8 k1
#pragma unroll
  for (int m2 = 1; m2 < 8; ++m2)
#pragma unroll
    for (int k1 = 1; k1 < 8; ++k1) v[m2 + 8 * k1] = cmulw<INV>(v[m2 + 8 * k1], c_w64[m2 * k1]);
  dft64_rows<INV, 0>(v);  // over m2 for each k1: position 8 k1 + k2
}
__device__ __forceinline__ int dft64_freq(int p) { return (p >> 3) + 8 * (p & 7); }

template <int M2>
__device__ __forceinline__ void dft32f_cols(float2 (&v)[32]) {
  dft8<false, M2, 4>(v);
  if constexpr (M2 + 1 < 4) dft32f_cols<M2 + 1>(v);
}
template <int Q1>
__device__ __forceinline__ void dft32f_rows(float2 (&v)[32]) {
  dft4<false, 4 * Q1, 1>(v);
  if constexpr (Q1 + 1 < 8) dft32f_rows<Q1 + 1>(v);
}
// Forward 32-point DFT (natural order in); position 4 q1 + q2 ends up holding
// frequency q1 + 8 q2.
__device__ __forceinline__ void dft32_fwd(float2 (&v)[32]) {
  dft32f_cols<0>(v);  // over m1 for each m2 (j = m2 + 4 m1): position m2 + 4 q1
#pragma unroll
  for (int m2 = 1; m2 < 4; ++m2)
#pragma unroll
    for (int q1 = 1; q1 < 8; ++q1) v[m2 + 4 * q1] = cmulw<false>(v[m2 + 4 * q1], c_w64[2 * m2 * q1]);
  dft32f_rows<0>(v);  // over m2 for each q1
}
template <int Q1>
__device__ __forceinline__ void dft32i_rows(float2 (&v)[32]) {
  dft4<true, 4 * Q1, 1>(v);
  if constexpr (Q1 + 1 < 8) dft32i_rows<Q1 + 1>(v);
}
template <int R1>
__device__ __forceinline__ void dft32i_cols(float2 (&v)[32]) {
  dft8<true, R1, 4>(v);
  if constexpr (R1 + 1 < 4) dft32i_cols<R1 + 1>(v);
}
// Inverse 32-point DFT whose input is in dft32_fwd's output order; the
// output is in natural order.
__device__ __forceinline__ void dft32_inv(float2 (&v)[32]) {
  dft32i_rows<0>(v);  // over q2 for each q1: position 4 q1 + r1
#pragma unroll
  for (int r1 = 1; r1 < 4; ++r1)
#pragma unroll
    for (int q1 = 1; q1 < 8; ++q1) v[4 * q1 + r1] = cmulw<true>(v[4 * q1 + r1], c_w64[2 * r1 * q1]);
  dft32i_cols<0>(v);  // over q1 for each r1: position r1 + 4 r2 = n
}
__device__ __forceinline__ int dft32_freq(int p) { return (p >> 2) + 8 * (p & 3); }

// Preweight table [ZL][YL] with the reference's float expression
// (src/filtering.cu:187-207); wt8 (if not null): the same values as
// [ZL / 8][YL][8].
__global__ void preweight_table_kernel(float* __restrict__ wt, float* __restrict__ wt8, int YL, int ZL, float PLC,
                                       float ZLC, float dYL, float dZL, float SO) {
  const float SO2 = SO * SO;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < YL * ZL; e += gridDim.x * blockDim.x) {
    const int k = e / YL, j = e - k * YL;
    const float b = ((float)k - ZLC) * dZL;
    const float t = ((float)j - PLC) * dYL;
    const float w = SO2 / sqrtf(SO2 * (SO2 + b * b) - b * t * b * t);
    wt[e] = w;
    if (wt8) wt8[((size_t)(k >> 3) * YL + j) * 8 + (k & 7)] = w;
  }
}

// STAGE (rebinning layout, ZL a multiple of 8): a CTA's four warps take the
// four row pairs of 8 consecutive rows k0..k0+7 of one view; those rows are
// 32 contiguous bytes per channel, so the CTA first copies the [YL][8] block
// into shared memory with coalesced 16-byte loads (over the exchange buffers,
// which are free between pairs) and each warp reads its two rows from there;
// without staging a lane's load touches a sector of its own.
template <int IN_LAYOUT, bool STAGE>
__global__ void __launch_bounds__(32 * kWarps, 2) filter2048_kernel(float* __restrict__ out, const float* __restrict__ in,
                                                                const float* __restrict__ gH,
                                                                const float2* __restrict__ gtw2,
                                                                const float* __restrict__ wt, int YL, int ZL,
                                                                long long rows, int view0) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* tw2 = reinterpret_cast<float2*>(smem_raw);             // [64][32]: W^(j c) at [c][j]
  float2* tw2t = tw2 + 64 * 32;                                  // [32][64]: W^(n c) at [n][c]
  float* H = reinterpret_cast<float*>(tw2t + 64 * 32);           // [2048]
  float2* xbuf = reinterpret_cast<float2*>(H + kN) + (threadIdx.x >> 5) * (32 * kStride);  // this warp's exchange
  for (int t = threadIdx.x; t < 64 * 32; t += blockDim.x) {
    tw2[t] = gtw2[t];
    tw2t[t] = gtw2[(t & 63) * 32 + (t >> 6)];
  }
  for (int t = threadIdx.x; t < kN; t += blockDim.x) H[t] = gH[t];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long pairs = (rows + 1) >> 1;
  // STAGE: rows is a multiple of 8, so every tile of kWarps pairs is full and the loop is CTA-uniform
  const long long first = STAGE ? (long long)blockIdx.x * kWarps : (long long)blockIdx.x * kWarps + warp;
  const long long step = (long long)gridDim.x * kWarps;
  float* stage = reinterpret_cast<float*>(H + kN);  // [YL][9] (STAGE), over the exchange buffers
  for (long long pt = first; pt < pairs; pt += step) {
    const long long pr = STAGE ? pt + warp : pt;
    const long long ra = 2 * pr, rb = ra + 1;
    const bool hasb = rb < rows;
    const int ka = (int)(ra % ZL), kb = (int)(rb % ZL);
    const long long va = ra / ZL, vb = rb / ZL;
    // ---- load x[n] = wa[n] a[n] + i wb[n] b[n], n = lane + 32 m, and the first
    // stage of the 64-point DFT (over m1, m = m2 + 8 m1) group by group --------
    const float* pa = IN_LAYOUT == HR_LAYOUT_ROWS ? in + ((size_t)(view0 + va) * ZL + ka) * YL
                                                  : in + (size_t)(view0 + va) * YL * ZL + ka;
    const float* pb = IN_LAYOUT == HR_LAYOUT_ROWS ? in + ((size_t)(view0 + vb) * ZL + kb) * YL
                                                  : in + (size_t)(view0 + vb) * YL * ZL + kb;
    const size_t es = IN_LAYOUT == HR_LAYOUT_ROWS ? 1 : (size_t)ZL;  // element stride along a row
    const float* wa = wt + (size_t)ka * YL;
    const float* wb = wt + (size_t)kb * YL;
    float2 v[64];
    if constexpr (STAGE) {
      // rows 2*pt .. 2*pt+7 are k0 .. k0+7 of view va0 (ZL % 8 == 0)
      const long long r0 = 2 * pt;
      const long long va0 = r0 / ZL;
      const int k0 = (int)(r0 - va0 * ZL);
      const float4* src = reinterpret_cast<const float4*>(in + (size_t)(view0 + va0) * YL * ZL + k0);
      __syncthreads();  // every warp has finished reading its exchange buffer (the previous tile)
      for (int t = threadIdx.x; t < 2 * YL; t += 32 * kWarps) {
        const int n = t >> 1, hq = t & 1;
        const float4 q = __ldg(src + (size_t)n * (ZL / 4) + hq);
        float* d = stage + n * 9 + 4 * hq;
        d[0] = q.x;
        d[1] = q.y;
        d[2] = q.z;
        d[3] = q.w;
      }
      __syncthreads();
#pragma unroll
      for (int m2 = 0; m2 < 8; ++m2) {
#pragma unroll
        for (int m1 = 0; m1 < 8; ++m1) {
          const int n = lane + 32 * (m2 + 8 * m1);
          float a = 0.0f, b = 0.0f;
          if (n < YL) {
            a = stage[n * 9 + 2 * warp] * __ldg(wa + n);
            b = stage[n * 9 + 2 * warp + 1] * __ldg(wb + n);
          }
          v[m2 + 8 * m1] = make_float2(a, b);
        }
      }
      __syncthreads();  // the staging area is read before any warp writes its exchange buffer
    } else {
#pragma unroll
      for (int m2 = 0; m2 < 8; ++m2) {
#pragma unroll
        for (int m1 = 0; m1 < 8; ++m1) {
          const int n = lane + 32 * (m2 + 8 * m1);
          float a = 0.0f, b = 0.0f;
          if (n < YL) {
            a = __ldg(pa + n * es) * __ldg(wa + n);
            if (hasb) b = __ldg(pb + n * es) * __ldg(wb + n);
          }
          v[m2 + 8 * m1] = make_float2(a, b);
        }
        asm volatile("" ::: "memory");  // keep each group's loads next to its use
      }
    }
    // ---- forward: 64-point DFTs over m, twiddle W_2048^(lane c), exchange ------
    dft64<false>(v);
    __syncwarp();  // the previous pair's reads of xbuf are done
#pragma unroll
    for (int k1 = 0; k1 < 8; k1 += 2)
#pragma unroll
      for (int k2 = 0; k2 < 8; ++k2) {
        const int c = k1 + 8 * k2;  // even
        const float2 x0 = cmulw<false>(v[8 * k1 + k2], tw2[c * 32 + lane]);
        const float2 x1 = cmulw<false>(v[8 * (k1 + 1) + k2], tw2[(c + 1) * 32 + lane]);
        *reinterpret_cast<float4*>(xbuf + lane * kStride + c) = make_float4(x0.x, x0.y, x1.x, x1.y);
      }
    __syncwarp();
    // lane t owns columns c = t and t + 32 (all j): it reads each, transforms
    // it and writes it back in place (no other lane touches the column)
#pragma unroll 1
    for (int half = 0; half < 2; ++half) {
      const int c = lane + 32 * half;
      float2 y[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) y[j] = xbuf[j * kStride + c];
      // ---- 32-point DFT over j, H, inverse 32-point DFT over q -------------
      dft32_fwd(y);
#pragma unroll
      for (int p = 0; p < 32; ++p) {
        const float h = H[c + 64 * dft32_freq(p)];
        y[p] = make_float2(y[p].x * h, y[p].y * h);
      }
      dft32_inv(y);
      // ---- twiddle conj(W_2048^(n c)), back into the column ------------------
#pragma unroll
      for (int n = 0; n < 32; ++n) xbuf[n * kStride + c] = cmulw<true>(y[n], tw2t[n * 64 + c]);
    }
    __syncwarp();
#pragma unroll
    for (int c = 0; c < 64; c += 2) {
      const float4 q = *reinterpret_cast<const float4*>(xbuf + lane * kStride + c);
      v[c] = make_float2(q.x, q.y);
      v[c + 1] = make_float2(q.z, q.w);
    }
    // ---- inverse 64-point DFTs over c: y[lane + 32 n] ------------------------
    dft64<true>(v);
    float* oa = out + (size_t)ra * YL;
    float* ob = out + (size_t)rb * YL;
#pragma unroll
    for (int p = 0; p < 64; ++p) {
      const int n = lane + 32 * dft64_freq(p);
      if (n < YL) {
        oa[n] = v[p].x;
        if (hasb) ob[n] = v[p].y;
      }
    }
  }
}

size_t smem_bytes() {
  return 2 * 64 * 32 * sizeof(float2) + kN * sizeof(float) + kWarps * 32 * kStride * sizeof(float2);
}

template <int IN_LAYOUT, bool STAGE>
int launch_k(const hr_filter_plan* p, float* out, const float* in, int view0, cudaStream_t s) {
  auto kern = filter2048_kernel<IN_LAYOUT, STAGE>;
  const size_t smem = smem_bytes();
  HR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long rows = (long long)p->ZL * p->ViewN;
  const long long tiles = ((rows + 1) / 2 + kWarps - 1) / kWarps;
  int per_sm = 0;
  HR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * kWarps, smem));
  if (per_sm < 1) per_sm = 1;
  const long long want = (long long)per_sm * hr::sm_count();
  const int grid = (int)(tiles < want ? tiles : want);
  kern<<<grid, 32 * kWarps, smem, s>>>(out, in, p->d_H, p->d_tw2, p->d_wt, p->YL, p->ZL, rows, view0);
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}

template <int IN_LAYOUT>
int launch(const hr_filter_plan* p, float* out, const float* in, int view0, cudaStream_t s) {
  // staging needs 8-row tiles inside one view and 16-byte aligned channel blocks
  if constexpr (IN_LAYOUT == HR_LAYOUT_REBIN)
    if (p->ZL % 8 == 0 && ((uintptr_t)in & 15) == 0) return launch_k<IN_LAYOUT, true>(p, out, in, view0, s);
  return launch_k<IN_LAYOUT, false>(p, out, in, view0, s);
}

// ---- two warps per row pair ------------------------------------------------
// N = 64 x 32 with 32 points per lane, so that a lane needs half the registers
// of the one-warp kernel (<= 128: 16 warps per SM instead of 8). The 64 lanes
// of a pair (j = lane + 32 h, h the warp of the pair) and x[n], n = j + 64 m:
//   A: lane j: 32-point DFT over m -> k1, times W_2048^(j k1), into row j of
//      the pair's exchange buffer [64][33].
//   B: column k1 (lane & 15 + 16 h) is shared by lanes l and l ^ 16 (e =
//      lane >> 4): lane e takes rows j = 2 j' + e and transforms over j' -> k
//      (E for e = 0, O for e = 1). The 64-point DFT over j is X[k1 + 32 k] =
//      E + W_64^k O and X[k1 + 32 (k + 32)] = E - W_64^k O; after the filter
//      (H0 = H[k1 + 32 k], H1 = H[k1 + 32 k + 1024]) the inverse over k2 needs
//      S = Y0 + Y1 = (H0 + H1) E + (H0 - H1) W_64^k O on the even rows and
//      D = W_64^-k (Y0 - Y1) = (H0 - H1) W_64^-k E + (H0 + H1) O on the odd
//      ones, so one exchange of E and O between the two lanes (a shuffle)
//      carries the forward radix-2 step, the filter and the inverse one. An
//      inverse 32-point DFT over k gives rows 2 j' + e, times
//      conj(W_2048^(j k1)), back into the buffer.
//   A': lane j: inverse 32-point DFT over k1 of row j -> y[j + 64 m].
// With YL <= 64 MNZ only m < MNZ carries samples (888 channels: 14 of 32), so
// the first forward stage and the last inverse one are pruned at compile time.
// Bank-conflict free: rows of 33 float2 for the row-wise stages, 16
// consecutive columns per half-warp for the column-wise one.
constexpr int kPairs = 4;             // row pairs per CTA, two warps each
constexpr int kThreads2 = 64 * kPairs;
constexpr int kS2 = 33;               // exchange row stride in float2

__device__ __forceinline__ void bar_pair(int pair) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + pair), "r"(64) : "memory");
}

template <int IN_LAYOUT, bool STAGE, int MNZ>
__global__ void __launch_bounds__(kThreads2, 2) filter2048x2_kernel(float* __restrict__ out,
                                                                   const float* __restrict__ in,
                                                                   const float2* __restrict__ gtw,
                                                                   const float2* __restrict__ gG,
                                                                   const float* __restrict__ wt, int YL, int ZL,
                                                                   long long rows, int view0) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* twA = reinterpret_cast<float2*>(smem_raw);  // [32][64]: W_2048^(j k1) at [k1][j]
  float2* twB = twA + 32 * 64;                        // [64][32]: the same at [j][k1]
  float2* G = twB + 64 * 32;                          // [32][32]: {H0 + H1, H0 - H1} at [k][k1]
  float2* xall = G + 32 * 32;                         // kPairs exchange buffers [64][kS2]
  for (int t = threadIdx.x; t < 32 * 64; t += kThreads2) {
    const float2 w = gtw[t];
    twA[t] = w;
    twB[(t & 63) * 32 + (t >> 6)] = w;
  }
  for (int t = threadIdx.x; t < 32 * 32; t += kThreads2) G[t] = gG[t];
  __syncthreads();
  const int pair = threadIdx.x >> 6, h = (threadIdx.x >> 5) & 1, lane = threadIdx.x & 31;
  const int j = lane + 32 * h;                      // stages A and A'
  const int kc = (lane & 15) + 16 * h, e = lane >> 4;  // stage B: column and row parity
  float2* xb = xall + pair * 64 * kS2;
  float* stage = reinterpret_cast<float*>(xall);    // [YL][10] (STAGE), over the exchange buffers
  const long long npairs = (rows + 1) >> 1;
  // STAGE: rows is a multiple of 8, so every tile of kPairs pairs is full and the loop is CTA-uniform
  const long long first = STAGE ? (long long)blockIdx.x * kPairs : (long long)blockIdx.x * kPairs + pair;
  const long long step = (long long)gridDim.x * kPairs;
  for (long long pt = first; pt < npairs; pt += step) {
    const long long pr = STAGE ? pt + pair : pt;
    const long long ra = 2 * pr, rb = ra + 1;
    const bool hasb = rb < rows;
    float2 v[32];
    if constexpr (STAGE) {
      // rows 2 pt .. 2 pt + 7 are k0 .. k0 + 7 of one view (ZL % 8 == 0): stage them preweighted
      const long long r0 = 2 * pt;
      const long long va0 = r0 / ZL;
      const int k0 = (int)(r0 - va0 * ZL);
      const float4* src = reinterpret_cast<const float4*>(in + (size_t)(view0 + va0) * YL * ZL + k0);
      __syncthreads();  // every pair has finished reading its exchange buffer (the previous tile)
      // wt here: the preweights as [ZL / 8][YL][8], the 8 rows of a channel in 32 contiguous bytes
      const float4* w8 = reinterpret_cast<const float4*>(wt + ((size_t)(k0 >> 3) * YL) * 8);
      for (int t = threadIdx.x; t < 2 * YL; t += kThreads2) {
        const int n = t >> 1, hq = t & 1;
        const float4 q = __ldg(src + (size_t)n * (ZL / 4) + hq);
        const float4 w = __ldg(w8 + 2 * n + hq);
        float2* d = reinterpret_cast<float2*>(stage + n * 10 + 4 * hq);
        d[0] = make_float2(q.x * w.x, q.y * w.y);
        d[1] = make_float2(q.z * w.z, q.w * w.w);
      }
      __syncthreads();
#pragma unroll
      for (int m = 0; m < 32; ++m) {
        const int n = j + 64 * m;
        v[m] = make_float2(0.f, 0.f);
        if (m < MNZ && n < YL) v[m] = *reinterpret_cast<const float2*>(stage + n * 10 + 2 * pair);
      }
      __syncthreads();  // the staging area is read before any pair writes its exchange buffer
    } else {
      bar_pair(pair);  // both warps of the pair have finished reading the buffer (the previous pair of rows)
      const int ka = (int)(ra % ZL), kb = (int)(rb % ZL);
      const long long va = ra / ZL, vb = rb / ZL;
      const float* pa = IN_LAYOUT == HR_LAYOUT_ROWS ? in + ((size_t)(view0 + va) * ZL + ka) * YL
                                                    : in + (size_t)(view0 + va) * YL * ZL + ka;
      const float* pb = IN_LAYOUT == HR_LAYOUT_ROWS ? in + ((size_t)(view0 + vb) * ZL + kb) * YL
                                                    : in + (size_t)(view0 + vb) * YL * ZL + kb;
      const size_t es = IN_LAYOUT == HR_LAYOUT_ROWS ? 1 : (size_t)ZL;  // element stride along a row
      const float* wa = wt + (size_t)ka * YL;
      const float* wb = wt + (size_t)kb * YL;
#pragma unroll
      for (int m = 0; m < 32; ++m) {
        const int n = j + 64 * m;
        float a = 0.0f, b = 0.0f;
        if (m < MNZ && n < YL) {
          a = __ldg(pa + n * es) * __ldg(wa + n);
          if (hasb) b = __ldg(pb + n * es) * __ldg(wb + n);
        }
        v[m] = make_float2(a, b);
      }
    }
    // ---- A: 32-point DFT over m, twiddle, row j of the buffer --------------
    dft32_fwd(v);
#pragma unroll
    for (int p = 0; p < 32; ++p) {
      const int k1 = dft32_freq(p);
      xb[j * kS2 + k1] = cmulw<false>(v[p], twA[k1 * 64 + j]);
    }
    bar_pair(pair);
    // ---- B: column kc, rows of parity e: DFT over j', exchange + filter, inverse
#pragma unroll
    for (int q = 0; q < 32; ++q) v[q] = xb[(2 * q + e) * kS2 + kc];
    dft32_fwd(v);
    const float sg = e ? -1.0f : 1.0f;  // lane e = 1 multiplies the other lane's E by W_64^-k
#pragma unroll
    for (int p = 0; p < 32; ++p) {
      const int k = dft32_freq(p);
      const float2 o = make_float2(__shfl_xor_sync(0xffffffffu, v[p].x, 16), __shfl_xor_sync(0xffffffffu, v[p].y, 16));
      const float2 g = G[k * 32 + kc];
      const float2 w = c_w64[k];
      const float wy = sg * w.y;
      const float2 ow = make_float2(o.x * w.x - o.y * wy, o.x * wy + o.y * w.x);  // o W_64^(+-k)
      v[p] = make_float2(g.x * v[p].x + g.y * ow.x, g.x * v[p].y + g.y * ow.y);
    }
    dft32_inv(v);
#pragma unroll
    for (int q = 0; q < 32; ++q) {
      const int jj = 2 * q + e;
      xb[jj * kS2 + kc] = cmulw<true>(v[q], twB[jj * 32 + kc]);
    }
    bar_pair(pair);
    // ---- A': inverse 32-point DFT over k1 of row j: y[j + 64 m] -------------
#pragma unroll
    for (int p = 0; p < 32; ++p) v[p] = xb[j * kS2 + dft32_freq(p)];
    dft32_inv(v);
    float* oa = out + (size_t)ra * YL;
    float* ob = out + (size_t)rb * YL;
#pragma unroll
    for (int m = 0; m < MNZ; ++m) {
      const int n = j + 64 * m;
      if (n < YL) {
        oa[n] = v[m].x;
        if (hasb) ob[n] = v[m].y;
      }
    }
  }
}

size_t smem_bytes2() { return (2 * 32 * 64 + 32 * 32 + kPairs * 64 * kS2) * sizeof(float2); }

template <int IN_LAYOUT, bool STAGE, int MNZ>
int launch_k2(const hr_filter_plan* p, float* out, const float* in, int view0, cudaStream_t s) {
  auto kern = filter2048x2_kernel<IN_LAYOUT, STAGE, MNZ>;
  const size_t smem = smem_bytes2();
  HR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long rows = (long long)p->ZL * p->ViewN;
  const long long tiles = ((rows + 1) / 2 + kPairs - 1) / kPairs;
  int per_sm = 0;
  HR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads2, smem));
  if (per_sm < 1) per_sm = 1;
  const long long want = (long long)per_sm * hr::sm_count();
  const int grid = (int)(tiles < want ? tiles : want);
  kern<<<grid, kThreads2, smem, s>>>(out, in, p->d_tw3, p->d_G, STAGE ? p->d_wt8 : p->d_wt, p->YL, p->ZL, rows,
                                     view0);
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}

template <int IN_LAYOUT, bool STAGE>
int launch_k2m(const hr_filter_plan* p, float* out, const float* in, int view0, cudaStream_t s) {
  if (p->YL <= 64 * 14) return launch_k2<IN_LAYOUT, STAGE, 14>(p, out, in, view0, s);
  return launch_k2<IN_LAYOUT, STAGE, 16>(p, out, in, view0, s);
}

template <int IN_LAYOUT>
int launch2(const hr_filter_plan* p, float* out, const float* in, int view0, cudaStream_t s) {
  if constexpr (IN_LAYOUT == HR_LAYOUT_REBIN)
    if (p->ZL % 8 == 0 && ((uintptr_t)in & 15) == 0) return launch_k2m<IN_LAYOUT, true>(p, out, in, view0, s);
  return launch_k2m<IN_LAYOUT, false>(p, out, in, view0, s);
}

}  // namespace fft2k

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
    case 11: return p->kernel2048 ? fft2k::launch<IN_LAYOUT>(p, out, in, view0, s)
                                  : fft2k::launch2<IN_LAYOUT>(p, out, in, view0, s);
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
  std::vector<double> Hd(N);
  for (int k = 0; k < N; ++k) {
    double acc = 0.0;
    for (int n = 0; n < N; ++n)
      if (hs[n] != 0.0) acc += hs[n] * ct[(size_t)k * n % N];
    Hd[k] = acc / N;
    H[k] = (float)Hd[k];
  }
  std::vector<float2> tw(N);
  for (int t = 0; t < N; ++t)
    tw[t] = make_float2((float)std::cos(2.0 * M_PI * t / N), (float)-std::sin(2.0 * M_PI * t / N));
  hr_filter_plan* p = new hr_filter_plan{};
  p->YL = YL; p->ZL = ZL; p->ViewN = ViewN; p->log2N = log2N;
  p->PLC = PLC; p->ZLC = ZLC; p->dYL = dYL; p->dZL = dZL; p->SO = SO;
  if (const char* ev = std::getenv("HELIXRECON_FILTER2048")) p->kernel2048 = std::atoi(ev) == 1 ? 1 : 0;
  cudaError_t e = cudaMalloc(&p->d_H, sizeof(float) * N);
  if (e == cudaSuccess) e = cudaMalloc(&p->d_tw, sizeof(float2) * N);
  if (e == cudaSuccess) e = cudaMemcpy(p->d_H, H.data(), sizeof(float) * N, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(p->d_tw, tw.data(), sizeof(float2) * N, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && N == fft2k::kN) {
    // the register kernel's tables: W_2048^(j c) by [c][j], W_64^x, the preweight of every sample
    std::vector<float2> tw2(64 * 32), w64(64);
    for (int c = 0; c < 64; ++c)
      for (int j = 0; j < 32; ++j) tw2[c * 32 + j] = tw[(size_t)c * j];
    for (int x = 0; x < 64; ++x)
      w64[x] = make_float2((float)std::cos(2.0 * M_PI * x / 64), (float)-std::sin(2.0 * M_PI * x / 64));
    // the two-warp kernel's tables: W_2048^(j k1) by [k1][j] (k1 < 32, j < 64); the filter folded with the
    // radix-2 step, {H[k1 + 32 k] + H[k1 + 32 k + 1024], H[k1 + 32 k] - H[k1 + 32 k + 1024]} by [k][k1]
    std::vector<float2> tw3(32 * 64), G(32 * 32);
    for (int k1 = 0; k1 < 32; ++k1)
      for (int j = 0; j < 64; ++j) tw3[k1 * 64 + j] = tw[(size_t)k1 * j];
    for (int k = 0; k < 32; ++k)
      for (int k1 = 0; k1 < 32; ++k1) {
        const double h0 = Hd[k1 + 32 * k], h1 = Hd[k1 + 32 * k + 1024];
        G[k * 32 + k1] = make_float2((float)(h0 + h1), (float)(h0 - h1));
      }
    e = cudaMalloc(&p->d_tw3, sizeof(float2) * tw3.size());
    if (e == cudaSuccess) e = cudaMalloc(&p->d_G, sizeof(float2) * G.size());
    if (e == cudaSuccess) e = cudaMemcpy(p->d_tw3, tw3.data(), sizeof(float2) * tw3.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_G, G.data(), sizeof(float2) * G.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_tw2, sizeof(float2) * tw2.size());
    if (e == cudaSuccess) e = cudaMalloc(&p->d_wt, sizeof(float) * (size_t)YL * ZL);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_tw2, tw2.data(), sizeof(float2) * tw2.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(fft2k::c_w64, w64.data(), sizeof(float2) * 64);
    if (e == cudaSuccess && ZL % 8 == 0) e = cudaMalloc(&p->d_wt8, sizeof(float) * (size_t)YL * ZL);
    if (e == cudaSuccess) {
      fft2k::preweight_table_kernel<<<64, 256>>>(p->d_wt, p->d_wt8, YL, ZL, PLC, ZLC, dYL, dZL, SO);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
  }
  if (e != cudaSuccess) {
    cudaFree(p->d_H);
    cudaFree(p->d_tw);
    cudaFree(p->d_tw2);
    cudaFree(p->d_tw3);
    cudaFree(p->d_G);
    cudaFree(p->d_wt);
    cudaFree(p->d_wt8);
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
  cudaFree(p->d_tw2);
  cudaFree(p->d_tw3);
  cudaFree(p->d_G);
  cudaFree(p->d_wt);
  cudaFree(p->d_wt8);
  delete p;
}
