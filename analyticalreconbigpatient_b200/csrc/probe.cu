// Device throughput probe for the texture-sampling backprojection's roofline:
// the rate at which the texture units return bilinear samples of an FP16
// layered texture (the format the backprojection samples), measured with CUDA
// events on a cache-resident texture with every lane active. Built into a
// measurement library of its own (libhelixprobe.so), outside the product's C
// ABI:
//   int hr_texture_sample_rate(double* samples_per_s, void* stream);
// synchronises the stream and writes the device-wide bilinear samples per second.
#include <cuda_fp16.h>

#include <algorithm>
#include <vector>

#include "hr_internal.h"

namespace {

constexpr int kW = 64, kH = 64, kLayers = 4, kPerThread = 8;

// Neighbouring lanes sample 0.75 texels apart (adjacent volume columns project
// to nearby detector channels in the backprojection); kPerThread independent
// samples per iteration keep the texture pipe's queue full.
__global__ void tex_rate_kernel(float* __restrict__ out, cudaTextureObject_t t, int iters) {
  const float x = 1.0f + (float)(threadIdx.x & 63) * 0.75f;
  const float y = 1.0f + (float)(threadIdx.x >> 6) * 0.5f;
  float acc[kPerThread];
#pragma unroll
  for (int k = 0; k < kPerThread; ++k) acc[k] = 0.0f;
  for (int it = 0; it < iters; ++it) {
    const float dy = (float)it * 1e-3f;
#pragma unroll
    for (int k = 0; k < kPerThread; ++k)
      acc[k] += tex2DLayered<float>(t, x + 0.37f * (float)k, y + 0.21f * (float)k + dy, k & (kLayers - 1));
  }
  float s = 0.0f;
#pragma unroll
  for (int k = 0; k < kPerThread; ++k) s += acc[k];
  out[blockIdx.x * (size_t)blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" int hr_texture_sample_rate(double* samples_per_s, void* stream) {
  HR_REQUIRE(samples_per_s != nullptr, "hr_texture_sample_rate: NULL argument");
  cudaStream_t s = hr::as_stream(stream);
  const int threads = 256, ctas = 8 * hr::sm_count(), iters = 256;
  cudaArray_t arr = nullptr;
  cudaTextureObject_t tex = 0;
  float* d_out = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  double best = 0.0;
  cudaError_t e = cudaSuccess;
  do {
    const cudaChannelFormatDesc desc = cudaCreateChannelDescHalf();
    if ((e = cudaMalloc3DArray(&arr, &desc, make_cudaExtent(kW, kH, kLayers), cudaArrayLayered)) != cudaSuccess) break;
    std::vector<unsigned short> h((size_t)kW * kH * kLayers);
    for (size_t i = 0; i < h.size(); ++i) h[i] = __half_as_ushort(__float2half((float)((i * 37) % 101) * 0.01f));
    cudaMemcpy3DParms cp{};
    cp.srcPtr = make_cudaPitchedPtr(h.data(), kW * sizeof(unsigned short), kW, kH);
    cp.dstArray = arr;
    cp.extent = make_cudaExtent(kW, kH, kLayers);
    cp.kind = cudaMemcpyHostToDevice;
    if ((e = cudaMemcpy3D(&cp)) != cudaSuccess) break;
    cudaResourceDesc rd{};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td{};
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    if ((e = cudaCreateTextureObject(&tex, &rd, &td, nullptr)) != cudaSuccess) break;
    if ((e = cudaMalloc(&d_out, sizeof(float) * (size_t)threads * ctas)) != cudaSuccess) break;
    if ((e = cudaEventCreate(&e0)) != cudaSuccess || (e = cudaEventCreate(&e1)) != cudaSuccess) break;
    for (int rep = 0; rep < 6 && e == cudaSuccess; ++rep) {
      cudaEventRecord(e0, s);
      tex_rate_kernel<<<ctas, threads, 0, s>>>(d_out, tex, iters);
      cudaEventRecord(e1, s);
      if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0 && ms > 0.f) best = std::max(best, (double)threads * ctas * iters * kPerThread / (ms * 1e-3));
    }
    if (e == cudaSuccess) e = cudaGetLastError();
  } while (false);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(d_out);
  if (tex) cudaDestroyTextureObject(tex);
  if (arr) cudaFreeArray(arr);
  if (e != cudaSuccess)
    return hr::fail(e == cudaErrorMemoryAllocation ? HR_ERR_OUT_OF_MEMORY : HR_ERR_CUDA, "hr_texture_sample_rate: %s",
                    cudaGetErrorString(e));
  *samples_per_s = best;
  return HR_OK;
}
