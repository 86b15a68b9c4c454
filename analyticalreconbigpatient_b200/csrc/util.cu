// Small element-wise device helpers of the host drivers.
#include "hr_internal.h"

namespace {

__global__ void accumulate_kernel(float* __restrict__ sum, const float* __restrict__ x, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    sum[i] += x[i];
}

}  // namespace

extern "C" int hr_accumulate(float* d_sum, const float* d_x, long long n, void* stream) {
  HR_REQUIRE(d_sum != nullptr && d_x != nullptr && n >= 0, "hr_accumulate: invalid argument");
  if (n == 0) return HR_OK;
  accumulate_kernel<<<8 * hr::sm_count(), 256, 0, hr::as_stream(stream)>>>(d_sum, d_x, n);
  HR_CUDA_TRY(cudaGetLastError());
  return HR_OK;
}
