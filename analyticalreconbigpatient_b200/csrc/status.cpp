// Error reporting and device helpers.
#include <cstring>
#include <string>

#include "hr_internal.h"

namespace hr {

static thread_local char g_last_error[1024] = {0};

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

void clear_error() { g_last_error[0] = 0; }

int require_device() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(HR_ERR_NO_DEVICE, "no CUDA device available (%s)",
                e == cudaSuccess ? "0 devices" : cudaGetErrorString(e));
  }
  return HR_OK;
}

int sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (cached[dev] == 0) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    cached[dev] = n > 0 ? n : 148;
  }
  return cached[dev];
}

}  // namespace hr

extern "C" const char* hr_last_error(void) { return hr::g_last_error; }

extern "C" int hr_version(void) { return 100; }
