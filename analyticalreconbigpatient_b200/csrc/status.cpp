// Error reporting and device helpers.
#include <cstdlib>
#include <cstring>
#include <string>

#include "hr_internal.h"

namespace hr {

static thread_local char g_last_error[1024] = {0};

int fail(int code, const char* fmt, ...) {
  // a failed runtime call (an allocation, a launch configuration) leaves its error as the thread's
  // last CUDA error; clear it so that it is not reported again by the caller's next CUDA call
  if (code == HR_ERR_CUDA || code == HR_ERR_OUT_OF_MEMORY) cudaGetLastError();
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

void clear_error() { g_last_error[0] = 0; }

// HELIXRECON_LOG=1 prints the plans' configuration choices to stderr.
bool log_enabled() {
  static const int on = [] {
    const char* e = std::getenv("HELIXRECON_LOG");
    return (e && *e && std::strcmp(e, "0") != 0) ? 1 : 0;
  }();
  return on != 0;
}

void log(const char* fmt, ...) {
  if (!log_enabled()) return;
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  std::fprintf(stderr, "[helixrecon] %s\n", buf);
}

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
