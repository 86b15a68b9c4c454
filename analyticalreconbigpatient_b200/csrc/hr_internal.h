// Internal helpers shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>

#include "helixrecon.h"

namespace hr {

// Records a printf-style message as the calling thread's last error and
// returns `code`, so that call sites can `return fail(...)`.
int fail(int code, const char* fmt, ...);
void clear_error();
// Diagnostic line on stderr when the environment variable HELIXRECON_LOG is set (and not "0").
bool log_enabled();
void log(const char* fmt, ...);

// Checks a CUDA runtime call; on failure records file:line and the CUDA
// message and returns HR_ERR_CUDA (HR_ERR_OUT_OF_MEMORY for allocation).
#define HR_CUDA_TRY(expr)                                                                             \
  do {                                                                                                \
    cudaError_t hr_e_ = (expr);                                                                       \
    if (hr_e_ != cudaSuccess) {                                                                       \
      return ::hr::fail(hr_e_ == cudaErrorMemoryAllocation ? HR_ERR_OUT_OF_MEMORY : HR_ERR_CUDA,      \
                        "%s:%d: %s failed: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(hr_e_)); \
    }                                                                                                 \
  } while (0)

#define HR_TRY(expr)            \
  do {                          \
    int hr_s_ = (expr);         \
    if (hr_s_ != HR_OK) return hr_s_; \
  } while (0)

#define HR_REQUIRE(cond, ...)                                              \
  do {                                                                     \
    if (!(cond)) return ::hr::fail(HR_ERR_INVALID_ARGUMENT, __VA_ARGS__); \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Checks that a CUDA device is usable; records HR_ERR_NO_DEVICE otherwise.
int require_device();

// RAII device buffer used by the host-pointer entries.
struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  int alloc(size_t n) {
    bytes = n;
    if (n == 0) return HR_OK;
    HR_CUDA_TRY(cudaMalloc(&ptr, n));
    return HR_OK;
  }
  ~DeviceBuffer() {
    if (ptr) cudaFree(ptr);
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(ptr);
  }
};

// Number of SMs of the current device (cached per device).
int sm_count();

// Tensor-core filter plans whose split-operand scratch (three buffers of
// filter_tc_scratch_bytes each) belongs to the caller and may be shared by
// plans that execute one after the other on one stream.
size_t filter_tc_scratch_bytes(int YL, int ZL, int ViewN);
int filter_tc_create_shared(hr_filter_tc_plan** plan, int YL, int ZL, int ViewN, float PLC, float ZLC, float dYL,
                            float dZL, float SO, void* const scratch[3]);

// Launches with a bounded number of CTAs (max_ctas <= 0: one CTA per tile, as
// the public entries): memory-bound stages that run beside a texture-bound
// backprojection leave it most of the SMs' CTA slots.
int rebin_execute_limited(const hr_rebin_plan* p, float* d_out, const float* d_proj, int max_ctas, cudaStream_t s);
// Output views [i0, i1) only (written at their place in d_out; the same bits as a whole-scan launch).
int rebin_execute_range(const hr_rebin_plan* p, float* d_out, const float* d_proj, int i0, int i1, int max_ctas,
                        cudaStream_t s);
// Fan views [*f0, *f1] (clamped to the scan) that output views [i0, i1) read; i0 < i1.
void rebin_fan_views(const hr_rebin_plan* p, int i0, int i1, int* f0, int* f1);
// The three split-operand buffers of a tensor-core filter plan (its own or a caller's scratch), for plans that
// share them with filter_tc_create_shared.
void filter_tc_scratch(const hr_filter_tc_plan* p, void* scratch[3]);
int filter_tc_execute_limited(const hr_filter_tc_plan* p, uint32_t* d_pairs, const float* d_in, int in_layout,
                              int view0, int max_prep_ctas, cudaStream_t s);

}  // namespace hr
