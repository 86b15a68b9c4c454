// Whole-chain plan: rebin -> crop -> preweight/filter -> backprojection.
//
// Restates the per-segment sequence of src/analyticalReconBigPatient.m:77-146
// (rebin with the MEX arguments, drop the segment overlap, filter with
// PLC-1/ZLC-1, backproject) as one device-resident plan: the three stage
// plans, the rebinned and filtered intermediates, and device copies of the
// fan data and volume for host-pointer execution are allocated once at
// creation; execution only enqueues kernels and copies on one stream.
#include <cstring>
#include <vector>

#include "hr_internal.h"
#include "bp_fast.h"

struct hr_recon_plan {
  hr_recon_desc d;
  hr_rebin_plan* rebin = nullptr;
  hr_filter_plan* filter = nullptr;        // plain form: FFT filter
  hr_filter_tc_plan* filter_tc = nullptr;  // fast form: tensor-core Toeplitz filter
  hr_bp_plan* bp = nullptr;
  float* d_rebinned = nullptr;  // [ViewN][YL][ZL]
  float* d_filtered = nullptr;  // [PN][ZL][YL]
  uint32_t* d_pairs = nullptr;  // [PN][ZL][YL] BF16 channel pairs (fast form)
  float* d_fan = nullptr;       // staging for host execution
  float* d_vol = nullptr;
  cudaStream_t stream = nullptr;
  size_t bytes = 0;
};

namespace {

void destroy(hr_recon_plan* p) {
  if (!p) return;
  hr_rebin_plan_destroy(p->rebin);
  hr_filter_plan_destroy(p->filter);
  hr_filter_tc_plan_destroy(p->filter_tc);
  hr_bp_plan_destroy(p->bp);
  cudaFree(p->d_rebinned);
  cudaFree(p->d_filtered);
  cudaFree(p->d_pairs);
  cudaFree(p->d_fan);
  cudaFree(p->d_vol);
  if (p->stream) cudaStreamDestroy(p->stream);
  delete p;
}

int alloc(hr_recon_plan* p, void** ptr, size_t bytes) {
  HR_CUDA_TRY(cudaMalloc(ptr, bytes));
  p->bytes += bytes;
  return HR_OK;
}

}  // namespace

extern "C" int hr_recon_plan_create(hr_recon_plan** plan, const hr_recon_desc* d) {
  hr::clear_error();
  HR_REQUIRE(plan != nullptr && d != nullptr && d->w != nullptr, "hr_recon_plan_create: NULL argument");
  *plan = nullptr;
  HR_REQUIRE(d->form == HR_FORM_PLAIN || d->form == HR_FORM_FAST,
             "hr_recon_plan_create: form %d not available for the whole chain (the FP64 data path is reached "
             "through the stage plans)", d->form);
  HR_REQUIRE(d->bp.YL == d->YL && d->bp.ZL == d->ZL, "hr_recon_plan_create: bp.YL/ZL differ from YL/ZL");
  HR_REQUIRE(d->view0 >= 0 && d->view0 + d->bp.PN <= d->ViewN,
             "hr_recon_plan_create: views [%d, %d) exceed the %d rebinned views", d->view0, d->view0 + d->bp.PN,
             d->ViewN);
  hr_recon_plan* p = new hr_recon_plan;
  p->d = *d;
  p->d.w = nullptr;
  int st = hr_rebin_plan_create(&p->rebin, d->YL, d->ZL, d->ViewN, d->YLC, d->dYA, d->DeltaTheta, d->PLC, d->DeltaT,
                                d->DeltaFai, d->SO);
  const bool fast = d->form == HR_FORM_FAST;
  if (st == HR_OK && fast)
    st = hr_filter_tc_plan_create(&p->filter_tc, d->YL, d->ZL, d->bp.PN, d->fPLC, d->fZLC, d->fdYL, d->fdZL, d->fSO);
  if (st == HR_OK && !fast)
    st = hr_filter_plan_create(&p->filter, d->YL, d->ZL, d->bp.PN, d->fPLC, d->fZLC, d->fdYL, d->fdZL, d->fSO);
  if (st == HR_OK) st = hr_bp_plan_create(&p->bp, &d->bp, d->w, d->form);
  const size_t nfan = (size_t)d->YL * d->ZL * d->ViewN;
  const size_t nfilt = (size_t)d->YL * d->ZL * d->bp.PN;
  const size_t nvol = (size_t)d->bp.XN * d->bp.YN * d->bp.ZN;
  if (st == HR_OK) st = alloc(p, (void**)&p->d_rebinned, nfan * sizeof(float));
  if (st == HR_OK && !fast) st = alloc(p, (void**)&p->d_filtered, nfilt * sizeof(float));
  if (st == HR_OK && fast) st = alloc(p, (void**)&p->d_pairs, nfilt * sizeof(uint32_t));
  if (st == HR_OK) st = alloc(p, (void**)&p->d_fan, nfan * sizeof(float));
  if (st == HR_OK) st = alloc(p, (void**)&p->d_vol, nvol * sizeof(float));
  if (st == HR_OK) {
    cudaError_t e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) st = hr::fail(HR_ERR_CUDA, "hr_recon_plan_create: %s", cudaGetErrorString(e));
  }
  if (st == HR_OK && fast) {
    // pick the backprojection variant on the plan's own (zeroed) buffers
    cudaError_t e = cudaMemsetAsync(p->d_pairs, 0, nfilt * sizeof(uint32_t), p->stream);
    if (e != cudaSuccess) st = hr::fail(HR_ERR_CUDA, "hr_recon_plan_create: %s", cudaGetErrorString(e));
    if (st == HR_OK) st = hr_bp_autotune(p->bp, p->d_vol, p->d_pairs, p->stream);
  }
  if (st != HR_OK) {
    destroy(p);
    return st;
  }
  if (hr::log_enabled()) {
    char desc[512];
    if (hr_recon_describe(p, desc, sizeof(desc)) == HR_OK)
      hr::log("recon plan: %d views -> %dx%dx%d, %.2f GB on the device; %s", d->ViewN, d->bp.XN, d->bp.YN, d->bp.ZN,
              hr_recon_device_bytes(p) / 1e9, desc);
  }
  *plan = p;
  return HR_OK;
}

extern "C" int hr_recon_describe(const hr_recon_plan* p, char* buf, int len) {
  HR_REQUIRE(p != nullptr, "hr_recon_describe: NULL plan");
  char bp[400];
  HR_TRY(hr_bp_describe(p->bp, bp, sizeof(bp)));
  if (buf && len > 0)
    snprintf(buf, (size_t)len, "filter=%s; backprojection: %s",
             p->filter_tc ? "tcgen05 split-BF16 Toeplitz" : "FP32 radix-4 FFT", bp);
  return HR_OK;
}

extern "C" int hr_recon_execute(const hr_recon_plan* p, float* d_vol, const float* d_fan, void* stream) {
  HR_REQUIRE(p != nullptr && d_vol != nullptr && d_fan != nullptr, "hr_recon_execute: NULL argument");
  HR_TRY(hr_rebin_execute(p->rebin, p->d_rebinned, d_fan, stream));
  if (p->d.form == HR_FORM_FAST) {
    HR_TRY(hr_filter_tc_execute(p->filter_tc, p->d_pairs, p->d_rebinned, HR_LAYOUT_REBIN, p->d.view0, stream));
    return hr_bp_execute(p->bp, d_vol, p->d_pairs, stream);
  }
  HR_TRY(hr_filter_execute(p->filter, p->d_filtered, p->d_rebinned, HR_LAYOUT_REBIN, p->d.view0, stream));
  return hr_bp_execute(p->bp, d_vol, p->d_filtered, stream);
}

extern "C" int hr_recon_execute_host(hr_recon_plan* p, float* h_vol, const float* h_fan) {
  hr::clear_error();
  HR_REQUIRE(p != nullptr && h_vol != nullptr && h_fan != nullptr, "hr_recon_execute_host: NULL argument");
  const size_t nfan = (size_t)p->d.YL * p->d.ZL * p->d.ViewN;
  const size_t nvol = (size_t)p->d.bp.XN * p->d.bp.YN * p->d.bp.ZN;
  HR_CUDA_TRY(cudaMemcpyAsync(p->d_fan, h_fan, nfan * sizeof(float), cudaMemcpyHostToDevice, p->stream));
  HR_TRY(hr_recon_execute(p, p->d_vol, p->d_fan, p->stream));
  HR_CUDA_TRY(cudaMemcpyAsync(h_vol, p->d_vol, nvol * sizeof(float), cudaMemcpyDeviceToHost, p->stream));
  HR_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return HR_OK;
}

extern "C" int hr_recon_check(const hr_recon_plan* p) {
  HR_REQUIRE(p != nullptr, "hr_recon_check: NULL plan");
  if (p->filter_tc) return hr_filter_tc_check(p->filter_tc);
  return HR_OK;
}

extern "C" size_t hr_recon_device_bytes(const hr_recon_plan* p) {
  if (!p) return 0;
  size_t b = p->bytes + (p->filter_tc ? hr_filter_tc_device_bytes(p->filter_tc) : 0);
  const hr::BpFastGeom* g;
  const hr::BpFast* f;
  if (p->d.form == HR_FORM_FAST && hr::bp_plan_fast_parts(p->bp, &g, &f) == HR_OK) b += hr::bp_fast_device_bytes(*f);
  return b;
}

extern "C" void hr_recon_plan_destroy(hr_recon_plan* p) { destroy(p); }
