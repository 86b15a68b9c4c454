// Whole-chain plan: rebin -> crop -> preweight/filter -> backprojection.
//
// Restates the per-segment sequence of src/analyticalReconBigPatient.m:77-146
// (rebin with the MEX arguments, drop the segment overlap, filter with
// PLC-1/ZLC-1, backproject) as one device-resident plan: the three stage
// plans, the rebinned and filtered intermediates, and device copies of the
// fan data and volume for host-pointer execution are allocated once at
// creation; execution only enqueues kernels and copies on one stream.
//
// Host-pointer execution of the fast form is streamed: the fan data cross the
// host link in chunks while the views that have arrived are rebinned and
// filtered (each view once, chunk by chunk, high-priority stream), the
// backprojection runs in z-block ranges as soon as every view of a range's
// windows is filtered (ranges growing from one block, so that the first starts
// after a few percent of the fan data), and each range's slices leave the
// device while later ranges compute. Rebinning and filtering give the bits of
// the whole-scan launches; the FP16 texture copy of a texture variant is filled
// range by range with a scale taken from the first chunk, with headroom
// (bp_fast_tex_fill_range), and refilled whole if a later chunk exceeds it.
#include <algorithm>
#include <cstdlib>
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
  // streamed host execution (fast form): chunk filter plans sharing filter_tc's split scratch (chunk views;
  // the last chunk's views when it is shorter), streams (sf: rebin + filter, high priority; sbp:
  // texture fill + backprojection; scopy: fan in; sout: volume out) and their events
  int chunk = 0;
  hr_filter_tc_plan* fchunk[2] = {nullptr, nullptr};
  cudaStream_t sf = nullptr, sbp = nullptr, scopy = nullptr, sout = nullptr;
  std::vector<cudaEvent_t> ev_in, ev_filt, ev_bp;
};

namespace {

void destroy(hr_recon_plan* p) {
  if (!p) return;
  for (hr_filter_tc_plan* f : p->fchunk) hr_filter_tc_plan_destroy(f);
  for (auto* v : {&p->ev_in, &p->ev_filt, &p->ev_bp})
    for (cudaEvent_t e : *v) cudaEventDestroy(e);
  for (cudaStream_t st : {p->sf, p->sbp, p->scopy, p->sout})
    if (st) cudaStreamDestroy(st);
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

// Parallel views per chunk of the streamed host execution (HELIXRECON_STREAM_CHUNK overrides: tests use short
// chunks on small scans; 0 turns streaming off).
int stream_chunk_views(int PN) {
  int c = 1024;
  if (const char* e = std::getenv("HELIXRECON_STREAM_CHUNK")) c = std::atoi(e);
  return c <= 0 ? 0 : std::min(c, PN);
}

int events(std::vector<cudaEvent_t>* v, size_t n) {
  while (v->size() < n) {
    cudaEvent_t e = nullptr;
    HR_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    v->push_back(e);
  }
  return HR_OK;
}

// Chunk plans and streams of the streamed host execution.
int stream_setup(hr_recon_plan* p) {
  const hr_recon_desc& d = p->d;
  p->chunk = stream_chunk_views(d.bp.PN);
  if (p->chunk == 0) return HR_OK;
  void* scratch[3];
  hr::filter_tc_scratch(p->filter_tc, scratch);
  const int last = d.bp.PN - (d.bp.PN - 1) / p->chunk * p->chunk;
  HR_TRY(hr::filter_tc_create_shared(&p->fchunk[0], d.YL, d.ZL, p->chunk, d.fPLC, d.fZLC, d.fdYL, d.fdZL, d.fSO,
                                     scratch));
  if (last != p->chunk)
    HR_TRY(hr::filter_tc_create_shared(&p->fchunk[1], d.YL, d.ZL, last, d.fPLC, d.fZLC, d.fdYL, d.fdZL, d.fSO,
                                       scratch));
  int prio_lo = 0, prio_hi = 0;
  HR_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
  HR_CUDA_TRY(cudaStreamCreateWithPriority(&p->sf, cudaStreamNonBlocking, prio_hi));
  HR_CUDA_TRY(cudaStreamCreateWithFlags(&p->sbp, cudaStreamNonBlocking));
  HR_CUDA_TRY(cudaStreamCreateWithFlags(&p->scopy, cudaStreamNonBlocking));
  HR_CUDA_TRY(cudaStreamCreateWithFlags(&p->sout, cudaStreamNonBlocking));
  const int nch = (d.bp.PN + p->chunk - 1) / p->chunk;
  HR_TRY(events(&p->ev_in, nch));
  HR_TRY(events(&p->ev_filt, nch));
  return HR_OK;
}

// One backprojection launch of the streamed execution: z blocks [b0, b1), after chunk `ready` is filtered.
struct BpRange {
  int b0, b1, ready;
};

// Ranges of z blocks in the order their windows complete (blocks in z order when the source moves towards
// larger z, reversed when it moves the other way), growing 1, 2, 4, ... blocks up to 48, the last one at most
// 8 blocks (its copy-out is the only one nothing overlaps). Empty when the windows do not complete in a
// monotone order (the caller then runs the chain whole).
std::vector<BpRange> bp_ranges(const std::vector<int>& zb, int nblocks, int chunk, int PN) {
  // chunk after which block b's window is filtered (-1: an empty window, slices outside the scan)
  std::vector<int> rc(nblocks);
  for (int b = 0; b < nblocks; ++b) {
    const int count = zb[2 * b + 1], hi = zb[2 * b] + count - 1;
    rc[b] = count > 0 ? std::min(hi, PN - 1) / chunk : -1;
  }
  bool up = true, down = true;
  for (int b = 0, last = -1; b < nblocks; ++b) {
    if (rc[b] < 0) continue;
    if (last >= 0) {
      up = up && rc[b] >= rc[last];
      down = down && rc[b] <= rc[last];
    }
    last = b;
  }
  std::vector<BpRange> r;
  if (!up && !down) return r;
  // an empty block is ready with the block before it in the processing order
  for (int i = 0, run = 0; i < nblocks; ++i) {
    int& x = rc[up ? i : nblocks - 1 - i];
    x = x < 0 ? run : x;
    run = x;
  }
  int done = 0, S = 1;
  while (done < nblocks) {
    const int rem = nblocks - done;
    const int n = rem <= 8 ? rem : rem <= S + 8 ? rem - 8 : S;
    const int b0 = up ? done : nblocks - done - n, b1 = b0 + n;
    r.push_back(BpRange{b0, b1, up ? rc[b1 - 1] : rc[b0]});
    done += n;
    S = std::min(2 * S, 48);
  }
  return r;
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
    if (st == HR_OK) st = stream_setup(p);
  }
  if (st != HR_OK) {
    destroy(p);
    return st;
  }
  if (hr::log_enabled()) {
    char desc[1024];
    if (hr_recon_describe(p, desc, sizeof(desc)) == HR_OK)
      hr::log("recon plan: %d views -> %dx%dx%d, %.2f GB on the device; %s", d->ViewN, d->bp.XN, d->bp.YN, d->bp.ZN,
              hr_recon_device_bytes(p) / 1e9, desc);
  }
  *plan = p;
  return HR_OK;
}

extern "C" int hr_recon_describe(const hr_recon_plan* p, char* buf, int len) {
  HR_REQUIRE(p != nullptr, "hr_recon_describe: NULL plan");
  char bp[640];
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

namespace {

// The streamed host execution of the fast form (see the top of this file). Returns HR_OK with *done = false,
// having enqueued nothing, when the plan's windows do not allow it.
int execute_host_streamed(hr_recon_plan* p, float* h_vol, const float* h_fan, bool* done) {
  *done = false;
  const hr_recon_desc& d = p->d;
  const hr::BpFastGeom* g = nullptr;
  const hr::BpFast* f = nullptr;
  HR_TRY(hr::bp_plan_fast_parts(p->bp, &g, &f));
  const hr::BpFastTables& t = hr::bp_fast_variant_tables(*f);
  const int PN = d.bp.PN, C = p->chunk, nch = (PN + C - 1) / C;
  const std::vector<BpRange> ranges = bp_ranges(t.h_zb, t.nblocks, C, PN);
  if (ranges.empty()) return HR_OK;
  HR_TRY(events(&p->ev_bp, ranges.size()));
  const bool tex = f->tex.kind != 0;
  const size_t per_view = (size_t)d.YL * d.ZL;
  const int ctas = 8 * hr::sm_count();  // rebin and split CTAs beside a running backprojection
  // Enqueues the copies and kernels; on a failure it returns with earlier work possibly in flight.
  auto enqueue = [&]() -> int {
    // everything before this call on the plan's own stream comes first
    HR_CUDA_TRY(cudaEventRecord(p->ev_in[0], p->stream));
    for (cudaStream_t st : {p->sf, p->sbp, p->scopy, p->sout}) HR_CUDA_TRY(cudaStreamWaitEvent(st, p->ev_in[0], 0));
    int copied = 0, filled = -1;
    size_t r = 0;
    for (int c = 0; c < nch; ++c) {
      const int p0 = c * C, p1 = std::min(PN, p0 + C);
      int f0 = 0, f1 = 0;
      hr::rebin_fan_views(p->rebin, d.view0 + p0, d.view0 + p1, &f0, &f1);
      if (c == nch - 1) f1 = d.ViewN - 1;
      if (f1 + 1 > copied) {
        HR_CUDA_TRY(cudaMemcpyAsync(p->d_fan + copied * per_view, h_fan + copied * per_view,
                                    (size_t)(f1 + 1 - copied) * per_view * sizeof(float), cudaMemcpyDefault,
                                    p->scopy));
        copied = f1 + 1;
      }
      HR_CUDA_TRY(cudaEventRecord(p->ev_in[c], p->scopy));
      HR_CUDA_TRY(cudaStreamWaitEvent(p->sf, p->ev_in[c], 0));
      HR_TRY(hr::rebin_execute_range(p->rebin, p->d_rebinned, p->d_fan, d.view0 + p0, d.view0 + p1, ctas, p->sf));
      HR_TRY(hr::filter_tc_execute_limited(p->fchunk[p1 - p0 == C ? 0 : 1], p->d_pairs + p0 * per_view,
                                           p->d_rebinned, HR_LAYOUT_REBIN, d.view0 + p0, ctas, p->sf));
      HR_CUDA_TRY(cudaEventRecord(p->ev_filt[c], p->sf));
      // backprojection ranges whose windows this chunk completes: fill the chunks they need, then launch
      for (; r < ranges.size() && ranges[r].ready <= c; ++r) {
        for (; filled < ranges[r].ready; ++filled) {
          const int q = filled + 1;
          HR_CUDA_TRY(cudaStreamWaitEvent(p->sbp, p->ev_filt[q], 0));
          if (tex)
            HR_TRY(hr::bp_fast_tex_fill_range(*f, *g, p->d_pairs, q * C, std::min(PN, (q + 1) * C), q == 0 ? 1 : 2,
                                              p->sbp));
        }
        HR_TRY(hr::bp_fast_execute_blocks(*f, *g, p->d_vol, p->d_pairs, ranges[r].b0, ranges[r].b1 - ranges[r].b0,
                                          p->sbp));
        HR_CUDA_TRY(cudaEventRecord(p->ev_bp[r], p->sbp));
      }
    }
    // volume out, range by range (enqueued last: a copy to pageable memory returns only when it is done); the
    // copies take their direction from the addresses, so h_vol (and h_fan) may also be device memory
    const size_t ld = (size_t)d.bp.ZN * sizeof(float);
    for (size_t j = 0; j < ranges.size(); ++j) {
      const int z0 = ranges[j].b0 * t.nz, z1 = std::min(d.bp.ZN, ranges[j].b1 * t.nz);
      if (z1 <= z0) continue;
      HR_CUDA_TRY(cudaStreamWaitEvent(p->sout, p->ev_bp[j], 0));
      HR_CUDA_TRY(cudaMemcpy2DAsync(h_vol + z0, ld, p->d_vol + z0, ld, (size_t)(z1 - z0) * sizeof(float),
                                    (size_t)d.bp.XN * d.bp.YN, cudaMemcpyDefault, p->sout));
    }
    return HR_OK;
  };
  int st = enqueue();
  // whether or not everything was enqueued, no copy may still read or write the caller's buffers on return
  for (cudaStream_t s2 : {p->scopy, p->sf, p->sbp, p->sout}) {
    const cudaError_t e = cudaStreamSynchronize(s2);
    if (e != cudaSuccess && st == HR_OK)
      st = hr::fail(HR_ERR_CUDA, "hr_recon_execute_host: %s", cudaGetErrorString(e));
  }
  HR_TRY(st);
  *done = true;
  for (hr_filter_tc_plan* fc : p->fchunk)
    if (fc) HR_TRY(hr_filter_tc_check(fc));
  bool refill = false;
  if (tex) HR_TRY(hr::bp_fast_tex_refill_needed(*f, &refill));
  if (refill) {
    // a later chunk outgrew the first chunk's FP16 scale: the whole copy again, with the scan's own scale
    hr::log("recon: streamed texture scale exceeded, refilling the whole copy");
    HR_TRY(hr::bp_fast_execute(*f, *g, p->d_vol, p->d_pairs, p->stream));
    const size_t nvol = (size_t)d.bp.XN * d.bp.YN * d.bp.ZN;
    HR_CUDA_TRY(cudaMemcpyAsync(h_vol, p->d_vol, nvol * sizeof(float), cudaMemcpyDefault, p->stream));
    HR_CUDA_TRY(cudaStreamSynchronize(p->stream));
  }
  return HR_OK;
}

}  // namespace

extern "C" int hr_recon_stream_schedule(const hr_recon_desc* d, int nz, int chunk, int* out, int cap, int* n) {
  hr::clear_error();
  HR_REQUIRE(d != nullptr && d->w != nullptr && n != nullptr, "hr_recon_stream_schedule: NULL argument");
  HR_REQUIRE(chunk > 0, "hr_recon_stream_schedule: chunk of %d views", chunk);
  int set = -1;
  for (int i = 0; i < hr::kFastTableSets; ++i)
    if (hr::kFastNz[i] == nz) set = i;
  HR_REQUIRE(set >= 0, "hr_recon_stream_schedule: %d slices per z block (16, 8 or 4)", nz);
  hr::BpFastGeom g;
  HR_TRY(hr::fast_geom_of(d->bp, &g));
  hr::BpFastHost h;  // the tables a fast backprojection plan builds, on the host
  HR_TRY(hr::bp_fast_host_tables(&h, g, d->w));
  const hr::BpFastHostSet& t = h.set[set];
  const std::vector<int> zb(t.zb.begin(), t.zb.begin() + 2 * (size_t)t.nblocks);
  const std::vector<BpRange> r = bp_ranges(zb, t.nblocks, std::min(chunk, d->bp.PN), d->bp.PN);
  *n = (int)r.size();
  if (out == nullptr) return HR_OK;
  HR_REQUIRE(cap >= (int)r.size(), "hr_recon_stream_schedule: %d ranges, room for %d", (int)r.size(), cap);
  for (size_t j = 0; j < r.size(); ++j) {
    out[3 * j] = r[j].b0;
    out[3 * j + 1] = r[j].b1;
    out[3 * j + 2] = r[j].ready;
  }
  return HR_OK;
}

extern "C" int hr_recon_execute_host(hr_recon_plan* p, float* h_vol, const float* h_fan) {
  hr::clear_error();
  HR_REQUIRE(p != nullptr && h_vol != nullptr && h_fan != nullptr, "hr_recon_execute_host: NULL argument");
  if (p->d.form == HR_FORM_FAST && p->chunk > 0) {
    bool done = false;
    HR_TRY(execute_host_streamed(p, h_vol, h_fan, &done));
    if (done) return HR_OK;
  }
  const size_t nfan = (size_t)p->d.YL * p->d.ZL * p->d.ViewN;
  const size_t nvol = (size_t)p->d.bp.XN * p->d.bp.YN * p->d.bp.ZN;
  auto enqueue = [&]() -> int {
    HR_CUDA_TRY(cudaMemcpyAsync(p->d_fan, h_fan, nfan * sizeof(float), cudaMemcpyDefault, p->stream));
    HR_TRY(hr_recon_execute(p, p->d_vol, p->d_fan, p->stream));
    HR_CUDA_TRY(cudaMemcpyAsync(h_vol, p->d_vol, nvol * sizeof(float), cudaMemcpyDefault, p->stream));
    return HR_OK;
  };
  const int st = enqueue();
  // no copy may still read or write the caller's buffers on return, also after a failure
  const cudaError_t e = cudaStreamSynchronize(p->stream);
  HR_TRY(st);
  HR_CUDA_TRY(e);
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
