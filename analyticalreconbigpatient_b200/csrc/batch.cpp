// Several helical scans of uneven length in one persistent backprojection launch.
//
// Each scan is the per-segment sequence of src/analyticalReconBigPatient.m:77-146
// (rebin, drop the overlap, filter, backproject). Rebinning and the tensor-core
// filter run scan after scan through one shared rebinned buffer and one shared
// split-operand scratch; every scan keeps its own BF16 filtered data, and one
// persistent launch then backprojects the (scan, z block, column tile) items of
// all scans, so small scans fill the GPU together instead of each leaving a tail.
// The sequence is captured into a CUDA graph for the buffer addresses it is
// given and replayed while they stay the same.

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "hr_internal.h"
#include "bp_fast.h"

struct hr_batch_plan {
  int n = 0;
  std::vector<hr_recon_desc> d;
  std::vector<hr_rebin_plan*> rebin;
  std::vector<hr_filter_tc_plan*> ftc;
  std::vector<hr_bp_plan*> bp;
  std::vector<uint32_t*> pairs;  // per scan: [PN][ZL][YL] BF16 channel pairs
  std::vector<int> nz;           // per scan: slices per thread of its backprojection (register gathers)
  std::vector<int> tv;           // per scan: its FP16 texture variant (batch variants with texture taps)
  std::vector<int> sv;           // per scan: the variant its own autotuner chose (per-scan launches)
  std::vector<cudaStream_t> ss;  // per scan: its stream for the per-scan launches
  std::vector<cudaEvent_t> ready, done;  // per scan: fork and join points of the per-scan launches
  float* d_rebinned = nullptr;   // shared: the largest scan's [ViewN][YL][ZL]
  int* d_counter = nullptr;      // work-item counter of the persistent launch
  void* d_split[3] = {};         // shared tensor-core filter operands
  int variant = 0, tuned = 0;
  int ctas[hr::kBatchVariants_n] = {};
  float tuned_ms[hr::kBatchVariants_n] = {};
  cudaStream_t sc = nullptr;  // capture stream
  // host-buffer execution (hr_batch_execute_host), allocated at its first call
  float* d_stage[2] = {};        // fan staging ring, each the largest scan's fan
  float* d_hvol = nullptr;       // every scan's volume, at voff[i]
  std::vector<size_t> voff;
  cudaStream_t sin = nullptr, sout = nullptr;
  cudaEvent_t copied[2] = {}, consumed[2] = {}, bp_done = nullptr;
  bool host_ready = false;
  cudaGraphExec_t graph = nullptr;
  std::vector<const void*> graph_ptrs;
  int graph_variant = -1;
  size_t bytes = 0;
};

namespace {

void destroy(hr_batch_plan* p) {
  if (!p) return;
  if (p->graph) cudaGraphExecDestroy(p->graph);
  for (auto* r : p->rebin) hr_rebin_plan_destroy(r);
  for (auto* f : p->ftc) hr_filter_tc_plan_destroy(f);
  for (auto* b : p->bp) hr_bp_plan_destroy(b);
  for (auto* q : p->pairs) cudaFree(q);
  cudaFree(p->d_rebinned);
  cudaFree(p->d_counter);
  for (void* q : p->d_split) cudaFree(q);
  for (cudaStream_t q : p->ss) cudaStreamDestroy(q);
  for (cudaEvent_t e : p->ready) cudaEventDestroy(e);
  for (cudaEvent_t e : p->done) cudaEventDestroy(e);
  for (int b = 0; b < 2; ++b) {
    cudaFree(p->d_stage[b]);
    if (p->copied[b]) cudaEventDestroy(p->copied[b]);
    if (p->consumed[b]) cudaEventDestroy(p->consumed[b]);
  }
  cudaFree(p->d_hvol);
  if (p->bp_done) cudaEventDestroy(p->bp_done);
  if (p->sin) cudaStreamDestroy(p->sin);
  if (p->sout) cudaStreamDestroy(p->sout);
  if (p->sc) cudaStreamDestroy(p->sc);
  delete p;
}

int alloc(hr_batch_plan* p, void** ptr, size_t bytes) {
  HR_CUDA_TRY(cudaMalloc(ptr, bytes));
  p->bytes += bytes;
  return HR_OK;
}

bool textured(int bv) { return hr::kBatchVariants[bv].tex != 0; }
bool per_scan(int bv) { return hr::kBatchVariants[bv].streams != 0; }

// The scans as batch variant bv sees them (slices per thread of its taps).
int scans_of(const hr_batch_plan* p, float* const* vols, int bv, std::vector<hr::BpFastBatchScan>* out) {
  out->resize(p->n);
  for (int i = 0; i < p->n; ++i) {
    hr::BpFastBatchScan& b = (*out)[i];
    HR_TRY(hr::bp_plan_fast_parts(p->bp[i], &b.g, &b.f));
    b.vol = vols[i];
    b.fpb = p->pairs[i];
    const int forced = hr::kBatchVariants[bv].chunk;
    b.nz = !textured(bv) ? p->nz[i] : forced ? forced : hr::bp_fast_variant_nz(p->tv[i]);
  }
  return HR_OK;
}

// Gives every scan's plan the variant batch variant bv runs: its own
// autotuner's choice (per-scan launches), its FP16 texture variant (which keeps
// a layered copy of the scan's filtered data), or a register-gather one.
int set_scan_variants(hr_batch_plan* p, int bv) {
  const int gather_v[3] = {0, 3, 8};  // per-slice variants with 16, 8, 4 slices per thread
  for (int i = 0; i < p->n; ++i) {
    int v = per_scan(bv) ? p->sv[i] : textured(bv) ? p->tv[i] : 3;
    for (int g : gather_v)
      if (!per_scan(bv) && !textured(bv) && hr::bp_fast_variant_nz(g) == p->nz[i]) v = g;
    HR_TRY(hr_bp_select(p->bp[i], v));
  }
  return HR_OK;
}

// Per-scan launches: scan i's backprojection waits for ready[i] on the batch's
// stream, runs on its own stream and is joined back through done[i].
int fork_bp(const hr_batch_plan* p, int i, float* vol, cudaStream_t s) {
  HR_CUDA_TRY(cudaEventRecord(p->ready[i], s));
  HR_CUDA_TRY(cudaStreamWaitEvent(p->ss[i], p->ready[i], 0));
  HR_TRY(hr_bp_execute(p->bp[i], vol, p->pairs[i], p->ss[i]));
  HR_CUDA_TRY(cudaEventRecord(p->done[i], p->ss[i]));
  return HR_OK;
}

int join_all(const hr_batch_plan* p, cudaStream_t s) {
  for (int i = 0; i < p->n; ++i) HR_CUDA_TRY(cudaStreamWaitEvent(s, p->done[i], 0));
  return HR_OK;
}

// The backprojection of batch variant bv from the scans' filtered data.
int backproject(const hr_batch_plan* p, float* const* vols, int bv, cudaStream_t s);

int fill_textures(const hr_batch_plan* p, cudaStream_t s) {
  for (int i = 0; i < p->n; ++i) {
    const hr::BpFastGeom* g;
    const hr::BpFast* f;
    HR_TRY(hr::bp_plan_fast_parts(p->bp[i], &g, &f));
    HR_TRY(hr::bp_fast_tex_fill(*f, *g, p->pairs[i], s));
  }
  return HR_OK;
}

int backproject(const hr_batch_plan* p, float* const* vols, int bv, cudaStream_t s) {
  if (per_scan(bv)) {
    for (int i = 0; i < p->n; ++i) HR_TRY(fork_bp(p, i, vols[i], s));
    return join_all(p, s);
  }
  if (textured(bv)) HR_TRY(fill_textures(p, s));
  std::vector<hr::BpFastBatchScan> sc;
  HR_TRY(scans_of(p, vols, bv, &sc));
  const long long items = hr::bp_fast_batch_items(sc.data(), p->n);
  return hr::bp_fast_batch_execute(sc.data(), p->n, bv, 0, (int)items, p->ctas[bv], p->d_counter, s);
}

// Per-scan launches start each scan's backprojection as soon as its filter
// is done, under the next scans' rebinning and filtering (they read only the
// scan's own filtered data).
int enqueue(const hr_batch_plan* p, float* const* vols, const float* const* fans, cudaStream_t s) {
  for (int i = 0; i < p->n; ++i) {
    HR_TRY(hr_rebin_execute(p->rebin[i], p->d_rebinned, fans[i], s));
    HR_TRY(hr_filter_tc_execute(p->ftc[i], p->pairs[i], p->d_rebinned, HR_LAYOUT_REBIN, p->d[i].view0, s));
    if (per_scan(p->variant)) HR_TRY(fork_bp(p, i, vols[i], s));
  }
  if (per_scan(p->variant)) return join_all(p, s);
  return backproject(p, vols, p->variant, s);
}

size_t fan_elems(const hr_recon_desc& d) { return (size_t)d.YL * d.ZL * d.ViewN; }
size_t vol_elems(const hr_recon_desc& d) { return (size_t)d.bp.XN * d.bp.YN * d.bp.ZN; }

// Staging for hr_batch_execute_host: two fan buffers (the copy of one scan's
// fan overlaps the rebinning of the previous one), the volumes, two streams.
int host_buffers(hr_batch_plan* p) {
  if (p->host_ready) return HR_OK;
  size_t nfan_max = 0, vtot = 0;
  p->voff.assign(p->n, 0);
  for (int i = 0; i < p->n; ++i) {
    nfan_max = std::max(nfan_max, fan_elems(p->d[i]));
    p->voff[i] = vtot;
    vtot += vol_elems(p->d[i]);
  }
  for (int b = 0; b < 2; ++b)
    if (!p->d_stage[b]) HR_TRY(alloc(p, (void**)&p->d_stage[b], nfan_max * sizeof(float)));
  if (!p->d_hvol) HR_TRY(alloc(p, (void**)&p->d_hvol, vtot * sizeof(float)));
  if (!p->sin) HR_CUDA_TRY(cudaStreamCreateWithFlags(&p->sin, cudaStreamNonBlocking));
  if (!p->sout) HR_CUDA_TRY(cudaStreamCreateWithFlags(&p->sout, cudaStreamNonBlocking));
  for (int b = 0; b < 2; ++b) {
    if (!p->copied[b]) HR_CUDA_TRY(cudaEventCreateWithFlags(&p->copied[b], cudaEventDisableTiming));
    if (!p->consumed[b]) HR_CUDA_TRY(cudaEventCreateWithFlags(&p->consumed[b], cudaEventDisableTiming));
  }
  if (!p->bp_done) HR_CUDA_TRY(cudaEventCreateWithFlags(&p->bp_done, cudaEventDisableTiming));
  p->host_ready = true;
  return HR_OK;
}

// The order in which hr_batch_execute_host streams the scans in: the smallest
// fan first (the first copy overlaps nothing), then the others largest first,
// so that the last scan, whose compute and copy-out overlap nothing, is small.
std::vector<int> host_order(const hr_batch_plan* p) {
  std::vector<int> o(p->n);
  for (int i = 0; i < p->n; ++i) o[i] = i;
  std::stable_sort(o.begin(), o.end(),
                   [p](int a, int b) { return fan_elems(p->d[a]) > fan_elems(p->d[b]); });
  std::rotate(o.rbegin(), o.rbegin() + 1, o.rend());
  return o;
}

// Picks each scan's slices per thread with its own plan's autotuner (the
// fastest per-slice variant on a band of its slices), then times every batch
// variant on the whole batch and keeps the fastest. Backprojects into scratch
// volumes. HELIXRECON_BATCH_VARIANT=<index> pins the batch variant (the
// per-scan choice still runs).
int autotune(hr_batch_plan* p) {
  size_t total = 0;
  std::vector<size_t> off(p->n);
  for (int i = 0; i < p->n; ++i) {
    off[i] = total;
    total += (size_t)p->d[i].bp.XN * p->d[i].bp.YN * p->d[i].bp.ZN;
  }
  hr::DeviceBuffer tmp;
  HR_TRY(tmp.alloc(total * sizeof(float)));
  std::vector<float*> vols(p->n);
  for (int i = 0; i < p->n; ++i) {
    vols[i] = tmp.as<float>() + off[i];
    HR_CUDA_TRY(cudaMemsetAsync(p->pairs[i], 0,
                                sizeof(uint32_t) * (size_t)p->d[i].bp.PN * p->d[i].ZL * p->d[i].YL, p->sc));
  }
  p->nz.assign(p->n, 8);
  p->tv.assign(p->n, 11);
  p->sv.assign(p->n, 3);
  for (int i = 0; i < p->n; ++i) {
    HR_TRY(hr_bp_autotune(p->bp[i], vols[i], p->pairs[i], p->sc));
    const hr::BpFastGeom* g;
    const hr::BpFast* f;
    HR_TRY(hr::bp_plan_fast_parts(p->bp[i], &g, &f));
    p->nz[i] = hr::bp_fast_best_per_slice_nz(*f);
    p->tv[i] = hr::bp_fast_best_tex_variant(*f);
    p->sv[i] = f->variant;
  }
  const int first_tex = 6;  // the texture variants follow the gather ones
  HR_TRY(set_scan_variants(p, first_tex));
  HR_TRY(fill_textures(p, p->sc));
  const char* pin = std::getenv("HELIXRECON_BATCH_VARIANT");
  if (pin && *pin) {
    char* end = nullptr;
    const long v = std::strtol(pin, &end, 10);
    HR_REQUIRE(*end == '\0' && v >= 0 && v < hr::kBatchVariants_n,
               "HELIXRECON_BATCH_VARIANT must be an integer in [0, %d)", hr::kBatchVariants_n);
    p->variant = (int)v;
    p->tuned = 2;
    return set_scan_variants(p, p->variant);
  }
  cudaEvent_t e0, e1;
  HR_CUDA_TRY(cudaEventCreate(&e0));
  HR_CUDA_TRY(cudaEventCreate(&e1));
  float best = 1e30f;
  int best_v = 0, st = HR_OK;
  for (int v = 0; v < hr::kBatchVariants_n && st == HR_OK; ++v) {
    // per-scan launches: each scan's own choice (fills inside its launch); texture variants: each scan's
    // FP16 texture variant (after the per-scan one, a scan may have switched to another copy)
    if (per_scan(v) || textured(v)) st = set_scan_variants(p, v);
    float ms = 1e30f;
    for (int rep = 0; rep < 2 && st == HR_OK; ++rep) {
      cudaEventRecord(e0, p->sc);
      st = backproject(p, vols.data(), v, p->sc);  // texture fills included
      cudaEventRecord(e1, p->sc);
      if (cudaEventSynchronize(e1) != cudaSuccess) st = hr::fail(HR_ERR_CUDA, "batch autotune: launch failed");
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      if (rep > 0) ms = t;
    }
    p->tuned_ms[v] = ms;
    if (ms < best) {
      best = ms;
      best_v = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != HR_OK) return st;
  p->variant = best_v;
  p->tuned = 1;
  return set_scan_variants(p, p->variant);
}

}  // namespace

extern "C" int hr_batch_plan_create(hr_batch_plan** plan, const hr_recon_desc* descs, int n) {
  hr::clear_error();
  HR_REQUIRE(plan != nullptr && descs != nullptr, "hr_batch_plan_create: NULL argument");
  *plan = nullptr;
  HR_REQUIRE(n >= 1 && n <= hr::kBatchMaxScans, "hr_batch_plan_create: %d scans (1..%d)", n, hr::kBatchMaxScans);
  for (int i = 0; i < n; ++i) {
    const hr_recon_desc& d = descs[i];
    HR_REQUIRE(d.w != nullptr, "hr_batch_plan_create: scan %d has no weight table", i);
    HR_REQUIRE(d.form == HR_FORM_FAST, "hr_batch_plan_create: scan %d: the batch runs the fast form only", i);
    HR_REQUIRE(d.bp.YL == d.YL && d.bp.ZL == d.ZL, "hr_batch_plan_create: scan %d: bp.YL/ZL differ from YL/ZL", i);
    HR_REQUIRE(d.view0 >= 0 && d.view0 + d.bp.PN <= d.ViewN,
               "hr_batch_plan_create: scan %d: views [%d, %d) exceed the %d rebinned views", i, d.view0,
               d.view0 + d.bp.PN, d.ViewN);
  }
  HR_TRY(hr::require_device());
  hr_batch_plan* p = new hr_batch_plan;
  p->n = n;
  p->d.assign(descs, descs + n);
  size_t nfan_max = 0, split_max = 0;
  for (int i = 0; i < n; ++i) {
    p->d[i].w = nullptr;
    nfan_max = std::max(nfan_max, (size_t)descs[i].YL * descs[i].ZL * descs[i].ViewN);
    split_max = std::max(split_max, hr::filter_tc_scratch_bytes(descs[i].YL, descs[i].ZL, descs[i].bp.PN));
  }
  int st = alloc(p, (void**)&p->d_rebinned, nfan_max * sizeof(float));
  if (st == HR_OK) st = alloc(p, (void**)&p->d_counter, sizeof(int));
  for (int k = 0; k < 3 && st == HR_OK; ++k) st = alloc(p, &p->d_split[k], split_max);
  for (int i = 0; i < n && st == HR_OK; ++i) {
    const hr_recon_desc& d = descs[i];
    hr_rebin_plan* r = nullptr;
    hr_filter_tc_plan* f = nullptr;
    hr_bp_plan* b = nullptr;
    uint32_t* q = nullptr;
    st = hr_rebin_plan_create(&r, d.YL, d.ZL, d.ViewN, d.YLC, d.dYA, d.DeltaTheta, d.PLC, d.DeltaT, d.DeltaFai,
                              d.SO);
    p->rebin.push_back(r);
    if (st == HR_OK)
      st = hr::filter_tc_create_shared(&f, d.YL, d.ZL, d.bp.PN, d.fPLC, d.fZLC, d.fdYL, d.fdZL, d.fSO, p->d_split);
    p->ftc.push_back(f);
    if (st == HR_OK) st = hr_bp_plan_create(&b, &d.bp, d.w, HR_FORM_FAST);
    p->bp.push_back(b);
    if (st == HR_OK) st = alloc(p, (void**)&q, sizeof(uint32_t) * (size_t)d.bp.PN * d.ZL * d.YL);
    p->pairs.push_back(q);
  }
  for (int v = 0; v < hr::kBatchVariants_n && st == HR_OK; ++v) st = hr::bp_fast_batch_grid(v, &p->ctas[v]);
  if (st == HR_OK) {
    cudaError_t e = cudaStreamCreateWithFlags(&p->sc, cudaStreamNonBlocking);
    p->ss.assign(n, nullptr);
    p->ready.assign(n, nullptr);
    p->done.assign(n, nullptr);
    for (int i = 0; i < n && e == cudaSuccess; ++i) {
      e = cudaStreamCreateWithFlags(&p->ss[i], cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ready[i], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->done[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) st = hr::fail(HR_ERR_CUDA, "hr_batch_plan_create: %s", cudaGetErrorString(e));
  }
  if (st == HR_OK) st = autotune(p);
  if (st != HR_OK) {
    destroy(p);
    return st;
  }
  if (hr::log_enabled()) {
    char desc[768];
    if (hr_batch_describe(p, desc, sizeof(desc)) == HR_OK)
      hr::log("batch plan: %.2f GB on the device; %s", hr_batch_device_bytes(p) / 1e9, desc);
  }
  *plan = p;
  return HR_OK;
}

extern "C" int hr_batch_execute(hr_batch_plan* p, float* const* d_vols, const float* const* d_fans, void* stream) {
  HR_REQUIRE(p != nullptr && d_vols != nullptr && d_fans != nullptr, "hr_batch_execute: NULL argument");
  std::vector<const void*> ptrs;
  for (int i = 0; i < p->n; ++i) {
    HR_REQUIRE(d_vols[i] != nullptr && d_fans[i] != nullptr, "hr_batch_execute: NULL buffer for scan %d", i);
    ptrs.push_back(d_vols[i]);
    ptrs.push_back(d_fans[i]);
  }
  cudaStream_t s = hr::as_stream(stream);
  if (!p->graph || ptrs != p->graph_ptrs || p->graph_variant != p->variant) {
    if (p->graph) cudaGraphExecDestroy(p->graph);
    p->graph = nullptr;
    cudaGraph_t gr = nullptr;
    HR_CUDA_TRY(cudaStreamBeginCapture(p->sc, cudaStreamCaptureModeRelaxed));
    const int st = enqueue(p, d_vols, d_fans, p->sc);
    const cudaError_t e = cudaStreamEndCapture(p->sc, &gr);
    if (st != HR_OK || e != cudaSuccess) {
      if (gr) cudaGraphDestroy(gr);
      return st != HR_OK ? st : hr::fail(HR_ERR_CUDA, "hr_batch_execute: capture failed: %s", cudaGetErrorString(e));
    }
    const cudaError_t ei = cudaGraphInstantiate(&p->graph, gr, 0);
    cudaGraphDestroy(gr);
    if (ei != cudaSuccess) {
      p->graph = nullptr;
      return hr::fail(HR_ERR_CUDA, "hr_batch_execute: graph instantiation failed: %s", cudaGetErrorString(ei));
    }
    p->graph_ptrs = ptrs;
    p->graph_variant = p->variant;
  }
  HR_CUDA_TRY(cudaGraphLaunch(p->graph, s));
  return HR_OK;
}

extern "C" int hr_batch_execute_host(hr_batch_plan* p, float* const* h_vols, const float* const* h_fans) {
  hr::clear_error();
  HR_REQUIRE(p != nullptr && h_vols != nullptr && h_fans != nullptr, "hr_batch_execute_host: NULL argument");
  for (int i = 0; i < p->n; ++i)
    HR_REQUIRE(h_vols[i] != nullptr && h_fans[i] != nullptr, "hr_batch_execute_host: NULL buffer for scan %d", i);
  HR_TRY(host_buffers(p));
  const std::vector<int> order = host_order(p);
  std::vector<float*> dv(p->n);
  for (int i = 0; i < p->n; ++i) dv[i] = p->d_hvol + p->voff[i];
  const bool fork = per_scan(p->variant);
  cudaStream_t s = p->sc;
  // Enqueues every scan; on a failure it returns with earlier work possibly in flight.
  auto enqueue = [&]() -> int {
    for (int j = 0; j < p->n; ++j) {
      const int i = order[j], b = j & 1;
      // the fan of scan j goes to staging buffer b once scan j-2's rebinning has read it
      HR_CUDA_TRY(cudaStreamWaitEvent(p->sin, p->consumed[b], 0));
      HR_CUDA_TRY(cudaMemcpyAsync(p->d_stage[b], h_fans[i], fan_elems(p->d[i]) * sizeof(float),
                                  cudaMemcpyHostToDevice, p->sin));
      HR_CUDA_TRY(cudaEventRecord(p->copied[b], p->sin));
      HR_CUDA_TRY(cudaStreamWaitEvent(s, p->copied[b], 0));
      HR_TRY(hr_rebin_execute(p->rebin[i], p->d_rebinned, p->d_stage[b], s));
      HR_CUDA_TRY(cudaEventRecord(p->consumed[b], s));
      HR_TRY(hr_filter_tc_execute(p->ftc[i], p->pairs[i], p->d_rebinned, HR_LAYOUT_REBIN, p->d[i].view0, s));
      if (fork) {
        // the scan's backprojection on its own stream, its volume out as soon as it is done
        HR_TRY(fork_bp(p, i, dv[i], s));
        HR_CUDA_TRY(cudaStreamWaitEvent(p->sout, p->done[i], 0));
        HR_CUDA_TRY(cudaMemcpyAsync(h_vols[i], dv[i], vol_elems(p->d[i]) * sizeof(float), cudaMemcpyDeviceToHost,
                                    p->sout));
      }
    }
    if (!fork) {
      HR_TRY(backproject(p, dv.data(), p->variant, s));
      HR_CUDA_TRY(cudaEventRecord(p->bp_done, s));
      HR_CUDA_TRY(cudaStreamWaitEvent(p->sout, p->bp_done, 0));
      for (int i = 0; i < p->n; ++i)
        HR_CUDA_TRY(cudaMemcpyAsync(h_vols[i], dv[i], vol_elems(p->d[i]) * sizeof(float), cudaMemcpyDeviceToHost,
                                    p->sout));
    } else {
      HR_TRY(join_all(p, s));
    }
    return HR_OK;
  };
  int st = enqueue();
  // whether or not everything was enqueued, no copy may still use the caller's buffers on return
  for (cudaStream_t s2 : {p->sout, s, p->sin}) {
    const cudaError_t e = cudaStreamSynchronize(s2);
    if (e != cudaSuccess && st == HR_OK)
      st = hr::fail(HR_ERR_CUDA, "hr_batch_execute_host: %s", cudaGetErrorString(e));
  }
  HR_TRY(st);
  return hr_batch_check(p);
}

extern "C" int hr_batch_backproject(hr_batch_plan* p, float* const* d_vols, void* stream) {
  HR_REQUIRE(p != nullptr && d_vols != nullptr, "hr_batch_backproject: NULL argument");
  for (int i = 0; i < p->n; ++i) HR_REQUIRE(d_vols[i] != nullptr, "hr_batch_backproject: NULL volume %d", i);
  return backproject(p, d_vols, p->variant, hr::as_stream(stream));
}

extern "C" int hr_batch_select(hr_batch_plan* p, int variant) {
  HR_REQUIRE(p != nullptr, "hr_batch_select: NULL plan");
  HR_REQUIRE(variant >= 0 && variant < hr::kBatchVariants_n, "hr_batch_select: variant %d out of range [0, %d)",
             variant, hr::kBatchVariants_n);
  HR_TRY(set_scan_variants(p, variant));
  p->variant = variant;
  return HR_OK;
}

extern "C" int hr_batch_describe(const hr_batch_plan* p, char* buf, int len) {
  HR_REQUIRE(p != nullptr, "hr_batch_describe: NULL plan");
  if (!buf || len <= 0) return HR_OK;
  std::vector<float*> vols(p->n, nullptr);
  std::vector<hr::BpFastBatchScan> sc;
  HR_TRY(scans_of(p, vols.data(), p->variant, &sc));
  const hr::BatchVariant& bv = hr::kBatchVariants[p->variant];
  int k = 0;
  if (bv.streams) {
    k = snprintf(buf, (size_t)len, "%d scans, each scan's own backprojection on a stream of its own (fork/join in "
                 "the graph); variant by scan:", p->n);
    for (int i = 0; i < p->n && k > 0 && k < len; ++i) k += snprintf(buf + k, (size_t)(len - k), " %d", p->sv[i]);
  } else {
    k = snprintf(buf, (size_t)len,
                 "%d scans, %lld work items in one persistent launch of %d CTAs (>= %d per SM, taps %s); "
                 "slices per thread by scan:", p->n, hr::bp_fast_batch_items(sc.data(), p->n),
                 p->ctas[p->variant], bv.min_ctas,
                 bv.tex ? (bv.seg ? "from FP16 textures, segmented view loop"
                           : bv.spec ? "from FP16 textures, code specialised per scan" : "from FP16 textures")
                 : bv.chunk > 0 ? "gathered in chunks of 4 slices" : "gathered per slice");
    for (int i = 0; i < p->n && k > 0 && k < len; ++i) k += snprintf(buf + k, (size_t)(len - k), " %d", sc[i].nz);
  }
  if (k > 0 && k < len)
    k += snprintf(buf + k, (size_t)(len - k), " %s",
                  p->tuned == 2 ? "(pinned by HELIXRECON_BATCH_VARIANT)"
                  : p->tuned ? "(autotuned; batch ms:" : "(selected)");
  if (p->tuned == 1) {
    for (int v = 0; v < hr::kBatchVariants_n && k > 0 && k < len; ++v)
      k += snprintf(buf + k, (size_t)(len - k), " v%d=%.2f", v, p->tuned_ms[v]);
    if (k > 0 && k < len) snprintf(buf + k, (size_t)(len - k), ")");
  }
  return HR_OK;
}

extern "C" int hr_batch_check(const hr_batch_plan* p) {
  HR_REQUIRE(p != nullptr, "hr_batch_check: NULL plan");
  for (auto* f : p->ftc) HR_TRY(hr_filter_tc_check(f));
  return HR_OK;
}

extern "C" size_t hr_batch_device_bytes(const hr_batch_plan* p) {
  if (!p) return 0;
  size_t b = p->bytes;
  for (auto* f : p->ftc) b += hr_filter_tc_device_bytes(f);
  for (auto* q : p->bp) {
    const hr::BpFastGeom* g;
    const hr::BpFast* f;
    if (hr::bp_plan_fast_parts(q, &g, &f) == HR_OK) b += hr::bp_fast_device_bytes(*f);
  }
  return b;
}

extern "C" void hr_batch_plan_destroy(hr_batch_plan* p) { destroy(p); }
