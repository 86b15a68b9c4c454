// Slab-batched reconstruction of long (big-patient) scans.
//
// The reference reconstructs a long scan by cutting the view stream into
// overlapping segments, reconstructing the WHOLE volume from each segment and
// summing the volumes on the host (src/analyticalRecon.m:15-25,
// src/readBigPatientData.m:15-34). Here the volume is cut instead: z slabs of
// S slices are disjoint in the output, and a slab needs only the views of its
// own window [s1(first slice), s2(last slice)] plus the half-fan rebinning
// margin, so nothing is summed and no view outside the window is touched.
//
// Every slab is processed with the same shapes: its backprojection window has
// a fixed length of Wbp views starting at a clamped first view, and its fan
// window is those views plus the half-fan margin on both sides (the margin is
// the crop of the whole-scan plan, so a fan window always lies inside the
// scan). The per-slab geometry (first view angle, z offset) lives only in the
// backprojection tables, so one captured CUDA graph -- rebin, preweight/split,
// tensor-core filter, backprojection -- serves every slab of a buffer parity.
// Each slab runs as two captured graphs on two streams: rebin + tensor-core
// filter (into one of two filtered buffers) on a high-priority stream, and the
// backprojection on another, so that slab k+1's filter (tensor cores) runs
// under slab k's backprojection (texture units): the scheduler places the
// filter's CTAs on SMs as backprojection CTAs retire. Fan windows are copied
// into ping-pong buffers on a third stream while earlier slabs compute, and
// each slab's volume leaves its own ping-pong buffer on a fourth stream; each
// slab's tables are built on the host in FP64 and uploaded in stream order
// before its backprojection. Consecutive slabs' fan windows overlap (by the backprojection window
// minus the slab advance, plus the margins): the overlap is copied on the
// device from the previous window's buffer and only the views a slab adds
// cross the host link.
//
// Several GPUs split one scan by slabs (one plan per rank, `part` of `nparts`):
// each rank rebins, filters and backprojects only its own slabs from its own
// fan windows and writes only their slices; there is nothing to exchange.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "bp_fast.h"
#include "hr_internal.h"

namespace {

// Slab decomposition of a scan: slab k holds slices [k S, min(ZN, (k+1) S));
// its backprojection window is Wbp views starting at p_start[k] (views of the
// cropped, rebinned scan) and its fan window Wfan = Wbp + 2 margin fan views
// starting at a0[k] = view0 + p_start[k] - margin.
struct SlabLayout {
  int S = 0, nslabs = 0, Wbp = 0, Wfan = 0, margin = 0, half = 0;
  std::vector<int> p_start, a0, first_slice, n_slices;
};

}  // namespace

struct hr_slab_plan {
  hr_recon_desc d;
  SlabLayout L;
  int part = 0, nparts = 1, assign = HR_SLAB_BLOCKS;
  int filter_ctas = 0;  // CTAs of the rebin and split launches beside the backprojection
  std::vector<int> mine;  // slabs of this plan, in z order
  int fan_first = 0, fan_count = 0;  // fan views the plan reads: [fan_first, fan_first + fan_count)
  size_t fan_bytes = 0;   // bytes copied from the caller's fan per execution
  hr_rebin_plan* rebin = nullptr;
  hr_filter_tc_plan* ftc = nullptr;
  hr::BpFast fast[2];
  hr::BpFastGeom gslab{};
  std::vector<double> w;
  float* d_fan[2] = {nullptr, nullptr};
  float* d_reb = nullptr;
  uint32_t* d_pairs[2] = {nullptr, nullptr};
  float* d_vslab[2] = {nullptr, nullptr};
  // sf: rebin + filter (high priority); sc: backprojection; scopy: fan in; sout: volume out
  cudaStream_t sf = nullptr, sc = nullptr, scopy = nullptr, sout = nullptr;
  cudaEvent_t copied[2] = {nullptr, nullptr}, consumed[2] = {nullptr, nullptr};
  cudaEvent_t filtered[2] = {nullptr, nullptr}, computed[2] = {nullptr, nullptr}, drained[2] = {nullptr, nullptr};
  cudaGraphExec_t gfilter[2] = {nullptr, nullptr}, gbp[2] = {nullptr, nullptr};
  size_t bytes = 0;
};

namespace {

int s0_of(const hr_bp_geom& g, int zi) {
  const double z = (zi - g.ZNC) * g.dz;
  const double beta0 = 2.0 * 3.14159265358979 * z / g.h;
  return (int)std::ceil((beta0 - g.BetaS) / g.DeltaFai - 0.5);
}

// Checks a whole-scan description for slab processing and computes its slab
// windows (host arithmetic only).
int slab_layout(const hr_recon_desc* d, int slab_slices, SlabLayout* L) {
  HR_REQUIRE(slab_slices > 0 && slab_slices <= 4096, "slab pipeline: slab of %d slices", slab_slices);
  HR_REQUIRE(d->DeltaTheta == d->DeltaFai,
             "slab pipeline: windowed rebinning needs DeltaTheta == DeltaFai (as the reference driver passes)");
  HR_REQUIRE(d->bp.YL == d->YL && d->bp.ZL == d->ZL, "slab pipeline: bp.YL/ZL differ from YL/ZL");
  HR_REQUIRE(d->view0 >= 0 && d->view0 + d->bp.PN + d->view0 <= d->ViewN,
             "slab pipeline: the crop must be symmetric (views [view0, view0+PN) plus view0 behind)");
  const hr_bp_geom& G = d->bp;
  HR_REQUIRE(G.ZN > 0 && G.PN > 0 && G.h != 0.0 && G.DeltaFai != 0.0, "slab pipeline: invalid geometry");
  *L = SlabLayout{};
  L->S = std::min(slab_slices, G.ZN);
  L->nslabs = (G.ZN + L->S - 1) / L->S;
  L->margin = d->view0;
  L->half = (int)std::ceil(G.N_pi * G.HSCoef);
  int wmax = 1;
  std::vector<int> lo(L->nslabs), hi(L->nslabs);
  for (int k = 0; k < L->nslabs; ++k) {
    const int z0 = k * L->S, z1 = std::min(G.ZN, z0 + L->S) - 1;
    const int sa = s0_of(G, z0), sb = s0_of(G, z1);
    lo[k] = std::max(0, std::min(sa, sb) - L->half);
    hi[k] = std::min(G.PN - 1, std::max(sa, sb) + L->half);
    if (hi[k] >= lo[k]) wmax = std::max(wmax, hi[k] - lo[k] + 1);
    L->first_slice.push_back(z0);
    L->n_slices.push_back(z1 - z0 + 1);
  }
  L->Wbp = std::min(wmax, G.PN);
  L->Wfan = L->Wbp + 2 * L->margin;
  for (int k = 0; k < L->nslabs; ++k) {
    const int ps = std::max(0, std::min(lo[k], G.PN - L->Wbp));
    L->p_start.push_back(ps);
    L->a0.push_back(d->view0 + ps - L->margin);  // >= 0, and a0 + Wfan <= ViewN
  }
  return HR_OK;
}

// Slabs of part `part` of `nparts`: contiguous blocks of slabs in z order
// (HR_SLAB_BLOCKS; the first nslabs % nparts parts take one slab more) or
// every nparts-th slab (HR_SLAB_ROUND_ROBIN).
int slab_part(int nslabs, int part, int nparts, int assign, std::vector<int>* mine) {
  HR_REQUIRE(nparts >= 1 && part >= 0 && part < nparts, "slab pipeline: part %d of %d", part, nparts);
  HR_REQUIRE(nparts <= nslabs, "slab pipeline: %d parts for %d slabs (every part needs a slab)", nparts, nslabs);
  HR_REQUIRE(assign == HR_SLAB_BLOCKS || assign == HR_SLAB_ROUND_ROBIN, "slab pipeline: unknown assignment %d",
             assign);
  mine->clear();
  if (assign == HR_SLAB_ROUND_ROBIN) {
    for (int k = part; k < nslabs; k += nparts) mine->push_back(k);
  } else {
    const int base = nslabs / nparts, extra = nslabs % nparts;
    const int first = part * base + std::min(part, extra);
    const int count = base + (part < extra ? 1 : 0);
    for (int k = first; k < first + count; ++k) mine->push_back(k);
  }
  return HR_OK;
}

// Fan views the j-th slab of a part shares with its (j-1)-th (0 for the first).
int overlap_views(const SlabLayout& L, const std::vector<int>& mine, int j) {
  if (j == 0) return 0;
  return std::max(0, std::min(L.Wfan, L.a0[mine[j - 1]] + L.Wfan - L.a0[mine[j]]));
}

void destroy(hr_slab_plan* p) {
  if (!p) return;
  for (int i = 0; i < 2; ++i) {
    if (p->gfilter[i]) cudaGraphExecDestroy(p->gfilter[i]);
    if (p->gbp[i]) cudaGraphExecDestroy(p->gbp[i]);
    hr::bp_fast_destroy(&p->fast[i]);
    cudaFree(p->d_fan[i]);
    cudaFree(p->d_vslab[i]);
    cudaFree(p->d_pairs[i]);
    if (p->copied[i]) cudaEventDestroy(p->copied[i]);
    if (p->consumed[i]) cudaEventDestroy(p->consumed[i]);
    if (p->filtered[i]) cudaEventDestroy(p->filtered[i]);
    if (p->computed[i]) cudaEventDestroy(p->computed[i]);
    if (p->drained[i]) cudaEventDestroy(p->drained[i]);
  }
  hr_rebin_plan_destroy(p->rebin);
  hr_filter_tc_plan_destroy(p->ftc);
  cudaFree(p->d_reb);
  if (p->sf) cudaStreamDestroy(p->sf);
  if (p->sc) cudaStreamDestroy(p->sc);
  if (p->scopy) cudaStreamDestroy(p->scopy);
  if (p->sout) cudaStreamDestroy(p->sout);
  delete p;
}

int alloc(hr_slab_plan* p, void** ptr, size_t bytes) {
  HR_CUDA_TRY(cudaMalloc(ptr, bytes));
  p->bytes += bytes;
  return HR_OK;
}

// Geometry of slab k for the fast backprojection tables.
hr::BpFastGeom slab_geom(const hr_slab_plan* p, int k) {
  hr::BpFastGeom g = p->gslab;
  const hr_bp_geom& G = p->d.bp;
  g.ZNC = G.ZNC - p->L.first_slice[k];
  g.BetaS = G.BetaS + p->L.p_start[k] * G.DeltaFai;
  g.ZN_valid = p->L.n_slices[k];
  return g;
}

// Fan window of the plan's j-th slab into buffer j & 1 on the copy stream.
// `fan` points at fan view `fan_view0`. With `incremental`, the views shared
// with slab j-1 come from the other buffer (device to device; that buffer was
// filled earlier on this stream) and only the new ones from `fan`.
int enqueue_fan_copy(hr_slab_plan* p, int j, const float* fan, int fan_view0, bool fan_on_host, bool incremental) {
  const SlabLayout& L = p->L;
  const int k = p->mine[j], b = j & 1;
  const size_t per_view = (size_t)p->d.YL * p->d.ZL;
  HR_CUDA_TRY(cudaStreamWaitEvent(p->scopy, p->consumed[b], 0));
  const int ov = incremental ? overlap_views(L, p->mine, j) : 0;
  if (ov > 0) {
    const int shift = L.a0[k] - L.a0[p->mine[j - 1]];
    HR_CUDA_TRY(cudaMemcpyAsync(p->d_fan[b], p->d_fan[b ^ 1] + (size_t)shift * per_view, (size_t)ov * per_view * 4,
                                cudaMemcpyDeviceToDevice, p->scopy));
  }
  if (ov < L.Wfan)
    HR_CUDA_TRY(cudaMemcpyAsync(p->d_fan[b] + (size_t)ov * per_view,
                                fan + (size_t)(L.a0[k] + ov - fan_view0) * per_view,
                                (size_t)(L.Wfan - ov) * per_view * 4,
                                fan_on_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, p->scopy));
  HR_CUDA_TRY(cudaEventRecord(p->copied[b], p->scopy));
  return HR_OK;
}

// The two halves of one slab for buffer parity b (what the graphs capture):
// rebin + filter from fan buffer b into filtered buffer b, and the
// backprojection of filtered buffer b into slab buffer b (for a texture
// variant with the fill of its layered copy first). Filling on the filter
// stream instead, under the previous slab's backprojection, measured slower
// (big patient 659 against 639 ms on the device, 1.43 against 1.03 s from
// host memory, same box).
int slab_filter(hr_slab_plan* p, int b, cudaStream_t s) {
  HR_TRY(hr::rebin_execute_limited(p->rebin, p->d_reb, p->d_fan[b], p->filter_ctas, s));
  return hr::filter_tc_execute_limited(p->ftc, p->d_pairs[b], p->d_reb, HR_LAYOUT_REBIN, p->L.margin,
                                       p->filter_ctas, s);
}
int slab_bp(hr_slab_plan* p, int b, cudaStream_t s) {
  return hr::bp_fast_execute(p->fast[b], p->gslab, p->d_vslab[b], p->d_pairs[b], s);
}

// Captures fn(p, b, s) on stream s into an executable graph.
int capture(hr_slab_plan* p, int b, cudaStream_t s, int (*fn)(hr_slab_plan*, int, cudaStream_t),
            cudaGraphExec_t* out) {
  cudaGraph_t gr = nullptr;
  HR_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
  const int st = fn(p, b, s);
  const cudaError_t e = cudaStreamEndCapture(s, &gr);
  if (st != HR_OK) {
    if (gr) cudaGraphDestroy(gr);
    return st;
  }
  HR_CUDA_TRY(e);
  const cudaError_t ei = cudaGraphInstantiate(out, gr, 0);
  cudaGraphDestroy(gr);
  HR_CUDA_TRY(ei);
  return HR_OK;
}

}  // namespace

extern "C" int hr_slab_windows(const hr_recon_desc* d, int slab_slices, int part, int nparts, int assign,
                               hr_slab_window* out, int cap, int* n) {
  hr::clear_error();
  HR_REQUIRE(d != nullptr && n != nullptr, "hr_slab_windows: NULL argument");
  SlabLayout L;
  HR_TRY(slab_layout(d, slab_slices, &L));
  std::vector<int> mine;
  HR_TRY(slab_part(L.nslabs, part, nparts, assign, &mine));
  *n = (int)mine.size();
  HR_REQUIRE(out == nullptr || cap >= (int)mine.size(), "hr_slab_windows: %d slabs, room for %d", (int)mine.size(),
             cap);
  if (out == nullptr) return HR_OK;
  for (size_t j = 0; j < mine.size(); ++j) {
    const int k = mine[j];
    out[j] = hr_slab_window{k, L.first_slice[k], L.n_slices[k], L.p_start[k], L.Wbp, L.a0[k], L.Wfan,
                            overlap_views(L, mine, (int)j)};
  }
  return HR_OK;
}

extern "C" int hr_slab_plan_create_part(hr_slab_plan** plan, const hr_recon_desc* d, int slab_slices, int part,
                                        int nparts, int assign) {
  hr::clear_error();
  HR_REQUIRE(plan != nullptr && d != nullptr && d->w != nullptr, "hr_slab_plan_create: NULL argument");
  *plan = nullptr;
  HR_REQUIRE(d->form == HR_FORM_FAST, "hr_slab_plan_create: the slab pipeline runs the fast form");
  SlabLayout L;
  HR_TRY(slab_layout(d, slab_slices, &L));
  std::vector<int> mine;
  HR_TRY(slab_part(L.nslabs, part, nparts, assign, &mine));
  HR_TRY(hr::require_device());
  hr_slab_plan* p = new hr_slab_plan;
  p->d = *d;
  p->d.w = nullptr;
  p->w.assign(d->w, d->w + d->bp.N_2pi);
  p->L = L;
  p->part = part;
  p->nparts = nparts;
  p->assign = assign;
  p->mine = mine;
  // The rebinning and the split stride over their views with 8 CTAs per SM instead of one CTA per tile:
  // the device time is the same, and from host memory the big patient took 0.86-0.88 s instead of 1.06 s
  // (A/B on one box; 1 CTA per SM was 1.36x slower on the device).
  p->filter_ctas = 8 * hr::sm_count();
  const hr_bp_geom& G = d->bp;
  const size_t per_view = (size_t)d->YL * d->ZL;
  p->fan_first = L.a0[mine.front()];
  p->fan_count = L.a0[mine.back()] + L.Wfan - p->fan_first;
  for (size_t j = 0; j < mine.size(); ++j)
    p->fan_bytes += (size_t)(L.Wfan - overlap_views(L, mine, (int)j)) * per_view * 4;
  // geometry template of a slab (the per-slab parts are set by slab_geom)
  hr::BpFastGeom& g = p->gslab;
  g.XN = G.XN; g.YN = G.YN; g.ZN = L.S; g.YL = G.YL; g.ZL = G.ZL; g.PN = L.Wbp; g.half = L.half;
  g.ZN_valid = L.S;
  g.XNC = G.XNC; g.YNC = G.YNC; g.ZNC = G.ZNC; g.dx = G.dx; g.dy = G.dy; g.dz = G.dz;
  g.YLC = G.YLC; g.ZLC = G.ZLC; g.dYL = G.dYL; g.dZL = G.dZL; g.h = G.h; g.BetaS = G.BetaS;
  g.DeltaFai = G.DeltaFai; g.N_pi = G.N_pi; g.SO = G.SO; g.SD = G.SD; g.k1 = G.k1;

  int st = hr_rebin_plan_create(&p->rebin, d->YL, d->ZL, L.Wfan, d->YLC, d->dYA, d->DeltaTheta, d->PLC, d->DeltaT,
                                d->DeltaFai, d->SO);
  if (st == HR_OK)
    st = hr_filter_tc_plan_create(&p->ftc, d->YL, d->ZL, L.Wbp, d->fPLC, d->fZLC, d->fdYL, d->fdZL, d->fSO);
  // table capacity: the largest tables over the plan's slabs
  size_t rows[hr::kFastTableSets] = {0};
  int nb[hr::kFastTableSets] = {0};
  for (size_t j = 0; j < mine.size() && st == HR_OK; ++j) {
    hr::BpFastHost h;
    st = hr::bp_fast_host_tables(&h, slab_geom(p, mine[j]), p->w.data());
    for (int i = 0; i < hr::kFastTableSets && st == HR_OK; ++i) {
      rows[i] = std::max(rows[i], h.set[i].mask.size());
      nb[i] = h.set[i].nblocks;
    }
  }
  for (int b = 0; b < 2 && st == HR_OK; ++b) st = hr::bp_fast_reserve(&p->fast[b], rows, nb, L.Wbp);
  for (int b = 0; b < 2 && st == HR_OK; ++b) st = alloc(p, (void**)&p->d_fan[b], (size_t)L.Wfan * per_view * 4);
  if (st == HR_OK) st = alloc(p, (void**)&p->d_reb, (size_t)L.Wfan * per_view * 4);
  for (int b = 0; b < 2 && st == HR_OK; ++b) st = alloc(p, (void**)&p->d_pairs[b], (size_t)L.Wbp * per_view * 4);
  for (int b = 0; b < 2 && st == HR_OK; ++b) st = alloc(p, (void**)&p->d_vslab[b], (size_t)G.XN * G.YN * L.S * 4);
  if (st == HR_OK) {
    int prio_lo = 0, prio_hi = 0;
    cudaError_t e = cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&p->sf, cudaStreamNonBlocking, prio_hi);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->sc, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->scopy, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->sout, cudaStreamNonBlocking);
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
      e = cudaEventCreateWithFlags(&p->copied[b], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->consumed[b], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->filtered[b], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->computed[b], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->drained[b], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) st = hr::fail(HR_ERR_CUDA, "hr_slab_plan_create: %s", cudaGetErrorString(e));
  }
  if (st != HR_OK) {
    destroy(p);
    return st;
  }
  *plan = p;
  return HR_OK;
}

extern "C" int hr_slab_plan_create(hr_slab_plan** plan, const hr_recon_desc* d, int slab_slices) {
  return hr_slab_plan_create_part(plan, d, slab_slices, 0, 1, HR_SLAB_BLOCKS);
}

// Picks the backprojection variant on the plan's middle slab's real data and
// captures the two per-parity graphs. Runs once, on the first execution.
static int prepare(hr_slab_plan* p, const float* fan, int fan_view0, bool fan_on_host) {
  const int j = (int)p->mine.size() / 2, k = p->mine[j], b = j & 1;
  HR_TRY(enqueue_fan_copy(p, j, fan, fan_view0, fan_on_host, false));
  HR_CUDA_TRY(cudaStreamWaitEvent(p->sc, p->copied[b], 0));
  hr::BpFastHost h;
  HR_TRY(hr::bp_fast_host_tables(&h, slab_geom(p, k), p->w.data()));
  HR_TRY(hr::bp_fast_upload(&p->fast[b], h, p->sc));
  HR_TRY(slab_filter(p, b, p->sc));
  HR_TRY(hr::bp_fast_autotune(&p->fast[b], p->gslab, p->d_vslab[b], p->d_pairs[b], p->sc));
  p->fast[b ^ 1].variant = p->fast[b].variant;
  p->fast[b ^ 1].tuned = p->fast[b].tuned;
  std::memcpy(p->fast[b ^ 1].tuned_ms, p->fast[b].tuned_ms, sizeof(p->fast[b].tuned_ms));
  HR_TRY(hr::bp_fast_tex_prepare(&p->fast[b ^ 1], p->gslab));
  HR_CUDA_TRY(cudaStreamSynchronize(p->sc));
  HR_CUDA_TRY(cudaStreamSynchronize(p->scopy));
  for (int bb = 0; bb < 2; ++bb) {
    HR_TRY(capture(p, bb, p->sf, slab_filter, &p->gfilter[bb]));
    HR_TRY(capture(p, bb, p->sc, slab_bp, &p->gbp[bb]));
  }
  if (hr::log_enabled()) {
    char desc[1024];
    if (hr_slab_describe(p, desc, sizeof(desc)) == HR_OK) hr::log("slab plan prepared: %s", desc);
  }
  return HR_OK;
}

extern "C" int hr_slab_execute_range(hr_slab_plan* p, float* vol, const float* fan, int fan_view0, int vol_on_host,
                                     int fan_on_host) {
  hr::clear_error();
  HR_REQUIRE(p != nullptr && vol != nullptr && fan != nullptr, "hr_slab_execute: NULL argument");
  HR_REQUIRE(fan_view0 >= 0 && fan_view0 <= p->fan_first,
             "hr_slab_execute: fan starts at view %d, the plan reads from view %d", fan_view0, p->fan_first);
  if (!p->gbp[0]) HR_TRY(prepare(p, fan, fan_view0, fan_on_host != 0));
  const hr_bp_geom& G = p->d.bp;
  const SlabLayout& L = p->L;
  const int n = (int)p->mine.size();
  // Enqueues every slab; on a failure it returns with earlier work possibly in flight.
  auto enqueue = [&]() -> int {
    HR_TRY(enqueue_fan_copy(p, 0, fan, fan_view0, fan_on_host != 0, true));
    for (int j = 0; j < n; ++j) {
      const int k = p->mine[j], b = j & 1;
      // rebin + filter of slab j on the filter stream (under slab j-1's backprojection)
      HR_CUDA_TRY(cudaStreamWaitEvent(p->sf, p->copied[b], 0));
      HR_CUDA_TRY(cudaStreamWaitEvent(p->sf, p->computed[b], 0));  // slab j-2's backprojection has read d_pairs[b]
      HR_CUDA_TRY(cudaGraphLaunch(p->gfilter[b], p->sf));
      HR_CUDA_TRY(cudaEventRecord(p->consumed[b], p->sf));
      HR_CUDA_TRY(cudaEventRecord(p->filtered[b], p->sf));
      if (j + 1 < n) HR_TRY(enqueue_fan_copy(p, j + 1, fan, fan_view0, fan_on_host != 0, true));
      // tables of slab k: host build (overlaps the GPU), stream-ordered upload, backprojection
      hr::BpFastHost h;
      HR_TRY(hr::bp_fast_host_tables(&h, slab_geom(p, k), p->w.data()));
      HR_CUDA_TRY(cudaStreamWaitEvent(p->sc, p->filtered[b], 0));
      HR_CUDA_TRY(cudaStreamWaitEvent(p->sc, p->drained[b], 0));  // slab j-2's volume has left d_vslab[b]
      HR_TRY(hr::bp_fast_upload(&p->fast[b], h, p->sc));
      HR_CUDA_TRY(cudaGraphLaunch(p->gbp[b], p->sc));
      HR_CUDA_TRY(cudaEventRecord(p->computed[b], p->sc));
      // the slab's slices are a strided block of the z-fastest volume; copied out
      // on the output stream while the next slab computes
      const size_t ld = (size_t)G.ZN * 4;
      HR_CUDA_TRY(cudaStreamWaitEvent(p->sout, p->computed[b], 0));
      HR_CUDA_TRY(cudaMemcpy2DAsync(vol + L.first_slice[k], ld, p->d_vslab[b], (size_t)L.S * 4,
                                    (size_t)L.n_slices[k] * 4, (size_t)G.XN * G.YN,
                                    vol_on_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, p->sout));
      HR_CUDA_TRY(cudaEventRecord(p->drained[b], p->sout));
    }
    return HR_OK;
  };
  int st = enqueue();
  // whether or not everything was enqueued, no copy may still use the caller's buffers on return
  for (cudaStream_t s2 : {p->sout, p->sc, p->sf, p->scopy}) {
    const cudaError_t e = cudaStreamSynchronize(s2);
    if (e != cudaSuccess && st == HR_OK) st = hr::fail(HR_ERR_CUDA, "hr_slab_execute: %s", cudaGetErrorString(e));
  }
  HR_TRY(st);
  return hr_filter_tc_check(p->ftc);
}

extern "C" int hr_slab_execute(hr_slab_plan* p, float* vol, const float* fan, int vol_on_host, int fan_on_host) {
  return hr_slab_execute_range(p, vol, fan, 0, vol_on_host, fan_on_host);
}

extern "C" int hr_slab_fan_range(const hr_slab_plan* p, int* first_view, int* nviews, size_t* bytes_per_execute) {
  HR_REQUIRE(p != nullptr, "hr_slab_fan_range: NULL plan");
  if (first_view) *first_view = p->fan_first;
  if (nviews) *nviews = p->fan_count;
  if (bytes_per_execute) *bytes_per_execute = p->fan_bytes;
  return HR_OK;
}

extern "C" int hr_slab_describe(const hr_slab_plan* p, char* buf, int len) {
  HR_REQUIRE(p != nullptr, "hr_slab_describe: NULL plan");
  char bp[640];
  HR_TRY(hr::bp_fast_describe(p->fast[0], bp, sizeof(bp)));
  if (buf && len > 0) {
    char part[96] = "";
    if (p->nparts > 1)
      snprintf(part, sizeof(part), " (part %d of %d, %s: %d slabs)", p->part, p->nparts,
               p->assign == HR_SLAB_ROUND_ROBIN ? "round robin" : "blocks", (int)p->mine.size());
    snprintf(buf, (size_t)len, "%d slabs of %d slices%s; window %d views (fan %d); graphs %s; backprojection: %s",
             p->L.nslabs, p->L.S, part, p->L.Wbp, p->L.Wfan,
             p->gbp[0] ? "captured (filter under backprojection)" : "not yet", bp);
  }
  return HR_OK;
}

extern "C" size_t hr_slab_device_bytes(const hr_slab_plan* p) {
  if (!p) return 0;
  return p->bytes + hr::bp_fast_device_bytes(p->fast[0]) + hr::bp_fast_device_bytes(p->fast[1]) +
         hr_filter_tc_device_bytes(p->ftc);
}

extern "C" void hr_slab_plan_destroy(hr_slab_plan* p) { destroy(p); }
