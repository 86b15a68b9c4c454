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
// Fan windows are copied into ping-pong buffers on a second stream while the
// previous slab computes, and each slab's volume leaves its own ping-pong
// buffer on a third stream while the next slab computes; each slab's tables
// are built on the host in FP64 and uploaded in stream order before its graph
// launch.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "bp_fast.h"
#include "hr_internal.h"

struct hr_slab_plan {
  hr_recon_desc d;
  int S = 0, nslabs = 0, Wbp = 0, Wfan = 0, margin = 0, half = 0;
  std::vector<int> p_start, a0, first_slice, n_slices;
  hr_rebin_plan* rebin = nullptr;
  hr_filter_tc_plan* ftc = nullptr;
  hr::BpFast fast[2];
  hr::BpFastGeom gslab{};
  std::vector<double> w;
  float* d_fan[2] = {nullptr, nullptr};
  float* d_reb = nullptr;
  uint32_t* d_pairs = nullptr;
  float* d_vslab[2] = {nullptr, nullptr};
  cudaStream_t sc = nullptr, scopy = nullptr, sout = nullptr;
  cudaEvent_t copied[2] = {nullptr, nullptr}, consumed[2] = {nullptr, nullptr};
  cudaEvent_t computed[2] = {nullptr, nullptr}, drained[2] = {nullptr, nullptr};
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  size_t bytes = 0;
};

namespace {

int s0_of(const hr_bp_geom& g, int zi) {
  const double z = (zi - g.ZNC) * g.dz;
  const double beta0 = 2.0 * 3.14159265358979 * z / g.h;
  return (int)std::ceil((beta0 - g.BetaS) / g.DeltaFai - 0.5);
}

void destroy(hr_slab_plan* p) {
  if (!p) return;
  for (int i = 0; i < 2; ++i) {
    if (p->graph[i]) cudaGraphExecDestroy(p->graph[i]);
    hr::bp_fast_destroy(&p->fast[i]);
    cudaFree(p->d_fan[i]);
    cudaFree(p->d_vslab[i]);
    if (p->copied[i]) cudaEventDestroy(p->copied[i]);
    if (p->consumed[i]) cudaEventDestroy(p->consumed[i]);
    if (p->computed[i]) cudaEventDestroy(p->computed[i]);
    if (p->drained[i]) cudaEventDestroy(p->drained[i]);
  }
  hr_rebin_plan_destroy(p->rebin);
  hr_filter_tc_plan_destroy(p->ftc);
  cudaFree(p->d_reb);
  cudaFree(p->d_pairs);
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
  g.ZNC = G.ZNC - p->first_slice[k];
  g.BetaS = G.BetaS + p->p_start[k] * G.DeltaFai;
  g.ZN_valid = p->n_slices[k];
  return g;
}

int enqueue_fan_copy(hr_slab_plan* p, int k, const float* fan, bool fan_on_host) {
  const int b = k & 1;
  const size_t per_view = (size_t)p->d.YL * p->d.ZL;
  HR_CUDA_TRY(cudaStreamWaitEvent(p->scopy, p->consumed[b], 0));
  HR_CUDA_TRY(cudaMemcpyAsync(p->d_fan[b], fan + (size_t)p->a0[k] * per_view, (size_t)p->Wfan * per_view * 4,
                              fan_on_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, p->scopy));
  HR_CUDA_TRY(cudaEventRecord(p->copied[b], p->scopy));
  return HR_OK;
}

// The three stages of one slab on stream s reading fan buffer b (what the
// graphs capture).
int slab_kernels(hr_slab_plan* p, int b, cudaStream_t s) {
  HR_TRY(hr_rebin_execute(p->rebin, p->d_reb, p->d_fan[b], s));
  HR_TRY(hr_filter_tc_execute(p->ftc, p->d_pairs, p->d_reb, HR_LAYOUT_REBIN, p->margin, s));
  return hr::bp_fast_execute(p->fast[b], p->gslab, p->d_vslab[b], p->d_pairs, s);
}

}  // namespace

extern "C" int hr_slab_plan_create(hr_slab_plan** plan, const hr_recon_desc* d, int slab_slices) {
  hr::clear_error();
  HR_REQUIRE(plan != nullptr && d != nullptr && d->w != nullptr, "hr_slab_plan_create: NULL argument");
  *plan = nullptr;
  HR_REQUIRE(d->form == HR_FORM_FAST, "hr_slab_plan_create: the slab pipeline runs the fast form");
  HR_REQUIRE(slab_slices > 0 && slab_slices <= 4096, "hr_slab_plan_create: slab of %d slices", slab_slices);
  HR_REQUIRE(d->DeltaTheta == d->DeltaFai,
             "hr_slab_plan_create: windowed rebinning needs DeltaTheta == DeltaFai (as the reference driver passes)");
  HR_REQUIRE(d->bp.YL == d->YL && d->bp.ZL == d->ZL, "hr_slab_plan_create: bp.YL/ZL differ from YL/ZL");
  HR_REQUIRE(d->view0 >= 0 && d->view0 + d->bp.PN + d->view0 <= d->ViewN,
             "hr_slab_plan_create: the crop must be symmetric (views [view0, view0+PN) plus view0 behind)");
  HR_TRY(hr::require_device());
  hr_slab_plan* p = new hr_slab_plan;
  p->d = *d;
  p->d.w = nullptr;
  p->w.assign(d->w, d->w + d->bp.N_2pi);
  const hr_bp_geom& G = d->bp;
  p->S = std::min(slab_slices, G.ZN);
  p->nslabs = (G.ZN + p->S - 1) / p->S;
  p->margin = d->view0;
  p->half = (int)std::ceil(G.N_pi * G.HSCoef);
  // per-slab windows
  int wmax = 1;
  std::vector<int> lo(p->nslabs), hi(p->nslabs);
  for (int k = 0; k < p->nslabs; ++k) {
    const int z0 = k * p->S, z1 = std::min(G.ZN, z0 + p->S) - 1;
    const int sa = s0_of(G, z0), sb = s0_of(G, z1);
    lo[k] = std::max(0, std::min(sa, sb) - p->half);
    hi[k] = std::min(G.PN - 1, std::max(sa, sb) + p->half);
    if (hi[k] >= lo[k]) wmax = std::max(wmax, hi[k] - lo[k] + 1);
    p->first_slice.push_back(z0);
    p->n_slices.push_back(z1 - z0 + 1);
  }
  p->Wbp = std::min(wmax, G.PN);
  p->Wfan = p->Wbp + 2 * p->margin;
  for (int k = 0; k < p->nslabs; ++k) {
    const int ps = std::max(0, std::min(lo[k], G.PN - p->Wbp));
    p->p_start.push_back(ps);
    p->a0.push_back(d->view0 + ps - p->margin);  // >= 0, and a0 + Wfan <= ViewN
  }
  // geometry template of a slab (the per-slab parts are set by slab_geom)
  hr::BpFastGeom& g = p->gslab;
  g.XN = G.XN; g.YN = G.YN; g.ZN = p->S; g.YL = G.YL; g.ZL = G.ZL; g.PN = p->Wbp; g.half = p->half;
  g.ZN_valid = p->S;
  g.XNC = G.XNC; g.YNC = G.YNC; g.ZNC = G.ZNC; g.dx = G.dx; g.dy = G.dy; g.dz = G.dz;
  g.YLC = G.YLC; g.ZLC = G.ZLC; g.dYL = G.dYL; g.dZL = G.dZL; g.h = G.h; g.BetaS = G.BetaS;
  g.DeltaFai = G.DeltaFai; g.N_pi = G.N_pi; g.SO = G.SO; g.SD = G.SD; g.k1 = G.k1;

  int st = hr_rebin_plan_create(&p->rebin, d->YL, d->ZL, p->Wfan, d->YLC, d->dYA, d->DeltaTheta, d->PLC, d->DeltaT,
                                d->DeltaFai, d->SO);
  if (st == HR_OK)
    st = hr_filter_tc_plan_create(&p->ftc, d->YL, d->ZL, p->Wbp, d->fPLC, d->fZLC, d->fdYL, d->fdZL, d->fSO);
  // table capacity: the largest tables over all slabs
  size_t rows[hr::kFastTableSets] = {0};
  int nb[hr::kFastTableSets] = {0};
  for (int k = 0; k < p->nslabs && st == HR_OK; ++k) {
    hr::BpFastHost h;
    st = hr::bp_fast_host_tables(&h, slab_geom(p, k), p->w.data());
    for (int i = 0; i < hr::kFastTableSets && st == HR_OK; ++i) {
      rows[i] = std::max(rows[i], h.set[i].mask.size());
      nb[i] = h.set[i].nblocks;
    }
  }
  for (int b = 0; b < 2 && st == HR_OK; ++b) st = hr::bp_fast_reserve(&p->fast[b], rows, nb, p->Wbp);
  const size_t per_view = (size_t)d->YL * d->ZL;
  for (int b = 0; b < 2 && st == HR_OK; ++b) st = alloc(p, (void**)&p->d_fan[b], (size_t)p->Wfan * per_view * 4);
  if (st == HR_OK) st = alloc(p, (void**)&p->d_reb, (size_t)p->Wfan * per_view * 4);
  if (st == HR_OK) st = alloc(p, (void**)&p->d_pairs, (size_t)p->Wbp * per_view * 4);
  for (int b = 0; b < 2 && st == HR_OK; ++b) st = alloc(p, (void**)&p->d_vslab[b], (size_t)G.XN * G.YN * p->S * 4);
  if (st == HR_OK) {
    cudaError_t e = cudaStreamCreateWithFlags(&p->sc, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->scopy, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->sout, cudaStreamNonBlocking);
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
      e = cudaEventCreateWithFlags(&p->copied[b], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->consumed[b], cudaEventDisableTiming);
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

// Picks the backprojection variant on the middle slab's real data and
// captures the two per-parity graphs. Runs once, on the first execution.
static int prepare(hr_slab_plan* p, const float* fan, bool fan_on_host) {
  const int k = p->nslabs / 2;
  HR_TRY(enqueue_fan_copy(p, k, fan, fan_on_host));
  HR_CUDA_TRY(cudaStreamWaitEvent(p->sc, p->copied[k & 1], 0));
  hr::BpFastHost h;
  HR_TRY(hr::bp_fast_host_tables(&h, slab_geom(p, k), p->w.data()));
  HR_TRY(hr::bp_fast_upload(&p->fast[k & 1], h, p->sc));
  HR_TRY(hr_rebin_execute(p->rebin, p->d_reb, p->d_fan[k & 1], p->sc));
  HR_TRY(hr_filter_tc_execute(p->ftc, p->d_pairs, p->d_reb, HR_LAYOUT_REBIN, p->margin, p->sc));
  HR_TRY(hr::bp_fast_autotune(&p->fast[k & 1], p->gslab, p->d_vslab[k & 1], p->d_pairs, p->sc));
  p->fast[(k & 1) ^ 1].variant = p->fast[k & 1].variant;
  p->fast[(k & 1) ^ 1].tuned = p->fast[k & 1].tuned;
  HR_TRY(hr::bp_fast_tex_prepare(&p->fast[(k & 1) ^ 1], p->gslab));
  HR_CUDA_TRY(cudaStreamSynchronize(p->sc));
  for (int b = 0; b < 2; ++b) {
    cudaGraph_t gr = nullptr;
    HR_CUDA_TRY(cudaStreamBeginCapture(p->sc, cudaStreamCaptureModeRelaxed));
    const int st = slab_kernels(p, b, p->sc);
    const cudaError_t e = cudaStreamEndCapture(p->sc, &gr);
    if (st != HR_OK) {
      if (gr) cudaGraphDestroy(gr);
      return st;
    }
    HR_CUDA_TRY(e);
    const cudaError_t ei = cudaGraphInstantiate(&p->graph[b], gr, 0);
    cudaGraphDestroy(gr);
    HR_CUDA_TRY(ei);
  }
  if (hr::log_enabled()) {
    char desc[768];
    if (hr_slab_describe(p, desc, sizeof(desc)) == HR_OK) hr::log("slab plan prepared: %s", desc);
  }
  return HR_OK;
}

extern "C" int hr_slab_execute(hr_slab_plan* p, float* vol, const float* fan, int vol_on_host, int fan_on_host) {
  hr::clear_error();
  HR_REQUIRE(p != nullptr && vol != nullptr && fan != nullptr, "hr_slab_execute: NULL argument");
  if (!p->graph[0]) HR_TRY(prepare(p, fan, fan_on_host != 0));
  const hr_bp_geom& G = p->d.bp;
  HR_TRY(enqueue_fan_copy(p, 0, fan, fan_on_host != 0));
  for (int k = 0; k < p->nslabs; ++k) {
    const int b = k & 1;
    // tables of slab k: host build (overlaps the previous slab on the GPU), stream-ordered upload
    hr::BpFastHost h;
    HR_TRY(hr::bp_fast_host_tables(&h, slab_geom(p, k), p->w.data()));
    HR_CUDA_TRY(cudaStreamWaitEvent(p->sc, p->copied[b], 0));
    HR_CUDA_TRY(cudaStreamWaitEvent(p->sc, p->drained[b], 0));  // slab k-2's volume has left d_vslab[b]
    HR_TRY(hr::bp_fast_upload(&p->fast[b], h, p->sc));
    HR_CUDA_TRY(cudaGraphLaunch(p->graph[b], p->sc));
    HR_CUDA_TRY(cudaEventRecord(p->consumed[b], p->sc));
    HR_CUDA_TRY(cudaEventRecord(p->computed[b], p->sc));
    if (k + 1 < p->nslabs) HR_TRY(enqueue_fan_copy(p, k + 1, fan, fan_on_host != 0));
    // the slab's slices are a strided block of the z-fastest volume; copied out
    // on the output stream while the next slab computes
    const size_t ld = (size_t)G.ZN * 4;
    HR_CUDA_TRY(cudaStreamWaitEvent(p->sout, p->computed[b], 0));
    HR_CUDA_TRY(cudaMemcpy2DAsync(vol + p->first_slice[k], ld, p->d_vslab[b], (size_t)p->S * 4,
                                  (size_t)p->n_slices[k] * 4, (size_t)G.XN * G.YN,
                                  vol_on_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, p->sout));
    HR_CUDA_TRY(cudaEventRecord(p->drained[b], p->sout));
  }
  HR_CUDA_TRY(cudaStreamSynchronize(p->sout));
  HR_CUDA_TRY(cudaStreamSynchronize(p->sc));
  return hr_filter_tc_check(p->ftc);
}

extern "C" int hr_slab_describe(const hr_slab_plan* p, char* buf, int len) {
  HR_REQUIRE(p != nullptr, "hr_slab_describe: NULL plan");
  char bp[384];
  HR_TRY(hr::bp_fast_describe(p->fast[0], bp, sizeof(bp)));
  if (buf && len > 0)
    snprintf(buf, (size_t)len, "%d slabs of %d slices; window %d views (fan %d); graphs %s; backprojection: %s",
             p->nslabs, p->S, p->Wbp, p->Wfan, p->graph[0] ? "captured" : "not yet", bp);
  return HR_OK;
}

extern "C" size_t hr_slab_device_bytes(const hr_slab_plan* p) {
  if (!p) return 0;
  return p->bytes + hr::bp_fast_device_bytes(p->fast[0]) + hr::bp_fast_device_bytes(p->fast[1]) +
         hr_filter_tc_device_bytes(p->ftc);
}

extern "C" void hr_slab_plan_destroy(hr_slab_plan* p) { destroy(p); }
