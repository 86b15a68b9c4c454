/*
 * helixrecon.h -- C ABI of the B200-native helical cone-beam FBP chain
 * (curved-detector fan->parallel rebinning, cosine preweight + ramp filter,
 * 3D-weighted helical FDK backprojection).
 *
 * Two layers:
 *
 * 1. Drop-in entry points with the exact names, argument lists and array
 *    layouts of the reference's extern "C" functions. They take HOST
 *    pointers, are synchronous, allocate their own device memory per call and
 *    return void, as the reference's do. They run on the calling thread's
 *    current CUDA device (device 0 in a fresh process, which is what the
 *    reference hard-codes). Failures are reported through hr_last_error()
 *    and, unlike the reference, never silently: the output is left untouched
 *    and an error message is printed to stderr.
 *
 * 2. hr_* entry points that return an hr_status: host-pointer twins of the
 *    drop-ins, and plan-based device-pointer entries that take a CUDA stream
 *    (passed as void*), allocate nothing at execute time and can be captured
 *    into CUDA graphs.
 *
 * Layouts (C order, last index fastest):
 *   fan / rebinned projections  [ViewN][YL][ZL]   (MATLAB [ZL,YL,ViewN])
 *   filter input / output       [ViewN][ZL][YL]   (MATLAB [YL,ZL,ViewN])
 *   volume                      [YN][XN][ZN]      (MATLAB [ZN,XN,YN])
 */
#ifndef HELIXRECON_H
#define HELIXRECON_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ======================================================================== */
/* 1. Reference drop-ins                                                    */
/* ======================================================================== */

/* Replaces src/ParallelRebinningCBCurve.h:4-8 / src/ParallelRebinningCBCurveGPU.cu:106-115.
 * Fan -> parallel rebinning; YLC and PLC 0-based. Clamp rule of the reference's
 * CPU path (src/ParallelRebinningCBCurve.cpp:55-85); result bit-identical to it. */
void ParallelRebinningCBCurve_GPU(float* outputProj, const float* Proj, const int YL, const int ZL, const int ViewN,
                                  const float YLC, const float dYA, const float DeltaTheta, const float PLC,
                                  const float DeltaT, const float DeltaFai, const float SO);

/* Replaces src/filtering.h:12-18 / src/filtering.cu:270-287. Cosine preweight and
 * Shepp-Logan ramp filter of every detector row, cuFFT-free (own radix-4 FFT). */
void filtering(float* hfpwd, const float* hProj, const int YL, const int ZL, const int ViewN, const float PLC,
               const float ZLC, const float dYL, const float dZL, const float SO);

/* Replaces src/ParallelFDKHelical3DWeightingGPU.h:4-13 / ...GPU.cu:125-140.
 * FP64 data path on the GPU; views s1..s2 as the reference's CPU loop. */
void ParallekFDKHelical3DWeighting_GPU_double(
    double* hctimage, const double* hfp, const double* hw, const int N_2pi, const int XN, const int YN,
    const int ZN, const double XNC, const double YNC, const double ZNC, const double dx, const double dy,
    const double dz, const int YL, const int ZL, const int PN, const double YLC, const double ZLC,
    const double dYL, const double dZL, const double h, const double BetaS, const double DeltaFai,
    const double N_pi, const double HSCoef, const double SO, const double SD, const double k1);

/* Replaces src/ParallelFDKHelical3DWeightingGPU.h:15-24 / ...GPU.cu:144-159.
 * FP32 data path; view/row/channel index selection computed in FP64 with the
 * reference CPU's expression order, so it is bit-exact to that path. */
void ParallekFDKHelical3DWeighting_GPU_float(
    float* hctimage, const float* hfp, const float* hw, const int N_2pi, const int XN, const int YN, const int ZN,
    const float XNC, const float YNC, const float ZNC, const float dx, const float dy, const float dz,
    const int YL, const int ZL, const int PN, const float YLC, const float ZLC, const float dYL, const float dZL,
    const float h, const float BetaS, const float DeltaFai, const float N_pi, const float HSCoef, const float SO,
    const float SD, const float k1);

/* Replaces src/Parallel_FDK_Helical_3DWeighting.cpp:117-200. Derives dx,dy,dz,
 * dYL,dZL,DeltaFai and the view weight w as the reference does. useGPU == 1
 * runs the FP32 data path (as the reference's GPU branch); any other value
 * runs the FP64 data path on the GPU (the reference's CPU branch semantics). */
void ParallelFDKHelical3DWeighting(double* ctimage, const double* fp, const double SO, const double DO,
                                   const int YL, const int ZL, const double DecWidth, const double DecHeigh,
                                   const double YLC, const double ZLC, const double h, const double BetaS,
                                   const int PN, const int N_2pi, const double ObjR, const int XN, const int YN,
                                   const int ZN, const double XNC, const double YNC, const double ZNC,
                                   const int delta, const double HSCoef, const double k1, const int useGPU);

/* ======================================================================== */
/* 2. Status-returning API                                                  */
/* ======================================================================== */

typedef enum hr_status {
  HR_OK = 0,
  HR_ERR_INVALID_ARGUMENT = 1,
  HR_ERR_CUDA = 2,
  HR_ERR_OUT_OF_MEMORY = 3,
  HR_ERR_NO_DEVICE = 4,
  HR_ERR_UNSUPPORTED = 5
} hr_status;

/* Precision forms of the chain. */
typedef enum hr_form {
  HR_FORM_PLAIN = 0, /* FP32 data, FFT filter, FP64 exact index selection (the drop-in) */
  HR_FORM_FP64 = 1,  /* FP64 data path */
  HR_FORM_FAST = 2   /* BF16 split Toeplitz filter on tcgen05, BF16 filtered data, fast BP */
} hr_form;

/* Message of the last failure on the calling thread ("" if none). */
const char* hr_last_error(void);
/* Library version (major*10000 + minor*100 + patch). */
int hr_version(void);

/* Host-pointer twins of the drop-ins. Same arguments; return an hr_status. */
int hr_rebin_host(float* outputProj, const float* Proj, int YL, int ZL, int ViewN, float YLC, float dYA,
                  float DeltaTheta, float PLC, float DeltaT, float DeltaFai, float SO);
int hr_filter_host(float* hfpwd, const float* hProj, int YL, int ZL, int ViewN, float PLC, float ZLC, float dYL,
                   float dZL, float SO);
int hr_bp_host_float(float* hctimage, const float* hfp, const float* hw, int N_2pi, int XN, int YN, int ZN,
                     float XNC, float YNC, float ZNC, float dx, float dy, float dz, int YL, int ZL, int PN,
                     float YLC, float ZLC, float dYL, float dZL, float h, float BetaS, float DeltaFai, float N_pi,
                     float HSCoef, float SO, float SD, float k1);
int hr_bp_host_double(double* hctimage, const double* hfp, const double* hw, int N_2pi, int XN, int YN, int ZN,
                      double XNC, double YNC, double ZNC, double dx, double dy, double dz, int YL, int ZL, int PN,
                      double YLC, double ZLC, double dYL, double dZL, double h, double BetaS, double DeltaFai,
                      double N_pi, double HSCoef, double SO, double SD, double k1);
/* Status twin of ParallelFDKHelical3DWeighting (same arguments). */
int hr_bp_host_reference(double* ctimage, const double* fp, double SO, double DO, int YL, int ZL, double DecWidth,
                         double DecHeigh, double YLC, double ZLC, double h, double BetaS, int PN, int N_2pi,
                         double ObjR, int XN, int YN, int ZN, double XNC, double YNC, double ZNC, int delta,
                         double HSCoef, double k1, int useGPU);

/* View weight table w[N_2pi] of src/Parallel_FDK_Helical_3DWeighting.cpp:156-170
 * (cos^2 tapers of `delta` views at both ends of a 2 ceil(N_pi HSCoef)+1 window). */
int hr_view_weights(double* w, int N_2pi, double HSCoef, int delta);

/* ---- rebinning plan ----------------------------------------------------- */
typedef struct hr_rebin_plan hr_rebin_plan;
int hr_rebin_plan_create(hr_rebin_plan** plan, int YL, int ZL, int ViewN, float YLC, float dYA, float DeltaTheta,
                         float PLC, float DeltaT, float DeltaFai, float SO);
/* d_out, d_proj: device [ViewN][YL][ZL]. */
int hr_rebin_execute(const hr_rebin_plan* plan, float* d_out, const float* d_proj, void* stream);
void hr_rebin_plan_destroy(hr_rebin_plan* plan);
/* Host only (no device needed): the fan views [*f0, *f1] that the rebinning of
 * output views [i0, i1) reads (its bilinear taps over every channel, clamped to
 * the scan, with a view or two of slack), for callers that stream the fan data
 * in by ranges of views, as hr_recon_execute_host does. Same arguments as the
 * rebinning (YLC, PLC 0-based). */
int hr_rebin_fan_views(int YL, int ViewN, float YLC, float dYA, float DeltaTheta, float PLC, float DeltaT,
                       float DeltaFai, float SO, int i0, int i1, int* f0, int* f1);

/* ---- filter plan -------------------------------------------------------- */
typedef struct hr_filter_plan hr_filter_plan;
/* Input layouts for hr_filter_execute. */
#define HR_LAYOUT_ROWS 0   /* [views][ZL][YL] (YL fastest), the reference filter layout */
#define HR_LAYOUT_REBIN 1  /* [views][YL][ZL] (ZL fastest), the rebinning output */
int hr_filter_plan_create(hr_filter_plan** plan, int YL, int ZL, int ViewN, float PLC, float ZLC, float dYL,
                          float dZL, float SO);
/* Filters views [view0, view0+ViewN) of d_in (laid out as in_layout, holding
 * at least view0+ViewN views) into d_out [ViewN][ZL][YL]. d_in and d_out must
 * not overlap (HR_ERR_INVALID_ARGUMENT otherwise). */
int hr_filter_execute(const hr_filter_plan* plan, float* d_out, const float* d_in, int in_layout, int view0,
                      void* stream);
void hr_filter_plan_destroy(hr_filter_plan* plan);

/* ---- tensor-core filter plan (fast form) -------------------------------- */
/* Preweight + ramp filter as a split-BF16 Toeplitz matrix product on the
 * tcgen05 tensor cores (FP32 accumulation in TMEM); writes the fast
 * backprojection's BF16 channel pairs [ViewN][ZL][YL] (uint32). Needs an
 * sm_100 device. The plan holds the split operands (4 bytes per sample of
 * workspace plus the Toeplitz matrix). */
typedef struct hr_filter_tc_plan hr_filter_tc_plan;
int hr_filter_tc_plan_create(hr_filter_tc_plan** plan, int YL, int ZL, int ViewN, float PLC, float ZLC, float dYL,
                             float dZL, float SO);
int hr_filter_tc_execute(const hr_filter_tc_plan* plan, uint32_t* d_pairs, const float* d_in, int in_layout,
                         int view0, void* stream);
/* Reads and clears the plan's device error flag (synchronous): HR_ERR_CUDA if
 * a kernel pipeline wait timed out in an earlier execution. */
int hr_filter_tc_check(const hr_filter_tc_plan* plan);
/* Test hook, no counterpart in the reference: from the next execution on, the
 * TMA producer of every CTA leaves K block k_block unloaded (a barrier nothing
 * completes) and pipeline waits give up after wait_polls polls, so the
 * bounded-wait abort path runs: the kernel flags the error, lets the copies
 * it issued land, frees its tensor memory and returns without writing its
 * tile. k_block < 0 restores normal operation. */
int hr_filter_tc_test_stall(hr_filter_tc_plan* plan, int k_block, unsigned int wait_polls);
size_t hr_filter_tc_device_bytes(const hr_filter_tc_plan* plan);
void hr_filter_tc_plan_destroy(hr_filter_tc_plan* plan);

/* ---- backprojection plan ------------------------------------------------ */
typedef struct hr_bp_geom {
  int N_2pi, XN, YN, ZN, YL, ZL, PN;
  double XNC, YNC, ZNC, dx, dy, dz;
  double YLC, ZLC, dYL, dZL, h, BetaS, DeltaFai, N_pi, HSCoef, SO, SD, k1;
} hr_bp_geom;

typedef struct hr_bp_plan hr_bp_plan;
/* w: host view weight table of N_2pi entries (as the reference's hw). form:
 * HR_FORM_PLAIN (fp float), HR_FORM_FP64 (fp double), HR_FORM_FAST (fp BF16
 * channel pairs, see hr_pack_bf16_pairs). */
int hr_bp_plan_create(hr_bp_plan** plan, const hr_bp_geom* g, const double* w, int form);
/* d_fp: device [PN][ZL][YL] (float; double for HR_FORM_FP64; uint32 BF16 pairs
 * for HR_FORM_FAST); d_vol: device [YN][XN][ZN] (double for HR_FORM_FP64, else float). */
int hr_bp_execute(const hr_bp_plan* plan, void* d_vol, const void* d_fp, void* stream);
void hr_bp_plan_destroy(hr_bp_plan* plan);
/* HR_FORM_FAST: times the kernel variants (slices per thread x register
 * gathers or texture-sampled taps, see hr_bp_select) on a 32-slice band of
 * d_vol and keeps the fastest for the plan's later executions; a texture
 * variant keeps an FP16 (2 bytes per sample) or FP32 layered copy of the
 * filtered data in the plan, refilled by every hr_bp_execute, so two
 * executions of one such plan must not overlap on the GPU. Synchronises the
 * stream and may allocate; call before graph capture. Other forms: no-op. */
int hr_bp_autotune(hr_bp_plan* plan, void* d_vol, const void* d_fp, void* stream);
/* Writes a one-line description of the kernel configuration into buf. */
int hr_bp_describe(const hr_bp_plan* plan, char* buf, int len);
/* Selects a fast-form kernel variant by index (the autotuner's candidates:
 * 0-2 sixteen slices per thread, 3-5 eight, gathers issued one, four or eight
 * slices at a time; 6-7 sixteen / eight slices per thread in packed FP32x2
 * slice pairs; 8-10 four slices per thread, per slice / pairs / batched;
 * 11-13 eight / sixteen / four slices per thread sampling an FP16 layered
 * texture copy of the data with the texture units' bilinear filtering, 14-15
 * eight / sixteen with an FP32 copy, 16-17 eight / four slices per thread
 * from the FP16 copy with the view loop cut into segments of a fixed set of
 * slices holding the view (thick slices), 18-19 eight / four slices per
 * thread as 16-17 with two views per iteration in segments of at most four
 * slices (thick slices: more taps in flight), 20 as 16 and 21 as 19 with
 * registers bounded for 6 CTAs per SM; the texture variants allocate the
 * copy, 2 or 4 bytes per sample, and fill it on every execution).
 * For tests and manual tuning. */
int hr_bp_select(hr_bp_plan* plan, int variant);

/* ---- backprojection that allocates nothing ------------------------------ */
/* No counterpart in the reference. For callers that cannot call cudaMalloc:
 * streaming pipelines that must not allocate once running (cudaMalloc and
 * cudaFree synchronise the whole device), hosts whose pooling allocator owns
 * all device memory (a MATLAB session, a framework's caching allocator), and
 * services held to a fixed device-memory budget. Same result, bit for bit, as
 * a HR_FORM_PLAIN plan: d_vol [YN][XN][ZN] float, d_fp [PN][ZL][YL] float,
 * d_w the N_2pi view weights as float on the device; the geometry checks are
 * the plan's. Its per-view table is computed on the host with the plan's C
 * library calls and copied (from pageable memory, so the call first waits for
 * the stream's earlier work) into a fixed 768 KiB device array inside the
 * library: PN is limited to 32768 views (HR_ERR_INVALID_ARGUMENT beyond). The
 * first call on a device looks up that array's address (cudaGetSymbolAddress).
 * All calls share the array and it keeps the last call's table: calls that
 * overlap on the GPU (other streams, other threads) race. */
int hr_bp_plain_noalloc(float* d_vol, const float* d_fp, const float* d_w, const hr_bp_geom* g, void* stream);

/* ---- BF16 channel pairs (the fast form's filtered-data layout) ---------- */
/* d_out[r][u] = bf16(d_in[r][u]) | bf16(d_in[r][u+1]) << 16 (round to nearest
 * even; channel YL pairs with 0), for rows r in [0, rows). The fast form's
 * backprojection plan reads this layout. */
int hr_pack_bf16_pairs(uint32_t* d_out, const float* d_in, long long rows, int YL, void* stream);

/* ---- whole chain: rebin -> crop -> preweight/filter -> backprojection ---- */
/* The per-scan driver of src/analyticalReconBigPatient.m:77-146 as one plan. */
typedef struct hr_recon_desc {
  /* rebinning: the arguments of ParallelRebinningCBCurve_GPU (YLC, PLC 0-based) */
  int YL, ZL, ViewN;
  float YLC, dYA, DeltaTheta, PLC, DeltaT, DeltaFai, SO;
  /* rebinned views [view0, view0 + bp.PN) are filtered and backprojected (the
   * segment-overlap crop of the m-file :80-93) */
  int view0;
  /* filter: the arguments of `filtering` (PLC, ZLC 0-based) */
  float fPLC, fZLC, fdYL, fdZL, fSO;
  /* backprojection geometry; bp.YL/ZL must equal YL/ZL */
  hr_bp_geom bp;
  const double* w; /* N_2pi view weights, copied at plan creation */
  int form;        /* hr_form */
} hr_recon_desc;

typedef struct hr_recon_plan hr_recon_plan;
int hr_recon_plan_create(hr_recon_plan** plan, const hr_recon_desc* desc);
/* Device pointers: d_fan [ViewN][YL][ZL] float, d_vol [YN][XN][ZN] float. */
int hr_recon_execute(const hr_recon_plan* plan, float* d_vol, const float* d_fan, void* stream);
/* Host pointers (pinned for full copy speed): copies the fan data in, runs the
 * chain, copies the volume out; returns when h_vol is written. Either pointer
 * may also be device memory (the copies take their direction from the
 * addresses: a host fan into a device volume, for instance). The fast form
 * streams: the fan crosses the host link in chunks of 1024 views
 * (HELIXRECON_STREAM_CHUNK at plan creation; 0: no streaming) while the chunks
 * that have arrived are rebinned and filtered, z-block ranges are
 * backprojected as soon as their view windows are filtered, and each range's
 * slices are copied out while later ranges compute. Rebinning and filtering
 * give the device entry's bits; a texture variant's FP16 copy is filled chunk
 * by chunk with a scale from the first chunk (2^4 of headroom), so its volume
 * equals the device entry's to FP32 rounding, and is refilled whole (the
 * device entry's bits) when a later chunk exceeds that scale. */
int hr_recon_execute_host(hr_recon_plan* plan, float* h_vol, const float* h_fan);
/* Host only (no device needed): the backprojection ranges of the streamed host
 * execution for a scan, with nz slices per z block (the chosen variant's: 16,
 * 8 or 4) and chunks of `chunk` parallel views: *n ranges, written to out as
 * {first z block, end z block, chunk after whose filtering the range may run}
 * (out may be NULL to count them; cap: triples out holds). Zero ranges: the
 * scan's view windows do not complete in z order, and the host execution runs
 * the chain unstreamed. */
int hr_recon_stream_schedule(const hr_recon_desc* desc, int nz, int chunk, int* out, int cap, int* n);
/* One-line description of the plan's kernel configuration (the fast form's
 * backprojection is autotuned at plan creation). */
int hr_recon_describe(const hr_recon_plan* plan, char* buf, int len);
/* Synchronous health check of the plan's kernels (tensor-core filter flag). */
int hr_recon_check(const hr_recon_plan* plan);
/* Device bytes the plan holds (tables + intermediate + host-staging buffers). */
size_t hr_recon_device_bytes(const hr_recon_plan* plan);
void hr_recon_plan_destroy(hr_recon_plan* plan);

/* ---- slab-batched long scans (big patients) ------------------------------ */
/* Replaces the segment loop of src/analyticalRecon.m:15-25 (segments of views,
 * each reconstructed into the whole volume and summed) by disjoint z slabs:
 * each slab of slab_slices slices is reconstructed from only its own view
 * window (plus the half-fan margin) through one captured CUDA graph (rebin ->
 * tensor-core filter -> fast backprojection, autotuned on the first call);
 * fan windows stream in on a second stream while the previous slab computes.
 * desc: the whole scan (form HR_FORM_FAST; the crop view0 must be the same at
 * both ends, as the geometry helpers make it). */
typedef struct hr_slab_plan hr_slab_plan;
int hr_slab_plan_create(hr_slab_plan** plan, const hr_recon_desc* desc, int slab_slices);
/* fan [ViewN][YL][ZL], vol [YN][XN][ZN]; each on the host (pinned for overlap)
 * or the device as the flags say. Synchronous. Consecutive slabs' fan windows
 * overlap; the shared views are copied on the device from the previous
 * window, so each fan view crosses the host link once. */
int hr_slab_execute(hr_slab_plan* plan, float* vol, const float* fan, int vol_on_host, int fan_on_host);
int hr_slab_describe(const hr_slab_plan* plan, char* buf, int len);
size_t hr_slab_device_bytes(const hr_slab_plan* plan);
void hr_slab_plan_destroy(hr_slab_plan* plan);

/* One scan on several GPUs: z slabs split between parts (one plan per GPU,
 * part p of nparts), each part rebinning, filtering and backprojecting only
 * its own slabs from its own fan windows and writing only their slices of the
 * volume. No data cross between parts: windows of neighbouring parts overlap
 * and the overlap is recomputed, which is cheaper than exchanging it. This
 * replaces the reference's only way to split a long scan, the sequential
 * segment loop (src/analyticalRecon.m:20-25), whose segments each need a
 * volume-sized sum. */
#define HR_SLAB_BLOCKS 0      /* part p takes a contiguous block of slabs (its fan views are one range) */
#define HR_SLAB_ROUND_ROBIN 1 /* part p takes slabs p, p + nparts, ... */
typedef struct hr_slab_window {
  int slab;          /* slab index k: slices [k S, k S + n_slices) */
  int first_slice, n_slices;
  int bp_view0;      /* first backprojected view (cropped, rebinned numbering) */
  int bp_views;      /* backprojection window length (the same for every slab) */
  int fan_view0;     /* first fan view of the slab's window (view0 + bp_view0 - margin) */
  int fan_views;     /* fan window length: bp_views + 2 margin (view0 of the desc) */
  int shared_views;  /* leading fan views shared with the part's previous slab (0 for its first) */
} hr_slab_window;
/* The slab windows of part `part` of `nparts` (host arithmetic only, needs no
 * GPU): *n = the part's slab count; out (cap entries, or NULL to query *n).
 * The same arithmetic as hr_slab_plan_create_part. */
int hr_slab_windows(const hr_recon_desc* desc, int slab_slices, int part, int nparts, int assign,
                    hr_slab_window* out, int cap, int* n);
/* Plan for part `part` of `nparts` (assign: HR_SLAB_BLOCKS or
 * HR_SLAB_ROUND_ROBIN; nparts <= number of slabs). hr_slab_plan_create is
 * part 0 of 1. */
int hr_slab_plan_create_part(hr_slab_plan** plan, const hr_recon_desc* desc, int slab_slices, int part, int nparts,
                             int assign);
/* As hr_slab_execute, with fan holding views [fan_view0, ...) of the scan
 * only (at least the range hr_slab_fan_range reports): a part needs only its
 * own views in memory. */
int hr_slab_execute_range(hr_slab_plan* plan, float* vol, const float* fan, int fan_view0, int vol_on_host,
                          int fan_on_host);
/* Fan views the plan reads, [first_view, first_view + nviews), and the bytes
 * one execution copies from the caller's fan (overlaps counted once). */
int hr_slab_fan_range(const hr_slab_plan* plan, int* first_view, int* nviews, size_t* bytes_per_execute);

/* ---- several scans of uneven size in one persistent launch --------------- */
/* n (1..16) independent scans, each described as for hr_recon_plan_create
 * (form HR_FORM_FAST): every scan's rebinning and tensor-core filter run one
 * after the other through shared scratch, then ONE persistent backprojection
 * launch covers all scans' (z block, column tile) work items. The sequence is
 * captured into a CUDA graph per set of buffer addresses and replayed. At
 * creation each scan's slices per thread are autotuned, then the batch kernel
 * variant on the whole batch (HELIXRECON_BATCH_VARIANT pins the latter). */
typedef struct hr_batch_plan hr_batch_plan;
int hr_batch_plan_create(hr_batch_plan** plan, const hr_recon_desc* descs, int n);
/* d_vols[i]: device [YN][XN][ZN] of scan i; d_fans[i]: device [ViewN][YL][ZL]. */
int hr_batch_execute(hr_batch_plan* plan, float* const* d_vols, const float* const* d_fans, void* stream);
/* The same batch from host memory, synchronous: h_fans[i] host [ViewN][YL][ZL],
 * h_vols[i] host [YN][XN][ZN]. The fans stream in through two device staging
 * buffers on a copy stream while earlier scans rebin, filter and backproject
 * (smallest scan first, then the largest ones); with per-scan backprojection
 * launches (variant 11) each volume is copied out as soon as its scan is done,
 * otherwise all after the persistent launch. Copies from page-locked host
 * memory overlap the computation; from pageable memory they are synchronous.
 * The staging buffers (2 x the largest fan) and the volumes are allocated at
 * the first call and kept with the plan. Not to be run concurrently with
 * another call on the same plan. */
int hr_batch_execute_host(hr_batch_plan* plan, float* const* h_vols, const float* const* h_fans);
/* Only the persistent backprojection launch, from the filtered data the last
 * hr_batch_execute left in the plan (not captured; for timing the kernel). */
int hr_batch_backproject(hr_batch_plan* plan, float* const* d_vols, void* stream);
/* Selects a batch backprojection variant (0..5: registers unconstrained, or
 * limited for 5 or 6 CTAs of 256 threads per SM; gathers per slice (0..2) or in
 * chunks of 4 slices (3..5); 6..10: taps sampled from each scan's FP16 layered
 * texture copy, with each scan's own slices per thread and registers
 * unconstrained or limited for 4 CTAs per SM (6, 7), or 4 slices per thread
 * for every scan and registers limited for 4, 5 or 6 CTAs per SM (8..10));
 * 11: no persistent launch, every scan's own plan kernel on a stream of its
 * own, forked after the scan's filter (under the next scans' rebinning and
 * filtering) and joined at the end; 12..14: one persistent launch with FP16
 * texture taps whose column code is specialised per scan (each scan's
 * constants read at a fixed descriptor index), each scan's own slices per
 * thread (12) or 4 for every scan, registers unconstrained (13) or limited
 * for 5 CTAs per SM (14); 15..16: one persistent launch running the
 * segmented view loop of the single-scan variants 16-17 with each scan's own
 * slices per thread, registers unconstrained (15) or limited for 4 CTAs per
 * SM (16). The gather variants keep the slices per thread each
 * scan's own autotuner chose. Switching variants allocates or frees the
 * scans' texture copies. */
int hr_batch_select(hr_batch_plan* plan, int variant);
int hr_batch_describe(const hr_batch_plan* plan, char* buf, int len);
int hr_batch_check(const hr_batch_plan* plan);
size_t hr_batch_device_bytes(const hr_batch_plan* plan);
void hr_batch_plan_destroy(hr_batch_plan* plan);

/* ---- analytic phantom projector (synthetic data source) ----------------- */
/* Objects: nobj rows of 17 doubles [type, cx, cy, cz, a, b, c, R(9, row-major,
 * columns = body axes), mu]; type 0 ellipsoid, type 1 elliptic cylinder (z in
 * cz +- c). Writes FP64 line integrals rounded to float into device
 * d_proj [ViewN][YL][ZL] for the fan geometry (source angle BetaS + i*dBeta,
 * fan angle (j - YLC0)*dYA, row rise (k - ZLC0)*dZL over SD, source height
 * h*angle/(2 pi)). d_obj: device copy of the object table. */
int hr_project_ellipsoids(float* d_proj, int YL, int ZL, int ViewN, double SO, double SD, double dYA, double YLC0,
                          double dZL, double ZLC0, double BetaS, double dBeta, double h, const double* d_obj,
                          int nobj, void* stream);

/* Photon noise of a transmission scan, in place: p -> -log(max(N, 1) / I0)
 * with N ~ Poisson(I0 exp(-p)) per sample (counter-based generator seeded by
 * `seed`; the result does not depend on the launch). */
int hr_add_poisson_noise(float* d_proj, long long n, double I0, unsigned long long seed, void* stream);

/* ---- learned artifact correction (2.5D residual CNN) -------------------- */
/* Corrects a half-view reconstruction toward the full-view one. Input: 5
 * adjacent slices (u = mu/mu_w - 1, NHWC BF16, channels padded to 16); 8 conv
 * layers 3x3 (16->32, 6 x 32->32 with ReLU, 32->16 of which channel 0 is the
 * residual); output = centre slice + mu_w * residual. Forward and backward
 * data passes run on the tensor cores (BF16 operands, FP32 accumulation),
 * weight gradients on the CUDA cores; Adam on FP32 master parameters.
 * Parameters: per layer W[co][tap][ci] (tap = 3*ky + kx) then b[co]. */
typedef struct hr_cnn hr_cnn;
size_t hr_cnn_param_count(void);
int hr_cnn_create(hr_cnn** net, const float* h_params);
int hr_cnn_get_params(const hr_cnn* net, float* h_params);
/* Gradients of the last hr_cnn_train_step. */
int hr_cnn_get_grads(const hr_cnn* net, float* h_grads);
/* Forward, loss = mean(((pred - target)/mu_w)^2) and parameter gradients; lr > 0
 * then applies one Adam step. d_x [B][H][W][16] BF16 (16-byte aligned),
 * d_base / d_target FP32 [B][H][W]; *loss_out (if not NULL) after a sync. */
int hr_cnn_train_step(hr_cnn* net, const uint16_t* d_x, const float* d_base, const float* d_target, int B, int H,
                      int W, float mu_w, float lr, float* loss_out, void* stream);
/* Inference: d_out[b*sb + (y*W+x)*sp] = base[same] + mu_w * residual. */
int hr_cnn_forward(hr_cnn* net, float* d_out, const uint16_t* d_x, const float* d_base, long long sb, long long sp,
                   int B, int H, int W, float mu_w, void* stream);
/* Corrects every slice of a volume [YN][XN][ZN] (z fastest), chunk slices per pass. */
int hr_cnn_apply_volume(hr_cnn* net, float* d_out, const float* d_vol, int XN, int YN, int ZN, float mu_w, int chunk,
                        void* stream);
/* Network input of slices [z0, z0+nz) of a volume (neighbours clamped at the ends). */
int hr_cnn_pack_input(uint16_t* d_x, const float* d_vol, int XN, int YN, int ZN, int z0, int nz, float mu_w,
                      void* stream);
/* Reads and clears the network's device error flag: HR_ERR_CUDA if a
 * tensor-core pipeline wait timed out in an earlier call. */
int hr_cnn_check(const hr_cnn* net);
/* Test hook, no counterpart in the reference: from the next call on, every
 * conv CTA leaves its input row number `row` unloaded (a barrier nothing
 * completes) and pipeline waits give up after wait_polls polls; the kernels
 * flag the error, let their issued copies and tensor-core operations finish,
 * free their tensor memory and return. row < 0 restores normal operation. */
int hr_cnn_test_stall(hr_cnn* net, int row, unsigned int wait_polls);
void hr_cnn_destroy(hr_cnn* net);

/* ---- GE raw data and the segment driver ---------------------------------- */
/* The header file of a GE scan: 18 floats (GetHeadofGeDataSet.m:20-30,
 * 0-based: [2] source-detector, [3] source-iso, [4] cell pitch at the detector
 * (mm), [5] first view angle (degrees), [8] views per rotation, [9] total
 * views, [10] channels per row, [11] iso channel (1-based), [12] rows, [13]
 * slice height at iso (mm), [14] helical pitch (table feed / slice height)).
 * The projection file: float32 [view][row][channel], no header. */
typedef struct hr_ge_header {
  float raw[18];
  double Source2DetDis, Source2IsoDis, DetCellPitch, BeginViewAngle;
  int NumberOfViewPerRotation, TotalViewNumber, NumberOfDetChannelPerRow, NumberOfDetectorRow;
  double IsoChannelLocation, SliceHeigh, HelicalPitch;
} hr_ge_header;
/* Reconstruction options of analyticalReconBigPatient.m:14-28 (NULL: k1 = 5,
 * delta = 60, HSCoef = 0.68). */
typedef struct hr_ge_options {
  double k1;
  int delta;
  double HSCoef;
} hr_ge_options;
int hr_ge_parse_header(const float* raw18, hr_ge_header* h);
int hr_ge_read_header(const char* path, hr_ge_header* h);
/* Segment overlap (half fan in views + 1) and count (analyticalRecon.m:15-17). */
int hr_ge_segments(const hr_ge_header* h, int seg_length, int* seg_overlap, int* seg_num);
/* First view and view count of segment seg_ind (1-based; readBigPatientData.m:16-23). */
int hr_ge_segment_views(const hr_ge_header* h, int seg_length, int seg_ind, int* first_view, int* dlength);
/* Reads segment seg_ind into fan [dlength][YL][ZL] with the channels flipped
 * (analyticalReconBigPatient.m:30), the layout the rebinning takes. fan holds
 * seg_length*YL*ZL floats. */
int hr_ge_read_segment(const char* path, const hr_ge_header* h, int seg_length, int seg_ind, float* fan,
                       int* dlength);
/* The whole-chain description of segment seg_ind (analyticalReconBigPatient.m:
 * 31-146 with the MEX field mapping): rebinning arguments, crop, filter
 * arguments, backprojection geometry (cubic voxels 2 objR/N, ZC = 10) and the
 * view weights w[N_2pi] (desc->w points at w). */
int hr_ge_segment_desc(const hr_ge_header* h, int seg_length, int seg_ind, double objR, int XN, int YN, int ZN,
                       const hr_ge_options* opt, int form, hr_recon_desc* desc, double* w);
/* analyticalRecon.m: every segment read, reconstructed on the GPU and summed
 * into h_vol [YN][XN][ZN]. */
int hr_ge_reconstruct(const char* proj_path, const char* head_path, int seg_length, double objR, int XN, int YN,
                      int ZN, const hr_ge_options* opt, int form, float* h_vol);
/* d_sum[i] += d_x[i] for i < n. */
int hr_accumulate(float* d_sum, const float* d_x, long long n, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* HELIXRECON_H */
