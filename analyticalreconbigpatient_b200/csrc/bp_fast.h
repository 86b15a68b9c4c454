// Fast-form backprojection (BF16 filtered data, FP32 arithmetic, FP64 tables).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "helixrecon.h"

struct hr_bp_plan;

namespace hr {

struct BpFastGeom {
  int XN, YN, ZN, YL, ZL, PN, half;
  int ZN_valid;  // slices >= ZN_valid (padding of a last, partial slab) get no views
  double XNC, YNC, ZNC, dx, dy, dz, YLC, ZLC, dYL, dZL, h, BetaS, DeltaFai, N_pi, SO, SD, k1;
};

// Slices per thread of the table sets (a CTA covers one z block of NZ slices);
// thin slices favour 8-16 (per-view work shared by more slices), thick slices
// 4 (adjacent slices' view windows overlap less).
constexpr int kFastTableSets = 3;
constexpr int kFastNz[kFastTableSets] = {16, 8, 4};

// Kernel variants the autotuner chooses from: table set and gather chunk
// (0 = one slice at a time, 4/8 = slices whose gathers are issued together,
// -1 = slice pairs in packed FP32x2 arithmetic); tex != 0: the taps come from
// the texture units' bilinear filtering of a layered copy of the filtered data
// (kTexHalf: FP16 scaled by a power of two; kTexFloat: FP32).
constexpr int kTexHalf = 1, kTexFloat = 2;
// seg != 0 (texture variants with 8 or 4 slices per thread): the view loop of
// a z block runs in segments over which the set of slices whose window holds
// the view is a fixed range [ma, mb], with code specialised for that range, so
// slices without the view cost nothing (thick slices: a block's union window
// is much longer than one slice's); seg = 2: segments whose range holds at
// most 4 slices run two views per iteration, both views' taps in flight
// together (thick slices: few taps per view). occ = 6: the segmented code with
// registers bounded for 6 CTAs per SM.
struct FastVariant {
  int table, chunk, tex, seg, occ;
};
constexpr FastVariant kFastVariants[] = {{0, 0}, {0, 4}, {0, 8}, {1, 0}, {1, 4}, {1, 8},
                                         {0, -1}, {1, -1}, {2, 0}, {2, -1}, {2, 4},
                                         {1, 0, kTexHalf}, {0, 0, kTexHalf}, {2, 0, kTexHalf},
                                         {1, 0, kTexFloat}, {0, 0, kTexFloat},
                                         {1, 0, kTexHalf, 1}, {2, 0, kTexHalf, 1},
                                         {1, 0, kTexHalf, 2}, {2, 0, kTexHalf, 2},
                                         {1, 0, kTexHalf, 1, 6}, {2, 0, kTexHalf, 2, 6}};
constexpr int kFastVariants_n = sizeof(kFastVariants) / sizeof(kFastVariants[0]);
constexpr int kFastDefaultVariant = 0;

// Scans one persistent batch launch covers (their descriptors travel as one
// kernel parameter block).
constexpr int kBatchMaxScans = 16;

// View segments per z block of the segmented variants: {q0, q1, ma, mb}, views
// [q0, q1) of the block's window with active slices [ma, mb] (q0 == q1: unused).
constexpr int kSegPerNz = 2;  // at most 2 NZ segments per block (NZ - 1 entering, 1 full, NZ - 1 leaving)

struct BpFastTables {
  int nz = 0, nblocks = 0;
  size_t cap_rows = 0;         // reserved table rows (views summed over blocks)
  float2* d_tab = nullptr;     // per z block and view of its window: NZ x {t2, 2^Q}
  uint32_t* d_mask = nullptr;  // per z block and view: slices whose [s1, s2] holds the view
  int* d_zblock = nullptr;     // [nblocks] {first view, count}, then [nblocks] table offsets
  int4* d_seg = nullptr;       // [nblocks][kSegPerNz NZ] view segments
  size_t bytes = 0;
  std::vector<int> h_zb;       // host copy of the [nblocks] {first view, count} of the last upload
};

// Host copies of one geometry's tables (built in FP64, uploaded as float).
struct BpFastHostSet {
  int nz = 0, nblocks = 0;
  std::vector<float2> tab;
  std::vector<uint32_t> mask;
  std::vector<int> zb;
  std::vector<int4> seg;
};
struct BpFastHost;

// Layered 2D textures holding the filtered data of the texture variants: n
// CUDA arrays of 2^lsh views (layers) of [ZL][YL] samples each.
struct BpFastTex {
  int kind = 0;  // 0 (none), kTexHalf or kTexFloat
  int lsh = 0, n = 0, YL = 0, ZL = 0, views = 0;
  std::vector<cudaArray_t> arr;
  std::vector<unsigned long long> tex, surf;  // texture and surface objects of the arrays
  unsigned long long* d_obj = nullptr;        // device copy: n texture objects, then n surface objects
  float* d_scale = nullptr;                   // device: {1 / FP16 scale, max |value| (bits)}
  size_t bytes = 0;
};

struct BpFast {
  BpFastTables t[kFastTableSets];
  float2* d_trig = nullptr;  // per view: {cos, sin}
  int cap_views = 0;
  int variant = kFastDefaultVariant;
  int tuned = 0;
  float tuned_ms[kFastVariants_n] = {};  // autotuner: ms per slice of each variant
  size_t bytes = 0;
  BpFastTex tex;
};

struct BpFastHost {
  BpFastHostSet set[kFastTableSets];
  std::vector<float2> trig;
};

// Device bytes the plan holds: tables and, for a texture variant, the layered copy.
inline size_t bp_fast_device_bytes(const BpFast& f) { return f.bytes + f.tex.bytes; }

int bp_fast_create(BpFast* f, const BpFastGeom& g, const double* w);
// Pieces of bp_fast_create for plans whose geometry changes between launches
// (z slabs): build the tables of a geometry on the host, reserve device
// capacity once, upload (stream-ordered) before each launch.
int bp_fast_host_tables(BpFastHost* h, const BpFastGeom& g, const double* w);
int bp_fast_reserve(BpFast* f, const size_t rows[kFastTableSets], const int nblocks[kFastTableSets], int PN);
int bp_fast_upload(BpFast* f, const BpFastHost& h, cudaStream_t s);
void bp_fast_destroy(BpFast* f);
int bp_fast_execute(const BpFast& f, const BpFastGeom& g, float* vol, const uint32_t* fpb, cudaStream_t s);
int bp_fast_autotune(BpFast* f, const BpFastGeom& g, float* vol, const uint32_t* fpb, cudaStream_t s);
int bp_fast_describe(const BpFast& f, char* buf, int len);
// Allocates (or frees) the layered textures the plan's variant samples
// (no-op for the gather variants); hr_bp_select and the slab pipeline call it
// after choosing a variant by hand.
int bp_fast_tex_prepare(BpFast* f, const BpFastGeom& g);
// Fills the plan's layered textures from BF16 pairs (stream-ordered).
int bp_fast_tex_fill(const BpFast& f, const BpFastGeom& g, const uint32_t* fpb, cudaStream_t s);
// Fills views [p0, p1) only. mode 0: the FP16 scale from these views' largest |value| (a whole fill); 1: the
// first range of a fill done range by range while later views are still being produced (its scale leaves
// headroom for larger values later); 2: a later range with the first range's scale. After a fill by ranges,
// bp_fast_tex_refill_needed (synchronous) says whether a later range's values exceeded the FP16 range of that
// scale (or the first range was all zeros); the copy must then be refilled whole (mode 0) before its samples
// are used again.
int bp_fast_tex_fill_range(const BpFast& f, const BpFastGeom& g, const uint32_t* fpb, int p0, int p1, int mode,
                           cudaStream_t s);
int bp_fast_tex_refill_needed(const BpFast& f, bool* needed);
// Backprojects z blocks [b_first, b_first + b_count) of the plan's variant (a texture variant samples the
// copy as it is: no fill).
int bp_fast_execute_blocks(const BpFast& f, const BpFastGeom& g, float* vol, const uint32_t* fpb, int b_first,
                           int b_count, cudaStream_t s);
// The z-block tables of the plan's variant (nz slices per block; h_zb: each block's view window).
const BpFastTables& bp_fast_variant_tables(const BpFast& f);
// Several scans in one persistent launch. Each scan runs the kernel body with
// its own slices per thread (16, 8 or 4; 8 or 4 with texture taps); batch
// variants differ in the CTAs (of 256 threads) per SM their registers must
// allow (1: unconstrained; 4; 5; 6), in the gathers issued together (one slice
// at a time, or chunks of 4 slices) and in the taps (register gathers, or
// samples of each scan's FP16 texture copy; for these, chunk = 4 runs every
// scan with 4 slices per thread). Variant 11 (streams = 1) is not a
// persistent launch: every scan runs its own plan's kernel on a stream of its
// own, forked from and joined back into the batch's stream (the batch plan
// drives it; bp_fast_batch_execute refuses it). Variants 12-14 (spec = 1) are
// persistent texture launches whose column code is specialised per scan (a
// constant descriptor index per copy, so each scan's constants are
// constant-bank operands, not registers): each scan's own slices per thread
// (12), or 4 for every scan with registers unconstrained (13) or limited for
// 5 CTAs per SM (14). Variants 15-16 (seg = 1) are persistent texture launches
// running the segmented view loop of the single-scan variants 16-17 with each
// scan's own slices per thread, registers unconstrained or limited for 4 CTAs
// per SM.
struct BatchVariant {
  int min_ctas, chunk, tex, streams, spec, seg;
};
constexpr BatchVariant kBatchVariants[] = {{1, 0}, {5, 0}, {6, 0}, {1, 4}, {5, 4}, {6, 4},
                                           {1, 0, kTexHalf}, {4, 0, kTexHalf}, {4, 4, kTexHalf},
                                           {5, 4, kTexHalf}, {6, 4, kTexHalf}, {0, 0, 0, 1},
                                           {1, 0, kTexHalf, 0, 1}, {1, 4, kTexHalf, 0, 1}, {5, 4, kTexHalf, 0, 1},
                                           {1, 0, kTexHalf, 0, 0, 1}, {4, 0, kTexHalf, 0, 0, 1}};
constexpr int kBatchVariants_n = sizeof(kBatchVariants) / sizeof(kBatchVariants[0]);
struct BpFastBatchScan {
  const BpFast* f;
  const BpFastGeom* g;
  float* vol;
  const uint32_t* fpb;
  int nz;  // slices per thread (a table set)
};
// Work items (scan, z block, 8 x 16 column tile) of the batch (-1: a bad nz).
long long bp_fast_batch_items(const BpFastBatchScan* scans, int n);
// Persistent CTAs a launch of batch variant bv keeps resident (occupancy x SMs).
int bp_fast_batch_grid(int bv, int* ctas);
// Backprojects items [begin, begin + count) of the batch with at most ctas CTAs;
// d_counter: a device int the launch consumes (zeroed on the stream first).
int bp_fast_batch_execute(const BpFastBatchScan* scans, int n, int bv, int begin, int count, int ctas,
                          int* d_counter, cudaStream_t s);
// Slices per thread of the fastest per-slice variant the plan's autotuner timed (8 if untuned).
int bp_fast_best_per_slice_nz(const BpFast& f);
// The faster of the FP16 texture variants with 8 and 4 slices per thread (11 if untuned).
int bp_fast_best_tex_variant(const BpFast& f);
// Slices per thread of variant v.
int bp_fast_variant_nz(int v);
// The fast-form geometry and tables of a backprojection plan (HR_FORM_FAST).
int bp_plan_fast_parts(const hr_bp_plan* plan, const BpFastGeom** g, const BpFast** f);
// The fast-form geometry of a backprojection geometry (checked as hr_bp_plan_create checks it), host only.
int fast_geom_of(const hr_bp_geom& g, BpFastGeom* f);
void fast_geom_fill(const hr_bp_geom& g, int half, BpFastGeom* f);
// FP32 rows [rows][YL] -> BF16 channel pairs: word u = bf16(x[u]) | bf16(x[u+1]) << 16.
int pack_pairs(uint32_t* out, const float* in, long long rows, int YL, cudaStream_t s);

}  // namespace hr
