// Fast-form backprojection (BF16 filtered data, FP32 arithmetic, FP64 tables).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

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
// -1 = slice pairs in packed FP32x2 arithmetic).
struct FastVariant {
  int table, chunk;
};
constexpr FastVariant kFastVariants[] = {{0, 0}, {0, 4}, {0, 8}, {1, 0}, {1, 4}, {1, 8},
                                         {0, -1}, {1, -1}, {2, 0}, {2, -1}, {2, 4}};
constexpr int kFastVariants_n = sizeof(kFastVariants) / sizeof(kFastVariants[0]);
constexpr int kFastDefaultVariant = 0;

struct BpFastTables {
  int nz = 0, nblocks = 0;
  size_t cap_rows = 0;         // reserved table rows (views summed over blocks)
  float2* d_tab = nullptr;     // per z block and view of its window: NZ x {t2, Q}
  uint32_t* d_mask = nullptr;  // per z block and view: slices whose [s1, s2] holds the view
  int* d_zblock = nullptr;     // [nblocks] {first view, count}, then [nblocks] table offsets
  size_t bytes = 0;
};

// Host copies of one geometry's tables (built in FP64, uploaded as float).
struct BpFastHostSet {
  int nz = 0, nblocks = 0;
  std::vector<float2> tab;
  std::vector<uint32_t> mask;
  std::vector<int> zb;
};
struct BpFastHost;

struct BpFast {
  BpFastTables t[kFastTableSets];
  float2* d_trig = nullptr;  // per view: {cos, sin}
  int cap_views = 0;
  int variant = kFastDefaultVariant;
  int tuned = 0;
  float tuned_ms[kFastVariants_n] = {};  // autotuner: ms per slice of each variant
  size_t bytes = 0;
};

struct BpFastHost {
  BpFastHostSet set[kFastTableSets];
  std::vector<float2> trig;
};

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
// FP32 rows [rows][YL] -> BF16 channel pairs: word u = bf16(x[u]) | bf16(x[u+1]) << 16.
int pack_pairs(uint32_t* out, const float* in, long long rows, int YL, cudaStream_t s);

}  // namespace hr
