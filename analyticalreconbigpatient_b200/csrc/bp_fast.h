// Fast-form backprojection (BF16 filtered data, FP32 arithmetic, FP64 tables).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace hr {

constexpr int kBpFastNz = 16;  // z slices per thread (one CTA covers one z block)

struct BpFastGeom {
  int XN, YN, ZN, YL, ZL, PN, half;
  double XNC, YNC, ZNC, dx, dy, dz, YLC, ZLC, dYL, dZL, h, BetaS, DeltaFai, N_pi, SO, SD, k1;
};

struct BpFast {
  int nblocks = 0;
  float2* d_tab = nullptr;     // per z block and view of its window: NZ x {t2, Q}
  uint32_t* d_mask = nullptr;  // per z block and view: slices whose [s1, s2] holds the view
  float2* d_trig = nullptr;    // per view: {cos, sin}
  int* d_zblock = nullptr;     // [nblocks] {first view, count}, then [nblocks] table offsets
  size_t bytes = 0;
};

int bp_fast_create(BpFast* f, const BpFastGeom& g, const double* w);
void bp_fast_destroy(BpFast* f);
int bp_fast_execute(const BpFast& f, const BpFastGeom& g, float* vol, const uint32_t* fpb, cudaStream_t s);
// FP32 rows [rows][YL] -> BF16 channel pairs: word u = bf16(x[u]) | bf16(x[u+1]) << 16.
int pack_pairs(uint32_t* out, const float* in, long long rows, int YL, cudaStream_t s);

}  // namespace hr
