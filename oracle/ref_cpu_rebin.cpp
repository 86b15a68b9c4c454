/*
 * Test infrastructure only (oracle). Compiles the reference's own rebinning
 * source, src/ParallelRebinningCBCurve.cpp, from where it lies (the include
 * path is set by oracle/Makefile) and exports its CPU template
 * ParallelRebinningCBCurve_CPU<T> (src/ParallelRebinningCBCurve.cpp:22-97)
 * under C names. The reference's mexFunction and GPU entry are renamed so
 * that they cannot collide with the product library's exports.
 */
#define mexFunction helix_ref_rebin_mexFunction
#define ParallelRebinningCBCurve_GPU helix_ref_rebin_gpu_unused
#include "ParallelRebinningCBCurve.cpp"
#undef ParallelRebinningCBCurve_GPU
#undef mexFunction

#include <cstdio>
#include <cstdlib>

extern "C" void helix_ref_rebin_gpu_unused(float*, const float*, const int, const int, const int, const float,
                                           const float, const float, const float, const float, const float,
                                           const float) {
  std::fprintf(stderr, "oracle: the reference GPU rebin is not part of the CPU oracle\n");
  std::abort();
}

extern "C" void ref_rebin_cpu_f32(float* out, const float* proj, int YL, int ZL, int ViewN, float YLC, float dYA,
                                  float DeltaTheta, float PLC, float DeltaT, float DeltaFai, float SO) {
  ParallelRebinningCBCurve_CPU<float>(out, proj, YL, ZL, ViewN, YLC, dYA, DeltaTheta, PLC, DeltaT, DeltaFai, SO);
}

extern "C" void ref_rebin_cpu_f64(double* out, const double* proj, int YL, int ZL, int ViewN, double YLC,
                                  double dYA, double DeltaTheta, double PLC, double DeltaT, double DeltaFai,
                                  double SO) {
  ParallelRebinningCBCurve_CPU<double>(out, proj, YL, ZL, ViewN, YLC, dYA, DeltaTheta, PLC, DeltaT, DeltaFai, SO);
}
