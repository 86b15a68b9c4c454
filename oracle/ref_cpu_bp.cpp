/*
 * Test infrastructure only (oracle). Compiles the reference's own
 * backprojection source, src/Parallel_FDK_Helical_3DWeighting.cpp, from where
 * it lies and exports:
 *   ref_bp_cpu_f64   -> ParallelFDKHelical3DWeightingCPU
 *                       (src/Parallel_FDK_Helical_3DWeighting.cpp:42-113)
 *   ref_ParallelFDKHelical3DWeighting -> the reference's extern "C"
 *                       ParallelFDKHelical3DWeighting (:117-200), renamed.
 * The reference's GPU entries are renamed to aborting stubs: the CPU oracle
 * only ever takes the useGPU==0 branch.
 */
#define mexFunction helix_ref_bp_mexFunction
#define ParallekFDKHelical3DWeighting_GPU_float helix_ref_bp_gpu_float_unused
#define ParallekFDKHelical3DWeighting_GPU_double helix_ref_bp_gpu_double_unused
#define ParallelFDKHelical3DWeighting ref_ParallelFDKHelical3DWeighting
#include "Parallel_FDK_Helical_3DWeighting.cpp"
#undef ParallelFDKHelical3DWeighting
#undef ParallekFDKHelical3DWeighting_GPU_double
#undef ParallekFDKHelical3DWeighting_GPU_float
#undef mexFunction

#include <cstdio>
#include <cstdlib>

static void ref_gpu_unused() {
  std::fprintf(stderr, "oracle: the reference GPU backprojection is not part of the CPU oracle\n");
  std::abort();
}

extern "C" void helix_ref_bp_gpu_float_unused(float*, const float*, const float*, const int, const int, const int,
                                              const int, const float, const float, const float, const float,
                                              const float, const float, const int, const int, const int,
                                              const float, const float, const float, const float, const float,
                                              const float, const float, const float, const float, const float,
                                              const float, const float) {
  ref_gpu_unused();
}

extern "C" void helix_ref_bp_gpu_double_unused(double*, const double*, const double*, const int, const int,
                                               const int, const int, const double, const double, const double,
                                               const double, const double, const double, const int, const int,
                                               const int, const double, const double, const double, const double,
                                               const double, const double, const double, const double,
                                               const double, const double, const double, const double) {
  ref_gpu_unused();
}

extern "C" void ref_bp_cpu_f64(double* ctimage, const double* fp, const double* w, int N_2pi, int XN, int YN, int ZN,
                               double XNC, double YNC, double ZNC, double dx, double dy, double dz, int YL, int ZL,
                               int PN, double YLC, double ZLC, double dYL, double dZL, double h, double BetaS,
                               double DeltaFai, double N_pi, double HSCoef, double SO, double SD, double k1) {
  ParallelFDKHelical3DWeightingCPU(ctimage, fp, w, N_2pi, XN, YN, ZN, XNC, YNC, ZNC, dx, dy, dz, YL, ZL, PN, YLC, ZLC,
                                   dYL, dZL, h, BetaS, DeltaFai, N_pi, HSCoef, SO, SD, k1);
}
