// Host-pointer entry points: the reference's extern "C" drop-ins and their
// status-returning twins. Each call allocates device buffers, copies in, runs
// the stage on the current device's default stream, copies out and frees, as
// the reference's thrust-based entries do -- but every CUDA call is checked.
#include <cmath>
#include <cstdio>
#include <memory>
#include <vector>

#include "hr_internal.h"

namespace {

void report(const char* entry, int status) {
  if (status != HR_OK) std::fprintf(stderr, "helixrecon: %s failed (status %d): %s\n", entry, status, hr_last_error());
}

template <class Plan, void (*Destroy)(Plan*)>
struct PlanGuard {
  Plan* p = nullptr;
  ~PlanGuard() {
    if (p) Destroy(p);
  }
};

// View weight table of src/Parallel_FDK_Helical_3DWeighting.cpp:156-170, with
// the file-level pi of :16 in the taper.
void view_weights(std::vector<double>& w, int N_2pi, double HSCoef, int delta) {
  const double pi_trunc = 3.14159265358979;
  const double N_pi = N_2pi / 2.0;
  w.assign(N_2pi, 0.0);
  const int L = (int)(2.0 * std::ceil(N_pi * HSCoef) + 1.0);
  const int Shift = (int)(N_pi - std::ceil(N_pi * HSCoef));
  for (int k = 0; k < L; ++k) {
    double v;
    if (0 <= k && k < delta)
      v = std::pow(std::cos((pi_trunc / 2) * (delta - k - 0.5) / delta), 2);
    else if (L - delta <= k && k < L)
      v = std::pow(std::cos((pi_trunc / 2) * (k - (L - delta) + 0.5) / delta), 2);
    else
      v = 1;
    const int idx = k + Shift;
    if (idx >= 0 && idx < N_2pi) w[idx] = v;
  }
}

int bp_host(void* hvol, size_t vol_elem, const void* hfp, size_t fp_elem, const hr_bp_geom& g,
            const double* w, int form) {
  PlanGuard<hr_bp_plan, hr_bp_plan_destroy> plan;
  HR_TRY(hr_bp_plan_create(&plan.p, &g, w, form));
  const size_t nvol = (size_t)g.XN * g.YN * g.ZN;
  const size_t nfp = (size_t)g.YL * g.ZL * g.PN;
  hr::DeviceBuffer dvol, dfp;
  HR_TRY(dvol.alloc(nvol * vol_elem));
  HR_TRY(dfp.alloc(nfp * fp_elem));
  HR_CUDA_TRY(cudaMemcpy(dfp.ptr, hfp, nfp * fp_elem, cudaMemcpyHostToDevice));
  HR_TRY(hr_bp_execute(plan.p, dvol.ptr, dfp.ptr, nullptr));
  HR_CUDA_TRY(cudaMemcpy(hvol, dvol.ptr, nvol * vol_elem, cudaMemcpyDeviceToHost));
  return HR_OK;
}

hr_bp_geom make_geom(int N_2pi, int XN, int YN, int ZN, double XNC, double YNC, double ZNC, double dx, double dy,
                     double dz, int YL, int ZL, int PN, double YLC, double ZLC, double dYL, double dZL, double h,
                     double BetaS, double DeltaFai, double N_pi, double HSCoef, double SO, double SD, double k1) {
  hr_bp_geom g;
  g.N_2pi = N_2pi; g.XN = XN; g.YN = YN; g.ZN = ZN; g.YL = YL; g.ZL = ZL; g.PN = PN;
  g.XNC = XNC; g.YNC = YNC; g.ZNC = ZNC; g.dx = dx; g.dy = dy; g.dz = dz;
  g.YLC = YLC; g.ZLC = ZLC; g.dYL = dYL; g.dZL = dZL; g.h = h; g.BetaS = BetaS; g.DeltaFai = DeltaFai;
  g.N_pi = N_pi; g.HSCoef = HSCoef; g.SO = SO; g.SD = SD; g.k1 = k1;
  return g;
}

}  // namespace

extern "C" int hr_view_weights(double* w, int N_2pi, double HSCoef, int delta) {
  hr::clear_error();
  HR_REQUIRE(w != nullptr && N_2pi > 0 && delta > 0, "hr_view_weights: invalid argument");
  std::vector<double> v;
  view_weights(v, N_2pi, HSCoef, delta);
  for (int i = 0; i < N_2pi; ++i) w[i] = v[i];
  return HR_OK;
}

extern "C" int hr_rebin_host(float* out, const float* in, int YL, int ZL, int ViewN, float YLC, float dYA,
                             float DeltaTheta, float PLC, float DeltaT, float DeltaFai, float SO) {
  hr::clear_error();
  HR_REQUIRE(out != nullptr && in != nullptr, "ParallelRebinningCBCurve_GPU: NULL pointer");
  PlanGuard<hr_rebin_plan, hr_rebin_plan_destroy> plan;
  HR_TRY(hr_rebin_plan_create(&plan.p, YL, ZL, ViewN, YLC, dYA, DeltaTheta, PLC, DeltaT, DeltaFai, SO));
  const size_t n = (size_t)YL * ZL * ViewN;
  hr::DeviceBuffer din, dout;
  HR_TRY(din.alloc(n * sizeof(float)));
  HR_TRY(dout.alloc(n * sizeof(float)));
  HR_CUDA_TRY(cudaMemcpy(din.ptr, in, n * sizeof(float), cudaMemcpyHostToDevice));
  HR_TRY(hr_rebin_execute(plan.p, dout.as<float>(), din.as<float>(), nullptr));
  HR_CUDA_TRY(cudaMemcpy(out, dout.ptr, n * sizeof(float), cudaMemcpyDeviceToHost));
  return HR_OK;
}

extern "C" int hr_filter_host(float* out, const float* in, int YL, int ZL, int ViewN, float PLC, float ZLC, float dYL,
                              float dZL, float SO) {
  hr::clear_error();
  HR_REQUIRE(out != nullptr && in != nullptr, "filtering: NULL pointer");
  PlanGuard<hr_filter_plan, hr_filter_plan_destroy> plan;
  HR_TRY(hr_filter_plan_create(&plan.p, YL, ZL, ViewN, PLC, ZLC, dYL, dZL, SO));
  const size_t n = (size_t)YL * ZL * ViewN;
  hr::DeviceBuffer din, dout;
  HR_TRY(din.alloc(n * sizeof(float)));
  HR_TRY(dout.alloc(n * sizeof(float)));
  HR_CUDA_TRY(cudaMemcpy(din.ptr, in, n * sizeof(float), cudaMemcpyHostToDevice));
  HR_TRY(hr_filter_execute(plan.p, dout.as<float>(), din.as<float>(), HR_LAYOUT_ROWS, 0, nullptr));
  HR_CUDA_TRY(cudaMemcpy(out, dout.ptr, n * sizeof(float), cudaMemcpyDeviceToHost));
  return HR_OK;
}

extern "C" int hr_bp_host_float(float* hctimage, const float* hfp, const float* hw, int N_2pi, int XN, int YN,
                                int ZN, float XNC, float YNC, float ZNC, float dx, float dy, float dz, int YL, int ZL,
                                int PN, float YLC, float ZLC, float dYL, float dZL, float h, float BetaS,
                                float DeltaFai, float N_pi, float HSCoef, float SO, float SD, float k1) {
  hr::clear_error();
  HR_REQUIRE(hctimage != nullptr && hfp != nullptr && hw != nullptr && N_2pi > 0,
             "ParallekFDKHelical3DWeighting_GPU_float: NULL pointer");
  const hr_bp_geom g = make_geom(N_2pi, XN, YN, ZN, XNC, YNC, ZNC, dx, dy, dz, YL, ZL, PN, YLC, ZLC, dYL, dZL, h,
                                 BetaS, DeltaFai, N_pi, HSCoef, SO, SD, k1);
  std::vector<double> w(hw, hw + N_2pi);
  return bp_host(hctimage, sizeof(float), hfp, sizeof(float), g, w.data(), HR_FORM_PLAIN);
}

extern "C" int hr_bp_host_double(double* hctimage, const double* hfp, const double* hw, int N_2pi, int XN, int YN,
                                 int ZN, double XNC, double YNC, double ZNC, double dx, double dy, double dz, int YL,
                                 int ZL, int PN, double YLC, double ZLC, double dYL, double dZL, double h,
                                 double BetaS, double DeltaFai, double N_pi, double HSCoef, double SO, double SD,
                                 double k1) {
  hr::clear_error();
  HR_REQUIRE(hctimage != nullptr && hfp != nullptr && hw != nullptr,
             "ParallekFDKHelical3DWeighting_GPU_double: NULL pointer");
  const hr_bp_geom g = make_geom(N_2pi, XN, YN, ZN, XNC, YNC, ZNC, dx, dy, dz, YL, ZL, PN, YLC, ZLC, dYL, dZL, h,
                                 BetaS, DeltaFai, N_pi, HSCoef, SO, SD, k1);
  return bp_host(hctimage, sizeof(double), hfp, sizeof(double), g, hw, HR_FORM_FP64);
}

// ---------------------------------------------------------------------------
// Reference drop-ins (void, as the reference's).
// ---------------------------------------------------------------------------
extern "C" void ParallelRebinningCBCurve_GPU(float* outputProj, const float* Proj, const int YL, const int ZL,
                                             const int ViewN, const float YLC, const float dYA,
                                             const float DeltaTheta, const float PLC, const float DeltaT,
                                             const float DeltaFai, const float SO) {
  report("ParallelRebinningCBCurve_GPU",
         hr_rebin_host(outputProj, Proj, YL, ZL, ViewN, YLC, dYA, DeltaTheta, PLC, DeltaT, DeltaFai, SO));
}

extern "C" void filtering(float* hfpwd, const float* hProj, const int YL, const int ZL, const int ViewN,
                          const float PLC, const float ZLC, const float dYL, const float dZL, const float SO) {
  report("filtering", hr_filter_host(hfpwd, hProj, YL, ZL, ViewN, PLC, ZLC, dYL, dZL, SO));
}

extern "C" void ParallekFDKHelical3DWeighting_GPU_float(
    float* hctimage, const float* hfp, const float* hw, const int N_2pi, const int XN, const int YN, const int ZN,
    const float XNC, const float YNC, const float ZNC, const float dx, const float dy, const float dz, const int YL,
    const int ZL, const int PN, const float YLC, const float ZLC, const float dYL, const float dZL, const float h,
    const float BetaS, const float DeltaFai, const float N_pi, const float HSCoef, const float SO, const float SD,
    const float k1) {
  report("ParallekFDKHelical3DWeighting_GPU_float",
         hr_bp_host_float(hctimage, hfp, hw, N_2pi, XN, YN, ZN, XNC, YNC, ZNC, dx, dy, dz, YL, ZL, PN, YLC, ZLC, dYL,
                          dZL, h, BetaS, DeltaFai, N_pi, HSCoef, SO, SD, k1));
}

extern "C" void ParallekFDKHelical3DWeighting_GPU_double(
    double* hctimage, const double* hfp, const double* hw, const int N_2pi, const int XN, const int YN,
    const int ZN, const double XNC, const double YNC, const double ZNC, const double dx, const double dy,
    const double dz, const int YL, const int ZL, const int PN, const double YLC, const double ZLC,
    const double dYL, const double dZL, const double h, const double BetaS, const double DeltaFai,
    const double N_pi, const double HSCoef, const double SO, const double SD, const double k1) {
  report("ParallekFDKHelical3DWeighting_GPU_double",
         hr_bp_host_double(hctimage, hfp, hw, N_2pi, XN, YN, ZN, XNC, YNC, ZNC, dx, dy, dz, YL, ZL, PN, YLC, ZLC,
                           dYL, dZL, h, BetaS, DeltaFai, N_pi, HSCoef, SO, SD, k1));
}

extern "C" int hr_bp_host_reference(double* ctimage, const double* fp, double SO, double DO, int YL, int ZL,
                                    double DecWidth, double DecHeigh, double YLC, double ZLC, double h, double BetaS,
                                    int PN, int N_2pi, double ObjR, int XN, int YN, int ZN, double XNC, double YNC,
                                    double ZNC, int delta, double HSCoef, double k1, int useGPU) {
  hr::clear_error();
  HR_REQUIRE(ctimage != nullptr && fp != nullptr, "ParallelFDKHelical3DWeighting: NULL pointer");
  HR_REQUIRE(XN > 0 && YN > 0 && ZN > 0 && YL > 0 && ZL > 0 && PN > 0 && N_2pi > 0 && delta > 0,
             "ParallelFDKHelical3DWeighting: invalid sizes");
  // Derived scalars of src/Parallel_FDK_Helical_3DWeighting.cpp:145-154.
  const double PI = 3.141592653589793;
  const double N_pi = N_2pi / 2.0;
  const hr_bp_geom g = make_geom(N_2pi, XN, YN, ZN, XNC, YNC, ZNC, 2.0 * ObjR / XN, 2.0 * ObjR / YN,
                                 2.0 * ObjR / ZN, YL, ZL, PN, YLC, ZLC, DecWidth / YL, DecHeigh / ZL, h, BetaS,
                                 2.0 * PI / N_2pi, N_pi, HSCoef, SO, SO + DO, k1);
  std::vector<double> w;
  view_weights(w, N_2pi, HSCoef, delta);
  if (useGPU == 1) {
    // FP32 data path, as the reference's GPU branch (:173-190).
    const size_t nfp = (size_t)YL * ZL * PN, nvol = (size_t)XN * YN * ZN;
    std::vector<float> ffp(fp, fp + nfp), fvol(nvol);
    HR_TRY(bp_host(fvol.data(), sizeof(float), ffp.data(), sizeof(float), g, w.data(), HR_FORM_PLAIN));
    for (size_t i = 0; i < nvol; ++i) ctimage[i] = fvol[i];
    return HR_OK;
  }
  return bp_host(ctimage, sizeof(double), fp, sizeof(double), g, w.data(), HR_FORM_FP64);
}

extern "C" void ParallelFDKHelical3DWeighting(double* ctimage, const double* fp, const double SO, const double DO,
                                              const int YL, const int ZL, const double DecWidth,
                                              const double DecHeigh, const double YLC, const double ZLC,
                                              const double h, const double BetaS, const int PN, const int N_2pi,
                                              const double ObjR, const int XN, const int YN, const int ZN,
                                              const double XNC, const double YNC, const double ZNC, const int delta,
                                              const double HSCoef, const double k1, const int useGPU) {
  report("ParallelFDKHelical3DWeighting",
         hr_bp_host_reference(ctimage, fp, SO, DO, YL, ZL, DecWidth, DecHeigh, YLC, ZLC, h, BetaS, PN, N_2pi, ObjR,
                              XN, YN, ZN, XNC, YNC, ZNC, delta, HSCoef, k1, useGPU));
}
