/*
 * helix_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's helical cone-beam FBP chain, used by
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
 * checker. Nothing in the product library links or calls this file.
 *
 * Parity pin: the rebin and backprojection restatements are checked
 * bit-for-bit / to FP64 round-off against the reference's own CPU functions
 * compiled from its sources (oracle/Makefile -> oracle/_ref/libref_cpu.so),
 * and against golden vectors committed under tests/golden/. The filter has no
 * C/C++ CPU implementation in the reference (only MATLAB and cuFFT), so it is
 * pinned to golden vectors produced by the reference's own cuFFT filter
 * (src/filtering.cu built unmodified into oracle/_ref/libref_gpu.so).
 *
 * Functions and the reference lines they restate:
 *   hxo_rebin_f32 / hxo_rebin_f64  src/ParallelRebinningCBCurve.cpp:22-97
 *   hxo_weight_table               src/Parallel_FDK_Helical_3DWeighting.cpp:156-170
 *   hxo_filter_f64                 src/analyticalReconBigPatient.m:107-134
 *                                  (kernel/wrap/cut: src/filtering.cu:15-25,57-84,117-125;
 *                                   preweight: src/filtering.cu:187-207)
 *   hxo_bp_f64                     src/Parallel_FDK_Helical_3DWeighting.cpp:42-113
 *   hxo_project_ellipsoids         analytic FP64 line integrals (project-written data source)
 *
 * Build flags keep IEEE semantics: no -ffast-math, -ffp-contract=off.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define HXO_PI 3.141592653589793

/* ------------------------------------------------------------------------ */
/* Rebinning (fan -> parallel), layouts [ViewN][YL][ZL], ZL fastest.          */
/* ParallelRebinningCBCurve.cpp:22-97. In the reference's float instance the  */
/* unqualified asin/atan/sqrt bind to the C double functions (the compiled    */
/* reference imports asin and atan, never asinf/atanf), so the trig runs in   */
/* double on float arguments and is rounded to float on assignment.           */
/* coeXU/coeYU go through double because the reference writes `1.0 - coeXB`.  */
/* ------------------------------------------------------------------------ */
void hxo_rebin_f32(float* out, const float* proj, int YL, int ZL, int ViewN, float YLC, float dYA, float DeltaTheta,
                   float PLC, float DeltaT, float DeltaFai, float SO) {
  for (int i = 0; i < ViewN; ++i) {
    const float Theta = (float)i * DeltaTheta;
    for (int j = 0; j < YL; ++j) {
      const float t = ((float)j - PLC) * DeltaT;
      const float Beta = (float)asin((double)(t / SO));
      const float Fai = Theta + Beta;
      const float a = (float)atan((double)t / sqrt((double)(SO * SO - t * t)));
      const float FaiIndex = Fai / DeltaFai;
      const float UIndex = a / dYA + YLC;
      const int FI = (int)ceilf(FaiIndex);
      const int UI = (int)ceilf(UIndex);
      const float coeXB = (float)FI - FaiIndex;
      const float coeXU = (float)(1.0 - (double)coeXB);
      const float coeYB = (float)UI - UIndex;
      const float coeYU = (float)(1.0 - (double)coeYB);
      int XU, XB, YU, YB;
      if (FI <= 0) { XU = 0; XB = 0; }
      else if (FI > ViewN - 1) { XU = ViewN - 1; XB = ViewN - 1; }
      else { XU = FI; XB = FI - 1; }
      if (UI <= 0) { YU = 0; YB = 0; }
      else if (UI > YL - 1) { YU = YL - 1; YB = YL - 1; }
      else { YU = UI; YB = UI - 1; }
      const float w_bb = coeXB * coeYB, w_ub = coeXU * coeYB, w_bu = coeXB * coeYU, w_uu = coeXU * coeYU;
      const float* p_bb = proj + ((size_t)XB * YL + YB) * ZL;
      const float* p_ub = proj + ((size_t)XU * YL + YB) * ZL;
      const float* p_bu = proj + ((size_t)XB * YL + YU) * ZL;
      const float* p_uu = proj + ((size_t)XU * YL + YU) * ZL;
      float* o = out + ((size_t)i * YL + j) * ZL;
      for (int k = 0; k < ZL; ++k) {
        float acc = w_bb * p_bb[k];
        acc = acc + w_ub * p_ub[k];
        acc = acc + w_bu * p_bu[k];
        acc = acc + w_uu * p_uu[k];
        o[k] = acc;
      }
    }
  }
}

void hxo_rebin_f64(double* out, const double* proj, int YL, int ZL, int ViewN, double YLC, double dYA,
                   double DeltaTheta, double PLC, double DeltaT, double DeltaFai, double SO, int nthreads) {
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
  for (int i = 0; i < ViewN; ++i) {
    const double Theta = i * DeltaTheta;
    for (int j = 0; j < YL; ++j) {
      const double t = (j - PLC) * DeltaT;
      const double Fai = Theta + asin(t / SO);
      const double a = atan(t / sqrt(SO * SO - t * t));
      const double FaiIndex = Fai / DeltaFai;
      const double UIndex = a / dYA + YLC;
      const int FI = (int)ceil(FaiIndex);
      const int UI = (int)ceil(UIndex);
      const double coeXB = FI - FaiIndex, coeXU = 1.0 - coeXB;
      const double coeYB = UI - UIndex, coeYU = 1.0 - coeYB;
      int XU, XB, YU, YB;
      if (FI <= 0) { XU = 0; XB = 0; }
      else if (FI > ViewN - 1) { XU = ViewN - 1; XB = ViewN - 1; }
      else { XU = FI; XB = FI - 1; }
      if (UI <= 0) { YU = 0; YB = 0; }
      else if (UI > YL - 1) { YU = YL - 1; YB = YL - 1; }
      else { YU = UI; YB = UI - 1; }
      for (int k = 0; k < ZL; ++k) {
        out[((size_t)i * YL + j) * ZL + k] = coeXB * coeYB * proj[((size_t)XB * YL + YB) * ZL + k] +
                                             coeXU * coeYB * proj[((size_t)XU * YL + YB) * ZL + k] +
                                             coeXB * coeYU * proj[((size_t)XB * YL + YU) * ZL + k] +
                                             coeXU * coeYU * proj[((size_t)XU * YL + YU) * ZL + k];
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* 3D-weighting view table w[N_2pi]: Parallel_FDK_Helical_3DWeighting.cpp     */
/* :145-170. The reference's taper uses its file-level `pi` = 3.14159265358979*/
/* (:16), not the full-precision constant of :145.                           */
/* ------------------------------------------------------------------------ */
void hxo_weight_table(double* w, int N_2pi, double HSCoef, int delta) {
  const double pi_trunc = 3.14159265358979;
  const double N_pi = N_2pi / 2.0;
  for (int i = 0; i < N_2pi; ++i) w[i] = 0.0;
  const int L = (int)(2.0 * ceil(N_pi * HSCoef) + 1.0);
  const int Shift = (int)(N_pi - ceil(N_pi * HSCoef));
  for (int k = 0; k < L; ++k) {
    double v;
    if (0 <= k && k < delta) v = pow(cos((pi_trunc / 2) * (delta - k - 0.5) / delta), 2);
    else if (L - delta <= k && k < L) v = pow(cos((pi_trunc / 2) * (k - (L - delta) + 0.5) / delta), 2);
    else v = 1;
    const int idx = k + Shift;
    if (idx >= 0 && idx < N_2pi) w[idx] = v;
  }
}

/* ------------------------------------------------------------------------ */
/* Cosine preweight + Shepp-Logan ramp filter, FP64, layout [ViewN][ZL][YL]  */
/* (YL fastest). analyticalReconBigPatient.m:107-134: preweight              */
/* SO^2/sqrt(SO^4+(SO b)^2-(b t)^2), then the real part of the first YL       */
/* samples of ifft(fft(HS) .* fft(p, NN)). With NN >= 3 YL that circular      */
/* product equals the linear convolution f[j] = sum_m p[m] h[j-m], |j-m|<YL,  */
/* h[n] = -2/(pi^2 (4 n^2 - 1))/dYL, which is what is summed here directly.   */
/* PLC, ZLC are 0-based (the caller passes PLC-1, ZLC-1, m-file :139).        */
/* ------------------------------------------------------------------------ */
void hxo_filter_f64(double* out, const double* proj, int YL, int ZL, int ViewN, double PLC, double ZLC, double dYL,
                    double dZL, double SO, int nthreads) {
  double* hk = (double*)malloc(sizeof(double) * (2 * (size_t)YL + 1));
  const double pi2 = HXO_PI * HXO_PI;
  for (int n = -YL; n <= YL; ++n) hk[n + YL] = -2.0 / (pi2 * (4.0 * n * n - 1.0)) / dYL;
  const long long rows = (long long)ZL * ViewN;
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
  {
    double* p = (double*)malloc(sizeof(double) * (size_t)YL);
#pragma omp for schedule(static)
    for (long long r = 0; r < rows; ++r) {
      const int k = (int)(r % ZL);
      const double b = (k - ZLC) * dZL;
      const double* src = proj + (size_t)r * YL;
      for (int j = 0; j < YL; ++j) {
        const double t = (j - PLC) * dYL;
        p[j] = src[j] * SO * SO / sqrt(pow(SO, 4) + (SO * b) * (SO * b) - (b * t) * (b * t));
      }
      double* dst = out + (size_t)r * YL;
      for (int j = 0; j < YL; ++j) {
        double acc = 0.0;
        const double* hj = hk + YL + j; /* hj[-m] = h[j-m] */
        for (int m = 0; m < YL; ++m) acc += p[m] * hj[-m];
        dst[j] = acc;
      }
    }
    free(p);
  }
  free(hk);
}

/* ------------------------------------------------------------------------ */
/* 3D-weighted helical parallel-cone backprojection, FP64.                   */
/* Parallel_FDK_Helical_3DWeighting.cpp:42-113, loop s1..s2 (the CPU form;   */
/* the reference GPU kernel starts at 0, see its :47 vs CPU :71).            */
/* fp holds views [fp_view0, fp_view0 + fp_nviews) in [view][ZL][YL] order.  */
/* vox == NULL: full volume, out[(yi*XN+xi)*ZN+zi]; else out[n] = voxel      */
/* vox[n] (same linear index). Returns 0, or -1 if a needed view is not held.*/
/* ------------------------------------------------------------------------ */
int hxo_bp_f64(double* out, const double* fp, int fp_view0, int fp_nviews, const double* w, int N_2pi, int XN,
               int YN, int ZN, double XNC, double YNC, double ZNC, double dx, double dy, double dz, int YL, int ZL,
               int PN, double YLC, double ZLC, double dYL, double dZL, double h, double BetaS, double DeltaFai,
               double N_pi, double HSCoef, double SO, double SD, double k1, const int64_t* vox, int64_t nvox,
               int nthreads) {
  const double pi_trunc = 3.14159265358979;               /* :16, used for Beta0 (:62) */
  const double invPI = 1.0 / (2.0 * 3.141592653589793);   /* :51, used for temp2 (:79) */
  const int64_t total = vox ? nvox : (int64_t)XN * YN * ZN;
  int bad = 0;
  (void)N_2pi;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads > 0 ? nthreads : 1) reduction(| : bad)
  for (int64_t n = 0; n < total; ++n) {
    const int64_t lin = vox ? vox[n] : n;
    const int zi = (int)(lin % ZN);
    const int xi = (int)((lin / ZN) % XN);
    const int yi = (int)(lin / ((int64_t)ZN * XN));
    const double y = (yi - YNC) * dy;
    const double x = (xi - XNC) * dx;
    const double z = (zi - ZNC) * dz;
    const double Beta0 = 2.0 * pi_trunc * z / h;
    const int s0 = (int)ceil((Beta0 - BetaS) / DeltaFai - 0.5);
    int s1 = (int)(s0 - ceil(N_pi * HSCoef));
    int s2 = (int)(s0 + ceil(N_pi * HSCoef));
    double res = 0;
    if ((s1 < PN) && (s2 > 0)) {
      s1 = (s1 < 0) ? 0 : s1;
      s2 = (s2 > PN - 1) ? PN - 1 : s2;
      for (int ProjInd = s1; ProjInd <= s2; ++ProjInd) {
        const double View = BetaS + ProjInd * DeltaFai;
        const int d1 = (int)(N_pi - (s0 - ProjInd));
        const int d2 = (ProjInd < s0) ? (int)(d1 + N_pi) : (int)(d1 - N_pi);
        const double UU = -x * cos(View) - y * sin(View);
        const double Yr = -x * sin(View) + y * cos(View);
        const double temp1 = sqrt(SO * SO - Yr * Yr);
        const double temp2 = (z - h * View * invPI);
        const double Zr = temp2 * (SO * SD) / (UU * temp1 + SO * SO - Yr * Yr);
        const double U1 = Yr / dYL + YLC;
        const int U = (int)ceil(U1);
        const double V1 = Zr / dZL + ZLC;
        const int V = (int)ceil(V1);
        const double Dey = U - U1;
        const double Dez = V - V1;
        if ((U > 0) && (U < YL) && (V > 0) && (V < ZL)) {
          const int pl = ProjInd - fp_view0;
          if (pl < 0 || pl >= fp_nviews) { bad = 1; continue; }
          const double* f0 = fp + ((size_t)pl * ZL + (V - 1)) * YL;
          const double* f1 = fp + ((size_t)pl * ZL + V) * YL;
          const double touying = Dey * Dez * f0[U - 1] + Dey * (1.0 - Dez) * f1[U - 1] +
                                 (1.0 - Dey) * Dez * f0[U] + (1.0 - Dey) * (1.0 - Dez) * f1[U];
          const double weight1 = w[d1];
          const double weight2 = w[d2];
          const double Gama = fabs(temp2 / (temp1 + UU));
          const double Gama_C =
              (ProjInd < s0) ? fabs((temp2 - 0.5) / (temp1 - UU)) : fabs((temp2 + 0.5) / (temp1 - UU));
          const double m1 = pow(Gama, k1);
          const double m2 = pow(Gama_C, k1);
          const double weight = (weight1 * m2) / (weight2 * m1 + weight1 * m2);
          res += weight * touying * DeltaFai;
        }
      }
    }
    out[n] = res;
  }
  return bad ? -1 : 0;
}

/* ------------------------------------------------------------------------ */
/* Analytic FP64 projector (project-written data source, no reference        */
/* counterpart). Curved (arc) detector centred on the source, helical       */
/* source orbit. Fan view i: source angle beta = BetaS + i*dBeta, source     */
/* S = (SO cos beta, SO sin beta, h beta / 2 pi). Channel j: fan angle       */
/* gamma = (j - YLC0) * dYA, in-plane ray direction -(cos(beta-gamma),       */
/* sin(beta-gamma)) -- the parallel view angle of that ray is beta - gamma,  */
/* which is the relation the rebinning inverts (Fai = Theta + asin(t/SO)).   */
/* Row k: rise (k - ZLC0) * dZL over the in-plane source-detector distance   */
/* SD. Output layout [ViewN][YL][ZL] (ZL fastest), the rebinning input.      */
/*                                                                           */
/* Objects: nobj records of 17 doubles                                       */
/*   [type, cx, cy, cz, a, b, c, R00, R01, R02, R10, R11, R12, R20, R21, R22, */
/*    mu]; R's columns are the body axes in world coordinates.               */
/*   type 0: ellipsoid with semi-axes a, b, c.                               */
/*   type 1: elliptic cylinder, in-plane semi-axes a, b (body axes 0, 1),    */
/*           z in [cz - c, cz + c].                                          */
/* Densities add where objects overlap.                                      */
/* ------------------------------------------------------------------------ */
static double hxo_chord(const double* o, const double S[3], const double D[3], double Dnorm) {
  const double p0[3] = {S[0] - o[1], S[1] - o[2], S[2] - o[3]};
  const double* R = o + 7;
  double q0[3], q1[3];
  for (int i = 0; i < 3; ++i) {
    q0[i] = R[0 * 3 + i] * p0[0] + R[1 * 3 + i] * p0[1] + R[2 * 3 + i] * p0[2];
    q1[i] = R[0 * 3 + i] * D[0] + R[1 * 3 + i] * D[1] + R[2 * 3 + i] * D[2];
  }
  const double ax[3] = {o[4], o[5], o[6]};
  const int type = (int)o[0];
  const int nd = (type == 1) ? 2 : 3;
  double A = 0, B = 0, C = -1.0;
  for (int i = 0; i < nd; ++i) {
    const double u0 = q0[i] / ax[i], u1 = q1[i] / ax[i];
    A += u1 * u1;
    B += u0 * u1;
    C += u0 * u0;
  }
  if (A <= 0) return 0.0;
  const double disc = B * B - A * C;
  if (disc <= 0) return 0.0;
  const double sq = sqrt(disc);
  double s_lo = (-B - sq) / A, s_hi = (-B + sq) / A;
  if (type == 1) {
    const double z_lo = o[3] - o[6], z_hi = o[3] + o[6];
    if (D[2] == 0.0) {
      if (S[2] < z_lo || S[2] > z_hi) return 0.0;
    } else {
      double t0 = (z_lo - S[2]) / D[2], t1 = (z_hi - S[2]) / D[2];
      if (t0 > t1) { const double tt = t0; t0 = t1; t1 = tt; }
      if (t0 > s_lo) s_lo = t0;
      if (t1 < s_hi) s_hi = t1;
    }
    if (s_hi <= s_lo) return 0.0;
  }
  return (s_hi - s_lo) * Dnorm;
}

void hxo_project_ellipsoids(float* proj, int YL, int ZL, int ViewN, double SO, double SD, double dYA, double YLC0,
                            double dZL, double ZLC0, double BetaS, double dBeta, double h, const double* obj,
                            int nobj, int nthreads) {
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
  for (int i = 0; i < ViewN; ++i) {
    const double beta = BetaS + i * dBeta;
    const double S[3] = {SO * cos(beta), SO * sin(beta), h * beta / (2.0 * HXO_PI)};
    for (int j = 0; j < YL; ++j) {
      const double gam = (j - YLC0) * dYA;
      const double th = beta - gam;
      const double dxy[2] = {-cos(th), -sin(th)};
      for (int k = 0; k < ZL; ++k) {
        const double slope = (k - ZLC0) * dZL / SD;
        const double D[3] = {dxy[0], dxy[1], slope};
        const double Dn = sqrt(1.0 + slope * slope);
        double acc = 0.0;
        for (int e = 0; e < nobj; ++e) {
          const double* o = obj + (size_t)e * 17;
          acc += o[16] * hxo_chord(o, S, D, Dn);
        }
        proj[((size_t)i * YL + j) * ZL + k] = (float)acc;
      }
    }
  }
}
