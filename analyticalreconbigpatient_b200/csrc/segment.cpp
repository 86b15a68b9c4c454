// GE raw-data reader and the segment-by-segment reconstruction driver.
//
// Restates the MATLAB host code around the three MEX calls so that a caller
// needs no MATLAB:
//   * GetHeadofGeDataSet.m:20-30    the 18-float header and its field map
//   * readBigPatientData.m:15-34    segment view ranges and the raw reads
//   * analyticalRecon.m:14-26       segment count/overlap and the summed volume
//   * analyticalReconBigPatient.m:30-146  channel flip, iso mirror, scan
//     geometry, rebinning arguments, crop, filter arguments, MEX field mapping
// The projection file holds float32 samples [view][row][channel] (channel
// fastest, as fread/reshape read them); the header file holds 18 floats.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "hr_internal.h"

namespace {

constexpr double kPi = 3.141592653589793;

struct FileCloser {
  FILE* f;
  ~FileCloser() {
    if (f) fclose(f);
  }
};

}  // namespace

extern "C" int hr_ge_parse_header(const float* raw, hr_ge_header* h) {
  HR_REQUIRE(raw != nullptr && h != nullptr, "hr_ge_parse_header: NULL argument");
  std::memset(h, 0, sizeof(*h));
  std::memcpy(h->raw, raw, sizeof(h->raw));
  h->Source2DetDis = raw[2];
  h->Source2IsoDis = raw[3];
  h->DetCellPitch = raw[4];
  h->BeginViewAngle = raw[5];
  h->NumberOfViewPerRotation = (int)raw[8];
  h->TotalViewNumber = (int)raw[9];
  h->NumberOfDetChannelPerRow = (int)raw[10];
  h->IsoChannelLocation = raw[11];
  h->NumberOfDetectorRow = (int)raw[12];
  h->SliceHeigh = raw[13];
  h->HelicalPitch = raw[14];
  HR_REQUIRE(h->Source2IsoDis > 0 && h->Source2DetDis > h->Source2IsoDis && h->DetCellPitch > 0 &&
                 h->NumberOfViewPerRotation > 1 && h->TotalViewNumber > 0 && h->NumberOfDetChannelPerRow > 1 &&
                 h->NumberOfDetectorRow > 0 && h->SliceHeigh > 0,
             "GE header: implausible geometry (SD=%g SO=%g pitch=%g views/rot=%d views=%d channels=%d rows=%d)",
             h->Source2DetDis, h->Source2IsoDis, h->DetCellPitch, h->NumberOfViewPerRotation, h->TotalViewNumber,
             h->NumberOfDetChannelPerRow, h->NumberOfDetectorRow);
  return HR_OK;
}

extern "C" int hr_ge_read_header(const char* path, hr_ge_header* h) {
  hr::clear_error();
  HR_REQUIRE(path != nullptr && h != nullptr, "hr_ge_read_header: NULL argument");
  FileCloser fc{std::fopen(path, "rb")};
  HR_REQUIRE(fc.f != nullptr, "hr_ge_read_header: cannot open %s", path);
  float raw[18];
  HR_REQUIRE(std::fread(raw, sizeof(float), 18, fc.f) == 18, "hr_ge_read_header: %s holds fewer than 18 floats",
             path);
  return hr_ge_parse_header(raw, h);
}

extern "C" int hr_ge_segments(const hr_ge_header* h, int seg_length, int* seg_overlap, int* seg_num) {
  HR_REQUIRE(h != nullptr && seg_overlap != nullptr && seg_num != nullptr, "hr_ge_segments: NULL argument");
  // analyticalRecon.m:15-17
  const double so = std::atan(h->DetCellPitch / h->Source2DetDis / 2.0) * h->NumberOfDetChannelPerRow;
  const int ov = (int)std::ceil(so * h->NumberOfViewPerRotation / (2.0 * kPi)) + 1;
  HR_REQUIRE(seg_length > 2 * ov, "hr_ge_segments: segment length %d must exceed twice the overlap (%d)", seg_length,
             ov);
  *seg_overlap = ov;
  *seg_num = (int)std::ceil(((double)h->TotalViewNumber - seg_length) / (double)(seg_length - 2 * ov)) + 1;
  if (*seg_num < 1) *seg_num = 1;
  return HR_OK;
}

extern "C" int hr_ge_segment_views(const hr_ge_header* h, int seg_length, int seg_ind, int* first_view,
                                   int* dlength) {
  int ov = 0, num = 0;
  HR_TRY(hr_ge_segments(h, seg_length, &ov, &num));
  HR_REQUIRE(seg_ind >= 1 && seg_ind <= num, "hr_ge_segment_views: segment %d outside 1..%d", seg_ind, num);
  // readBigPatientData.m:16-23
  *first_view = (seg_length - 2 * ov) * (seg_ind - 1);
  *dlength = seg_ind < num ? seg_length : h->TotalViewNumber - *first_view;
  HR_REQUIRE(*dlength > 0 && *first_view + *dlength <= h->TotalViewNumber,
             "hr_ge_segment_views: segment %d has no views", seg_ind);
  return HR_OK;
}

extern "C" int hr_ge_read_segment(const char* path, const hr_ge_header* h, int seg_length, int seg_ind, float* fan,
                                  int* dlength) {
  hr::clear_error();
  HR_REQUIRE(path != nullptr && h != nullptr && fan != nullptr && dlength != nullptr,
             "hr_ge_read_segment: NULL argument");
  int first = 0;
  HR_TRY(hr_ge_segment_views(h, seg_length, seg_ind, &first, dlength));
  const int YL = h->NumberOfDetChannelPerRow, ZL = h->NumberOfDetectorRow;
  const size_t view = (size_t)YL * ZL;
  FileCloser fc{std::fopen(path, "rb")};
  HR_REQUIRE(fc.f != nullptr, "hr_ge_read_segment: cannot open %s", path);
  HR_REQUIRE(std::fseek(fc.f, (long)(first * view * sizeof(float)), SEEK_SET) == 0,
             "hr_ge_read_segment: cannot seek to view %d of %s", first, path);
  // file [view][row][channel] -> fan [view][channel flipped][row] (analyticalReconBigPatient.m:30 and the
  // permute to the rebinning MEX's [ZL, YL, ViewN] order)
  std::vector<float> buf(view);
  for (int v = 0; v < *dlength; ++v) {
    HR_REQUIRE(std::fread(buf.data(), sizeof(float), view, fc.f) == view,
               "hr_ge_read_segment: %s ends inside view %d", path, first + v);
    float* out = fan + (size_t)v * view;
    for (int k = 0; k < ZL; ++k)
      for (int j = 0; j < YL; ++j) out[(size_t)(YL - 1 - j) * ZL + k] = buf[(size_t)k * YL + j];
  }
  return HR_OK;
}

extern "C" int hr_ge_segment_desc(const hr_ge_header* h, int seg_length, int seg_ind, double objR, int XN, int YN,
                                  int ZN, const hr_ge_options* opt, int form, hr_recon_desc* d, double* w) {
  hr::clear_error();
  HR_REQUIRE(h != nullptr && d != nullptr && w != nullptr, "hr_ge_segment_desc: NULL argument");
  HR_REQUIRE(XN > 0 && YN > 0 && ZN > 0 && objR > 0, "hr_ge_segment_desc: invalid volume");
  const hr_ge_options def = {5.0, 60, 0.68};
  const hr_ge_options& o = opt ? *opt : def;
  int ov = 0, num = 0, first = 0, DLength = 0;
  HR_TRY(hr_ge_segments(h, seg_length, &ov, &num));
  HR_TRY(hr_ge_segment_views(h, seg_length, seg_ind, &first, &DLength));
  // analyticalReconBigPatient.m:30-75 (after the channel flip and iso mirror)
  const double SO = h->Source2IsoDis, DO = h->Source2DetDis - h->Source2IsoDis;
  const int YL = h->NumberOfDetChannelPerRow, ZL = h->NumberOfDetectorRow;
  const double YLC = YL - h->IsoChannelLocation;
  const double ZLC = (1 + ZL) * 0.5;
  const double DetWid = h->DetCellPitch;
  const double DetHei = h->SliceHeigh * (DO + SO) / SO;
  const double DecAngle = std::atan(DetWid / (SO + DO) / 2.0) * YL * 2.0;
  const double DecHeigh = DetHei * ZL;
  const int N_2pi = h->NumberOfViewPerRotation;
  const double hn = h->HelicalPitch / ZL * SO / (DO + SO);
  const double dView = 2.0 * kPi / N_2pi;
  int ViewN = DLength;
  double BetaS = kPi - h->BeginViewAngle * kPi / 180.0 + (double)(seg_ind - 1) * (seg_length - 2 * ov) * dView;
  double BetaE = BetaS + ViewN * dView;
  // rebinning arguments (Parallel_Rebinning_CB_Curve.m:8-18; the MEX subtracts 1 in float)
  d->YL = YL;
  d->ZL = ZL;
  d->ViewN = ViewN;
  d->YLC = (float)YLC - 1.0f;
  d->dYA = (float)(DecAngle / YL);
  d->DeltaFai = (float)((BetaE - BetaS) / (ViewN - 1));
  d->DeltaTheta = d->DeltaFai;
  d->DeltaT = (float)(std::tan(DecAngle * 0.5) * SO * 1.5 * 2.0 / YL);
  d->PLC = (float)((1 + YL) * 0.5) - 1.0f;
  d->SO = (float)SO;
  // crop (analyticalReconBigPatient.m:80-93): first segment drops its tail overlap, the last its head, the
  // others both
  int view0 = 0;
  if (seg_ind == 1) {
    ViewN -= ov;
    BetaE -= ov * dView;
  } else if (seg_ind == num) {
    view0 = ov;
    ViewN -= ov;
    BetaS += ov * dView;
  } else {
    view0 = ov;
    ViewN -= 2 * ov;
    BetaS += ov * dView;
    BetaE -= ov * dView;
  }
  HR_REQUIRE(ViewN > 0, "hr_ge_segment_desc: segment %d keeps no views after the crop", seg_ind);
  d->view0 = view0;
  // filter arguments (:95-105, :139)
  const double DecWidth = std::tan(DecAngle * 0.5) * SO * 2.0 * 1.5;
  const double dYL = DecWidth / YL, dZL = DecHeigh / ZL;
  d->fPLC = (float)((1 + YL) * 0.5 - 1.0);
  d->fZLC = (float)(ZLC - 1.0);
  d->fdYL = (float)dYL;
  d->fdZL = (float)dZL;
  d->fSO = (float)SO;
  // backprojection: the MEX's field mapping (Parallel_FDK_Helical_3DWeighting.cpp:222-263) and the derived
  // scalars of ParallelFDKHelical3DWeighting (:145-154): cubic voxels 2 ObjR / N, XC = (N+1)/2, ZC = 10
  hr_bp_geom& g = d->bp;
  g.N_2pi = N_2pi;
  g.XN = XN;
  g.YN = YN;
  g.ZN = ZN;
  g.YL = YL;
  g.ZL = ZL;
  g.PN = ViewN;
  g.XNC = (XN + 1) * 0.5 - 1.0;
  g.YNC = (YN + 1) * 0.5 - 1.0;
  g.ZNC = 10.0 - 1.0;
  g.dx = 2.0 * objR / XN;
  g.dy = 2.0 * objR / YN;
  g.dz = 2.0 * objR / ZN;
  g.YLC = (YL - 1) * 0.5;
  g.ZLC = ZLC - 1.0;
  g.dYL = dYL;
  g.dZL = dZL;
  g.h = hn * DecHeigh;
  g.BetaS = BetaS;
  g.DeltaFai = 2.0 * kPi / N_2pi;
  g.N_pi = N_2pi / 2.0;
  g.HSCoef = o.HSCoef;
  g.SO = SO;
  g.SD = SO + DO;
  g.k1 = o.k1 * hn;
  d->form = form;
  d->w = w;
  return hr_view_weights(w, N_2pi, o.HSCoef, o.delta);
}

extern "C" int hr_ge_reconstruct(const char* proj_path, const char* head_path, int seg_length, double objR, int XN,
                                 int YN, int ZN, const hr_ge_options* opt, int form, float* h_vol) {
  hr::clear_error();
  HR_REQUIRE(proj_path != nullptr && head_path != nullptr && h_vol != nullptr, "hr_ge_reconstruct: NULL argument");
  hr_ge_header h;
  HR_TRY(hr_ge_read_header(head_path, &h));
  int ov = 0, num = 0;
  HR_TRY(hr_ge_segments(&h, seg_length, &ov, &num));
  HR_TRY(hr::require_device());
  const size_t nvol = (size_t)XN * YN * ZN;
  const size_t view = (size_t)h.NumberOfDetChannelPerRow * h.NumberOfDetectorRow;
  hr::DeviceBuffer d_sum, d_vol, d_fan;
  HR_TRY(d_sum.alloc(nvol * sizeof(float)));
  HR_TRY(d_vol.alloc(nvol * sizeof(float)));
  HR_TRY(d_fan.alloc((size_t)seg_length * view * sizeof(float)));
  HR_CUDA_TRY(cudaMemset(d_sum.ptr, 0, nvol * sizeof(float)));
  std::vector<float> fan((size_t)seg_length * view);
  std::vector<double> w(h.NumberOfViewPerRotation);
  // analyticalRecon.m:21-25: each segment reconstructs the whole grid from its own views; the volumes add up
  for (int s = 1; s <= num; ++s) {
    int DLength = 0;
    HR_TRY(hr_ge_read_segment(proj_path, &h, seg_length, s, fan.data(), &DLength));
    hr_recon_desc d;
    HR_TRY(hr_ge_segment_desc(&h, seg_length, s, objR, XN, YN, ZN, opt, form, &d, w.data()));
    HR_CUDA_TRY(cudaMemcpy(d_fan.ptr, fan.data(), (size_t)DLength * view * sizeof(float), cudaMemcpyHostToDevice));
    hr_recon_plan* plan = nullptr;
    HR_TRY(hr_recon_plan_create(&plan, &d));
    int st = hr_recon_execute(plan, d_vol.as<float>(), d_fan.as<float>(), nullptr);
    if (st == HR_OK) st = hr_accumulate(d_sum.as<float>(), d_vol.as<float>(), (long long)nvol, nullptr);
    if (st == HR_OK && cudaDeviceSynchronize() != cudaSuccess)
      st = hr::fail(HR_ERR_CUDA, "hr_ge_reconstruct: segment %d failed on the device", s);
    hr_recon_plan_destroy(plan);
    HR_TRY(st);
  }
  HR_CUDA_TRY(cudaMemcpy(h_vol, d_sum.ptr, nvol * sizeof(float), cudaMemcpyDeviceToHost));
  return HR_OK;
}
