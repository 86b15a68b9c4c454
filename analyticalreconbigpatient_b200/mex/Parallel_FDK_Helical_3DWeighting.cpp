// MEX shim: Parallel_FDK_Helical_3DWeighting(ScanGeom, double fpwd[YL,ZL,PN],
//     double ctimage[XN,YN,ZN], int32 useGPU)
// Same arguments as the reference MEX (src/Parallel_FDK_Helical_3DWeighting.cpp:204-262),
// with its ScanGeom field mapping:
//   ScDet = [SO DO YL ZL DecWidth DecHeigh YLC ZLC h]  (YLC is ignored: (YL-1)/2 is used)
//   Proj  = [BetaS BetaE ViewN N_2pi]                  (ViewN is the filtered view count PN)
//   Obj   = [ObjR XN YN ZN XC YC ZC]                   (1-based centres)
//   Rec   = [delta HSCoef k1]                          (k1 is scaled by the pitch ScDet(9))
// and, like it, no output: the volume is written in place into ctimage. useGPU == 1 runs
// the FP32 data path of the reference GPU branch, any other value its FP64 path.
#include "mex_args.h"

static const double* field(const mxArray* s, int k, size_t n, const char* id, const char* what) {
  const mxArray* f = mxGetFieldByNumber(s, 0, k);
  return static_cast<const double*>(hrmex::data_of(f, mxDOUBLE_CLASS, n, id, what));
}

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  (void)plhs;
  const char* id = "helixrecon:Parallel_FDK_Helical_3DWeighting";
  hrmex::require(nrhs == 4, id, "Backward projection needs 4 inputs.");
  hrmex::require(nlhs == 0, id, "Backward projection does not need any output.");
  hrmex::require(prhs[0] != nullptr && mxIsStruct(prhs[0]) && mxGetNumberOfFields(prhs[0]) >= 4, id,
                 "ScanGeom must be a struct with fields ScDet, Proj, Obj, Rec");
  const double* sc = field(prhs[0], 0, 9, id, "ScanGeom.ScDet must hold 9 doubles");
  const double* pj = field(prhs[0], 1, 4, id, "ScanGeom.Proj must hold 4 doubles");
  const double* ob = field(prhs[0], 2, 7, id, "ScanGeom.Obj must hold 7 doubles");
  const double* rc = field(prhs[0], 3, 3, id, "ScanGeom.Rec must hold 3 doubles");
  const double SO = sc[0], DO = sc[1];
  const int YL = (int)(sc[2] + 0.5), ZL = (int)(sc[3] + 0.5);
  const double DecWidth = sc[4], DecHeigh = sc[5];
  const double YLC = (YL - 1) * 0.5;
  const double ZLC = sc[7] - 1.0;
  const double h = sc[8] * DecHeigh;
  const double BetaS = pj[0];
  const int PN = (int)pj[2], N_2pi = (int)pj[3];
  const double ObjR = ob[0];
  const int XN = (int)(ob[1] + 0.5), YN = (int)(ob[2] + 0.5), ZN = (int)(ob[3] + 0.5);
  const double XNC = ob[4] - 1.0, YNC = ob[5] - 1.0, ZNC = ob[6] - 1.0;
  const int delta = (int)(rc[0] + 0.5);
  const double HSCoef = rc[1];
  const double k1 = rc[2] * sc[8];
  hrmex::require(YL > 0 && ZL > 0 && PN > 0 && XN > 0 && YN > 0 && ZN > 0 && N_2pi > 0, id,
                 "ScanGeom sizes must be positive");
  const double* fp = static_cast<const double*>(
      hrmex::data_of(prhs[1], mxDOUBLE_CLASS, (size_t)YL * ZL * PN, id, "fpwd must be double [YL,ZL,PN]"));
  const mxArray* img = prhs[2];
  hrmex::data_of(img, mxDOUBLE_CLASS, (size_t)XN * YN * ZN, id, "ctimage must be double [XN,YN,ZN]");
  double* ctimage = static_cast<double*>(mxGetData(img));
  const int useGPU = hrmex::i32(prhs[3], id, "useGPU must be int32");
  hrmex::check(hr_bp_host_reference(ctimage, fp, SO, DO, YL, ZL, DecWidth, DecHeigh, YLC, ZLC, h, BetaS, PN, N_2pi,
                                    ObjR, XN, YN, ZN, XNC, YNC, ZNC, delta, HSCoef, k1, useGPU),
               id);
}
