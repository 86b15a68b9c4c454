// MEX shim: out = ParallelRebinningCBCurve(single Proj[ZL,YL,ViewN], int32 YL, int32 ZL,
//     int32 ViewN, single YLC, single dYA, single DeltaTheta, single PLC, single DeltaT,
//     single DeltaFai, single SO, int32 useGPU)
// Same arguments and output as the reference MEX (src/ParallelRebinningCBCurve.cpp:101-129):
// YLC and PLC arrive 1-based and are passed 0-based; the output is a new single
// [ZL,YL,ViewN] array. Both useGPU values run the GPU rebinning, which follows the
// reference CPU branch's clamp rule (its result is bit-identical to that branch).
#include "mex_args.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  const char* id = "helixrecon:ParallelRebinningCBCurve";
  hrmex::require(nrhs == 12 && nlhs <= 1, id, "ParallelRebinningCBCurve needs 12 inputs and gives one output");
  const int YL = hrmex::i32(prhs[1], id, "YL must be int32");
  const int ZL = hrmex::i32(prhs[2], id, "ZL must be int32");
  const int ViewN = hrmex::i32(prhs[3], id, "ViewN must be int32");
  hrmex::require(YL > 0 && ZL > 0 && ViewN > 0, id, "YL, ZL and ViewN must be positive");
  const size_t n = (size_t)YL * ZL * ViewN;
  const float* Proj = static_cast<const float*>(
      hrmex::data_of(prhs[0], mxSINGLE_CLASS, n, id, "Proj must be single with ZL*YL*ViewN elements"));
  const float YLC = hrmex::f32(prhs[4], id, "YLC must be single");
  const float dYA = hrmex::f32(prhs[5], id, "dYA must be single");
  const float DeltaTheta = hrmex::f32(prhs[6], id, "DeltaTheta must be single");
  const float PLC = hrmex::f32(prhs[7], id, "PLC must be single");
  const float DeltaT = hrmex::f32(prhs[8], id, "DeltaT must be single");
  const float DeltaFai = hrmex::f32(prhs[9], id, "DeltaFai must be single");
  const float SO = hrmex::f32(prhs[10], id, "SO must be single");
  (void)hrmex::i32(prhs[11], id, "useGPU must be int32");
  const mwSize dims[] = {(mwSize)ZL, (mwSize)YL, (mwSize)ViewN};
  plhs[0] = mxCreateNumericArray(3, dims, mxSINGLE_CLASS, mxREAL);
  float* out = static_cast<float*>(mxGetData(plhs[0]));
  hrmex::check(hr_rebin_host(out, Proj, YL, ZL, ViewN, YLC - 1.0f, dYA, DeltaTheta, PLC - 1.0f, DeltaT, DeltaFai, SO),
               id);
}
