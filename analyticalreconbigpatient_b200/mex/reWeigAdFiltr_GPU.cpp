// MEX shim: fpwd = reWeigAdFiltr_GPU(single Proj[YL,ZL,ViewN], single PLC, single ZLC,
//     single dYL, single dZL, single SO)
// Same arguments and output as the reference MEX (src/reWeigAdFiltr_GPU.cpp:33-60): PLC and
// ZLC are passed through as given (the MATLAB driver already subtracts 1). The reference
// prints to stderr and calls exit(-1) on a wrong argument count; this shim raises a MATLAB
// error instead.
#include "mex_args.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  const char* id = "helixrecon:reWeigAdFiltr_GPU";
  hrmex::require(nlhs == 1 && nrhs == 6, id, "reWeigAdFiltr_GPU needs 6 inputs and gives one output");
  hrmex::require(prhs[0] != nullptr && mxGetNumberOfDimensions(prhs[0]) >= 2, id,
                 "Proj must be a single [YL,ZL,ViewN] array");
  const mwSize* siz = mxGetDimensions(prhs[0]);
  const int YL = (int)siz[0];
  const int ZL = (int)siz[1];
  const int ViewN = mxGetNumberOfDimensions(prhs[0]) >= 3 ? (int)siz[2] : 1;
  const size_t n = (size_t)YL * ZL * ViewN;
  const float* Proj = static_cast<const float*>(
      hrmex::data_of(prhs[0], mxSINGLE_CLASS, n, id, "Proj must be a single [YL,ZL,ViewN] array"));
  const float PLC = hrmex::f32(prhs[1], id, "PLC must be single");
  const float ZLC = hrmex::f32(prhs[2], id, "ZLC must be single");
  const float dYL = hrmex::f32(prhs[3], id, "dYL must be single");
  const float dZL = hrmex::f32(prhs[4], id, "dZL must be single");
  const float SO = hrmex::f32(prhs[5], id, "SO must be single");
  const mwSize dims[] = {(mwSize)YL, (mwSize)ZL, (mwSize)ViewN};
  plhs[0] = mxCreateNumericArray(3, dims, mxSINGLE_CLASS, mxREAL);
  float* fpwd = static_cast<float*>(mxGetData(plhs[0]));
  hrmex::check(hr_filter_host(fpwd, Proj, YL, ZL, ViewN, PLC, ZLC, dYL, dZL, SO), id);
}
