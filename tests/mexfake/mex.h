// Test double of MATLAB's mex.h (errors become C++ exceptions caught by mxf_call).
#pragma once
#include "matrix.h"

extern "C" void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);
void mexErrMsgTxt(const char* msg);
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);
