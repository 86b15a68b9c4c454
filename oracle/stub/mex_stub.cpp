/*
 * Test infrastructure only: definitions behind the stand-in mex.h. The oracle
 * never runs a mexFunction, so every entry aborts loudly if reached.
 */
#include <cstdio>
#include <cstdlib>
#include "mex.h"

static void stub_abort(const char* what) {
  std::fprintf(stderr, "oracle mex stub: %s called outside MATLAB\n", what);
  std::abort();
}

extern "C" {
double* mxGetPr(const mxArray*) { stub_abort("mxGetPr"); return nullptr; }
void* mxGetData(const mxArray*) { stub_abort("mxGetData"); return nullptr; }
const mwSize* mxGetDimensions(const mxArray*) { stub_abort("mxGetDimensions"); return nullptr; }
mxArray* mxCreateNumericArray(mwSize, const mwSize*, mxClassID, mxComplexity) {
  stub_abort("mxCreateNumericArray");
  return nullptr;
}
mxArray* mxGetFieldByNumber(const mxArray*, mwIndex, int) { stub_abort("mxGetFieldByNumber"); return nullptr; }
void mexErrMsgTxt(const char* msg) { stub_abort(msg); }
}
