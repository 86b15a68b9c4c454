/*
 * Test infrastructure only: a minimal, project-written stand-in for MATLAB's
 * mex.h / matrix.h so that the reference's C++ CPU sources can be compiled
 * without MATLAB. Only declarations the reference sources mention are given;
 * the matching definitions in mex_stub.cpp abort if ever called (the oracle
 * calls the reference's CPU functions directly, never its mexFunction).
 */
#ifndef HELIX_ORACLE_STUB_MEX_H
#define HELIX_ORACLE_STUB_MEX_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef size_t mwIndex;

typedef enum { mxUNKNOWN_CLASS = 0, mxDOUBLE_CLASS = 6, mxSINGLE_CLASS = 7, mxINT32_CLASS = 12 } mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

double* mxGetPr(const mxArray* a);
void* mxGetData(const mxArray* a);
const mwSize* mxGetDimensions(const mxArray* a);
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cplx);
mxArray* mxGetFieldByNumber(const mxArray* a, mwIndex index, int field);
void mexErrMsgTxt(const char* msg);

#ifdef __cplusplus
}
#endif

#endif
