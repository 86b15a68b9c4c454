// Test double of MATLAB's matrix.h: the subset of the mx API the MEX shims use.
#pragma once
#include <cstddef>

typedef size_t mwSize;
typedef size_t mwIndex;
typedef enum {
  mxUNKNOWN_CLASS = 0, mxCELL_CLASS, mxSTRUCT_CLASS, mxLOGICAL_CLASS, mxCHAR_CLASS, mxVOID_CLASS,
  mxDOUBLE_CLASS, mxSINGLE_CLASS, mxINT8_CLASS, mxUINT8_CLASS, mxINT16_CLASS, mxUINT16_CLASS,
  mxINT32_CLASS, mxUINT32_CLASS, mxINT64_CLASS, mxUINT64_CLASS
} mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX } mxComplexity;
struct mxArray_tag;
typedef struct mxArray_tag mxArray;

void* mxGetData(const mxArray* a);
double* mxGetPr(const mxArray* a);
const mwSize* mxGetDimensions(const mxArray* a);
mwSize mxGetNumberOfDimensions(const mxArray* a);
size_t mxGetNumberOfElements(const mxArray* a);
mxClassID mxGetClassID(const mxArray* a);
bool mxIsComplex(const mxArray* a);
bool mxIsStruct(const mxArray* a);
int mxGetNumberOfFields(const mxArray* a);
mxArray* mxGetFieldByNumber(const mxArray* a, mwIndex i, int field);
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity c);
