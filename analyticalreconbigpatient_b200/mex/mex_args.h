// Argument checks shared by the MEX shims. The reference MEX files read their
// arguments through raw pointer casts without checks; these shims read the
// same arguments in the same order and raise a MATLAB error instead of
// reading a wrongly typed or short array.
#pragma once

#include "mex.h"
#include "matrix.h"

#include "helixrecon.h"

namespace hrmex {

inline void require(bool ok, const char* id, const char* msg) {
  if (!ok) mexErrMsgIdAndTxt(id, "%s", msg);
}

inline const void* data_of(const mxArray* a, mxClassID cls, size_t min_elems, const char* id, const char* what) {
  require(a != nullptr && mxGetClassID(a) == cls && !mxIsComplex(a) && mxGetNumberOfElements(a) >= min_elems, id,
          what);
  return mxGetData(a);
}

inline float f32(const mxArray* a, const char* id, const char* what) {
  return *static_cast<const float*>(data_of(a, mxSINGLE_CLASS, 1, id, what));
}

inline int i32(const mxArray* a, const char* id, const char* what) {
  return *static_cast<const int*>(data_of(a, mxINT32_CLASS, 1, id, what));
}

// Raises the library's message for a failed call.
inline void check(int status, const char* id) {
  if (status != HR_OK) mexErrMsgIdAndTxt(id, "%s", hr_last_error());
}

}  // namespace hrmex
