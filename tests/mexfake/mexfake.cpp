// Minimal in-process stand-in for MATLAB's mx/mex runtime, linked into each MEX shim
// for tests: numeric arrays wrap caller memory (column-major dims, as MATLAB stores
// them), structs hold field arrays, mex errors are thrown and reported by mxf_call.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "mex.h"

struct mxArray_tag {
  mxClassID cls = mxUNKNOWN_CLASS;
  std::vector<mwSize> dims;
  void* data = nullptr;
  bool owns = false;
  std::vector<mxArray*> fields;
};

namespace {
std::string g_error;
size_t elem_size(mxClassID c) {
  switch (c) {
    case mxDOUBLE_CLASS: case mxINT64_CLASS: case mxUINT64_CLASS: return 8;
    case mxSINGLE_CLASS: case mxINT32_CLASS: case mxUINT32_CLASS: return 4;
    case mxINT16_CLASS: case mxUINT16_CLASS: return 2;
    default: return 1;
  }
}
struct MexError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
}  // namespace

void* mxGetData(const mxArray* a) { return a ? a->data : nullptr; }
double* mxGetPr(const mxArray* a) { return static_cast<double*>(mxGetData(a)); }
const mwSize* mxGetDimensions(const mxArray* a) { return a->dims.data(); }
mwSize mxGetNumberOfDimensions(const mxArray* a) { return a->dims.size(); }
size_t mxGetNumberOfElements(const mxArray* a) {
  size_t n = 1;
  for (mwSize d : a->dims) n *= d;
  return n;
}
mxClassID mxGetClassID(const mxArray* a) { return a->cls; }
bool mxIsComplex(const mxArray*) { return false; }
bool mxIsStruct(const mxArray* a) { return a && a->cls == mxSTRUCT_CLASS; }
int mxGetNumberOfFields(const mxArray* a) { return (int)a->fields.size(); }
mxArray* mxGetFieldByNumber(const mxArray* a, mwIndex i, int f) {
  if (!a || i != 0 || f < 0 || f >= (int)a->fields.size()) return nullptr;
  return a->fields[f];
}
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity) {
  mxArray* a = new mxArray_tag;
  a->cls = cls;
  a->dims.assign(dims, dims + ndim);
  a->data = std::calloc(mxGetNumberOfElements(a) ? mxGetNumberOfElements(a) : 1, elem_size(cls));
  a->owns = true;
  return a;
}
void mexErrMsgTxt(const char* msg) { throw MexError(msg); }
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  throw MexError(std::string(id) + ": " + buf);
}

extern "C" {
// Wraps caller memory (not owned) as a numeric array with MATLAB (column-major) dims.
mxArray* mxf_wrap(int cls, int ndim, const long long* dims, void* data) {
  mxArray* a = new mxArray_tag;
  a->cls = (mxClassID)cls;
  for (int i = 0; i < ndim; ++i) a->dims.push_back((mwSize)dims[i]);
  a->data = data;
  return a;
}
mxArray* mxf_struct(int nfields, mxArray** fields) {
  mxArray* a = new mxArray_tag;
  a->cls = mxSTRUCT_CLASS;
  a->dims = {1, 1};
  a->fields.assign(fields, fields + nfields);
  return a;
}
void* mxf_data(mxArray* a) { return a->data; }
long long mxf_numel(mxArray* a) { return (long long)mxGetNumberOfElements(a); }
void mxf_free(mxArray* a) {
  if (!a) return;
  if (a->owns) std::free(a->data);
  delete a;
}
// Calls the shim's mexFunction; 0 on success, 1 with mxf_error() set on a mex error.
int mxf_call(int nlhs, mxArray** plhs, int nrhs, mxArray** prhs) {
  try {
    mexFunction(nlhs, plhs, nrhs, const_cast<const mxArray**>(prhs));
  } catch (const MexError& e) {
    g_error = e.what();
    return 1;
  }
  return 0;
}
const char* mxf_error() { return g_error.c_str(); }
}
