// Test stand-in for the MATLAB MEX runtime (see mex.h here): column-major 2-D mxArrays of
// the classes the gateway uses, MATLAB's error unwinding as a C++ exception, and a small C
// interface (mexrt_*) through which pytest builds arguments, calls mexFunction and reads the
// outputs.  Test infrastructure only; the gateway itself is 3d-stereo-aldic_b200/mex/.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "mex.h"

struct mxArray {
  mxClassID cls = mxDOUBLE_CLASS;
  mwSize m = 0, n = 0;
  std::vector<unsigned char> bytes;
};

namespace {
size_t elem_size(mxClassID c) {
  switch (c) {
    case mxDOUBLE_CLASS: return 8;
    case mxINT32_CLASS: return 4;
    case mxUINT8_CLASS:
    case mxLOGICAL_CLASS:
    case mxCHAR_CLASS: return 1;
    default: return 1;
  }
}
mxArray* make(mxClassID cls, mwSize m, mwSize n) {
  mxArray* a = new mxArray;
  a->cls = cls;
  a->m = m;
  a->n = n;
  a->bytes.assign(m * n * elem_size(cls) + 1, 0);
  return a;
}
void (*g_exit_fn)(void) = nullptr;
}  // namespace

mwSize mxGetM(const mxArray* a) { return a->m; }
mwSize mxGetN(const mxArray* a) { return a->n; }
mwSize mxGetNumberOfElements(const mxArray* a) { return a->m * a->n; }
mxClassID mxGetClassID(const mxArray* a) { return a->cls; }
bool mxIsDouble(const mxArray* a) { return a->cls == mxDOUBLE_CLASS; }
bool mxIsComplex(const mxArray*) { return false; }
bool mxIsLogical(const mxArray* a) { return a->cls == mxLOGICAL_CLASS; }
bool mxIsChar(const mxArray* a) { return a->cls == mxCHAR_CLASS; }
double* mxGetDoubles(const mxArray* a) {
  return a->cls == mxDOUBLE_CLASS ? (double*)const_cast<unsigned char*>(a->bytes.data()) : nullptr;
}
mxLogical* mxGetLogicals(const mxArray* a) {
  return a->cls == mxLOGICAL_CLASS ? (mxLogical*)const_cast<unsigned char*>(a->bytes.data()) : nullptr;
}
void* mxGetData(const mxArray* a) { return const_cast<unsigned char*>(a->bytes.data()); }
double mxGetScalar(const mxArray* a) {
  if (a->m * a->n == 0) return 0.0;
  switch (a->cls) {
    case mxDOUBLE_CLASS: return ((const double*)a->bytes.data())[0];
    case mxINT32_CLASS: return ((const int32_t*)a->bytes.data())[0];
    default: return a->bytes[0];
  }
}
char* mxArrayToString(const mxArray* a) {
  if (a->cls != mxCHAR_CLASS) return nullptr;
  char* s = (char*)std::malloc(a->m * a->n + 1);
  std::memcpy(s, a->bytes.data(), a->m * a->n);
  s[a->m * a->n] = 0;
  return s;
}
void mxFree(void* p) { std::free(p); }
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity) { return make(mxDOUBLE_CLASS, m, n); }
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID cls, mxComplexity) { return make(cls, m, n); }
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  throw std::runtime_error(std::string(id) + ": " + buf);
}
int mexAtExit(void (*fn)(void)) {
  g_exit_fn = fn;
  return 0;
}

extern "C" {
// An m x n array of class cls (mxClassID values) holding a copy of data (column-major).
mxArray* mexrt_array(int cls, int64_t m, int64_t n, const void* data) {
  mxArray* a = make((mxClassID)cls, (mwSize)m, (mwSize)n);
  if (data) std::memcpy(a->bytes.data(), data, (size_t)(m * n) * elem_size((mxClassID)cls));
  return a;
}
mxArray* mexrt_string(const char* s) { return mexrt_array(mxCHAR_CLASS, 1, (int64_t)std::strlen(s), s); }
void* mexrt_data(mxArray* a) { return a->bytes.data(); }
int64_t mexrt_rows(mxArray* a) { return (int64_t)a->m; }
int64_t mexrt_cols(mxArray* a) { return (int64_t)a->n; }
int mexrt_class(mxArray* a) { return (int)a->cls; }
void mexrt_free(mxArray* a) { delete a; }
// mexFunction(nlhs, plhs, nrhs, prhs); 0, or 1 with the error text in err.
int mexrt_call(int nlhs, mxArray** plhs, int nrhs, const mxArray** prhs, char* err, int errlen) {
  try {
    mexFunction(nlhs, plhs, nrhs, prhs);
  } catch (const std::exception& e) {
    std::snprintf(err, errlen, "%s", e.what());
    return 1;
  }
  return 0;
}
// MATLAB's clear mex: the gateway's exit handler.
void mexrt_exit() {
  if (g_exit_fn) g_exit_fn();
  g_exit_fn = nullptr;
}
}
