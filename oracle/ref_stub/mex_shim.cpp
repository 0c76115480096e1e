// Host shim that lets the reference MEX entry point run outside MATLAB (test oracle
// only).  mxArray is a small owned-or-borrowed N-d array; mexErrMsgTxt throws.  The
// exported C function ref_interp2 mirrors the MATLAB call Z = ba_interp2_spline(F, X, Y)
// for a double M x N image and n query points.
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
#include "mex.h"

struct mxArray {
  std::vector<mwSize> dims;
  mxClassID cls;
  void* data;
  std::vector<unsigned char> own;
};

const mwSize* mxGetDimensions(const mxArray* a) { return a->dims.data(); }
mwSize mxGetNumberOfDimensions(const mxArray* a) { return a->dims.size(); }
mwSize mxGetNumberOfElements(const mxArray* a) {
  mwSize n = 1;
  for (mwSize d : a->dims) n *= d;
  return n;
}
void* mxGetData(const mxArray* a) { return a->data; }
bool mxIsDouble(const mxArray* a) { return a->cls == mxDOUBLE_CLASS; }
bool mxIsSingle(const mxArray* a) { return a->cls == mxSINGLE_CLASS; }
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity) {
  mxArray* a = new mxArray;
  a->dims.assign(dims, dims + ndim);
  a->cls = cls;
  a->own.assign(mxGetNumberOfElements(a) * (cls == mxDOUBLE_CLASS ? 8 : 4), 0);
  a->data = a->own.data();
  return a;
}
void mexErrMsgTxt(const char* msg) { throw std::runtime_error(msg); }

extern "C" int ref_interp2(const double* F, long M, long N, const double* X, const double* Y, long n,
                           double* out) {
  mxArray f{{(mwSize)M, (mwSize)N}, mxDOUBLE_CLASS, const_cast<double*>(F), {}};
  mxArray x{{(mwSize)n, 1}, mxDOUBLE_CLASS, const_cast<double*>(X), {}};
  mxArray y{{(mwSize)n, 1}, mxDOUBLE_CLASS, const_cast<double*>(Y), {}};
  const mxArray* prhs[3] = {&f, &x, &y};
  mxArray* plhs[1] = {nullptr};
  try {
    mexFunction(1, plhs, 3, prhs);
  } catch (const std::exception&) {
    return -1;
  }
  std::memcpy(out, plhs[0]->data, sizeof(double) * n);
  delete plhs[0];
  return 0;
}
