// Minimal stand-in for MATLAB's mex.h so that the reference's ba_interp2_spline.cpp can
// be compiled, unmodified, into a CPU library used only as a test oracle.  Declares just
// the mx* / mex* calls that file makes; oracle/ref_stub/mex_shim.cpp defines them.
#pragma once
#include <cstddef>
typedef std::size_t mwSize;
struct mxArray;
enum mxClassID { mxDOUBLE_CLASS = 6, mxSINGLE_CLASS = 7 };
enum mxComplexity { mxREAL = 0 };
const mwSize* mxGetDimensions(const mxArray* a);
mwSize mxGetNumberOfDimensions(const mxArray* a);
mwSize mxGetNumberOfElements(const mxArray* a);
void* mxGetData(const mxArray* a);
bool mxIsDouble(const mxArray* a);
bool mxIsSingle(const mxArray* a);
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cplx);
void mexErrMsgTxt(const char* msg);
void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);
