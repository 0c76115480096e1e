// Test stand-in for MATLAB's mex.h (R2018a interleaved API): the mx* / mex* calls that
// 3d-stereo-aldic_b200/mex/aldic_mex.cpp makes, with MATLAB's names and signatures, so the
// gateway compiles and runs outside MATLAB under pytest.  tests/mex/mex_runtime.cpp defines
// them; mexErrMsgIdAndTxt throws, as MATLAB unwinds the MEX call on an error.
#pragma once
#include <cstddef>
#include <cstdint>

typedef std::size_t mwSize;
typedef bool mxLogical;
struct mxArray;
enum mxClassID {
  mxUNKNOWN_CLASS = 0,
  mxLOGICAL_CLASS = 3,
  mxCHAR_CLASS = 4,
  mxDOUBLE_CLASS = 6,
  mxINT32_CLASS = 12,
  mxUINT8_CLASS = 9
};
enum mxComplexity { mxREAL = 0, mxCOMPLEX = 1 };

mwSize mxGetM(const mxArray* a);
mwSize mxGetN(const mxArray* a);
mwSize mxGetNumberOfElements(const mxArray* a);
mxClassID mxGetClassID(const mxArray* a);
bool mxIsDouble(const mxArray* a);
bool mxIsComplex(const mxArray* a);
bool mxIsLogical(const mxArray* a);
bool mxIsChar(const mxArray* a);
double* mxGetDoubles(const mxArray* a);
mxLogical* mxGetLogicals(const mxArray* a);
void* mxGetData(const mxArray* a);
double mxGetScalar(const mxArray* a);
char* mxArrayToString(const mxArray* a);
void mxFree(void* p);
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c);
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID cls, mxComplexity c);
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);
int mexAtExit(void (*fn)(void));
// C linkage, as MATLAB declares the gateway
extern "C" void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);
