// Declarations of the MATLAB MEX C API (interleaved-complex, -R2018a) that
// the gateway inverse_solver_b200/mex/odt_mex.cpp uses, written from the
// public MEX documentation so that the gateway can be compile-checked where
// MATLAB is absent.  Declarations only: nothing here links or runs.
#pragma once
#include <cstddef>

typedef size_t mwSize;
typedef struct mxArray_tag mxArray;
typedef enum {
  mxUNKNOWN_CLASS = 0, mxCELL_CLASS, mxSTRUCT_CLASS, mxLOGICAL_CLASS, mxCHAR_CLASS, mxVOID_CLASS,
  mxDOUBLE_CLASS, mxSINGLE_CLASS, mxINT8_CLASS, mxUINT8_CLASS, mxINT16_CLASS, mxUINT16_CLASS,
  mxINT32_CLASS, mxUINT32_CLASS, mxINT64_CLASS, mxUINT64_CLASS
} mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX } mxComplexity;
typedef struct { float real, imag; } mxComplexSingle;
typedef struct { double real, imag; } mxComplexDouble;
typedef float mxSingle;

mxArray* mxGetField(const mxArray* pm, size_t index, const char* fieldname);
double mxGetScalar(const mxArray* pm);
size_t mxGetNumberOfElements(const mxArray* pm);
mwSize mxGetNumberOfDimensions(const mxArray* pm);
const mwSize* mxGetDimensions(const mxArray* pm);
double* mxGetPr(const mxArray* pm);
void* mxGetData(const mxArray* pm);
mxClassID mxGetClassID(const mxArray* pm);
bool mxIsComplex(const mxArray* pm);
mxSingle* mxGetSingles(const mxArray* pm);
mxComplexSingle* mxGetComplexSingles(const mxArray* pm);
mxComplexDouble* mxGetComplexDoubles(const mxArray* pm);
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID classid, mxComplexity flag);
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID classid, mxComplexity flag);
mxArray* mxCreateDoubleScalar(double value);
void mexErrMsgIdAndTxt(const char* errorid, const char* errormsg, ...);
