/*
 * mex.h -- a minimal stand-in for MATLAB's MEX API.
 *
 * TEST INFRASTRUCTURE ONLY.  MATLAB is not available on the build machine or on
 * the GPU machines, so the reference's MEX sources (src/mex/*.cpp) and this
 * project's own MEX shims are compiled against this header and driven by the
 * small mxArray host in mxhost.c.  Only the handful of calls those sources use
 * are provided: mxGetPr, mxGetM, mxGetN, mxGetScalar, mxGetNumberOfElements,
 * mxGetNumberOfDimensions, mxGetDimensions, mxIsDouble, mxIsComplex,
 * mxCreateNumericArray, mxCreateDoubleMatrix, mxCreateDoubleScalar, mxDestroyArray
 * and mexErrMsgIdAndTxt.
 *
 * mexFunction is declared with C linkage so that a C++ translation unit that
 * defines it (as every reference MEX source does) exports an unmangled symbol.
 * Compile each source with -DmexFunction=<unique_name> to link several into
 * one shared library.
 */
#ifndef CF_ORACLE_MEX_H
#define CF_ORACLE_MEX_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t mwSize;
typedef size_t mwIndex;

typedef enum {
    mxUNKNOWN_CLASS = 0,
    mxDOUBLE_CLASS = 6
} mxClassID;

typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

typedef struct mxArray_tag mxArray;

double*        mxGetPr(const mxArray* a);
size_t         mxGetM(const mxArray* a);
size_t         mxGetN(const mxArray* a);
double         mxGetScalar(const mxArray* a);
size_t         mxGetNumberOfElements(const mxArray* a);
mwSize         mxGetNumberOfDimensions(const mxArray* a);
const mwSize*  mxGetDimensions(const mxArray* a);
int            mxIsDouble(const mxArray* a);
int            mxIsComplex(const mxArray* a);
mxArray*       mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cplx);
mxArray*       mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity cplx);
mxArray*       mxCreateDoubleScalar(double v);
void           mxDestroyArray(mxArray* a);
void           mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);

#ifdef __cplusplus
}
#endif

#endif /* CF_ORACLE_MEX_H */
