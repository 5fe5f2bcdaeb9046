/*
 * mxhost.c -- a tiny mxArray host that runs MEX functions without MATLAB.
 *
 * TEST INFRASTRUCTURE ONLY (see mex.h).  An mxArray here is a column-major
 * double array with up to 8 dimensions.  Arrays made by mxh_wrap() borrow the
 * caller's buffer, which is how MATLAB hands its arrays to a MEX function: a MEX
 * function that writes into prhs[0] (the reference contraction kernels do,
 * src/mex/angular_first_collision_kernel_mex.cpp:68) writes straight into the
 * caller's memory.
 *
 * mexErrMsgIdAndTxt records the message and long-jumps back into mxh_call(),
 * which then returns 1, so a MEX error surfaces as a return code on the host.
 */
#include "mex.h"

#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MXH_MAXDIM 8

struct mxArray_tag {
    mxClassID cls;
    mwSize ndim;
    mwSize dims[MXH_MAXDIM];
    double* pr;
    int owns;
};

static _Thread_local jmp_buf* mxh_jmp = NULL;
static _Thread_local char mxh_msg[1024];
static _Thread_local char mxh_id[256];

static size_t numel(const mxArray* a) {
    size_t n = 1;
    for (mwSize i = 0; i < a->ndim; ++i) n *= a->dims[i];
    return n;
}

double* mxGetPr(const mxArray* a) { return a->pr; }
size_t mxGetM(const mxArray* a) { return a->ndim > 0 ? a->dims[0] : 0; }
size_t mxGetN(const mxArray* a) {
    /* MATLAB: product of all dimensions after the first */
    size_t n = 1;
    for (mwSize i = 1; i < a->ndim; ++i) n *= a->dims[i];
    return n;
}
double mxGetScalar(const mxArray* a) { return numel(a) > 0 ? a->pr[0] : 0.0; }
size_t mxGetNumberOfElements(const mxArray* a) { return numel(a); }
mwSize mxGetNumberOfDimensions(const mxArray* a) { return a->ndim; }
const mwSize* mxGetDimensions(const mxArray* a) { return a->dims; }
int mxIsDouble(const mxArray* a) { return a->cls == mxDOUBLE_CLASS; }
int mxIsComplex(const mxArray* a) { (void)a; return 0; }

static mxArray* make(mwSize ndim, const mwSize* dims, double* data, int owns) {
    mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
    if (!a) return NULL;
    a->cls = mxDOUBLE_CLASS;
    a->ndim = ndim < 2 ? 2 : (ndim > MXH_MAXDIM ? MXH_MAXDIM : ndim);
    for (mwSize i = 0; i < a->ndim; ++i) a->dims[i] = (i < ndim) ? dims[i] : 1;
    a->pr = data;
    a->owns = owns;
    return a;
}

mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cplx) {
    (void)cls; (void)cplx;
    mwSize nd = ndim < 2 ? 2 : ndim;
    mwSize d[MXH_MAXDIM];
    size_t n = 1;
    for (mwSize i = 0; i < nd && i < MXH_MAXDIM; ++i) {
        d[i] = (i < ndim) ? dims[i] : 1;
        n *= d[i];
    }
    double* data = (double*)calloc(n > 0 ? n : 1, sizeof(double));
    return make(nd, d, data, 1);
}

mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity cplx) {
    mwSize d[2] = {m, n};
    return mxCreateNumericArray(2, d, mxDOUBLE_CLASS, cplx);
}

mxArray* mxCreateDoubleScalar(double v) {
    mxArray* a = mxCreateDoubleMatrix(1, 1, mxREAL);
    if (a) a->pr[0] = v;
    return a;
}

void mxDestroyArray(mxArray* a) {
    if (!a) return;
    if (a->owns) free(a->pr);
    free(a);
}

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(mxh_msg, sizeof(mxh_msg), fmt, ap);
    va_end(ap);
    snprintf(mxh_id, sizeof(mxh_id), "%s", id ? id : "");
    if (mxh_jmp) longjmp(*mxh_jmp, 1);
    fprintf(stderr, "mexErrMsgIdAndTxt outside mxh_call: %s: %s\n", mxh_id, mxh_msg);
    abort();
}

/* ---------------- host-side API (called from C harnesses and ctypes) ---------------- */

typedef void (*mxh_mexfn)(int, mxArray**, int, const mxArray**);

/* Wrap a caller-owned column-major double buffer (no copy). */
mxArray* mxh_wrap(double* data, int ndim, const size_t* dims) {
    mwSize d[MXH_MAXDIM];
    int nd = ndim > MXH_MAXDIM ? MXH_MAXDIM : ndim;
    for (int i = 0; i < nd; ++i) d[i] = dims[i];
    return make((mwSize)nd, d, data, 0);
}

/* Run a MEX function; 0 on success, 1 if it raised mexErrMsgIdAndTxt. */
int mxh_call(mxh_mexfn fn, int nlhs, mxArray** plhs, int nrhs, const mxArray** prhs) {
    jmp_buf env;
    jmp_buf* saved = mxh_jmp;
    mxh_msg[0] = 0;
    mxh_id[0] = 0;
    mxh_jmp = &env;
    if (setjmp(env)) {
        mxh_jmp = saved;
        return 1;
    }
    fn(nlhs, plhs, nrhs, prhs);
    mxh_jmp = saved;
    return 0;
}

const char* mxh_last_error(void) { return mxh_msg; }
const char* mxh_last_error_id(void) { return mxh_id; }
double* mxh_data(mxArray* a) { return a->pr; }
size_t mxh_numel(const mxArray* a) { return numel(a); }
int mxh_ndim(const mxArray* a) { return (int)a->ndim; }
size_t mxh_dim(const mxArray* a, int i) { return (i >= 0 && (mwSize)i < a->ndim) ? a->dims[i] : 1; }
