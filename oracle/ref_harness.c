/*
 * oracle/ref_harness.c -- drive the reference's own MEX contraction kernels.
 *
 * TEST INFRASTRUCTURE and CPU BASELINE.  Linked into oracle/_ref/libref_*.so
 * together with the reference sources (compiled unmodified by oracle/Makefile,
 * each with -DmexFunction=<name>) and the mxArray host (mexhost/mxhost.c).
 *
 * refh_batch() calls one reference kernel once per cell, exactly as the
 * reference's benchmark harness calls it for one f
 * (benchmark_collision_contraction_scaling.m:96-108): Q_out (in place, +=), f,
 * labels, vals, ic_map, R, N_Q, K.  The reference kernels are single threaded;
 * the OpenMP loop over cells is this harness's, not the reference's.
 */
#include "mexhost/mex.h"

#include <stdint.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

void ref_af_mexFunction(int, mxArray**, int, const mxArray**);
void ref_rf_mexFunction(int, mxArray**, int, const mxArray**);
void ref_naive_mexFunction(int, mxArray**, int, const mxArray**);
void ref_dense_mexFunction(int, mxArray**, int, const mxArray**);
void ref_sumfac_mexFunction(int, mxArray**, int, const mxArray**);

mxArray* mxh_wrap(double* data, int ndim, const size_t* dims);

typedef void (*mexfn_t)(int, mxArray**, int, const mxArray**);

static mexfn_t pick(int which) {
    switch (which) {
        case 0: return ref_af_mexFunction;
        case 1: return ref_rf_mexFunction;
        case 2: return ref_naive_mexFunction;
        default: return NULL;
    }
}

/* which: 0 = angular_first, 1 = radial_first, 2 = naive.  Arrays are column-major;
 * Q and f are [N_Q x K x B].  Returns 0 on success. */
int refh_batch(int which, double* Q, const double* f, int64_t B, const double* labels,
               const double* vals, const double* ic_map, const double* R, int64_t NG, int NL,
               int NQ, int K, int nthreads) {
    mexfn_t fn = pick(which);
    if (!fn) return 2;
    const size_t M = (size_t)NQ * (size_t)K;
    int err = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads) reduction(| : err)
#endif
    {
        double nq = (double)NQ, kk = (double)K;
        size_t d_lab[2] = {(size_t)NG, 3}, d_vec[2] = {(size_t)NG, 1};
        size_t d_R[4] = {(size_t)K, (size_t)K, (size_t)K, (size_t)NL};
        size_t d_s[2] = {1, 1}, d_f[2] = {(size_t)NQ, (size_t)K};
        mxArray* a_lab = mxh_wrap((double*)labels, 2, d_lab);
        mxArray* a_val = mxh_wrap((double*)vals, 2, d_vec);
        mxArray* a_ic = mxh_wrap((double*)ic_map, 2, d_vec);
        mxArray* a_R = mxh_wrap((double*)R, 4, d_R);
        mxArray* a_nq = mxh_wrap(&nq, 2, d_s);
        mxArray* a_k = mxh_wrap(&kk, 2, d_s);
        if (!a_lab || !a_val || !a_ic || !a_R || !a_nq || !a_k) {
            err |= 1;
        } else {
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
            for (int64_t b = 0; b < B; ++b) {
                mxArray* q = mxh_wrap(Q + (size_t)b * M, 2, d_f);
                mxArray* fv = mxh_wrap((double*)f + (size_t)b * M, 2, d_f);
                const mxArray* prhs[8] = {q, fv, a_lab, a_val, a_ic, a_R, a_nq, a_k};
                fn(0, NULL, 8, prhs);
                mxDestroyArray(q);
                mxDestroyArray(fv);
            }
        }
        mxDestroyArray(a_lab); mxDestroyArray(a_val); mxDestroyArray(a_ic); mxDestroyArray(a_R);
        mxDestroyArray(a_nq); mxDestroyArray(a_k);
    }
    return err;
}

int refh_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
