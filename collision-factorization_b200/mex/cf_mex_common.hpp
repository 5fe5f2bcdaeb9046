// cf_mex_common.hpp -- argument handling shared by the MEX shims over libcf_b200.
//
// The shims keep the reference's MEX calling convention exactly
// (src/mex/angular_first_collision_kernel_mex.cpp:5-16): eight real double arguments
// (Q_out, f, labels, vals, ic_map, R, N_Q, K_len), Q_out updated IN PLACE with +=, nothing
// returned.  N_G is mxGetM(labels) and N_L is numel(R)/K^3, as the reference implies.
// Unlike the reference, every argument is checked and a failure raises a MATLAB error through
// mexErrMsgIdAndTxt instead of reading out of bounds.  f and Q_out may also be N_Q x K x B
// arrays: the B cells are contracted in one GPU call.
#pragma once
#include <cstdint>

#include "cf_b200.h"
#include "mex.h"

namespace cfmex {

inline void require(bool ok, const char* id, const char* msg) {
    if (!ok) mexErrMsgIdAndTxt(id, "%s", msg);
}

inline bool is_real_double(const mxArray* a) { return mxIsDouble(a) && !mxIsComplex(a); }

struct OperatorArgs {
    const double *labels, *vals, *ic_map, *R;
    int64_t n_g;
    int32_t n_l, n_q, k;
};

// prhs[first..first+5] = labels, vals, ic_map, R, N_Q, K_len
inline OperatorArgs operator_args(const mxArray* const* prhs, int first, const char* id) {
    for (int i = 0; i < 6; ++i) require(is_real_double(prhs[first + i]), id, "all arguments must be real double arrays");
    OperatorArgs o;
    const mxArray* lab = prhs[first];
    o.n_g = (int64_t)mxGetM(lab);
    require(o.n_g == 0 || mxGetN(lab) == 3, id, "labels must be N_G x 3");
    require(mxGetNumberOfElements(prhs[first + 1]) == (size_t)o.n_g, id, "vals must have N_G elements");
    require(mxGetNumberOfElements(prhs[first + 2]) == (size_t)o.n_g, id, "ic_map must have N_G elements");
    const double nq = mxGetScalar(prhs[first + 4]), kk = mxGetScalar(prhs[first + 5]);
    require(nq >= 1 && nq <= 65535 && (double)(int32_t)nq == nq, id, "N_Q must be a positive integer");
    require(kk >= 1 && kk <= 16 && (double)(int32_t)kk == kk, id, "K_len must be an integer in [1, 16]");
    o.n_q = (int32_t)nq;
    o.k = (int32_t)kk;
    const size_t k3 = (size_t)o.k * o.k * o.k;
    const size_t nr = mxGetNumberOfElements(prhs[first + 3]);
    require(nr % k3 == 0, id, "numel(R_tensor) must be a multiple of K_len^3");
    o.n_l = (int32_t)(nr / k3);
    o.labels = mxGetPr(lab);
    o.vals = mxGetPr(prhs[first + 1]);
    o.ic_map = mxGetPr(prhs[first + 2]);
    o.R = mxGetPr(prhs[first + 3]);
    return o;
}

inline int64_t cells(const mxArray* a, const OperatorArgs& o, const char* id) {
    const size_t m = (size_t)o.n_q * o.k, n = mxGetNumberOfElements(a);
    require(is_real_double(a), id, "cell arrays must be real double");
    require(n % m == 0, id, "cell arrays must be N_Q x K_len (x B)");
    return (int64_t)(n / m);
}

inline void raise_status(int st, const char* id) {
    if (st != CF_OK) mexErrMsgIdAndTxt(id, "%s: %s", cf_status_string(st), cf_last_error());
}

// Q_out += contraction(f); prhs = (Q_out, f, labels, vals, ic_map, R, N_Q, K_len)
inline void contract(int nrhs, const mxArray* prhs[], int form, const char* id) {
    require(nrhs == 8, id, "expected 8 inputs: (Q_out, f, labels, vals, ic_map, R_tensor, N_Q, K_len)");
    const OperatorArgs o = operator_args(prhs, 2, id);
    const int64_t b = cells(prhs[1], o, id);
    require(cells(prhs[0], o, id) == b, id, "Q_out and f must have the same size");
    raise_status(cf_contract_host(mxGetPr(prhs[0]), mxGetPr(prhs[1]), b, o.labels, o.vals, o.ic_map, o.R, o.n_g,
                                  o.n_l, o.n_q, o.k, form),
                 id);
}

}  // namespace cfmex
