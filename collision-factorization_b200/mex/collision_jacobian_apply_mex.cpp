// collision_jacobian_apply_mex.cpp -- J(f).v = Q(v,f) + Q(f,v) on the GPU (no reference counterpart).
// Signature: collision_jacobian_apply_mex(out, f, v, labels, vals, ic_map, R_tensor, N_Q, K_len)
// out is updated in place (out += J(f).v), in the same convention as the contraction MEX functions.
#include "cf_mex_common.hpp"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    (void)nlhs;
    (void)plhs;
    const char* id = "cf_b200:jacobian_apply";
    cfmex::require(nrhs == 9, id, "expected 9 inputs: (out, f, v, labels, vals, ic_map, R_tensor, N_Q, K_len)");
    const cfmex::OperatorArgs o = cfmex::operator_args(prhs, 3, id);
    const int64_t b = cfmex::cells(prhs[1], o, id);
    cfmex::require(cfmex::cells(prhs[0], o, id) == b && cfmex::cells(prhs[2], o, id) == b, id,
                   "out, f and v must have the same size");
    cfmex::raise_status(cf_jacobian_apply_host(mxGetPr(prhs[0]), mxGetPr(prhs[1]), mxGetPr(prhs[2]), b, o.labels,
                                               o.vals, o.ic_map, o.R, o.n_g, o.n_l, o.n_q, o.k, 0),
                        id);
}
