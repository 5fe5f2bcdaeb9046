// radial_first_collision_kernel_mex.cpp -- GPU drop-in for the reference MEX of the same name.
// Signature: radial_first_collision_kernel_mex(Q_out, f, labels_sorted, vals_sorted, ic_map_sorted,
//                                              R_tensor, N_Q, K_len)       (Q_out updated in place)
#include "cf_mex_common.hpp"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    (void)nlhs;
    (void)plhs;
    cfmex::contract(nrhs, prhs, CF_FORM_RF, "cf_b200:radial_first");
}
