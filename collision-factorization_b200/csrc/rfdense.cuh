// rfdense.cuh -- the radial-first form with its radial step as a dense GEMM over cells
// (CF_FORM_RF_DENSE): host interface of rfdense.cu.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace cf {

struct RfDensePlan;

// Builds the tables of the form from a plan's device operator (downloaded to the host, regrouped by
// (l-triplet, q2), uploaded).  Returns a cf_status; on failure the message is set.
int rfdense_build(RfDensePlan** out, const DevOp& op, int64_t n_g, int64_t n_slices, int device);
void rfdense_destroy(RfDensePlan* rp);
int64_t rfdense_device_bytes(const RfDensePlan* rp);
// Q_cm += Q(f_cm) for B cells, cell-major [N_Q x K x B] device arrays.  Grows the plan's scratch on
// first use at a batch size (allocation); successive calls are ordered on the device by an event, so
// calls on different streams do not share the scratch at the same time.
int rfdense_run(RfDensePlan* rp, double* q_cm, const double* f_cm, int64_t B, cudaStream_t st, int64_t* launches);
// Whether the form is built for this K.
bool rfdense_supported_k(int k);

}  // namespace cf
