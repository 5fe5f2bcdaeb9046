// split.cuh -- the exact-split form (CF_FORM_AF_SYM_I8): host interface of split.cu.
//
// Q(f) on the q2 <-> q3 folded operator with the Phi step in FP64 on the CUDA cores and the
// K^3 step on the int8 tensor cores (tcgen05.mma kind::i8): Phi and R_t are written as
// 47-bit fixed-point integers split into six bytes each, the byte products are summed exactly
// in int32 tensor-memory accumulators, and the accumulators are recombined in FP64.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace cf {

struct SplitPlan;

// Builds the split operator from a folded plan's device operator (downloaded to the host, split,
// uploaded).  Returns a cf_status; on failure the message is set with cf_set_last_error.
int split_build(SplitPlan** out, const DevOp& folded, int64_t n_g, int64_t n_slices, int device);
void split_destroy(SplitPlan* sp);
int64_t split_device_bytes(const SplitPlan* sp);
// Q_cm += Q(f_cm) for B cells, cell-major [N_Q x K x B] device arrays; no allocation, no
// synchronisation.  Returns a cf_status (message set on failure).
int split_run(const SplitPlan* sp, double* q_cm, const double* f_cm, int64_t B, cudaStream_t st,
              int64_t* launches);
// The FP64 band kernel on the same units: Q_cm += Q(f_cm) with the K^3 step in FP64 (the plan's own
// G and R, plain or folded).  No allocation, no synchronisation.
int band64_run(const SplitPlan* sp, double* q_cm, const double* f_cm, int64_t B, cudaStream_t st,
               int64_t* launches);
// The BF16-split band kernel on the same units: Q_cm += Q(f_cm) with the K^3 step on the BF16 tensor
// cores (R_t and Phi as BF16 hi + lo, FP32 accumulation in tensor memory).  CF_EUNSUPPORTED where its
// shared memory does not fit.  No allocation, no synchronisation.
int bf16_band_run(const SplitPlan* sp, double* q_cm, const double* f_cm, int64_t B, cudaStream_t st,
                  int64_t* launches);
// The l-block kernels (K = 8 and 12): one CTA per (l1 band, cell group) -- 8 cells in FP64, 16 in the
// FP32 forms -- with R_t and the f rows of bands l2 and l3 staged per l-triplet by bulk copies, the
// band's (t, row) slices taken by the warps one at a time and summed per row in t order into FP64 Q.
// pf is a device workspace of at least lblock_pack_bytes(sp, B, f32) bytes for the packed f.  No
// allocation, no synchronisation.
int lblock_run(const SplitPlan* sp, double* q_cm, const double* f_cm, void* pf, size_t pf_bytes, int64_t B, bool f32,
               cudaStream_t st, int64_t* launches);
size_t lblock_pack_bytes(const SplitPlan* sp, int64_t B, bool f32);
// Self-test of the l-block kernel's bounded waits: the FP64 kernel on B cells with no stage ever
// filled and each wait limited to wait_cycles SM clocks; synchronises, and returns CF_ETIMEOUT (the
// error word cleared) when the waits ran out and the kernel returned, as they must.
int lblock_selftest(const SplitPlan* sp, double* q_cm, const double* f_cm, void* pf, size_t pf_bytes, int64_t B,
                    long long wait_cycles, cudaStream_t st, int64_t* launches);
bool lblock_available(const SplitPlan* sp, bool f32);
// After the stream has been synchronised: CF_ETIMEOUT (and the flag cleared) if a CTA of an
// earlier launch gave up a bounded wait, else CF_OK.
int split_check(const SplitPlan* sp);
// Whether the split form exists for this K (K divisible by 4, K <= 12).
bool split_supported_k(int k);

}  // namespace cf
