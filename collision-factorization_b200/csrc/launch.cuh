// launch.cuh -- per-K launch entry points.  Each K is instantiated in its own translation unit
// (inst_k<K>.cu) so the kernels compile in parallel; plan.cu calls them through cf_launch().
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace cf {

enum Op { OP_AF = 0, OP_RF = 1, OP_JV = 2 };

// Kernel families for the angular-first / Jacobian forms.
enum Path { PATH_AUTO = 0, PATH_GATHER = 1, PATH_TILE = 2, PATH_PAIR = 3, PATH_PAIR_L1 = 4, PATH_PAIR_SPLIT = 5, PATH_TILE_MMA = 6,
           PATH_BF16_MMA = 7 /* reported only: the BF16-split form's kernel */,
           PATH_TILE4 = 8 /* reported only: the quarter-tile kernel, where the 16-cell tile does not fit */,
           PATH_FEW = 9 /* reported only: the few-cell kernel (a handful of cells per call) */,
           PATH_SPLIT_I8 = 10 /* reported only: the exact-split form's kernel (split.cu) */,
           PATH_BAND = 11 /* the band kernels on the cell-major arrays (split.cu): the FP64 forms on request */,
           PATH_BAND_BF16 = 12 /* reported only: the BF16-split form on the band kernel (tcgen05, split.cu) */,
           PATH_RF_DENSE = 13 /* reported only: the radial-first dense form (rfdense.cu) */,
           PATH_LBLOCK = 14 /* the l-block kernel (split.cu): band units, f staged per l-triplet, K = 8 and 12 */ };

struct LaunchArgs {
    DevOp op;
    const double* fT;
    const double* vT;
    double* QT;
    int64_t n_tiles;
    int64_t n_cells;
    cudaStream_t stream;
    int what;    // Op
    bool exact;  // reference operation order, no FMA
    int path;    // Path
    // tile-resident kernels: q1 bins, work-queue counter, device limits
    const int* bin_begin;
    const int* bin_q1;
    int* counter;
    int n_sms;
    size_t max_smem;
    // pair kernels: bins over pair items, items (qa, qb)
    const int* pbin_begin;
    const int* pbin_item;
    const int2* pitems;
    // FP32 form: tiled FP32 copies of f (and v) in place of fT / vT
    bool f32;
    const float* fT32;
    // automatic order for the fast Q form: false = pair kernel first, true = tile kernel first
    bool tile_first;
    // BF16-split form (f32 is set too: FP32 tiles of f)
    bool bf16;
    // streamed host path: the tile kernel on cell-major f and Q while they are copied in and out
    const StreamSync* ss = nullptr;
    const double* f_cm = nullptr;
    double* q_cm = nullptr;
    const double* v_cm = nullptr;  // the exact J.v above K = 8 (rows): v, cell-major like f_cm
    // a handful of cells: the few-cell kernel on cell-major f_cm and q_cm (status -1 where it does not apply);
    // with few_host_f / few_host_q set, f and Q_in are those host arrays, passed in the launch's
    // parameter block, and q_cm receives Q_out
    bool few = false;
    const double* few_host_f = nullptr;
    const double* few_host_q = nullptr;
    // FP32 J.v: tiled FP32 copy of v
    const float* vT32 = nullptr;
    // with few: the exact form of any number of cells on the row kernel (one CTA per (q1, pair of cells), on the
    // cell-major arrays), the exact route where the batch kernels' register tiles do not fit (K > 8)
    bool rows = false;
};

// Status codes mirror cf_status: 0 ok, 5 CUDA error, 8 unsupported, 2 shape.
struct LaunchResult {
    int status;
    int launches;
    cudaError_t cuda;
    int path;  // the kernel family that ran
};

#define CF_DECLARE_K(KK) LaunchResult launch_k##KK(const LaunchArgs& a);
CF_DECLARE_K(1) CF_DECLARE_K(2) CF_DECLARE_K(3) CF_DECLARE_K(4) CF_DECLARE_K(5) CF_DECLARE_K(6)
CF_DECLARE_K(7) CF_DECLARE_K(8) CF_DECLARE_K(9) CF_DECLARE_K(10) CF_DECLARE_K(11) CF_DECLARE_K(12)
CF_DECLARE_K(13) CF_DECLARE_K(14) CF_DECLARE_K(15) CF_DECLARE_K(16)
#undef CF_DECLARE_K

// Lanes per cell (P) of the fast kernels: the K x K Phi accumulator is split over P lanes by
// k3 column once it no longer fits one lane's registers.
constexpr int af_P(int K) { return K <= 8 ? 1 : (K <= 12 ? 2 : 4); }
constexpr int jv_P(int K) { return K <= 6 ? 1 : (K <= 8 ? 2 : 4); }

}  // namespace cf
