// inst.cuh -- the body of one per-K translation unit (included by inst_k<K>.cu with CF_K defined).
#pragma once
#include <cstring>
#include <mutex>
#include <vector>

#include "kernels.cuh"
#include "launch.cuh"
#include "tile_kernels.cuh"
#include "pair_kernels.cuh"
#include "mma_kernels.cuh"
#include "bf16_kernels.cuh"
#include "few_kernels.cuh"

namespace cf {

// The dynamic shared-memory attribute and the resident CTAs per SM of a kernel, set and queried on
// its first launch with a given shared-memory size on a device and remembered, so that later
// launches (and launches recorded into a CUDA graph) make no attribute or occupancy calls.
struct ResidentEntry {
    const void* fn;
    int dev;
    size_t smem;
    int per_sm;
};
static cudaError_t resident_ctas(const void* fn, int threads, size_t smem, int* per_sm) {
    static std::mutex mu;
    static std::vector<ResidentEntry> seen;
    static std::vector<ResidentEntry> attr;  // per (fn, dev): the largest size the attribute allows
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    for (const ResidentEntry& r : seen)
        if (r.fn == fn && r.dev == dev && r.smem == smem) {
            *per_sm = r.per_sm;
            return cudaSuccess;
        }
    ResidentEntry* a = nullptr;
    for (ResidentEntry& r : attr)
        if (r.fn == fn && r.dev == dev) a = &r;
    if (!a || a->smem < smem) {
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        if (a)
            a->smem = smem;
        else
            attr.push_back({fn, dev, smem, 0});
    }
    int n = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, smem);
    if (e != cudaSuccess) return e;
    seen.push_back({fn, dev, smem, n});
    *per_sm = n;
    return cudaSuccess;
}

template <int K, int P, bool EXACT, bool JV>
static LaunchResult launch_af(const LaunchArgs& a) {
    const int64_t warps = (int64_t)a.op.n_items * a.n_tiles * P;
    if (warps == 0) return {0, 0, cudaSuccess, PATH_GATHER};
    const int64_t blocks = (warps + 3) / 4;
    if (blocks > INT32_MAX) return {2, 0, cudaSuccess, PATH_GATHER};
    af_kernel<K, P, EXACT, JV><<<(unsigned)blocks, 128, 0, a.stream>>>(a.op, a.fT, a.vT, a.QT, (int)a.n_tiles);
    const cudaError_t e = cudaGetLastError();
    return {e == cudaSuccess ? 0 : 5, 1, e, PATH_GATHER};
}

// Tile-resident persistent kernel.  Returns status -1 when it does not fit (shared memory or
// occupancy), in which case the caller uses the gather kernel.
template <int K, int W, bool EXACT, bool JV>
static LaunchResult launch_tile(const LaunchArgs& a) {
    const int M = a.op.n_q * K;
    const size_t smem = tile_smem_bytes<K>(M, W, JV);
    if (smem + 256 > a.max_smem || a.counter == nullptr) return {-1, 0, cudaSuccess, PATH_TILE};
    auto kern = af_tile_kernel<K, W, EXACT, JV>;
    int per_sm = 0;
    cudaError_t e = resident_ctas((const void*)kern, W * 32, smem, &per_sm);
    if (e != cudaSuccess) return {5, 0, e, PATH_TILE};
    if (per_sm < 1) return {-1, 0, cudaSuccess, PATH_TILE};
    const int64_t ctas = (int64_t)per_sm * a.n_sms;
    const int64_t n_ht = (a.n_cells + kTileCells - 1) / kTileCells;
    TileSched sc;
    sc.bin_begin = a.bin_begin;
    sc.bin_q1 = a.bin_q1;
    sc.n_ht = (int)n_ht;
    const int64_t n_whole = n_ht > ctas ? n_ht - ctas : 0;
    const int64_t rem = n_ht - n_whole;
    sc.split = rem * 4 >= ctas ? 4 : 16;
    sc.n_whole = (int)n_whole;
    const int64_t n_units = n_whole + rem * sc.split;
    if (n_units > INT32_MAX) return {2, 0, cudaSuccess, PATH_TILE};
    sc.n_units = (int)n_units;
    sc.counter = a.counter;
    e = cudaMemsetAsync(a.counter, 0, sizeof(int), a.stream);
    if (e != cudaSuccess) return {5, 0, e, PATH_TILE};
    const unsigned grid = (unsigned)(n_units < ctas ? n_units : ctas);
    kern<<<grid, W * 32, smem, a.stream>>>(a.op, sc, a.fT, a.vT, a.QT);
    e = cudaGetLastError();
    return {e == cudaSuccess ? 0 : 5, 1, e, PATH_TILE};
}

// Tile kernel on cell-major f and Q (a.f_cm, a.q_cm).  Streamed (a.ss->ready set): every half-tile
// split into 4 q1 bins, chunk flags in a.ss.  Resident (a.ss->ready null): the tile kernel's own
// schedule, no waits.  Status -1 when the tile does not fit.
template <int K, int W>
static LaunchResult launch_tile_stream(const LaunchArgs& a) {
    const int M = a.op.n_q * K;
    const size_t smem = tile_smem_bytes<K>(M, W, false);
    if (smem + 256 > a.max_smem || a.counter == nullptr) return {-1, 0, cudaSuccess, PATH_TILE};
    auto kern = af_tile_stream_kernel<K, W>;
    int per_sm = 0;
    cudaError_t e = resident_ctas((const void*)kern, W * 32, smem, &per_sm);
    if (e != cudaSuccess) return {5, 0, e, PATH_TILE};
    if (per_sm < 1) return {-1, 0, cudaSuccess, PATH_TILE};
    const int64_t ctas = (int64_t)per_sm * a.n_sms;
    const int64_t n_ht = (a.n_cells + kTileCells - 1) / kTileCells;
    TileSched sc;
    sc.bin_begin = a.bin_begin;
    sc.bin_q1 = a.bin_q1;
    sc.n_ht = (int)n_ht;
    if (a.ss->ready) {
        sc.n_whole = 0;
        sc.split = 4;
    } else {
        const int64_t n_whole = n_ht > ctas ? n_ht - ctas : 0;
        sc.n_whole = (int)n_whole;
        sc.split = (n_ht - n_whole) * 4 >= ctas ? 4 : 16;
    }
    const int64_t n_units = sc.n_whole + (n_ht - sc.n_whole) * sc.split;
    if (n_units > INT32_MAX) return {2, 0, cudaSuccess, PATH_TILE};
    sc.n_units = (int)n_units;
    sc.counter = a.counter;
    e = cudaMemsetAsync(a.counter, 0, sizeof(int), a.stream);
    if (e != cudaSuccess) return {5, 0, e, PATH_TILE};
    const unsigned grid = (unsigned)(n_units < ctas ? n_units : ctas);
    kern<<<grid, W * 32, smem, a.stream>>>(a.op, sc, *a.ss, a.f_cm, a.q_cm, (long long)a.n_cells);
    e = cudaGetLastError();
    return {e == cudaSuccess ? 0 : 5, 1, e, PATH_TILE};
}

// Quarter-tile kernel (8 cells per CTA, fast forms, K % 4 == 0).  Status -1 when it does not fit.
template <int K, int W, bool JV>
static LaunchResult launch_tile4(const LaunchArgs& a) {
    const int M = a.op.n_q * K;
    const size_t smem = tile4_smem_bytes<K>(M, W, JV);
    if (smem + 256 > a.max_smem || a.counter == nullptr) return {-1, 0, cudaSuccess, PATH_TILE4};
    auto kern = af_tile4_kernel<K, W, JV>;
    int per_sm = 0;
    cudaError_t e = resident_ctas((const void*)kern, W * 32, smem, &per_sm);
    if (e != cudaSuccess) return {5, 0, e, PATH_TILE4};
    if (per_sm < 1) return {-1, 0, cudaSuccess, PATH_TILE4};
    const int64_t ctas = (int64_t)per_sm * a.n_sms;
    const int64_t n_qt = (a.n_cells + kQuarterCells - 1) / kQuarterCells;
    TileSched sc;
    sc.bin_begin = a.bin_begin;
    sc.bin_q1 = a.bin_q1;
    sc.n_ht = (int)n_qt;
    const int64_t n_whole = n_qt > ctas ? n_qt - ctas : 0;
    const int64_t rem = n_qt - n_whole;
    sc.split = rem * 4 >= ctas ? 4 : 16;
    sc.n_whole = (int)n_whole;
    const int64_t n_units = n_whole + rem * sc.split;
    if (n_units > INT32_MAX) return {2, 0, cudaSuccess, PATH_TILE4};
    sc.n_units = (int)n_units;
    sc.counter = a.counter;
    e = cudaMemsetAsync(a.counter, 0, sizeof(int), a.stream);
    if (e != cudaSuccess) return {5, 0, e, PATH_TILE4};
    const unsigned grid = (unsigned)(n_units < ctas ? n_units : ctas);
    kern<<<grid, W * 32, smem, a.stream>>>(a.op, sc, a.fT, a.vT, a.QT);
    e = cudaGetLastError();
    return {e == cudaSuccess ? 0 : 5, 1, e, PATH_TILE4};
}

// Work-unit schedule shared by the persistent kernels: whole half-tiles while there are more
// half-tiles than CTAs, then the last `ctas` half-tiles split into 4 (or 16) bins each.
struct UnitPlan {
    int n_ht, n_whole, split, n_units;
};
static inline UnitPlan plan_units(int64_t n_cells, int64_t ctas) {
    const int64_t n_ht = (n_cells + kTileCells - 1) / kTileCells;
    const int64_t n_whole = n_ht > ctas ? n_ht - ctas : 0;
    const int64_t rem = n_ht - n_whole;
    const int split = rem * 4 >= ctas ? 4 : 16;
    return {(int)n_ht, (int)n_whole, split, (int)(n_whole + rem * split)};
}

template <int K, int W, bool EXACT, bool JV, bool RG, typename T = double, bool SPLIT = false>
static LaunchResult launch_pair(const LaunchArgs& a) {
    const int M = a.op.n_q * K;
    const size_t smem = pair_smem_bytes<K, T>(M, W, JV, RG);
    if (smem + 256 > a.max_smem || a.counter == nullptr || a.pitems == nullptr) return {-1, 0, cudaSuccess, PATH_PAIR};
    static_assert(!SPLIT || (!EXACT && !JV && !RG && K % 2 == 0), "the split variant is the fast Q form");
    auto kern = af_pair_kernel<K, W, EXACT, JV, RG, T, SPLIT>;
    int per_sm = 0;
    cudaError_t e = resident_ctas((const void*)kern, W * 32, smem, &per_sm);
    if (e != cudaSuccess) return {5, 0, e, PATH_PAIR};
    if (per_sm < 1) return {-1, 0, cudaSuccess, PATH_PAIR};
    const int64_t ctas = (int64_t)per_sm * a.n_sms;
    if ((a.n_cells + kTileCells - 1) / kTileCells * 16 > INT32_MAX) return {2, 0, cudaSuccess, PATH_PAIR};
    const UnitPlan up = plan_units(a.n_cells, ctas);
    PairSched sc{a.pbin_begin, a.pbin_item, a.pitems, up.n_ht, up.n_whole, up.split, up.n_units, a.counter};
    e = cudaMemsetAsync(a.counter, 0, sizeof(int), a.stream);
    if (e != cudaSuccess) return {5, 0, e, PATH_PAIR};
    const unsigned grid = (unsigned)(up.n_units < ctas ? up.n_units : ctas);
    const T* fT;
    const T* vT;
    if constexpr (sizeof(T) == 8) {
        fT = a.fT;
        vT = a.vT;
    } else {
        fT = a.fT32;
        vT = a.vT32;
    }
    kern<<<grid, W * 32, smem, a.stream>>>(a.op, sc, fT, vT, a.QT);
    e = cudaGetLastError();
    return {e == cudaSuccess ? 0 : 5, 1, e, SPLIT ? PATH_PAIR_SPLIT : (RG ? PATH_PAIR_L1 : PATH_PAIR)};
}

// Tile-resident kernel with the K^3 step on the FP64 MMA (K = 8, fast Q form).
template <int W>
static LaunchResult launch_mma(const LaunchArgs& a) {
    const int M = a.op.n_q * kMmaK;
    const size_t smem = mma_smem_bytes(M, W);
    if (smem + 256 > a.max_smem || a.counter == nullptr || a.op.RT == nullptr) return {-1, 0, cudaSuccess, PATH_TILE_MMA};
    auto kern = af_mma_kernel<W>;
    int per_sm = 0;
    cudaError_t e = resident_ctas((const void*)kern, W * 32, smem, &per_sm);
    if (e != cudaSuccess) return {5, 0, e, PATH_TILE_MMA};
    if (per_sm < 1) return {-1, 0, cudaSuccess, PATH_TILE_MMA};
    const int64_t ctas = (int64_t)per_sm * a.n_sms;
    const UnitPlan up = plan_units(a.n_cells, ctas);
    TileSched sc{a.bin_begin, a.bin_q1, up.n_ht, up.n_whole, up.split, up.n_units, a.counter};
    e = cudaMemsetAsync(a.counter, 0, sizeof(int), a.stream);
    if (e != cudaSuccess) return {5, 0, e, PATH_TILE_MMA};
    const unsigned grid = (unsigned)(up.n_units < ctas ? up.n_units : ctas);
    kern<<<grid, W * 32, smem, a.stream>>>(a.op, sc, a.fT, a.QT);
    e = cudaGetLastError();
    return {e == cudaSuccess ? 0 : 5, 1, e, PATH_TILE_MMA};
}

// BF16-split form: the K^3 step on the BF16 tensor cores (K = 8).
template <int W>
static LaunchResult launch_bf16(const LaunchArgs& a) {
    const int M = a.op.n_q * kBfK;
    const size_t smem = bf16_smem_bytes(M, W);
    if (smem + 256 > a.max_smem || a.counter == nullptr || a.op.RTbf == nullptr || a.fT32 == nullptr)
        return {-1, 0, cudaSuccess, PATH_BF16_MMA};
    auto kern = af_bf16_kernel<W>;
    int per_sm = 0;
    cudaError_t e = resident_ctas((const void*)kern, W * 32, smem, &per_sm);
    if (e != cudaSuccess) return {5, 0, e, PATH_BF16_MMA};
    if (per_sm < 1) return {-1, 0, cudaSuccess, PATH_BF16_MMA};
    const int64_t ctas = (int64_t)per_sm * a.n_sms;
    const UnitPlan up = plan_units(a.n_cells, ctas);
    TileSched sc{a.bin_begin, a.bin_q1, up.n_ht, up.n_whole, up.split, up.n_units, a.counter};
    e = cudaMemsetAsync(a.counter, 0, sizeof(int), a.stream);
    if (e != cudaSuccess) return {5, 0, e, PATH_BF16_MMA};
    const unsigned grid = (unsigned)(up.n_units < ctas ? up.n_units : ctas);
    kern<<<grid, W * 32, smem, a.stream>>>(a.op, sc, a.fT32, a.QT);
    e = cudaGetLastError();
    return {e == cudaSuccess ? 0 : 5, 1, e, PATH_BF16_MMA};
}

template <int K, bool EXACT>
static LaunchResult launch_rf(const LaunchArgs& a) {
    const int64_t warps = (int64_t)a.op.n_items * a.n_tiles;
    if (warps == 0) return {0, 0, cudaSuccess, PATH_GATHER};
    const int64_t blocks = (warps + 3) / 4;
    if (blocks > INT32_MAX) return {2, 0, cudaSuccess, PATH_GATHER};
    rf_kernel<K, EXACT><<<(unsigned)blocks, 128, 0, a.stream>>>(a.op, a.fT, a.QT, (int)a.n_tiles);
    const cudaError_t e = cudaGetLastError();
    return {e == cudaSuccess ? 0 : 5, 1, e, PATH_GATHER};
}

// The few-cell kernel with f and Q_in (host arrays a.few_host_f, a.few_host_q) copied into its
// parameter block; Q_out to a.q_cm.  A launch the driver refuses (status -1) leaves the caller to
// take the copy route; the refusal is not sticky.
// A parameter-block launch that the device refuses for its size or resources (cudaErrorInvalidValue,
// cudaErrorLaunchOutOfResources) does not apply, and the caller falls back to the copy route; any
// other launch error is a failure, reported with its CUDA code.
static LaunchResult few_param_status(cudaError_t e) {
    if (e == cudaSuccess) return {0, 1, cudaSuccess, PATH_FEW};
    if (e == cudaErrorInvalidValue || e == cudaErrorLaunchOutOfResources) return {-1, 0, cudaSuccess, PATH_FEW};
    return {5, 0, e, PATH_FEW};
}

template <int K, bool RF, int CAP>
static LaunchResult launch_few_param(const LaunchArgs& a, dim3 grid, size_t smem, size_t need) {
    static_assert(sizeof(FewPayload<CAP>) + sizeof(DevOp) + 16 <= 32764, "parameter block too large");
    auto kern = af_few_param_kernel<K, RF, CAP>;
    if (smem > 48 * 1024) {
        int per_sm = 0;
        const cudaError_t e = resident_ctas((const void*)kern, kFewWarps * 32, smem, &per_sm);
        if (e != cudaSuccess) return {5, 0, e, PATH_FEW};
        if (per_sm < 1) return {-1, 0, cudaSuccess, PATH_FEW};
    }
    FewPayload<CAP> pay;
    const size_t half = need / 2;
    std::memcpy(pay.v, a.few_host_f, half * sizeof(double));
    std::memcpy(pay.v + half, a.few_host_q, half * sizeof(double));
    std::memset(pay.v + need, 0, (CAP - need) * sizeof(double));
    kern<<<grid, kFewWarps * 32, smem, a.stream>>>(a.op, pay, (int)a.n_cells, a.q_cm);
    return few_param_status(cudaGetLastError());
}

// Few-cell kernel on the cell-major arrays: one CTA per (q1 row, cell).  Status -1 where
// it does not apply (more than kFewCells cells, the radial-first form above K = 8, or f of one cell
// larger than the shared memory).
template <int K, bool RF>
static LaunchResult launch_few(const LaunchArgs& a) {
    if constexpr (RF && K > 8) {
        return {-1, 0, cudaSuccess, PATH_FEW};
    } else {
        if (a.n_cells > kFewCells || a.q_cm == nullptr || (a.f_cm == nullptr && a.few_host_f == nullptr))
            return {-1, 0, cudaSuccess, PATH_FEW};
        if (a.op.n_items == 0 || a.n_cells == 0) return {0, 0, cudaSuccess, PATH_FEW};
        const size_t smem = sizeof(double) * (size_t)a.op.n_q * K;
        if (smem + 256 + sizeof(double) * kFewWarps * K > a.max_smem) return {-1, 0, cudaSuccess, PATH_FEW};
        const dim3 grid((unsigned)a.op.n_q, (unsigned)a.n_cells);
        if (a.few_host_f) {
            // f and Q_in ride in the parameter block: the smallest block that holds them
            const size_t need = 2 * (size_t)a.n_cells * a.op.n_q * K;
            if (need <= 512) return launch_few_param<K, RF, 512>(a, grid, smem, need);
            if (need <= 2048) return launch_few_param<K, RF, 2048>(a, grid, smem, need);
            if (need <= (size_t)kFewPayloadMax) return launch_few_param<K, RF, kFewPayloadMax>(a, grid, smem, need);
            return {-1, 0, cudaSuccess, PATH_FEW};
        }
        auto kern = af_few_kernel<K, RF>;
        if (smem > 48 * 1024) {
            int per_sm = 0;
            const cudaError_t e = resident_ctas((const void*)kern, kFewWarps * 32, smem, &per_sm);
            if (e != cudaSuccess) return {5, 0, e, PATH_FEW};
            if (per_sm < 1) return {-1, 0, cudaSuccess, PATH_FEW};
        }
        kern<<<grid, kFewWarps * 32, smem, a.stream>>>(a.op, a.f_cm, a.q_cm);
        const cudaError_t e = cudaGetLastError();
        return {e == cudaSuccess ? 0 : 5, 1, e, PATH_FEW};
    }
}

// The exact form of the few-cell kernel (one CTA per (row, cell)), in place on device arrays or
// with f and Q_in in the parameter block as launch_few does.  Status -1 where it does not apply.
template <int K, int CAP>
static LaunchResult launch_few_exact_param(const LaunchArgs& a, dim3 grid, size_t smem, size_t need) {
    auto kern = af_few_exact_param_kernel<K, CAP>;
    if (smem > 48 * 1024) {
        int per_sm = 0;
        const cudaError_t e = resident_ctas((const void*)kern, kFewWarps * 32, smem, &per_sm);
        if (e != cudaSuccess) return {5, 0, e, PATH_FEW};
        if (per_sm < 1) return {-1, 0, cudaSuccess, PATH_FEW};
    }
    FewPayload<CAP> pay;
    const size_t half = need / 2;
    std::memcpy(pay.v, a.few_host_f, half * sizeof(double));
    std::memcpy(pay.v + half, a.few_host_q, half * sizeof(double));
    std::memset(pay.v + need, 0, (CAP - need) * sizeof(double));
    kern<<<grid, kFewWarps * 32, smem, a.stream>>>(a.op, pay, (int)a.n_cells, a.q_cm);
    return few_param_status(cudaGetLastError());
}

template <int K>
static LaunchResult launch_few_exact(const LaunchArgs& a) {
    {
        if ((a.n_cells > kFewCells && !a.rows) || a.q_cm == nullptr || (a.f_cm == nullptr && a.few_host_f == nullptr))
            return {-1, 0, cudaSuccess, PATH_FEW};
        // the exact J.v has this route only above K = 8, on the two-cell kernel (the batch kernels take
        // it up to K = 8)
        const bool jv = a.what == OP_JV;
        if (jv && (K <= 8 || !a.rows || a.v_cm == nullptr || a.f_cm == nullptr)) return {-1, 0, cudaSuccess, PATH_FEW};
        if (a.n_cells > 65535) return {2, 0, cudaSuccess, PATH_FEW};
        if (a.op.n_items == 0 || a.n_cells == 0) return {0, 0, cudaSuccess, PATH_FEW};
        const size_t smem = sizeof(double) * ((size_t)a.op.n_q * K + kFewWarps * (K * K + K));
        if (smem + 256 > a.max_smem) return {-1, 0, cudaSuccess, PATH_FEW};
        const dim3 grid((unsigned)a.op.n_q, (unsigned)a.n_cells);
        if (a.few_host_f) {
            const size_t need = 2 * (size_t)a.n_cells * a.op.n_q * K;
            if (need <= 512) return launch_few_exact_param<K, 512>(a, grid, smem, need);
            if (need <= 2048) return launch_few_exact_param<K, 2048>(a, grid, smem, need);
            if (need <= (size_t)kFewPayloadMax) return launch_few_exact_param<K, kFewPayloadMax>(a, grid, smem, need);
            return {-1, 0, cudaSuccess, PATH_FEW};
        }
        if constexpr (K > 8) {
            // the batch route above K = 8: two cells per CTA where their f (and v) fit (the same bits)
            if (a.rows) {
                const size_t arrays = jv ? 4 : 2;
                const size_t smem2 =
                    sizeof(double) * (arrays * (size_t)a.op.n_q * K + 2 * kFewWarps * (K * K + K));
                if (smem2 + 256 <= a.max_smem) {
                    auto kern2 = jv ? af_few_exact2_kernel<K, true> : af_few_exact2_kernel<K, false>;
                    int per_sm = 0;
                    const cudaError_t e = resident_ctas((const void*)kern2, kFewWarps * 32, smem2, &per_sm);
                    if (e != cudaSuccess) return {5, 0, e, PATH_FEW};
                    if (per_sm >= 1) {
                        const dim3 grid2((unsigned)a.op.n_q, (unsigned)((a.n_cells + 1) / 2));
                        kern2<<<grid2, kFewWarps * 32, smem2, a.stream>>>(a.op, a.f_cm, jv ? a.v_cm : nullptr, a.q_cm,
                                                                           (long long)a.n_cells);
                        const cudaError_t e2 = cudaGetLastError();
                        return {e2 == cudaSuccess ? 0 : 5, 1, e2, PATH_FEW};
                    }
                }
                if (jv) return {8, 0, cudaSuccess, PATH_FEW};  // f and v of two cells do not fit
            }
        }
        auto kern = af_few_exact_kernel<K>;
        if (smem > 48 * 1024) {
            int per_sm = 0;
            const cudaError_t e = resident_ctas((const void*)kern, kFewWarps * 32, smem, &per_sm);
            if (e != cudaSuccess) return {5, 0, e, PATH_FEW};
            if (per_sm < 1) return {-1, 0, cudaSuccess, PATH_FEW};
        }
        kern<<<grid, kFewWarps * 32, smem, a.stream>>>(a.op, a.f_cm, a.q_cm);
        const cudaError_t e = cudaGetLastError();
        return {e == cudaSuccess ? 0 : 5, 1, e, PATH_FEW};
    }
}

// Warps per CTA of the tile kernel (registers: 16 warps leave 128 per thread).
constexpr int tile_W(int K, bool jv) { return jv ? (K >= 8 ? 12 : 16) : 16; }

template <int K>
static LaunchResult launch_for_k(const LaunchArgs& a) {
    if (a.few) {
        if (a.f32 || a.bf16 || (a.what == OP_JV && !(a.exact && a.rows))) return {-1, 0, cudaSuccess, PATH_FEW};
        if (a.exact)
            return a.what == OP_AF || a.what == OP_JV ? launch_few_exact<K>(a) : LaunchResult{-1, 0, cudaSuccess, PATH_FEW};
        return a.what == OP_RF ? launch_few<K, true>(a) : launch_few<K, false>(a);
    }
    if (a.ss) {
        if (a.what != OP_AF || a.exact || a.f32) return {8, 0, cudaSuccess, PATH_TILE};
        if constexpr (K % 2 == 0 && K <= 8) {
            const LaunchResult r = launch_tile_stream<K, tile_W(K, false)>(a);
            if (r.status == -1) return {8, 0, cudaSuccess, PATH_TILE};
            return r;
        } else {
            return {8, 0, cudaSuccess, PATH_TILE};
        }
    }
    if (a.bf16) {
        if (a.what != OP_AF || a.exact) return {8, 0, cudaSuccess, PATH_BF16_MMA};
        if constexpr (K == kBfK) {
            const LaunchResult r = launch_bf16<16>(a);
            if (r.status == -1) return {8, 0, cudaSuccess, PATH_BF16_MMA};
            return r;
        } else {
            return {8, 0, cudaSuccess, PATH_BF16_MMA};
        }
    }
    if (a.f32) {
        // FP32 form: the pair kernel in FP32 (angular first only), R staged in shared memory when the
        // FP32 tile leaves room for it, else read through L1
        if constexpr (K % 2 == 0 && K <= 12) {
            if ((a.what != OP_AF && a.what != OP_JV) || a.exact) return {8, 0, cudaSuccess, PATH_PAIR};
            LaunchResult r{-1, 0, cudaSuccess, PATH_PAIR};
            if (a.what == OP_JV) {
                // FP32 J.v: Phi = sum G (f (x) v + v (x) f) in FP32 on the pair kernel
                if (a.vT32 == nullptr) return {8, 0, cudaSuccess, PATH_PAIR};
                r = launch_pair<K, 8, false, true, false, float>(a);
                if (r.status == -1) r = launch_pair<K, 8, false, true, true, float>(a);
                if (r.status == -1) return {8, 0, cudaSuccess, PATH_PAIR};
                return r;
            }
            if constexpr (K <= 8)
                if (a.path == PATH_PAIR_SPLIT) r = launch_pair<K, 8, false, false, false, float, true>(a);
            if (r.status == -1) r = launch_pair<K, 8, false, false, false, float>(a);
            if (r.status == -1) r = launch_pair<K, 8, false, false, true, float>(a);
            if (r.status == -1) return {8, 0, cudaSuccess, PATH_PAIR};
            return r;
        } else {
            return {8, 0, cudaSuccess, PATH_PAIR};
        }
    }
    if (a.what == OP_RF) return a.exact ? launch_rf<K, true>(a) : launch_rf<K, false>(a);
    const bool jv = a.what == OP_JV;
    if (a.path == PATH_TILE_MMA) {
        if constexpr (K == kMmaK) {
            if (!jv && !a.exact) {
                const LaunchResult r = launch_mma<16>(a);
                if (r.status != -1) return r;
            }
        }
        // the MMA kernel is the fast Q form at K = 8: anything else runs as PATH_TILE
        LaunchArgs b = a;
        b.path = PATH_TILE;
        return launch_for_k<K>(b);
    }
    if constexpr (K % 2 == 0 && K <= 8) {
        if (a.path == PATH_AUTO && a.tile_first && !a.exact) {
            const LaunchResult r = jv ? launch_tile<K, tile_W(K, true), false, true>(a)
                                      : launch_tile<K, tile_W(K, false), false, false>(a);
            if (r.status != -1) return r;
        }
    }
    if constexpr (K <= 8 && K % 2 == 0) {
        if (a.path == PATH_PAIR_SPLIT && !jv && !a.exact) {
            const LaunchResult r = launch_pair<K, 8, false, false, false, double, true>(a);
            if (r.status != -1) return r;
        }
    }
    // PATH_PAIR_SPLIT: the split variant where it applies (fast Q form, K even), else the pair kernel
    if constexpr (K <= 8) {
        if (a.path == PATH_AUTO || a.path == PATH_PAIR || a.path == PATH_PAIR_L1 || a.path == PATH_PAIR_SPLIT) {
            LaunchResult r;
            if (a.path == PATH_PAIR_L1) {
                if (jv)
                    r = a.exact ? launch_pair<K, 8, true, true, true>(a) : launch_pair<K, 8, false, true, true>(a);
                else
                    r = a.exact ? launch_pair<K, 8, true, false, true>(a) : launch_pair<K, 8, false, false, true>(a);
            } else {
                if (jv)
                    r = a.exact ? launch_pair<K, 8, true, true, false>(a) : launch_pair<K, 8, false, true, false>(a);
                else
                    r = a.exact ? launch_pair<K, 8, true, false, false>(a) : launch_pair<K, 8, false, false, false>(a);
            }
            if (r.status != -1) return r;
            if (a.path != PATH_AUTO) return {8, 0, cudaSuccess, a.path};
        }
    } else {
        if (a.path == PATH_PAIR || a.path == PATH_PAIR_L1 || a.path == PATH_PAIR_SPLIT) return {8, 0, cudaSuccess, a.path};
    }
    if constexpr (K % 2 == 0 && K <= 8) {
        if (a.path == PATH_AUTO || a.path == PATH_TILE) {
            LaunchResult r;
            if (jv)
                r = a.exact ? launch_tile<K, tile_W(K, true), true, true>(a)
                            : launch_tile<K, tile_W(K, true), false, true>(a);
            else
                r = a.exact ? launch_tile<K, tile_W(K, false), true, false>(a)
                            : launch_tile<K, tile_W(K, false), false, false>(a);
            if (r.status != -1) return r;
            if (a.path == PATH_TILE) return {8, 0, cudaSuccess, PATH_TILE};
        }
    } else {
        if (a.path == PATH_TILE) return {8, 0, cudaSuccess, PATH_TILE};
    }
    // the 16-cell tile (and the pair kernel) did not fit: 8-cell quarter tiles before the gather kernel
    if constexpr (K % 4 == 0 && K <= 8) {
        if (a.path == PATH_AUTO && !a.exact && !a.f32) {
            const LaunchResult r = jv ? launch_tile4<K, 16, true>(a) : launch_tile4<K, 16, false>(a);
            if (r.status != -1) return r;
        }
    }
    if constexpr (K <= 8) {
        if (a.exact)
            return jv ? launch_af<K, 1, true, true>(a) : launch_af<K, 1, true, false>(a);
    } else {
        if (a.exact) return {8, 0, cudaSuccess, PATH_GATHER};
    }
    return jv ? launch_af<K, jv_P(K), false, true>(a) : launch_af<K, af_P(K), false, false>(a);
}

}  // namespace cf

#define CF_CAT2(a, b) a##b
#define CF_CAT(a, b) CF_CAT2(a, b)
namespace cf {
LaunchResult CF_CAT(launch_k, CF_K)(const LaunchArgs& a) { return launch_for_k<CF_K>(a); }
}  // namespace cf
