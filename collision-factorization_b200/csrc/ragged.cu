// ragged.cu -- one persistent launch over cells of several resolutions (L, K).
//
// A ragged batch is a set of buckets, each a plan (one (L, K) operator) with its own cells and its
// own form.  Buckets in the angular-first forms CF_FORM_AF / CF_FORM_AF_SYM with K <= 8 are "fused":
// one kernel runs the pair or tile routine of the plans for all of them in a single launch.  The work
// units of the fused buckets -- whole 16-cell half-tiles first, heaviest buckets first, then the last
// half-tiles split into 4 or 16 q1-pair bins (or not split) -- sit in one table that persistent CTAs
// drain through a device counter; a unit names its bucket, and the CTA stages that bucket's tile and
// switches to the routine compiled for the bucket's K: the pair routine (8 warps per CTA) or the
// tile routine (16 warps, even K only), chosen per batch.  Shared memory and registers are sized
// for the largest fused bucket.  Any other bucket (radial-first, the exact forms, K > 8) runs its
// own plan's kernels on its tiled buffers in the same step.
//
// Each step is: pack every bucket's cells into its tiled buffer, the fused launch, the separate
// buckets, unpack.  The sequence has no host synchronisation and no allocation, so it is recorded
// once into a CUDA graph (cf_ragged_graph_launch) and replayed per time step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/cf_b200.h"
#include "common.cuh"
#include "layout.cuh"
#include "pair_kernels.cuh"

void cf_set_last_error(const char* msg);
int cf_plan_internal_view(const cf_plan* plan, DevOp* op, const int** pbin_begin, const int** pbin_item,
                          const int2** pitems, const int** bin_begin, const int** bin_q1, int* n_sms,
                          size_t* max_smem);
int cf_plan_folded(cf_plan* plan, cf_plan** folded);
void cf_add_launches(int64_t n);

namespace {

constexpr int kRW = 8;                  // warps per CTA, pair routine
constexpr int kTW = 16;                 // warps per CTA, tile routine
constexpr int kMaxK = 8;                // fused buckets have K <= 8 (FP64 pair / tile routines)
constexpr int kRBufPair = kMaxK * kMaxK * kMaxK;
constexpr int kRBufTile = cf::RBuf<kMaxK>::SIZE;

struct Bucket {
    DevOp op;
    const int* pbin_begin;  // pair routine: bins over mirrored-row items
    const int* pbin_item;
    const int2* pitems;
    const int* bin_begin;   // tile routine: bins over q1 rows
    const int* bin_q1;
    const double* fT;
    double* QT;
    int K, M;
    // host entry point (cf_ragged_q_host): the bucket's cell-major device copies and its chunks
    const double* f_cm;
    double* q_cm;
    long long cells;
};

struct Unit {
    int bucket, ht, bin;
    int chunk;  // the streamed host call's upload chunk holding the half-tile (0 elsewhere)
};

// TILE = false: the pair routine (8 warps, one mirrored row pair per warp, whole Phi per lane);
// TILE = true: the tile routine (16 warps, one q1 row per warp, Phi split over two lanes per cell;
// even K only).  Both are the routines the buckets' own plans run, so a bucket's result is the same
// bit for bit as its plan's pair or tile kernel.
template <bool TILE>
__global__ void __launch_bounds__((TILE ? kTW : kRW) * 32, 1)
    af_ragged_kernel(const Bucket* __restrict__ buckets, const Unit* __restrict__ units, int n_units,
                     int* __restrict__ counter) {
    constexpr int W = TILE ? kTW : kRW;
    constexpr int RBS = TILE ? kRBufTile : kRBufPair;
    extern __shared__ __align__(16) double smem[];
    __shared__ int s_unit, s_next;
    __shared__ Bucket s_bk;  // the current unit's bucket (uniform shared loads inside the routines)
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    double* fs = smem + W * RBS;
    double* rb = smem + warp * RBS;
    int staged_b = -1, staged_ht = -1;
    for (;;) {
        if (tid == 0) {
            const int uu = atomicAdd(counter, 1);
            s_unit = uu;
            if (uu < n_units) s_bk = buckets[units[uu].bucket];
        }
        __syncthreads();
        const int u = s_unit;
        if (u >= n_units) break;
        const Unit un = units[u];
        const Bucket& bk = s_bk;
        const int M = bk.M;
        const size_t tile_base = (size_t)(un.ht >> 1) * M * CF_TILE + (size_t)(un.ht & 1) * cf::kTileCells;
        if (un.bucket != staged_b || un.ht != staged_ht) {
            const double* srcf = bk.fT + tile_base;
            for (int i = tid; i < M * 8; i += W * 32) {
                const int r = i >> 3, w = (i & 7) * 2;
                cf::cp_async16(fs + r * cf::kTileCells + w, srcf + (size_t)r * CF_TILE + w);
            }
            cf::cp_async_commit();
            cf::cp_async_wait_all();
            staged_b = un.bucket;
            staged_ht = un.ht;
        }
        if (tid == 0) s_next = 0;
        __syncthreads();
        const int* bb = TILE ? bk.bin_begin : bk.pbin_begin;
        const int b0 = bb[un.bin], nb = bb[un.bin + 1] - b0;
        double* qtc = bk.QT + tile_base + (lane & 15);
        for (;;) {
            int i = 0;
            if (lane == 0) i = atomicAdd(&s_next, 1);
            i = __shfl_sync(0xffffffffu, i, 0);
            if (i >= nb) break;
            if constexpr (TILE) {
                const int q1 = bk.bin_q1[b0 + i];
                switch (bk.K) {
                    case 2: cf::tile_q1<2, false, false>(bk.op, q1, fs, nullptr, rb, qtc, lane); break;
                    case 4: cf::tile_q1<4, false, false>(bk.op, q1, fs, nullptr, rb, qtc, lane); break;
                    case 6: cf::tile_q1<6, false, false>(bk.op, q1, fs, nullptr, rb, qtc, lane); break;
                    case 8: cf::tile_q1<8, false, false>(bk.op, q1, fs, nullptr, rb, qtc, lane); break;
                    default: break;
                }
            } else {
                const int2 item = bk.pitems[bk.pbin_item[b0 + i]];
                switch (bk.K) {
                    case 1: cf::pair_item<1, false, false, false, double>(bk.op, item, fs, nullptr, rb, qtc, lane); break;
                    case 2: cf::pair_item<2, false, false, false, double>(bk.op, item, fs, nullptr, rb, qtc, lane); break;
                    case 3: cf::pair_item<3, false, false, false, double>(bk.op, item, fs, nullptr, rb, qtc, lane); break;
                    case 4: cf::pair_item<4, false, false, false, double>(bk.op, item, fs, nullptr, rb, qtc, lane); break;
                    case 5: cf::pair_item<5, false, false, false, double>(bk.op, item, fs, nullptr, rb, qtc, lane); break;
                    case 6: cf::pair_item<6, false, false, false, double>(bk.op, item, fs, nullptr, rb, qtc, lane); break;
                    case 7: cf::pair_item<7, false, false, false, double>(bk.op, item, fs, nullptr, rb, qtc, lane); break;
                    case 8: cf::pair_item<8, false, false, false, double>(bk.op, item, fs, nullptr, rb, qtc, lane); break;
                    default: break;
                }
            }
        }
        __syncthreads();
    }
}

// The callers' cell-major arrays of a resident launch (cf_ragged_q / cf_ragged_graph_launch), by bucket.
struct CmPtrs {
    const double* f[64];
    double* q[64];
};

// Words of the streamed launch of cf_ragged_q_host (per upload chunk; see af_ragged_stream_kernel).
struct RaggedSync {
    const int* ready;        // [n_chunks] device; == epoch once the chunk's f and Q are in
    int* done;               // [n_chunks] device; units finished (zeroed before the launch)
    const int* chunk_units;  // [n_chunks] device; units of the work table that read the chunk
    int* host_done;          // [n_chunks] mapped host memory; set to epoch once the chunk is final
    int* err;                // mapped host memory; set to 1 if a wait gave up
    int* abort;              // device; == epoch once a wait gave up
    int epoch;
    long long wait_cycles;
};

// The tile routine of af_ragged_kernel over the buckets' cell-major arrays while they are being
// copied in and out (cf_ragged_q_host).  Its work table holds the buckets' half-tiles heaviest
// bucket first, each cut into 4 q1 bins, and the host uploads every bucket in chunks of whole
// half-tiles in that order, each chunk followed by a 4-byte copy that sets its ready word.  A CTA waits (bounded by wait_cycles of the SM clock; past that it records err and
// abort, and later waits return at once) for the chunk of its unit, stages the half-tile from the
// cell-major rows and contracts its rows with the same per-row code as af_ragged_kernel, reading Q_in
// at each row's start and writing Q in place, so a bucket's result equals the resident step's bit
// for bit.  The CTA that finishes a chunk's last unit fences at system scope and writes the epoch
// into the chunk's mapped host word; the host then queues that chunk's download.
//
// Resident (rs.ready null; the device steps): the same routine on the callers' cell-major arrays in
// `ptrs`, with the handle's own work table, no waits and no chunk words -- the whole step in one
// launch, without layout passes.
__global__ void __launch_bounds__(kTW * 32, 1)
    af_ragged_stream_kernel(const Bucket* __restrict__ buckets, const Unit* __restrict__ units, int n_units,
                            int* __restrict__ counter, RaggedSync rs, CmPtrs ptrs) {
    constexpr int W = kTW;
    extern __shared__ __align__(16) double smem[];
    __shared__ int s_unit, s_next;
    __shared__ Bucket s_bk;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    double* fs = smem + W * kRBufTile;
    double* rb = smem + warp * kRBufTile;
    int staged_b = -1, staged_ht = -1;
    for (;;) {
        if (tid == 0) {
            const int uu = atomicAdd(counter, 1);
            s_unit = uu;
            if (uu < n_units) s_bk = buckets[units[uu].bucket];
        }
        __syncthreads();
        const int u = s_unit;
        if (u >= n_units) break;
        const Unit un = units[u];
        const Bucket& bk = s_bk;
        const int M = bk.M, NQ = bk.op.n_q, K = bk.K;
        const int chunk = un.chunk;
        const long long cell0 = (long long)un.ht * cf::kTileCells;
        const double* fb = rs.ready ? bk.f_cm : ptrs.f[un.bucket];
        double* qb = rs.ready ? bk.q_cm : ptrs.q[un.bucket];
        if (un.bucket != staged_b || un.ht != staged_ht) {
            if (tid == 0 && rs.ready) {
                const long long t0 = clock64();
                while (cf::ld_acquire(rs.ready + chunk) != rs.epoch) {
                    if (*reinterpret_cast<volatile int*>(rs.abort) == rs.epoch) break;
                    if (clock64() - t0 > rs.wait_cycles) {
                        *reinterpret_cast<volatile int*>(rs.abort) = rs.epoch;
                        *reinterpret_cast<volatile int*>(rs.err) = 1;
                        break;
                    }
                    __nanosleep(256);
                }
            }
            __syncthreads();
            // element j = q + N_Q k of cell c goes to row q K + k of the tile
            for (int i = tid; i < M * cf::kTileCells; i += W * 32) {
                const int c = i & 15, j = i >> 4;
                const int r = (j % NQ) * K + j / NQ;
                if (cell0 + c < bk.cells)
                    cf::cp_async8(fs + r * cf::kTileCells + c, fb + (size_t)(cell0 + c) * M + j);
                else
                    fs[r * cf::kTileCells + c] = 0.0;
            }
            cf::cp_async_commit();
            cf::cp_async_wait_all();
            staged_b = un.bucket;
            staged_ht = un.ht;
        }
        if (tid == 0) s_next = 0;
        __syncthreads();
        const int b0 = bk.bin_begin[un.bin], nb = bk.bin_begin[un.bin + 1] - b0;
        const long long cell = cell0 + (lane & 15);
        const bool live = cell < bk.cells;
        double* qc = qb + (size_t)(live ? cell : 0) * M;
        for (;;) {
            int i = 0;
            if (lane == 0) i = atomicAdd(&s_next, 1);
            i = __shfl_sync(0xffffffffu, i, 0);
            if (i >= nb) break;
            const int q1 = bk.bin_q1[b0 + i];
            switch (K) {
                case 2: cf::tile_q1<2, false, false, true>(bk.op, q1, fs, nullptr, rb, qc, lane, live); break;
                case 4: cf::tile_q1<4, false, false, true>(bk.op, q1, fs, nullptr, rb, qc, lane, live); break;
                case 6: cf::tile_q1<6, false, false, true>(bk.op, q1, fs, nullptr, rb, qc, lane, live); break;
                case 8: cf::tile_q1<8, false, false, true>(bk.op, q1, fs, nullptr, rb, qc, lane, live); break;
                default: break;
            }
        }
        if (rs.done) __threadfence();
        __syncthreads();
        if (tid == 0 && rs.done && atomicAdd(rs.done + chunk, 1) == rs.chunk_units[chunk] - 1) {
            __threadfence_system();
            *reinterpret_cast<volatile int*>(rs.host_done + chunk) = rs.epoch;
        }
    }
}

#define RCHECK(expr)                                                                                    \
    do {                                                                                                \
        cudaError_t e_ = (expr);                                                                        \
        if (e_ != cudaSuccess) {                                                                        \
            char m_[256];                                                                               \
            snprintf(m_, sizeof(m_), "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
            cf_set_last_error(m_);                                                                      \
            return e_ == cudaErrorMemoryAllocation ? CF_ENOMEM : CF_ECUDA;                              \
        }                                                                                               \
    } while (0)

}  // namespace

struct cf_ragged {
    int device = 0;
    int n_buckets = 0;
    std::vector<cf_plan*> plans;
    std::vector<int64_t> cells;
    std::vector<int> K, NQ;
    std::vector<int> form;     // per bucket: the form it is contracted in
    std::vector<char> fused;   // per bucket: part of the fused launch
    std::vector<double> cost;  // relative cost of one half-tile of each bucket
    int tail_split = 4;
    int family = 0;  // 0: pair routine, 1: tile routine
    Bucket* d_buckets = nullptr;
    Unit* d_units = nullptr;
    int* d_counter = nullptr;
    double* d_tiles = nullptr;  // per bucket: tiled f, tiled Q
    std::vector<size_t> tile_off;
    int n_units = 0, ctas = 0;
    size_t smem = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int64_t step_kernels = 0;  // layout passes and fused launch of the last step enqueued
    // every non-empty bucket fused on the tile routine: a device step is one resident launch of
    // af_ragged_stream_kernel on the callers' cell-major arrays (the last ones kept for
    // cf_ragged_q_resident)
    bool cell_major = false;
    CmPtrs last_ptrs{};
    bool have_last = false;
    std::vector<const double*> graph_f;
    std::vector<double*> graph_q;
    cudaStream_t graph_stream = nullptr;
    // host entry point (cf_ragged_q_host), set up on its first call: cell-major device copies of
    // every bucket's f and Q; for the streamed launch, the upload chunks and their words
    std::vector<Unit> h_units;
    std::vector<Bucket> h_buckets;
    bool host_ready = false, host_stream = false;
    double* d_io = nullptr;
    std::vector<size_t> io_off;
    std::vector<int> chunk_bucket, chunk_ht0, chunk_ht1;  // upload order = the work table's order
    Unit* d_xunits = nullptr;  // the streamed launch's work table: every half-tile in 4 q1 bins
    int n_xunits = 0;
    cudaStream_t xs[3] = {};
    int* d_xsync = nullptr;   // ready[kHostChunks], done[kHostChunks], chunk_units[kHostChunks], abort
    int* h_xepoch = nullptr;  // pinned: the epoch values the ready copies read
    int* h_xsync = nullptr;   // mapped: chunk completion words [kHostChunks], then the error word
    int* h_xsync_dev = nullptr;
    int xepoch = 0;
    long long xwait = 0;
    std::mutex mu;
};

namespace {

int64_t ntiles(int64_t B) { return (B + CF_TILE - 1) / CF_TILE; }

constexpr int kHostChunks = 128;            // upload chunks of the streamed host call, at most
// Upload chunks by bytes (f and Q_in of whole half-tiles): the first ones small, so that the kernel
// starts early, growing to kChunkMaxBytes, and small again over the last 2 kChunkMaxBytes, so that
// the last contraction and download are short.  Every copy costs a few microseconds of copy-engine
// time beyond its bytes, so the chunks are as large as the ramp allows.
constexpr size_t kChunkFirstBytes = size_t(2) << 20;
constexpr size_t kChunkMaxBytes = size_t(8) << 20;

using StreamWriteValue32 = int (*)(cudaStream_t, unsigned long long, unsigned int, unsigned int);

// cuStreamWriteValue32 through the runtime's driver entry point (no link to the driver library), or
// null where it is not available: the streamed host call then sets its ready words by 4-byte copies.
StreamWriteValue32 stream_write_value32() {
    static StreamWriteValue32 fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuStreamWriteValue32", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (StreamWriteValue32) nullptr;
        }
        return reinterpret_cast<StreamWriteValue32>(f);
    }();
    return fn;
}
constexpr double kHostWaitSeconds = 5.0;     // a CTA gives up on a chunk's ready word after this

void free_ragged(cf_ragged* r) {
    if (r->graph_exec) cudaGraphExecDestroy(r->graph_exec);
    if (r->graph) cudaGraphDestroy(r->graph);
    cudaFree(r->d_buckets);
    cudaFree(r->d_units);
    cudaFree(r->d_counter);
    cudaFree(r->d_tiles);
    cudaFree(r->d_io);
    cudaFree(r->d_xunits);
    cudaFree(r->d_xsync);
    if (r->h_xepoch) cudaFreeHost(r->h_xepoch);
    if (r->h_xsync) cudaFreeHost(r->h_xsync);
    for (cudaStream_t& s : r->xs)
        if (s) cudaStreamDestroy(s);
}

double* tiled_f(cf_ragged* r, int b) { return r->d_tiles + r->tile_off[b]; }
double* tiled_q(cf_ragged* r, int b) {
    return r->d_tiles + r->tile_off[b] + (size_t)ntiles(r->cells[b]) * CF_TILE * r->NQ[b] * r->K[b];
}

// the contraction on the handle's tiled buffers: the fused launch, then the separate buckets (whose
// plans count their own kernels)
int enqueue_contract(cf_ragged* r, cudaStream_t s, bool count = true) {
    if (r->n_units > 0) {
        if (count) cf_add_launches(1);
        RCHECK(cudaMemsetAsync(r->d_counter, 0, sizeof(int), s));
        const unsigned grid = (unsigned)std::min(r->n_units, r->ctas);
        if (r->family == 1)
            af_ragged_kernel<true><<<grid, kTW * 32, r->smem, s>>>(r->d_buckets, r->d_units, r->n_units, r->d_counter);
        else
            af_ragged_kernel<false><<<grid, kRW * 32, r->smem, s>>>(r->d_buckets, r->d_units, r->n_units, r->d_counter);
        RCHECK(cudaGetLastError());
    }
    for (int b = 0; b < r->n_buckets; ++b) {
        if (r->fused[b] || r->cells[b] == 0) continue;
        const int st = cf_q_tiled(r->plans[b], tiled_q(r, b), tiled_f(r, b), r->cells[b], r->form[b], s);
        if (st != CF_OK) return st;
    }
    return CF_OK;
}

// pack every bucket, the contraction, unpack (q += Q(f) per bucket), all on stream s; count: add the
// step's kernels to the launch counter now (false while recording a graph: each replay adds them)
int enqueue_resident_cm(cf_ragged* r, cudaStream_t s, bool count) {
    RCHECK(cudaMemsetAsync(r->d_counter, 0, sizeof(int), s));
    const RaggedSync none{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0, 0};
    const unsigned grid = (unsigned)std::min(r->n_units, r->ctas);
    af_ragged_stream_kernel<<<grid, kTW * 32, r->smem, s>>>(r->d_buckets, r->d_units, r->n_units, r->d_counter,
                                                            none, r->last_ptrs);
    RCHECK(cudaGetLastError());
    if (count) cf_add_launches(1);
    return CF_OK;
}

int enqueue_step(cf_ragged* r, double* const* q, const double* const* f, cudaStream_t s, bool count = true) {
    if (r->cell_major) {
        for (int b = 0; b < r->n_buckets; ++b) {
            r->last_ptrs.f[b] = f[b];
            r->last_ptrs.q[b] = q[b];
        }
        r->have_last = true;
        r->step_kernels = 1;
        return enqueue_resident_cm(r, s, count);
    }
    int64_t nk = r->n_units > 0 ? 1 : 0;
    for (int b = 0; b < r->n_buckets; ++b) nk += r->cells[b] > 0 ? 3 : 0;
    r->step_kernels = nk;
    if (count) cf_add_launches(nk - (r->n_units > 0 ? 1 : 0));
    for (int b = 0; b < r->n_buckets; ++b) {
        if (r->cells[b] == 0) continue;
        const int M = r->NQ[b] * r->K[b];
        dim3 grid((M + 31) / 32, (unsigned)ntiles(r->cells[b])), block(32, 8);
        cf::pack_tiles_kernel<double><<<grid, block, 0, s>>>(f[b], tiled_f(r, b), r->cells[b], r->NQ[b], r->K[b]);
        cf::pack_tiles_kernel<double><<<grid, block, 0, s>>>(q[b], tiled_q(r, b), r->cells[b], r->NQ[b], r->K[b]);
    }
    RCHECK(cudaGetLastError());
    const int st = enqueue_contract(r, s, count);
    if (st != CF_OK) return st;
    for (int b = 0; b < r->n_buckets; ++b) {
        if (r->cells[b] == 0) continue;
        const int M = r->NQ[b] * r->K[b];
        dim3 grid((M + 31) / 32, (unsigned)ntiles(r->cells[b])), block(32, 8);
        cf::unpack_tiles_kernel<<<grid, block, 0, s>>>(tiled_q(r, b), q[b], r->cells[b], r->NQ[b], r->K[b]);
    }
    RCHECK(cudaGetLastError());
    return CF_OK;
}

// First host call: cell-major device copies of every bucket's f and Q; and, when every non-empty
// bucket runs in the fused launch on the tile routine, the streamed launch's work table, its upload
// chunks (whole half-tiles, about kTargetChunks, in the table's order) and their words.
int host_setup(cf_ragged* r) {
    if (r->host_ready) return CF_OK;
    size_t total = 0;
    r->io_off.clear();
    for (int b = 0; b < r->n_buckets; ++b) {
        r->io_off.push_back(total);
        total += 2 * (size_t)r->cells[b] * r->NQ[b] * r->K[b];
    }
    if (!r->d_io) RCHECK(cudaMalloc(&r->d_io, std::max<size_t>(total, 1) * sizeof(double)));
    for (cudaStream_t& s : r->xs)
        if (!s) RCHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    bool stream = r->family == 1 && r->n_units > 0;
    for (int b = 0; b < r->n_buckets; ++b)
        if (r->cells[b] > 0 && !r->fused[b]) stream = false;
    if (stream) {
        // buckets in the order the work table first names them; the table runs over each bucket's
        // half-tiles in ascending order, so chunks uploaded in this order arrive in the order the
        // CTAs take them
        std::vector<int> order;
        std::vector<char> seen(r->n_buckets, 0);
        for (const Unit& u : r->h_units)
            if (!seen[u.bucket]) {
                seen[u.bucket] = 1;
                order.push_back(u.bucket);
            }
        // chunks of whole half-tiles within one bucket, sized by bytes (f and Q_in): ramped up from
        // kChunkFirstBytes to kChunkMaxBytes and down again at the end
        size_t remaining = 0;
        for (int b : order) remaining += (size_t)r->cells[b] * r->NQ[b] * r->K[b] * 2 * sizeof(double);
        size_t first = kChunkFirstBytes, maxb = kChunkMaxBytes;
        for (;;) {
            // the largest count the ramp can produce: every chunk at least `first`, plus one per bucket
            if (remaining / first + (size_t)order.size() + 1 <= (size_t)kHostChunks) break;
            first *= 2;
            maxb = std::max(maxb, first);
        }
        r->chunk_bucket.clear();
        r->chunk_ht0.clear();
        r->chunk_ht1.clear();
        std::vector<int> first_chunk(r->n_buckets, 0);
        for (int b : order) {
            const int n_ht = (int)((r->cells[b] + 15) / 16);
            const size_t ht_bytes = (size_t)16 * r->NQ[b] * r->K[b] * 2 * sizeof(double);
            first_chunk[b] = (int)r->chunk_bucket.size();
            for (int h = 0; h < n_ht;) {
                const int i = (int)r->chunk_bucket.size();
                size_t target = std::min(maxb, first << std::min(i, 16));
                if (remaining < 2 * maxb) target = std::min(target, std::max(first, remaining / 2));
                int n = (int)std::max<size_t>(1, target / ht_bytes);
                n = std::min(n, n_ht - h);
                // no sliver of a chunk at the end of a bucket
                if (n_ht - h - n > 0 && (size_t)(n_ht - h - n) * ht_bytes < first / 2) n = n_ht - h;
                r->chunk_bucket.push_back(b);
                r->chunk_ht0.push_back(h);
                r->chunk_ht1.push_back(h + n);
                remaining -= std::min(remaining, (size_t)n * ht_bytes);
                h += n;
            }
        }
        const int n_chunks = (int)r->chunk_bucket.size();
        if (n_chunks > kHostChunks) {
            cf_set_last_error("cf_ragged_q_host: too many upload chunks");
            return CF_EINVAL;
        }
        // the streamed work table: the buckets' half-tiles in the upload order, each in 4 q1 bins, so
        // that the first chunk already feeds every SM and results complete (and go back) steadily
        std::vector<Unit> xunits;
        for (int c = 0; c < n_chunks; ++c)
            for (int h = r->chunk_ht0[c]; h < r->chunk_ht1[c]; ++h)
                for (int k = 0; k < 4; ++k) xunits.push_back({r->chunk_bucket[c], h, 1 + k, c});
        r->n_xunits = (int)xunits.size();
        if (!r->d_xunits) RCHECK(cudaMalloc(&r->d_xunits, std::max<size_t>(xunits.size(), 1) * sizeof(Unit)));
        RCHECK(cudaMemcpy(r->d_xunits, xunits.data(), xunits.size() * sizeof(Unit), cudaMemcpyHostToDevice));
        std::vector<int> chunk_units(kHostChunks, 0);
        for (const Unit& u : xunits) chunk_units[u.chunk]++;
        if (!r->d_xsync) RCHECK(cudaMalloc(&r->d_xsync, (3 * kHostChunks + 1) * sizeof(int)));
        RCHECK(cudaMemset(r->d_xsync, 0, (3 * kHostChunks + 1) * sizeof(int)));
        RCHECK(cudaMemcpy(r->d_xsync + 2 * kHostChunks, chunk_units.data(), kHostChunks * sizeof(int),
                          cudaMemcpyHostToDevice));
        if (!r->h_xepoch) RCHECK(cudaHostAlloc((void**)&r->h_xepoch, kHostChunks * sizeof(int), cudaHostAllocDefault));
        if (!r->h_xsync) RCHECK(cudaHostAlloc((void**)&r->h_xsync, (kHostChunks + 1) * sizeof(int), cudaHostAllocMapped));
        RCHECK(cudaHostGetDevicePointer((void**)&r->h_xsync_dev, r->h_xsync, 0));
        int khz = 0;
        RCHECK(cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, r->device));
        r->xwait = (long long)((double)std::max(khz, 1000000) * 1e3 * kHostWaitSeconds);
        RCHECK(cudaFuncSetAttribute(af_ragged_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)r->smem));
    }
    for (int b = 0; b < r->n_buckets; ++b) {
        r->h_buckets[b].f_cm = r->d_io + r->io_off[b];
        r->h_buckets[b].q_cm = r->d_io + r->io_off[b] + (size_t)r->cells[b] * r->NQ[b] * r->K[b];
    }
    RCHECK(cudaMemcpy(r->d_buckets, r->h_buckets.data(), r->n_buckets * sizeof(Bucket), cudaMemcpyHostToDevice));
    r->host_stream = stream;
    r->host_ready = true;
    return CF_OK;
}

// q_host[b] += Q(f_host[b]) through the streamed launch (see af_ragged_stream_kernel).  Every upload
// is queued before the launch, so the copies stay ahead of the kernel even where the copy and kernel
// streams share a hardware queue; the host polls the chunks' completion words only while the kernel
// runs, and the kernel's own waits are bounded, so the call always ends.
int host_streamed(cf_ragged* r, double* const* q_host, const double* const* f_host) {
    const int n_chunks = (int)r->chunk_bucket.size();
    r->xepoch = r->xepoch % 0x3fffffff + 1;
    const int epoch = r->xepoch;
    volatile int* hs = r->h_xsync;
    for (int c = 0; c < n_chunks; ++c) {
        r->h_xepoch[c] = epoch;
        hs[c] = 0;
    }
    hs[kHostChunks] = 0;
    cudaStream_t s_in = r->xs[0], s_k = r->xs[1], s_out = r->xs[2];
    int* d_ready = r->d_xsync;
    int* d_done = r->d_xsync + kHostChunks;
    const int* d_units = r->d_xsync + 2 * kHostChunks;
    int* d_abort = r->d_xsync + 3 * kHostChunks;
    RCHECK(cudaMemsetAsync(d_done, 0, n_chunks * sizeof(int), s_k));
    const StreamWriteValue32 wv = stream_write_value32();
    auto span = [&](int c, size_t& off, size_t& nb) {
        const int b = r->chunk_bucket[c];
        const int64_t c0 = (int64_t)r->chunk_ht0[c] * 16, c1 = std::min<int64_t>(r->cells[b], (int64_t)r->chunk_ht1[c] * 16);
        const size_t M = (size_t)r->NQ[b] * r->K[b];
        off = (size_t)c0 * M;
        nb = (size_t)(c1 - c0) * M * sizeof(double);
    };
    for (int c = 0; c < n_chunks; ++c) {
        const int b = r->chunk_bucket[c];
        size_t off, nb;
        span(c, off, nb);
        const Bucket& bk = r->h_buckets[b];
        RCHECK(cudaMemcpyAsync(const_cast<double*>(bk.f_cm) + off, f_host[b] + off, nb, cudaMemcpyHostToDevice, s_in));
        RCHECK(cudaMemcpyAsync(bk.q_cm + off, q_host[b] + off, nb, cudaMemcpyHostToDevice, s_in));
        // the chunk's ready word, ordered after its two copies: a stream memory write (with the fence
        // that orders the copies' data before it), else a 4-byte copy
        if (!wv || wv(s_in, (unsigned long long)(uintptr_t)(d_ready + c), (unsigned)epoch, 0u) != 0)
            RCHECK(cudaMemcpyAsync(d_ready + c, r->h_xepoch + c, sizeof(int), cudaMemcpyHostToDevice, s_in));
    }
    RCHECK(cudaMemsetAsync(r->d_counter, 0, sizeof(int), s_k));
    const RaggedSync rs{d_ready, d_done, d_units, r->h_xsync_dev, r->h_xsync_dev + kHostChunks, d_abort, epoch,
                        r->xwait};
    const unsigned grid = (unsigned)std::min(r->n_xunits, r->ctas);
    af_ragged_stream_kernel<<<grid, kTW * 32, r->smem, s_k>>>(r->d_buckets, r->d_xunits, r->n_xunits, r->d_counter,
                                                              rs, CmPtrs{});
    cf_add_launches(1);
    int st = CF_OK;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        cf_set_last_error(cudaGetErrorString(e));
        st = CF_ECUDA;
    }
    std::vector<char> sent(n_chunks, 0);
    int left = st == CF_OK ? n_chunks : 0;
    while (left > 0) {
        bool progress = false;
        for (int c = 0; c < n_chunks; ++c) {
            if (sent[c] || hs[c] != epoch) continue;
            size_t off, nb;
            span(c, off, nb);
            const int b = r->chunk_bucket[c];
            e = cudaMemcpyAsync(q_host[b] + off, r->h_buckets[b].q_cm + off, nb, cudaMemcpyDeviceToHost, s_out);
            if (e != cudaSuccess) break;
            sent[c] = 1;
            --left;
            progress = true;
        }
        if (e != cudaSuccess) {
            cf_set_last_error(cudaGetErrorString(e));
            st = CF_ECUDA;
            break;
        }
        if (progress || left == 0) continue;
        const cudaError_t q = cudaStreamQuery(s_k);
        if (q == cudaErrorNotReady) {
            std::this_thread::yield();
            continue;
        }
        if (q != cudaSuccess) {
            cf_set_last_error(cudaGetErrorString(q));
            st = CF_ECUDA;
            break;
        }
        // the kernel has ended: every chunk is final
        for (int c = 0; c < n_chunks && st == CF_OK; ++c) {
            if (sent[c]) continue;
            size_t off, nb;
            span(c, off, nb);
            const int b = r->chunk_bucket[c];
            e = cudaMemcpyAsync(q_host[b] + off, r->h_buckets[b].q_cm + off, nb, cudaMemcpyDeviceToHost, s_out);
            if (e != cudaSuccess) {
                cf_set_last_error(cudaGetErrorString(e));
                st = CF_ECUDA;
            }
            sent[c] = 1;
        }
        left = 0;
    }
    for (cudaStream_t x : r->xs) {
        const cudaError_t ex = cudaStreamSynchronize(x);
        if (ex != cudaSuccess && st == CF_OK) {
            cf_set_last_error(cudaGetErrorString(ex));
            st = CF_ECUDA;
        }
    }
    if (st == CF_OK && hs[kHostChunks] != 0) {
        cf_set_last_error("cf_ragged_q_host: a chunk's data did not arrive within the wait limit");
        st = CF_ETIMEOUT;
    }
    return st;
}

// Any other handle: every bucket up, the ordinary step on the device copies, every bucket back.
int host_plain(cf_ragged* r, double* const* q_host, const double* const* f_host) {
    cudaStream_t s = r->xs[0];
    std::vector<double*> qd(r->n_buckets);
    std::vector<const double*> fd(r->n_buckets);
    for (int b = 0; b < r->n_buckets; ++b) {
        fd[b] = r->h_buckets[b].f_cm;
        qd[b] = r->h_buckets[b].q_cm;
        const size_t nb = (size_t)r->cells[b] * r->NQ[b] * r->K[b] * sizeof(double);
        if (nb == 0) continue;
        RCHECK(cudaMemcpyAsync(const_cast<double*>(fd[b]), f_host[b], nb, cudaMemcpyHostToDevice, s));
        RCHECK(cudaMemcpyAsync(qd[b], q_host[b], nb, cudaMemcpyHostToDevice, s));
    }
    const int st = enqueue_step(r, qd.data(), fd.data(), s);
    if (st != CF_OK) return st;
    for (int b = 0; b < r->n_buckets; ++b) {
        const size_t nb = (size_t)r->cells[b] * r->NQ[b] * r->K[b] * sizeof(double);
        if (nb) RCHECK(cudaMemcpyAsync(q_host[b], qd[b], nb, cudaMemcpyDeviceToHost, s));
    }
    RCHECK(cudaStreamSynchronize(s));
    return CF_OK;
}

}  // namespace

extern "C" {

int cf_ragged_create(cf_ragged** out, cf_plan* const* plans, const int64_t* cells, const int32_t* forms,
                     int32_t n_buckets, int32_t tail_split, int32_t family) {
    if (!out || !plans || !cells || n_buckets < 1 || n_buckets > 64) {
        cf_set_last_error("cf_ragged_create: need 1..64 buckets");
        return CF_EINVAL;
    }
    if (tail_split != 0 && tail_split != 4 && tail_split != 16) {
        cf_set_last_error("cf_ragged_create: tail_split must be 0, 4 or 16");
        return CF_EINVAL;
    }
    if (family != 0 && family != 1) {
        cf_set_last_error("cf_ragged_create: family must be 0 (pair routine) or 1 (tile routine)");
        return CF_EINVAL;
    }
    *out = nullptr;
    cf_ragged* r = new cf_ragged();
    r->n_buckets = n_buckets;
    r->tail_split = tail_split;
    r->family = family;
    std::vector<Bucket> hb(n_buckets);
    int dev = -1;
    size_t max_smem = 0;
    int n_sms = 0;
    size_t tiles_total = 0;
    size_t max_M = 0;
    for (int b = 0; b < n_buckets; ++b) {
        cf_plan_info info;
        if (!plans[b] || cf_plan_get_info(plans[b], &info) != CF_OK || cells[b] < 0 ||
            ntiles(cells[b]) > 65535) {
            delete r;
            cf_set_last_error("cf_ragged_create: invalid plan or cell count");
            return CF_EINVAL;
        }
        const int form = forms ? forms[b] : CF_FORM_AF;
        if (form < CF_FORM_AF || form > CF_FORM_AF_SYM) {
            delete r;
            cf_set_last_error("cf_ragged_create: bucket forms must be one of the FP64 forms (0..4)");
            return CF_EINVAL;
        }
        if (dev < 0) dev = info.device;
        if (info.device != dev) {
            delete r;
            cf_set_last_error("cf_ragged_create: all plans must live on one device");
            return CF_EINVAL;
        }
        const bool fused = (form == CF_FORM_AF || form == CF_FORM_AF_SYM) && info.k <= kMaxK && info.k >= 1 &&
                           (family == 0 || info.k % 2 == 0);
        DevOp op{};
        const int* pbb = nullptr;
        const int* pbi = nullptr;
        const int2* pit = nullptr;
        const int* tbb = nullptr;
        const int* tbq = nullptr;
        cf_plan* view = plans[b];
        if (form == CF_FORM_AF_SYM) {
            // built here, never inside a graph recording (the build copies from the host)
            cf_plan* folded = nullptr;
            const int fs = cf_plan_folded(plans[b], &folded);
            if (fs != CF_OK) {
                delete r;
                return fs;
            }
            if (fused) view = folded;
        }
        cf_plan_internal_view(view, &op, &pbb, &pbi, &pit, &tbb, &tbq, &n_sms, &max_smem);
        hb[b] = Bucket{op, pbb, pbi, pit, tbb, tbq, nullptr, nullptr, info.k, info.n_q * info.k};
        r->form.push_back(form);
        r->fused.push_back(fused ? 1 : 0);
        r->plans.push_back(plans[b]);
        r->cells.push_back(cells[b]);
        r->K.push_back(info.k);
        r->NQ.push_back(info.n_q);
        // cost of one half-tile ~ its FLOPs (16 cells)
        r->cost.push_back(info.flops_q * 16.0);
        r->tile_off.push_back(tiles_total);
        tiles_total += 2 * (size_t)ntiles(cells[b]) * CF_TILE * info.n_q * info.k;
        if (fused) max_M = std::max(max_M, (size_t)info.n_q * info.k);
    }
    r->device = dev;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
    int st = CF_OK;
    const int W = family == 1 ? kTW : kRW;
    r->smem = sizeof(double) * ((size_t)W * (family == 1 ? kRBufTile : kRBufPair) + max_M * cf::kTileCells);
    const void* kern = family == 1 ? (const void*)af_ragged_kernel<true> : (const void*)af_ragged_kernel<false>;
    do {
        if (max_M > 0 && r->smem + 256 > max_smem) {
            cf_set_last_error("cf_ragged_create: the largest bucket's 16-cell tile does not fit in shared memory");
            st = CF_EUNSUPPORTED;
            break;
        }
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)r->smem);
        int per_sm = 0;
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, W * 32, r->smem);
        if (e != cudaSuccess || per_sm < 1) {
            cf_set_last_error("cf_ragged_create: fused kernel does not fit on this device");
            st = CF_EUNSUPPORTED;
            break;
        }
        r->ctas = per_sm * n_sms;
        // work units: whole half-tiles of every fused bucket, heaviest bucket first; the last `ctas`
        // half-tiles (in that order) are split into tail_split q1-pair bins each
        std::vector<int> order;
        for (int b = 0; b < n_buckets; ++b)
            if (r->fused[b]) order.push_back(b);
        std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return r->cost[a] > r->cost[c]; });
        std::vector<std::pair<int, int>> hts;
        for (int b : order)
            for (int64_t h = 0; h < (r->cells[b] + 15) / 16; ++h) hts.push_back({b, (int)h});
        const size_t n_ht = hts.size();
        const size_t n_whole = (tail_split == 0 || n_ht <= (size_t)r->ctas) ? (tail_split == 0 ? n_ht : 0)
                                                                              : n_ht - r->ctas;
        std::vector<Unit> units;
        for (size_t i = 0; i < n_ht; ++i) {
            if (i < n_whole) {
                units.push_back({hts[i].first, hts[i].second, 0, 0});
            } else {
                const int base = tail_split == 4 ? 1 : 5;  // bin layout of the plan: 0 whole, 1..4, 5..20
                for (int k = 0; k < tail_split; ++k) units.push_back({hts[i].first, hts[i].second, base + k, 0});
            }
        }
        r->n_units = (int)units.size();
        r->h_units = units;
        bool cm = family == 1 && r->n_units > 0;
        for (int b = 0; b < n_buckets; ++b)
            if (r->cells[b] > 0 && !r->fused[b]) cm = false;
        if (cm) {
            e = cudaFuncSetAttribute(af_ragged_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)r->smem);
            if (e != cudaSuccess) {
                cf_set_last_error(cudaGetErrorString(e));
                st = CF_ECUDA;
                break;
            }
        }
        r->cell_major = cm;
        e = cudaMalloc(&r->d_tiles, std::max<size_t>(tiles_total, 1) * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&r->d_buckets, n_buckets * sizeof(Bucket));
        if (e == cudaSuccess) e = cudaMalloc(&r->d_units, std::max<size_t>(units.size(), 1) * sizeof(Unit));
        if (e == cudaSuccess) e = cudaMalloc(&r->d_counter, sizeof(int));
        if (e != cudaSuccess) {
            cf_set_last_error(cudaGetErrorString(e));
            st = CF_ENOMEM;
            break;
        }
        for (int b = 0; b < n_buckets; ++b) {
            hb[b].fT = r->d_tiles + r->tile_off[b];
            hb[b].QT = r->d_tiles + r->tile_off[b] + (size_t)ntiles(r->cells[b]) * CF_TILE * r->NQ[b] * r->K[b];
            hb[b].cells = r->cells[b];
        }
        r->h_buckets = hb;
        e = cudaMemcpy(r->d_buckets, hb.data(), n_buckets * sizeof(Bucket), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !units.empty())
            e = cudaMemcpy(r->d_units, units.data(), units.size() * sizeof(Unit), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cf_set_last_error(cudaGetErrorString(e));
            st = CF_ECUDA;
            break;
        }
    } while (false);
    if (cur != dev) cudaSetDevice(cur);
    if (st != CF_OK) {
        free_ragged(r);
        delete r;
        return st;
    }
    *out = r;
    return CF_OK;
}

int cf_ragged_destroy(cf_ragged* r) {
    if (!r) return CF_OK;
    free_ragged(r);
    if (r->graph_stream) cudaStreamDestroy(r->graph_stream);
    delete r;
    return CF_OK;
}

// q[b] += Q(f[b]) for every bucket b (device arrays [N_Q x K x B_b]), one fused launch.
int cf_ragged_q(cf_ragged* r, double* const* q_dev, const double* const* f_dev, void* stream) {
    if (!r || !q_dev || !f_dev) return CF_EINVAL;
    std::lock_guard<std::mutex> lk(r->mu);
    return enqueue_step(r, q_dev, f_dev, (cudaStream_t)stream);
}

// The same step replayed from a CUDA graph recorded on first use for these buffers (re-recorded when
// the buffers change).  The recording does not allocate or synchronise inside the step.
int cf_ragged_graph_launch(cf_ragged* r, double* const* q_dev, const double* const* f_dev, void* stream) {
    if (!r || !q_dev || !f_dev) return CF_EINVAL;
    std::lock_guard<std::mutex> lk(r->mu);
    bool same = r->graph_exec != nullptr && (int)r->graph_f.size() == r->n_buckets;
    for (int b = 0; same && b < r->n_buckets; ++b) same = r->graph_f[b] == f_dev[b] && r->graph_q[b] == q_dev[b];
    if (!same) {
        if (r->graph_exec) cudaGraphExecDestroy(r->graph_exec);
        if (r->graph) cudaGraphDestroy(r->graph);
        r->graph_exec = nullptr;
        r->graph = nullptr;
        if (!r->graph_stream) RCHECK(cudaStreamCreateWithFlags(&r->graph_stream, cudaStreamNonBlocking));
        RCHECK(cudaStreamBeginCapture(r->graph_stream, cudaStreamCaptureModeThreadLocal));
        const int st = enqueue_step(r, q_dev, f_dev, r->graph_stream, false);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(r->graph_stream, &g);
        if (st != CF_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        RCHECK(e);
        r->graph = g;
        RCHECK(cudaGraphInstantiate(&r->graph_exec, g, 0));
        r->graph_f.assign(f_dev, f_dev + r->n_buckets);
        r->graph_q.assign(q_dev, q_dev + r->n_buckets);
    }
    RCHECK(cudaGraphLaunch(r->graph_exec, (cudaStream_t)stream));
    cf_add_launches(r->step_kernels);
    return CF_OK;
}

// The contraction alone on the handle's resident tiled buffers, as the last cf_ragged_q or
// cf_ragged_graph_launch left them (Q_tiled += Q(f_tiled)): the step without its layout passes.
int cf_ragged_q_resident(cf_ragged* r, void* stream) {
    if (!r) return CF_EINVAL;
    std::lock_guard<std::mutex> lk(r->mu);
    if (r->cell_major) {
        if (!r->have_last) {
            cf_set_last_error("cf_ragged_q_resident: no step has run on this handle yet");
            return CF_EINVAL;
        }
        return enqueue_resident_cm(r, (cudaStream_t)stream, true);
    }
    return enqueue_contract(r, (cudaStream_t)stream);
}

// q_host[b] += Q(f_host[b]) for every bucket, host arrays; synchronous.
int cf_ragged_q_host(cf_ragged* r, double* const* q_host, const double* const* f_host) {
    if (!r || !q_host || !f_host) return CF_EINVAL;
    for (int b = 0; b < r->n_buckets; ++b)
        if (r->cells[b] > 0 && (!q_host[b] || !f_host[b])) {
            cf_set_last_error("cf_ragged_q_host: null host array");
            return CF_EINVAL;
        }
    std::lock_guard<std::mutex> lk(r->mu);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != r->device) cudaSetDevice(r->device);
    int st = host_setup(r);
    if (st == CF_OK) st = r->host_stream ? host_streamed(r, q_host, f_host) : host_plain(r, q_host, f_host);
    if (cur != r->device) cudaSetDevice(cur);
    return st;
}

int cf_ragged_info(const cf_ragged* r, int32_t* n_units, int32_t* ctas, int64_t* smem_bytes, int32_t* n_fused) {
    if (!r) return CF_EINVAL;
    if (n_units) *n_units = r->n_units;
    if (ctas) *ctas = r->ctas;
    if (smem_bytes) *smem_bytes = (int64_t)r->smem;
    if (n_fused) {
        int n = 0;
        for (int b = 0; b < r->n_buckets; ++b) n += r->fused[b] ? 1 : 0;
        *n_fused = n;
    }
    return CF_OK;
}

}  // extern "C"
