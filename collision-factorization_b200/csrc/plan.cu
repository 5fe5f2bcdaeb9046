// plan.cu -- host side of libcf_b200: validation, COO re-bucketing, device plans, C ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <thread>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <list>
#include <map>
#include <unordered_map>
#include <array>
#include <mutex>
#include <string>
#include <vector>

#include "rfdense.cuh"
#include "split.cuh"
#include "../../include/cf_b200.h"
#include "common.cuh"
#include "launch.cuh"
#include "layout.cuh"

namespace {

thread_local std::string g_last_error;
std::atomic<int64_t> g_launches{0};
thread_local int g_few_route = 0;  // cf_few_route_last()

int fail(int status, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return status;
}

#define CF_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(e_ == cudaErrorMemoryAllocation ? CF_ENOMEM : CF_ECUDA, "%s: %s (%s:%d)", \
                        #call, cudaGetErrorString(e_), __FILE__, __LINE__);                    \
    } while (0)

#define CF_TRY(expr)              \
    do {                          \
        int s_ = (expr);          \
        if (s_ != CF_OK) return s_; \
    } while (0)

constexpr int kMaxK = 16;

// BF16 bits of a finite float, rounded to nearest even; and back
static unsigned short bf16_bits(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    u += 0x7fffu + ((u >> 16) & 1u);
    return (unsigned short)(u >> 16);
}
static float bf16_value(unsigned short b) {
    const uint32_t u = (uint32_t)b << 16;
    float x;
    std::memcpy(&x, &u, 4);
    return x;
}
constexpr int kCounterSlots = 64;  // work-queue heads per plan (one per stream in use)
#ifndef CF_HOST_STREAMS
#define CF_HOST_STREAMS 3
#endif
#ifndef CF_HOST_CHUNK_MIN
#define CF_HOST_CHUNK_MIN 256
#endif
#ifndef CF_HOST_MAX_CHUNKS
#define CF_HOST_MAX_CHUNKS 16
#endif
constexpr int kStreamChunks = 16;  // chunks of the streamed host path (at most)
constexpr double kStreamWaitSeconds = 5.0;  // a streamed-kernel CTA gives up on a chunk flag after this
constexpr int kHostStreams = CF_HOST_STREAMS;        // streams of the chunked host entry points
constexpr int64_t kHostChunkMin = CF_HOST_CHUNK_MIN;  // cells per chunk at least
constexpr int64_t kHostMaxChunks = CF_HOST_MAX_CHUNKS;

}  // namespace

// Internal view of a plan for the ragged (multi-operator) launcher in ragged.cu.
__attribute__((visibility("hidden"))) int cf_plan_internal_view(const cf_plan* plan, DevOp* op,
                                                                const int** pbin_begin, const int** pbin_item,
                                                                const int2** pitems, int* n_sms, size_t* max_smem);

// Lets the other translation units of the library report through cf_last_error().
__attribute__((visibility("hidden"))) void cf_set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }

// ------------------------------------------------------------------------------------------
// The plan: one operator resident on one device
// ------------------------------------------------------------------------------------------
struct cf_plan {
    int device = 0;
    int n_q = 0, k = 0, n_l = 0;
    int64_t n_g = 0, n_slices = 0;
    int n_items = 0;
    double flops_q = 0, flops_jv = 0;
    int64_t dev_bytes = 0;
    // device operator
    int* d_q1_begin = nullptr;
    int* d_slice_t = nullptr;
    int* d_slice_e = nullptr;
    uint32_t* d_e_q23 = nullptr;
    double* d_e_g = nullptr;
    double* d_R = nullptr;
    float* d_R32 = nullptr;  // FP32 copy of R for CF_FORM_AF_F32
    double* d_RT = nullptr;  // K = 8: R_t as [k1][8 k2 + k3] for the MMA kernel
    unsigned short* d_RTbf = nullptr;  // K = 8: the same split into BF16 hi and lo parts
    int* d_item_q1 = nullptr;
    int* d_bin_begin = nullptr;  // q1 bins of the tile kernel's work units (bin 0 = all, 1..4, 5..20)
    int* d_bin_q1 = nullptr;
    // work-queue heads of the persistent kernels: one slot per stream (kCounterSlots slots, assigned
    // on first use of a stream, least recently assigned slot reused beyond that), so launches on
    // different streams never share a counter; allocated with the plan, nothing is allocated later
    int* d_counter = nullptr;
    std::vector<std::pair<cudaStream_t, int>> counter_slots;  // most recently assigned last
    std::mutex counter_mu;
    int* d_pbin_begin = nullptr; // bins over pair items (same layout as the q1 bins)
    int* d_pbin_item = nullptr;
    int2* d_pitems = nullptr;    // (qa, qb) rows contracted by the two half-warps; qb = -1: no mirror
    int n_pairs = 0, n_pair_items = 0;
    int n_sms = 0;
    size_t max_smem = 0;
    int grouped = 0;  // folded plan, entries of each slice sorted by (q2, q3): bit 0 Q, bit 1 J.v (DevOp::grouped)
    int path = 0;  // cf::Path requested: 0 automatic, 1 gather, 2 tile, 3 pair, 4 pair (R via L1), 5 split pair
    int last_path = 0;  // family of the last angular-first / J.v launch (of this plan or its folded twin)
    cf_plan* parent = nullptr;  // for a folded twin: the plan it folds
    // scratch owned by the plan (tiled copies; device copies of host inputs)
    void* d_ws = nullptr;
    size_t ws_bytes = 0;
    double* d_io = nullptr;
    size_t io_bytes = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t host_streams[kHostStreams] = {};  // chunked host path: copies overlap the contraction
    cudaEvent_t chunk_done[CF_HOST_MAX_CHUNKS] = {};  // chunked host path: a chunk's contraction is done
    // streamed host path: copy-in, kernel and copy-out streams; per chunk a ready flag (device) and
    // a completion word (mapped pinned host memory); the epoch values the flag copies read (pinned)
    cudaStream_t xs[3] = {};
    int* d_xready = nullptr;
    int* d_xdone = nullptr;
    int* h_xepoch = nullptr;
    int* h_xsync = nullptr;      // [kStreamChunks] completion words, then the error word
    int* h_xsync_dev = nullptr;  // device alias of h_xsync
    int xepoch = 0;
    long long xwait_cycles = 0;
    // few-cell host path: Q then f of up to kFewCells cells in mapped pinned memory, which the
    // few-cell kernel reads and writes in place (no copy operations); h_few_dev is its device alias
    double* h_few = nullptr;
    double* h_few_dev = nullptr;
    std::mutex mu;
    // q2 <-> q3 folded operator (built on first use of CF_FORM_AF_SYM); fold_status != 0 if the
    // COO list is not symmetric in its last two indices
    cf_plan* sym = nullptr;
    int fold_status = -1;
    std::mutex sym_mu;
    // exact-split form (CF_FORM_AF_SYM_I8): built on the folded twin on first use
    cf::SplitPlan* split = nullptr;
    int split_status = -1;
    std::mutex split_mu;
    // radial-first dense form (CF_FORM_RF_DENSE): built on first use on the plan it runs on
    cf::RfDensePlan* rfd = nullptr;
    int rfd_status = -1;
    std::mutex rfd_mu;
    std::vector<double> h_labels, h_vals, h_ic, h_R;  // host copies kept for building the folded operator

    DevOp op() const {
        DevOp o;
        o.q1_begin = d_q1_begin;
        o.slice_t = d_slice_t;
        o.slice_e = d_slice_e;
        o.e_q23 = d_e_q23;
        o.e_g = d_e_g;
        o.R = d_R;
        o.R32 = d_R32;
        o.RT = d_RT;
        o.RTbf = d_RTbf;
        o.item_q1 = d_item_q1;
        o.grouped = grouped;
        o.n_items = n_items;
        o.n_q = n_q;
        o.k = k;
        o.n_l = n_l;
        return o;
    }
};

namespace {

struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) ok = (cudaSetDevice(dev) == cudaSuccess);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

int check_device_available() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
        return fail(CF_ENODEVICE, "no CUDA device available (%s)", cudaGetErrorString(e));
    return CF_OK;
}

bool is_index(double x, int hi) {
    if (!(x >= 1.0 && x <= (double)hi)) return false;
    return std::floor(x) == x;
}

int validate(const double* labels, const double* vals, const double* ic_map, const double* R,
             int64_t n_g, int32_t n_l, int32_t n_q, int32_t k) {
    if (n_g < 0) return fail(CF_ESHAPE, "N_G = %lld is negative", (long long)n_g);
    if (n_q < 1 || n_q > 65535) return fail(CF_ESHAPE, "N_Q = %d outside [1, 65535]", n_q);
    if (k < 1 || k > kMaxK) return fail(CF_EUNSUPPORTED, "K = %d outside [1, %d]", k, kMaxK);
    if (n_g > INT32_MAX - 64) return fail(CF_ESHAPE, "N_G = %lld too large", (long long)n_g);
    if (n_g == 0) return CF_OK;
    if (!labels || !vals || !ic_map || !R) return fail(CF_EINVAL, "null operator array");
    if (n_l < 1) return fail(CF_ESHAPE, "N_L = %d must be >= 1", n_l);
    for (int64_t z = 0; z < n_g; ++z) {
        for (int c = 0; c < 3; ++c) {
            const double q = labels[z + c * n_g];
            if (!is_index(q, n_q))
                return fail(CF_EBADIDX, "labels(%lld,%d) = %g is not an integer in [1, %d]", (long long)z + 1,
                            c + 1, q, n_q);
        }
        if (!is_index(ic_map[z], n_l))
            return fail(CF_EBADIDX, "ic_map(%lld) = %g is not an integer in [1, %d]", (long long)z + 1, ic_map[z],
                        n_l);
        if (!std::isfinite(vals[z])) return fail(CF_ENONFINITE, "vals(%lld) is not finite", (long long)z + 1);
    }
    const int64_t nr = (int64_t)k * k * k * n_l;
    for (int64_t i = 0; i < nr; ++i)
        if (!std::isfinite(R[i])) return fail(CF_ENONFINITE, "R(%lld) is not finite", (long long)i + 1);
    return CF_OK;
}

template <typename T>
int upload(T** dst, const std::vector<T>& src, int64_t& bytes) {
    const size_t nb = std::max<size_t>(src.size(), 1) * sizeof(T);
    CF_CUDA(cudaMalloc((void**)dst, nb));
    if (!src.empty()) CF_CUDA(cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
    bytes += (int64_t)nb;
    return CF_OK;
}

void free_plan_memory(cf_plan* p);
void free_plan_memory(cf_plan* p) {
    if (p->rfd) {
        cf::rfdense_destroy(p->rfd);
        p->rfd = nullptr;
    }
    if (p->split) {
        cf::split_destroy(p->split);
        p->split = nullptr;
    }
    if (p->sym) {
        free_plan_memory(p->sym);
        delete p->sym;
        p->sym = nullptr;
    }
    cudaFree(p->d_q1_begin);
    cudaFree(p->d_slice_t);
    cudaFree(p->d_slice_e);
    cudaFree(p->d_e_q23);
    cudaFree(p->d_e_g);
    cudaFree(p->d_R);
    cudaFree(p->d_R32);
    cudaFree(p->d_RT);
    cudaFree(p->d_RTbf);
    cudaFree(p->d_item_q1);
    cudaFree(p->d_bin_begin);
    cudaFree(p->d_bin_q1);
    cudaFree(p->d_counter);
    cudaFree(p->d_pbin_begin);
    cudaFree(p->d_pbin_item);
    cudaFree(p->d_pitems);
    cudaFree(p->d_ws);
    cudaFree(p->d_io);
    cudaFree(p->d_xready);
    if (p->h_xepoch) cudaFreeHost(p->h_xepoch);
    if (p->h_xsync) cudaFreeHost(p->h_xsync);
    if (p->h_few) cudaFreeHost(p->h_few);
    if (p->stream) cudaStreamDestroy(p->stream);
    for (cudaStream_t& hs : p->host_streams)
        if (hs) cudaStreamDestroy(hs);
    for (cudaEvent_t& ev : p->chunk_done)
        if (ev) cudaEventDestroy(ev);
    for (cudaStream_t& hs : p->xs)
        if (hs) cudaStreamDestroy(hs);
}

// Build the q1-grouped run structure (host) and upload it.
int build_plan(cf_plan* p, const double* labels, const double* vals, const double* ic_map, const double* R) {
    const int64_t NG = p->n_g;
    const int NQ = p->n_q, K = p->k;
    struct Run {
        int q1, t;
        int64_t z0, z1;
    };
    std::vector<Run> runs;
    for (int64_t z = 0; z < NG;) {
        const int t = (int)ic_map[z] - 1, q1 = (int)labels[z] - 1;
        int64_t e = z + 1;
        while (e < NG && (int)ic_map[e] - 1 == t && (int)labels[e] - 1 == q1) ++e;
        runs.push_back({q1, t, z, e});
        z = e;
    }
    // group runs by q1, keeping the caller's order inside each q1
    std::vector<int> count(NQ + 1, 0);
    for (const Run& r : runs) count[r.q1 + 1]++;
    std::vector<int> q1_begin(NQ + 1, 0);
    for (int q = 0; q < NQ; ++q) q1_begin[q + 1] = q1_begin[q] + count[q + 1];
    std::vector<int> fill(q1_begin.begin(), q1_begin.end() - 1);
    std::vector<int> order(runs.size());
    for (size_t i = 0; i < runs.size(); ++i) order[fill[runs[i].q1]++] = (int)i;

    const int64_t S = (int64_t)runs.size();
    std::vector<int> slice_t(S), slice_e(S + 1);
    std::vector<uint32_t> e_q23(NG);
    std::vector<double> e_g(NG);
    std::vector<double> cost(NQ, 0.0);
    int64_t pos = 0;
    for (int64_t s = 0; s < S; ++s) {
        const Run& r = runs[order[s]];
        slice_t[s] = r.t;
        slice_e[s] = (int)pos;
        for (int64_t z = r.z0; z < r.z1; ++z, ++pos) {
            const uint32_t q2 = (uint32_t)labels[z + NG] - 1, q3 = (uint32_t)labels[z + 2 * NG] - 1;
            e_q23[pos] = q2 | (q3 << 16);
            e_g[pos] = vals[z];
        }
        cost[r.q1] += (double)(r.z1 - r.z0) * K * K + (double)K * K * K;
    }
    slice_e[S] = (int)pos;

    std::vector<int> items;
    for (int q = 0; q < NQ; ++q)
        if (q1_begin[q + 1] > q1_begin[q]) items.push_back(q);
    std::stable_sort(items.begin(), items.end(), [&](int a, int b) { return cost[a] > cost[b]; });

    p->n_slices = S;
    p->n_items = (int)items.size();
    p->flops_q = (double)NG * (2.0 * K * K + K) + (double)S * 2.0 * K * K * K;
    p->flops_jv = (double)NG * (4.0 * K * K + 2.0 * K) + (double)S * 2.0 * K * K * K;

    // q1 bins of the tile kernel: bin 0 = every q1 heaviest first; bins 1..4 and 5..20 split the
    // q1 values into 4 and 16 bins of near-equal cost (longest-processing-time assignment)
    std::vector<int> bin_begin(1, 0), bin_q1;
    bin_q1.insert(bin_q1.end(), items.begin(), items.end());
    bin_begin.push_back((int)bin_q1.size());
    for (int nb : {4, 16}) {
        std::vector<std::vector<int>> bins(nb);
        std::vector<double> load(nb, 0.0);
        for (int q : items) {
            const int b = (int)(std::min_element(load.begin(), load.end()) - load.begin());
            bins[b].push_back(q);
            load[b] += cost[q];
        }
        for (auto& bl : bins) {
            bin_q1.insert(bin_q1.end(), bl.begin(), bl.end());
            bin_begin.push_back((int)bin_q1.size());
        }
    }

    // pair items: rows (l1,+m1) and (l1,-m1) whose slices have the same t sequence and lengths
    std::vector<std::vector<std::pair<int, int>>> shape(NQ);
    for (int q = 0; q < NQ; ++q)
        for (int s = q1_begin[q]; s < q1_begin[q + 1]; ++s) shape[q].push_back({slice_t[s], slice_e[s + 1] - slice_e[s]});
    std::vector<int2> pitems;
    std::vector<double> pcost;
    std::vector<char> used(NQ, 0);
    for (int l = 0; l * l < NQ; ++l) {
        for (int m = 1; m <= l; ++m) {
            const int qa = l * l + l + m, qb = l * l + l - m;
            if (qa >= NQ || qb >= NQ) continue;
            if (!shape[qa].empty() && shape[qa] == shape[qb]) {
                pitems.push_back(make_int2(qa, qb));
                pcost.push_back(cost[qa]);
                used[qa] = used[qb] = 1;
            }
        }
    }
    for (int q = 0; q < NQ; ++q)
        if (!used[q] && !shape[q].empty()) {
            pitems.push_back(make_int2(q, -1));
            pcost.push_back(cost[q]);
        }
    std::vector<int> porder(pitems.size());
    for (size_t i = 0; i < porder.size(); ++i) porder[i] = (int)i;
    std::stable_sort(porder.begin(), porder.end(), [&](int a, int b) { return pcost[a] > pcost[b]; });
    std::vector<int> pbin_begin(1, 0), pbin_item(porder.begin(), porder.end());
    pbin_begin.push_back((int)pbin_item.size());
    for (int nb : {4, 16}) {
        std::vector<std::vector<int>> bins(nb);
        std::vector<double> load(nb, 0.0);
        for (int i : porder) {
            const int b = (int)(std::min_element(load.begin(), load.end()) - load.begin());
            bins[b].push_back(i);
            load[b] += pcost[i];
        }
        for (auto& bl : bins) {
            pbin_item.insert(pbin_item.end(), bl.begin(), bl.end());
            pbin_begin.push_back((int)pbin_item.size());
        }
    }
    p->n_pair_items = (int)pitems.size();
    p->n_pairs = 0;
    for (const int2& it : pitems) p->n_pairs += it.y >= 0;

    std::vector<double> Rv((size_t)K * K * K * p->n_l);
    if (NG > 0) std::memcpy(Rv.data(), R, Rv.size() * sizeof(double));
    int64_t bytes = 0;
    CF_TRY(upload(&p->d_q1_begin, q1_begin, bytes));
    CF_TRY(upload(&p->d_slice_t, slice_t, bytes));
    CF_TRY(upload(&p->d_slice_e, slice_e, bytes));
    CF_TRY(upload(&p->d_e_q23, e_q23, bytes));
    CF_TRY(upload(&p->d_e_g, e_g, bytes));
    CF_TRY(upload(&p->d_R, Rv, bytes));
    std::vector<float> R32(Rv.begin(), Rv.end());
    CF_TRY(upload(&p->d_R32, R32, bytes));
    if (K == 8) {
        std::vector<double> RT(Rv.size());
        for (int t = 0; t < p->n_l; ++t)
            for (int k1 = 0; k1 < 8; ++k1)
                for (int k2 = 0; k2 < 8; ++k2)
                    for (int k3 = 0; k3 < 8; ++k3)
                        RT[(size_t)t * 512 + k1 * 64 + 8 * k2 + k3] = Rv[(size_t)t * 512 + k1 + 8 * k2 + 64 * k3];
        CF_TRY(upload(&p->d_RT, RT, bytes));
        // R_t^T = hi + lo in BF16 (round to nearest even), [t][hi, lo][k1][kk]
        std::vector<unsigned short> RTbf(2 * RT.size());
        for (int t = 0; t < p->n_l; ++t)
            for (int e = 0; e < 512; ++e) {
                const double r = RT[(size_t)t * 512 + e];
                const unsigned short hi = bf16_bits((float)r);
                const unsigned short lo = bf16_bits((float)(r - (double)bf16_value(hi)));
                RTbf[(size_t)t * 1024 + e] = hi;
                RTbf[(size_t)t * 1024 + 512 + e] = lo;
            }
        CF_TRY(upload(&p->d_RTbf, RTbf, bytes));
    }
    CF_TRY(upload(&p->d_item_q1, items, bytes));
    CF_TRY(upload(&p->d_bin_begin, bin_begin, bytes));
    CF_TRY(upload(&p->d_bin_q1, bin_q1, bytes));
    CF_TRY(upload(&p->d_pbin_begin, pbin_begin, bytes));
    CF_TRY(upload(&p->d_pbin_item, pbin_item, bytes));
    CF_TRY(upload(&p->d_pitems, pitems, bytes));
    CF_CUDA(cudaMalloc((void**)&p->d_counter, kCounterSlots * sizeof(int)));
    bytes += kCounterSlots * sizeof(int);
    int dev = 0, optin = 0;
    CF_CUDA(cudaGetDevice(&dev));
    CF_CUDA(cudaDeviceGetAttribute(&p->n_sms, cudaDevAttrMultiProcessorCount, dev));
    CF_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    p->max_smem = (size_t)optin;
    p->dev_bytes = bytes;
    return CF_OK;
}

int64_t n_tiles_for(int64_t B) { return (B + CF_TILE - 1) / CF_TILE; }

size_t tiled_bytes(const cf_plan* p, int64_t B) {
    return (size_t)n_tiles_for(B) * CF_TILE * (size_t)p->n_q * p->k * sizeof(double);
}

// ------------------------------------------------------------------------------------------
// Kernel dispatch over K (each K lives in its own translation unit, inst.cu)
// ------------------------------------------------------------------------------------------
int* counter_for(const cf_plan* pc, cudaStream_t st) {
    cf_plan* p = const_cast<cf_plan*>(pc);
    std::lock_guard<std::mutex> lk(p->counter_mu);
    auto& v = p->counter_slots;
    for (size_t i = 0; i < v.size(); ++i)
        if (v[i].first == st) return p->d_counter + v[i].second;
    int slot;
    if ((int)v.size() < kCounterSlots) {
        slot = (int)v.size();
    } else {
        slot = v.front().second;
        v.erase(v.begin());
    }
    v.push_back({st, slot});
    return p->d_counter + slot;
}

// dispatch() with `few` set: the few-cell kernel does not apply (the caller takes another route)
constexpr int kNoFew = -2;

int dispatch(const cf_plan* p, int what, bool exact, const double* fT, const double* vT, double* QT, int64_t B,
             cudaStream_t st, const float* fT32 = nullptr, bool bf16 = false, const StreamSync* ss = nullptr,
             const double* f_cm = nullptr, double* q_cm = nullptr, bool few = false,
             const double* few_host_f = nullptr, const double* few_host_q = nullptr, const float* vT32 = nullptr,
             bool rows = false, const double* v_cm = nullptr) {
    const int64_t nt = n_tiles_for(B);
    // The folded operator has about half the COO entries per slice of the plain one, and its tile
    // routine groups them by q2, so its Phi step is light next to the K^3 step; there the tile kernel
    // (16 warps per SM) runs ahead of the pair kernel (8 warps per SM): Q 2.50 M against 1.92 M
    // cells/s at L=10, K=8 on B200, J.v 0.59 against 0.75 ms for 2048 cells at L=8, K=8.
    const bool tile_first = p->parent != nullptr && (what == cf::OP_AF || what == cf::OP_JV) && !exact;
    cf::LaunchArgs a{p->op(), fT, vT, QT, nt, B, st, what, exact, p->path, p->d_bin_begin, p->d_bin_q1,
                     counter_for(p, st), p->n_sms, p->max_smem, p->d_pbin_begin, p->d_pbin_item, p->d_pitems,
                     fT32 != nullptr, fT32, tile_first, bf16};
    a.ss = ss;
    a.f_cm = f_cm;
    a.q_cm = q_cm;
    a.few = few;
    a.few_host_f = few_host_f;
    a.few_host_q = few_host_q;
    a.vT32 = vT32;
    a.rows = rows;
    a.v_cm = v_cm;
    cf::LaunchResult r{8, 0, cudaSuccess};
    switch (p->k) {
#define CF_K(KK) \
    case KK: r = cf::launch_k##KK(a); break;
        CF_K(1) CF_K(2) CF_K(3) CF_K(4) CF_K(5) CF_K(6) CF_K(7) CF_K(8)
        CF_K(9) CF_K(10) CF_K(11) CF_K(12) CF_K(13) CF_K(14) CF_K(15) CF_K(16)
#undef CF_K
        default: return fail(CF_EUNSUPPORTED, "K = %d not built", p->k);
    }
    g_launches += r.launches;
    if (few && r.status == -1) return kNoFew;
    if (r.status == CF_OK && r.launches > 0 && what != cf::OP_RF) {
        cf_plan* pm = const_cast<cf_plan*>(p);
        pm->last_path = r.path;
        if (pm->parent) pm->parent->last_path = r.path;
    }
    if (r.status == CF_ECUDA) return fail(CF_ECUDA, "kernel launch: %s", cudaGetErrorString(r.cuda));
    if (r.status == CF_EUNSUPPORTED)
        return fail(CF_EUNSUPPORTED, "form or kernel path not built for K = %d ("
                    "the tile-resident kernels need an even K <= 8 and a tile that fits in shared memory)", p->k);
    if (r.status != CF_OK) return fail(r.status, "launch failed for K = %d", p->k);
    return CF_OK;
}

int launch_pack(const cf_plan* p, const double* src, double* dst, int64_t B, cudaStream_t st) {
    const int M = p->n_q * p->k;
    const int64_t nt = n_tiles_for(B);
    if (nt == 0) return CF_OK;
    if (nt > 65535) return fail(CF_ESHAPE, "B = %lld exceeds %d cells per call", (long long)B, 65535 * CF_TILE);
    dim3 grid((M + 31) / 32, (unsigned)nt), block(32, 8);
    cf::pack_tiles_kernel<double><<<grid, block, 0, st>>>(src, dst, B, p->n_q, p->k);
    g_launches++;
    CF_CUDA(cudaGetLastError());
    return CF_OK;
}

int launch_pack32(const cf_plan* p, const double* src, float* dst, int64_t B, cudaStream_t st) {
    const int M = p->n_q * p->k;
    const int64_t nt = n_tiles_for(B);
    if (nt == 0) return CF_OK;
    if (nt > 65535) return fail(CF_ESHAPE, "B = %lld exceeds %d cells per call", (long long)B, 65535 * CF_TILE);
    dim3 grid((M + 31) / 32, (unsigned)nt), block(32, 8);
    cf::pack_tiles_kernel<float><<<grid, block, 0, st>>>(src, dst, B, p->n_q, p->k);
    g_launches++;
    CF_CUDA(cudaGetLastError());
    return CF_OK;
}

int launch_unpack(const cf_plan* p, const double* src, double* dst, int64_t B, cudaStream_t st) {
    const int M = p->n_q * p->k;
    const int64_t nt = n_tiles_for(B);
    if (nt == 0) return CF_OK;
    dim3 grid((M + 31) / 32, (unsigned)nt), block(32, 8);
    cf::unpack_tiles_kernel<<<grid, block, 0, st>>>(src, dst, B, p->n_q, p->k);
    g_launches++;
    CF_CUDA(cudaGetLastError());
    return CF_OK;
}

// Q_dev (cell-major) += op(f_dev[, v_dev]) using the tiled workspace ws (>= 2 or 3 tiled buffers).
// The forms that run on the tile kernel skip the layout passes: the kernel reads f and updates Q in
// the caller's cell-major arrays (the same per-row operations, so the same bits).  So do the fast
// FP64 Q forms on at most kFewCells cells, on the few-cell kernel (one launch).
int get_sym(cf_plan* p, cf_plan** out);
bool streamable(const cf_plan* p, const cf_plan* target, int what, bool exact, int f32);
int run_split(cf_plan* p, double* q_dev, const double* f_dev, int64_t B, cudaStream_t st);
int run_band64(cf_plan* target, double* q_dev, const double* f_dev, int64_t B, cudaStream_t st);
int run_lblock(cf_plan* target, double* q_dev, const double* f_dev, int64_t B, void* ws, size_t ws_bytes,
               cudaStream_t st, bool f32);
int run_bf16_band(cf_plan* target, double* q_dev, const double* f_dev, int64_t B, cudaStream_t st);
int run_rfdense(cf_plan* p, double* q_dev, const double* f_dev, int64_t B, cudaStream_t st);
int check_split(cf_plan* p);

// The fast FP64 angular-first (plain or folded) or radial-first form, or the exact angular-first
// form, of at most kFewCells cells on the few-cell kernel; kNoFew where that kernel does not apply.  With host_f and host_q (host
// arrays), f and Q_in travel in the launch's parameter block and Q_out goes to q; else Q is
// updated in place in the device arrays f, q.
int run_few(cf_plan* p, int what, bool exact, double* q, const double* f, int64_t B, cudaStream_t st, bool sym,
            int f32, const double* host_f = nullptr, const double* host_q = nullptr) {
    if (what == 2 || (exact && what != 0) || f32 != 0 || B > kFewCells) return kNoFew;
    cf_plan* target = p;
    if (sym) CF_TRY(get_sym(p, &target));
    return dispatch(target, what, exact, nullptr, nullptr, nullptr, B, st, nullptr, false, nullptr, f, q, true, host_f,
                    host_q);
}

// The kernel paths that run on the band units (their bounded waits report through check_split).
bool band_path(int path) { return path == cf::PATH_BAND || path == cf::PATH_LBLOCK; }

int run_device(cf_plan* p, int what, bool exact, double* q_dev, const double* f_dev, const double* v_dev,
               int64_t B, void* ws, size_t ws_bytes, cudaStream_t st, bool sym = false, int f32 = 0) {
    // f32: 0 the FP64 forms, 1 the FP32 forms, 2 the BF16-split forms (both read FP32 tiles of f)
    if (B < 0) return fail(CF_ESHAPE, "B = %lld is negative", (long long)B);
    if (B == 0 || p->n_g == 0) return CF_OK;
    if (!q_dev || !f_dev || (what == 2 && !v_dev)) return fail(CF_EINVAL, "null device buffer");
    if (f32 == 3) {
        if (what != 0) return fail(CF_EUNSUPPORTED, "the split form computes Q only");
        return run_split(p, q_dev, f_dev, B, st);
    }
    if (f32 == 4) {
        if (what != 0) return fail(CF_EUNSUPPORTED, "the radial-first dense form computes Q only");
        return run_rfdense(p, q_dev, f_dev, B, st);
    }
    {
        const int r = run_few(p, what, exact, q_dev, f_dev, B, st, sym, f32);
        if (r != kNoFew) return r;
    }
    // The exact angular-first form and the exact J.v above K = 8, where the batch kernels' per-lane
    // K x K Phi does not fit in registers: the row kernel of the few-cell route (one CTA per (q1, pair of
    // cells), the reference's operation order) on the cell-major arrays, for any number of cells.
    if (exact && (what == 0 || what == 2) && f32 == 0 && !sym && p->k > 8) {
        if (B > 65535)
            return fail(CF_ESHAPE, "the exact forms above K = 8 take at most 65535 cells per call (B = %lld)",
                        (long long)B);
        const int r = dispatch(p, what, true, nullptr, nullptr, nullptr, B, st, nullptr, false, nullptr, f_dev, q_dev,
                               true, nullptr, nullptr, nullptr, true, what == 2 ? v_dev : nullptr);
        if (r != kNoFew) return r;
    }
    const size_t tb = tiled_bytes(p, B);
    const size_t need = tb * (what == 2 ? 3 : 2);
    if (ws_bytes < need) return fail(CF_EINVAL, "workspace of %zu bytes is smaller than %zu", ws_bytes, need);
    double* fT = (double*)ws;
    double* QT = (double*)((char*)ws + tb);
    double* vT = what == 2 ? (double*)((char*)ws + 2 * tb) : nullptr;
    float* fT32 = f32 ? reinterpret_cast<float*>(fT) : nullptr;  // FP32 tiles use half of the f slot
    if (what == 0) {
        cf_plan* target = p;
        if (sym) CF_TRY(get_sym(p, &target));
        if (!exact && f32 == 0) {
            int r = run_band64(target, q_dev, f_dev, B, st);
            if (r != kNoFew) return r;
            r = run_lblock(target, q_dev, f_dev, B, ws, ws_bytes, st, false);
            if (r != kNoFew) return r;
        }
        if (!exact && f32 == 1) {
            const int r = run_lblock(target, q_dev, f_dev, B, ws, ws_bytes, st, true);
            if (r != kNoFew) return r;
        }
        if (!exact && f32 == 2) {
            const int r = run_bf16_band(target, q_dev, f_dev, B, st);
            if (r != kNoFew) return r;
        }
        if (streamable(p, target, what, exact, f32)) {
            const StreamSync resident{nullptr, nullptr, nullptr, nullptr, nullptr, 0, 1, 0};
            return dispatch(target, 0, false, nullptr, nullptr, nullptr, B, st, nullptr, false, &resident, f_dev,
                            q_dev);
        }
    }
    float* vT32 = (f32 && what == 2) ? reinterpret_cast<float*>(vT) : nullptr;  // FP32 J.v: v's FP32 tiles
    if (f32)
        CF_TRY(launch_pack32(p, f_dev, fT32, B, st));
    else
        CF_TRY(launch_pack(p, f_dev, fT, B, st));
    if (what == 2) {
        if (vT32)
            CF_TRY(launch_pack32(p, v_dev, vT32, B, st));
        else
            CF_TRY(launch_pack(p, v_dev, vT, B, st));
    }
    CF_TRY(launch_pack(p, q_dev, QT, B, st));
    cf_plan* target = p;
    if (sym) CF_TRY(get_sym(p, &target));
    CF_TRY(dispatch(target, what, exact, fT, vT, QT, B, st, fT32, f32 == 2, nullptr, nullptr, nullptr, false, nullptr,
                    nullptr, vT32));
    CF_TRY(launch_unpack(p, QT, q_dev, B, st));
    return CF_OK;
}

int ensure_ws(cf_plan* p, size_t need) {
    if (p->ws_bytes >= need) return CF_OK;
    if (p->d_ws) {
        CF_CUDA(cudaStreamSynchronize(p->stream));
        cudaFree(p->d_ws);
        p->d_ws = nullptr;
        p->ws_bytes = 0;
    }
    CF_CUDA(cudaMalloc(&p->d_ws, need));
    p->ws_bytes = need;
    return CF_OK;
}

int ensure_io(cf_plan* p, size_t need) {
    if (p->io_bytes >= need) return CF_OK;
    if (p->d_io) {
        CF_CUDA(cudaStreamSynchronize(p->stream));
        cudaFree(p->d_io);
        p->d_io = nullptr;
        p->io_bytes = 0;
    }
    CF_CUDA(cudaMalloc((void**)&p->d_io, need));
    p->io_bytes = need;
    return CF_OK;
}

int plan_create(cf_plan** out, const double* labels, const double* vals, const double* ic_map, const double* R,
                int64_t n_g, int32_t n_l, int32_t n_q, int32_t k, int32_t device) {
    if (!out) return fail(CF_EINVAL, "null plan pointer");
    *out = nullptr;
    CF_TRY(check_device_available());
    CF_TRY(validate(labels, vals, ic_map, R, n_g, n_l, n_q, k));
    if (device < 0) CF_CUDA(cudaGetDevice(&device));
    DeviceGuard guard(device);
    if (!guard.ok) return fail(CF_ENODEVICE, "cannot select device %d", device);
    cf_plan* p = new cf_plan();
    p->device = device;
    p->n_q = n_q;
    p->k = k;
    p->n_l = n_g > 0 ? n_l : std::max(n_l, 0);
    p->n_g = n_g;
    int s = build_plan(p, labels, vals, ic_map, R);
    if (s == CF_OK && n_g > 0) {
        p->h_labels.assign(labels, labels + 3 * n_g);
        p->h_vals.assign(vals, vals + n_g);
        p->h_ic.assign(ic_map, ic_map + n_g);
        p->h_R.assign(R, R + (size_t)k * k * k * n_l);
    }
    if (s == CF_OK) {
        cudaError_t e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) s = fail(CF_ECUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
    }
    if (s != CF_OK) {
        free_plan_memory(p);
        delete p;
        return s;
    }
    *out = p;
    return CF_OK;
}

// ------------------------------------------------------------------------------------------
// q2 <-> q3 folding.  The real Gaunt coefficients are symmetric in their last two indices, so
// the entries (q1,q2,q3,t = (l1,l2,l3)) and (q1,q3,q2,t' = (l1,l3,l2)) contribute
//   G R_t.(f2 (x) f3) + G' R_t'.(f3 (x) f2) = G (R_t + R_t'^T23).(f2 (x) f3)   (G = G').
// The folded operator keeps the entries with l2 < l3, or l2 = l3 and q2 <= q3 (diagonal q2 = q3
// at G/2), against R^S_t = R_t + R_t'^T23: about half the entries and half the slices, the same
// quadratic form.  J.v on it is the same Jacobian (the folded bilinear form is not symmetric, but
// its symmetric part is).
// ------------------------------------------------------------------------------------------
int isqrt_l(double q) {
    int64_t x = (int64_t)q - 1, l = (int64_t)std::sqrt((double)x);
    while ((l + 1) * (l + 1) <= x) ++l;
    while (l * l > x) --l;
    return (int)l;
}

int build_folded(const cf_plan* p, std::vector<double>& lab2, std::vector<double>& val2, std::vector<double>& ic2,
                 std::vector<double>& R2, int64_t& ng2, int& nl2) {
    const int64_t NG = p->n_g;
    const int K = p->k, NL = p->n_l, NQ = p->n_q;
    const size_t K3 = (size_t)K * K * K;
    const double* lab = p->h_labels.data();
    const double* val = p->h_vals.data();
    const double* ic = p->h_ic.data();
    std::vector<std::array<int, 3>> trip(NL, {-1, -1, -1});
    std::unordered_map<int64_t, int64_t> where;
    where.reserve((size_t)NG * 2);
    double gmax = 0.0;
    for (int64_t z = 0; z < NG; ++z) {
        const int t = (int)ic[z] - 1;
        const std::array<int, 3> l = {isqrt_l(lab[z]), isqrt_l(lab[z + NG]), isqrt_l(lab[z + 2 * NG])};
        if (trip[t][0] < 0) trip[t] = l;
        else if (trip[t] != l) return fail(CF_EUNSUPPORTED, "fold: ic_map %d mixes l-triplets", t + 1);
        const int64_t key = (((int64_t)lab[z] - 1) * NQ + ((int64_t)lab[z + NG] - 1)) * NQ + ((int64_t)lab[z + 2 * NG] - 1);
        where[key] = z;
        gmax = std::max(gmax, std::fabs(val[z]));
    }
    std::map<std::array<int, 3>, int> tindex;
    for (int t = 0; t < NL; ++t)
        if (trip[t][0] >= 0) tindex[trip[t]] = t;
    std::vector<int> tnew(NL, -1);
    nl2 = 0;
    R2.clear();
    for (int t = 0; t < NL; ++t) {
        if (trip[t][0] < 0 || trip[t][1] > trip[t][2]) continue;
        auto it = tindex.find({trip[t][0], trip[t][2], trip[t][1]});
        if (it == tindex.end()) return fail(CF_EUNSUPPORTED, "fold: l-triplet of ic_map %d has no mirror", t + 1);
        const int tp = it->second;
        tnew[t] = nl2++;
        const double* Rt = p->h_R.data() + (size_t)t * K3;
        const double* Rp = p->h_R.data() + (size_t)tp * K3;
        for (int k3 = 0; k3 < K; ++k3)
            for (int k2 = 0; k2 < K; ++k2)
                for (int k1 = 0; k1 < K; ++k1)
                    R2.push_back(Rt[k1 + K * k2 + K * K * k3] + Rp[k1 + K * k3 + K * K * k2]);
    }
    std::vector<double> q1v, q2v, q3v;
    val2.clear();
    ic2.clear();
    for (int64_t z = 0; z < NG; ++z) {
        const int t = (int)ic[z] - 1;
        const int l2 = trip[t][1], l3 = trip[t][2];
        const double q1 = lab[z], q2 = lab[z + NG], q3 = lab[z + 2 * NG];
        const int64_t key = (((int64_t)q1 - 1) * NQ + ((int64_t)q3 - 1)) * NQ + ((int64_t)q2 - 1);
        auto it = where.find(key);
        // every entry needs its mirror, also the ones the folded list drops (a dropped entry whose
        // kept mirror is missing would otherwise vanish from Q without a word)
        if (it == where.end()) return fail(CF_EUNSUPPORTED, "fold: entry %lld has no (q1,q3,q2) mirror", (long long)z + 1);
        if (!(l2 < l3 || (l2 == l3 && q2 <= q3))) continue;
        const double gp = val[it->second];
        if (std::fabs(gp - val[z]) > 1e-10 * gmax)
            return fail(CF_EUNSUPPORTED, "fold: G(q1,q2,q3) and G(q1,q3,q2) differ at entry %lld", (long long)z + 1);
        q1v.push_back(q1);
        q2v.push_back(q2);
        q3v.push_back(q3);
        val2.push_back(q2 == q3 ? 0.5 * val[z] : 0.5 * (val[z] + gp));
        ic2.push_back((double)(tnew[t] + 1));
    }
    // inside each run of equal (l-triplet, q1) the entries are ordered by (q2, q3), so that runs of
    // equal q2 are as long as they can be (the tile routine's grouped Phi step); the folded operator
    // has no exact form, so the order is free
    ng2 = (int64_t)q1v.size();
    {
        std::vector<int64_t> perm(ng2);
        for (int64_t i = 0; i < ng2; ++i) perm[i] = i;
        for (int64_t a = 0; a < ng2;) {
            int64_t b = a + 1;
            while (b < ng2 && ic2[b] == ic2[a] && q1v[b] == q1v[a]) ++b;
            std::stable_sort(perm.begin() + a, perm.begin() + b, [&](int64_t x, int64_t y) {
                return q2v[x] != q2v[y] ? q2v[x] < q2v[y] : q3v[x] < q3v[y];
            });
            a = b;
        }
        auto apply = [&](std::vector<double>& v) {
            std::vector<double> w(v.size());
            for (int64_t i = 0; i < ng2; ++i) w[i] = v[perm[i]];
            v.swap(w);
        };
        apply(q1v);
        apply(q2v);
        apply(q3v);
        apply(val2);
        apply(ic2);
    }
    lab2.clear();
    lab2.insert(lab2.end(), q1v.begin(), q1v.end());
    lab2.insert(lab2.end(), q2v.begin(), q2v.end());
    lab2.insert(lab2.end(), q3v.begin(), q3v.end());
    return CF_OK;
}

// The folded plan of p (created on first use).
int get_sym(cf_plan* p, cf_plan** out) {
    std::lock_guard<std::mutex> lk(p->sym_mu);
    if (p->sym) {
        *out = p->sym;
        return CF_OK;
    }
    if (p->fold_status > 0) return fail(p->fold_status, "this operator cannot be folded (see the first failure)");
    std::vector<double> lab2, val2, ic2, R2;
    int64_t ng2 = 0;
    int nl2 = 0;
    int st = build_folded(p, lab2, val2, ic2, R2, ng2, nl2);
    if (st != CF_OK) {
        p->fold_status = st;
        return st;
    }
    cf_plan* s = nullptr;
    st = plan_create(&s, lab2.data(), val2.data(), ic2.data(), R2.data(), ng2, nl2, p->n_q, p->k, p->device);
    if (st != CF_OK) return st;
    s->path = p->path;
    s->parent = p;
    // Grouping the Phi step by q2 pays where it was measured to (B200, folded hard-sphere operators):
    // for Q at K = 8 with long slices (L = 10: 12.8 entries per slice, 1.654 against 1.699 ms for
    // 4096 cells), not with short ones (L = 8: 9.8 per slice, 0.483 against 0.471 ms) or at K = 4
    // (0.373 against 0.324 ms at L = 8); for J.v from K = 6 on (L = 8, K = 8: 0.619 against 0.655 ms).
    // (The gather kernel, the automatic family for K > 8, was measured slower grouped: 13.23 against
    // 12.08 ms at L = 16, K = 12, 1024 cells; its entries' independent gathers hide its L1 latency.)
    const double per_slice = s->n_slices > 0 ? (double)s->n_g / (double)s->n_slices : 0.0;
    s->grouped = ((s->k == 8 && per_slice >= 12.0) ? 1 : 0) | (s->k >= 6 ? 2 : 0);
    s->h_labels.clear();  // the folded plan is never folded again
    p->sym = s;
    p->fold_status = 0;
    *out = s;
    return CF_OK;
}

// The split operator of a folded plan (created on first use).
int get_split(cf_plan* s, cf::SplitPlan** out) {
    std::lock_guard<std::mutex> lk(s->split_mu);
    if (s->split) {
        *out = s->split;
        return CF_OK;
    }
    if (s->split_status > 0) return fail(s->split_status, "the split form is not available for this operator");
    const int st = cf::split_build(&s->split, s->op(), s->n_g, s->n_slices, s->device);
    if (st != CF_OK) {
        s->split_status = st;
        return st;  // message set by split_build
    }
    s->split_status = 0;
    s->dev_bytes += cf::split_device_bytes(s->split);
    *out = s->split;
    return CF_OK;
}

// Q += Q(f) in the split form on cell-major device arrays (one launch of af_split_kernel).
int run_split(cf_plan* p, double* q_dev, const double* f_dev, int64_t B, cudaStream_t st) {
    if (!cf::split_supported_k(p->k)) return fail(CF_EUNSUPPORTED, "the split form needs K = 4, 8 or 12 (K = %d)", p->k);
    cf_plan* target = nullptr;
    CF_TRY(get_sym(p, &target));
    cf::SplitPlan* sp = nullptr;
    CF_TRY(get_split(target, &sp));
    int64_t launches = 0;
    CF_TRY(cf::split_run(sp, q_dev, f_dev, B, st, &launches));
    g_launches += launches;
    if (launches > 0) {
        target->last_path = cf::PATH_SPLIT_I8;
        p->last_path = cf::PATH_SPLIT_I8;
    }
    return CF_OK;
}

// The FP64 band kernel (af_band64_kernel) takes the fast angular-first Q forms at K = 4, 8 and 12 on
// kernel path PATH_BAND.  Where its operator has no unique (t, q1) slices it does not apply.
int run_band64(cf_plan* target, double* q_dev, const double* f_dev, int64_t B, cudaStream_t st) {
    const bool wanted = cf::split_supported_k(target->k) && target->path == cf::PATH_BAND;
    if (!wanted) return kNoFew;
    cf::SplitPlan* sp = nullptr;
    const int st_build = get_split(target, &sp);
    if (st_build != CF_OK) {
        if (target->path == cf::PATH_BAND) return st_build;
        g_last_error.clear();
        return kNoFew;
    }
    int64_t launches = 0;
    CF_TRY(cf::band64_run(sp, q_dev, f_dev, B, st, &launches));
    g_launches += launches;
    if (launches > 0) {
        target->last_path = cf::PATH_BAND;
        if (target->parent) target->parent->last_path = cf::PATH_BAND;
    }
    return CF_OK;
}

// The l-block kernels (af_lblock64_kernel, and af_lblock32_kernel for the FP32 forms) take the fast
// angular-first Q forms at K = 8 and 12 on kernel path PATH_LBLOCK: one CTA per (l1 band, cell group:
// 8 cells in FP64, 16 in FP32) with R_t and the f rows of bands l2 and l3 staged per l-triplet, from f
// packed per cell group into the workspace, and the band's slices handed to the warps one at a time.
//
// The automatic order also takes it for the fast Q forms (plain and folded) at K = 12, where the
// gather kernel is the other family (B200, ms per launch, l-block with its K^3 step on the FP64 tensor
// cores against gather, folded / plain: L = 16, 1024 cells 6.89 / 15.93 against 12.10 / 23.11;
// L = 12, 1024 cells 2.29 / 5.07 against 3.86 / 7.37; L = 8, 2048 cells 0.96 / 1.82 against
// 1.69 / 3.07; L = 6, 2048 cells 0.39 / 0.66 against 0.68 / 1.18; L = 4, 4096 cells 0.27 / 0.38
// against - / 0.63).  Operators whose (t, q1) pairs come in several runs (an unsorted COO list) have
// no band tables and stay on the gather kernel.
bool lblock_auto(const cf_plan* target) { return target->path == cf::PATH_AUTO && target->k == 12; }

int run_lblock(cf_plan* target, double* q_dev, const double* f_dev, int64_t B, void* ws, size_t ws_bytes,
               cudaStream_t st, bool f32) {
    const bool automatic = lblock_auto(target);
    if (target->path != cf::PATH_LBLOCK && !automatic) return kNoFew;
    if (target->k != 8 && target->k != 12)
        return fail(CF_EUNSUPPORTED, "the l-block kernel needs K = 8 or 12 (K = %d)", target->k);
    cf::SplitPlan* sp = nullptr;
    const int st_build = get_split(target, &sp);
    if (st_build != CF_OK || (automatic && !cf::lblock_available(sp, f32))) {
        if (!automatic) return st_build;
        g_last_error.clear();  // the automatic order goes on to the gather kernel
        return kNoFew;
    }
    int64_t launches = 0;
    CF_TRY(cf::lblock_run(sp, q_dev, f_dev, ws, ws_bytes, B, f32, st, &launches));
    g_launches += launches;
    if (launches > 0) {
        target->last_path = cf::PATH_LBLOCK;
        if (target->parent) target->parent->last_path = cf::PATH_LBLOCK;
    }
    return CF_OK;
}

// The BF16-split forms at K = 4 and 12 (and at K = 8 on kernel path PATH_BAND) run on the band kernel
// with the K^3 step on the BF16 tensor cores (af_bf16_band_kernel); K = 8 otherwise keeps the warp-level
// BF16 kernel.
int run_bf16_band(cf_plan* target, double* q_dev, const double* f_dev, int64_t B, cudaStream_t st) {
    if (!cf::split_supported_k(target->k) || (target->k == 8 && target->path != cf::PATH_BAND)) return kNoFew;
    cf::SplitPlan* sp = nullptr;
    CF_TRY(get_split(target, &sp));
    int64_t launches = 0;
    CF_TRY(cf::bf16_band_run(sp, q_dev, f_dev, B, st, &launches));
    g_launches += launches;
    if (launches > 0) {
        target->last_path = cf::PATH_BAND_BF16;
        if (target->parent) target->parent->last_path = cf::PATH_BAND_BF16;
    }
    return CF_OK;
}

// The radial-first dense form on the plan's folded twin where the operator folds, else on the plan.
int run_rfdense(cf_plan* p, double* q_dev, const double* f_dev, int64_t B, cudaStream_t st) {
    if (!cf::rfdense_supported_k(p->k)) return fail(CF_EUNSUPPORTED, "the radial-first dense form needs K <= 16");
    cf_plan* target = nullptr;
    if (get_sym(p, &target) != CF_OK) {
        g_last_error.clear();
        target = p;
    }
    cf::RfDensePlan* rp = nullptr;
    {
        std::lock_guard<std::mutex> lk(target->rfd_mu);
        if (!target->rfd) {
            if (target->rfd_status > 0) return fail(target->rfd_status, "the radial-first dense form is not available for this operator");
            const int st_b = cf::rfdense_build(&target->rfd, target->op(), target->n_g, target->n_slices, target->device);
            if (st_b != CF_OK) {
                target->rfd_status = st_b;
                return st_b;  // message set by rfdense_build
            }
            target->rfd_status = 0;
            target->dev_bytes += cf::rfdense_device_bytes(target->rfd);
        }
        rp = target->rfd;
    }
    int64_t launches = 0;
    CF_TRY(cf::rfdense_run(rp, q_dev, f_dev, B, st, &launches));
    g_launches += launches;
    if (launches > 0) {
        target->last_path = cf::PATH_RF_DENSE;
        p->last_path = cf::PATH_RF_DENSE;
    }
    return CF_OK;
}

// After a synchronised call on a band kernel (split, FP64 or BF16): the error word of its launches,
// on the plan's own band units and on those of its folded twin.
int check_split(cf_plan* p) {
    int st = CF_OK;
    if (p->split) st = cf::split_check(p->split);
    if (st == CF_OK && p->sym && p->sym->split) st = cf::split_check(p->sym->split);
    return st;
}

// ------------------------------------------------------------------------------------------
// Content-keyed cache of plans for the MEX-style host entry points
// ------------------------------------------------------------------------------------------
uint64_t hash_words(const double* a, int64_t n, uint64_t h) {
    // eight independent multiply-xorshift lanes, so the multiplier's throughput rather than one
    // lane's dependency chain bounds the speed
    constexpr int NL = 8;
    const uint64_t* w = reinterpret_cast<const uint64_t*>(a);
    uint64_t l[NL];
    for (int j = 0; j < NL; ++j) l[j] = h ^ (0x9e3779b97f4a7c15ULL * (uint64_t)(j + 1));
    int64_t i = 0;
    for (; i + NL <= n; i += NL)
        for (int j = 0; j < NL; ++j) {
            l[j] ^= w[i + j];
            l[j] *= 0x100000001b3ULL;
            l[j] ^= l[j] >> 29;
        }
    uint64_t r = (uint64_t)n ^ h;
    for (; i < n; ++i) {
        r ^= w[i];
        r *= 0x100000001b3ULL;
        r ^= r >> 29;
    }
    for (int j = 0; j < NL; ++j) {
        r ^= l[j];
        r *= 0x100000001b3ULL;
        r ^= r >> 31;
    }
    return r;
}

// Content key of an operator: the four arrays hashed separately and combined in a fixed order.
// Above 1 MB a helper thread hashes labels and vals while the caller hashes ic_map and R (the
// key does not depend on which thread hashed what).
uint64_t hash_operator(const double* labels, const double* vals, const double* ic_map, const double* R, int64_t n_g,
                       int64_t n_r) {
    uint64_t hl = 0, hv = 0;
    auto first = [&] {
        hl = hash_words(labels, 3 * n_g, 0x11);
        hv = hash_words(vals, n_g, 0x22);
    };
    bool threaded = (5 * n_g + n_r) * (int64_t)sizeof(double) > ((int64_t)1 << 20);
    std::thread helper;
    if (threaded) {
        try {
            helper = std::thread(first);
        } catch (...) {
            threaded = false;
        }
    }
    if (!threaded) first();
    const uint64_t hi = hash_words(ic_map, n_g, 0x33), hr = hash_words(R, n_r, 0x44);
    if (threaded) helper.join();
    uint64_t r = 0xcbf29ce484222325ULL;
    for (uint64_t x : {hl, hv, hi, hr}) {
        r ^= x;
        r *= 0x100000001b3ULL;
        r ^= r >> 31;
    }
    return r;
}

struct CacheEntry {
    uint64_t key;
    int64_t n_g;
    int n_l, n_q, k, device;
    cf_plan* plan;
    const void* ptrs[4];  // labels, vals, ic_map, R of the last call that found this entry by content
};

std::mutex g_cache_mu;
std::list<CacheEntry> g_cache;  // most recent first
constexpr size_t kCacheMax = 8;

int cached_plan(cf_plan** out, const double* labels, const double* vals, const double* ic_map, const double* R,
                int64_t n_g, int32_t n_l, int32_t n_q, int32_t k) {
    CF_TRY(check_device_available());
    int device = 0;
    CF_CUDA(cudaGetDevice(&device));
    if (n_g < 0 || k < 1 || k > kMaxK || n_l < 0) return validate(labels, vals, ic_map, R, n_g, n_l, n_q, k);
    uint64_t h = 0xcbf29ce484222325ULL;
    if (n_g > 0 && labels && vals && ic_map && R) h = hash_operator(labels, vals, ic_map, R, n_g, (int64_t)k * k * k * n_l);
    const void* ptrs[4] = {labels, vals, ic_map, R};
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (CacheEntry& e : g_cache)  // these pointers now belong to the entry found or made below
        if (std::equal(e.ptrs, e.ptrs + 4, ptrs)) std::fill(e.ptrs, e.ptrs + 4, nullptr);
    for (auto it = g_cache.begin(); it != g_cache.end(); ++it) {
        if (it->key == h && it->n_g == n_g && it->n_l == n_l && it->n_q == n_q && it->k == k && it->device == device) {
            g_cache.splice(g_cache.begin(), g_cache, it);
            std::copy(ptrs, ptrs + 4, g_cache.front().ptrs);
            *out = g_cache.front().plan;
            return CF_OK;
        }
    }
    cf_plan* p = nullptr;
    CF_TRY(plan_create(&p, labels, vals, ic_map, R, n_g, n_l, n_q, k, device));
    g_cache.push_front({h, n_g, n_l, n_q, k, device, p, {labels, vals, ic_map, R}});
    while (g_cache.size() > kCacheMax) {
        cf_plan* old = g_cache.back().plan;
        g_cache.pop_back();
        {
            std::lock_guard<std::mutex> pl(old->mu);
            DeviceGuard g(old->device);
            cudaStreamSynchronize(old->stream);
            free_plan_memory(old);
        }
        delete old;
    }
    *out = p;
    return CF_OK;
}

// The plan that the last content lookup with these very pointers (and sizes, on the current device)
// found, with its content key: a guess that the arrays did not change since, which the streamed
// host path verifies while the GPU already works on it.
bool plan_by_pointers(cf_plan** out, uint64_t* key, const double* labels, const double* vals, const double* ic_map,
                      const double* R, int64_t n_g, int32_t n_l, int32_t n_q, int32_t k) {
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return false;
    const void* ptrs[4] = {labels, vals, ic_map, R};
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (auto it = g_cache.begin(); it != g_cache.end(); ++it)
        if (std::equal(it->ptrs, it->ptrs + 4, ptrs) && it->n_g == n_g && it->n_l == n_l && it->n_q == n_q &&
            it->k == k && it->device == device) {
            g_cache.splice(g_cache.begin(), g_cache, it);
            *out = g_cache.front().plan;
            *key = g_cache.front().key;
            return true;
        }
    return false;
}

// Streamed host path: whether the fast angular-first form on `target` runs on the tile kernel (so the
// streamed kernel reproduces the device path bit for bit) and the tile fits in shared memory.
bool streamable(const cf_plan* p, const cf_plan* target, int what, bool exact, int f32) {
    if (what != 0 || exact || f32 != 0 || p->k % 2 != 0 || p->k > 8) return false;
    const bool tile = target->parent != nullptr ? (p->path == 0 || p->path == cf::PATH_TILE) : p->path == cf::PATH_TILE;
    if (!tile) return false;
    const size_t smem = sizeof(double) * ((size_t)p->n_q * p->k * 16 + (size_t)16 * p->k * (p->k * p->k + 2));
    return smem + 256 <= p->max_smem;
}

int ensure_stream_sync(cf_plan* p) {
    if (p->d_xready) return CF_OK;
    for (cudaStream_t& s : p->xs)
        if (!s) CF_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    int khz = 0;
    CF_CUDA(cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, p->device));
    p->xwait_cycles = (long long)((double)std::max(khz, 1000000) * 1e3 * kStreamWaitSeconds);
    // each allocation is kept once made, so a call after a failed set-up does not allocate it twice
    if (!p->h_xepoch) CF_CUDA(cudaHostAlloc((void**)&p->h_xepoch, kStreamChunks * sizeof(int), cudaHostAllocDefault));
    if (!p->h_xsync)
        CF_CUDA(cudaHostAlloc((void**)&p->h_xsync, (kStreamChunks + 1) * sizeof(int), cudaHostAllocMapped));
    CF_CUDA(cudaHostGetDevicePointer((void**)&p->h_xsync_dev, p->h_xsync, 0));
    int* d = nullptr;
    CF_CUDA(cudaMalloc((void**)&d, (2 * kStreamChunks + 1) * sizeof(int)));
    const cudaError_t e = cudaMemset(d, 0, (2 * kStreamChunks + 1) * sizeof(int));
    if (e != cudaSuccess) {
        cudaFree(d);
        return fail(CF_ECUDA, "cudaMemset: %s", cudaGetErrorString(e));
    }
    p->d_xready = d;
    p->d_xdone = d + kStreamChunks;
    return CF_OK;
}

// Q += op(f) for B cells in host memory with one launch of the streamed tile kernel: every chunk's
// uploads and ready flag are queued first (copy-in stream), then the kernel (kernel stream), then
// each chunk's download as soon as the kernel marks it final (copy-out stream).  Queueing every
// upload before the launch keeps the copies ahead of the kernel even where the two streams share a
// hardware queue.  The host waits for a chunk's completion word only while the kernel is still
// running, and the kernel's own waits are bounded, so the call always ends.
//
// send = false (the self-test) queues no uploads and no flags, so the kernel's waits run out after
// wait_cycles; the call then returns CF_ETIMEOUT with Q untouched on the host.
//
// gate (speculative calls): no chunk goes back to Q before *gate is 1 (the operator's content was
// verified); 2 means it changed: the call copies nothing back, waits for the kernel and returns
// kRetry, and the caller contracts again with the right plan.
constexpr int kRetry = -1;
int run_host_streamed(cf_plan* p, cf_plan* target, double* Q, const double* f, int64_t B, double* dQ, double* df,
                      bool send = true, long long wait_cycles = 0, const std::atomic<int>* gate = nullptr) {
    CF_TRY(ensure_stream_sync(p));
    const int64_t M = (int64_t)p->n_q * p->k;
    const int64_t n_ht = (B + 15) / 16;
    const int64_t hpc = (n_ht + kStreamChunks - 1) / kStreamChunks;
    const int n_chunks = (int)((n_ht + hpc - 1) / hpc);
    p->xepoch = p->xepoch % 0x3fffffff + 1;
    const int epoch = p->xepoch;
    volatile int* hs = p->h_xsync;
    for (int c = 0; c < n_chunks; ++c) {
        p->h_xepoch[c] = epoch;
        hs[c] = 0;
    }
    hs[kStreamChunks] = 0;
    cudaStream_t s_in = p->xs[0], s_k = p->xs[1], s_out = p->xs[2];
    CF_CUDA(cudaMemsetAsync(p->d_xdone, 0, n_chunks * sizeof(int), s_k));
    auto span = [&](int c, int64_t& off, size_t& nb) {
        const int64_t b0 = (int64_t)c * hpc * 16, b1 = std::min<int64_t>(B, (int64_t)(c + 1) * hpc * 16);
        off = b0 * M;
        nb = (size_t)(b1 - b0) * M * sizeof(double);
    };
    for (int c = 0; c < n_chunks && send; ++c) {
        int64_t off;
        size_t nb;
        span(c, off, nb);
        CF_CUDA(cudaMemcpyAsync(df + off, f + off, nb, cudaMemcpyHostToDevice, s_in));
        CF_CUDA(cudaMemcpyAsync(dQ + off, Q + off, nb, cudaMemcpyHostToDevice, s_in));
        CF_CUDA(cudaMemcpyAsync(p->d_xready + c, p->h_xepoch + c, sizeof(int), cudaMemcpyHostToDevice, s_in));
    }
    StreamSync ss{p->d_xready, p->d_xdone, p->h_xsync_dev, p->h_xsync_dev + kStreamChunks,
                  p->d_xdone + kStreamChunks, epoch, (int)hpc, wait_cycles > 0 ? wait_cycles : p->xwait_cycles};
    int st = dispatch(target, 0, false, nullptr, nullptr, nullptr, B, s_k, nullptr, false, &ss, df, dQ);
    int next = 0;
    while (st == CF_OK && next < n_chunks) {
        if (gate) {
            const int g = gate->load(std::memory_order_acquire);
            if (g == 2) {
                st = kRetry;
                break;
            }
            if (g == 0) {
                std::this_thread::yield();
                continue;
            }
        }
        bool all = false;
        if (hs[next] != epoch) {
            const cudaError_t q = cudaStreamQuery(s_k);
            if (q == cudaErrorNotReady) {
                std::this_thread::yield();
                continue;
            }
            if (q != cudaSuccess) {
                st = fail(CF_ECUDA, "streamed contraction: %s", cudaGetErrorString(q));
                break;
            }
            all = true;  // the kernel has ended: every chunk is final
        }
        for (int c = next; c < (all ? n_chunks : next + 1) && send; ++c) {
            int64_t off;
            size_t nb;
            span(c, off, nb);
            const cudaError_t e = cudaMemcpyAsync(Q + off, dQ + off, nb, cudaMemcpyDeviceToHost, s_out);
            if (e != cudaSuccess) st = fail(CF_ECUDA, "%s", cudaGetErrorString(e));
        }
        next = all ? n_chunks : next + 1;
    }
    for (cudaStream_t s : p->xs) {
        const cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess && (st == CF_OK || st == kRetry)) st = fail(CF_ECUDA, "%s", cudaGetErrorString(e));
    }
    if (st == CF_OK && hs[kStreamChunks] != 0)
        st = fail(CF_ETIMEOUT, "streamed contraction: a chunk's data did not arrive within the wait limit");
    return st;
}

// The streamed contraction with the plan these pointers had last time, while a helper thread checks
// the operator's content hash; nothing reaches Q before the check passes.  kRetry: no guess, the
// guess does not stream, or the content changed (Q untouched) -- contract the ordinary way.
// Chunked host pipeline on plan p (p->mu held): chunk c goes up, is contracted and comes back on stream
// c mod kHostStreams, so the host<->device copies of one chunk overlap the contraction of the others
// (pinned host memory makes the copies asynchronous; pageable memory still gives the right answer,
// serialised).  With a gate (p is a guess from the operator's pointers, its content hash computed on
// another thread), the downloads wait: once the gate reads 1, every chunk's download is queued on the
// plan's stream behind an event of its contraction; if it reads 2, nothing is copied back and kRetry
// is returned.
int run_host_chunked(cf_plan* p, int what, bool exact, double* Q, const double* f, const double* v, int64_t B,
                     double* dQ, double* df, double* dv, bool sym, int f32, const std::atomic<int>* gate) {
    const int64_t M = (int64_t)p->n_q * p->k;
    const int nbuf = what == 2 ? 3 : 2;
    for (cudaStream_t& hs : p->host_streams)
        if (!hs) CF_CUDA(cudaStreamCreateWithFlags(&hs, cudaStreamNonBlocking));
    int64_t n_chunks = std::min<int64_t>(kHostMaxChunks, B / kHostChunkMin);
    const int64_t per = (B + n_chunks - 1) / n_chunks;
    const int64_t chunk = (per + CF_TILE - 1) / CF_TILE * CF_TILE;  // whole 32-cell tiles per chunk
    n_chunks = (B + chunk - 1) / chunk;
    const size_t tbc = tiled_bytes(p, chunk) * nbuf;
    CF_TRY(ensure_ws(p, tbc * kHostStreams));
    if (gate)
        for (int64_t c = 0; c < n_chunks; ++c)
            if (!p->chunk_done[c]) CF_CUDA(cudaEventCreateWithFlags(&p->chunk_done[c], cudaEventDisableTiming));
    int st = CF_OK;
    for (int64_t c = 0; c < n_chunks && st == CF_OK; ++c) {
        cudaStream_t s = p->host_streams[c % kHostStreams];
        const int64_t b0 = c * chunk, bc = std::min(chunk, B - b0);
        const size_t off = (size_t)b0 * M, nb = (size_t)bc * M * sizeof(double);
        void* ws = (char*)p->d_ws + (size_t)(c % kHostStreams) * tbc;
        cudaError_t e = cudaMemcpyAsync(dQ + off, Q + off, nb, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(df + off, f + off, nb, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && dv) e = cudaMemcpyAsync(dv + off, v + off, nb, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) {
            st = fail(CF_ECUDA, "%s", cudaGetErrorString(e));
            break;
        }
        st = run_device(p, what, exact, dQ + off, df + off, dv ? dv + off : nullptr, bc, ws, tbc, s, sym, f32);
        if (st == CF_OK) {
            e = gate ? cudaEventRecord(p->chunk_done[c], s) : cudaMemcpyAsync(Q + off, dQ + off, nb, cudaMemcpyDeviceToHost, s);
            if (e != cudaSuccess) st = fail(CF_ECUDA, "%s", cudaGetErrorString(e));
        }
    }
    bool retry = false;
    if (gate) {
        while (gate->load(std::memory_order_acquire) == 0) std::this_thread::yield();
        retry = gate->load(std::memory_order_acquire) == 2;
        for (int64_t c = 0; c < n_chunks && st == CF_OK && !retry; ++c) {
            const int64_t b0 = c * chunk, bc = std::min(chunk, B - b0);
            const size_t off = (size_t)b0 * M, nb = (size_t)bc * M * sizeof(double);
            cudaError_t e = cudaStreamWaitEvent(p->stream, p->chunk_done[c], 0);
            if (e == cudaSuccess) e = cudaMemcpyAsync(Q + off, dQ + off, nb, cudaMemcpyDeviceToHost, p->stream);
            if (e != cudaSuccess) st = fail(CF_ECUDA, "%s", cudaGetErrorString(e));
        }
    }
    for (cudaStream_t hs : p->host_streams) {
        const cudaError_t e = cudaStreamSynchronize(hs);
        if (e != cudaSuccess && st == CF_OK) st = fail(CF_ECUDA, "%s", cudaGetErrorString(e));
    }
    if (gate) {
        const cudaError_t e = cudaStreamSynchronize(p->stream);
        if (e != cudaSuccess && st == CF_OK) st = fail(CF_ECUDA, "%s", cudaGetErrorString(e));
    }
    if (st == CF_OK && (f32 >= 2 || band_path(p->path) || band_path(p->last_path))) st = check_split(p);
    if (st == CF_OK && retry) return kRetry;
    return st;
}

int run_host_speculative(double* Q, const double* f, int64_t B, const double* labels, const double* vals,
                         const double* ic_map, const double* R, int64_t n_g, int32_t n_l, int32_t n_q, int32_t k,
                         bool sym) {
    cf_plan* p = nullptr;
    uint64_t key = 0;
    if (n_g <= 0 || !labels || !vals || !ic_map || !R) return kRetry;
    if (!plan_by_pointers(&p, &key, labels, vals, ic_map, R, n_g, n_l, n_q, k)) return kRetry;
    std::lock_guard<std::mutex> lk(p->mu);
    DeviceGuard guard(p->device);
    if (!guard.ok) return kRetry;
    cf_plan* target = p;
    if (sym && get_sym(p, &target) != CF_OK) return kRetry;
    const bool streamed = streamable(p, target, 0, false, 0);
    const size_t cell_bytes = (size_t)B * p->n_q * p->k * sizeof(double);
    if (ensure_io(p, 2 * cell_bytes) != CF_OK) return kRetry;
    std::atomic<int> gate{0};
    std::thread check;
    try {
        check = std::thread([&] {
            const uint64_t h = hash_operator(labels, vals, ic_map, R, n_g, (int64_t)k * k * k * n_l);
            gate.store(h == key ? 1 : 2, std::memory_order_release);
        });
    } catch (...) {
        return kRetry;
    }
    double* dQ = p->d_io;
    double* df = (double*)((char*)p->d_io + cell_bytes);
    // the streamed tile kernel where the form runs on it, else the chunked pipeline with its
    // downloads held back until the hash has matched
    const int st = streamed ? run_host_streamed(p, target, Q, f, B, dQ, df, true, 0, &gate)
                            : run_host_chunked(p, 0, false, Q, f, nullptr, B, dQ, df, nullptr, sym, 0, &gate);
    check.join();
    if (gate.load() == 2) return kRetry;  // nothing was copied back: Q is as the caller passed it
    return st;
}

// A handful of cells on plan p from host arrays, one launch and one wait.  Where f and Q_in fit in
// the launch's parameter block they travel there and the kernel writes Q_out to the plan's mapped
// pinned staging; else they go up through the staging and a device buffer with two copies, and Q
// comes back the same way.  With key_check set, p is a guess from the pointers of an earlier call,
// and the operator's content hash is computed here while the kernel runs; on a mismatch Q is left
// as it was and kRetry returned.
int few_on_plan(cf_plan* p, int what, bool exact, double* Q, const double* f, int64_t B, bool sym, const uint64_t* key_check,
                const double* labels, const double* vals, const double* ic_map, const double* R) {
    std::lock_guard<std::mutex> lk(p->mu);
    DeviceGuard guard(p->device);
    if (!guard.ok) return fail(CF_ENODEVICE, "cannot select device %d", p->device);
    const size_t M = (size_t)p->n_q * p->k, nb = (size_t)B * M * sizeof(double);
    if (!p->h_few) {
        CF_CUDA(cudaHostAlloc((void**)&p->h_few, 2 * kFewCells * M * sizeof(double), cudaHostAllocMapped));
        const cudaError_t e = cudaHostGetDevicePointer((void**)&p->h_few_dev, p->h_few, 0);
        if (e != cudaSuccess) {
            cudaFreeHost(p->h_few);
            p->h_few = nullptr;
            return fail(CF_ECUDA, "cudaHostGetDevicePointer: %s", cudaGetErrorString(e));
        }
    }
    int st = run_few(p, what, exact, p->h_few_dev, nullptr, B, p->stream, sym, 0, f, Q);
    int route = 1;
    if (st == kNoFew) {
        route = 2;
        // the copy route: pinned staging [Q | f] -> device buffer [Q | f] -> kernel -> staging
        CF_TRY(ensure_io(p, 2 * nb));
        std::memcpy(p->h_few, Q, nb);
        std::memcpy(p->h_few + kFewCells * M, f, nb);
        double* dq = p->d_io;
        double* df = p->d_io + B * M;
        CF_CUDA(cudaMemcpyAsync(dq, p->h_few, nb, cudaMemcpyHostToDevice, p->stream));
        CF_CUDA(cudaMemcpyAsync(df, p->h_few + kFewCells * M, nb, cudaMemcpyHostToDevice, p->stream));
        st = run_few(p, what, exact, dq, df, B, p->stream, sym, 0);
        if (st == CF_OK) CF_CUDA(cudaMemcpyAsync(p->h_few, dq, nb, cudaMemcpyDeviceToHost, p->stream));
    }
    if (st != CF_OK) {  // kNoFew included: the caller takes the ordinary route
        cudaStreamSynchronize(p->stream);
        return st;
    }
    const bool same = !key_check ||
                      hash_operator(labels, vals, ic_map, R, p->n_g, (int64_t)p->k * p->k * p->k * p->n_l) == *key_check;
    CF_CUDA(cudaStreamSynchronize(p->stream));
    if (!same) return kRetry;
    std::memcpy(Q, p->h_few, nb);
    g_few_route = route;
    return CF_OK;
}

// The fast angular-first (plain or folded) and radial-first forms, and the exact angular-first
// form, of at most kFewCells cells from host arrays; kNoFew where the few-cell kernel does not apply.
int run_host_few(int what, bool exact, double* Q, const double* f, int64_t B, const double* labels, const double* vals,
                 const double* ic_map, const double* R, int64_t n_g, int32_t n_l, int32_t n_q, int32_t k, bool sym) {
    cf_plan* p = nullptr;
    uint64_t key = 0;
    if (n_g > 0 && labels && vals && ic_map && R && plan_by_pointers(&p, &key, labels, vals, ic_map, R, n_g, n_l, n_q, k)) {
        const int st = few_on_plan(p, what, exact, Q, f, B, sym, &key, labels, vals, ic_map, R);
        if (st != kRetry) return st;
    }
    CF_TRY(cached_plan(&p, labels, vals, ic_map, R, n_g, n_l, n_q, k));
    if (n_g == 0) return CF_OK;
    return few_on_plan(p, what, exact, Q, f, B, sym, nullptr, labels, vals, ic_map, R);
}

// Host-pointer contraction: upload, run, download.  what: 0 AF, 1 RF, 2 JV.
int run_host(int what, bool exact, double* Q, const double* f, const double* v, int64_t B, const double* labels,
             const double* vals, const double* ic_map, const double* R, int64_t n_g, int32_t n_l, int32_t n_q,
             int32_t k, bool sym = false, int f32 = 0) {
    if (B < 0) return fail(CF_ESHAPE, "B = %lld is negative", (long long)B);
    if (!Q || !f || (what == 2 && !v)) return fail(CF_EINVAL, "null host buffer");
    g_few_route = 0;
    if (B >= 1 && B <= kFewCells && what != 2 && (!exact || what == 0) && f32 == 0) {
        const int r = run_host_few(what, exact, Q, f, B, labels, vals, ic_map, R, n_g, n_l, n_q, k, sym);
        if (r != kNoFew) return r;
    }
    if (what == 0 && !exact && f32 == 0 && B >= 2 * kHostChunkMin) {
        const int r = run_host_speculative(Q, f, B, labels, vals, ic_map, R, n_g, n_l, n_q, k, sym);
        if (r != kRetry) return r;
    }
    cf_plan* p = nullptr;
    CF_TRY(cached_plan(&p, labels, vals, ic_map, R, n_g, n_l, n_q, k));
    if (B == 0 || n_g == 0) return CF_OK;
    std::lock_guard<std::mutex> lk(p->mu);
    DeviceGuard guard(p->device);
    const int64_t M = (int64_t)n_q * k;
    const size_t cell_bytes = (size_t)B * M * sizeof(double);
    const int nbuf = what == 2 ? 3 : 2;
    CF_TRY(ensure_io(p, cell_bytes * nbuf));
    double* dQ = p->d_io;
    double* df = (double*)((char*)p->d_io + cell_bytes);
    double* dv = what == 2 ? (double*)((char*)p->d_io + 2 * cell_bytes) : nullptr;
    if (B < 2 * kHostChunkMin) {
        const size_t tb = tiled_bytes(p, B);
        CF_TRY(ensure_ws(p, tb * nbuf));
        CF_CUDA(cudaMemcpyAsync(dQ, Q, cell_bytes, cudaMemcpyHostToDevice, p->stream));
        CF_CUDA(cudaMemcpyAsync(df, f, cell_bytes, cudaMemcpyHostToDevice, p->stream));
        if (dv) CF_CUDA(cudaMemcpyAsync(dv, v, cell_bytes, cudaMemcpyHostToDevice, p->stream));
        CF_TRY(run_device(p, what, exact, dQ, df, dv, B, p->d_ws, p->ws_bytes, p->stream, sym, f32));
        CF_CUDA(cudaMemcpyAsync(Q, dQ, cell_bytes, cudaMemcpyDeviceToHost, p->stream));
        CF_CUDA(cudaStreamSynchronize(p->stream));
        return f32 >= 2 || band_path(p->path) || band_path(p->last_path) ? check_split(p) : CF_OK;
    }
    if (B >= 2 * kHostChunkMin) {
        cf_plan* target = p;
        if (sym) CF_TRY(get_sym(p, &target));
        if (streamable(p, target, what, exact, f32)) return run_host_streamed(p, target, Q, f, B, dQ, df);
    }
    return run_host_chunked(p, what, exact, Q, f, v, B, dQ, df, dv, sym, f32, nullptr);
}

int form_what(int form, bool& exact, bool& sym, int& f32) {
    sym = false;
    f32 = 0;
    switch (form) {
        case CF_FORM_AF_F32: exact = false; f32 = 1; return 0;
        case CF_FORM_AF_SYM_F32: exact = false; f32 = 1; sym = true; return 0;
        case CF_FORM_AF_BF16: exact = false; f32 = 2; return 0;
        case CF_FORM_AF_SYM_BF16: exact = false; f32 = 2; sym = true; return 0;
        case CF_FORM_AF: exact = false; return 0;
        case CF_FORM_RF: exact = false; return 1;
        case CF_FORM_AF_EXACT: exact = true; return 0;
        case CF_FORM_RF_EXACT: exact = true; return 1;
        case CF_FORM_AF_SYM: exact = false; sym = true; return 0;
        case CF_FORM_AF_SYM_I8: exact = false; sym = true; f32 = 3; return 0;
        case CF_FORM_RF_DENSE: exact = false; sym = true; f32 = 4; return 0;
        default: return -1;
    }
}

// J.v mode argument: 0 fast, 1 exact operation order, 2 folded operator, 3 FP32, 4 FP32 folded
bool jv_mode(int mode, bool& exact, bool& sym, int& f32) {
    exact = mode == 1;
    sym = mode == 2 || mode == 4;
    f32 = mode >= 3 ? 1 : 0;
    return mode >= 0 && mode <= 4;
}

}  // namespace

// ------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------
extern "C" {

int cf_angular_first(double* Q, const double* f, const double* labels, const double* vals, const double* ic_map,
                     const double* R, int64_t n_g, int32_t n_l, int32_t n_q, int32_t k) {
    g_last_error.clear();
    return run_host(0, false, Q, f, nullptr, 1, labels, vals, ic_map, R, n_g, n_l, n_q, k);
}

int cf_radial_first(double* Q, const double* f, const double* labels, const double* vals, const double* ic_map,
                    const double* R, int64_t n_g, int32_t n_l, int32_t n_q, int32_t k) {
    g_last_error.clear();
    return run_host(1, false, Q, f, nullptr, 1, labels, vals, ic_map, R, n_g, n_l, n_q, k);
}

int cf_contract_host(double* Q, const double* f, int64_t b, const double* labels, const double* vals,
                     const double* ic_map, const double* R, int64_t n_g, int32_t n_l, int32_t n_q, int32_t k,
                     int32_t form) {
    g_last_error.clear();
    bool exact = false, sym = false;
    int f32 = 0;
    const int what = form_what(form, exact, sym, f32);
    if (what < 0) return fail(CF_EINVAL, "unknown form %d", form);
    return run_host(what, exact, Q, f, nullptr, b, labels, vals, ic_map, R, n_g, n_l, n_q, k, sym, f32);
}

int cf_time_contract_host(int64_t n_calls, double* seconds, double* Q, const double* f, int64_t b,
                          const double* labels, const double* vals, const double* ic_map, const double* R,
                          int64_t n_g, int32_t n_l, int32_t n_q, int32_t k, int32_t form) {
    if (!seconds || n_calls < 0) return fail(CF_EINVAL, "null seconds or negative n_calls");
    *seconds = 0.0;
    const auto t0 = std::chrono::steady_clock::now();
    for (int64_t i = 0; i < n_calls; ++i) {
        const int st = cf_contract_host(Q, f, b, labels, vals, ic_map, R, n_g, n_l, n_q, k, form);
        if (st != CF_OK) return st;
    }
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return CF_OK;
}

int cf_jacobian_apply_host(double* out, const double* f, const double* v, int64_t b, const double* labels,
                           const double* vals, const double* ic_map, const double* R, int64_t n_g, int32_t n_l,
                           int32_t n_q, int32_t k, int32_t exact) {
    g_last_error.clear();
    bool ex = false, sym = false;
    int f32 = 0;
    if (!jv_mode(exact, ex, sym, f32))
        return fail(CF_EINVAL, "J.v mode %d is not 0 (fast), 1 (exact), 2 (folded), 3 (FP32) or 4 (FP32 folded)", exact);
    return run_host(2, ex, out, f, v, b, labels, vals, ic_map, R, n_g, n_l, n_q, k, sym, f32);
}

int cf_plan_create(cf_plan** plan, const double* labels, const double* vals, const double* ic_map, const double* R,
                   int64_t n_g, int32_t n_l, int32_t n_q, int32_t k, int32_t device) {
    g_last_error.clear();
    return plan_create(plan, labels, vals, ic_map, R, n_g, n_l, n_q, k, device);
}

int cf_plan_destroy(cf_plan* plan) {
    if (!plan) return CF_OK;
    {
        std::lock_guard<std::mutex> lk(plan->mu);
        DeviceGuard g(plan->device);
        if (plan->stream) cudaStreamSynchronize(plan->stream);
        free_plan_memory(plan);
    }
    delete plan;
    return CF_OK;
}

int cf_plan_get_info(const cf_plan* plan, cf_plan_info* info) {
    if (!plan || !info) return fail(CF_EINVAL, "null argument");
    info->n_g = plan->n_g;
    info->n_slices = plan->n_slices;
    info->n_l = plan->n_l;
    info->n_q = plan->n_q;
    info->k = plan->k;
    info->device = plan->device;
    info->flops_q = plan->flops_q;
    info->flops_jv = plan->flops_jv;
    info->device_bytes = plan->dev_bytes + (int64_t)plan->ws_bytes + (int64_t)plan->io_bytes;
    info->last_path = plan->last_path;
    info->reserved = 0;
    return CF_OK;
}

int cf_plan_workspace_size(const cf_plan* plan, int64_t b, int32_t jacobian, size_t* bytes) {
    if (!plan || !bytes) return fail(CF_EINVAL, "null argument");
    if (b < 0) return fail(CF_ESHAPE, "B is negative");
    *bytes = tiled_bytes(plan, b) * (jacobian ? 3 : 2);
    return CF_OK;
}

int cf_q_device_ws(cf_plan* plan, double* q_dev, const double* f_dev, int64_t b, int32_t form, void* workspace,
                   size_t workspace_bytes, void* stream) {
    g_last_error.clear();
    if (!plan) return fail(CF_EINVAL, "null plan");
    bool exact = false, sym = false;
    int f32 = 0;
    const int what = form_what(form, exact, sym, f32);
    if (what < 0) return fail(CF_EINVAL, "unknown form %d", form);
    std::lock_guard<std::mutex> lk(plan->mu);
    DeviceGuard guard(plan->device);
    return run_device(plan, what, exact, q_dev, f_dev, nullptr, b, workspace, workspace_bytes, (cudaStream_t)stream,
                      sym, f32);
}

int cf_q_device(cf_plan* plan, double* q_dev, const double* f_dev, int64_t b, int32_t form, void* stream) {
    g_last_error.clear();
    if (!plan) return fail(CF_EINVAL, "null plan");
    bool exact = false, sym = false;
    int f32 = 0;
    const int what = form_what(form, exact, sym, f32);
    if (what < 0) return fail(CF_EINVAL, "unknown form %d", form);
    std::lock_guard<std::mutex> lk(plan->mu);
    DeviceGuard guard(plan->device);
    CF_TRY(ensure_ws(plan, tiled_bytes(plan, b) * 2));
    return run_device(plan, what, exact, q_dev, f_dev, nullptr, b, plan->d_ws, plan->ws_bytes, (cudaStream_t)stream,
                      sym, f32);
}

int cf_jv_device(cf_plan* plan, double* out_dev, const double* f_dev, const double* v_dev, int64_t b, int32_t exact,
                 void* stream) {
    g_last_error.clear();
    if (!plan) return fail(CF_EINVAL, "null plan");
    bool ex = false, sym = false;
    int f32 = 0;
    if (!jv_mode(exact, ex, sym, f32))
        return fail(CF_EINVAL, "J.v mode %d is not 0 (fast), 1 (exact), 2 (folded), 3 (FP32) or 4 (FP32 folded)", exact);
    std::lock_guard<std::mutex> lk(plan->mu);
    DeviceGuard guard(plan->device);
    CF_TRY(ensure_ws(plan, tiled_bytes(plan, b) * 3));
    return run_device(plan, 2, ex, out_dev, f_dev, v_dev, b, plan->d_ws, plan->ws_bytes, (cudaStream_t)stream, sym,
                      f32);
}

int cf_pack_cells(const cf_plan* plan, double* dst_tiled, const double* src_cells, int64_t b, void* stream) {
    g_last_error.clear();
    if (!plan) return fail(CF_EINVAL, "null plan");
    if (b < 0) return fail(CF_ESHAPE, "B is negative");
    if (b > 0 && (!dst_tiled || !src_cells)) return fail(CF_EINVAL, "null device buffer");
    DeviceGuard guard(plan->device);
    return launch_pack(plan, src_cells, dst_tiled, b, (cudaStream_t)stream);
}

int cf_unpack_cells(const cf_plan* plan, double* dst_cells, const double* src_tiled, int64_t b, void* stream) {
    g_last_error.clear();
    if (!plan) return fail(CF_EINVAL, "null plan");
    if (b < 0) return fail(CF_ESHAPE, "B is negative");
    if (b > 0 && (!dst_cells || !src_tiled)) return fail(CF_EINVAL, "null device buffer");
    DeviceGuard guard(plan->device);
    return launch_unpack(plan, src_tiled, dst_cells, b, (cudaStream_t)stream);
}

int cf_q_tiled(cf_plan* plan, double* q_tiled, const double* f_tiled, int64_t b, int32_t form, void* stream) {
    g_last_error.clear();
    if (!plan) return fail(CF_EINVAL, "null plan");
    bool exact = false, sym = false;
    int f32 = 0;
    const int what = form_what(form, exact, sym, f32);
    if (what < 0) return fail(CF_EINVAL, "unknown form %d", form);
    if (f32) return fail(CF_EUNSUPPORTED, "the FP32, BF16 and split forms read FP64 cells through cf_q_device / cf_contract_host");
    if (b < 0) return fail(CF_ESHAPE, "B is negative");
    if (b == 0 || plan->n_g == 0) return CF_OK;
    if (!q_tiled || !f_tiled) return fail(CF_EINVAL, "null device buffer");
    DeviceGuard guard(plan->device);
    cf_plan* target = plan;
    if (sym) CF_TRY(get_sym(plan, &target));
    return dispatch(target, what, exact, f_tiled, nullptr, q_tiled, b, (cudaStream_t)stream);
}

int cf_jv_tiled(cf_plan* plan, double* out_tiled, const double* f_tiled, const double* v_tiled, int64_t b,
                int32_t exact, void* stream) {
    g_last_error.clear();
    if (!plan) return fail(CF_EINVAL, "null plan");
    if (b < 0) return fail(CF_ESHAPE, "B is negative");
    if (b == 0 || plan->n_g == 0) return CF_OK;
    if (!out_tiled || !f_tiled || !v_tiled) return fail(CF_EINVAL, "null device buffer");
    bool ex = false, sym = false;
    int f32 = 0;
    if (!jv_mode(exact, ex, sym, f32))
        return fail(CF_EINVAL, "J.v mode %d is not 0 (fast), 1 (exact), 2 (folded), 3 (FP32) or 4 (FP32 folded)", exact);
    if (f32) return fail(CF_EUNSUPPORTED, "the FP32 J.v modes read FP64 cells through cf_jv_device / cf_jacobian_apply_host");
    DeviceGuard guard(plan->device);
    cf_plan* target = plan;
    if (sym) CF_TRY(get_sym(plan, &target));
    return dispatch(target, cf::OP_JV, ex, f_tiled, v_tiled, out_tiled, b, (cudaStream_t)stream);
}

}  // extern "C"

__attribute__((visibility("hidden"))) int cf_plan_internal_view(const cf_plan* plan, DevOp* op,
                                                                const int** pbin_begin, const int** pbin_item,
                                                                const int2** pitems, const int** bin_begin,
                                                                const int** bin_q1, int* n_sms, size_t* max_smem) {
    *op = plan->op();
    *pbin_begin = plan->d_pbin_begin;
    *pbin_item = plan->d_pbin_item;
    *pitems = plan->d_pitems;
    *bin_begin = plan->d_bin_begin;
    *bin_q1 = plan->d_bin_q1;
    *n_sms = plan->n_sms;
    *max_smem = plan->max_smem;
    return CF_OK;
}

// The plan's q2 <-> q3 folded twin (built on first use, owned by the plan).
__attribute__((visibility("hidden"))) int cf_plan_folded(cf_plan* plan, cf_plan** folded) {
    DeviceGuard guard(plan->device);
    return get_sym(plan, folded);
}

// Kernels launched by the other translation units (ragged.cu), for cf_launch_count().
__attribute__((visibility("hidden"))) void cf_add_launches(int64_t n) { g_launches += n; }

// Whether the folded twin exists already (building it allocates device memory).
__attribute__((visibility("hidden"))) bool cf_plan_folded_built(cf_plan* plan) {
    std::lock_guard<std::mutex> lk(plan->sym_mu);
    return plan->sym != nullptr;
}

// Whether a call in this form would first build the plan's band units (the tables of the band
// kernels, which allocate device memory): the BF16-split forms at K = 4 and 12 (and at K = 8 on path
// PATH_BAND), the fast FP64 forms on path PATH_BAND.  A folded form whose twin is not built yet
// answers false (that case is refused on its own).
__attribute__((visibility("hidden"))) bool cf_plan_band_pending(cf_plan* plan, int form) {
    bool exact = false, sym = false;
    int f32 = 0;
    if (form_what(form, exact, sym, f32) != 0 || exact || !cf::split_supported_k(plan->k)) return false;
    const bool band = plan->path == cf::PATH_BAND;
    const bool lblock = (plan->path == cf::PATH_LBLOCK && (plan->k == 8 || plan->k == 12)) ||
                        (plan->path == cf::PATH_AUTO && plan->k == 12);
    if (!((f32 == 2 && (plan->k != 8 || band)) || (f32 == 0 && (band || lblock)) || (f32 == 1 && lblock))) return false;
    cf_plan* target = plan;
    if (sym) {
        std::lock_guard<std::mutex> lk(plan->sym_mu);
        target = plan->sym;
    }
    if (!target) return false;
    std::lock_guard<std::mutex> lk(target->split_mu);
    return target->split == nullptr && target->split_status <= 0;
}

extern "C" {

int cf_plan_set_kernel_path(cf_plan* plan, int32_t path) {
    g_last_error.clear();
    if (!plan) return fail(CF_EINVAL, "null plan");
    if (path < 0 || (path > 6 && path != cf::PATH_BAND && path != cf::PATH_LBLOCK))
        return fail(CF_EINVAL,
                    "kernel path %d is not 0 (auto), 1 (gather), 2 (tile), 3 (pair), 4 (pair, R via L1), 5 (pair, "
                    "split rows), 6 (tile, K^3 step on the FP64 MMA), 11 (band) or 14 (l-block)",
                    path);
    std::lock_guard<std::mutex> lk(plan->mu);
    plan->path = path;
    if (plan->sym) plan->sym->path = path;
    return CF_OK;
}

int cf_plan_stream_selftest(cf_plan* plan, double wait_seconds) {
    g_last_error.clear();
    if (!plan) return fail(CF_EINVAL, "null plan");
    if (!(wait_seconds > 0.0 && wait_seconds <= 10.0)) return fail(CF_EINVAL, "wait_seconds must be in (0, 10]");
    std::lock_guard<std::mutex> lk(plan->mu);
    DeviceGuard guard(plan->device);
    if (!guard.ok) return fail(CF_ENODEVICE, "cannot select device %d", plan->device);
    if (plan->n_g == 0 || plan->k % 2 != 0 || plan->k > 8)
        return fail(CF_EUNSUPPORTED, "the streamed tile kernel needs an even K <= 8 and a non-empty operator");
    const int64_t B = 64;
    const size_t cell_bytes = (size_t)B * plan->n_q * plan->k * sizeof(double);
    CF_TRY(ensure_io(plan, 2 * cell_bytes));
    CF_TRY(ensure_stream_sync(plan));
    int khz = 0;
    CF_CUDA(cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, plan->device));
    const long long cycles = std::max(1LL, (long long)((double)std::max(khz, 1000000) * 1e3 * wait_seconds));
    double* dQ = plan->d_io;
    double* df = (double*)((char*)plan->d_io + cell_bytes);
    return run_host_streamed(plan, plan, nullptr, nullptr, B, dQ, df, false, cycles);
}

int cf_plan_lblock_selftest(cf_plan* plan, double wait_seconds) {
    g_last_error.clear();
    if (!plan) return fail(CF_EINVAL, "null plan");
    if (!(wait_seconds > 0.0 && wait_seconds <= 10.0)) return fail(CF_EINVAL, "wait_seconds must be in (0, 10]");
    std::lock_guard<std::mutex> lk(plan->mu);
    DeviceGuard guard(plan->device);
    if (!guard.ok) return fail(CF_ENODEVICE, "cannot select device %d", plan->device);
    if (plan->n_g == 0 || (plan->k != 8 && plan->k != 12))
        return fail(CF_EUNSUPPORTED, "the l-block kernel needs K = 8 or 12 and a non-empty operator");
    cf::SplitPlan* sp = nullptr;
    CF_TRY(get_split(plan, &sp));
    const int64_t B = 16;
    const size_t cell_bytes = (size_t)B * plan->n_q * plan->k * sizeof(double);
    CF_TRY(ensure_io(plan, 2 * cell_bytes));
    CF_TRY(ensure_ws(plan, tiled_bytes(plan, B) * 2));
    int khz = 0;
    CF_CUDA(cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, plan->device));
    const long long cycles = std::max(1LL, (long long)((double)std::max(khz, 1000000) * 1e3 * wait_seconds));
    double* dQ = plan->d_io;
    double* df = (double*)((char*)plan->d_io + cell_bytes);
    CF_CUDA(cudaMemsetAsync(plan->d_io, 0, 2 * cell_bytes, plan->stream));
    int64_t launches = 0;
    const int st = cf::lblock_selftest(sp, dQ, df, plan->d_ws, plan->ws_bytes, B, cycles, plan->stream, &launches);
    g_launches += launches;
    return st;
}

int cf_fp64_fma_peak(int32_t device, double* tflops) {
    g_last_error.clear();
    if (!tflops) return fail(CF_EINVAL, "null output");
    CF_TRY(check_device_available());
    DeviceGuard guard(device);
    if (!guard.ok) return fail(CF_ENODEVICE, "cannot select device %d", device);
    int sms = 0;
    CF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int blocks = sms * 8, threads = 256, iters = 4096;
    double* sink = nullptr;
    CF_CUDA(cudaMalloc(&sink, sizeof(double) * blocks * threads));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 6; ++rep) {
        cudaEventRecord(e0);
        cf::fp64_fma_probe_kernel<<<blocks, threads>>>(sink, iters, 1.0 + 1e-12 * rep);
        g_launches++;
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0) best = std::min(best, ms);
    }
    const cudaError_t e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (e != cudaSuccess) return fail(CF_ECUDA, "probe: %s", cudaGetErrorString(e));
    const double flops = 2.0 * cf::kProbeChains * (double)iters * blocks * threads;
    *tflops = flops / (best * 1e-3) / 1e12;
    return CF_OK;
}

const char* cf_status_string(int status) {
    switch (status) {
        case CF_OK: return "ok";
        case CF_EINVAL: return "invalid argument";
        case CF_ESHAPE: return "inconsistent sizes";
        case CF_EBADIDX: return "index out of range";
        case CF_ENONFINITE: return "non-finite operator value";
        case CF_ECUDA: return "CUDA error";
        case CF_ENOMEM: return "out of memory";
        case CF_ENODEVICE: return "no usable CUDA device";
        case CF_EUNSUPPORTED: return "unsupported form or size";
        case CF_ETIMEOUT: return "device wait timed out";
        default: return "unknown status";
    }
}

const char* cf_last_error(void) { return g_last_error.c_str(); }
int64_t cf_launch_count(void) { return g_launches.load(); }
int cf_few_route_last(void) { return g_few_route; }
const char* cf_version(void) { return "cf_b200 0.1 (sm_100a)"; }

}  // extern "C"
