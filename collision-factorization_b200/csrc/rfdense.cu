// rfdense.cu -- the radial-first form with its radial step as a dense GEMM over cells
// (CF_FORM_RF_DENSE).
//
// The reference's radial-first kernel (radial_first_collision_kernel_mex.cpp:41-59) forms, per COO
// entry z of l-triplet t,  Psi[z][k1] = sum_{k2,k3} R_t[k1,k2,k3] f[q2,k2] f[q3,k3]  (K^3 per entry),
// then routes  Q[q1][k1] += G_z Psi[z][k1]  (:64-73).  Here the k2 sum is factored out of the
// entries: for every pair (t, q2) and cell b,
//
//     C_{t,q2}[k1,k3; b] = sum_k2 R_t[k1,k2,k3] f[q2,k2; b]           (step 1)
//
// is one dense [K^2 x K] x [K x cells] product shared by every entry of the pair, and each entry
// then costs K^2 per cell:
//
//     Q[q1,k1; b] += G_z sum_k3 C_{t,q2}[k1,k3; b] f[q3,k3; b]         (step 2)
//
// Work per cell: pairs x 2K^3 + N_G x 2K^2 (on the folded operator at L = 16, K = 12: 11 313 pairs and
// 302 389 entries, 126 MFLOP, against 111 MFLOP for the angular-first form grouped by q2).
//
// Kernel: a CTA owns 32 cells (one per lane) and a part of the l-triplet list of one l1 band; warp w
// is row k1 = w.  Per t: R_t is staged in shared memory; per pair (t, q2) each lane forms its row of
// C (K^2 FMAs, R_t read warp-uniform) and keeps it in registers; per entry it reads f(q3) (one
// coalesced 256-byte load per k3 across the warp) and adds G sum_k3 C f(q3) into its own slot of
// the band's Q rows in shared memory.  The band's parts write partial sums, which a second kernel
// adds into Q in a fixed order (deterministic, no atomics).  f is first packed cell-fastest,
// [k][q][cell], so that every load is coalesced over the warp's 32 cells.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/cf_b200.h"
#include "rfdense.cuh"

void cf_set_last_error(const char* msg);

namespace cf {

namespace {

constexpr int kCellsPerCta = 32;

struct RfUnit {
    int l1;      // band
    int t0, t1;  // range of the band's l-triplets in band_t
    long long part_off;  // the unit's partial sums start at part_off x (padded cells) doubles
};

struct RfArgs {
    const RfUnit* units;
    const int* unit_order;   // units, heaviest first
    const int* band_t;       // l-triplets of each band, band after band
    const int* t_pair;       // [n_l + 1] pair range of each l-triplet
    const int* pair_q2;      // q2 of each pair
    const int* pair_e;       // [n_pairs + 1] entry range of each pair
    const uint32_t* ent_q13;  // q1 - l1^2 | q3 << 16, per entry, grouped by pair
    const double* ent_g;     // G per entry
    const double* R;         // R_t[k1 + K k2 + K^2 k3 + K^3 t]
    const double* F;         // packed f: [k][q][cell], cells padded to a multiple of 32
    double* part;            // partial sums
    int n_cb;                // cell blocks (padded cells / 32)
    int n_q;
    long long bp;            // padded cells
};

// f (cell-major [B][K][N_Q]) -> F[(k N_Q + q) bp + cell], zero past the batch.
__global__ void rf_pack_kernel(const double* __restrict__ f, double* __restrict__ F, long long B, long long bp, int M) {
    const long long n = (long long)M * bp;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long cell = i % bp, r = i / bp;  // r = k N_Q + q: the cell-major element index
        F[i] = cell < B ? f[cell * M + r] : 0.0;
    }
}

template <int K>
__global__ void __launch_bounds__(K * 32) rf_dense_kernel(RfArgs a) {
    extern __shared__ __align__(16) double smem[];
    const int u = a.unit_order[blockIdx.x / a.n_cb], cb = blockIdx.x % a.n_cb;
    const RfUnit un = a.units[u];
    const int nq1 = 2 * un.l1 + 1;
    double* Rs = smem;                 // K^3
    double* Qs = smem + K * K * K;     // [q1 - l1^2][k1][lane]
    const int tid = threadIdx.x, k1 = tid >> 5, lane = tid & 31;
    for (int i = tid; i < nq1 * K * kCellsPerCta; i += K * 32) Qs[i] = 0.0;
    const long long cell = (long long)cb * kCellsPerCta + lane;
    const double* __restrict__ Fc = a.F + cell;
    const long long qstride = a.bp;    // next q
    const long long kstride = (long long)a.n_q * a.bp;  // next k
    for (int ti = un.t0; ti < un.t1; ++ti) {
        const int t = a.band_t[ti];
        __syncthreads();  // the previous t's reads of Rs are done
        for (int i = tid; i < K * K * K; i += K * 32) Rs[i] = __ldg(a.R + (size_t)t * K * K * K + i);
        __syncthreads();
        const int p1 = __ldg(a.t_pair + t + 1);
        for (int p = __ldg(a.t_pair + t); p < p1; ++p) {
            const int q2 = __ldg(a.pair_q2 + p);
            double f2[K];
#pragma unroll
            for (int k2 = 0; k2 < K; ++k2) f2[k2] = __ldg(Fc + k2 * kstride + q2 * qstride);
            // row k1 of C_{t,q2} for this lane's cell
            double c[K];
#pragma unroll
            for (int k3 = 0; k3 < K; ++k3) {
                double s = 0.0;
#pragma unroll
                for (int k2 = 0; k2 < K; ++k2) s = fma(Rs[k1 + K * k2 + K * K * k3], f2[k2], s);
                c[k3] = s;
            }
            const int e1 = __ldg(a.pair_e + p + 1);
            for (int e = __ldg(a.pair_e + p); e < e1; ++e) {
                const uint32_t w = __ldg(a.ent_q13 + e);
                const double g = __ldg(a.ent_g + e);
                const int q1l = (int)(w & 0xffffu), q3 = (int)(w >> 16);
                double s = 0.0;
#pragma unroll
                for (int k3 = 0; k3 < K; ++k3) s = fma(c[k3], __ldg(Fc + k3 * kstride + q3 * qstride), s);
                double& qv = Qs[(q1l * K + k1) * kCellsPerCta + lane];
                qv = fma(g, s, qv);
            }
        }
    }
    __syncthreads();
    // partial sums of this unit and cell block: part[part_off + (cell K + k1) nq1 + q1l]
    const int n = kCellsPerCta * K * nq1;
    double* pb = a.part + un.part_off * a.bp + (long long)cb * kCellsPerCta * K * nq1;
    for (int i = tid; i < n; i += K * 32) {
        const int c = i / (K * nq1), r = i % (K * nq1), kk = r / nq1, q1l = r % nq1;
        pb[i] = Qs[(q1l * K + kk) * kCellsPerCta + c];
    }
}

// Q[cell][k1][q1] += the band's partial sums of (cell, k1, q1), its units in order.
__global__ void rf_reduce_kernel(const RfUnit* __restrict__ units, const int* __restrict__ band_u, const double* __restrict__ part,
                                 double* __restrict__ q, long long B, long long bp, int n_q, int K) {
    const long long n = B * n_q;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long cell = i / n_q;
        const int q1 = (int)(i % n_q);
        int l1 = (int)sqrtf((float)q1);
        while (l1 * l1 > q1) --l1;
        while ((l1 + 1) * (l1 + 1) <= q1) ++l1;
        const int nq1 = 2 * l1 + 1, q1l = q1 - l1 * l1;
        const int u0 = band_u[l1], u1 = band_u[l1 + 1];
        for (int k1 = 0; k1 < K; ++k1) {
            double s = 0.0;
            for (int uu = u0; uu < u1; ++uu) s += part[units[uu].part_off * bp + (cell * K + k1) * nq1 + q1l];
            if (u1 > u0) q[cell * (long long)K * n_q + (long long)k1 * n_q + q1] += s;
        }
    }
}

int fail_rf(int st, const std::string& msg) {
    cf_set_last_error(msg.c_str());
    return st;
}

template <typename T>
cudaError_t upload(T** dst, const std::vector<T>& v, int64_t& bytes) {
    *dst = nullptr;
    const size_t n = std::max<size_t>(v.size(), 1);
    cudaError_t e = cudaMalloc((void**)dst, n * sizeof(T));
    if (e != cudaSuccess) return e;
    bytes += (int64_t)(n * sizeof(T));
    if (!v.empty()) e = cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    return e;
}

template <typename T>
cudaError_t download(std::vector<T>& v, const T* src, size_t n) {
    v.resize(n);
    return n ? cudaMemcpy(v.data(), src, n * sizeof(T), cudaMemcpyDeviceToHost) : cudaSuccess;
}

int isqrt_i(int q) {
    int l = (int)std::sqrt((double)q);
    while (l * l > q) --l;
    while ((l + 1) * (l + 1) <= q) ++l;
    return l;
}

}  // namespace

struct RfDensePlan {
    int device = 0, k = 0, n_q = 0, L = 0, n_units = 0;
    int64_t bytes = 0;
    const double* R = nullptr;  // borrowed from the plan's operator
    RfUnit* d_units = nullptr;
    int* d_unit_order = nullptr;
    int* d_band_t = nullptr;
    int* d_t_pair = nullptr;
    int* d_pair_q2 = nullptr;
    int* d_pair_e = nullptr;
    uint32_t* d_ent_q13 = nullptr;
    double* d_ent_g = nullptr;
    int* d_band_u = nullptr;
    long long part_per_cell = 0;   // sum over units of K (2 l1 + 1)
    int max_nq1 = 1;
    // scratch, grown on demand: packed f and the partial sums for cap_bp padded cells
    double* d_F = nullptr;
    double* d_part = nullptr;
    long long cap_bp = 0;
    cudaEvent_t done = nullptr;     // the last run's completion (orders runs on different streams)
    bool have_done = false;
};

bool rfdense_supported_k(int k) { return k >= 1 && k <= 16; }

int rfdense_build(RfDensePlan** out, const DevOp& op, int64_t n_g, int64_t n_slices, int device) {
    *out = nullptr;
    const int K = op.k, NQ = op.n_q, NL = op.n_l;
    if (!rfdense_supported_k(K)) return fail_rf(CF_EUNSUPPORTED, "radial-first dense form: K must be 1 .. 16");
    const int L = isqrt_i(NQ) - 1;
    if ((L + 1) * (L + 1) != NQ) return fail_rf(CF_EUNSUPPORTED, "radial-first dense form: N_Q is not (L+1)^2");
    std::vector<int> q1_begin, slice_t, slice_e;
    std::vector<uint32_t> e_q23;
    std::vector<double> e_g;
    cudaError_t ce = download(q1_begin, op.q1_begin, (size_t)NQ + 1);
    if (ce == cudaSuccess) ce = download(slice_t, op.slice_t, (size_t)n_slices);
    if (ce == cudaSuccess) ce = download(slice_e, op.slice_e, (size_t)n_slices + 1);
    if (ce == cudaSuccess) ce = download(e_q23, op.e_q23, (size_t)n_g);
    if (ce == cudaSuccess) ce = download(e_g, op.e_g, (size_t)n_g);
    if (ce != cudaSuccess) return fail_rf(CF_ECUDA, std::string("radial-first dense form: download: ") + cudaGetErrorString(ce));

    // entries regrouped per l-triplet by (q2, q1, q3), keeping the operator's order within equal keys
    struct Ent {
        int t, q2, q1, q3;
        double g;
        int64_t z;
    };
    std::vector<Ent> ents;
    ents.reserve((size_t)n_g);
    std::vector<int> t_l1(NL, -1);
    for (int q = 0; q < NQ; ++q)
        for (int s = q1_begin[q]; s < q1_begin[q + 1]; ++s) {
            const int t = slice_t[s];
            const int l1 = isqrt_i(q);
            if (t_l1[t] >= 0 && t_l1[t] != l1)
                return fail_rf(CF_EUNSUPPORTED, "radial-first dense form: an l-triplet spans two l1 bands");
            t_l1[t] = l1;
            for (int z = slice_e[s]; z < slice_e[s + 1]; ++z)
                ents.push_back({t, (int)(e_q23[z] & 0xffffu), q, (int)(e_q23[z] >> 16), e_g[z], z});
        }
    std::stable_sort(ents.begin(), ents.end(), [](const Ent& x, const Ent& y) {
        if (x.t != y.t) return x.t < y.t;
        if (x.q2 != y.q2) return x.q2 < y.q2;
        if (x.q1 != y.q1) return x.q1 < y.q1;
        return x.q3 < y.q3;
    });
    std::vector<int> t_pair(NL + 1, 0), pair_q2, pair_e;
    std::vector<uint32_t> ent_q13(ents.size());
    std::vector<double> ent_g(ents.size());
    std::vector<double> t_work(NL, 0.0);
    for (size_t i = 0; i < ents.size(); ++i) {
        const Ent& e = ents[i];
        if (i == 0 || e.t != ents[i - 1].t || e.q2 != ents[i - 1].q2) {
            pair_q2.push_back(e.q2);
            pair_e.push_back((int)i);
            t_work[e.t] += (double)K * K * K;
        }
        const int l1 = t_l1[e.t];
        ent_q13[i] = (uint32_t)(e.q1 - l1 * l1) | ((uint32_t)e.q3 << 16);
        ent_g[i] = e.g;
        t_work[e.t] += (double)K * K;
    }
    pair_e.push_back((int)ents.size());
    {
        size_t p = 0;
        for (int t = 0; t < NL; ++t) {
            t_pair[t] = (int)p;
            while (p < pair_q2.size() && ents[pair_e[p]].t == t) ++p;
        }
        t_pair[NL] = (int)pair_q2.size();
    }
    // units: each band's l-triplets in parts of about equal work, about 48 parts in all
    double total = 0.0;
    for (int t = 0; t < NL; ++t) total += t_work[t];
    const double target = std::max(total / 48.0, 1.0);
    std::vector<int> band_t, band_u(L + 2, 0);
    std::vector<RfUnit> units;
    std::vector<double> unit_work;
    long long part_per_cell = 0;
    int max_nq1 = 1;
    for (int l1 = 0; l1 <= L; ++l1) {
        band_u[l1] = (int)units.size();
        const int b0 = (int)band_t.size();
        for (int t = 0; t < NL; ++t)
            if (t_l1[t] == l1) band_t.push_back(t);
        const int b1 = (int)band_t.size();
        double w = 0.0;
        int start = b0;
        for (int i = b0; i < b1; ++i) {
            w += t_work[band_t[i]];
            if (w >= target || i == b1 - 1) {
                units.push_back({l1, start, i + 1, part_per_cell});
                unit_work.push_back(w);
                part_per_cell += (long long)K * (2 * l1 + 1);
                max_nq1 = std::max(max_nq1, 2 * l1 + 1);
                w = 0.0;
                start = i + 1;
            }
        }
    }
    band_u[L + 1] = (int)units.size();
    std::vector<int> order(units.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return unit_work[x] > unit_work[y]; });

    RfDensePlan* rp = new RfDensePlan();
    rp->device = device;
    rp->k = K;
    rp->n_q = NQ;
    rp->L = L;
    rp->R = op.R;
    rp->n_units = (int)units.size();
    rp->part_per_cell = part_per_cell;
    rp->max_nq1 = max_nq1;
    int64_t bytes = 0;
    if ((ce = upload(&rp->d_units, units, bytes)) != cudaSuccess ||
        (ce = upload(&rp->d_unit_order, order, bytes)) != cudaSuccess ||
        (ce = upload(&rp->d_band_t, band_t, bytes)) != cudaSuccess ||
        (ce = upload(&rp->d_t_pair, t_pair, bytes)) != cudaSuccess ||
        (ce = upload(&rp->d_pair_q2, pair_q2, bytes)) != cudaSuccess ||
        (ce = upload(&rp->d_pair_e, pair_e, bytes)) != cudaSuccess ||
        (ce = upload(&rp->d_ent_q13, ent_q13, bytes)) != cudaSuccess ||
        (ce = upload(&rp->d_ent_g, ent_g, bytes)) != cudaSuccess ||
        (ce = upload(&rp->d_band_u, band_u, bytes)) != cudaSuccess ||
        (ce = cudaEventCreateWithFlags(&rp->done, cudaEventDisableTiming)) != cudaSuccess) {
        rfdense_destroy(rp);
        return fail_rf(ce == cudaErrorMemoryAllocation ? CF_ENOMEM : CF_ECUDA,
                       std::string("radial-first dense form: upload: ") + cudaGetErrorString(ce));
    }
    rp->bytes = bytes;
    *out = rp;
    return CF_OK;
}

void rfdense_destroy(RfDensePlan* rp) {
    if (!rp) return;
    void* ptrs[] = {rp->d_units, rp->d_unit_order, rp->d_band_t, rp->d_t_pair, rp->d_pair_q2, rp->d_pair_e,
                    rp->d_ent_q13, rp->d_ent_g, rp->d_band_u, rp->d_F, rp->d_part};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (rp->done) cudaEventDestroy(rp->done);
    delete rp;
}

int64_t rfdense_device_bytes(const RfDensePlan* rp) { return rp ? rp->bytes : 0; }

namespace {

template <int K>
int launch_rf(RfDensePlan* rp, const RfArgs& a, unsigned blocks, cudaStream_t st) {
    const size_t smem = ((size_t)K * K * K + (size_t)rp->max_nq1 * K * kCellsPerCta) * sizeof(double);
    static bool attr_set[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        const cudaError_t e =
            cudaFuncSetAttribute(rf_dense_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        if (e != cudaSuccess) return fail_rf(CF_ECUDA, std::string("radial-first dense form: ") + cudaGetErrorString(e));
        attr_set[dev] = true;
    }
    if (smem > 227 * 1024) return fail_rf(CF_EUNSUPPORTED, "radial-first dense form: the band's Q rows do not fit");
    rf_dense_kernel<K><<<blocks, K * 32, smem, st>>>(a);
    return CF_OK;
}

}  // namespace

int rfdense_run(RfDensePlan* rp, double* q_cm, const double* f_cm, int64_t B, cudaStream_t st, int64_t* launches) {
    if (B <= 0 || rp->n_units == 0) return CF_OK;
    const int K = rp->k, NQ = rp->n_q, M = NQ * K;
    const long long bp = (B + kCellsPerCta - 1) / kCellsPerCta * kCellsPerCta;
    if (rp->have_done) {
        const cudaError_t e = cudaStreamWaitEvent(st, rp->done, 0);
        if (e != cudaSuccess) return fail_rf(CF_ECUDA, std::string("radial-first dense form: ") + cudaGetErrorString(e));
    }
    if (bp > rp->cap_bp) {
        // grow the scratch: packed f and the partial sums for bp cells (after the last run is done)
        if (rp->have_done) cudaEventSynchronize(rp->done);
        cudaFree(rp->d_F);
        cudaFree(rp->d_part);
        rp->d_F = rp->d_part = nullptr;
        rp->cap_bp = 0;
        cudaError_t e = cudaMalloc(&rp->d_F, (size_t)M * bp * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&rp->d_part, (size_t)rp->part_per_cell * bp * sizeof(double));
        if (e != cudaSuccess)
            return fail_rf(e == cudaErrorMemoryAllocation ? CF_ENOMEM : CF_ECUDA,
                           std::string("radial-first dense form: scratch: ") + cudaGetErrorString(e));
        rp->cap_bp = bp;
    }
    rf_pack_kernel<<<std::min<long long>((M * bp + 255) / 256, 148LL * 16), 256, 0, st>>>(f_cm, rp->d_F, B, bp, M);
    RfArgs a{};
    a.units = rp->d_units;
    a.unit_order = rp->d_unit_order;
    a.band_t = rp->d_band_t;
    a.t_pair = rp->d_t_pair;
    a.pair_q2 = rp->d_pair_q2;
    a.pair_e = rp->d_pair_e;
    a.ent_q13 = rp->d_ent_q13;
    a.ent_g = rp->d_ent_g;
    a.R = rp->R;
    a.F = rp->d_F;
    a.part = rp->d_part;
    a.n_cb = (int)(bp / kCellsPerCta);
    a.n_q = NQ;
    a.bp = bp;
    const long long blocks = (long long)rp->n_units * a.n_cb;
    if (blocks > 0x7fffffffLL) return fail_rf(CF_ESHAPE, "radial-first dense form: batch too large for one launch");
    int s = CF_OK;
    switch (K) {
#define CF_RF_CASE(k) \
    case k: s = launch_rf<k>(rp, a, (unsigned)blocks, st); break;
        CF_RF_CASE(1) CF_RF_CASE(2) CF_RF_CASE(3) CF_RF_CASE(4) CF_RF_CASE(5) CF_RF_CASE(6) CF_RF_CASE(7)
        CF_RF_CASE(8) CF_RF_CASE(9) CF_RF_CASE(10) CF_RF_CASE(11) CF_RF_CASE(12) CF_RF_CASE(13) CF_RF_CASE(14)
        CF_RF_CASE(15) CF_RF_CASE(16)
#undef CF_RF_CASE
        default: s = fail_rf(CF_EUNSUPPORTED, "radial-first dense form: K must be 1 .. 16");
    }
    if (s != CF_OK) return s;
    rf_reduce_kernel<<<std::min<long long>((B * NQ + 255) / 256, 148LL * 16), 256, 0, st>>>(rp->d_units, rp->d_band_u,
                                                                                        rp->d_part, q_cm, B, bp, NQ, K);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecord(rp->done, st);
    if (e != cudaSuccess) return fail_rf(CF_ECUDA, std::string("radial-first dense form: launch: ") + cudaGetErrorString(e));
    rp->have_done = true;
    if (launches) *launches += 3;
    return CF_OK;
}

}  // namespace cf
