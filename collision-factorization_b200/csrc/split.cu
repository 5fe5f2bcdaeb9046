// split.cu -- the exact-split form CF_FORM_AF_SYM_I8: Q(f) to ~1e-11 with the K^3 step on the
// int8 tensor cores.
//
// What is computed (angular first on the q2 <-> q3 folded operator, as CF_FORM_AF_SYM):
//
//   Q[q1,k1] += sum_t sum_kk R_t[k1,kk] Phi_{t,q1}[kk],  Phi_{t,q1} = sum_z G_z f[q2] (x) f[q3]
//
// (src/mex/angular_first_collision_kernel_mex.cpp:45-69 is the reference's per-slice loop).  The
// Phi step runs in FP64 on the CUDA cores.  The K^3 step is a sum of products with exact integer
// operands on the tensor cores:
//
//   * R_t is scaled by a power of two s_t so that |R_t s_t| < 1 (1/s_t goes into G), rounded to
//     R_int = rint(R_t s_t 2^46) and written as six balanced signed bytes r_0..r_5 at plan time;
//   * Phi' = sum_z (G_z / s_t) f (x) f of one (row, cell) is scaled by 2^e, e fixed per (row, cell)
//     from an a-priori bound (below) so that |X| < 2^47, X = rint(Phi' 2^e), and X is split into its
//     two's-complement bytes a_0..a_4 (unsigned) and a_5 (signed);
//   * sum_kk X R_int = sum_{i,j} 2^{8(i+j)} sum_kk a_i r_j: every product of bytes is exact, and the
//     sums over kk accumulate exactly in int32 (tcgen05.mma kind::i8) in tensor memory, one
//     accumulator block per weight d = i + j over the whole t-list of a row group;
//   * the blocks are recombined in FP64: Q += sum_d 2^{8d} D_d / 2^{e+46}.  Blocks d < 4 (weights
//     below 2^-48 of the top) are not formed.
//
// The bound: |Phi'_{t,q1}[kk]| <= (sum_z |G_z/s_t|) * max|f(band l2)| * max|f(band l3)|, where the
// band maxima are taken over the cell's staged coefficients; e = 46 - ceil(log2(bound over the
// row's slices)).  The error left is the rounding of X and R_int: measured 1.1e-11 of max|Q| on the
// hard-sphere L = 10, K = 8 operator against 5.6e-10 with one more block dropped.
//
// Work decomposition: a CTA (16 warps) owns C cells (4, or 8 at K = 8 where their f fits; f resident
// in shared memory) and a row group of one l1 band: up to 16 "slots" (a row, or a contiguous chunk of
// a row's entries when a band has few rows), one per warp.  The band's l-triplets t are walked in
// order; per t every warp computes its slot's Phi (C cells x 32/C lanes, each lane a part of K^2: a
// (k2 half, k3 quarter) for C = 4, a k3 quarter for C = 8), quantises it, and its six byte planes go
// into a shared-memory A buffer (M = 16 C rows: 16 slots x C cells; two buffers where shared memory
// allows).  After one barrier, one thread issues, per plane and 32-byte
// K step, one MMA against a window of the six R planes (B, staged per t into a 2-deep ring by one
// cp.async.bulk each), into the accumulator blocks d = i + j the window reaches.
// Accumulators are drained when the row group is done (or earlier, before int32 could overflow),
// and the slots of one row are summed in a fixed order, so results are deterministic.
//
// Every wait (mbarriers of the copies and of the MMAs) is bounded by a clock budget; a CTA that
// gives up records an error word, stops issuing work and leaves through the normal exit path.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/cf_b200.h"
#include "split.cuh"
#include "tc05.cuh"

void cf_set_last_error(const char* msg);

namespace cf {

namespace {

constexpr int kSlots = 16;       // row slots per CTA, one per warp
constexpr int kWarps = 16;
constexpr int kThreads = kWarps * 32;
constexpr int kPlanes = 6;       // bytes of X and of R_int
constexpr int kDMin = 4;         // lowest block weight kept
constexpr int kNB = 16;          // B rows per R plane (k1, padded)
constexpr int kDBlocks = 11 - kDMin;
constexpr int kTmemCols = 128;   // >= kDBlocks * kNB = 112
constexpr int kBRing = 2;
constexpr int kBStep = kPlanes * kNB * 32;  // one K step of the six R planes
constexpr int kRShift = 46;               // R_int = rint(R_t s_t 2^46)
constexpr int kXBits = 46;                // |X| <= 2^46 (1 bit of margin below the 47 the bytes hold)
constexpr long long kWaitCycles = 2000000000LL;  // ~1 s of SM clock per wait

// Per (K, C): C cells per CTA (4, or 8 at K = 8), P = 32 / C lanes per cell, each lane holding a part of
// the K x K Phi: (k2 half, k3 quarter) for P = 8, a k3 quarter for P = 4.
template <int K, int C>
struct Shape {
    static_assert((C == 4 && K % 4 == 0 && K <= 12) || (C == 8 && (K == 8 || K == 12)),
                  "the band kernels take K in {4, 8, 12} with 4 cells per CTA, or K = 8 and 12 with 8");
    static constexpr int P = 32 / C;                // lanes (parts) per cell
    static constexpr int KH = P == 8 ? K / 2 : K;   // k2 per lane
    static constexpr int KQ = K / 4;                // k3 per lane
    static constexpr int E = KH * KQ;               // Phi elements per lane
    static constexpr int EP = (E + 3) / 4 * 4;      // bytes per lane in a plane (word aligned)
    static constexpr int KK = P * EP;               // K dimension of the MMA (kk = part * EP + e)
    static constexpr int NKS = KK / 32;             // 32-byte K steps of the int8 planes (whole
                                                    // steps checked where they are used)
    static constexpr int M = 16 * C;                // MMA rows: 16 slots x C cells
    static constexpr int ATILE = M * 32;            // one 32-byte K step of an A plane
    static constexpr int PS = E * K + 2;            // FP64 R: doubles per part (16 bytes of padding
                                                    // keep the parts' 16-byte loads on distinct banks)
    static constexpr int RT_BYTES = P * PS * 8;     // FP64 R_t of one t
    // the first k2 and k3 of part p
    __host__ __device__ static constexpr int k2_of(int p) { return P == 8 ? (p & 1) * KH : 0; }
    __host__ __device__ static constexpr int k3_of(int p) { return P == 8 ? (p >> 1) * KQ : p * KQ; }
};

struct SplitArgs {
    const int* slice_e;
    const uint32_t* e_q23;
    const double* e_gs;        // G_z / s_t, in slice order (the split kernel)
    const double* e_g;         // G_z, in slice order (the FP64 band kernel)
    const double* rfp64;       // FP64 R_t per t as [part][e][k1], parts kPartStride<K> doubles apart
    const uint8_t* rplanes;    // [t][NKS][K step: 6 planes x 16 rows x 32 bytes, canonical]
    const uint8_t* rbf;        // [t][NKS][K step: R hi, R lo, each 16 rows x 16 BF16, canonical]
    const int* rb_off;         // per row q1: its slices' bound factors at rb_off[q1] .. rb_off[q1 + 1]
    const double* rb_gs;       // per slice of a row: sum |G_z / s_t|
    const int* rb_l23;         // per slice of a row: l2 | l3 << 8 of its l-triplet
    const int* units;          // per row group: 8 ints (unit_*)
    const int* unit_order;     // row groups, heaviest first
    const int* band_tl;        // t-lists of the bands
    const int* band_rng;       // per band: [n_t][2 l1 + 1] the slice's entries (begin, end) as int2, (0, 0) if none
    const double* f;           // cell-major [B][K][N_Q]
    double* q;
    int* err;
    long long n_cells;
    int n_cg;                  // cell groups: ceil(B / 4)
    int n_q, L;
    int tseg;                  // t per accumulation segment (int32 bound)
    int n_abuf;                // A buffers of six planes each (2 where shared memory allows, else 1)
    // the l-block kernel: f packed per cell group as [q][k][cell], one stage per l-triplet
    const double* pf;          // [n_cg][N_Q][K][C]
    const int* t_l23;          // per l-triplet: l2 | l3 << 8
    int n_ring, stage_bytes;   // stages in the ring, bytes per stage (R_t first, then the f rows)
    const int4* items;         // per band, its (t, row) slices in t-major order (lbi_*)
    const int* t_items;        // per t-list position of a band: its number of items
    int max_rows, max_t;       // sizes of the per-CTA row and t tables
    long long wait_cycles;     // the l-block kernel's budget per bounded wait (SM clocks)
    int no_copy;               // self-test: no stage is ever filled, so every wait runs out
    // shared-memory offsets (bytes)
    int off_a, off_b, off_f, off_mb, off_red, off_scale, off_eexp, off_bar, off_misc;
};

enum { U_L1 = 0, U_R0, U_NR, U_S, U_TLOFF, U_NT, U_TABOFF, U_BROWS, U_REM, U_INTS };

struct Layout {
    int off_a, off_b, off_f, off_mb, off_red, off_scale, off_eexp, off_bar, off_misc, total;
};

template <int K, int C>
Layout smem_layout(int n_q, int L, int n_abuf) {
    using S = Shape<K, C>;
    Layout l{};
    int o = 0;
    auto take = [&](int bytes, int align) {
        o = (o + align - 1) / align * align;
        const int r = o;
        o += bytes;
        return r;
    };
    l.off_a = take(n_abuf * kPlanes * S::NKS * S::ATILE, 1024);
    l.off_b = take(kBRing * S::NKS * kBStep, 1024);
    l.off_f = take(C * n_q * K * (int)sizeof(double), 16);
    l.off_mb = take(C * (L + 1) * (int)sizeof(double), 16);
    l.off_red = take(kSlots * C * K * (int)sizeof(double), 16);
    l.off_scale = take(kSlots * C * (int)sizeof(double), 16);
    l.off_eexp = take(kSlots * C * (int)sizeof(int), 16);
    l.off_bar = take(16 * (int)sizeof(uint64_t), 16);
    l.off_misc = take(16 * (int)sizeof(int), 16);
    l.total = o;
    return l;
}

// Warps per CTA of the FP64 band kernel.  16 at every K: its K^3 step keeps K accumulators and a part
// of Phi (18 doubles at K = 12) live, so more warps (64 or 80 registers each) spill hundreds of bytes.
__host__ __device__ constexpr int band64_warps(int) { return 16; }

template <int K, int C>
Layout band64_layout(int n_q, int warps) {
    using S = Shape<K, C>;
    Layout l{};
    int o = 0;
    auto take = [&](int bytes, int align) {
        o = (o + align - 1) / align * align;
        const int r = o;
        o += bytes;
        return r;
    };
    l.off_b = take(2 * S::RT_BYTES, 1024);
    l.off_f = take(C * n_q * K * (int)sizeof(double), 16);
    l.off_red = take(warps * C * K * (int)sizeof(double), 16);
    l.off_bar = take(16 * (int)sizeof(uint64_t), 16);
    l.off_misc = take(16 * (int)sizeof(int), 16);
    l.total = o;
    return l;
}

// The l-block kernels (K = 8 and 12): 16 warps, a ring of up to 8 stages; 8 cells per CTA in FP64,
// 16 in FP32 (the same bytes per packed f row).
constexpr int kLbCells = 8;
constexpr int kLbWarps = 16;
constexpr int kLbMaxRing = 8;

__host__ __device__ constexpr bool lblock_supported_k(int k) { return k == 8 || k == 12; }

// The l-block kernel's shared memory: the ring of stages (R_t as the kernel reads it, then at most
// max_rows packed f rows of K x cells values each), the band's FP64 Q rows of the CTA's cells, and the
// counter, done words, row tickets, per-t item totals and stage assignments.
inline Layout lblock_layout(int n_ring, int stage_bytes, int k, int max_rows, int max_t, int cells) {
    Layout l{};
    int o = 0;
    auto take = [&](int bytes, int align) {
        o = (o + align - 1) / align * align;
        const int r = o;
        o += bytes;
        return r;
    };
    l.off_b = take(n_ring * stage_bytes, 1024);
    l.off_red = take(max_rows * k * cells * (int)sizeof(double), 16);
    l.off_bar = take(16 * (int)sizeof(uint64_t), 16);
    l.off_misc = take((2 + 2 * kLbMaxRing + max_rows + max_t) * (int)sizeof(int), 16);
    l.total = o;
    return l;
}

// Bounded wait on an mbarrier phase; on timeout (or if another thread already gave up) sets the
// CTA's abort word and the error word, and returns false.
__device__ __forceinline__ bool wait_bar(uint64_t* bar, uint32_t parity, volatile int* abort_flag, int* err,
                                         long long budget = kWaitCycles) {
    if (*abort_flag) return false;
    const long long t0 = clock64();
    for (;;) {
        if (tc05::mbar_try_wait_sleep(bar, parity, 2000u)) return true;
        if (*abort_flag) return false;
        if (clock64() - t0 > budget) {
            *abort_flag = 1;
            atomicExch(err, 1);
            return false;
        }
    }
}

__device__ __forceinline__ uint32_t byte_word(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3, int ib) {
    // byte ib of x0..x3, packed little-endian
    const uint32_t sel = (uint32_t)ib | ((uint32_t)(ib + 4) << 4);
    const uint32_t t01 = __byte_perm(x0, x1, sel);
    const uint32_t t23 = __byte_perm(x2, x3, sel);
    return __byte_perm(t01, t23, 0x5410);
}

// A slot's entries of one l-triplet and the first 32 of them, loaded one l-triplet ahead of their use
// (the band kernels walk a row group's t-list in lockstep, so the next t's metadata and entries are
// known a whole Phi step before they are needed; without this, three dependent global loads per t
// sat exposed on every warp).
struct SlotEntries {
    int cb, ce;     // the slot's entries cb .. ce - 1
    uint32_t q23;   // entry cb + lane (if < ce)
    double g;
};

// Slots of a row group of nr rows on W warps: q = W / nr chunks per row, and one more for the first
// rem = W % nr rows, so that every warp has a slot.  Slot w -> (local row, chunk, chunks of the row).
__device__ __forceinline__ void slot_of(int w, int q, int rem, int& rl, int& ch, int& nch) {
    const int big = rem * (q + 1);
    if (w < big) {
        rl = w / (q + 1);
        ch = w % (q + 1);
        nch = q + 1;
    } else {
        rl = rem + (w - big) / q;
        ch = (w - big) % q;
        nch = q;
    }
}

// The first slot of local row rl and its number of chunks.
__device__ __forceinline__ int row_first_slot(int rl, int q, int rem) {
    return rl < rem ? rl * (q + 1) : rem * (q + 1) + (rl - rem) * q;
}
__device__ __forceinline__ int row_chunks(int rl, int q, int rem) { return rl < rem ? q + 1 : q; }

// The entry range of slot (row, chunk ch of nS) at t-list position ti of the unit's band.
__device__ __forceinline__ void slot_range(const SplitArgs& a, int tab_off, int brows, int ti, int row, int ch, int nS,
                                           int& cb, int& ce) {
    const int2 r = __ldg(reinterpret_cast<const int2*>(a.band_rng) + tab_off + ti * brows + row);
    const int n = r.y - r.x;
    cb = r.x + (int)(((long long)n * ch) / nS);
    ce = r.x + (int)(((long long)n * (ch + 1)) / nS);
}

__device__ __forceinline__ SlotEntries slot_fetch(const SplitArgs& a, const double* __restrict__ gv, int cb, int ce,
                                                  int lane) {
    SlotEntries se{cb, ce, 0u, 0.0};
    if (cb + lane < ce) {
        se.q23 = __ldg(a.e_q23 + cb + lane);
        se.g = __ldg(gv + cb + lane);
    }
    return se;
}

// Phi of one slot for this lane's part (k2 = k2o .. k2o + KH - 1, k3 = k3o .. k3o + KQ - 1) of cell c:
// the slot's entries, grouped by q2 (h = sum G f(q3) over a run of equal q2, then phi += f(q2) (x) h).
template <int K, int C, typename T = double>
__device__ __forceinline__ void slot_phi(const SplitArgs& a, const double* __restrict__ gv,
                                         const T* __restrict__ fs, int NQ, const SlotEntries& se, int lane,
                                         int c, int k2o, int k3o,
                                         T (&phi)[Shape<K, C>::KH][Shape<K, C>::KQ]) {
    constexpr int KH = Shape<K, C>::KH, KQ = Shape<K, C>::KQ;
#pragma unroll
    for (int x = 0; x < KH; ++x)
#pragma unroll
        for (int y = 0; y < KQ; ++y) phi[x][y] = (T)0;
    const int cb = se.cb, ce = se.ce;
    if (cb >= ce) return;
    T h[KQ];
#pragma unroll
    for (int y = 0; y < KQ; ++y) h[y] = (T)0;
    int cur = -1;
    auto flush = [&]() {
#pragma unroll
        for (int x = 0; x < KH; ++x) {
            const T f2 = fs[((k2o + x) * NQ + cur) * C + c];
#pragma unroll
            for (int y = 0; y < KQ; ++y) phi[x][y] = fma(f2, h[y], phi[x][y]);
        }
#pragma unroll
        for (int y = 0; y < KQ; ++y) h[y] = (T)0;
    };
    for (int eb = cb; eb < ce; eb += 32) {
        const int nb = min(32, ce - eb);
        uint32_t my_q23 = se.q23;
        double my_g = se.g;
        if (eb != cb) {
            my_q23 = 0;
            my_g = 0.0;
            if (lane < nb) {
                my_q23 = __ldg(a.e_q23 + eb + lane);
                my_g = __ldg(gv + eb + lane);
            }
        }
        for (int j = 0; j < nb; ++j) {
            const uint32_t q23 = __shfl_sync(0xffffffffu, my_q23, j);
            const T g = (T)__shfl_sync(0xffffffffu, my_g, j);
            const int q2 = (int)(q23 & 0xffffu), q3 = (int)(q23 >> 16);
            if (q2 != cur) {
                if (cur >= 0) flush();
                cur = q2;
            }
#pragma unroll
            for (int y = 0; y < KQ; ++y) h[y] = fma(g, fs[((k3o + y) * NQ + q3) * C + c], h[y]);
        }
    }
    if (cur >= 0) flush();
}

// The C cells' f (cell-major in global memory) into shared memory as fs[(k N_Q + q) C + cell], zero
// past the end of the batch.
template <int C, int NT = kThreads>
__device__ __forceinline__ void stage_f(const SplitArgs& a, double* fs, int M, long long cell0, int tid) {
    for (int i = tid; i < C * M; i += NT) {
        const int cc = i % C, r = i / C;  // r = k N_Q + q: the cell-major element index
        const long long cell = cell0 + cc;
        fs[i] = cell < a.n_cells ? __ldg(a.f + cell * M + r) : 0.0;
    }
}

template <int K, int C>
__global__ void __launch_bounds__(kThreads, 1) af_split_kernel(SplitArgs a) {
    using S = Shape<K, C>;
    static_assert(S::KK % 32 == 0, "whole 32-byte K steps of the int8 planes");
    constexpr int KH = S::KH, KQ = S::KQ, E = S::E, EP = S::EP, NKS = S::NKS;
    extern __shared__ __align__(1024) unsigned char smem[];
    uint8_t* sA = smem + a.off_a;
    uint8_t* sB = smem + a.off_b;
    double* fs = reinterpret_cast<double*>(smem + a.off_f);
    double* mb = reinterpret_cast<double*>(smem + a.off_mb);
    double* red = reinterpret_cast<double*>(smem + a.off_red);
    double* scale = reinterpret_cast<double*>(smem + a.off_scale);
    int* eexp = reinterpret_cast<int*>(smem + a.off_eexp);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + a.off_bar);
    uint64_t* bfull = bars;        // [2] R planes of a t have landed
    uint64_t* bfree = bars + 2;    // [2] the MMAs reading a B slot are done
    uint64_t* afree = bars + 4;    // [2] the MMAs reading an A buffer are done
    int* misc = reinterpret_cast<int*>(smem + a.off_misc);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(misc);
    volatile int* abort_flag = misc + 1;
    int* acount = misc + 2;  // [2] warps that have written an A buffer, summed over its uses

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int c = lane % C, part = lane / C, k2o = S::k2_of(part), k3o = S::k3_of(part);
    const int NQ = a.n_q, L = a.L, M = NQ * K;
    const int rg = a.unit_order[blockIdx.x / a.n_cg];
    const int cg = blockIdx.x % a.n_cg;
    const int* u = a.units + (size_t)rg * U_INTS;
    const int l1 = u[U_L1], r0 = u[U_R0], nr = u[U_NR], cq = u[U_S], crem = u[U_REM], tl_off = u[U_TLOFF],
              n_t = u[U_NT], tab_off = u[U_TABOFF], brows = u[U_BROWS];
    const int n_slots = nr * cq + crem;
    const long long cell0 = (long long)cg * C;

    // ---- set-up: barriers, tensor memory, zero A tiles, f staged -----------------------------
    if (tid == 0) {
        for (int i = 0; i < 8; ++i) tc05::mbar_init(&bars[i], 1);
        tc05::fence_mbar_init();
        *abort_flag = 0;
        acount[0] = acount[1] = 0;
    }
    if (warp == 0) {
        tc05::tmem_alloc(tslot, kTmemCols);
        tc05::tmem_relinquish();
    }
    {
        uint4* z = reinterpret_cast<uint4*>(sA);
        for (int i = tid; i < a.n_abuf * kPlanes * NKS * S::ATILE / 16; i += kThreads) z[i] = make_uint4(0, 0, 0, 0);
    }
    stage_f<C>(a, fs, M, cell0, tid);
    tc05::tc_fence_before();
    __syncthreads();
    tc05::tc_fence_after();
    const uint32_t tbase = *tslot;
    const int bbytes = NKS * kBStep;
    if (tid == 0) {
        for (int ti = 0; ti < min(n_t, kBRing); ++ti) {
            const int t = a.band_tl[tl_off + ti];
            tc05::mbar_arrive_expect_tx(&bfull[ti], (uint32_t)bbytes);
            tc05::bulk_g2s(sB + ti * bbytes, a.rplanes + (size_t)t * bbytes, (uint32_t)bbytes, &bfull[ti]);
        }
    }
    // band maxima of |f| per cell: mb[cell][l]
    for (int pr = warp; pr < C * (L + 1); pr += kWarps) {
        const int cc = pr / (L + 1), l = pr % (L + 1);
        const int q0 = l * l, nq = 2 * l + 1;
        double m = 0.0;
        for (int i = lane; i < nq * K; i += 32) {
            const int k = i / nq, q = q0 + i % nq;
            m = fmax(m, fabs(fs[(k * NQ + q) * C + cc]));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) mb[cc * (L + 1) + l] = m;
    }
    __syncthreads();
    // per (slot, cell): the exponent e from the a-priori bound over the row's slices
    if (tid < kSlots * C) {
        const int s = tid / C, cc = tid % C;
        int e = 0;
        if (s < n_slots) {
            int srl, sch, snc;
            slot_of(s, cq, crem, srl, sch, snc);
            const int q1 = l1 * l1 + r0 + srl;
            double bound = 0.0;
            const int i1 = __ldg(a.rb_off + q1 + 1);
#pragma unroll 4
            for (int i = __ldg(a.rb_off + q1); i < i1; ++i) {
                const int l23 = __ldg(a.rb_l23 + i);
                bound = fmax(bound, __ldg(a.rb_gs + i) * mb[cc * (L + 1) + (l23 & 0xff)] * mb[cc * (L + 1) + (l23 >> 8)]);
            }
            if (bound > 0.0) {
                int x;
                frexp(bound, &x);  // bound < 2^x
                e = min(max(kXBits - x, -1000), 1000);
            }
        }
        eexp[tid] = e;
        scale[tid] = ldexp(1.0, e);
    }
    // zero the accumulators (lanes 0-63: quadrants 0 and 1)
    auto zero_d = [&]() {
        const uint32_t lb = (uint32_t)(32 * (warp & 3)) << 16;
        for (int col = (warp >> 2) * 4; col < kDBlocks * kNB; col += 16)
            tc05::tmem_st4(tbase + lb + col, 0u, 0u, 0u, 0u);
        tc05::tmem_wait_st();
    };
    zero_d();
    tc05::tc_fence_before();
    __syncthreads();
    tc05::tc_fence_after();

    // ---- drain: accumulators -> FP64 -> Q (rows summed over their slots in a fixed order) ----
    // every MMA issued up to l-triplet ti is done once the commits of the last uses of the A buffers
    // (those of ti and, with two buffers, ti - 1) have landed: each earlier use was waited for before
    // its buffer was written again
    auto drain = [&](int ti) {
        bool done = true;
        for (int x = ti; x >= 0 && x > ti - a.n_abuf; --x)
            done = wait_bar(&afree[x % a.n_abuf], (uint32_t)((x / a.n_abuf) & 1), abort_flag, a.err) && done;
        const bool ok = __all_sync(0xffffffffu, done);
        tc05::tc_fence_after();
        constexpr int KG = (K + 3) / 4;  // k1 per drain warp
        // the accumulator row m in TMEM lane 32 (warp % 4) + lane: M = 64 keeps rows 16q..16q+15 in
        // lanes 0-15 of quadrant q; M = 128 keeps row m in lane m
        const int m = S::M == 64 ? 16 * (warp & 3) + (lane & 15) : 32 * (warp & 3) + lane;
        const bool holds = S::M == 64 ? lane < 16 : true;
        if (ok) {
            const int s = m / C, cc = m % C;
            const int kg = warp >> 2;
            const uint32_t lb = (uint32_t)(32 * (warp & 3)) << 16;
            double acc[KG];
#pragma unroll
            for (int j = 0; j < KG; ++j) acc[j] = 0.0;
#pragma unroll
            for (int d = kDMin; d <= 10; ++d) {
                // the block's 16 columns; this warp keeps k1 = kg * KG .. kg * KG + KG - 1
                uint32_t r16[16];
                uint32_t* lo8 = r16;
                uint32_t* hi8 = r16 + 8;
                tc05::tmem_ld8(tbase + lb + (uint32_t)((d - kDMin) * kNB), *reinterpret_cast<uint32_t(*)[8]>(lo8));
                tc05::tmem_ld8(tbase + lb + (uint32_t)((d - kDMin) * kNB + 8), *reinterpret_cast<uint32_t(*)[8]>(hi8));
                tc05::tmem_wait_ld();
                const double w = ldexp(1.0, 8 * d - kRShift - eexp[m]);
#pragma unroll
                for (int j = 0; j < KG; ++j) {
                    const int want = kg * KG + j;
                    uint32_t v = 0;
#pragma unroll
                    for (int x = 0; x < 16; ++x) v = (x == want) ? r16[x] : v;
                    acc[j] += (double)(int)v * w;
                }
            }
            if (holds && s < n_slots)
#pragma unroll
                for (int j = 0; j < KG; ++j)
                    if (kg * KG + j < K) red[(s * C + cc) * K + kg * KG + j] = acc[j];
        }
        tc05::tc_fence_before();
        __syncthreads();
        if (tid < nr * C) {
            const int rl = tid / C, cc = tid % C;
            const long long cell = cell0 + cc;
            if (cell < a.n_cells) {
                const int q1 = l1 * l1 + r0 + rl;
                double* qc = a.q + cell * M + q1;
                for (int k1 = 0; k1 < K; ++k1) {
                    double sum = 0.0;
                    const int s0 = row_first_slot(rl, cq, crem), nc = row_chunks(rl, cq, crem);
                    for (int ch = 0; ch < nc; ++ch) sum += red[((s0 + ch) * C + cc) * K + k1];
                    qc[(size_t)k1 * NQ] += sum;
                }
            }
        }
        zero_d();
        tc05::tc_fence_before();
        __syncthreads();
        tc05::tc_fence_after();
    };

    // ---- main loop over the band's l-triplets ------------------------------------------------
    const bool active = warp < n_slots;
    int srow = 0, ch = 0, nS = 1;
    if (active) slot_of(warp, cq, crem, srow, ch, nS);
    const int row = r0 + srow;
    const int m_row = warp * C + c;  // A row of this lane's (slot, cell)
    const double sc = scale[m_row];
    constexpr double kMagic = 6755399441055744.0;  // 1.5 * 2^52: adding it rounds to an integer
    // the slot's entries of t-list position ti in cur, of ti + 1 fetched during ti, the range of ti + 2
    SlotEntries cur{0, 0, 0u, 0.0}, nxt{0, 0, 0u, 0.0};
    int ncb = 0, nce = 0;
    if (active) {
        int cb, ce;
        slot_range(a, tab_off, brows, 0, row, ch, nS, cb, ce);
        cur = slot_fetch(a, a.e_gs, cb, ce, lane);
        if (n_t > 1) slot_range(a, tab_off, brows, 1, row, ch, nS, ncb, nce);
    }
    for (int ti = 0; ti < n_t; ++ti) {
        uint32_t lo[E], hi[E];
        if (active) {
            if (ti + 1 < n_t) nxt = slot_fetch(a, a.e_gs, ncb, nce, lane);
            if (ti + 2 < n_t) slot_range(a, tab_off, brows, ti + 2, row, ch, nS, ncb, nce);
            double phi[KH][KQ];
            slot_phi<K, C>(a, a.e_gs, fs, NQ, cur, lane, c, k2o, k3o, phi);
            cur = nxt;
#pragma unroll
            for (int x = 0; x < KH; ++x)
#pragma unroll
                for (int y = 0; y < KQ; ++y) {
                    const double yv = fma(phi[x][y], sc, kMagic);
                    lo[x * KQ + y] = (uint32_t)__double2loint(yv);
                    hi[x * KQ + y] = (uint32_t)(__double2hiint(yv) - 0x43380000);
                }
        }
        // all six planes of this t into A buffer b (the buffer's previous MMAs must be done), one barrier,
        // then one thread issues the t's MMAs: per plane i and 32-byte K step, A plane i against the
        // window of R planes j = j0..5 into the accumulator blocks d = i + j
        const int b = ti % a.n_abuf, use = ti / a.n_abuf;
        if (use >= 1) wait_bar(&afree[b], (uint32_t)((use - 1) & 1), abort_flag, a.err);
        uint8_t* abuf = sA + b * kPlanes * NKS * S::ATILE;
        if (active) {
#pragma unroll
            for (int i = 0; i < kPlanes; ++i) {
                uint8_t* tile = abuf + i * NKS * S::ATILE;
#pragma unroll
                for (int w = 0; w < EP / 4; ++w) {
                    uint32_t v[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int e = 4 * w + j;
                        v[j] = e < E ? (i < 4 ? lo[e < E ? e : 0] : hi[e < E ? e : 0]) : 0u;
                    }
                    const uint32_t word = byte_word(v[0], v[1], v[2], v[3], i & 3);
                    const int kk = part * EP + 4 * w;
                    const int off = (kk >> 5) * S::ATILE + (m_row >> 3) * 256 + ((kk & 31) >> 4) * 128 + (m_row & 7) * 16 +
                                    (kk & 15);
                    *reinterpret_cast<uint32_t*>(tile + off) = word;
                }
            }
        }
        // the warp that writes an A buffer last (per use) issues its MMAs: no CTA-wide barrier, a warp
        // runs ahead until the ring of A buffers holds it back
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncwarp();
        int last = 0;
        if (lane == 0) {
            __threadfence_block();
            last = atomicAdd(&acount[b], 1) == kWarps * (use + 1) - 1;
        }
        last = __shfl_sync(0xffffffffu, last, 0);
        if (last && lane == 0 && !*abort_flag) {
            __threadfence_block();
            tc05::tc_fence_after();
            // refill the other B slot with the next t (its MMAs, of t - 1, were issued a Phi step ago)
            const int tn = ti + 1;
            if (tn >= kBRing && tn < n_t) {
                const int sb = tn % kBRing, useb = tn / kBRing;
                if (wait_bar(&bfree[sb], (uint32_t)((useb - 1) & 1), abort_flag, a.err)) {
                    const int t = a.band_tl[tl_off + tn];
                    tc05::mbar_arrive_expect_tx(&bfull[sb], (uint32_t)bbytes);
                    tc05::bulk_g2s(sB + sb * bbytes, a.rplanes + (size_t)t * bbytes, (uint32_t)bbytes, &bfull[sb]);
                }
            }
            wait_bar(&bfull[ti % kBRing], (uint32_t)((ti / kBRing) & 1), abort_flag, a.err);
            if (!*abort_flag) {
                const uint8_t* bslot = sB + (ti % kBRing) * bbytes;
#pragma unroll
                for (int i = 0; i < kPlanes; ++i) {
                    const uint8_t* tile = abuf + i * NKS * S::ATILE;
                    const int j0 = i < kDMin ? kDMin - i : 0;
                    const int n = (kPlanes - j0) * kNB;
                    const uint32_t idesc = tc05::idesc_i8(S::M, n, i == kPlanes - 1, true);
                    const uint32_t dcol = (uint32_t)((i + j0 - kDMin) * kNB);
#pragma unroll
                    for (int ks = 0; ks < NKS; ++ks) {
                        const uint64_t ad = tc05::smem_desc_kmajor(tile + ks * S::ATILE, 128, 256);
                        const uint64_t bd = tc05::smem_desc_kmajor(bslot + ks * kBStep + j0 * (kNB / 8) * 256, 128, 256);
                        tc05::mma_i8_ss(tbase + dcol, ad, bd, idesc, true);
                    }
                }
            }
            // always arrive, so that waiters are released also on the error path
            tc05::mma_commit(&afree[b]);
            tc05::mma_commit(&bfree[ti % kBRing]);
        }
        __syncwarp();
        if ((ti + 1) % a.tseg == 0 && ti + 1 < n_t) drain(ti);
    }
    drain(n_t - 1);

    // ---- tear-down --------------------------------------------------------------------------
    tc05::tc_fence_before();
    __syncthreads();
    if (warp == 0) tc05::tmem_dealloc(tbase, kTmemCols);
}

// The FP64 band kernel: the same units and Phi step, the K^3 step in FP64 on the CUDA cores from R_t
// staged per t into a 2-deep shared-memory ring by one cp.async.bulk each ([part][e][k1], so a lane
// reads its part's K x E block with 16-byte loads shared by the part's 4 cells).  Each lane
// accumulates its part's share of Q(row, cell) over the band's t-list; the 8 parts and the slots of
// a row are summed in a fixed order at the end.
template <int K, int C, int W>
__global__ void __launch_bounds__(W * 32, 1) af_band64_kernel(SplitArgs a) {
    using S = Shape<K, C>;
    constexpr int KH = S::KH, KQ = S::KQ, PS = S::PS, RTB = S::RT_BYTES;
    extern __shared__ __align__(1024) unsigned char smem[];
    double* rring = reinterpret_cast<double*>(smem + a.off_b);
    double* fs = reinterpret_cast<double*>(smem + a.off_f);
    double* red = reinterpret_cast<double*>(smem + a.off_red);
    uint64_t* bfull = reinterpret_cast<uint64_t*>(smem + a.off_bar);
    int* misc = reinterpret_cast<int*>(smem + a.off_misc);
    volatile int* abort_flag = misc + 1;
    int* rcount = misc + 2;  // [2] warps done with an R slot, summed over its uses

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int c = lane % C, part = lane / C, k2o = S::k2_of(part), k3o = S::k3_of(part);
    const int NQ = a.n_q, M = NQ * K;
    const int rg = a.unit_order[blockIdx.x / a.n_cg];
    const int cg = blockIdx.x % a.n_cg;
    const int* u = a.units + (size_t)rg * U_INTS;
    const int l1 = u[U_L1], r0 = u[U_R0], nr = u[U_NR], cq = u[U_S], crem = u[U_REM], tl_off = u[U_TLOFF],
              n_t = u[U_NT], tab_off = u[U_TABOFF], brows = u[U_BROWS];
    const int n_slots = nr * cq + crem;
    const long long cell0 = (long long)cg * C;

    if (tid == 0) {
        tc05::mbar_init(&bfull[0], 1);
        tc05::mbar_init(&bfull[1], 1);
        tc05::fence_mbar_init();
        *abort_flag = 0;
        rcount[0] = rcount[1] = 0;
    }
    stage_f<C, W * 32>(a, fs, M, cell0, tid);
    __syncthreads();
    if (tid == 0)
        for (int ti = 0; ti < min(n_t, 2); ++ti) {
            const int t = a.band_tl[tl_off + ti];
            tc05::mbar_arrive_expect_tx(&bfull[ti], (uint32_t)RTB);
            tc05::bulk_g2s(rring + ti * (RTB / 8), a.rfp64 + (size_t)t * (RTB / 8), (uint32_t)RTB, &bfull[ti]);
        }

    const bool active = warp < n_slots;
    int srow = 0, ch = 0, nS = 1;
    if (active) slot_of(warp, cq, crem, srow, ch, nS);
    const int row = r0 + srow;
    double acc[K];
#pragma unroll
    for (int k1 = 0; k1 < K; ++k1) acc[k1] = 0.0;
    // the slot's entries of t-list position ti in cur, of ti + 1 fetched during ti, the range of ti + 2
    SlotEntries cur{0, 0, 0u, 0.0}, nxt{0, 0, 0u, 0.0};
    int ncb = 0, nce = 0;
    if (active) {
        int cb, ce;
        slot_range(a, tab_off, brows, 0, row, ch, nS, cb, ce);
        cur = slot_fetch(a, a.e_g, cb, ce, lane);
        if (n_t > 1) slot_range(a, tab_off, brows, 1, row, ch, nS, ncb, nce);
    }
    for (int ti = 0; ti < n_t; ++ti) {
        const int sb = ti & 1;
        const SlotEntries se = cur;
        double phi[KH][KQ];
        if (active) {
            if (ti + 1 < n_t) nxt = slot_fetch(a, a.e_g, ncb, nce, lane);
            if (ti + 2 < n_t) slot_range(a, tab_off, brows, ti + 2, row, ch, nS, ncb, nce);
            slot_phi<K, C>(a, a.e_g, fs, NQ, se, lane, c, k2o, k3o, phi);
            cur = nxt;
        }
        // every warp sees slot sb's copy land before it counts itself done with the slot (the refill of
        // the slot is armed only after that), also where it reads nothing from it
        const bool ok = wait_bar(&bfull[sb], (uint32_t)((ti >> 1) & 1), abort_flag, a.err);
        if (active && ok && se.cb < se.ce) {
            const double* rp = rring + sb * (RTB / 8) + part * PS;
#pragma unroll
            for (int x = 0; x < KH; ++x)
#pragma unroll
                for (int y = 0; y < KQ; ++y) {
                    const double2* r2 = reinterpret_cast<const double2*>(rp + (x * KQ + y) * K);
#pragma unroll
                    for (int j = 0; j < K / 2; ++j) {
                        const double2 r = r2[j];
                        acc[2 * j] = fma(r.x, phi[x][y], acc[2 * j]);
                        acc[2 * j + 1] = fma(r.y, phi[x][y], acc[2 * j + 1]);
                    }
                }
        }
        // the last warp done with slot sb refills it with t + 2 (no CTA-wide barrier)
        __syncwarp();
        if (lane == 0) {
            __threadfence_block();
            if (atomicAdd(&rcount[sb], 1) == W * ((ti >> 1) + 1) - 1 && ti + 2 < n_t && !*abort_flag) {
                __threadfence_block();
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                const int t = a.band_tl[tl_off + ti + 2];
                tc05::mbar_arrive_expect_tx(&bfull[sb], (uint32_t)RTB);
                tc05::bulk_g2s(rring + sb * (RTB / 8), a.rfp64 + (size_t)t * (RTB / 8), (uint32_t)RTB, &bfull[sb]);
            }
        }
        __syncwarp();
    }
    // the parts of a cell sit in lanes c, c + C, c + 2C, ...
#pragma unroll
    for (int k1 = 0; k1 < K; ++k1)
#pragma unroll
        for (int o = C; o < 32; o <<= 1) acc[k1] += __shfl_xor_sync(0xffffffffu, acc[k1], o);
    if (active && lane < C)
#pragma unroll
        for (int k1 = 0; k1 < K; ++k1) red[(warp * C + lane) * K + k1] = acc[k1];
    __syncthreads();
    if (tid < nr * C) {
        const int rl = tid / C, cc = tid % C;
        const long long cell = cell0 + cc;
        if (cell < a.n_cells) {
            double* qc = a.q + cell * M + (l1 * l1 + r0 + rl);
            for (int k1 = 0; k1 < K; ++k1) {
                double sum = 0.0;
                const int s0 = row_first_slot(rl, cq, crem), nc = row_chunks(rl, cq, crem);
                for (int chk = 0; chk < nc; ++chk) sum += red[((s0 + chk) * C + cc) * K + k1];
                qc[(size_t)k1 * NQ] += sum;
            }
        }
    }
}

// ------------------------------------------------------------------------------------------
// The l-block kernel: l1-band units with f staged per l-triplet, and a band's slices as work items
// ------------------------------------------------------------------------------------------
//
// A slice of l-triplet t = (l1, l2, l3) reads f only in the rows of band l2 (q2) and band l3 (q3):
// at most 4L rows of the cell's N_Q = (L+1)^2.  So instead of holding all of f for 4 cells (which is
// what fits at L = 16, K = 12: 27.7 KB of FP64 f per cell), a CTA holds C = 8 cells and stages, per
// t of its band's t-list, R_t and those two row blocks into a ring of shared-memory stages: three
// cp.async.bulk copies per stage on one mbarrier (transaction bytes), from f packed per cell group as
// [q][k][cell] so that a band's rows are one contiguous run.  Every COO entry's index work and every
// R_t load then serves 8 cells instead of 4.
//
// One CTA takes one (l1 band, 8-cell group).  A band's rows do not divide evenly over the warps of a
// CTA (33 rows at l1 = 16), and the entries of a (t, row) slice vary widely between rows, so its
// warps take the band's (t, row) slices one at a time from a shared counter, in t-major order.  A
// warp computes the slice's Phi and K^3 step, sums the parts of each cell, and adds the result into
// the band's Q rows, kept in shared memory for the CTA's 8 cells.  Each row takes its slices' results
// in t order (a ticket per row: the warp holding the row's slice number ord waits until ord - 1 has
// been added), so the sums, and the bits of Q, do not depend on which warp ran which item.  The stage
// of t-list position ti is refilled with ti + n_ring by the warp that finishes the last item of ti.

// f cell-major [B][K][N_Q] -> packed [cg][q][k][C], or with CELLROWS [cg][q][C][k] (zero past the
// end of the batch).  One CTA per
// (cell group, 32 rows q), in a one-dimensional grid: the C cells' K x 32 block is read along q
// (coalesced) into shared memory and written out as one contiguous run.
template <int C, typename T, bool CELLROWS = false>
__global__ void __launch_bounds__(256) pack_cg_kernel(const double* __restrict__ f, T* __restrict__ pf,
                                                      long long n_cells, int n_q, int K) {
    extern __shared__ __align__(16) unsigned char tile_raw[];
    T* tile = reinterpret_cast<T*>(tile_raw);  // [32][K][C]
    const int nqb = (n_q + 31) / 32;
    const long long cg = (long long)blockIdx.x / nqb;
    const int q0 = (int)(blockIdx.x % nqb) * 32;
    const int nq = min(32, n_q - q0);
    const long long M = (long long)n_q * K;
    for (int i = threadIdx.x; i < 32 * K * C; i += blockDim.x) {
        const int qq = i % 32, k = (i / 32) % K, c = i / (32 * K);
        const long long cell = cg * C + c;
        double v = 0.0;
        if (qq < nq && cell < n_cells) v = __ldg(f + cell * M + (long long)k * n_q + q0 + qq);
        tile[CELLROWS ? (qq * C + c) * K + k : (qq * K + k) * C + c] = (T)v;
    }
    __syncthreads();
    T* out = pf + (cg * n_q + q0) * K * C;
    for (int i = threadIdx.x; i < nq * K * C; i += blockDim.x) out[i] = tile[i];
}

// The lane layout of the l-block kernels: C cells per CTA, P = 32 / C lanes (parts) per cell, each
// holding all K values of k2 and KQ = K / P values of k3 of the cell's Phi.  FP64 (C = 8): part p
// owns k3 = p KQ .. p KQ + KQ - 1 (the packed rows k3 of the four parts fall on distinct banks);
// FP32 (C = 16): part p owns k3 = p, p + 2, ... (blocked halves would put both half-warps' 32-bit
// loads on the same 16 banks).  R_t per stage is [part][e = k2 KQ + y][k1] in T, 16 bytes of padding
// after each part.
template <int K, int C, typename T>
struct LbShape {
    static constexpr int P = 32 / C;
    static constexpr int KH = K;
    static constexpr int KQ = K / P;
    static constexpr int E = KH * KQ;
    static constexpr int PS = E * K + 16 / (int)sizeof(T);  // T words per part
    static constexpr int RT_BYTES = P * PS * (int)sizeof(T);
    static constexpr bool INTERLEAVED = sizeof(T) == 4;
    __host__ __device__ static constexpr int k3_base(int p) { return INTERLEAVED ? p : p * KQ; }
    static constexpr int K3_STEP = INTERLEAVED ? P : 1;
    __host__ __device__ static constexpr int k3(int p, int y) { return k3_base(p) + y * K3_STEP; }
};

// Phi of one slot on a stage: rows of the stage are local (q2 - b2, q3 - b3), f at
// fsg[(row K + k) C + cell]; grouped by q2 as slot_phi.
template <int K, int C, typename T>
__device__ __forceinline__ void slot_phi_staged(const double* __restrict__ gv, const uint32_t* __restrict__ eq23,
                                                const T* __restrict__ fsg, const SlotEntries& se, int lane,
                                                int c, int part, int b2, int b3,
                                                T (&phi)[LbShape<K, C, T>::KH][LbShape<K, C, T>::KQ]) {
    using S = LbShape<K, C, T>;
    constexpr int KH = S::KH, KQ = S::KQ;
    const int k3o = S::k3_base(part);
#pragma unroll
    for (int x = 0; x < KH; ++x)
#pragma unroll
        for (int y = 0; y < KQ; ++y) phi[x][y] = (T)0;
    const int cb = se.cb, ce = se.ce;
    if (cb >= ce) return;
    T h[KQ];
#pragma unroll
    for (int y = 0; y < KQ; ++y) h[y] = (T)0;
    int cur = -1;
    auto flush = [&]() {
        const T* __restrict__ f2p = fsg + (size_t)cur * K * C + c;
#pragma unroll
        for (int x = 0; x < KH; ++x) {
            const T f2 = f2p[x * C];
#pragma unroll
            for (int y = 0; y < KQ; ++y) phi[x][y] = fma(f2, h[y], phi[x][y]);
        }
#pragma unroll
        for (int y = 0; y < KQ; ++y) h[y] = (T)0;
    };
    for (int eb = cb; eb < ce; eb += 32) {
        const int nb = min(32, ce - eb);
        uint32_t my_q23 = se.q23;
        double my_g = se.g;
        if (eb != cb) {
            my_q23 = 0;
            my_g = 0.0;
            if (lane < nb) {
                my_q23 = __ldg(eq23 + eb + lane);
                my_g = __ldg(gv + eb + lane);
            }
        }
        for (int j = 0; j < nb; ++j) {
            const uint32_t q23 = __shfl_sync(0xffffffffu, my_q23, j);
            const T g = (T)__shfl_sync(0xffffffffu, my_g, j);
            const int q2 = (int)(q23 & 0xffffu) - b2, q3 = (int)(q23 >> 16) - b3;
            if (q2 != cur) {
                if (cur >= 0) flush();
                cur = q2;
            }
            const T* __restrict__ f3p = fsg + ((size_t)q3 * K + k3o) * C + c;
#pragma unroll
            for (int y = 0; y < KQ; ++y) h[y] = fma(g, f3p[y * S::K3_STEP * C], h[y]);
        }
    }
    if (cur >= 0) flush();
}

// The FP64 l-block kernel's K^3 step on the FP64 tensor cores (warp-level mma.sync m8n8k4; B200's
// tcgen05 has no FP64 kind).  Lane l = (g = l >> 2, p = l & 3) holds cell g's Phi for all k2 and
// k3 = p KQ .. p KQ + KQ - 1: at k-step s = k2 KQ + y that is exactly the B fragment B[k = p][n = g]
// of the MMA whose K index is kk' = 4 s + p.  Per l-triplet the stage holds R_t as A fragments,
// [m-tile][s][lane] with A[m = g][k = p] = R_t[k1 = g + 8 m-tile][k2][k3 = p KQ + y] (zero for
// k1 >= K), so a warp reads each fragment as 32 consecutive doubles.  The product lands in the C
// fragments D[k1 = g + 8 m-tile][cells 2p, 2p + 1]: the sum over the parts of a cell is the MMA's
// own, and no lane exchanges anything.  f rows are staged as [q][cell][k], so the four lanes of a
// cell read their k3 on distinct banks and a run's f(q2) comes in 16-byte pairs.
template <int K>
struct LbMma {
    static constexpr int C = 8;
    static constexpr int KQ = K / 4;                  // k3 per lane
    static constexpr int MT = (K + 7) / 8;            // m-tiles of k1
    static constexpr int S = K * KQ;                  // k-steps of four kk'
    static constexpr int RT_BYTES = MT * S * 32 * 8;  // A fragments of one R_t
};

// Phi of one item on an FP64 cell-rows stage (f at fsg[(row C + cell) K + k], rows local as in
// slot_phi_staged), for lane (cell c, part p): phi[k2][y], k3 = p KQ + y; grouped by q2.
template <int K>
__device__ __forceinline__ void slot_phi_cellrows(const double* __restrict__ gv, const uint32_t* __restrict__ eq23,
                                                  const double* __restrict__ fsg, const SlotEntries& se, int lane,
                                                  int c, int part, int b2, int b3, double (&phi)[K][K / 4]) {
    constexpr int C = LbMma<K>::C, KQ = LbMma<K>::KQ;
    const int k3o = part * KQ;
#pragma unroll
    for (int x = 0; x < K; ++x)
#pragma unroll
        for (int y = 0; y < KQ; ++y) phi[x][y] = 0.0;
    const int cb = se.cb, ce = se.ce;
    if (cb >= ce) return;
    double h[KQ];
#pragma unroll
    for (int y = 0; y < KQ; ++y) h[y] = 0.0;
    int cur = -1;
    auto flush = [&]() {
        const double2* __restrict__ f2p = reinterpret_cast<const double2*>(fsg + ((size_t)cur * C + c) * K);
#pragma unroll
        for (int x = 0; x < K / 2; ++x) {
            const double2 f2 = f2p[x];
#pragma unroll
            for (int y = 0; y < KQ; ++y) {
                phi[2 * x][y] = fma(f2.x, h[y], phi[2 * x][y]);
                phi[2 * x + 1][y] = fma(f2.y, h[y], phi[2 * x + 1][y]);
            }
        }
#pragma unroll
        for (int y = 0; y < KQ; ++y) h[y] = 0.0;
    };
    for (int eb = cb; eb < ce; eb += 32) {
        const int nb = min(32, ce - eb);
        uint32_t my_q23 = se.q23;
        double my_g = se.g;
        if (eb != cb) {
            my_q23 = 0;
            my_g = 0.0;
            if (lane < nb) {
                my_q23 = __ldg(eq23 + eb + lane);
                my_g = __ldg(gv + eb + lane);
            }
        }
        for (int j = 0; j < nb; ++j) {
            const uint32_t q23 = __shfl_sync(0xffffffffu, my_q23, j);
            const double g = __shfl_sync(0xffffffffu, my_g, j);
            const int q2 = (int)(q23 & 0xffffu) - b2, q3 = (int)(q23 >> 16) - b3;
            if (q2 != cur) {
                if (cur >= 0) flush();
                cur = q2;
            }
            const double* __restrict__ f3p = fsg + ((size_t)q3 * C + c) * K + k3o;
#pragma unroll
            for (int y = 0; y < KQ; ++y) h[y] = fma(g, f3p[y], h[y]);
        }
    }
    if (cur >= 0) flush();
}

__device__ __forceinline__ void lb_dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

enum { LBI_TR = 0, LBI_ORD, LBI_BEGIN, LBI_END };  // item: t | row << 16, ord | l2 << 16 | l3 << 24, entries
enum { LBU_L1 = 0, LBU_BROWS, LBU_TLOFF, LBU_NT, LBU_ITOFF, LBU_NIT, LBU_INTS = 8 };

template <int K, int C, typename T, int W, bool MMA = false>
__device__ __forceinline__ void lblock_body(const SplitArgs& a) {
    using S = LbShape<K, C, T>;
    static_assert(!MMA || (C == LbMma<K>::C && sizeof(T) == 8), "the FP64 tensor-core K^3 step takes 8 FP64 cells");
    constexpr int KH = S::KH, KQ = S::KQ, PS = S::PS, RTB = MMA ? LbMma<K>::RT_BYTES : S::RT_BYTES;
    constexpr int ROWB = K * C * (int)sizeof(T);
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* ring = smem + a.off_b;
    double* qacc = reinterpret_cast<double*>(smem + a.off_red);  // [brows][K][C]
    uint64_t* bfull = reinterpret_cast<uint64_t*>(smem + a.off_bar);
    int* misc = reinterpret_cast<int*>(smem + a.off_misc);
    int* counter = misc;
    volatile int* abort_flag = misc + 1;
    int* done = misc + 2;                        // [kLbMaxRing] items finished per stage, summed over uses
    volatile int* ticket = misc + 2 + kLbMaxRing;  // [max_rows] slices of each row added so far
    int* cum = misc + 2 + kLbMaxRing + a.max_rows;  // [max_t] items of the stage's uses up to ti
    // [kLbMaxRing] the t-list position each stage holds or is being filled with.  An item of ti may be
    // taken while its stage still holds ti - D (items are handed out ahead of the copies), and an
    // mbarrier cannot tell that phase from the one of ti: a parity wait on a phase two ahead of the
    // current one returns at once.  So an item first waits for its stage to be assigned ti.
    volatile int* stage_ti = misc + 2 + kLbMaxRing + a.max_rows + a.max_t;

    const int tid = threadIdx.x, lane = tid & 31;
    const int c = MMA ? lane >> 2 : lane % C, part = MMA ? lane & 3 : lane / C;
    const int NQ = a.n_q, M = NQ * K, D = a.n_ring;
    const int unit = a.unit_order[blockIdx.x / a.n_cg];
    const int cg = blockIdx.x % a.n_cg;
    const int* u = a.units + (size_t)unit * LBU_INTS;
    const int l1 = u[LBU_L1], brows = u[LBU_BROWS], tl_off = u[LBU_TLOFF], n_t = u[LBU_NT], it_off = u[LBU_ITOFF],
              n_it = u[LBU_NIT];
    const long long cell0 = (long long)cg * C;
    const T* __restrict__ pcg = reinterpret_cast<const T*>(a.pf) + (size_t)cg * M * C;
    const T* __restrict__ rsrc = reinterpret_cast<const T*>(a.rfp64);
    const int4* __restrict__ items = a.items + it_off;

    auto issue = [&](int ti, int sb) {
        const int t = a.band_tl[tl_off + ti];
        const int l23 = a.t_l23[t], l2 = l23 & 0xff, l3 = l23 >> 8;
        const uint32_t fb2 = (uint32_t)((2 * l2 + 1) * ROWB), fb3 = l3 != l2 ? (uint32_t)((2 * l3 + 1) * ROWB) : 0u;
        unsigned char* st = ring + (size_t)sb * a.stage_bytes;
        if (a.no_copy) return;  // self-test: the stage never fills
        tc05::mbar_arrive_expect_tx(&bfull[sb], (uint32_t)RTB + fb2 + fb3);
        tc05::bulk_g2s(st, rsrc + (size_t)t * (RTB / sizeof(T)), (uint32_t)RTB, &bfull[sb]);
        tc05::bulk_g2s(st + RTB, pcg + (size_t)l2 * l2 * K * C, fb2, &bfull[sb]);
        if (fb3) tc05::bulk_g2s(st + RTB + fb2, pcg + (size_t)l3 * l3 * K * C, fb3, &bfull[sb]);
    };

    for (int i = tid; i < brows * K * C; i += W * 32) qacc[i] = 0.0;
    for (int i = tid; i < brows; i += W * 32) ticket[i] = 0;
    if (tid == 0) {
        for (int i = 0; i < D; ++i) {
            tc05::mbar_init(&bfull[i], 1);
            done[i] = 0;
            stage_ti[i] = i;
        }
        tc05::fence_mbar_init();
        *abort_flag = 0;
        *counter = 0;
        // cum[ti]: the items of every use of stage ti % D up to and including ti
        int run[kLbMaxRing] = {};
        for (int ti = 0; ti < n_t; ++ti) {
            run[ti % D] += __ldg(a.t_items + tl_off + ti);
            cum[ti] = run[ti % D];
        }
    }
    __syncthreads();
    if (tid == 0)
        for (int ti = 0; ti < min(n_t, D); ++ti) issue(ti, ti);

    // the warp's item and, fetched while it works on it, the next one
    auto grab = [&]() {
        int v = 0;
        if (lane == 0) v = atomicAdd(counter, 1);
        return __shfl_sync(0xffffffffu, v, 0);
    };
    int cur_i = grab();
    int4 it = cur_i < n_it ? __ldg(items + cur_i) : make_int4(0, 0, 0, 0);
    SlotEntries se = cur_i < n_it ? slot_fetch(a, a.e_g, it.z, it.w, lane) : SlotEntries{0, 0, 0u, 0.0};
    while (cur_i < n_it) {
        const int nxt_i = grab();
        int4 nit = make_int4(0, 0, 0, 0);
        SlotEntries nse{0, 0, 0u, 0.0};
        if (nxt_i < n_it) {
            nit = __ldg(items + nxt_i);
            nse = slot_fetch(a, a.e_g, nit.z, nit.w, lane);
        }
        const int ti = it.x & 0xffff, row = it.x >> 16, ord = it.y & 0xffff;
        const int l2 = (it.y >> 16) & 0xff, l3 = (it.y >> 24) & 0xff;
        const int sb = ti % D;
        if (lane == 0) {
            const long long t0 = clock64();
            while (stage_ti[sb] != ti) {
                if (*abort_flag || clock64() - t0 > a.wait_cycles) {
                    *abort_flag = 1;
                    atomicExch(a.err, 1);
                    break;
                }
                __nanosleep(128);
            }
        }
        __syncwarp();
        bool ok = wait_bar(&bfull[sb], (uint32_t)((ti / D) & 1), abort_flag, a.err, a.wait_cycles);
        if (ok) {
            const unsigned char* st = ring + (size_t)sb * a.stage_bytes;
            const int b2 = l2 * l2, b3 = l3 * l3 - (l3 != l2 ? 2 * l2 + 1 : 0);
            T acc[K];
            double dq[MMA ? LbMma<K>::MT : 1][2];
            if constexpr (MMA) {
                constexpr int MT = LbMma<K>::MT, SS = LbMma<K>::S, QQ = LbMma<K>::KQ;
                double phi[K][QQ];
                slot_phi_cellrows<K>(a.e_g, a.e_q23, reinterpret_cast<const double*>(st + RTB), se, lane, c, part,
                                     b2, b3, phi);
                const double* __restrict__ ra = reinterpret_cast<const double*>(st) + lane;
                // two accumulator sets per m-tile (even and odd k-steps): two MMA chains instead of one
                double d[MT][2][2];
#pragma unroll
                for (int mt = 0; mt < MT; ++mt)
#pragma unroll
                    for (int h2 = 0; h2 < 2; ++h2) d[mt][h2][0] = d[mt][h2][1] = 0.0;
#pragma unroll
                for (int ks = 0; ks < SS; ++ks)
#pragma unroll
                    for (int mt = 0; mt < MT; ++mt)
                        lb_dmma(d[mt][ks & 1][0], d[mt][ks & 1][1], ra[(mt * SS + ks) * 32], phi[ks / QQ][ks % QQ]);
#pragma unroll
                for (int mt = 0; mt < MT; ++mt) {
                    dq[mt][0] = d[mt][0][0] + d[mt][1][0];
                    dq[mt][1] = d[mt][0][1] + d[mt][1][1];
                }
            } else {
                T phi[KH][KQ];
                slot_phi_staged<K, C, T>(a.e_g, a.e_q23, reinterpret_cast<const T*>(st + RTB), se, lane, c, part, b2,
                                         b3, phi);
                const T* rp = reinterpret_cast<const T*>(st) + part * PS;
#pragma unroll
                for (int k1 = 0; k1 < K; ++k1) acc[k1] = (T)0;
#pragma unroll
                for (int x = 0; x < KH; ++x)
#pragma unroll
                    for (int y = 0; y < KQ; ++y) {
                        const T* rr = rp + (x * KQ + y) * K;
                        if constexpr (sizeof(T) == 8) {
#pragma unroll
                            for (int j = 0; j < K / 2; ++j) {
                                const double2 r = reinterpret_cast<const double2*>(rr)[j];
                                acc[2 * j] = fma((T)r.x, phi[x][y], acc[2 * j]);
                                acc[2 * j + 1] = fma((T)r.y, phi[x][y], acc[2 * j + 1]);
                            }
                        } else {
#pragma unroll
                            for (int j = 0; j < K / 4; ++j) {
                                const float4 r = reinterpret_cast<const float4*>(rr)[j];
                                acc[4 * j] = fma((T)r.x, phi[x][y], acc[4 * j]);
                                acc[4 * j + 1] = fma((T)r.y, phi[x][y], acc[4 * j + 1]);
                                acc[4 * j + 2] = fma((T)r.z, phi[x][y], acc[4 * j + 2]);
                                acc[4 * j + 3] = fma((T)r.w, phi[x][y], acc[4 * j + 3]);
                            }
                        }
                    }
            }
            // the parts of a cell sit in lanes c, c + C, c + 2C, ...: sum them, then part p adds the
            // k1 of its quarter once this row's earlier slices are in (the MMA has summed them already)
            if constexpr (!MMA) {
#pragma unroll
                for (int k1 = 0; k1 < K; ++k1)
#pragma unroll
                    for (int o = C; o < 32; o <<= 1) acc[k1] += __shfl_xor_sync(0xffffffffu, acc[k1], o);
            }
            if (lane == 0) {
                const long long t0 = clock64();
                while (ticket[row] != ord) {
                    if (*abort_flag || clock64() - t0 > a.wait_cycles) {
                        *abort_flag = 1;
                        atomicExch(a.err, 1);
                        break;
                    }
                    __nanosleep(64);
                }
            }
            __syncwarp();
            __threadfence_block();
            ok = !*abort_flag;
            if (ok) {
                if constexpr (MMA) {
                    // this lane's C fragments: k1 = c + 8 m-tile, cells 2 part and 2 part + 1
#pragma unroll
                    for (int mt = 0; mt < LbMma<K>::MT; ++mt) {
                        const int k1 = c + 8 * mt;
                        if (k1 < K) {
                            double* qr = qacc + ((size_t)row * K + k1) * C + 2 * part;
                            qr[0] += dq[mt][0];
                            qr[1] += dq[mt][1];
                        }
                    }
                } else {
                    double* qr = qacc + (size_t)row * K * C + c;
                    constexpr int KP = K / (32 / C);  // k1 per part
#pragma unroll
                    for (int k1 = 0; k1 < K; ++k1)
                        if (k1 / KP == part) qr[k1 * C] += (double)acc[k1];
                }
            }
            __syncwarp();
            if (lane == 0) {
                __threadfence_block();
                ticket[row] = ord + 1;
            }
        }
        // the warp that finishes the last item of ti refills its stage with ti + D
        __syncwarp();
        if (lane == 0) {
            __threadfence_block();
            if (atomicAdd(&done[sb], 1) == cum[ti] - 1 && ti + D < n_t && !*abort_flag) {
                __threadfence_block();
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                stage_ti[sb] = ti + D;
                issue(ti + D, sb);
            }
        }
        __syncwarp();
        cur_i = nxt_i;
        it = nit;
        se = nse;
    }
    __syncthreads();
    if (*abort_flag) return;
    // Q += the band's rows of the CTA's cells (cell-major, in place)
    for (int i = tid; i < brows * K * C; i += W * 32) {
        const int cc = i % C, k1 = (i / C) % K, r = i / (C * K);
        const long long cell = cell0 + cc;
        if (cell < a.n_cells) a.q[cell * M + (size_t)k1 * NQ + l1 * l1 + r] += qacc[i];
    }
}

// FP64: 8 cells per CTA.  FP32 (the FP32 forms: f, Phi and the K^3 step in FP32, each item's result
// added into the FP64 Q rows): 16 cells per CTA, the same shared memory.
template <int K>
__global__ void __launch_bounds__(kLbWarps * 32, 1) af_lblock64_kernel(SplitArgs a) {
    lblock_body<K, kLbCells, double, kLbWarps, true>(a);
}
template <int K>
__global__ void __launch_bounds__(kLbWarps * 32, 1) af_lblock32_kernel(SplitArgs a) {
    lblock_body<K, 2 * kLbCells, float, kLbWarps>(a);
}

// The BF16-split band kernel (CF_FORM_AF_SYM_BF16 / CF_FORM_AF_BF16 where the warp-level BF16 kernel
// does not exist, K = 12): the same units and FP64 Phi step; Phi = hi + lo and R_t = hi + lo in BF16
// (round to nearest even), and per 16-element K step the four cross products hi*hi, hi*lo, lo*hi,
// lo*lo as MMAs (tcgen05.mma kind::f16) into one FP32 accumulator in tensor memory, which runs over
// the row group's t-list and is added to the FP64 Q at the end.  About 16 significant bits per
// operand and FP32 accumulation: a reduced-precision form (~1e-5 relative to max|Q|, as the BF16
// form at K = 8); zero rows of R stay exactly zero.
template <int K, int C>
struct ShapeB {
    using S = Shape<K, C>;
    static constexpr int KK = S::KK;        // BF16 elements along K (part * EP + e)
    static constexpr int NKS = KK / 16;     // 16-element (32-byte) K steps
    static constexpr int ABYTES = 2 * NKS * S::ATILE;  // hi and lo planes of one t
    static constexpr int BSTEP = 2 * kNB * 32;          // one K step of R hi and lo: 2 x 16 rows x 32 B
    static constexpr int BBYTES = NKS * BSTEP;
};

template <int K, int C, typename T = double>
Layout bf16_layout(int n_q, int n_abuf = 2) {
    using S = Shape<K, C>;
    using SB = ShapeB<K, C>;
    Layout l{};
    int o = 0;
    auto take = [&](int bytes, int align) {
        o = (o + align - 1) / align * align;
        const int r = o;
        o += bytes;
        return r;
    };
    l.off_a = take(n_abuf * SB::ABYTES, 1024);
    l.off_b = take(kBRing * SB::BBYTES, 1024);
    l.off_f = take(C * n_q * K * (int)sizeof(T), 16);
    l.off_red = take(kSlots * C * K * (int)sizeof(double), 16);
    l.off_bar = take(16 * (int)sizeof(uint64_t), 16);
    l.off_misc = take(16 * (int)sizeof(int), 16);
    l.total = o;
    (void)S::M;
    return l;
}

// The C cells' f as T (FP64, or FP32 for the FP32 Phi step) into shared memory, as stage_f.
template <int C, typename T>
__device__ __forceinline__ void stage_f_t(const SplitArgs& a, T* fs, int M, long long cell0, int tid) {
    for (int i = tid; i < C * M; i += kThreads) {
        const int cc = i % C, r = i / C;
        const long long cell = cell0 + cc;
        fs[i] = cell < a.n_cells ? (T)__ldg(a.f + cell * M + r) : (T)0;
    }
}

__device__ __forceinline__ uint32_t bf16_bits(float x) { return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x)); }

// T: the arithmetic of the Phi step (double, or float with f staged in FP32, which halves f's
// shared memory: 8 cells per CTA at L = 16, K = 12, and an M = 128 MMA).  NAB: A buffers (1 or 2).
template <int K, int C, typename T = double, int NAB = 2>
__global__ void __launch_bounds__(kThreads, 1) af_bf16_band_kernel(SplitArgs a) {
    using S = Shape<K, C>;
    using SB = ShapeB<K, C>;
    static_assert(S::KK % 16 == 0, "whole 16-element K steps");
    static_assert(NAB == 1 || NAB == 2, "one or two A buffers");
    constexpr int KH = S::KH, KQ = S::KQ, E = S::E, EP = S::EP, NKS = SB::NKS;
    extern __shared__ __align__(1024) unsigned char smem[];
    uint8_t* sA = smem + a.off_a;
    uint8_t* sB = smem + a.off_b;
    T* fs = reinterpret_cast<T*>(smem + a.off_f);
    double* red = reinterpret_cast<double*>(smem + a.off_red);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + a.off_bar);
    uint64_t* bfull = bars;      // [2]
    uint64_t* bfree = bars + 2;  // [2]
    uint64_t* afree = bars + 4;  // [2]
    int* misc = reinterpret_cast<int*>(smem + a.off_misc);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(misc);
    volatile int* abort_flag = misc + 1;
    int* acount = misc + 2;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int c = lane % C, part = lane / C, k2o = S::k2_of(part), k3o = S::k3_of(part);
    const int NQ = a.n_q, M = NQ * K;
    const int rg = a.unit_order[blockIdx.x / a.n_cg];
    const int cg = blockIdx.x % a.n_cg;
    const int* u = a.units + (size_t)rg * U_INTS;
    const int l1 = u[U_L1], r0 = u[U_R0], nr = u[U_NR], cq = u[U_S], crem = u[U_REM], tl_off = u[U_TLOFF],
              n_t = u[U_NT], tab_off = u[U_TABOFF], brows = u[U_BROWS];
    const int n_slots = nr * cq + crem;
    const long long cell0 = (long long)cg * C;
    const int bbytes = SB::BBYTES;

    if (tid == 0) {
        for (int i = 0; i < 6; ++i) tc05::mbar_init(&bars[i], 1);
        tc05::fence_mbar_init();
        *abort_flag = 0;
        acount[0] = acount[1] = 0;
    }
    if (warp == 0) {
        tc05::tmem_alloc(tslot, 32);
        tc05::tmem_relinquish();
    }
    {
        uint4* z = reinterpret_cast<uint4*>(sA);
        for (int i = tid; i < NAB * SB::ABYTES / 16; i += kThreads) z[i] = make_uint4(0, 0, 0, 0);
    }
    stage_f_t<C, T>(a, fs, M, cell0, tid);
    tc05::tc_fence_before();
    __syncthreads();
    tc05::tc_fence_after();
    const uint32_t tbase = *tslot;
    if (tid == 0)
        for (int ti = 0; ti < min(n_t, kBRing); ++ti) {
            const int t = a.band_tl[tl_off + ti];
            tc05::mbar_arrive_expect_tx(&bfull[ti], (uint32_t)bbytes);
            tc05::bulk_g2s(sB + ti * bbytes, a.rbf + (size_t)t * bbytes, (uint32_t)bbytes, &bfull[ti]);
        }
    {   // zero the accumulator (16 FP32 columns)
        const uint32_t lb = (uint32_t)(32 * (warp & 3)) << 16;
        if (warp < 4) {
            tc05::tmem_st4(tbase + lb + 0, 0u, 0u, 0u, 0u);
            tc05::tmem_st4(tbase + lb + 4, 0u, 0u, 0u, 0u);
            tc05::tmem_st4(tbase + lb + 8, 0u, 0u, 0u, 0u);
            tc05::tmem_st4(tbase + lb + 12, 0u, 0u, 0u, 0u);
            tc05::tmem_wait_st();
        }
    }
    tc05::tc_fence_before();
    __syncthreads();
    tc05::tc_fence_after();

    const bool active = warp < n_slots;
    int srow = 0, ch = 0, nS = 1;
    if (active) slot_of(warp, cq, crem, srow, ch, nS);
    const int row = r0 + srow;
    const int m_row = warp * C + c;
    // the slot's entries of t-list position ti in cur, of ti + 1 fetched during ti, the range of ti + 2
    SlotEntries cur{0, 0, 0u, 0.0}, nxt{0, 0, 0u, 0.0};
    int ncb = 0, nce = 0;
    if (active) {
        int cb, ce;
        slot_range(a, tab_off, brows, 0, row, ch, nS, cb, ce);
        cur = slot_fetch(a, a.e_g, cb, ce, lane);
        if (n_t > 1) slot_range(a, tab_off, brows, 1, row, ch, nS, ncb, nce);
    }
    for (int ti = 0; ti < n_t; ++ti) {
        T phi[KH][KQ];
        if (active) {
            if (ti + 1 < n_t) nxt = slot_fetch(a, a.e_g, ncb, nce, lane);
            if (ti + 2 < n_t) slot_range(a, tab_off, brows, ti + 2, row, ch, nS, ncb, nce);
            slot_phi<K, C, T>(a, a.e_g, fs, NQ, cur, lane, c, k2o, k3o, phi);
            cur = nxt;
        }
        const int b = ti % NAB, use = ti / NAB;
        if (use >= 1) wait_bar(&afree[b], (uint32_t)((use - 1) & 1), abort_flag, a.err);
        uint8_t* abuf = sA + b * SB::ABYTES;
        if (active) {
            // Phi = hi + lo in BF16 (round to nearest even), two elements per 32-bit word
            auto part_bits = [&](int e, int pl) -> uint32_t {
                if (e >= E) return 0u;
                const T x = phi[(e < E ? e : 0) / KQ][(e < E ? e : 0) % KQ];
                const float hf = __bfloat162float(__float2bfloat16_rn((float)x));
                return pl == 0 ? bf16_bits(hf) : bf16_bits((float)(x - (T)hf));
            };
#pragma unroll
            for (int pl = 0; pl < 2; ++pl) {
                uint8_t* tile = abuf + pl * NKS * S::ATILE;
#pragma unroll
                for (int w = 0; w < EP / 2; ++w) {
                    const uint32_t v0 = part_bits(2 * w, pl), v1 = part_bits(2 * w + 1, pl);
                    const int byte = 2 * (part * EP + 2 * w);  // element kk = part EP + e at byte 2 kk
                    const int off = (byte >> 5) * S::ATILE + (m_row >> 3) * 256 + ((byte & 31) >> 4) * 128 +
                                    (m_row & 7) * 16 + (byte & 15);
                    *reinterpret_cast<uint32_t*>(tile + off) = v0 | (v1 << 16);
                }
            }
        }
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncwarp();
        int last = 0;
        if (lane == 0) {
            __threadfence_block();
            last = atomicAdd(&acount[b], 1) == kWarps * (use + 1) - 1;
        }
        last = __shfl_sync(0xffffffffu, last, 0);
        if (last && lane == 0 && !*abort_flag) {
            __threadfence_block();
            tc05::tc_fence_after();
            const int tn = ti + 1;
            if (tn >= kBRing && tn < n_t) {
                const int sb = tn % kBRing, useb = tn / kBRing;
                if (wait_bar(&bfree[sb], (uint32_t)((useb - 1) & 1), abort_flag, a.err)) {
                    const int t = a.band_tl[tl_off + tn];
                    tc05::mbar_arrive_expect_tx(&bfull[sb], (uint32_t)bbytes);
                    tc05::bulk_g2s(sB + sb * bbytes, a.rbf + (size_t)t * bbytes, (uint32_t)bbytes, &bfull[sb]);
                }
            }
            wait_bar(&bfull[ti % kBRing], (uint32_t)((ti / kBRing) & 1), abort_flag, a.err);
            if (!*abort_flag) {
                const uint8_t* bslot = sB + (ti % kBRing) * bbytes;
                const uint32_t idesc = tc05::idesc_bf16(S::M, kNB);
#pragma unroll
                for (int ks = 0; ks < NKS; ++ks) {
                    const uint64_t a_hi = tc05::smem_desc_kmajor(abuf + ks * S::ATILE, 128, 256);
                    const uint64_t a_lo = tc05::smem_desc_kmajor(abuf + NKS * S::ATILE + ks * S::ATILE, 128, 256);
                    const uint64_t b_hi = tc05::smem_desc_kmajor(bslot + ks * SB::BSTEP, 128, 256);
                    const uint64_t b_lo = tc05::smem_desc_kmajor(bslot + ks * SB::BSTEP + kNB * 32, 128, 256);
                    tc05::mma_bf16_ss(tbase, a_hi, b_hi, idesc, true);
                    tc05::mma_bf16_ss(tbase, a_hi, b_lo, idesc, true);
                    tc05::mma_bf16_ss(tbase, a_lo, b_hi, idesc, true);
                    tc05::mma_bf16_ss(tbase, a_lo, b_lo, idesc, true);
                }
            }
            tc05::mma_commit(&afree[b]);
            tc05::mma_commit(&bfree[ti % kBRing]);
        }
        __syncwarp();
    }
    // drain: the last uses of both A buffers cover every MMA
    bool done = true;
    for (int x = n_t - 1; x >= 0 && x > n_t - 1 - NAB; --x)
        done = wait_bar(&afree[x % NAB], (uint32_t)((x / NAB) & 1), abort_flag, a.err) && done;
    const bool ok = __all_sync(0xffffffffu, done);
    tc05::tc_fence_after();
    {
        constexpr int KG = (K + 3) / 4;
        const int m = S::M == 64 ? 16 * (warp & 3) + (lane & 15) : 32 * (warp & 3) + lane;
        const bool holds = S::M == 64 ? lane < 16 : true;
        const int s = m / C, cc = m % C, kg = warp >> 2;
        if (ok) {
            uint32_t r16[16];
            const uint32_t lb = (uint32_t)(32 * (warp & 3)) << 16;
            tc05::tmem_ld8(tbase + lb, *reinterpret_cast<uint32_t(*)[8]>(r16));
            tc05::tmem_ld8(tbase + lb + 8, *reinterpret_cast<uint32_t(*)[8]>(r16 + 8));
            tc05::tmem_wait_ld();
            if (holds && s < n_slots)
#pragma unroll
                for (int j = 0; j < KG; ++j) {
                    const int want = kg * KG + j;
                    uint32_t v = 0;
#pragma unroll
                    for (int x = 0; x < 16; ++x) v = (x == want) ? r16[x] : v;
                    if (want < K) red[(s * C + cc) * K + want] = (double)__uint_as_float(v);
                }
        }
    }
    tc05::tc_fence_before();
    __syncthreads();
    if (tid < nr * C) {
        const int rl = tid / C, cc = tid % C;
        const long long cell = cell0 + cc;
        if (cell < a.n_cells) {
            double* qc = a.q + cell * M + (l1 * l1 + r0 + rl);
            for (int k1 = 0; k1 < K; ++k1) {
                double sum = 0.0;
                const int s0 = row_first_slot(rl, cq, crem), nc = row_chunks(rl, cq, crem);
                for (int chk = 0; chk < nc; ++chk) sum += red[((s0 + chk) * C + cc) * K + k1];
                qc[(size_t)k1 * NQ] += sum;
            }
        }
    }
    tc05::tc_fence_before();
    __syncthreads();
    if (warp == 0) tc05::tmem_dealloc(tbase, 32);
}

}  // namespace

// ------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------
struct SplitPlan {
    int device = 0, n_q = 0, k = 0, n_l = 0, L = 0;
    int n_rg = 0, tseg = 1, n_abuf = 1;
    int n_rg64 = 0, w64 = 16;         // the FP64 band kernel's row groups and warps per CTA
    int cells = 4;                    // cells per CTA (C)
    int64_t bytes = 0;
    int smem = 0;
    const int* slice_e = nullptr;     // borrowed from the folded plan
    const uint32_t* e_q23 = nullptr;  // borrowed
    uint8_t* d_rplanes = nullptr;
    double* d_e_gs = nullptr;
    int* d_rb_off = nullptr;
    double* d_rb_gs = nullptr;
    int* d_rb_l23 = nullptr;
    int* d_units = nullptr;
    int* d_unit_order = nullptr;
    int* d_units64 = nullptr;         // the FP64 band kernel's row groups (w64 slots each) and their order
    int* d_unit_order64 = nullptr;
    int* d_band_tl = nullptr;
    int* d_band_rng = nullptr;        // per band: [n_t][rows] (begin, end) of the (t, row) slice's entries
    int* d_err = nullptr;             // set to 1 by a CTA whose bounded wait gave up
    const double* e_g = nullptr;      // borrowed: G in slice order (FP64 band kernel)
    double* d_rfp64 = nullptr;        // FP64 R_t per t as [part][e][k1] (FP64 band kernel)
    uint8_t* d_rbf = nullptr;         // BF16 hi and lo planes of R_t (BF16-split band kernel)
    uint8_t* d_rbf8 = nullptr;        // K = 12: the same for 8 cells per CTA (Phi in FP32)
    double* d_rfl = nullptr;          // the FP64 l-block kernel: R_t as MMA A fragments [t][m-tile][k-step][lane]
    int* d_t_l23 = nullptr;           // per l-triplet: l2 | l3 << 8
    // the l-block kernel (0 bands: unsupported)
    int lb_bands = 0, lb_rows = 0, lb_t = 0;  // bands, rows of the largest band, longest t-list
    int lb_ring = 0, lb_stage = 0;    // stages in the ring, bytes per stage (FP64, 8 cells per CTA)
    int lb32_ring = 0, lb32_stage = 0;  // the same for the FP32 forms (16 cells per CTA)
    float* d_rfl32 = nullptr;         // FP32 R_t as [part][e][k1] for 16 cells per CTA
    Layout laylb32{};
    int* d_lb_units = nullptr;        // per band: LBU_INTS ints
    int* d_lb_order = nullptr;        // bands, heaviest first
    int4* d_lb_items = nullptr;       // per band: its (t, row) slices in t-major order
    int* d_lb_titems = nullptr;       // per t-list position: its items
    Layout lay{};
    Layout lay64{};
    Layout laybf{};
    Layout laybf8{};                  // K = 12: 8 cells per CTA, f and Phi in FP32, one A buffer
    Layout laylb{};                   // the l-block kernel
};

namespace {

int fail_split(int st, const std::string& msg) {
    cf_set_last_error(msg.c_str());
    return st;
}

template <typename T>
cudaError_t upload_vec(T** dst, const std::vector<T>& v, int64_t& bytes) {
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

int isqrt_int(int q) {
    int l = (int)std::sqrt((double)q);
    while (l * l > q) --l;
    while ((l + 1) * (l + 1) <= q) ++l;
    return l;
}

template <int K, int C>
void split_r_planes(const std::vector<double>& R, int n_l, std::vector<uint8_t>& planes, std::vector<double>& st_scale) {
    using S = Shape<K, C>;
    const size_t per_t = (size_t)S::NKS * kBStep;
    planes.assign(per_t * n_l, 0);
    st_scale.assign(n_l, 1.0);
    for (int t = 0; t < n_l; ++t) {
        const double* Rt = R.data() + (size_t)t * K * K * K;
        double mx = 0.0;
        for (int i = 0; i < K * K * K; ++i) mx = std::max(mx, std::fabs(Rt[i]));
        int x = 0;
        if (mx > 0.0) std::frexp(mx, &x);  // mx < 2^x
        const double s = std::ldexp(1.0, -x);
        st_scale[t] = s;
        uint8_t* pt = planes.data() + per_t * t;
        for (int p = 0; p < S::P; ++p)
            for (int e = 0; e < S::E; ++e) {
                const int k2 = S::k2_of(p) + e / S::KQ, k3 = S::k3_of(p) + e % S::KQ;
                const int kk = p * S::EP + e;
                const int ks = kk >> 5, kb = kk & 31;
                for (int k1 = 0; k1 < K; ++k1) {
                    long long X = (long long)std::nearbyint(std::ldexp(Rt[k1 + K * k2 + K * K * k3] * s, kRShift));
                    for (int j = 0; j < kPlanes; ++j) {
                        long long d = ((X % 256) + 256) % 256;  // 0..255
                        if (d >= 128) d -= 256;                 // balanced digit in [-128, 127]
                        X = (X - d) / 256;
                        const int n = j * kNB + k1;
                        const size_t off = (size_t)ks * kBStep + (n >> 3) * 256 + (kb >> 4) * 128 + (n & 7) * 16 + (kb & 15);
                        pt[off] = (uint8_t)(int8_t)d;
                    }
                }
            }
    }
}

// BF16 bits of a finite float, rounded to nearest even, and back
uint16_t host_bf16_bits(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    u += 0x7fffu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

float host_bf16_value(uint16_t b) {
    const uint32_t u = (uint32_t)b << 16;
    float x;
    std::memcpy(&x, &u, 4);
    return x;
}

// R_t = hi + lo in BF16 as the B operand of the BF16-split band kernel: per t and 16-element K step,
// the hi plane then the lo plane, each 16 rows (k1, zero past K) x 32 bytes in the canonical K-major
// layout; element kk = part EP + e holds (k2, k3) of part's e-th Phi element, zero for e >= E.
template <int K, int C>
void split_r_bf16(const std::vector<double>& R, int n_l, std::vector<uint8_t>& planes) {
    using S = Shape<K, C>;
    using SB = ShapeB<K, C>;
    const size_t per_t = (size_t)SB::BBYTES;
    planes.assign(per_t * n_l, 0);
    for (int t = 0; t < n_l; ++t) {
        const double* Rt = R.data() + (size_t)t * K * K * K;
        uint8_t* pt = planes.data() + per_t * t;
        for (int p = 0; p < S::P; ++p)
            for (int e = 0; e < S::E; ++e) {
                const int k2 = S::k2_of(p) + e / S::KQ, k3 = S::k3_of(p) + e % S::KQ;
                const int byte = 2 * (p * S::EP + e);
                const int ks = byte >> 5, kb = byte & 31;
                for (int k1 = 0; k1 < K; ++k1) {
                    const double r = Rt[k1 + K * k2 + K * K * k3];
                    const uint16_t hi = host_bf16_bits((float)r);
                    const uint16_t lo = host_bf16_bits((float)(r - (double)host_bf16_value(hi)));
                    for (int pl = 0; pl < 2; ++pl) {
                        const size_t off = (size_t)ks * SB::BSTEP + pl * kNB * 32 + (k1 >> 3) * 256 + (kb >> 4) * 128 +
                                           (k1 & 7) * 16 + (kb & 15);
                        const uint16_t v = pl == 0 ? hi : lo;
                        std::memcpy(pt + off, &v, 2);
                    }
                }
            }
    }
}

template <int K, int C>
int build_impl(SplitPlan* sp, const DevOp& op, int64_t n_g, int64_t n_slices) {
    using S = Shape<K, C>;
    const int NQ = op.n_q, NL = op.n_l;
    const int L = isqrt_int(NQ) - 1;
    if ((L + 1) * (L + 1) != NQ) return fail_split(CF_EUNSUPPORTED, "split form: N_Q is not (L+1)^2");
    std::vector<int> q1_begin, slice_t, slice_e;
    std::vector<uint32_t> e_q23;
    std::vector<double> e_g, R;
    cudaError_t ce = download(q1_begin, op.q1_begin, (size_t)NQ + 1);
    if (ce == cudaSuccess) ce = download(slice_t, op.slice_t, (size_t)n_slices);
    if (ce == cudaSuccess) ce = download(slice_e, op.slice_e, (size_t)n_slices + 1);
    if (ce == cudaSuccess) ce = download(e_q23, op.e_q23, (size_t)n_g);
    if (ce == cudaSuccess) ce = download(e_g, op.e_g, (size_t)n_g);
    if (ce == cudaSuccess) ce = download(R, op.R, (size_t)K * K * K * NL);
    if (ce != cudaSuccess) return fail_split(CF_ECUDA, std::string("split form: download: ") + cudaGetErrorString(ce));

    std::vector<uint8_t> planes, rbf;
    std::vector<double> st;
    split_r_planes<K, C>(R, NL, planes, st);
    split_r_bf16<K, C>(R, NL, rbf);
    std::vector<uint8_t> rbf8;
    if constexpr (K == 12) split_r_bf16<12, 8>(R, NL, rbf8);
    // FP64 R_t per t as [part][e][k1] with zero padding after each part
    std::vector<double> rfp64((size_t)NL * S::P * S::PS, 0.0);
    for (int t = 0; t < NL; ++t)
        for (int pp = 0; pp < S::P; ++pp)
            for (int e = 0; e < S::E; ++e) {
                const int k2 = S::k2_of(pp) + e / S::KQ, k3 = S::k3_of(pp) + e % S::KQ;
                for (int k1 = 0; k1 < K; ++k1)
                    rfp64[((size_t)t * S::P + pp) * S::PS + (size_t)e * K + k1] =
                        R[(size_t)t * K * K * K + k1 + (size_t)K * k2 + (size_t)K * K * k3];
            }
    // the l-block kernels' R_t: FP32 for 16 cells per CTA (LbShape), FP64 for 8 as MMA A fragments
    std::vector<double> rfl;
    std::vector<float> rfl32;
    if constexpr (lblock_supported_k(K)) {
        auto fill = [&](auto shape, auto& out) {
            using S8 = decltype(shape);
            out.assign((size_t)NL * S8::P * S8::PS, 0);
            for (int t = 0; t < NL; ++t)
                for (int pp = 0; pp < S8::P; ++pp)
                    for (int e = 0; e < S8::E; ++e) {
                        const int k2 = e / S8::KQ, k3 = S8::k3(pp, e % S8::KQ);
                        for (int k1 = 0; k1 < K; ++k1)
                            out[((size_t)t * S8::P + pp) * S8::PS + (size_t)e * K + k1] =
                                (typename std::decay_t<decltype(out)>::value_type)R[(size_t)t * K * K * K + k1 +
                                                                                   (size_t)K * k2 + (size_t)K * K * k3];
                    }
        };
        fill(LbShape<K, 2 * kLbCells, float>{}, rfl32);
        // FP64: A fragments of the m8n8k4 MMAs, [t][m-tile][k-step][lane] (LbMma)
        using LM = LbMma<K>;
        rfl.assign((size_t)NL * LM::MT * LM::S * 32, 0.0);
        for (int t = 0; t < NL; ++t)
            for (int mt = 0; mt < LM::MT; ++mt)
                for (int ks = 0; ks < LM::S; ++ks)
                    for (int ln = 0; ln < 32; ++ln) {
                        const int k1 = (ln >> 2) + 8 * mt, p4 = ln & 3;
                        const int k2 = ks / LM::KQ, k3 = p4 * LM::KQ + ks % LM::KQ;
                        if (k1 < K)
                            rfl[(((size_t)t * LM::MT + mt) * LM::S + ks) * 32 + ln] =
                                R[(size_t)t * K * K * K + k1 + (size_t)K * k2 + (size_t)K * K * k3];
                    }
    }
    // G / s_t per entry, |G / s_t| summed per slice, (l2, l3) per t
    std::vector<double> e_gs(n_g), gs(n_slices, 0.0);
    std::vector<int> t_l23(NL, -1);
    std::vector<int> slice_q1(n_slices, -1);
    for (int q = 0; q < NQ; ++q)
        for (int s = q1_begin[q]; s < q1_begin[q + 1]; ++s) slice_q1[s] = q;
    for (int64_t s = 0; s < n_slices; ++s) {
        const int t = slice_t[s];
        for (int z = slice_e[s]; z < slice_e[s + 1]; ++z) {
            e_gs[z] = e_g[z] / st[t];
            gs[s] += std::fabs(e_gs[z]);
            const int l2 = isqrt_int((int)(e_q23[z] & 0xffffu)), l3 = isqrt_int((int)(e_q23[z] >> 16));
            const int v = l2 | (l3 << 8);
            if (t_l23[t] < 0) t_l23[t] = v;
            if (t_l23[t] != v) return fail_split(CF_EUNSUPPORTED, "split form: an l-triplet's entries mix (l2, l3)");
        }
    }
    for (int t = 0; t < NL; ++t)
        if (t_l23[t] < 0) t_l23[t] = 0;
    // per row, its slices' bound factors, contiguous (the kernel reads them once per (row, cell))
    std::vector<int> rb_off(NQ + 1, 0), rb_l23;
    std::vector<double> rb_gs;
    for (int q = 0; q < NQ; ++q) {
        for (int s2 = q1_begin[q]; s2 < q1_begin[q + 1]; ++s2) {
            rb_gs.push_back(gs[s2]);
            rb_l23.push_back(t_l23[slice_t[s2]]);
        }
        rb_off[q + 1] = (int)rb_gs.size();
    }
    // bands: t-lists and the (t, row) -> slice tables
    struct BandInfo {
        int l1, brows, tl_off, n_t, tab_off;
        std::vector<double> row_work;
    };
    std::vector<BandInfo> bands;
    std::vector<int> band_tl, band_slice;
    for (int l1 = 0; l1 <= L; ++l1) {
        const int qa = l1 * l1, brows = 2 * l1 + 1;
        std::vector<int> ts;
        for (int r = 0; r < brows; ++r)
            for (int s = q1_begin[qa + r]; s < q1_begin[qa + r + 1]; ++s) ts.push_back(slice_t[s]);
        std::sort(ts.begin(), ts.end());
        ts.erase(std::unique(ts.begin(), ts.end()), ts.end());
        if (ts.empty()) continue;
        const int tl_off = (int)band_tl.size(), tab_off = (int)band_slice.size();
        band_tl.insert(band_tl.end(), ts.begin(), ts.end());
        band_slice.insert(band_slice.end(), ts.size() * brows, -1);
        std::vector<double> row_work(brows, 0.0);
        for (int r = 0; r < brows; ++r)
            for (int s = q1_begin[qa + r]; s < q1_begin[qa + r + 1]; ++s) {
                const int ti = (int)(std::lower_bound(ts.begin(), ts.end(), slice_t[s]) - ts.begin());
                int& cell = band_slice[tab_off + (size_t)ti * brows + r];
                if (cell >= 0) return fail_split(CF_EUNSUPPORTED, "split form: a (t, q1) pair has two slices");
                cell = s;
                row_work[r] += (double)(slice_e[s + 1] - slice_e[s]);
            }
        bands.push_back({l1, brows, tl_off, (int)ts.size(), tab_off, row_work});
    }
    // row groups for a kernel of `cap` slots (one per warp): as few as the slots allow (every group
    // walks the whole t-list, so the per-t costs scale with the number of groups); a group of
    // nr < cap rows splits each row's entries into cap / nr chunks, one more for the first cap % nr
    // rows, so that every warp has work.
    // Returns the units and their order, heaviest first.
    auto make_units = [&](int cap, std::vector<int>& units, std::vector<int>& order) {
        std::vector<double> work;
        units.clear();
        for (const BandInfo& bd : bands) {
            const int best_g = (bd.brows + cap - 1) / cap;
            int r = 0;
            for (int gi = 0; gi < best_g; ++gi) {
                const int nr = (bd.brows - r + (best_g - gi) - 1) / (best_g - gi);
                const int uu[U_INTS] = {bd.l1, r, nr, cap / nr, bd.tl_off, bd.n_t, bd.tab_off, bd.brows, cap % nr};
                units.insert(units.end(), uu, uu + U_INTS);
                double w = 0.0;
                for (int x = r; x < r + nr; ++x) w += bd.row_work[x];
                work.push_back(w * K * K + (double)bd.n_t * 4096.0);
                r += nr;
            }
        }
        order.resize(work.size());
        for (size_t i = 0; i < work.size(); ++i) order[i] = (int)i;
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return work[x] > work[y]; });
        return (int)work.size();
    };
    std::vector<int> units, order, units64, order64;
    const int n_rg = make_units(kSlots, units, order);
    const int w64 = band64_warps(K);
    const int n_rg64 = make_units(w64, units64, order64);
    // the l-block kernel: per band, its (t, row) slices in t-major order, each with its ordinal among
    // its row's slices (the row's ticket) and the (l2, l3) of its t
    std::vector<int> units_lb, order_lb, titems_lb(band_tl.size(), 0);
    std::vector<int4> items_lb;
    std::vector<double> work_lb;
    int lb_rows = 0, lb_t = 0;
    bool lb_ok = L < 128;
    for (const BandInfo& bd : bands) {
        const int it_off = (int)items_lb.size();
        std::vector<int> ord(bd.brows, 0);
        for (int ti = 0; ti < bd.n_t; ++ti) {
            const int t = band_tl[bd.tl_off + ti];
            const int l23 = t_l23[t];
            for (int r = 0; r < bd.brows; ++r) {
                const int sl = band_slice[bd.tab_off + (size_t)ti * bd.brows + r];
                if (sl < 0) continue;
                items_lb.push_back(make_int4(ti | (r << 16), ord[r]++ | ((l23 & 0xff) << 16) | ((l23 >> 8) << 24),
                                              slice_e[sl], slice_e[sl + 1]));
                ++titems_lb[bd.tl_off + ti];
            }
        }
        const int uu[LBU_INTS] = {bd.l1, bd.brows, bd.tl_off, bd.n_t, it_off, (int)items_lb.size() - it_off, 0, 0};
        units_lb.insert(units_lb.end(), uu, uu + LBU_INTS);
        double w = 0.0;
        for (double x : bd.row_work) w += x;
        work_lb.push_back(w * K * K + (double)(items_lb.size() - it_off) * K * K * K);
        lb_rows = std::max(lb_rows, bd.brows);
        lb_t = std::max(lb_t, bd.n_t);
        if (bd.n_t > 0xffff || bd.brows > 0x7fff) lb_ok = false;
    }
    order_lb.resize(work_lb.size());
    for (size_t i = 0; i < work_lb.size(); ++i) order_lb[i] = (int)i;
    std::stable_sort(order_lb.begin(), order_lb.end(), [&](int x, int y) { return work_lb[x] > work_lb[y]; });
    // the (t, row) tables as entry ranges (begin, end), empty where the row has no slice of t
    std::vector<int> band_rng(2 * band_slice.size(), 0);
    for (size_t i = 0; i < band_slice.size(); ++i)
        if (band_slice[i] >= 0) {
            band_rng[2 * i] = slice_e[band_slice[i]];
            band_rng[2 * i + 1] = slice_e[band_slice[i] + 1];
        }
    sp->n_q = NQ;
    sp->k = K;
    sp->n_l = NL;
    sp->L = L;
    sp->n_rg = n_rg;
    sp->n_rg64 = n_rg64;
    sp->lb_bands = lb_ok && lblock_supported_k(K) ? (int)work_lb.size() : 0;
    sp->lb_rows = lb_rows;
    sp->lb_t = lb_t;
    sp->w64 = w64;
    // int32 accumulators: at most 6 byte products of |255 * 128| per K element and weight
    sp->tseg = std::max(1, (int)(2147483647LL / (6LL * 255 * 128 * S::KK)));
    sp->slice_e = op.slice_e;
    sp->e_q23 = op.e_q23;
    sp->e_g = op.e_g;
    int optin = 0;
    cudaGetDevice(&sp->device);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, sp->device);
    sp->cells = C;
    sp->n_abuf = 2;
    sp->lay = smem_layout<K, C>(NQ, L, 2);
    if (sp->lay.total > optin) {
        sp->n_abuf = 1;
        sp->lay = smem_layout<K, C>(NQ, L, 1);
    }
    sp->lay64 = band64_layout<K, C>(NQ, w64);
    // the l-block kernel: a stage holds R_t and the row blocks of bands l2 and l3 of one t
    if constexpr (lblock_supported_k(K)) {
        int max_rows = 0;
        for (int t : band_tl) {
            const int l2 = t_l23[t] & 0xff, l3 = t_l23[t] >> 8;
            max_rows = std::max(max_rows, 2 * l2 + 1 + (l3 != l2 ? 2 * l3 + 1 : 0));
        }
        // FP64, 8 cells; FP32, 16 cells: the same bytes per f row
        const int stage = (LbMma<K>::RT_BYTES + max_rows * K * kLbCells * (int)sizeof(double) + 127) / 128 * 128;
        const int stage32 =
            (LbShape<K, 2 * kLbCells, float>::RT_BYTES + max_rows * K * 2 * kLbCells * (int)sizeof(float) + 127) / 128 *
            128;
        int ring = kLbMaxRing, ring32 = kLbMaxRing;
        while (ring >= 2 && lblock_layout(ring, stage, K, lb_rows, lb_t, kLbCells).total > optin) --ring;
        while (ring32 >= 2 && lblock_layout(ring32, stage32, K, lb_rows, lb_t, 2 * kLbCells).total > optin) --ring32;
        if (ring >= 2) {
            sp->lb_ring = ring;
            sp->lb_stage = stage;
            sp->laylb = lblock_layout(ring, stage, K, lb_rows, lb_t, kLbCells);
        }
        if (ring32 >= 2) {
            sp->lb32_ring = ring32;
            sp->lb32_stage = stage32;
            sp->laylb32 = lblock_layout(ring32, stage32, K, lb_rows, lb_t, 2 * kLbCells);
        }
    }
    sp->laybf = bf16_layout<K, C>(NQ);
    if constexpr (K == 12) sp->laybf8 = bf16_layout<12, 8, float>(NQ, 1);
    sp->smem = sp->lay.total;
    int64_t bytes = 0;
    if ((ce = upload_vec(&sp->d_rplanes, planes, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_e_gs, e_gs, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_rb_off, rb_off, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_rb_gs, rb_gs, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_rb_l23, rb_l23, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_units, units, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_unit_order, order, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_units64, units64, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_unit_order64, order64, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_band_tl, band_tl, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_band_rng, band_rng, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_err, std::vector<int>(1, 0), bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_rfp64, rfp64, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_rbf, rbf, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_rbf8, rbf8, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_rfl, rfl, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_rfl32, rfl32, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_lb_units, units_lb, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_lb_order, order_lb, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_lb_items, items_lb, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_lb_titems, titems_lb, bytes)) != cudaSuccess ||
        (ce = upload_vec(&sp->d_t_l23, t_l23, bytes)) != cudaSuccess)
        return fail_split(ce == cudaErrorMemoryAllocation ? CF_ENOMEM : CF_ECUDA,
                          std::string("split form: upload: ") + cudaGetErrorString(ce));
    sp->bytes = bytes;
    return CF_OK;
}

template <int K, int C>
int run_impl(const SplitPlan* sp, double* q_cm, const double* f_cm, int64_t B, cudaStream_t st, int64_t* launches) {
    static bool attr_set[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        const cudaError_t e = cudaFuncSetAttribute(af_split_kernel<K, C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   227 * 1024);
        if (e != cudaSuccess)
            return fail_split(CF_ECUDA, std::string("split form: smem attribute: ") + cudaGetErrorString(e));
        attr_set[dev] = true;
    }
    SplitArgs a{};
    a.slice_e = sp->slice_e;
    a.e_q23 = sp->e_q23;
    a.e_gs = sp->d_e_gs;
    a.rplanes = sp->d_rplanes;
    a.rb_off = sp->d_rb_off;
    a.rb_gs = sp->d_rb_gs;
    a.rb_l23 = sp->d_rb_l23;
    a.units = sp->d_units;
    a.unit_order = sp->d_unit_order;
    a.band_tl = sp->d_band_tl;
    a.band_rng = sp->d_band_rng;
    a.f = f_cm;
    a.q = q_cm;
    a.err = sp->d_err;
    a.n_cells = B;
    a.n_cg = (int)((B + C - 1) / C);
    a.n_q = sp->n_q;
    a.L = sp->L;
    a.tseg = sp->tseg;
    a.n_abuf = sp->n_abuf;
    a.off_a = sp->lay.off_a;
    a.off_b = sp->lay.off_b;
    a.off_f = sp->lay.off_f;
    a.off_mb = sp->lay.off_mb;
    a.off_red = sp->lay.off_red;
    a.off_scale = sp->lay.off_scale;
    a.off_eexp = sp->lay.off_eexp;
    a.off_bar = sp->lay.off_bar;
    a.off_misc = sp->lay.off_misc;
    const long long blocks = (long long)sp->n_rg * a.n_cg;
    if (blocks > 0x7fffffffLL) return fail_split(CF_ESHAPE, "split form: batch too large for one launch");
    af_split_kernel<K, C><<<(unsigned)blocks, kThreads, sp->smem, st>>>(a);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_split(CF_ECUDA, std::string("split form: launch: ") + cudaGetErrorString(e));
    if (launches) ++*launches;
    return CF_OK;
}

template <int K, int C>
int run64_impl(const SplitPlan* sp, double* q_cm, const double* f_cm, int64_t B, cudaStream_t st, int64_t* launches) {
    constexpr int W = band64_warps(K);
    static bool attr_set[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        const cudaError_t e = cudaFuncSetAttribute(af_band64_kernel<K, C, W>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        if (e != cudaSuccess)
            return fail_split(CF_ECUDA, std::string("band kernel: smem attribute: ") + cudaGetErrorString(e));
        attr_set[dev] = true;
    }
    SplitArgs a{};
    a.slice_e = sp->slice_e;
    a.e_q23 = sp->e_q23;
    a.e_g = sp->e_g;
    a.rfp64 = sp->d_rfp64;
    a.units = sp->d_units64;
    a.unit_order = sp->d_unit_order64;
    a.band_tl = sp->d_band_tl;
    a.band_rng = sp->d_band_rng;
    a.f = f_cm;
    a.q = q_cm;
    a.err = sp->d_err;
    a.n_cells = B;
    a.n_cg = (int)((B + C - 1) / C);
    a.n_q = sp->n_q;
    a.L = sp->L;
    a.off_b = sp->lay64.off_b;
    a.off_f = sp->lay64.off_f;
    a.off_red = sp->lay64.off_red;
    a.off_bar = sp->lay64.off_bar;
    a.off_misc = sp->lay64.off_misc;
    const long long blocks = (long long)sp->n_rg64 * a.n_cg;
    if (blocks > 0x7fffffffLL) return fail_split(CF_ESHAPE, "band kernel: batch too large for one launch");
    af_band64_kernel<K, C, W><<<(unsigned)blocks, W * 32, sp->lay64.total, st>>>(a);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_split(CF_ECUDA, std::string("band kernel: launch: ") + cudaGetErrorString(e));
    if (launches) ++*launches;
    return CF_OK;
}

// Bytes of the packed f that the l-block kernels read: [ceil(B / C)][N_Q][K][C] of T.
size_t lblock_pack_bytes_of(int n_q, int k, int64_t B, bool f32) {
    const int C = f32 ? 2 * kLbCells : kLbCells;
    return (size_t)((B + C - 1) / C) * (size_t)n_q * k * C * (f32 ? sizeof(float) : sizeof(double));
}

template <int K, typename T>
int runlb_impl(const SplitPlan* sp, double* q_cm, const double* f_cm, void* pf, int64_t B, cudaStream_t st,
               int64_t* launches, long long wait_cycles = kWaitCycles, bool no_copy = false) {
    constexpr bool F32 = sizeof(T) == 4;
    constexpr int C = F32 ? 2 * kLbCells : kLbCells, W = kLbWarps;
    auto kern = F32 ? (void (*)(SplitArgs))af_lblock32_kernel<K> : (void (*)(SplitArgs))af_lblock64_kernel<K>;
    const Layout& lay = F32 ? sp->laylb32 : sp->laylb;
    static bool attr_set[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        const cudaError_t e = cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   227 * 1024);
        if (e != cudaSuccess)
            return fail_split(CF_ECUDA, std::string("l-block kernel: smem attribute: ") + cudaGetErrorString(e));
        attr_set[dev] = true;
    }
    const long long n_cg = (B + C - 1) / C;
    const long long pblocks = n_cg * ((sp->n_q + 31) / 32);
    if (pblocks > 0x7fffffffLL || (long long)sp->lb_bands * n_cg > 0x7fffffffLL)
        return fail_split(CF_ESHAPE, "l-block kernel: batch too large for one launch");
    const unsigned pgrid = (unsigned)pblocks;
    static_assert(32 * K * C * sizeof(T) <= 48 * 1024, "the pack kernel's tile fits the default shared memory");
    // FP64: [q][cell][k] rows for the tensor-core kernel; FP32: [q][k][cell]
    pack_cg_kernel<C, T, !F32><<<pgrid, 256, 32 * K * C * sizeof(T), st>>>(f_cm, static_cast<T*>(pf), B, sp->n_q, K);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_split(CF_ECUDA, std::string("l-block pack: launch: ") + cudaGetErrorString(e));
    if (launches) ++*launches;
    SplitArgs a{};
    a.slice_e = sp->slice_e;
    a.e_q23 = sp->e_q23;
    a.e_g = sp->e_g;
    a.rfp64 = F32 ? reinterpret_cast<const double*>(sp->d_rfl32) : sp->d_rfl;  // read as T by the kernel
    a.units = sp->d_lb_units;
    a.unit_order = sp->d_lb_order;
    a.band_tl = sp->d_band_tl;
    a.items = sp->d_lb_items;
    a.t_items = sp->d_lb_titems;
    a.pf = static_cast<const double*>(pf);  // read as T by the kernel
    a.t_l23 = sp->d_t_l23;
    a.q = q_cm;
    a.err = sp->d_err;
    a.n_cells = B;
    a.n_cg = (int)n_cg;
    a.n_q = sp->n_q;
    a.L = sp->L;
    a.n_ring = F32 ? sp->lb32_ring : sp->lb_ring;
    a.stage_bytes = F32 ? sp->lb32_stage : sp->lb_stage;
    a.max_rows = sp->lb_rows;
    a.max_t = sp->lb_t;
    a.wait_cycles = wait_cycles;
    a.no_copy = no_copy ? 1 : 0;
    a.off_b = lay.off_b;
    a.off_red = lay.off_red;
    a.off_bar = lay.off_bar;
    a.off_misc = lay.off_misc;
    const long long blocks = (long long)sp->lb_bands * n_cg;
    kern<<<(unsigned)blocks, W * 32, lay.total, st>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail_split(CF_ECUDA, std::string("l-block kernel: launch: ") + cudaGetErrorString(e));
    if (launches) ++*launches;
    return CF_OK;
}

template <int K, int C, typename T = double, int NAB = 2>
int runbf_impl(const SplitPlan* sp, double* q_cm, const double* f_cm, int64_t B, cudaStream_t st, int64_t* launches) {
    const Layout& lay = (std::is_same<T, float>::value && K == 12) ? sp->laybf8 : sp->laybf;
    const uint8_t* planes = (std::is_same<T, float>::value && K == 12) ? sp->d_rbf8 : sp->d_rbf;
    static bool attr_set[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        const cudaError_t e = cudaFuncSetAttribute(af_bf16_band_kernel<K, C, T, NAB>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        if (e != cudaSuccess)
            return fail_split(CF_ECUDA, std::string("BF16 band kernel: smem attribute: ") + cudaGetErrorString(e));
        attr_set[dev] = true;
    }
    SplitArgs a{};
    a.slice_e = sp->slice_e;
    a.e_q23 = sp->e_q23;
    a.e_g = sp->e_g;
    a.rbf = planes;
    a.units = sp->d_units;
    a.unit_order = sp->d_unit_order;
    a.band_tl = sp->d_band_tl;
    a.band_rng = sp->d_band_rng;
    a.f = f_cm;
    a.q = q_cm;
    a.err = sp->d_err;
    a.n_cells = B;
    a.n_cg = (int)((B + C - 1) / C);
    a.n_q = sp->n_q;
    a.L = sp->L;
    a.off_a = lay.off_a;
    a.off_b = lay.off_b;
    a.off_f = lay.off_f;
    a.off_red = lay.off_red;
    a.off_bar = lay.off_bar;
    a.off_misc = lay.off_misc;
    const long long blocks = (long long)sp->n_rg * a.n_cg;
    if (blocks > 0x7fffffffLL) return fail_split(CF_ESHAPE, "BF16 band kernel: batch too large for one launch");
    af_bf16_band_kernel<K, C, T, NAB><<<(unsigned)blocks, kThreads, lay.total, st>>>(a);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_split(CF_ECUDA, std::string("BF16 band kernel: launch: ") + cudaGetErrorString(e));
    if (launches) ++*launches;
    return CF_OK;
}

}  // namespace

bool split_supported_k(int k) { return k == 4 || k == 8 || k == 12; }

int bf16_band_run(const SplitPlan* sp, double* q_cm, const double* f_cm, int64_t B, cudaStream_t st, int64_t* launches) {
    if (B <= 0 || sp->n_rg == 0) return CF_OK;
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, sp->device);
    // K = 12: Phi in FP32 on 8 cells per CTA (M = 128) where its shared memory fits
    if (sp->k == 12 && sp->laybf8.total > 0 && sp->laybf8.total <= optin)
        return runbf_impl<12, 8, float, 1>(sp, q_cm, f_cm, B, st, launches);
    if (sp->laybf.total > optin) {
        char msg[160];
        snprintf(msg, sizeof(msg), "BF16 band kernel: %d bytes of shared memory needed, %d available", sp->laybf.total,
                 optin);
        return fail_split(CF_EUNSUPPORTED, msg);
    }
    switch (sp->k) {
        case 4: return runbf_impl<4, 4>(sp, q_cm, f_cm, B, st, launches);
        case 8: return sp->cells == 8 ? runbf_impl<8, 8>(sp, q_cm, f_cm, B, st, launches)
                                      : runbf_impl<8, 4>(sp, q_cm, f_cm, B, st, launches);
        default: return runbf_impl<12, 4>(sp, q_cm, f_cm, B, st, launches);
    }
}

int band64_run(const SplitPlan* sp, double* q_cm, const double* f_cm, int64_t B, cudaStream_t st, int64_t* launches) {
    if (B <= 0 || sp->n_rg64 == 0) return CF_OK;
    switch (sp->k) {
        case 4: return run64_impl<4, 4>(sp, q_cm, f_cm, B, st, launches);
        case 8: return sp->cells == 8 ? run64_impl<8, 8>(sp, q_cm, f_cm, B, st, launches)
                                      : run64_impl<8, 4>(sp, q_cm, f_cm, B, st, launches);
        default: return run64_impl<12, 4>(sp, q_cm, f_cm, B, st, launches);
    }
}

size_t lblock_pack_bytes(const SplitPlan* sp, int64_t B, bool f32) { return lblock_pack_bytes_of(sp->n_q, sp->k, B, f32); }

bool lblock_available(const SplitPlan* sp, bool f32) {
    return sp && lblock_supported_k(sp->k) && sp->lb_bands > 0 && (f32 ? sp->lb32_ring : sp->lb_ring) >= 2;
}

int lblock_run(const SplitPlan* sp, double* q_cm, const double* f_cm, void* pf, size_t pf_bytes, int64_t B, bool f32,
               cudaStream_t st, int64_t* launches) {
    if (B <= 0) return CF_OK;
    if (!lblock_available(sp, f32))
        return fail_split(CF_EUNSUPPORTED, "l-block kernel: needs K = 8 or 12 and two stages of shared memory");
    if (pf_bytes < lblock_pack_bytes(sp, B, f32))
        return fail_split(CF_EINVAL, "l-block kernel: packed-f workspace too small");
    if (f32)
        return sp->k == 8 ? runlb_impl<8, float>(sp, q_cm, f_cm, pf, B, st, launches)
                          : runlb_impl<12, float>(sp, q_cm, f_cm, pf, B, st, launches);
    return sp->k == 8 ? runlb_impl<8, double>(sp, q_cm, f_cm, pf, B, st, launches)
                      : runlb_impl<12, double>(sp, q_cm, f_cm, pf, B, st, launches);
}

int lblock_selftest(const SplitPlan* sp, double* q_cm, const double* f_cm, void* pf, size_t pf_bytes, int64_t B,
                    long long wait_cycles, cudaStream_t st, int64_t* launches) {
    if (B <= 0) return fail_split(CF_EINVAL, "l-block self-test: no cells");
    if (!lblock_available(sp, false))
        return fail_split(CF_EUNSUPPORTED, "l-block kernel: needs K = 8 or 12 and two stages of shared memory");
    if (pf_bytes < lblock_pack_bytes(sp, B, false))
        return fail_split(CF_EINVAL, "l-block kernel: packed-f workspace too small");
    const int r = sp->k == 8 ? runlb_impl<8, double>(sp, q_cm, f_cm, pf, B, st, launches, wait_cycles, true)
                             : runlb_impl<12, double>(sp, q_cm, f_cm, pf, B, st, launches, wait_cycles, true);
    if (r != CF_OK) return r;
    const cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail_split(CF_ECUDA, std::string("l-block self-test: ") + cudaGetErrorString(e));
    return split_check(sp);
}

int split_build(SplitPlan** out, const DevOp& folded, int64_t n_g, int64_t n_slices, int device) {
    *out = nullptr;
    if (!split_supported_k(folded.k))
        return fail_split(CF_EUNSUPPORTED, "split form: K must be 4, 8 or 12");
    SplitPlan* sp = new SplitPlan();
    sp->device = device;
    int st = CF_OK;
    switch (folded.k) {
        case 4: st = build_impl<4, 4>(sp, folded, n_g, n_slices); break;
        case 8: {
            // 8 cells per CTA where their f fits beside one six-plane A buffer and the B ring
            int optin = 0;
            cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
            const int L = isqrt_int(folded.n_q) - 1;
            st = smem_layout<8, 8>(folded.n_q, L, 1).total <= optin ? build_impl<8, 8>(sp, folded, n_g, n_slices)
                                                                    : build_impl<8, 4>(sp, folded, n_g, n_slices);
            break;
        }
        default: st = build_impl<12, 4>(sp, folded, n_g, n_slices); break;
    }
    if (st == CF_OK) {
        int optin = 0;
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
        if (sp->smem > optin) {
            char msg[160];
            snprintf(msg, sizeof(msg), "split form: %d bytes of shared memory needed, %d available", sp->smem, optin);
            st = fail_split(CF_EUNSUPPORTED, msg);
        }
    }
    if (st != CF_OK) {
        split_destroy(sp);
        return st;
    }
    *out = sp;
    return CF_OK;
}

void split_destroy(SplitPlan* sp) {
    if (!sp) return;
    void* ptrs[] = {sp->d_rplanes, sp->d_e_gs, sp->d_rb_off, sp->d_rb_gs, sp->d_rb_l23, sp->d_units, sp->d_unit_order, sp->d_band_tl,
                    sp->d_band_rng, sp->d_err, sp->d_rfp64, sp->d_rbf, sp->d_units64, sp->d_unit_order64,
                    sp->d_rbf8, sp->d_rfl, sp->d_rfl32, sp->d_t_l23, sp->d_lb_units, sp->d_lb_order, sp->d_lb_items,
                    sp->d_lb_titems};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete sp;
}

int64_t split_device_bytes(const SplitPlan* sp) { return sp ? sp->bytes : 0; }

int split_check(const SplitPlan* sp) {
    int v = 0;
    if (!sp || cudaMemcpy(&v, sp->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return CF_ECUDA;
    if (v != 0) {
        cudaMemset(sp->d_err, 0, sizeof(int));
        return fail_split(CF_ETIMEOUT, "split form: a bounded wait on the tensor-core pipeline gave up");
    }
    return CF_OK;
}

int split_run(const SplitPlan* sp, double* q_cm, const double* f_cm, int64_t B, cudaStream_t st, int64_t* launches) {
    if (B <= 0 || sp->n_rg == 0) return CF_OK;
    switch (sp->k) {
        case 4: return run_impl<4, 4>(sp, q_cm, f_cm, B, st, launches);
        case 8: return sp->cells == 8 ? run_impl<8, 8>(sp, q_cm, f_cm, B, st, launches)
                                      : run_impl<8, 4>(sp, q_cm, f_cm, B, st, launches);
        default: return run_impl<12, 4>(sp, q_cm, f_cm, B, st, launches);
    }
}

}  // namespace cf
