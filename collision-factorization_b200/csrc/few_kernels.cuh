// few_kernels.cuh -- the contraction of a handful of cells (one f per call, as the reference's MEX
// is called) in one launch.
//
// A 32-cell tile with one live cell leaves the batch kernels one warp or one CTA walking every slice
// of a row in turn, each slice a chain of dependent loads (slice bounds, entries, R_t).  Here the
// work is spread the other way: one CTA per (q1 row, cell), its warps taking the row's slices in
// turn, and the lanes of a warp taking the K x K (k2, k3) pairs of the slice's Phi.  A warp reads
// the bounds of all its slices in one step and R_t before the entries (K <= 8), so a call is three
// dependent loads deep: the row's slice range (beside f and Q), the slice bounds, the entries.
//
// Angular first (src/mex/angular_first_collision_kernel_mex.cpp:45-69), per slice (t, q1):
//   Phi[k2,k3] = sum_{z in slice} G_z f[q2,k2] f[q3,k3]        a lane's own pairs only
//   acc[k1]   += sum_{own pairs} R_t[k1,k2,k3] Phi[k2,k3]      per lane, over all its slices
// Radial first (src/mex/radial_first_collision_kernel_mex.cpp:41-72), per entry:
//   acc[k1]   += G_z sum_{own pairs} R_t[k1,k2,k3] f[q2,k2] f[q3,k3]
// The lane sums are reduced over the warp (butterfly) and the warps' sums over the CTA in a fixed
// order, then added to Q[q1, :], so the result does not depend on scheduling.
//
// Two entry kernels share the body.  af_few_kernel updates Q in place in the caller's cell-major
// device arrays.  af_few_param_kernel serves the host entry points: f and Q_in of the cells travel
// inside the launch's parameter block (at most kFewPayloadMax doubles), so nothing is copied or read
// over the host link before the contraction, and Q_out is written to mapped pinned host memory
// (every row, those without slices as they came in).
#pragma once
#include "common.cuh"

namespace cf {

constexpr int kFewWarps = 16;
constexpr int kFewPayloadMax = 3968;  // doubles: with DevOp, the largest block under the 32,764-byte limit

template <int CAP>
struct FewPayload {
    double v[CAP];  // f of the cells, then Q_in of the cells, each [cell][K][N_Q]
};

template <int K>
__host__ __device__ constexpr int few_pairs_per_lane() { return (K * K + 31) / 32; }

// One (q1 row, cell): q_out[k1 * N_Q + q1] = q_in[k1 * N_Q + q1] + (row q1 of the contraction of f).
// With pass_through, a row without slices is still written (q_out is not q_in).
template <int K, bool RF>
__device__ __forceinline__ void few_row(const DevOp& op, const double* f, const double* q_in, double* q_out,
                                        bool pass_through) {
    constexpr int NP = few_pairs_per_lane<K>();
    constexpr bool R_AHEAD = K <= 8;  // R_t held in registers from the start of the slice
    static_assert(!RF || R_AHEAD, "the radial-first form is built for K <= 8");
    extern __shared__ double fs[];  // this cell's f, [K][N_Q] as in the cell-major array
    __shared__ double red[kFewWarps][K];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n_q = op.n_q, M = n_q * K;
    const int q1 = blockIdx.x;
    const int s0 = op.q1_begin[q1], s1 = op.q1_begin[q1 + 1];
    // this row of Q is read up front, beside f
    double qv = 0.0;
    if (threadIdx.x < K) qv = q_in[threadIdx.x * n_q + q1];
    if (s0 == s1) {  // no slice: the row is unchanged (the whole CTA leaves together)
        if (pass_through && threadIdx.x < K) q_out[threadIdx.x * n_q + q1] = qv;
        return;
    }
    for (int i = threadIdx.x; i < M; i += blockDim.x) fs[i] = f[i];

    // bounds of this warp's slices s0 + warp + kFewWarps i, lane i holding the i-th (32 at a time)
    const int n_mine = s1 - s0 > warp ? (s1 - s0 - warp + kFewWarps - 1) / kFewWarps : 0;

    // the lane's (k2, k3) pairs: p = lane + 32 j, k2 = p mod K, k3 = p / K
    int k2o[NP], k3o[NP];
    bool live[NP];
#pragma unroll
    for (int j = 0; j < NP; ++j) {
        const int p = lane + 32 * j;
        live[j] = p < K * K;
        k2o[j] = live[j] ? p % K : 0;
        k3o[j] = live[j] ? p / K : 0;
    }
    double acc[K];
#pragma unroll
    for (int k1 = 0; k1 < K; ++k1) acc[k1] = 0.0;
    __syncthreads();

    for (int base = 0; base < n_mine; base += 32) {
        int my_t = 0, my_e0 = 0, my_e1 = 0;
        if (base + lane < n_mine) {
            const int s = s0 + warp + kFewWarps * (base + lane);
            my_t = __ldg(op.slice_t + s);
            my_e0 = __ldg(op.slice_e + s);
            my_e1 = __ldg(op.slice_e + s + 1);
        }
        const int n_here = min(32, n_mine - base);
        for (int i = 0; i < n_here; ++i) {
            const int t = __shfl_sync(0xffffffffu, my_t, i);
            const int e0 = __shfl_sync(0xffffffffu, my_e0, i);
            const int e1 = __shfl_sync(0xffffffffu, my_e1, i);
            const double* __restrict__ Rt = op.R + (size_t)t * K * K * K;
            double r[R_AHEAD ? K : 1][NP];
            if constexpr (R_AHEAD) {
#pragma unroll
                for (int k1 = 0; k1 < K; ++k1)
#pragma unroll
                    for (int j = 0; j < NP; ++j) r[k1][j] = live[j] ? __ldg(Rt + k1 + K * (lane + 32 * j)) : 0.0;
            }
            double phi[NP];
#pragma unroll
            for (int j = 0; j < NP; ++j) phi[j] = 0.0;
            for (int eb = e0; eb < e1; eb += 32) {
                const int n = min(32, e1 - eb);
                uint32_t my_q23 = 0;
                double my_g = 0.0;
                if (lane < n) {
                    my_q23 = __ldg(op.e_q23 + eb + lane);
                    my_g = __ldg(op.e_g + eb + lane);
                }
                for (int z = 0; z < n; ++z) {
                    const uint32_t q23 = __shfl_sync(0xffffffffu, my_q23, z);
                    const double g = __shfl_sync(0xffffffffu, my_g, z);
                    const double* f2 = fs + (q23 & 0xffffu);
                    const double* f3 = fs + (q23 >> 16);
                    if constexpr (RF) {
                        double psi[K];
#pragma unroll
                        for (int k1 = 0; k1 < K; ++k1) psi[k1] = 0.0;
#pragma unroll
                        for (int j = 0; j < NP; ++j) {
                            const double w = f2[k2o[j] * n_q] * f3[k3o[j] * n_q];
#pragma unroll
                            for (int k1 = 0; k1 < K; ++k1) psi[k1] = fma(r[k1][j], w, psi[k1]);
                        }
#pragma unroll
                        for (int k1 = 0; k1 < K; ++k1) acc[k1] = fma(g, psi[k1], acc[k1]);
                    } else {
#pragma unroll
                        for (int j = 0; j < NP; ++j) phi[j] = fma(f2[k2o[j] * n_q], g * f3[k3o[j] * n_q], phi[j]);
                    }
                }
            }
            if constexpr (!RF) {
#pragma unroll
                for (int k1 = 0; k1 < K; ++k1)
#pragma unroll
                    for (int j = 0; j < NP; ++j) {
                        if constexpr (R_AHEAD)
                            acc[k1] = fma(r[k1][j], phi[j], acc[k1]);
                        else if (live[j])
                            acc[k1] = fma(__ldg(Rt + k1 + K * (lane + 32 * j)), phi[j], acc[k1]);
                    }
            }
        }
    }

#pragma unroll
    for (int k1 = 0; k1 < K; ++k1) {
        double v = acc[k1];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0) red[warp][k1] = v;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        const int k1 = threadIdx.x;
        double sum = 0.0;
#pragma unroll
        for (int w = 0; w < kFewWarps; ++w) sum += red[w][k1];
        q_out[k1 * n_q + q1] = qv + sum;
    }
}

// The exact form of one (q1 row, cell), in the reference's operation order
// (src/mex/angular_first_collision_kernel_mex.cpp:45-69).  Each warp takes one slice of the row at a
// time (16 at once): lane p owns Phi[k2][k3] (p = k2 + K k3) and sums (G f[q2,k2]) f[q3,k3] over the
// slice's entries in order, each product and sum rounded separately; lane k1 then sums
// R_t[k1,k2,k3] Phi[k2][k3] over k3 (outer) and k2 (inner) into the slice's row sum.  Thread k1 of
// the CTA adds the row sums to Q[q1,k1] in slice order, so the result is the reference's bit for
// bit.  Shared memory: f of the cell, each warp's Phi, each warp's row sum.
template <int K>
__device__ __forceinline__ void few_row_exact(const DevOp& op, const double* f, const double* q_in, double* q_out,
                                              bool pass_through) {
    constexpr int NP = few_pairs_per_lane<K>();
    extern __shared__ double fs[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n_q = op.n_q, M = n_q * K;
    double* phis = fs + M + warp * K * K;
    double* sums = fs + M + kFewWarps * K * K;  // [kFewWarps][K]
    const int q1 = blockIdx.x;
    const int s0 = op.q1_begin[q1], s1 = op.q1_begin[q1 + 1];
    double acc = 0.0;
    if (threadIdx.x < K) acc = q_in[threadIdx.x * n_q + q1];
    if (s0 == s1) {
        if (pass_through && threadIdx.x < K) q_out[threadIdx.x * n_q + q1] = acc;
        return;
    }
    for (int i = threadIdx.x; i < M; i += blockDim.x) fs[i] = f[i];
    __syncthreads();
    for (int base = s0; base < s1; base += kFewWarps) {
        const int s = base + warp;
        if (s < s1) {
            const int t = op.slice_t[s];
            const int e0 = op.slice_e[s], e1 = op.slice_e[s + 1];
            double phi[NP];
#pragma unroll
            for (int j = 0; j < NP; ++j) phi[j] = 0.0;
            for (int eb = e0; eb < e1; eb += 32) {
                const int n = min(32, e1 - eb);
                uint32_t my_q23 = 0;
                double my_g = 0.0;
                if (lane < n) {
                    my_q23 = __ldg(op.e_q23 + eb + lane);
                    my_g = __ldg(op.e_g + eb + lane);
                }
                for (int z = 0; z < n; ++z) {
                    const uint32_t q23 = __shfl_sync(0xffffffffu, my_q23, z);
                    const double g = __shfl_sync(0xffffffffu, my_g, z);
                    const double* f2 = fs + (q23 & 0xffffu);
                    const double* f3 = fs + (q23 >> 16);
#pragma unroll
                    for (int j = 0; j < NP; ++j) {
                        const int p = lane + 32 * j;
                        if (p < K * K)
                            phi[j] = __dadd_rn(phi[j], __dmul_rn(__dmul_rn(g, f2[(p % K) * n_q]), f3[(p / K) * n_q]));
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < NP; ++j)
                if (lane + 32 * j < K * K) phis[lane + 32 * j] = phi[j];
            __syncwarp();
            if (lane < K) {
                const double* __restrict__ Rt = op.R + (size_t)t * K * K * K;
                double sacc = 0.0;
                for (int k3 = 0; k3 < K; ++k3)
#pragma unroll
                    for (int k2 = 0; k2 < K; ++k2)
                        sacc = __dadd_rn(sacc, __dmul_rn(__ldg(Rt + lane + K * k2 + K * K * k3), phis[k2 + K * k3]));
                sums[warp * K + lane] = sacc;
            }
        }
        __syncthreads();
        if (threadIdx.x < K) {
            const int n = min(kFewWarps, s1 - base);
            for (int w = 0; w < n; ++w) acc = __dadd_rn(acc, sums[w * K + threadIdx.x]);
        }
        __syncthreads();
    }
    if (threadIdx.x < K) q_out[threadIdx.x * n_q + q1] = acc;
}

// The exact form in place on the caller's cell-major device arrays; grid (N_Q, cells).
template <int K>
__global__ void __launch_bounds__(kFewWarps * 32) af_few_exact_kernel(DevOp op, const double* __restrict__ f, double* q) {
    const size_t off = (size_t)blockIdx.y * op.n_q * K;
    few_row_exact<K>(op, f + off, q + off, q + off, false);
}

// The exact form of one (q1 row, pair of cells) in place, for the batch route above K = 8: each cell's
// operations are those of few_row_exact, in the same order, so the bits are the same; the pair shares
// the entry shuffles and the R_t loads, and lanes c 16 + k1 (k1 < K) run the K^3 sums of cell c, where
// one cell leaves 20 of 32 lanes idle.  JV: the exact J(f) v instead, Phi summing
// G ((v[q2,k2] f[q3,k3]) + (f[q2,k2] v[q3,k3])) with each product and sum rounded separately (the
// order of the exact J.v of the batch kernels).  nc (1 or 2) cells from f (and v) and q; shared
// memory: f (and v) of both cells (zero for a missing second cell), each warp's two Phi, each warp's
// two row sums.
template <int K, bool JV>
__device__ __forceinline__ void few_row_exact2(const DevOp& op, const double* __restrict__ f,
                                               const double* __restrict__ v, double* q, int nc) {
    static_assert(K <= 16, "a cell's K^3 sums take lanes c 16 .. c 16 + K - 1");
    constexpr int NP = few_pairs_per_lane<K>();
    constexpr int NA = JV ? 2 : 1;  // staged arrays per cell: f (and v)
    extern __shared__ double fs[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n_q = op.n_q, M = n_q * K;
    const double* vs = fs + 2 * M;                      // JV: v of both cells
    double* phis = fs + NA * 2 * M + warp * 2 * K * K;  // [2][K K]
    double* sums = fs + NA * 2 * M + kFewWarps * 2 * K * K;  // [kFewWarps][2][K]
    const int q1 = blockIdx.x;
    const int s0 = op.q1_begin[q1], s1 = op.q1_begin[q1 + 1];
    if (s0 == s1) return;  // in place: the row has no slices
    // thread c 16 + k (c < nc, k < K) carries Q[q1, k] of cell c
    const int my_c = threadIdx.x >> 4, my_k = threadIdx.x & 15;
    const bool q_thread = threadIdx.x < 32 && my_k < K && my_c < nc;
    double acc = 0.0;
    if (q_thread) acc = q[(size_t)my_c * M + (size_t)my_k * n_q + q1];
    for (int i = threadIdx.x; i < 2 * M; i += blockDim.x) fs[i] = i < nc * M ? f[i] : 0.0;
    if constexpr (JV)
        for (int i = threadIdx.x; i < 2 * M; i += blockDim.x) fs[2 * M + i] = i < nc * M ? v[i] : 0.0;
    __syncthreads();
    for (int base = s0; base < s1; base += kFewWarps) {
        const int s = base + warp;
        if (s < s1) {
            const int t = op.slice_t[s];
            const int e0 = op.slice_e[s], e1 = op.slice_e[s + 1];
            double phi[2][NP];
#pragma unroll
            for (int j = 0; j < NP; ++j) phi[0][j] = phi[1][j] = 0.0;
            for (int eb = e0; eb < e1; eb += 32) {
                const int n = min(32, e1 - eb);
                uint32_t my_q23 = 0;
                double my_g = 0.0;
                if (lane < n) {
                    my_q23 = __ldg(op.e_q23 + eb + lane);
                    my_g = __ldg(op.e_g + eb + lane);
                }
                for (int z = 0; z < n; ++z) {
                    const uint32_t q23 = __shfl_sync(0xffffffffu, my_q23, z);
                    const double g = __shfl_sync(0xffffffffu, my_g, z);
                    const double* f2 = fs + (q23 & 0xffffu);
                    const double* f3 = fs + (q23 >> 16);
                    if constexpr (JV) {
                        const double* v2 = vs + (q23 & 0xffffu);
                        const double* v3 = vs + (q23 >> 16);
#pragma unroll
                        for (int j = 0; j < NP; ++j) {
                            const int p = lane + 32 * j;
                            if (p < K * K) {
                                const int i2 = (p % K) * n_q, i3 = (p / K) * n_q;
#pragma unroll
                                for (int c = 0; c < 2; ++c) {
                                    const int o2 = c * M + i2, o3 = c * M + i3;
                                    phi[c][j] = __dadd_rn(phi[c][j], __dmul_rn(g, __dadd_rn(__dmul_rn(v2[o2], f3[o3]),
                                                                                            __dmul_rn(f2[o2], v3[o3]))));
                                }
                            }
                        }
                    } else {
#pragma unroll
                        for (int j = 0; j < NP; ++j) {
                            const int p = lane + 32 * j;
                            if (p < K * K) {
                                const int i2 = (p % K) * n_q, i3 = (p / K) * n_q;
                                phi[0][j] = __dadd_rn(phi[0][j], __dmul_rn(__dmul_rn(g, f2[i2]), f3[i3]));
                                phi[1][j] = __dadd_rn(phi[1][j], __dmul_rn(__dmul_rn(g, f2[M + i2]), f3[M + i3]));
                            }
                        }
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < NP; ++j)
                if (lane + 32 * j < K * K) {
                    phis[lane + 32 * j] = phi[0][j];
                    phis[K * K + lane + 32 * j] = phi[1][j];
                }
            __syncwarp();
            const int c = lane >> 4, k1 = lane & 15;
            if (k1 < K) {
                const double* __restrict__ Rt = op.R + (size_t)t * K * K * K;
                const double* ph = phis + c * K * K;
                double sacc = 0.0;
                for (int k3 = 0; k3 < K; ++k3)
#pragma unroll
                    for (int k2 = 0; k2 < K; ++k2)
                        sacc = __dadd_rn(sacc, __dmul_rn(__ldg(Rt + k1 + K * k2 + K * K * k3), ph[k2 + K * k3]));
                sums[(warp * 2 + c) * K + k1] = sacc;
            }
        }
        __syncthreads();
        if (q_thread) {
            const int n = min(kFewWarps, s1 - base);
            for (int w = 0; w < n; ++w) acc = __dadd_rn(acc, sums[(w * 2 + my_c) * K + my_k]);
        }
        __syncthreads();
    }
    if (q_thread) q[(size_t)my_c * M + (size_t)my_k * n_q + q1] = acc;
}

// The exact form (JV: the exact J(f) v, v non-null) in place on the caller's cell-major device arrays,
// two cells per CTA; grid (N_Q, ceil(cells / 2)).  The Q form's shared memory leaves room for two
// CTAs per SM at L = 16, K = 12 (95 KB each), so up to K = 13 its registers are held to what two CTAs
// of 16 warps allow (64 a thread; with 76 only one CTA fitted and the launch took 95.7 ms instead of
// 70.0).  Above K = 13 (Phi and f of two cells take about twice the memory) and for the J.v form
// (f and v: 151 KB at L = 16, K = 12) one CTA per SM is what shared memory leaves anyway.
template <int K, bool JV>
__global__ void __launch_bounds__(kFewWarps * 32, (JV || K > 13) ? 1 : 2) af_few_exact2_kernel(DevOp op, const double* __restrict__ f,
                                                                        const double* __restrict__ v, double* q,
                                                                        long long n_cells) {
    const long long c0 = 2LL * blockIdx.y;
    const int nc = (int)(n_cells - c0 < 2 ? n_cells - c0 : 2);
    const size_t off = (size_t)c0 * op.n_q * K;
    few_row_exact2<K, JV>(op, f + off, JV ? v + off : nullptr, q + off, nc);
}

// The exact form with f and Q_in in the parameter block, Q_out to q_out; grid (N_Q, n_cells).
template <int K, int CAP>
__global__ void __launch_bounds__(kFewWarps * 32) af_few_exact_param_kernel(DevOp op, const __grid_constant__ FewPayload<CAP> pay,
                                                                int n_cells, double* q_out) {
    const size_t M = (size_t)op.n_q * K, off = (size_t)blockIdx.y * M;
    few_row_exact<K>(op, pay.v + off, pay.v + (size_t)n_cells * M + off, q_out + off, true);
}

// Q += contraction of f, in the caller's cell-major device arrays; grid (N_Q, cells).
template <int K, bool RF>
__global__ void __launch_bounds__(kFewWarps * 32) af_few_kernel(DevOp op, const double* __restrict__ f,
                                                                 double* q) {
    const size_t off = (size_t)blockIdx.y * op.n_q * K;
    few_row<K, RF>(op, f + off, q + off, q + off, false);
}

// q_out = Q_in + contraction of f, f and Q_in in the parameter block; grid (N_Q, n_cells).
template <int K, bool RF, int CAP>
__global__ void __launch_bounds__(kFewWarps * 32) af_few_param_kernel(DevOp op, const __grid_constant__ FewPayload<CAP> pay,
                                                                       int n_cells, double* q_out) {
    const size_t M = (size_t)op.n_q * K, off = (size_t)blockIdx.y * M;
    few_row<K, RF>(op, pay.v + off, pay.v + (size_t)n_cells * M + off, q_out + off, true);
}

}  // namespace cf
