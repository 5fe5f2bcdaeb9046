// kernels.cuh -- FP64 contraction kernels for sm_100a.
//
// Work decomposition: one warp per (q1, tile of 32 cells[, lane group]).  A warp walks every
// (t, q1) slice of its q1 and every COO entry of those slices; the entry (q2, q3, G) is uniform
// across the warp, each lane handles one cell (or a column block of one cell's Phi when Phi is
// split over P lanes).  Q[q1] is accumulated in registers from the caller's Q and written once,
// so no atomics are needed and the result does not depend on scheduling.
//
// Angular first (src/mex/angular_first_collision_kernel_mex.cpp:45-69):
//   Phi[k2,k3]  = sum_{z in slice} G_z f[q2,k2] f[q3,k3]       K^2 FMA per entry
//   Q[q1,k1]   += sum_{k2,k3} R_t[k1,k2,k3] Phi[k2,k3]          K^3 FMA per slice
// Radial first (src/mex/radial_first_collision_kernel_mex.cpp:41-72):
//   Psi[k1]     = sum_{k3,k2} R_t[k1,k2,k3] f[q2,k2] f[q3,k3]   K^3 FMA per entry
//   Q[q1,k1]   += G_z Psi[k1]
// Jacobian apply (no reference counterpart): the angular-first loop with
//   Phi[k2,k3]  = sum G_z (v[q2,k2] f[q3,k3] + f[q2,k2] v[q3,k3]).
//
// EXACT variants perform the reference's operations in the reference's order with every
// product and sum rounded separately (no FMA), so their output equals the compiled reference
// kernels' bit for bit.  The fast variants hoist G into f3 and use FMA.
#pragma once
#include "common.cuh"

namespace cf {

// ----------------------------------------------------------------------------------------
// Work item decoding shared by the kernels
// ----------------------------------------------------------------------------------------
struct Item {
    int q1, tile, sub;
};

__device__ __forceinline__ bool decode_item(const DevOp& op, int n_tiles, int P, Item& it) {
    const int64_t item = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int64_t per_q1 = (int64_t)n_tiles * P;
    if (item >= (int64_t)op.n_items * per_q1) return false;
    it.q1 = op.item_q1[item / per_q1];
    const int rem = (int)(item % per_q1);
    it.tile = rem / P;
    it.sub = rem % P;
    return true;
}

// ----------------------------------------------------------------------------------------
// Angular first (and its bilinear Jacobian twin when JV = true)
// ----------------------------------------------------------------------------------------
template <int K, int P, bool EXACT, bool JV>
__global__ void __launch_bounds__(128) af_kernel(DevOp op, const double* __restrict__ fT,
                                                 const double* __restrict__ vT,
                                                 double* __restrict__ QT, int n_tiles) {
    constexpr int CPW = CF_TILE / P;       // cells per warp
    constexpr int KC = (K + P - 1) / P;    // k3 columns of Phi held per lane
    static_assert(!EXACT || P == 1, "the exact order needs one lane per cell");

    Item it;
    if (!decode_item(op, n_tiles, P, it)) return;
    const int lane = threadIdx.x & 31;
    const int part = (P == 1) ? 0 : lane / CPW;
    const int cell = it.sub * CPW + (lane % CPW);
    const int k3base = part * KC;
    const size_t tile_off = (size_t)it.tile * op.n_q * K * CF_TILE + cell;
    const double* __restrict__ fb = fT + tile_off;
    const double* __restrict__ vb = JV ? vT + tile_off : nullptr;
    double* qb = QT + tile_off;

    double acc[K];
#pragma unroll
    for (int k1 = 0; k1 < K; ++k1) acc[k1] = (part == 0) ? qb[(size_t)(it.q1 * K + k1) * CF_TILE] : 0.0;

    const int s0 = op.q1_begin[it.q1], s1 = op.q1_begin[it.q1 + 1];
    for (int s = s0; s < s1; ++s) {
        const int t = op.slice_t[s];
        const int e0 = op.slice_e[s], e1 = op.slice_e[s + 1];
        double phi[K][KC];
#pragma unroll
        for (int a = 0; a < K; ++a)
#pragma unroll
            for (int c = 0; c < KC; ++c) phi[a][c] = 0.0;

        for (int eb = e0; eb < e1; eb += 32) {
            const int n = min(32, e1 - eb);
            uint32_t my_q23 = 0;
            double my_g = 0.0;
            if (lane < n) {
                my_q23 = __ldg(op.e_q23 + eb + lane);
                my_g = __ldg(op.e_g + eb + lane);
            }
            for (int j = 0; j < n; ++j) {
                const uint32_t q23 = __shfl_sync(0xffffffffu, my_q23, j);
                const double g = __shfl_sync(0xffffffffu, my_g, j);
                const double* __restrict__ f2p = fb + (size_t)(q23 & 0xffffu) * K * CF_TILE;
                const double* __restrict__ f3p = fb + (size_t)(q23 >> 16) * K * CF_TILE;
                double f2[K], f3[KC];
#pragma unroll
                for (int k = 0; k < K; ++k) f2[k] = __ldg(f2p + k * CF_TILE);
#pragma unroll
                for (int c = 0; c < KC; ++c)
                    f3[c] = (k3base + c < K) ? __ldg(f3p + (k3base + c) * CF_TILE) : 0.0;
                if constexpr (JV) {
                    const double* __restrict__ v2p = vb + (size_t)(q23 & 0xffffu) * K * CF_TILE;
                    const double* __restrict__ v3p = vb + (size_t)(q23 >> 16) * K * CF_TILE;
                    double v2[K], v3[KC];
#pragma unroll
                    for (int k = 0; k < K; ++k) v2[k] = __ldg(v2p + k * CF_TILE);
#pragma unroll
                    for (int c = 0; c < KC; ++c)
                        v3[c] = (k3base + c < K) ? __ldg(v3p + (k3base + c) * CF_TILE) : 0.0;
                    if constexpr (EXACT) {
                        // phi += g * (v2 f3 + f2 v3), each operation rounded (oracle orc_jv order)
#pragma unroll
                        for (int c = 0; c < KC; ++c)
#pragma unroll
                            for (int k2 = 0; k2 < K; ++k2)
                                phi[k2][c] = __dadd_rn(
                                    phi[k2][c],
                                    __dmul_rn(g, __dadd_rn(__dmul_rn(v2[k2], f3[c]), __dmul_rn(f2[k2], v3[c]))));
                    } else {
#pragma unroll
                        for (int c = 0; c < KC; ++c) {
                            const double gf3 = g * f3[c], gv3 = g * v3[c];
#pragma unroll
                            for (int k2 = 0; k2 < K; ++k2) phi[k2][c] = fma(v2[k2], gf3, fma(f2[k2], gv3, phi[k2][c]));
                        }
                    }
                } else {
                    if constexpr (EXACT) {
                        // Phi[k2,k3] += (g * f2[k2]) * f3[k3]   (reference :55, no FMA)
                        double gf2[K];
#pragma unroll
                        for (int k2 = 0; k2 < K; ++k2) gf2[k2] = __dmul_rn(g, f2[k2]);
#pragma unroll
                        for (int c = 0; c < KC; ++c)
#pragma unroll
                            for (int k2 = 0; k2 < K; ++k2)
                                phi[k2][c] = __dadd_rn(phi[k2][c], __dmul_rn(gf2[k2], f3[c]));
                    } else {
#pragma unroll
                        for (int c = 0; c < KC; ++c) {
                            const double gf3 = g * f3[c];
#pragma unroll
                            for (int k2 = 0; k2 < K; ++k2) phi[k2][c] = fma(f2[k2], gf3, phi[k2][c]);
                        }
                    }
                }
            }
        }

        // K^3 step: acc[k1] += sum_{k3 (outer), k2 (inner)} R_t[k1,k2,k3] Phi[k2,k3]
        const double* __restrict__ Rt = op.R + (size_t)t * K * K * K;
#pragma unroll
        for (int k1 = 0; k1 < K; ++k1) {
            double sacc = 0.0;
#pragma unroll
            for (int c = 0; c < KC; ++c) {
                const int k3 = k3base + c;
                if (P == 1 || k3 < K) {
#pragma unroll
                    for (int k2 = 0; k2 < K; ++k2) {
                        const double r = __ldg(Rt + k1 + K * k2 + K * K * k3);
                        if constexpr (EXACT)
                            sacc = __dadd_rn(sacc, __dmul_rn(r, phi[k2][c]));
                        else
                            sacc = fma(r, phi[k2][c], sacc);
                    }
                }
            }
            acc[k1] = EXACT ? __dadd_rn(acc[k1], sacc) : acc[k1] + sacc;
        }
    }

    if constexpr (P > 1) {
#pragma unroll
        for (int k1 = 0; k1 < K; ++k1)
#pragma unroll
            for (int off = CPW; off < 32; off <<= 1) acc[k1] += __shfl_xor_sync(0xffffffffu, acc[k1], off);
    }
    if (part == 0) {
#pragma unroll
        for (int k1 = 0; k1 < K; ++k1) qb[(size_t)(it.q1 * K + k1) * CF_TILE] = acc[k1];
    }
}

// ----------------------------------------------------------------------------------------
// Radial first
// ----------------------------------------------------------------------------------------
template <int K, bool EXACT>
__global__ void __launch_bounds__(128) rf_kernel(DevOp op, const double* __restrict__ fT,
                                                 double* __restrict__ QT, int n_tiles) {
    Item it;
    if (!decode_item(op, n_tiles, 1, it)) return;
    const int lane = threadIdx.x & 31;
    const size_t tile_off = (size_t)it.tile * op.n_q * K * CF_TILE + lane;
    const double* __restrict__ fb = fT + tile_off;
    double* qb = QT + tile_off;

    double acc[K];
#pragma unroll
    for (int k1 = 0; k1 < K; ++k1) acc[k1] = qb[(size_t)(it.q1 * K + k1) * CF_TILE];

    const int s0 = op.q1_begin[it.q1], s1 = op.q1_begin[it.q1 + 1];
    for (int s = s0; s < s1; ++s) {
        const int t = op.slice_t[s];
        const double* __restrict__ Rt = op.R + (size_t)t * K * K * K;
        const int e0 = op.slice_e[s], e1 = op.slice_e[s + 1];
        for (int eb = e0; eb < e1; eb += 32) {
            const int n = min(32, e1 - eb);
            uint32_t my_q23 = 0;
            double my_g = 0.0;
            if (lane < n) {
                my_q23 = __ldg(op.e_q23 + eb + lane);
                my_g = __ldg(op.e_g + eb + lane);
            }
            for (int j = 0; j < n; ++j) {
                const uint32_t q23 = __shfl_sync(0xffffffffu, my_q23, j);
                const double g = __shfl_sync(0xffffffffu, my_g, j);
                const double* __restrict__ f2p = fb + (size_t)(q23 & 0xffffu) * K * CF_TILE;
                const double* __restrict__ f3p = fb + (size_t)(q23 >> 16) * K * CF_TILE;
                double f2[K], psi[K];
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    f2[k] = __ldg(f2p + k * CF_TILE);
                    psi[k] = 0.0;
                }
                // every psi[k1] accumulates over k3 (outer) then k2 (inner), the reference's order
#pragma unroll 1
                for (int k3 = 0; k3 < K; ++k3) {
                    const double f3 = __ldg(f3p + k3 * CF_TILE);
                    const double* __restrict__ Rk3 = Rt + K * K * k3;
#pragma unroll
                    for (int k1 = 0; k1 < K; ++k1) {
                        if constexpr (EXACT) {
#pragma unroll
                            for (int k2 = 0; k2 < K; ++k2)
                                psi[k1] = __dadd_rn(psi[k1], __dmul_rn(__dmul_rn(__ldg(Rk3 + k1 + K * k2), f2[k2]), f3));
                        } else {
                            double inner = 0.0;
#pragma unroll
                            for (int k2 = 0; k2 < K; ++k2) inner = fma(__ldg(Rk3 + k1 + K * k2), f2[k2], inner);
                            psi[k1] = fma(inner, f3, psi[k1]);
                        }
                    }
                }
#pragma unroll
                for (int k1 = 0; k1 < K; ++k1)
                    acc[k1] = EXACT ? __dadd_rn(acc[k1], __dmul_rn(g, psi[k1])) : fma(g, psi[k1], acc[k1]);
            }
        }
    }
#pragma unroll
    for (int k1 = 0; k1 < K; ++k1) qb[(size_t)(it.q1 * K + k1) * CF_TILE] = acc[k1];
}

}  // namespace cf
