// pair_kernels.cuh -- tile-resident angular-first kernels over pairs of mirrored output rows.
//
// In the real spherical-harmonic basis the rows q1 = (l1, +m1) and (l1, -m1) have identical slice
// structure: the same l-triplets t in the same order with the same number of COO entries per slice
// (the cos/sin parity of the real Gaunt coefficients maps one row's entries onto the other's).
// plan.cu verifies this per operator and pairs only rows whose structure matches.
//
// A warp owns one pair for the 16 cells of the CTA's resident half-tile: lanes 0-15 contract row
// qa, lanes 16-31 contract row qb, one cell per lane, each lane holding the whole K x K Phi of its
// cell.  Both halves are at the same slice, hence the same t, so the K^3 step reads R_t with
// warp-uniform shared loads, and each f row read by a half-warp is one 128-byte wavefront.  Rows
// without a mirror (m1 = 0, or a structure mismatch) run with the upper half idle.
//
// The rest follows tile_kernels.cuh: 16-cell half-tile resident in shared memory, R_t staged per
// warp with cp.async, persistent CTAs pulling whole half-tiles and then binned half-tiles from a
// device counter, warps pulling pair items from a shared counter.
#pragma once
#include "common.cuh"
#include "tile_kernels.cuh"

namespace cf {

struct PairSched {
    const int* bin_begin;  // bins over pair items: 0 = all (heaviest first), 1..4, 5..20
    const int* bin_item;   // item indices
    const int2* items;     // (qa, qb); qb = -1 for a row without a mirror
    int n_ht, n_whole, split, n_units;
    int* counter;
};

template <int K>
struct RPair {
    static constexpr int SIZE = K * K * K + (K % 2);  // keep each warp's buffer 16-byte aligned
};

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}

// RG = false: R_t is staged into the warp's shared buffer with cp.async.  RG = true: R_t is read
// straight from global memory with warp-uniform loads through L1 (prefetched into L1 at the start
// of the slice), which keeps the K^3 step off the shared-memory wavefront budget.
template <int K, bool EXACT, bool JV, bool RG>
__device__ __forceinline__ void pair_item(const DevOp& op, int2 item, const double* __restrict__ fs,
                                          const double* __restrict__ vs, double* rb, double* qtc, int lane) {
    const int half = lane >> 4;
    const int c = lane & 15;
    const bool active = half == 0 || item.y >= 0;
    const int q1 = half == 0 ? item.x : (item.y >= 0 ? item.y : item.x);

    double acc[K];
#pragma unroll
    for (int k1 = 0; k1 < K; ++k1) acc[k1] = active ? qtc[(size_t)(q1 * K + k1) * CF_TILE] : 0.0;

    // slices of qa and qb correspond one to one (same t, same length)
    const int sa0 = op.q1_begin[item.x], sa1 = op.q1_begin[item.x + 1];
    const int sb0 = item.y >= 0 ? op.q1_begin[item.y] : sa0;
    for (int i = 0; i < sa1 - sa0; ++i) {
        const int sa = sa0 + i, sb = sb0 + i;
        const int t = op.slice_t[sa];
        const int ea = op.slice_e[sa], n_e = op.slice_e[sa + 1] - ea;
        const int eb_ = op.slice_e[sb];
        const int my_e0 = half == 0 ? ea : eb_;

        const double* __restrict__ Rt = op.R + (size_t)t * K * K * K;
        if constexpr (RG) {
            const char* rbytes = reinterpret_cast<const char*>(Rt);
            for (int off = lane * 128; off < K * K * K * 8; off += 32 * 128)
                asm volatile("prefetch.global.L1 [%0];\n" ::"l"(rbytes + off));
        } else {
            __syncwarp();
            if constexpr (K % 2 == 0) {
                for (int j = lane; j < K * K * K / 2; j += 32) cp_async16(rb + 2 * j, Rt + 2 * j);
            } else {
                for (int j = lane; j < K * K * K; j += 32) cp_async8(rb + j, Rt + j);
            }
            cp_async_commit();
        }

        double phi[K][K];
#pragma unroll
        for (int a = 0; a < K; ++a)
#pragma unroll
            for (int b = 0; b < K; ++b) phi[a][b] = 0.0;

        for (int e0 = 0; e0 < n_e; e0 += 16) {
            const int n = min(16, n_e - e0);
            uint32_t my_q23 = 0;
            double my_g = 0.0;
            if (c < n && active) {
                my_q23 = __ldg(op.e_q23 + my_e0 + e0 + c);
                my_g = __ldg(op.e_g + my_e0 + e0 + c);
            }
            for (int j = 0; j < n; ++j) {
                const uint32_t q23 = __shfl_sync(0xffffffffu, my_q23, j + 16 * half);
                const double g = __shfl_sync(0xffffffffu, my_g, j + 16 * half);
                const int r2 = (int)(q23 & 0xffffu) * K, r3 = (int)(q23 >> 16) * K;
                double f2[K], f3[K];
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    f2[k] = fs[(r2 + k) * kTileCells + c];
                    f3[k] = fs[(r3 + k) * kTileCells + c];
                }
                if constexpr (JV) {
                    double v2[K], v3[K];
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        v2[k] = vs[(r2 + k) * kTileCells + c];
                        v3[k] = vs[(r3 + k) * kTileCells + c];
                    }
                    if constexpr (EXACT) {
#pragma unroll
                        for (int b = 0; b < K; ++b)
#pragma unroll
                            for (int a = 0; a < K; ++a)
                                phi[a][b] = __dadd_rn(
                                    phi[a][b], __dmul_rn(g, __dadd_rn(__dmul_rn(v2[a], f3[b]), __dmul_rn(f2[a], v3[b]))));
                    } else {
#pragma unroll
                        for (int b = 0; b < K; ++b) {
                            const double gf3 = g * f3[b], gv3 = g * v3[b];
#pragma unroll
                            for (int a = 0; a < K; ++a) phi[a][b] = fma(v2[a], gf3, fma(f2[a], gv3, phi[a][b]));
                        }
                    }
                } else if constexpr (EXACT) {
                    // Phi[k2,k3] += (g * f2[k2]) * f3[k3], reference operation order
                    double gf2[K];
#pragma unroll
                    for (int a = 0; a < K; ++a) gf2[a] = __dmul_rn(g, f2[a]);
#pragma unroll
                    for (int b = 0; b < K; ++b)
#pragma unroll
                        for (int a = 0; a < K; ++a) phi[a][b] = __dadd_rn(phi[a][b], __dmul_rn(gf2[a], f3[b]));
                } else {
#pragma unroll
                    for (int b = 0; b < K; ++b) {
                        const double gf3 = g * f3[b];
#pragma unroll
                        for (int a = 0; a < K; ++a) phi[a][b] = fma(f2[a], gf3, phi[a][b]);
                    }
                }
            }
        }
        if constexpr (!RG) {
            cp_async_wait_all();
            __syncwarp();
        }
        const double* __restrict__ rsrc = RG ? Rt : rb;

        // K^3 step: R_t element (k1,k2,k3) at rsrc[k1 + K k2 + K^2 k3]; the address is warp-uniform
        if constexpr (EXACT) {
#pragma unroll
            for (int k1 = 0; k1 < K; ++k1) {
                double sacc = 0.0;
#pragma unroll
                for (int b = 0; b < K; ++b)
#pragma unroll
                    for (int a = 0; a < K; ++a) {
                        const double r = RG ? __ldg(rsrc + k1 + K * a + K * K * b) : rsrc[k1 + K * a + K * K * b];
                        sacc = __dadd_rn(sacc, __dmul_rn(r, phi[a][b]));
                    }
                acc[k1] = __dadd_rn(acc[k1], sacc);
            }
        } else if constexpr (K % 2 == 0) {
#pragma unroll
            for (int b = 0; b < K; ++b)
#pragma unroll
                for (int a = 0; a < K; ++a) {
                    const double2* r2v = reinterpret_cast<const double2*>(rsrc + K * a + K * K * b);
#pragma unroll
                    for (int h = 0; h < K / 2; ++h) {
                        const double2 r = RG ? __ldg(r2v + h) : r2v[h];
                        acc[2 * h] = fma(r.x, phi[a][b], acc[2 * h]);
                        acc[2 * h + 1] = fma(r.y, phi[a][b], acc[2 * h + 1]);
                    }
                }
        } else {
#pragma unroll
            for (int b = 0; b < K; ++b)
#pragma unroll
                for (int a = 0; a < K; ++a)
#pragma unroll
                    for (int k1 = 0; k1 < K; ++k1) {
                        const double r = RG ? __ldg(rsrc + k1 + K * a + K * K * b) : rsrc[k1 + K * a + K * K * b];
                        acc[k1] = fma(r, phi[a][b], acc[k1]);
                    }
        }
    }
    if (active) {
#pragma unroll
        for (int k1 = 0; k1 < K; ++k1) qtc[(size_t)(q1 * K + k1) * CF_TILE] = acc[k1];
    }
}

template <int K, int W, bool EXACT, bool JV, bool RG>
__global__ void __launch_bounds__(W * 32, 1)
    af_pair_kernel(DevOp op, PairSched sc, const double* __restrict__ fT, const double* __restrict__ vT,
                   double* __restrict__ QT) {
    extern __shared__ __align__(16) double smem[];
    __shared__ int s_unit, s_next;
    const int M = op.n_q * K;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    double* fs = smem;
    double* vs = JV ? smem + (size_t)M * kTileCells : nullptr;
    double* rb = smem + (size_t)(JV ? 2 : 1) * M * kTileCells + (size_t)warp * RPair<K>::SIZE;
    int staged = -1;

    for (;;) {
        if (tid == 0) s_unit = atomicAdd(sc.counter, 1);
        __syncthreads();
        const int u = s_unit;
        if (u >= sc.n_units) break;
        int ht, bin;
        if (u < sc.n_whole) {
            ht = u;
            bin = 0;
        } else {
            const int v = u - sc.n_whole;
            ht = sc.n_whole + v / sc.split;
            bin = bin_base(sc.split) + v % sc.split;
        }
        const size_t tile_base = (size_t)(ht >> 1) * M * CF_TILE + (size_t)(ht & 1) * kTileCells;
        if (ht != staged) {
            const double* srcf = fT + tile_base;
            for (int i = tid; i < M * 8; i += W * 32) {
                const int r = i >> 3, w = (i & 7) * 2;
                cp_async16(fs + r * kTileCells + w, srcf + (size_t)r * CF_TILE + w);
            }
            if constexpr (JV) {
                const double* srcv = vT + tile_base;
                for (int i = tid; i < M * 8; i += W * 32) {
                    const int r = i >> 3, w = (i & 7) * 2;
                    cp_async16(vs + r * kTileCells + w, srcv + (size_t)r * CF_TILE + w);
                }
            }
            cp_async_commit();
            cp_async_wait_all();
            staged = ht;
        }
        if (tid == 0) s_next = 0;
        __syncthreads();
        const int b0 = sc.bin_begin[bin], nb = sc.bin_begin[bin + 1] - b0;
        double* qtc = QT + tile_base + (lane & 15);
        for (;;) {
            int i = 0;
            if (lane == 0) i = atomicAdd(&s_next, 1);
            i = __shfl_sync(0xffffffffu, i, 0);
            if (i >= nb) break;
            pair_item<K, EXACT, JV, RG>(op, sc.items[sc.bin_item[b0 + i]], fs, vs, rb, qtc, lane);
        }
        __syncthreads();
    }
}

template <int K>
constexpr size_t pair_smem_bytes(int M, int W, bool jv, bool rg) {
    return sizeof(double) * ((size_t)(jv ? 2 : 1) * M * kTileCells + (rg ? 0 : (size_t)W * RPair<K>::SIZE));
}

}  // namespace cf
