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
#include <type_traits>

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

template <int K, typename T = double>
struct RPair {
    // keep each warp's buffer 16-byte aligned
    static constexpr int SIZE = (K * K * K * (int)sizeof(T) + 15) / 16 * 16 / (int)sizeof(T);
};

// R_t as read by the kernels: FP64 R, or the plan's FP32 copy for the FP32 form
template <typename T>
__device__ __forceinline__ const T* r_tensor(const DevOp& op);
template <>
__device__ __forceinline__ const double* r_tensor<double>(const DevOp& op) { return op.R; }
template <>
__device__ __forceinline__ const float* r_tensor<float>(const DevOp& op) { return op.R32; }

// RG = false: R_t is staged into the warp's shared buffer with cp.async.  RG = true: R_t is read
// straight from global memory with warp-uniform loads through L1 (prefetched into L1 at the start
// of the slice), which keeps the K^3 step off the shared-memory wavefront budget.
// T = double: the FP64 forms (accumulating from the caller's Q).  T = float: the FP32 form (f, R,
// Phi and the per-row sums in FP32; the FP32 result is added to the caller's FP64 Q at the end).
template <int K, bool EXACT, bool JV, bool RG, typename T = double>
__device__ __forceinline__ void pair_item(const DevOp& op, int2 item, const T* __restrict__ fs,
                                          const T* __restrict__ vs, T* rb, double* qtc, int lane) {
    static_assert(!EXACT || sizeof(T) == 8, "the exact order is FP64");
    constexpr bool F64 = sizeof(T) == 8;
    const int half = lane >> 4;
    const int c = lane & 15;
    const bool active = half == 0 || item.y >= 0;
    const int q1 = half == 0 ? item.x : (item.y >= 0 ? item.y : item.x);

    T acc[K];
#pragma unroll
    for (int k1 = 0; k1 < K; ++k1) acc[k1] = (F64 && active) ? (T)qtc[(size_t)(q1 * K + k1) * CF_TILE] : (T)0;

    // slices of qa and qb correspond one to one (same t, same length)
    const int sa0 = op.q1_begin[item.x], sa1 = op.q1_begin[item.x + 1];
    const int sb0 = item.y >= 0 ? op.q1_begin[item.y] : sa0;
    for (int i = 0; i < sa1 - sa0; ++i) {
        const int sa = sa0 + i, sb = sb0 + i;
        const int t = op.slice_t[sa];
        const int ea = op.slice_e[sa], n_e = op.slice_e[sa + 1] - ea;
        const int eb_ = op.slice_e[sb];
        const int my_e0 = half == 0 ? ea : eb_;

        const T* __restrict__ Rt = r_tensor<T>(op) + (size_t)t * K * K * K;
        if constexpr (RG) {
            const char* rbytes = reinterpret_cast<const char*>(Rt);
            for (int off = lane * 128; off < K * K * K * (int)sizeof(T); off += 32 * 128)
                asm volatile("prefetch.global.L1 [%0];\n" ::"l"(rbytes + off));
        } else {
            __syncwarp();
            constexpr int PER16 = 16 / (int)sizeof(T);  // elements per 16-byte copy
            if constexpr ((K * K * K) % PER16 == 0) {
                for (int j = lane; j < K * K * K / PER16; j += 32) cp_async16(rb + PER16 * j, Rt + PER16 * j);
            } else if constexpr (F64) {
                for (int j = lane; j < K * K * K; j += 32) cp_async8(rb + j, Rt + j);
            } else {
                for (int j = lane; j < K * K * K; j += 32) rb[j] = Rt[j];
            }
            cp_async_commit();
        }

        T phi[K][K];
#pragma unroll
        for (int a = 0; a < K; ++a)
#pragma unroll
            for (int b = 0; b < K; ++b) phi[a][b] = (T)0;

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
                const T g = (T)__shfl_sync(0xffffffffu, my_g, j + 16 * half);
                const int r2 = (int)(q23 & 0xffffu) * K, r3 = (int)(q23 >> 16) * K;
                T f2[K], f3[K];
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    f2[k] = fs[(r2 + k) * kTileCells + c];
                    f3[k] = fs[(r3 + k) * kTileCells + c];
                }
                if constexpr (JV) {
                    T v2[K], v3[K];
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
                            const T gf3 = g * f3[b], gv3 = g * v3[b];
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
                        const T gf3 = g * f3[b];
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
        const T* __restrict__ rsrc = RG ? Rt : rb;

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
        } else if constexpr (!F64 && K % 4 == 0) {
#pragma unroll
            for (int b = 0; b < K; ++b)
#pragma unroll
                for (int a = 0; a < K; ++a) {
                    const float4* r4v = reinterpret_cast<const float4*>(rsrc + K * a + K * K * b);
#pragma unroll
                    for (int h = 0; h < K / 4; ++h) {
                        const float4 r = RG ? __ldg(r4v + h) : r4v[h];
                        acc[4 * h] = fmaf(r.x, phi[a][b], acc[4 * h]);
                        acc[4 * h + 1] = fmaf(r.y, phi[a][b], acc[4 * h + 1]);
                        acc[4 * h + 2] = fmaf(r.z, phi[a][b], acc[4 * h + 2]);
                        acc[4 * h + 3] = fmaf(r.w, phi[a][b], acc[4 * h + 3]);
                    }
                }
        } else if constexpr (F64 && K % 2 == 0) {
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
                        const T r = RG ? __ldg(rsrc + k1 + K * a + K * K * b) : rsrc[k1 + K * a + K * K * b];
                        acc[k1] = fma(r, phi[a][b], acc[k1]);
                    }
        }
    }
    if (active) {
#pragma unroll
        for (int k1 = 0; k1 < K; ++k1) {
            double* out = qtc + (size_t)(q1 * K + k1) * CF_TILE;
            *out = F64 ? (double)acc[k1] : *out + (double)acc[k1];
        }
    }
}

// Split variant (fast Q forms, K even): each lane holds BOTH rows of the pair for its cell, over half
// of the k3 range (lanes 0-15 the lower half, lanes 16-31 the upper half, same 16 cells).  Every R_t
// value a lane loads in the K^3 step then feeds two FMAs (rows qa and qb) instead of one, which
// halves the K^3 step's shared-memory wavefronts; the Phi step reads the same bytes as pair_item
// (f2 rows are shared by the two halves, f3 rows split between them).  The two halves' partial row
// sums are added with one shuffle per k1 at the end of the item.  Rows without a mirror use all 32
// lanes on the one row.
template <int K, typename T = double>
__device__ __forceinline__ void pair_split_item(const DevOp& op, int2 item, const T* __restrict__ fs, T* rb,
                                                double* qtc, int lane) {
    static_assert(K % 2 == 0, "the k3 range is split in two halves");
    constexpr int KH = K / 2;
    constexpr bool F64 = sizeof(T) == 8;
    const int h = lane >> 4;
    const int c = lane & 15;
    const bool has_b = item.y >= 0;  // warp-uniform
    const int qa = item.x, qb = has_b ? item.y : item.x;

    T acc_a[K], acc_b[K];
#pragma unroll
    for (int k1 = 0; k1 < K; ++k1) {
        acc_a[k1] = (F64 && h == 0) ? (T)qtc[(size_t)(qa * K + k1) * CF_TILE] : (T)0;
        acc_b[k1] = (F64 && h == 1 && has_b) ? (T)qtc[(size_t)(qb * K + k1) * CF_TILE] : (T)0;
    }

    const int sa0 = op.q1_begin[qa], sa1 = op.q1_begin[qa + 1];
    const int sb0 = has_b ? op.q1_begin[qb] : sa0;
    for (int i = 0; i < sa1 - sa0; ++i) {
        const int sa = sa0 + i, sb = sb0 + i;
        const int t = op.slice_t[sa];
        const int ea = op.slice_e[sa], n_e = op.slice_e[sa + 1] - ea;
        const int eb = op.slice_e[sb];

        const T* __restrict__ Rt = r_tensor<T>(op) + (size_t)t * K * K * K;
        __syncwarp();
        {
            constexpr int PER16 = 16 / (int)sizeof(T);
            if constexpr ((K * K * K) % PER16 == 0) {
                for (int j = lane; j < K * K * K / PER16; j += 32) cp_async16(rb + PER16 * j, Rt + PER16 * j);
            } else if constexpr (F64) {
                for (int j = lane; j < K * K * K; j += 32) cp_async8(rb + j, Rt + j);
            } else {
                for (int j = lane; j < K * K * K; j += 32) rb[j] = Rt[j];
            }
            cp_async_commit();
        }

        T pa[K][KH], pb[K][KH];
#pragma unroll
        for (int a = 0; a < K; ++a)
#pragma unroll
            for (int b = 0; b < KH; ++b) {
                pa[a][b] = (T)0;
                pb[a][b] = (T)0;
            }

        for (int e0 = 0; e0 < n_e; e0 += 16) {
            const int n = min(16, n_e - e0);
            // lanes 0-15 hold row qa's next entries, lanes 16-31 row qb's
            uint32_t my_q23 = 0;
            double my_g = 0.0;
            if (c < n && (h == 0 || has_b)) {
                const int e = (h == 0 ? ea : eb) + e0 + c;
                my_q23 = __ldg(op.e_q23 + e);
                my_g = __ldg(op.e_g + e);
            }
            for (int j = 0; j < n; ++j) {
                // both rows' rows of f are read before the FMAs, so each entry is one burst of
                // 2 K KH FMAs behind one set of loads (as in pair_item), not two half bursts
                const uint32_t qa23 = __shfl_sync(0xffffffffu, my_q23, j);
                const T ga = (T)__shfl_sync(0xffffffffu, my_g, j);
                const uint32_t qb23 = __shfl_sync(0xffffffffu, my_q23, 16 + j);
                const T gb = (T)__shfl_sync(0xffffffffu, my_g, 16 + j);
                const int ra2 = (int)(qa23 & 0xffffu) * K, ra3 = (int)(qa23 >> 16) * K + h * KH;
                const int rb2 = has_b ? (int)(qb23 & 0xffffu) * K : ra2;
                const int rb3 = has_b ? (int)(qb23 >> 16) * K + h * KH : ra3;
                T fa2[K], fa3[KH], fb2[K], fb3[KH];
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    fa2[k] = fs[(ra2 + k) * kTileCells + c];
                    fb2[k] = fs[(rb2 + k) * kTileCells + c];
                }
#pragma unroll
                for (int k = 0; k < KH; ++k) {
                    fa3[k] = fs[(ra3 + k) * kTileCells + c];
                    fb3[k] = fs[(rb3 + k) * kTileCells + c];
                }
                const T gbe = has_b ? gb : (T)0;  // a row without a mirror adds nothing to pb
#pragma unroll
                for (int b = 0; b < KH; ++b) {
                    const T gfa = ga * fa3[b], gfb = gbe * fb3[b];
#pragma unroll
                    for (int a = 0; a < K; ++a) {
                        pa[a][b] = fma(fa2[a], gfa, pa[a][b]);
                        pb[a][b] = fma(fb2[a], gfb, pb[a][b]);
                    }
                }
            }
        }
        cp_async_wait_all();
        __syncwarp();

        // K^3 step over this half's k3: R_t element (k1, k2=a, k3 = h KH + b) at rb[k1 + K a + K^2 k3];
        // the address is uniform over each half-warp
        if constexpr (!F64 && K % 4 == 0) {
#pragma unroll
            for (int b = 0; b < KH; ++b)
#pragma unroll
                for (int a = 0; a < K; ++a) {
                    const float4* r4v = reinterpret_cast<const float4*>(rb + K * a + K * K * (h * KH + b));
#pragma unroll
                    for (int hh = 0; hh < K / 4; ++hh) {
                        const float4 r = r4v[hh];
                        acc_a[4 * hh] = fmaf(r.x, pa[a][b], acc_a[4 * hh]);
                        acc_a[4 * hh + 1] = fmaf(r.y, pa[a][b], acc_a[4 * hh + 1]);
                        acc_a[4 * hh + 2] = fmaf(r.z, pa[a][b], acc_a[4 * hh + 2]);
                        acc_a[4 * hh + 3] = fmaf(r.w, pa[a][b], acc_a[4 * hh + 3]);
                        acc_b[4 * hh] = fmaf(r.x, pb[a][b], acc_b[4 * hh]);
                        acc_b[4 * hh + 1] = fmaf(r.y, pb[a][b], acc_b[4 * hh + 1]);
                        acc_b[4 * hh + 2] = fmaf(r.z, pb[a][b], acc_b[4 * hh + 2]);
                        acc_b[4 * hh + 3] = fmaf(r.w, pb[a][b], acc_b[4 * hh + 3]);
                    }
                }
        } else {
            using T2 = typename std::conditional<F64, double2, float2>::type;
#pragma unroll
            for (int b = 0; b < KH; ++b)
#pragma unroll
                for (int a = 0; a < K; ++a) {
                    const T2* r2v = reinterpret_cast<const T2*>(rb + K * a + K * K * (h * KH + b));
#pragma unroll
                    for (int hh = 0; hh < K / 2; ++hh) {
                        const T2 r = r2v[hh];
                        acc_a[2 * hh] = fma(r.x, pa[a][b], acc_a[2 * hh]);
                        acc_a[2 * hh + 1] = fma(r.y, pa[a][b], acc_a[2 * hh + 1]);
                        acc_b[2 * hh] = fma(r.x, pb[a][b], acc_b[2 * hh]);
                        acc_b[2 * hh + 1] = fma(r.y, pb[a][b], acc_b[2 * hh + 1]);
                    }
                }
        }
    }
    // half 0 owns row qa, half 1 row qb: each receives the other half's partial sum of its row
#pragma unroll
    for (int k1 = 0; k1 < K; ++k1) {
        const T send = h == 0 ? acc_b[k1] : acc_a[k1];
        const T recv = __shfl_xor_sync(0xffffffffu, send, 16);
        const T tot = (h == 0 ? acc_a[k1] : acc_b[k1]) + recv;
        if (h == 0 || has_b) {
            double* out = qtc + (size_t)((h == 0 ? qa : qb) * K + k1) * CF_TILE;
            *out = F64 ? (double)tot : *out + (double)tot;
        }
    }
}

// fT, vT: tiled cells in T (FP64 tiles for the FP64 forms, FP32 tiles for the FP32 form); QT: FP64.
template <int K, int W, bool EXACT, bool JV, bool RG, typename T = double, bool SPLIT = false>
__global__ void __launch_bounds__(W * 32, 1)
    af_pair_kernel(DevOp op, PairSched sc, const T* __restrict__ fT, const T* __restrict__ vT,
                   double* __restrict__ QT) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    __shared__ int s_unit, s_next;
    const int M = op.n_q * K;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    T* fs = smem;
    T* vs = JV ? smem + (size_t)M * kTileCells : nullptr;
    T* rb = smem + (size_t)(JV ? 2 : 1) * M * kTileCells + (size_t)warp * RPair<K, T>::SIZE;
    constexpr int PER16 = 16 / (int)sizeof(T);    // elements per 16-byte copy
    constexpr int CPR = kTileCells / PER16;       // 16-byte copies per 16-cell row
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
            const T* srcf = fT + tile_base;
            for (int i = tid; i < M * CPR; i += W * 32) {
                const int r = i / CPR, w = (i % CPR) * PER16;
                cp_async16(fs + r * kTileCells + w, srcf + (size_t)r * CF_TILE + w);
            }
            if constexpr (JV) {
                const T* srcv = vT + tile_base;
                for (int i = tid; i < M * CPR; i += W * 32) {
                    const int r = i / CPR, w = (i % CPR) * PER16;
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
            if constexpr (SPLIT)
                pair_split_item<K, T>(op, sc.items[sc.bin_item[b0 + i]], fs, rb, qtc, lane);
            else
                pair_item<K, EXACT, JV, RG, T>(op, sc.items[sc.bin_item[b0 + i]], fs, vs, rb, qtc, lane);
        }
        __syncthreads();
    }
}

template <int K, typename T = double>
constexpr size_t pair_smem_bytes(int M, int W, bool jv, bool rg) {
    return sizeof(T) * ((size_t)(jv ? 2 : 1) * M * kTileCells + (rg ? 0 : (size_t)W * RPair<K, T>::SIZE));
}

}  // namespace cf
