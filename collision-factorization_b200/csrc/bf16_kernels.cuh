// bf16_kernels.cuh -- the BF16-split angular-first form: the Phi step in FP32 on the CUDA cores,
// the K^3 step on the BF16 tensor cores as a two-term split, for K = 8.
//
// Per q1 row and 8-cell tile the K^3 step is C[k1][cell] += sum_kk R_t^T[k1][kk] Phi[kk][cell]
// (kk = K k2 + k3, 64 values).  With R_t^T = R_hi + R_lo and Phi = Phi_hi + Phi_lo in BF16 (each
// pair carries about 16 significant bits), the product is taken by the warp-level MMA
// m16n8k16 (BF16 in, FP32 accumulate) with the A operand stacking R_hi^T (rows 0-7) over R_lo^T
// (rows 8-15): one MMA against Phi_hi and one against Phi_lo per 16-wide slice of kk give all four
// cross terms, and row k1 of the result is the sum of accumulator rows k1 and 8 + k1.  Relative
// error ~1e-5 (FP32 accumulation of the cancelling terms of Q dominates, as in the FP32 form); the
// invariant rows stay exactly zero because both halves of a zero row of R are zero.
//
// Lane i = (g = i >> 2, t = i & 3) accumulates Phi for cells g and g + 8, all k2, and k3 in
// {2t, 2t + 1}: the B fragments of m16n8k16 (B[k = 2t + e (+8)][col = g]).  The half-tile of f is
// staged in FP32 as [q][cell][k] so that a lane's k-runs are contiguous (float4 / float2 loads).
// R_t^T's BF16 halves are staged per warp with a padded row (36 words: conflict-free A loads).
#pragma once
#include <cuda_bf16.h>

#include "tile_kernels.cuh"

namespace cf {

constexpr int kBfK = 8;
constexpr int kBfRow = 72;                     // bf16 per staged R row (64 + 8 pad)
constexpr int kBfWarpBuf = 2 * kBfK * kBfRow;  // bf16 per warp: hi rows then lo rows

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void bmma(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                     uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// hi and lo BF16 pairs of two FP32 values (lower index in the low half)
__device__ __forceinline__ void split2(float x, float y, uint32_t& hi, uint32_t& lo) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(x, y);
    const __nv_bfloat162 l = __floats2bfloat162_rn(x - __bfloat162float(h.x), y - __bfloat162float(h.y));
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = *reinterpret_cast<const uint32_t*>(&l);
}

// Contract every slice of q1 for the resident half-tile (fs: FP32 [q][16 cells][K]); qt points at
// cell 0 of the half-tile in the tiled FP64 output; the FP32 row sums are added to it.
__device__ __forceinline__ void bf16_q1(const DevOp& op, int q1, const float* __restrict__ fs,
                                        unsigned short* rb, double* qt, int lane) {
    constexpr int K = kBfK;
    const int g = lane >> 2, t = lane & 3;
    float c[2][4];
#pragma unroll
    for (int tl = 0; tl < 2; ++tl)
#pragma unroll
        for (int u = 0; u < 4; ++u) c[tl][u] = 0.f;
    const uint32_t* rw = reinterpret_cast<const uint32_t*>(rb);  // rows of kBfRow / 2 words

    const int s0 = op.q1_begin[q1], s1 = op.q1_begin[q1 + 1];
    for (int s = s0; s < s1; ++s) {
        const int tt = op.slice_t[s];
        const int e0 = op.slice_e[s], e1 = op.slice_e[s + 1];
        __syncwarp();
        // stage R_t^T hi and lo: 16 rows of 64 bf16 (128 B = 8 x 16 B each)
        const unsigned short* src = op.RTbf + (size_t)tt * 2 * K * 64;
        for (int i = lane; i < 16 * 8; i += 32) {
            const int row = i >> 3, w = (i & 7) * 8;
            cp_async16(rb + row * kBfRow + w, src + row * 64 + w);
        }
        cp_async_commit();

        float phi[2][K][2];
#pragma unroll
        for (int tl = 0; tl < 2; ++tl)
#pragma unroll
            for (int a = 0; a < K; ++a) {
                phi[tl][a][0] = 0.f;
                phi[tl][a][1] = 0.f;
            }
        for (int eb = e0; eb < e1; eb += 32) {
            const int nb = min(32, e1 - eb);
            uint32_t my_q23 = 0;
            float my_g = 0.f;
            if (lane < nb) {
                my_q23 = __ldg(op.e_q23 + eb + lane);
                my_g = (float)__ldg(op.e_g + eb + lane);
            }
            for (int j = 0; j < nb; ++j) {
                const uint32_t q23 = __shfl_sync(0xffffffffu, my_q23, j);
                const float gv = __shfl_sync(0xffffffffu, my_g, j);
                const int q2 = (int)(q23 & 0xffffu), q3 = (int)(q23 >> 16);
#pragma unroll
                for (int tl = 0; tl < 2; ++tl) {
                    const int cell = g + 8 * tl;
                    const float2 f3 = *reinterpret_cast<const float2*>(fs + ((size_t)q3 * 16 + cell) * K + 2 * t);
                    const float gf0 = gv * f3.x, gf1 = gv * f3.y;
                    const float4* f2v = reinterpret_cast<const float4*>(fs + ((size_t)q2 * 16 + cell) * K);
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const float4 f2 = f2v[h];
                        phi[tl][4 * h][0] = fmaf(f2.x, gf0, phi[tl][4 * h][0]);
                        phi[tl][4 * h][1] = fmaf(f2.x, gf1, phi[tl][4 * h][1]);
                        phi[tl][4 * h + 1][0] = fmaf(f2.y, gf0, phi[tl][4 * h + 1][0]);
                        phi[tl][4 * h + 1][1] = fmaf(f2.y, gf1, phi[tl][4 * h + 1][1]);
                        phi[tl][4 * h + 2][0] = fmaf(f2.z, gf0, phi[tl][4 * h + 2][0]);
                        phi[tl][4 * h + 2][1] = fmaf(f2.z, gf1, phi[tl][4 * h + 2][1]);
                        phi[tl][4 * h + 3][0] = fmaf(f2.w, gf0, phi[tl][4 * h + 3][0]);
                        phi[tl][4 * h + 3][1] = fmaf(f2.w, gf1, phi[tl][4 * h + 3][1]);
                    }
                }
            }
        }
        cp_async_wait_all();
        __syncwarp();

        // K^3 step: 4 slices of 16 kk; A rows 0-7 R_hi^T, rows 8-15 R_lo^T
#pragma unroll
        for (int ch = 0; ch < K / 2; ++ch) {
            const int wbase = g * (kBfRow / 2) + 8 * ch + t;  // word of (k1 = g, kk = 16 ch + 2 t)
            const uint32_t a0 = rw[wbase];
            const uint32_t a1 = rw[K * (kBfRow / 2) + wbase];
            const uint32_t a2 = rw[wbase + 4];
            const uint32_t a3 = rw[K * (kBfRow / 2) + wbase + 4];
#pragma unroll
            for (int tl = 0; tl < 2; ++tl) {
                uint32_t b0h, b0l, b1h, b1l;
                split2(phi[tl][2 * ch][0], phi[tl][2 * ch][1], b0h, b0l);          // kk = 16 ch + 2t + {0,1}
                split2(phi[tl][2 * ch + 1][0], phi[tl][2 * ch + 1][1], b1h, b1l);  // kk = 16 ch + 8 + 2t + {0,1}
                bmma(c[tl], a0, a1, a2, a3, b0h, b1h);
                bmma(c[tl], a0, a1, a2, a3, b0l, b1l);
            }
        }
    }
    // row k1 = g of the product: accumulator rows g (R_hi) and 8 + g (R_lo)
#pragma unroll
    for (int tl = 0; tl < 2; ++tl) {
        double* out = qt + (size_t)(q1 * K + g) * CF_TILE + 8 * tl + 2 * t;
        out[0] += (double)(c[tl][0] + c[tl][2]);
        out[1] += (double)(c[tl][1] + c[tl][3]);
    }
}

template <int W>
__global__ void __launch_bounds__(W * 32, 1)
    af_bf16_kernel(DevOp op, TileSched sc, const float* __restrict__ fT32, double* __restrict__ QT) {
    constexpr int K = kBfK;
    extern __shared__ __align__(16) unsigned char bsm[];
    __shared__ int s_unit, s_next;
    const int M = op.n_q * K;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    float* fs = reinterpret_cast<float*>(bsm);
    unsigned short* rb = reinterpret_cast<unsigned short*>(bsm + (size_t)M * kTileCells * sizeof(float)) +
                         (size_t)warp * kBfWarpBuf;
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
            // tiled FP32 rows (row = q K + k, 16 cells) -> [q][cell][k]
            const float* srcf = fT32 + tile_base;
            for (int i = tid; i < M * kTileCells; i += W * 32) {
                const int row = i >> 4, cell = i & 15;
                cp_async4(fs + ((size_t)(row / K) * kTileCells + cell) * K + row % K, srcf + (size_t)row * CF_TILE + cell);
            }
            cp_async_commit();
            cp_async_wait_all();
            staged = ht;
        }
        if (tid == 0) s_next = 0;
        __syncthreads();
        const int b0 = sc.bin_begin[bin], nb = sc.bin_begin[bin + 1] - b0;
        double* qt = QT + tile_base;
        for (;;) {
            int i = 0;
            if (lane == 0) i = atomicAdd(&s_next, 1);
            i = __shfl_sync(0xffffffffu, i, 0);
            if (i >= nb) break;
            bf16_q1(op, sc.bin_q1[b0 + i], fs, rb, qt, lane);
        }
        __syncthreads();
    }
}

constexpr size_t bf16_smem_bytes(int M, int W) {
    return sizeof(float) * (size_t)M * kTileCells + sizeof(unsigned short) * (size_t)W * kBfWarpBuf;
}

}  // namespace cf
