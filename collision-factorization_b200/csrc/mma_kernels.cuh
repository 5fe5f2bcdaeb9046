// mma_kernels.cuh -- the tile-resident angular-first kernel with its K^3 step on the FP64 tensor
// cores (warp-level mma.sync m8n8k4 f64), for K = 8.
//
// Per q1 row and 16 resident cells the K^3 step is a product
//     C[k1][cell] += sum_kk R_t^T[k1][kk] Phi[kk][cell],   kk = K k2 + k3 (64 values),
// i.e. 16 MMAs of m8n8k4 per 8-cell tile.  B200's tensor cores have no FP64 tcgen05 kind; the
// warp-level FP64 MMA is the tensor path for double precision.  What it buys here is shared-memory
// bandwidth: a lane loads one R_t value per MMA (32 distinct values per warp load) instead of the
// warp-uniform broadcasts of the SIMT K^3 step, which bound the tile kernel.
//
// Lane i = (n = i >> 2, r = i & 3) accumulates Phi for cells n and n + 8, all k2, and k3 in
// {r, r + 4}: exactly the B fragments (B[k = r][col = n], kk = 4 j + r) of the MMAs, so Phi never
// moves between lanes.  A fragments (A[row = k1 = i >> 2][col = r]) come from R_t^T staged per warp
// with a padded row (68 doubles: conflict-free).  The four lanes of a cell read four consecutive
// f rows in the Phi step, so the half-tile is staged with its cells XOR-swizzled by 4 (row & 3).
#pragma once
#include "tile_kernels.cuh"

namespace cf {

constexpr int kMmaK = 8;
constexpr int kRaStride = 68;
constexpr int kRaSize = kMmaK * kRaStride;  // doubles per warp

// position of (row, cell) in the swizzled half-tile
__device__ __forceinline__ int swz(int row, int cell) { return row * kTileCells + (cell ^ ((row & 3) << 2)); }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Contract every slice of q1 for the resident (swizzled) half-tile; qt points at cell 0 of the
// half-tile in the tiled output (rows CF_TILE apart); out += ...
__device__ __forceinline__ void mma_q1(const DevOp& op, int q1, const double* __restrict__ fs, double* ra,
                                       double* qt, int lane) {
    constexpr int K = kMmaK;
    const int n = lane >> 2, r = lane & 3;
    const int k1c = lane >> 2;  // C fragment row
    // two accumulator sets per 8-cell tile (even and odd K-slices): the MMAs of one tile form two
    // independent chains instead of one, halving the wait on the MMA latency
    double c[2][2], c2[2][2];
#pragma unroll
    for (int t = 0; t < 2; ++t)
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            c[t][u] = qt[(size_t)(q1 * K + k1c) * CF_TILE + 8 * t + 2 * r + u];
            c2[t][u] = 0.0;
        }

    const int s0 = op.q1_begin[q1], s1 = op.q1_begin[q1 + 1];
    for (int s = s0; s < s1; ++s) {
        const int tt = op.slice_t[s];
        const int e0 = op.slice_e[s], e1 = op.slice_e[s + 1];
        __syncwarp();
        const double* __restrict__ RTt = op.RT + (size_t)tt * K * K * K;
        for (int i = lane; i < K * K * K / 2; i += 32) {
            const int k1 = i >> 5, kk = (i & 31) * 2;
            cp_async16(ra + k1 * kRaStride + kk, RTt + k1 * K * K + kk);
        }
        cp_async_commit();

        double phi[2][K][2];
#pragma unroll
        for (int t = 0; t < 2; ++t)
#pragma unroll
            for (int a = 0; a < K; ++a) {
                phi[t][a][0] = 0.0;
                phi[t][a][1] = 0.0;
            }

        for (int eb = e0; eb < e1; eb += 32) {
            const int nb = min(32, e1 - eb);
            uint32_t my_q23 = 0;
            double my_g = 0.0;
            if (lane < nb) {
                my_q23 = __ldg(op.e_q23 + eb + lane);
                my_g = __ldg(op.e_g + eb + lane);
            }
            for (int j = 0; j < nb; ++j) {
                const uint32_t q23 = __shfl_sync(0xffffffffu, my_q23, j);
                const double g = __shfl_sync(0xffffffffu, my_g, j);
                const int r2 = (int)(q23 & 0xffffu) * K, r3 = (int)(q23 >> 16) * K + r;
                double gf3[2][2];
#pragma unroll
                for (int t = 0; t < 2; ++t)
#pragma unroll
                    for (int h = 0; h < 2; ++h) gf3[t][h] = g * fs[swz(r3 + 4 * h, n + 8 * t)];
#pragma unroll
                for (int k2 = 0; k2 < K; ++k2) {
                    const double f20 = fs[swz(r2 + k2, n)], f21 = fs[swz(r2 + k2, n + 8)];
                    phi[0][k2][0] = fma(f20, gf3[0][0], phi[0][k2][0]);
                    phi[0][k2][1] = fma(f20, gf3[0][1], phi[0][k2][1]);
                    phi[1][k2][0] = fma(f21, gf3[1][0], phi[1][k2][0]);
                    phi[1][k2][1] = fma(f21, gf3[1][1], phi[1][k2][1]);
                }
            }
        }
        cp_async_wait_all();
        __syncwarp();

        // K^3 step: 16 K-slices of 4 kk each, two 8-cell tiles
        const double* __restrict__ arow = ra + k1c * kRaStride + r;
#pragma unroll
        for (int j = 0; j < 2 * K; j += 2) {
            const double a0 = arow[4 * j], a1 = arow[4 * j + 4];
            dmma(c[0][0], c[0][1], a0, phi[0][j >> 1][0]);
            dmma(c[1][0], c[1][1], a0, phi[1][j >> 1][0]);
            dmma(c2[0][0], c2[0][1], a1, phi[0][j >> 1][1]);
            dmma(c2[1][0], c2[1][1], a1, phi[1][j >> 1][1]);
        }
    }
#pragma unroll
    for (int t = 0; t < 2; ++t) {
        double2* out = reinterpret_cast<double2*>(qt + (size_t)(q1 * K + k1c) * CF_TILE + 8 * t + 2 * r);
        *out = make_double2(c[t][0] + c2[t][0], c[t][1] + c2[t][1]);
    }
}

template <int W>
__global__ void __launch_bounds__(W * 32, 1)
    af_mma_kernel(DevOp op, TileSched sc, const double* __restrict__ fT, double* __restrict__ QT) {
    constexpr int K = kMmaK;
    extern __shared__ __align__(16) double smem[];
    __shared__ int s_unit, s_next;
    const int M = op.n_q * K;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    double* fs = smem;
    double* ra = smem + (size_t)M * kTileCells + (size_t)warp * kRaSize;
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
                const int row = i >> 3, w = (i & 7) * 2;
                cp_async16(fs + swz(row, w), srcf + (size_t)row * CF_TILE + w);
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
            mma_q1(op, sc.bin_q1[b0 + i], fs, ra, qt, lane);
        }
        __syncthreads();
    }
}

constexpr size_t mma_smem_bytes(int M, int W) {
    return sizeof(double) * ((size_t)M * kTileCells + (size_t)W * kRaSize);
}

}  // namespace cf
