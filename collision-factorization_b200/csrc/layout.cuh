// layout.cuh -- layout passes between the MEX-native cell-major arrays and the tiled
// cell-fastest layout the contraction kernels read (see common.cuh).  Included by plan.cu only.
#pragma once
#include "common.cuh"

namespace cf {

// ----------------------------------------------------------------------------------------
// Layout passes: MEX-native cell-major [B][N_Q*K] (m = q + k*N_Q)  <->  tiled [tile][q*K+k][32]
// ----------------------------------------------------------------------------------------
template <typename TO>
__global__ void __launch_bounds__(256) pack_tiles_kernel(const double* __restrict__ src,
                                                         TO* __restrict__ dst, int64_t B,
                                                         int nq, int K) {
    __shared__ double sm[32][33];
    const int M = nq * K;
    const int64_t tile = blockIdx.y;
    const int m0 = blockIdx.x * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int c = ty; c < 32; c += 8) {
        const int64_t b = tile * 32 + c;
        const int m = m0 + tx;
        sm[c][tx] = (b < B && m < M) ? src[b * M + m] : 0.0;
    }
    __syncthreads();
    for (int j = ty; j < 32; j += 8) {
        const int m = m0 + j;
        if (m < M) {
            const int q = m % nq, k = m / nq;
            dst[(tile * M + (int64_t)q * K + k) * 32 + tx] = (TO)sm[tx][j];
        }
    }
}

static __global__ void __launch_bounds__(256) unpack_tiles_kernel(const double* __restrict__ src,
                                                           double* __restrict__ dst, int64_t B,
                                                           int nq, int K) {
    __shared__ double sm[32][33];
    const int M = nq * K;
    const int64_t tile = blockIdx.y;
    const int m0 = blockIdx.x * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int j = ty; j < 32; j += 8) {
        const int m = m0 + j;
        double v = 0.0;
        if (m < M) {
            const int q = m % nq, k = m / nq;
            v = src[(tile * M + (int64_t)q * K + k) * 32 + tx];
        }
        sm[j][tx] = v;
    }
    __syncthreads();
    for (int c = ty; c < 32; c += 8) {
        const int64_t b = tile * 32 + c;
        const int m = m0 + tx;
        if (b < B && m < M) dst[b * M + m] = sm[tx][c];
    }
}

// FP64 FMA throughput probe: kProbeChains independent DFMA chains per thread.
constexpr int kProbeChains = 8;
static __global__ void __launch_bounds__(256) fp64_fma_probe_kernel(double* sink, int iters, double a) {
    double x[kProbeChains];
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c) x[c] = threadIdx.x * 1e-3 + c;
    const double b = 1e-9;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kProbeChains; ++c) x[c] = fma(x[c], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c) s += x[c];
    sink[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace cf
