// mlp.cu -- the learned block preconditioner's network: forward, backward and Adam, in FP32.
//
// Architecture: x [n_in] -> Linear -> GELU -> Linear -> GELU -> Linear -> y [n_out]
// (two hidden layers of n_hidden, exact erf GELU).  Weights follow the [out][in] convention.
// Every matrix product is the tiled SIMT SGEMM below (64 x 64 output tile per CTA, 4 x 4 outputs
// per thread, K in steps of 16 through shared memory); the network is small (0.6 M + 0.26 M + 2.7 M
// weights at n_in = 649, n_hidden = 512, n_out = 5184), so these kernels are not on the hot path
// of a time step: inference is one forward pass per cell per step.
//
// The loss that trains it lives here too: for a cell with probe pairs (v_p, a_p = A v_p) of the
// implicit operator A = I - dt J(f), the preconditioner P = P_eq + s * Delta(f) is fitted block by
// block to map a_p back to v_p:
//     L = (1/n_p) sum_p sum_q |P_q a_{p,q} - v_{p,q}|^2 / |v_p|^2.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <random>
#include <vector>

#include "../../include/cf_b200.h"

void cf_set_last_error(const char* msg);

namespace {

constexpr int TM = 64, TN = 64, TK = 16;

// C[M x N] = alpha * op(A)[M x K] op(B)[K x N] + beta * C, then + bias[N], then GELU (pre-activation
// stored in Z when given).  op(A)(i,k) = TA ? A[k*lda + i] : A[i*lda + k]; op(B)(k,j) = TB ? B[j*ldb + k] : B[k*ldb + j].
template <bool TA, bool TB>
__global__ void __launch_bounds__(256) k_sgemm(int M, int N, int K, const float* __restrict__ A, int lda,
                                               const float* __restrict__ B, int ldb, float* __restrict__ C, int ldc,
                                               float alpha, float beta, const float* __restrict__ bias, int gelu,
                                               float* __restrict__ Z) {
    __shared__ float As[TK][TM + 4];
    __shared__ float Bs[TK][TN + 4];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int i0 = blockIdx.y * TM, j0 = blockIdx.x * TN;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += TK) {
        for (int t = threadIdx.x; t < TM * TK; t += 256) {
            const int ii = TA ? (t % TM) : (t / TK), kk = TA ? (t / TM) : (t % TK);
            const int gi = i0 + ii, gk = k0 + kk;
            float v = 0.f;
            if (gi < M && gk < K) v = TA ? A[(size_t)gk * lda + gi] : A[(size_t)gi * lda + gk];
            As[kk][ii] = v;
        }
        for (int t = threadIdx.x; t < TN * TK; t += 256) {
            const int jj = TB ? (t / TK) : (t % TN), kk = TB ? (t % TK) : (t / TN);
            const int gj = j0 + jj, gk = k0 + kk;
            float v = 0.f;
            if (gj < N && gk < K) v = TB ? B[(size_t)gj * ldb + gk] : B[(size_t)gk * ldb + gj];
            Bs[kk][jj] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TK; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) a[r] = As[kk][ty * 4 + r];
#pragma unroll
            for (int c = 0; c < 4; ++c) b[c] = Bs[kk][tx * 4 + c];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[r][c] = fmaf(a[r], b[c], acc[r][c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int i = i0 + ty * 4 + r;
        if (i >= M) continue;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int j = j0 + tx * 4 + c;
            if (j >= N) continue;
            float v = alpha * acc[r][c];
            if (beta != 0.f) v += beta * C[(size_t)i * ldc + j];
            if (bias) v += bias[j];
            if (Z) Z[(size_t)i * ldc + j] = v;
            if (gelu) v = 0.5f * v * (1.f + erff(v * 0.70710678118654752f));
            C[(size_t)i * ldc + j] = v;
        }
    }
}

// dZ = dY * GELU'(Z) in place on dY
__global__ void k_gelu_back(float* __restrict__ dy, const float* __restrict__ z, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float x = z[i];
        const float cdf = 0.5f * (1.f + erff(x * 0.70710678118654752f));
        const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
        dy[i] *= cdf + x * pdf;
    }
}

// db[j] = sum_i dZ[i][j]
__global__ void k_colsum(const float* __restrict__ dz, float* __restrict__ db, int n, int cols) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= cols) return;
    float s = 0.f;
    for (int i = 0; i < n; ++i) s += dz[(size_t)i * cols + j];
    db[j] = s;
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       size_t n, float lr, float b1, float b2, float eps, float c1, float c2, float wd) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i] + wd * w[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// Probe loss and its gradient with respect to Delta (one thread per (sample, q)).
// delta: [n][nq][K][K]; peq: [nq][K][K] (FP64); av, v: [n][np][nq*K] with block q at q*K.
__global__ void k_probe_loss(const float* __restrict__ delta, const double* __restrict__ peq,
                             const float* __restrict__ av, const float* __restrict__ v,
                             const float* __restrict__ vnorm2, float scale, int n, int np, int nq, int K,
                             float* __restrict__ grad, double* __restrict__ loss) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)n * nq) return;
    const int s = (int)(idx / nq), q = (int)(idx % nq);
    const float* D = delta + ((size_t)s * nq + q) * K * K;
    const double* Pe = peq + (size_t)q * K * K;
    float G[16 * 16];
    for (int i = 0; i < K * K; ++i) G[i] = 0.f;
    double l = 0.0;
    for (int p = 0; p < np; ++p) {
        const float* a = av + ((size_t)s * np + p) * nq * K + (size_t)q * K;
        const float* t = v + ((size_t)s * np + p) * nq * K + (size_t)q * K;
        const float w = 1.f / (vnorm2[(size_t)s * np + p] * np);
        for (int i = 0; i < K; ++i) {
            double r = -(double)t[i];
            for (int j = 0; j < K; ++j) r += ((double)Pe[i * K + j] + (double)scale * D[i * K + j]) * a[j];
            l += w * r * r;
            for (int j = 0; j < K; ++j) G[i * K + j] += 2.f * w * (float)r * a[j] * scale;
        }
    }
    float* Go = grad + ((size_t)s * nq + q) * K * K;
    for (int i = 0; i < K * K; ++i) Go[i] = G[i] / n;
    atomicAdd(loss, l / n);
}

// P[cell][q] = Peq[q] + scale * Delta[cell][q] in FP64 (the per-cell preconditioner GMRES applies)
__global__ void k_assemble_precond(const float* __restrict__ delta, const double* __restrict__ peq, double* __restrict__ P,
                                   float scale, size_t n_cells, int nqkk) {
    const size_t n = n_cells * nqkk;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        P[i] = peq[i % nqkk] + (double)scale * (double)delta[i];
}

int grid1d(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

}  // namespace

// ------------------------------------------------------------------------------------------------
struct cf_mlp {
    int device = 0;
    int n_in = 0, n_hid = 0, n_out = 0, max_batch = 0;
    // parameters, gradients and Adam moments in one device allocation each
    float* params = nullptr;
    float* grads = nullptr;
    float* m1 = nullptr;
    float* m2 = nullptr;
    size_t n_params = 0;
    size_t off[6] = {};  // W1, b1, W2, b2, W3, b3
    // activations for backward: Z1, H1, Z2, H2 (each [max_batch][n_hid]) and dY/dH scratch
    float* act = nullptr;
    float* scratch = nullptr;
    int adam_t = 0;
    std::mutex mu;
};

namespace {

#define MCHECK(expr)                                                                                    \
    do {                                                                                                \
        cudaError_t e_ = (expr);                                                                        \
        if (e_ != cudaSuccess) {                                                                        \
            char m_[256];                                                                               \
            snprintf(m_, sizeof(m_), "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
            cf_set_last_error(m_);                                                                      \
            return e_ == cudaErrorMemoryAllocation ? CF_ENOMEM : CF_ECUDA;                              \
        }                                                                                               \
    } while (0)

template <bool TA, bool TB>
int gemm(cudaStream_t s, int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C, int ldc,
         float alpha, float beta, const float* bias, int gelu, float* Z) {
    if (M == 0 || N == 0) return CF_OK;
    dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM);
    k_sgemm<TA, TB><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, alpha, beta, bias, gelu, Z);
    MCHECK(cudaGetLastError());
    return CF_OK;
}

float* W(cf_mlp* m, int i) { return m->params + m->off[i]; }
float* dW(cf_mlp* m, int i) { return m->grads + m->off[i]; }

}  // namespace

extern "C" {

int cf_mlp_create(cf_mlp** out, int32_t n_in, int32_t n_hidden, int32_t n_out, int32_t max_batch, uint64_t seed,
                  int32_t device) {
    if (!out || n_in < 1 || n_hidden < 1 || n_out < 1 || max_batch < 1) {
        cf_set_last_error("cf_mlp_create: sizes must be positive");
        return CF_EINVAL;
    }
    *out = nullptr;
    int cur = 0;
    MCHECK(cudaGetDevice(&cur));
    if (device < 0) device = cur;
    if (device != cur) MCHECK(cudaSetDevice(device));
    cf_mlp* m = new cf_mlp();
    m->device = device;
    m->n_in = n_in;
    m->n_hid = n_hidden;
    m->n_out = n_out;
    m->max_batch = max_batch;
    const size_t sizes[6] = {(size_t)n_hidden * n_in, (size_t)n_hidden, (size_t)n_hidden * n_hidden, (size_t)n_hidden,
                             (size_t)n_out * n_hidden, (size_t)n_out};
    size_t o = 0;
    for (int i = 0; i < 6; ++i) {
        m->off[i] = o;
        o += (sizes[i] + 63) & ~size_t(63);
    }
    m->n_params = o;
    // Kaiming-uniform-like init (U(-1/sqrt(fan_in), 1/sqrt(fan_in))); last layer scaled down so the
    // network starts near Delta = 0, i.e. near the Maxwellian preconditioner
    std::vector<float> h(o, 0.f);
    std::mt19937_64 rng(seed);
    const int fan[3] = {n_in, n_hidden, n_hidden};
    for (int layer = 0; layer < 3; ++layer) {
        const float bound = 1.f / std::sqrt((float)fan[layer]) * (layer == 2 ? 0.01f : 1.f);
        std::uniform_real_distribution<float> U(-bound, bound);
        for (size_t i = 0; i < sizes[2 * layer]; ++i) h[m->off[2 * layer] + i] = U(rng);
        for (size_t i = 0; i < sizes[2 * layer + 1]; ++i) h[m->off[2 * layer + 1] + i] = layer == 2 ? 0.f : U(rng);
    }
    cudaError_t e = cudaSuccess;
    e = e ? e : cudaMalloc(&m->params, o * sizeof(float));
    e = e ? e : cudaMalloc(&m->grads, o * sizeof(float));
    e = e ? e : cudaMalloc(&m->m1, o * sizeof(float));
    e = e ? e : cudaMalloc(&m->m2, o * sizeof(float));
    e = e ? e : cudaMalloc(&m->act, (size_t)4 * max_batch * n_hidden * sizeof(float));
    e = e ? e : cudaMalloc(&m->scratch, (size_t)max_batch * (n_out > n_hidden ? n_out : n_hidden) * 2 * sizeof(float));
    e = e ? e : cudaMemcpy(m->params, h.data(), o * sizeof(float), cudaMemcpyHostToDevice);
    e = e ? e : cudaMemset(m->grads, 0, o * sizeof(float));
    e = e ? e : cudaMemset(m->m1, 0, o * sizeof(float));
    e = e ? e : cudaMemset(m->m2, 0, o * sizeof(float));
    if (device != cur) cudaSetDevice(cur);
    if (e != cudaSuccess) {
        cf_set_last_error(cudaGetErrorString(e));
        cudaFree(m->params); cudaFree(m->grads); cudaFree(m->m1); cudaFree(m->m2); cudaFree(m->act); cudaFree(m->scratch);
        delete m;
        return e == cudaErrorMemoryAllocation ? CF_ENOMEM : CF_ECUDA;
    }
    *out = m;
    return CF_OK;
}

int cf_mlp_destroy(cf_mlp* m) {
    if (!m) return CF_OK;
    cudaFree(m->params); cudaFree(m->grads); cudaFree(m->m1); cudaFree(m->m2); cudaFree(m->act); cudaFree(m->scratch);
    delete m;
    return CF_OK;
}

int cf_mlp_num_params(const cf_mlp* m, int64_t* n) {
    if (!m || !n) return CF_EINVAL;
    *n = (int64_t)m->n_params;
    return CF_OK;
}

// Copy parameters (dir = 0: device -> host, 1: host -> device) or gradients (dir = 2: device -> host).
// The flat layout is W1[n_hid][n_in], b1, W2[n_hid][n_hid], b2, W3[n_out][n_hid], b3, each padded to 64.
int cf_mlp_copy(cf_mlp* m, float* host, int32_t dir) {
    if (!m || !host || dir < 0 || dir > 2) return CF_EINVAL;
    const size_t nb = m->n_params * sizeof(float);
    if (dir == 0) MCHECK(cudaMemcpy(host, m->params, nb, cudaMemcpyDeviceToHost));
    if (dir == 1) MCHECK(cudaMemcpy(m->params, host, nb, cudaMemcpyHostToDevice));
    if (dir == 2) MCHECK(cudaMemcpy(host, m->grads, nb, cudaMemcpyDeviceToHost));
    return CF_OK;
}

// y[n][n_out] = net(x[n][n_in]); with train != 0 the activations are kept for cf_mlp_backward.
int cf_mlp_forward(cf_mlp* m, const float* x, float* y, int64_t n, int32_t train, void* stream) {
    if (!m || (n > 0 && (!x || !y))) return CF_EINVAL;
    if (n > m->max_batch) {
        cf_set_last_error("cf_mlp_forward: batch larger than the network's max_batch");
        return CF_ESHAPE;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int H = m->n_hid;
    float* Z1 = m->act;
    float* H1 = Z1 + (size_t)m->max_batch * H;
    float* Z2 = H1 + (size_t)m->max_batch * H;
    float* H2 = Z2 + (size_t)m->max_batch * H;
    int rc;
    rc = gemm<false, true>(s, (int)n, H, m->n_in, x, m->n_in, W(m, 0), m->n_in, H1, H, 1.f, 0.f, W(m, 1), 1,
                           train ? Z1 : nullptr);
    if (rc) return rc;
    rc = gemm<false, true>(s, (int)n, H, H, H1, H, W(m, 2), H, H2, H, 1.f, 0.f, W(m, 3), 1, train ? Z2 : nullptr);
    if (rc) return rc;
    return gemm<false, true>(s, (int)n, m->n_out, H, H2, H, W(m, 4), H, y, m->n_out, 1.f, 0.f, W(m, 5), 0, nullptr);
}

// Gradients of sum(dy * y) for the last training forward pass, given dy[n][n_out]; stored in the
// network's gradient buffer (overwritten).  x must be the same input as in that forward pass.
int cf_mlp_backward(cf_mlp* m, const float* x, const float* dy, int64_t n, void* stream) {
    if (!m || !x || !dy || n < 1 || n > m->max_batch) return CF_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    const int H = m->n_hid, O = m->n_out, I = m->n_in;
    float* Z1 = m->act;
    float* H1 = Z1 + (size_t)m->max_batch * H;
    float* Z2 = H1 + (size_t)m->max_batch * H;
    float* H2 = Z2 + (size_t)m->max_batch * H;
    float* dH2 = m->scratch;
    float* dH1 = m->scratch + (size_t)m->max_batch * (O > H ? O : H);
    int rc;
    // layer 3: dW3 = dy^T H2, db3 = colsum dy, dH2 = dy W3
    rc = gemm<true, false>(s, O, H, (int)n, dy, O, H2, H, dW(m, 4), H, 1.f, 0.f, nullptr, 0, nullptr);
    if (rc) return rc;
    k_colsum<<<(O + 255) / 256, 256, 0, s>>>(dy, dW(m, 5), (int)n, O);
    MCHECK(cudaGetLastError());
    rc = gemm<false, false>(s, (int)n, H, O, dy, O, W(m, 4), H, dH2, H, 1.f, 0.f, nullptr, 0, nullptr);
    if (rc) return rc;
    k_gelu_back<<<grid1d((size_t)n * H), 256, 0, s>>>(dH2, Z2, (size_t)n * H);
    MCHECK(cudaGetLastError());
    // layer 2
    rc = gemm<true, false>(s, H, H, (int)n, dH2, H, H1, H, dW(m, 2), H, 1.f, 0.f, nullptr, 0, nullptr);
    if (rc) return rc;
    k_colsum<<<(H + 255) / 256, 256, 0, s>>>(dH2, dW(m, 3), (int)n, H);
    MCHECK(cudaGetLastError());
    rc = gemm<false, false>(s, (int)n, H, H, dH2, H, W(m, 2), H, dH1, H, 1.f, 0.f, nullptr, 0, nullptr);
    if (rc) return rc;
    k_gelu_back<<<grid1d((size_t)n * H), 256, 0, s>>>(dH1, Z1, (size_t)n * H);
    MCHECK(cudaGetLastError());
    // layer 1
    rc = gemm<true, false>(s, H, I, (int)n, dH1, H, x, I, dW(m, 0), I, 1.f, 0.f, nullptr, 0, nullptr);
    if (rc) return rc;
    k_colsum<<<(H + 255) / 256, 256, 0, s>>>(dH1, dW(m, 1), (int)n, H);
    MCHECK(cudaGetLastError());
    return CF_OK;
}

int cf_mlp_adam_step(cf_mlp* m, float lr, float beta1, float beta2, float eps, float weight_decay, void* stream) {
    if (!m) return CF_EINVAL;
    m->adam_t += 1;
    const float c1 = 1.f - std::pow(beta1, (float)m->adam_t), c2 = 1.f - std::pow(beta2, (float)m->adam_t);
    k_adam<<<grid1d(m->n_params), 256, 0, (cudaStream_t)stream>>>(m->params, m->grads, m->m1, m->m2, m->n_params, lr,
                                                                  beta1, beta2, eps, c1, c2, weight_decay);
    MCHECK(cudaGetLastError());
    return CF_OK;
}

int cf_precond_probe_loss(const float* delta, const double* peq, const float* av, const float* v, const float* vnorm2,
                          float scale, int64_t n, int32_t n_probes, int32_t n_q, int32_t k, float* grad,
                          double* loss_dev, void* stream) {
    if (k < 1 || k > 16 || n < 0 || n_probes < 1 || n_q < 1) return CF_EINVAL;
    if (n == 0) return CF_OK;
    const size_t threads = (size_t)n * n_q;
    k_probe_loss<<<(unsigned)((threads + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
        delta, peq, av, v, vnorm2, scale, (int)n, n_probes, n_q, k, grad, loss_dev);
    MCHECK(cudaGetLastError());
    return CF_OK;
}

int cf_precond_assemble(const float* delta, const double* peq, double* P, float scale, int64_t n, int32_t n_q,
                        int32_t k, void* stream) {
    if (n < 0 || n_q < 1 || k < 1) return CF_EINVAL;
    if (n == 0) return CF_OK;
    k_assemble_precond<<<grid1d((size_t)n * n_q * k * k), 256, 0, (cudaStream_t)stream>>>(delta, peq, P, scale,
                                                                                          (size_t)n, n_q * k * k);
    MCHECK(cudaGetLastError());
    return CF_OK;
}

}  // extern "C"
