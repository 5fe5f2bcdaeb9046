// stepping.cu -- batched explicit time stepping df/dt = Q(f) with Heun's method (RK2), on the GPU.
//
// The reference steps one cell with a dense tensor, c <- c + dt/2 (C(c,c) + C(ct,ct)),
// ct = c + dt C(c,c) (tutorial_stress_relaxation.m:77-91, tutorial_collisions_bwu_solution.m:77-92).
// Here every cell of a batch steps at once with the factorised operator: the state stays in the
// tiled cell layout [ceil(B/32)][N_Q*K][32] between steps, each stage is one contraction launch of
// the library (cf_q_tiled) into a zeroed buffer, and the two vector updates are one coalesced pass
// each.  A step makes no allocation, no host synchronisation and no host read, so a caller can
// record n steps into a CUDA graph and replay them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>

#include "../../include/cf_b200.h"

void cf_set_last_error(const char* msg);

namespace {

// ft = f + dt * q1
__global__ void k_stage(double* __restrict__ ft, const double* __restrict__ f, const double* __restrict__ q1,
                        double dt, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        ft[i] = fma(dt, q1[i], f[i]);
}

// f += (dt / 2) * (q1 + q2)
__global__ void k_finish(double* __restrict__ f, const double* __restrict__ q1, const double* __restrict__ q2,
                         double half_dt, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        f[i] = fma(half_dt, q1[i] + q2[i], f[i]);
}

int grid_for(size_t n) { return (int)std::min<size_t>((n + 255) / 256, (size_t)148 * 8); }

#define SCHECK(expr)                                                                                    \
    do {                                                                                                \
        cudaError_t e_ = (expr);                                                                        \
        if (e_ != cudaSuccess) {                                                                        \
            char m_[256];                                                                               \
            snprintf(m_, sizeof(m_), "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
            cf_set_last_error(m_);                                                                      \
            return CF_ECUDA;                                                                            \
        }                                                                                               \
    } while (0)

size_t tiled_doubles(const cf_plan_info& info, int64_t b) {
    return (size_t)((b + 31) / 32) * 32 * (size_t)info.n_q * info.k;
}

}  // namespace

extern "C" {

int cf_rk2_workspace_size(const cf_plan* plan, int64_t b, size_t* bytes) {
    if (!plan || !bytes || b < 0) return CF_EINVAL;
    cf_plan_info info;
    const int st = cf_plan_get_info(plan, &info);
    if (st != CF_OK) return st;
    *bytes = 3 * tiled_doubles(info, b) * sizeof(double);  // q1, q2, ft
    return CF_OK;
}

int cf_rk2_steps_tiled(cf_plan* plan, double* f_tiled, int64_t b, double dt, int32_t n_steps, int32_t form,
                       void* workspace, size_t workspace_bytes, void* stream) {
    if (!plan || !f_tiled || b < 0 || n_steps < 0) return CF_EINVAL;
    if (b == 0 || n_steps == 0) return CF_OK;
    size_t need = 0;
    int st = cf_rk2_workspace_size(plan, b, &need);
    if (st != CF_OK) return st;
    if (!workspace || workspace_bytes < need) {
        cf_set_last_error("cf_rk2_steps_tiled: workspace smaller than cf_rk2_workspace_size");
        return CF_EINVAL;
    }
    cf_plan_info info;
    cf_plan_get_info(plan, &info);
    const size_t n = tiled_doubles(info, b);
    double* q1 = static_cast<double*>(workspace);
    double* q2 = q1 + n;
    double* ft = q2 + n;
    cudaStream_t s = (cudaStream_t)stream;
    const int g = grid_for(n);
    for (int i = 0; i < n_steps; ++i) {
        SCHECK(cudaMemsetAsync(q1, 0, n * sizeof(double), s));
        st = cf_q_tiled(plan, q1, f_tiled, b, form, stream);
        if (st != CF_OK) return st;
        k_stage<<<g, 256, 0, s>>>(ft, f_tiled, q1, dt, n);
        SCHECK(cudaGetLastError());
        SCHECK(cudaMemsetAsync(q2, 0, n * sizeof(double), s));
        st = cf_q_tiled(plan, q2, ft, b, form, stream);
        if (st != CF_OK) return st;
        k_finish<<<g, 256, 0, s>>>(f_tiled, q1, q2, 0.5 * dt, n);
        SCHECK(cudaGetLastError());
    }
    return CF_OK;
}

}  // extern "C"
