// krylov.cu -- batched implicit solves (I - dt J(f)) x = b with restarted GMRES, FP64, on the GPU.
//
// Every cell has its own f, hence its own Jacobian, and its own Krylov space.  All vectors live in
// the tiled cell layout [ceil(B/32)][N_Q*K][32] (lane = cell), so every vector kernel below is a
// coalesced stream with one cell per lane, and a matrix-vector product is one batched J.v launch
// of the contraction library (cf_jv_tiled) plus an axpy.
//
//   * right preconditioning: A P^-1 u = b, x = P^-1 u, so the Arnoldi residual is the true one;
//   * P^-1 is block-Jacobi over the angular modes q: N_Q blocks of K x K, either shared by all
//     cells (the Maxwellian-linearised blocks of I - dt J_eq, tutorial_chapman_enscog_decay_rates.m:42-48
//     generalised) or one set per cell (the learned preconditioner);
//   * classical Gram-Schmidt with one re-orthogonalisation (CGS2), FP64;
//   * Givens rotations per cell; a cell stops extending its Krylov space once its estimated residual
//     reaches tol * |b|, and the restart's true residual b - A x is recomputed in FP64.
//
// The host drives the iteration; each Arnoldi step is a handful of launches on one stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/cf_b200.h"

void cf_set_last_error(const char* msg);

namespace {

constexpr int kLanes = 32;
constexpr int kDotWarps = 8;  // warps per tile in the reduction kernels
constexpr int kVB = 8;        // vectors per register block

// ---------------------------------------------------------------------------------------------
// h[i][cell] = <V_i, w> for i < nv (V_i at V + i * vstride), one CTA per tile, rows split over warps
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kDotWarps * 32) k_dots(const double* __restrict__ V, size_t vstride, int nv,
                                                         const double* __restrict__ w, double* __restrict__ h,
                                                         int M, int n_cells_pad) {
    __shared__ double red[kDotWarps][kVB][kLanes];
    const int tile = blockIdx.x, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const size_t base = (size_t)tile * M * kLanes + lane;
    for (int i0 = 0; i0 < nv; i0 += kVB) {
        const int nb = min(kVB, nv - i0);
        double acc[kVB];
#pragma unroll
        for (int i = 0; i < kVB; ++i) acc[i] = 0.0;
        for (int r = warp; r < M; r += kDotWarps) {
            const double wr = w[base + (size_t)r * kLanes];
#pragma unroll
            for (int i = 0; i < kVB; ++i)
                if (i < nb) acc[i] = fma(V[(size_t)(i0 + i) * vstride + base + (size_t)r * kLanes], wr, acc[i]);
        }
#pragma unroll
        for (int i = 0; i < kVB; ++i) red[warp][i][lane] = acc[i];
        __syncthreads();
        if (warp == 0) {
            for (int i = 0; i < nb; ++i) {
                double s = 0.0;
#pragma unroll
                for (int q = 0; q < kDotWarps; ++q) s += red[q][i][lane];
                h[(size_t)(i0 + i) * n_cells_pad + (size_t)tile * kLanes + lane] = s;
            }
        }
        __syncthreads();
    }
}

// w -= sum_i h[i][cell] V_i (sign = -1) or w += ... (sign = +1)
__global__ void k_combine(double* __restrict__ w, const double* __restrict__ V, size_t vstride, int nv,
                          const double* __restrict__ h, double sign, int M, int n_tiles, int n_cells_pad) {
    const size_t n = (size_t)n_tiles * M * kLanes;
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        const int lane = (int)(idx & 31);
        const size_t tile = idx / ((size_t)M * kLanes);
        const size_t cell = tile * kLanes + lane;
        double s = 0.0;
        for (int i = 0; i < nv; ++i) s = fma(h[(size_t)i * n_cells_pad + cell], V[(size_t)i * vstride + idx], s);
        w[idx] = fma(sign, s, w[idx]);
    }
}

// y = x * scale[cell]
__global__ void k_scale(double* __restrict__ y, const double* __restrict__ x, const double* __restrict__ scale,
                        int M, int n_tiles) {
    const size_t n = (size_t)n_tiles * M * kLanes;
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        const size_t cell = (idx / ((size_t)M * kLanes)) * kLanes + (idx & 31);
        y[idx] = x[idx] * scale[cell];
    }
}

// y = a * x + b * y (uniform scalars)
__global__ void k_axpby(double* __restrict__ y, const double* __restrict__ x, double a, double b, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = fma(a, x[i], b * y[i]);
}

// Block-Jacobi apply: out[q*K .. q*K+K) = P_q in[...] per cell; blocks shared (per_cell = 0) or per cell.
// P is [N_Q][K][K] (row-major k_out, k_in) or [B][N_Q][K][K].
__global__ void k_block_apply(double* __restrict__ out, const double* __restrict__ in, const double* __restrict__ P,
                              int per_cell, int nq, int K, int n_tiles, int n_cells) {
    const size_t n = (size_t)n_tiles * nq * kLanes;
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        const int lane = (int)(idx & 31);
        const size_t tq = idx >> 5;
        const int q = (int)(tq % nq);
        const size_t tile = tq / nq;
        const size_t cell = tile * kLanes + lane;
        const size_t row0 = (tile * nq + q) * K;
        const double* Pq = P + ((per_cell ? (cell < (size_t)n_cells ? cell : 0) * (size_t)nq : 0) + q) * (size_t)K * K;
        for (int a = 0; a < K; ++a) {
            double s = 0.0;
            for (int b = 0; b < K; ++b) s = fma(Pq[a * K + b], in[(row0 + b) * kLanes + lane], s);
            out[(row0 + a) * kLanes + lane] = s;
        }
    }
}

// Per-cell Arnoldi tail: store column j of H, apply the previous Givens rotations, form the new one,
// update the residual estimate and freeze cells that reached tol * |b|.
struct CellState {
    double* H;        // [m+1][m][cells]   H[i][j] at (i*m + j)*cells + c
    double* cs;       // [m][cells]
    double* sn;       // [m][cells]
    double* g;        // [m+1][cells]
    double* bnorm;    // [cells]
    double* inv;      // [cells] 1 / H[j+1][j] (0 when frozen or breakdown)
    int* kdim;        // [cells] Krylov dimension in use (frozen cells keep theirs)
    int* active;      // [cells]
    int* n_active;    // [1]
};

__global__ void k_arnoldi_tail(CellState st, const double* __restrict__ h, const double* __restrict__ hh,
                               const double* __restrict__ wnorm2, int j, int m, int n_cells_pad, double tol) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells_pad) return;
    const size_t C = n_cells_pad;
    if (!st.active[c]) {
        st.inv[c] = 0.0;
        return;
    }
    double col[64];  // m <= 63
    for (int i = 0; i <= j; ++i) col[i] = h[(size_t)i * C + c] + hh[(size_t)i * C + c];
    const double hn = sqrt(fmax(wnorm2[c], 0.0));
    for (int i = 0; i < j; ++i) {
        const double a = col[i], b = col[i + 1];
        const double cs = st.cs[(size_t)i * C + c], sn = st.sn[(size_t)i * C + c];
        col[i] = cs * a + sn * b;
        col[i + 1] = -sn * a + cs * b;
    }
    const double a = col[j], b = hn;
    const double rr = hypot(a, b);
    const double cs = rr > 0 ? a / rr : 1.0, sn = rr > 0 ? b / rr : 0.0;
    col[j] = rr;
    for (int i = 0; i <= j; ++i) st.H[((size_t)i * m + j) * C + c] = col[i];
    st.cs[(size_t)j * C + c] = cs;
    st.sn[(size_t)j * C + c] = sn;
    const double gj = st.g[(size_t)j * C + c];
    st.g[(size_t)j * C + c] = cs * gj;
    st.g[(size_t)(j + 1) * C + c] = -sn * gj;
    st.kdim[c] = j + 1;
    const double res = fabs(sn * gj);
    const bool done = res <= tol * st.bnorm[c] || hn == 0.0 || j + 1 == m;
    st.inv[c] = (hn > 0.0) ? 1.0 / hn : 0.0;
    if (done) {
        st.active[c] = 0;
        if (res <= tol * st.bnorm[c] || hn == 0.0) atomicSub(st.n_active, 1);
    }
}

// y = H^-1 g (back substitution per cell, size kdim), written as coefficients h_out[i][cell]
__global__ void k_solve_y(CellState st, double* __restrict__ y, int m, int n_cells_pad) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells_pad) return;
    const size_t C = n_cells_pad;
    const int k = st.kdim[c];
    double yy[64];
    for (int i = k - 1; i >= 0; --i) {
        double s = st.g[(size_t)i * C + c];
        for (int l = i + 1; l < k; ++l) s -= st.H[((size_t)i * m + l) * C + c] * yy[l];
        const double d = st.H[((size_t)i * m + i) * C + c];
        yy[i] = d != 0.0 ? s / d : 0.0;
    }
    for (int i = 0; i < m; ++i) y[(size_t)i * C + c] = i < k ? yy[i] : 0.0;
}

// start of a cycle: bnorm given, beta = |r|, g = [beta, 0, ...], V0 scale = 1/beta; active = beta > tol*|b|
__global__ void k_cycle_start(CellState st, const double* __restrict__ rnorm2, double* __restrict__ scale, int m,
                              int n_cells_pad, int n_cells, double tol) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells_pad) return;
    const size_t C = n_cells_pad;
    const double beta = sqrt(fmax(rnorm2[c], 0.0));
    for (int i = 0; i <= m; ++i) st.g[(size_t)i * C + c] = 0.0;
    st.g[c] = beta;
    st.kdim[c] = 0;
    const bool act = c < n_cells && beta > tol * st.bnorm[c];
    st.active[c] = act ? 1 : 0;
    scale[c] = act ? 1.0 / beta : 0.0;
    if (act) atomicAdd(st.n_active, 1);
}

__global__ void k_sqrt_copy(double* __restrict__ out, const double* __restrict__ in, int n) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n) out[c] = sqrt(fmax(in[c], 0.0));
}

// relres[cell] = sqrt(rn2) / bnorm, and the count of cells still above tol
__global__ void k_relres(const double* __restrict__ rn2, const double* __restrict__ bnorm, double* __restrict__ rel,
                         int* __restrict__ n_bad, int n_cells, double tol) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells) return;
    const double r = sqrt(fmax(rn2[c], 0.0));
    const double b = bnorm[c];
    const double v = b > 0 ? r / b : r;
    rel[c] = v;
    if (v > tol) atomicAdd(n_bad, 1);
}

__global__ void k_add_iters(int* __restrict__ iters, const int* __restrict__ kdim, int n_cells) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n_cells) iters[c] += kdim[c];
}

int grid_for(size_t n, int threads = 256) {
    size_t g = (n + threads - 1) / threads;
    return (int)std::min<size_t>(g, 148 * 32);
}

#define KCHECK(expr)                                                                                      \
    do {                                                                                                  \
        cudaError_t e_ = (expr);                                                                          \
        if (e_ != cudaSuccess) {                                                                          \
            char m_[256];                                                                                 \
            snprintf(m_, sizeof(m_), "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
            cf_set_last_error(m_);                                                                        \
            return e_ == cudaErrorMemoryAllocation ? CF_ENOMEM : CF_ECUDA;                                \
        }                                                                                                 \
    } while (0)

#define KLAUNCH() KCHECK(cudaGetLastError())

}  // namespace

extern "C" int cf_gmres_workspace_size(const cf_plan* plan, int64_t b, int32_t restart, size_t* bytes) {
    if (!plan || !bytes || b < 0 || restart < 1 || restart > 63) return CF_EINVAL;
    cf_plan_info info;
    int st = cf_plan_get_info(plan, &info);
    if (st != CF_OK) return st;
    const size_t nt = (size_t)((b + kLanes - 1) / kLanes);
    const size_t vec = nt * kLanes * (size_t)info.n_q * info.k;  // doubles per vector
    const size_t C = nt * kLanes;
    const size_t m = (size_t)restart;
    size_t d = vec * (m + 1)      // V
               + vec * 3          // w, z, r
               + C * (m + 1) * m  // H
               + C * m * 2        // cs, sn
               + C * (m + 1)      // g
               + C * (m + 1) * 3  // h, hh, y
               + C * 6;           // bnorm, inv, scale, norms, rel
    *bytes = d * sizeof(double) + C * 3 * sizeof(int) + 64 * sizeof(int) + 32 * 256;  // + alignment of 25 pieces
    return CF_OK;
}

extern "C" int cf_gmres_solve_tiled(cf_plan* plan, const double* f_t, double dt, const double* b_t, double* x_t,
                                    int64_t b, int32_t restart, int32_t max_iters, double tol,
                                    const double* precond, int32_t precond_per_cell, int32_t* iters_out,
                                    double* relres_out, void* workspace, size_t workspace_bytes, void* stream) {
    if (!plan || (b > 0 && (!f_t || !b_t || !x_t))) {
        cf_set_last_error("cf_gmres_solve_tiled: null argument");
        return CF_EINVAL;
    }
    if (restart < 1 || restart > 63 || max_iters < 1 || !(tol > 0)) {
        cf_set_last_error("cf_gmres_solve_tiled: restart must be in [1, 63], max_iters >= 1, tol > 0");
        return CF_EINVAL;
    }
    if (b == 0) return CF_OK;
    cf_plan_info info;
    int st = cf_plan_get_info(plan, &info);
    if (st != CF_OK) return st;
    size_t need = 0;
    st = cf_gmres_workspace_size(plan, b, restart, &need);
    if (st != CF_OK) return st;
    if (!workspace || workspace_bytes < need) {
        char msg[160];
        snprintf(msg, sizeof(msg), "cf_gmres_solve_tiled: workspace of %zu bytes, %zu needed", workspace_bytes, need);
        cf_set_last_error(msg);
        return CF_EINVAL;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int M = info.n_q * info.k;
    const int nt = (int)((b + kLanes - 1) / kLanes);
    const size_t C = (size_t)nt * kLanes;
    const size_t vec = C * M;
    const int m = restart;
    const int n_cells = (int)b;

    // carve the workspace
    char* p = (char*)workspace;
    auto take = [&](size_t nbytes) {
        char* q = p;
        p += (nbytes + 255) & ~size_t(255);
        return q;
    };
    double* V = (double*)take(vec * (m + 1) * sizeof(double));
    double* w = (double*)take(vec * sizeof(double));
    double* z = (double*)take(vec * sizeof(double));
    double* r = (double*)take(vec * sizeof(double));
    CellState cs;
    cs.H = (double*)take(C * (m + 1) * m * sizeof(double));
    cs.cs = (double*)take(C * m * sizeof(double));
    cs.sn = (double*)take(C * m * sizeof(double));
    cs.g = (double*)take(C * (m + 1) * sizeof(double));
    double* h = (double*)take(C * (m + 1) * sizeof(double));
    double* hh = (double*)take(C * (m + 1) * sizeof(double));
    double* y = (double*)take(C * (m + 1) * sizeof(double));
    cs.bnorm = (double*)take(C * sizeof(double));
    cs.inv = (double*)take(C * sizeof(double));
    double* scale = (double*)take(C * sizeof(double));
    double* norm2 = (double*)take(C * sizeof(double));
    double* rel = (double*)take(C * sizeof(double));
    cs.kdim = (int*)take(C * sizeof(int));
    cs.active = (int*)take(C * sizeof(int));
    int* iters = (int*)take(C * sizeof(int));
    cs.n_active = (int*)take(64 * sizeof(int));
    int* n_bad = cs.n_active + 16;
    if ((size_t)(p - (char*)workspace) > workspace_bytes) {
        cf_set_last_error("cf_gmres_solve_tiled: internal workspace layout overflow");
        return CF_EINVAL;
    }

    const int gv = grid_for(vec);
    const int gc = (int)((C + 255) / 256);
    KCHECK(cudaMemsetAsync(iters, 0, C * sizeof(int), s));

    // A u = u - dt * J(f) u, preconditioned operand z = P^-1 u.  J(f) u runs on the q2 <-> q3 folded
    // operator (the same bilinear form on half the entries) when the operator folds, else on the
    // plain one.
    int jv_mode = 2;
    auto apply_A = [&](double* out, const double* u) -> int {
        KCHECK(cudaMemsetAsync(out, 0, vec * sizeof(double), s));
        int rc = cf_jv_tiled(plan, out, f_t, u, b, jv_mode, s);
        if (rc == CF_EUNSUPPORTED && jv_mode == 2) {
            jv_mode = 0;
            cf_set_last_error("");
            rc = cf_jv_tiled(plan, out, f_t, u, b, jv_mode, s);
        }
        if (rc != CF_OK) return rc;
        k_axpby<<<gv, 256, 0, s>>>(out, u, 1.0, -dt, vec);
        KLAUNCH();
        return CF_OK;
    };
    auto apply_P = [&](double* out, const double* in) -> int {
        if (!precond) {
            KCHECK(cudaMemcpyAsync(out, in, vec * sizeof(double), cudaMemcpyDeviceToDevice, s));
            return CF_OK;
        }
        k_block_apply<<<grid_for(C * info.n_q), 256, 0, s>>>(out, in, precond, precond_per_cell, info.n_q, info.k, nt,
                                                            n_cells);
        KLAUNCH();
        return CF_OK;
    };
    auto norms2 = [&](const double* v, double* out) -> int {
        k_dots<<<nt, kDotWarps * 32, 0, s>>>(v, 0, 1, v, out, M, (int)C);
        KLAUNCH();
        return CF_OK;
    };

    // |b| per cell
    int rc = norms2(b_t, norm2);
    if (rc) return rc;
    k_sqrt_copy<<<gc, 256, 0, s>>>(cs.bnorm, norm2, (int)C);
    KLAUNCH();

    int total = 0;
    int host_bad = n_cells;
    for (;;) {
        // true residual r = b - A x, per-cell relative residual, count of cells above tol
        rc = apply_A(r, x_t);
        if (rc) return rc;
        k_axpby<<<gv, 256, 0, s>>>(r, b_t, 1.0, -1.0, vec);
        KLAUNCH();
        rc = norms2(r, norm2);
        if (rc) return rc;
        KCHECK(cudaMemsetAsync(n_bad, 0, sizeof(int), s));
        k_relres<<<gc, 256, 0, s>>>(norm2, cs.bnorm, rel, n_bad, n_cells, tol);
        KLAUNCH();
        KCHECK(cudaMemcpyAsync(&host_bad, n_bad, sizeof(int), cudaMemcpyDeviceToHost, s));
        KCHECK(cudaStreamSynchronize(s));
        if (host_bad == 0 || total >= max_iters) break;

        // new cycle: V0 = r / |r| for the cells above tol
        KCHECK(cudaMemsetAsync(cs.n_active, 0, sizeof(int), s));
        k_cycle_start<<<gc, 256, 0, s>>>(cs, norm2, scale, m, (int)C, n_cells, tol);
        KLAUNCH();
        k_scale<<<gv, 256, 0, s>>>(V, r, scale, M, nt);
        KLAUNCH();
        int host_active = 0;
        for (int j = 0; j < m && total < max_iters; ++j, ++total) {
            double* Vj = V + (size_t)j * vec;
            rc = apply_P(z, Vj);
            if (rc) return rc;
            rc = apply_A(w, z);
            if (rc) return rc;
            // classical Gram-Schmidt, twice
            k_dots<<<nt, kDotWarps * 32, 0, s>>>(V, vec, j + 1, w, h, M, (int)C);
            KLAUNCH();
            k_combine<<<gv, 256, 0, s>>>(w, V, vec, j + 1, h, -1.0, M, nt, (int)C);
            KLAUNCH();
            k_dots<<<nt, kDotWarps * 32, 0, s>>>(V, vec, j + 1, w, hh, M, (int)C);
            KLAUNCH();
            k_combine<<<gv, 256, 0, s>>>(w, V, vec, j + 1, hh, -1.0, M, nt, (int)C);
            KLAUNCH();
            rc = norms2(w, norm2);
            if (rc) return rc;
            k_arnoldi_tail<<<gc, 256, 0, s>>>(cs, h, hh, norm2, j, m, (int)C, tol);
            KLAUNCH();
            k_scale<<<gv, 256, 0, s>>>(V + (size_t)(j + 1) * vec, w, cs.inv, M, nt);
            KLAUNCH();
            if ((j & 3) == 3) {
                KCHECK(cudaMemcpyAsync(&host_active, cs.n_active, sizeof(int), cudaMemcpyDeviceToHost, s));
                KCHECK(cudaStreamSynchronize(s));
                if (host_active <= 0) {
                    ++total;
                    break;
                }
            }
        }
        // x += P^-1 (V y), y from each cell's own Krylov dimension
        k_solve_y<<<gc, 256, 0, s>>>(cs, y, m, (int)C);
        KLAUNCH();
        k_add_iters<<<gc, 256, 0, s>>>(iters, cs.kdim, n_cells);
        KLAUNCH();
        KCHECK(cudaMemsetAsync(w, 0, vec * sizeof(double), s));
        k_combine<<<gv, 256, 0, s>>>(w, V, vec, m, y, 1.0, M, nt, (int)C);
        KLAUNCH();
        rc = apply_P(z, w);
        if (rc) return rc;
        k_axpby<<<gv, 256, 0, s>>>(x_t, z, 1.0, 1.0, vec);
        KLAUNCH();
    }
    if (iters_out) KCHECK(cudaMemcpyAsync(iters_out, iters, (size_t)n_cells * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (relres_out) KCHECK(cudaMemcpyAsync(relres_out, rel, (size_t)n_cells * sizeof(double), cudaMemcpyDeviceToHost, s));
    KCHECK(cudaStreamSynchronize(s));
    if (host_bad > 0) {
        char msg[160];
        snprintf(msg, sizeof(msg), "cf_gmres_solve_tiled: %d of %d cells above tol after %d iterations", host_bad,
                 n_cells, total);
        cf_set_last_error(msg);
        return CF_ETIMEOUT;
    }
    return CF_OK;
}
