// tile_kernels.cuh -- tile-resident angular-first kernels (persistent, device work queue).
//
// A CTA keeps the f (and, for J.v, the v) coefficients of a 16-cell half-tile resident in shared
// memory and its W warps contract every q1 of those cells out of it:
//
//   * one warp per q1; each cell is handled by two lanes (lane = 16*part + cell) that split the
//     K x K Phi accumulator by k3 column, so the f2 row is a broadcast between the two halves and a
//     lane holds K*K/2 accumulators;
//   * per (t, q1) slice the warp copies R_t into its own shared buffer with cp.async while it
//     accumulates Phi, so the K^3 step reads R from shared memory (k3 slices padded by two doubles
//     so the two lane halves hit different banks);
//   * CTAs are persistent and pull work units from a device counter: whole half-tiles first, then
//     half-tiles split into q1 bins, so the last wave is made of small units.  Inside a unit the
//     warps pull q1 values (heaviest first) from a shared counter.
//
// The counter is the only inter-CTA interaction; nothing waits on another CTA.  The streamed
// variant at the end also waits, with a bound, on flags that the host's copies set.
#pragma once
#include "common.cuh"

namespace cf {

constexpr int kTileCells = 16;

struct TileSched {
    const int* bin_begin;  // bin b = q1 list bin_q1[bin_begin[b] .. bin_begin[b+1])
    const int* bin_q1;     // bin 0: every q1, heaviest first; bins 1..4: quarters; bins 5..20: sixteenths
    int n_ht;              // half-tiles: ceil(B / 16)
    int n_whole;           // units [0, n_whole) are whole half-tiles
    int split;             // later units split a half-tile into `split` bins (4 or 16)
    int n_units;
    int* counter;          // zeroed before the launch
};

__host__ __device__ constexpr int bin_base(int split) { return split == 4 ? 1 : 5; }

template <int K>
struct RBuf {
    static constexpr int SL = K * K + 2;  // padded k3 slice (keeps 16-byte alignment for even K)
    static constexpr int SIZE = K * SL;
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Offset of Q[q1][k1] from a lane's cell: tiled rows (stride CF_TILE) or, with CELL_MAJOR, the
// caller's [N_Q x K x B] layout (qtc then points at the cell's first element).
template <int K, bool CELL_MAJOR>
__device__ __forceinline__ size_t q_off(int q1, int k1, int n_q) {
    return CELL_MAJOR ? (size_t)q1 + (size_t)k1 * n_q : (size_t)(q1 * K + k1) * CF_TILE;
}

// Contract every slice of one q1 for the resident half-tile.  qtc points at this lane's cell of
// the output; the result is accumulated into it (out += ...).  live = false: the lane's cell is
// past the end of the batch (cell-major output only), and Q is neither read nor written.
template <int K, bool EXACT, bool JV, bool CELL_MAJOR = false>
__device__ __forceinline__ void tile_q1(const DevOp& op, int q1, const double* __restrict__ fs,
                                        const double* __restrict__ vs, double* rb, double* qtc, int lane,
                                        bool live = true) {
    constexpr int KC = K / 2;
    constexpr int SL = RBuf<K>::SL;
    const int c = lane & 15;
    const int part = lane >> 4;
    const int k3b = part * KC;
    const int owner = EXACT ? 1 : 0;  // the lane half that holds the caller's Q and writes it back

    double acc[K];
#pragma unroll
    for (int k1 = 0; k1 < K; ++k1)
        acc[k1] = (part == owner && live) ? qtc[q_off<K, CELL_MAJOR>(q1, k1, op.n_q)] : 0.0;

    const int s0 = op.q1_begin[q1], s1 = op.q1_begin[q1 + 1];
    for (int s = s0; s < s1; ++s) {
        const int t = op.slice_t[s];
        const int e0 = op.slice_e[s], e1 = op.slice_e[s + 1];
        // stage R_t (K^3 doubles) into this warp's padded buffer while Phi accumulates
        __syncwarp();
        const double* __restrict__ Rt = op.R + (size_t)t * K * K * K;
        for (int i = lane; i < K * K * K / 2; i += 32) {
            const int j = (2 * i) / (K * K), w = (2 * i) % (K * K);
            cp_async16(rb + j * SL + w, Rt + 2 * i);
        }
        cp_async_commit();

        double phi[K][KC];
#pragma unroll
        for (int a = 0; a < K; ++a)
#pragma unroll
            for (int b = 0; b < KC; ++b) phi[a][b] = 0.0;

        bool phi_done = false;
        if constexpr (!EXACT) {
            if (op.grouped & (JV ? 2 : 1)) {
                // entries sorted by q2: over a run of equal q2, hf = sum G f(q3) (and, for J.v,
                // hv = sum G v(q3)); then Phi += f(q2) (x) hf (J.v: v(q2) (x) hf + f(q2) (x) hv) once
                // per run -- the q2 loads and the K x K/2 FMAs once per run instead of once per
                // entry (the run index is warp-uniform)
                double hf[KC], hv[KC];
#pragma unroll
                for (int b = 0; b < KC; ++b) hf[b] = hv[b] = 0.0;
                int cur = -1;
                auto flush = [&]() {
                    const int r2 = cur * K;
#pragma unroll
                    for (int k2 = 0; k2 < K; ++k2) {
                        const double f2 = fs[(r2 + k2) * kTileCells + c];
                        if constexpr (JV) {
                            const double v2 = vs[(r2 + k2) * kTileCells + c];
#pragma unroll
                            for (int b = 0; b < KC; ++b) phi[k2][b] = fma(v2, hf[b], fma(f2, hv[b], phi[k2][b]));
                        } else {
#pragma unroll
                            for (int b = 0; b < KC; ++b) phi[k2][b] = fma(f2, hf[b], phi[k2][b]);
                        }
                    }
#pragma unroll
                    for (int b = 0; b < KC; ++b) hf[b] = hv[b] = 0.0;
                };
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
                        const int q2 = (int)(q23 & 0xffffu), r3 = (int)(q23 >> 16) * K + k3b;
                        if (q2 != cur) {
                            if (cur >= 0) flush();
                            cur = q2;
                        }
#pragma unroll
                        for (int b = 0; b < KC; ++b) {
                            hf[b] = fma(g, fs[(r3 + b) * kTileCells + c], hf[b]);
                            if constexpr (JV) hv[b] = fma(g, vs[(r3 + b) * kTileCells + c], hv[b]);
                        }
                    }
                }
                if (cur >= 0) flush();
                phi_done = true;
            }
        }
        for (int eb = e0; eb < e1 && !phi_done; eb += 32) {
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
                const int r2 = (int)(q23 & 0xffffu) * K, r3 = (int)(q23 >> 16) * K + k3b;
                double f2[K], f3[KC];
#pragma unroll
                for (int k = 0; k < K; ++k) f2[k] = fs[(r2 + k) * kTileCells + c];
#pragma unroll
                for (int b = 0; b < KC; ++b) f3[b] = fs[(r3 + b) * kTileCells + c];
                if constexpr (JV) {
                    double v2[K], v3[KC];
#pragma unroll
                    for (int k = 0; k < K; ++k) v2[k] = vs[(r2 + k) * kTileCells + c];
#pragma unroll
                    for (int b = 0; b < KC; ++b) v3[b] = vs[(r3 + b) * kTileCells + c];
                    if constexpr (EXACT) {
#pragma unroll
                        for (int b = 0; b < KC; ++b)
#pragma unroll
                            for (int k2 = 0; k2 < K; ++k2)
                                phi[k2][b] = __dadd_rn(
                                    phi[k2][b],
                                    __dmul_rn(g, __dadd_rn(__dmul_rn(v2[k2], f3[b]), __dmul_rn(f2[k2], v3[b]))));
                    } else {
#pragma unroll
                        for (int b = 0; b < KC; ++b) {
                            const double gf3 = g * f3[b], gv3 = g * v3[b];
#pragma unroll
                            for (int k2 = 0; k2 < K; ++k2) phi[k2][b] = fma(v2[k2], gf3, fma(f2[k2], gv3, phi[k2][b]));
                        }
                    }
                } else if constexpr (EXACT) {
                    double gf2[K];
#pragma unroll
                    for (int k2 = 0; k2 < K; ++k2) gf2[k2] = __dmul_rn(g, f2[k2]);
#pragma unroll
                    for (int b = 0; b < KC; ++b)
#pragma unroll
                        for (int k2 = 0; k2 < K; ++k2) phi[k2][b] = __dadd_rn(phi[k2][b], __dmul_rn(gf2[k2], f3[b]));
                } else {
#pragma unroll
                    for (int b = 0; b < KC; ++b) {
                        const double gf3 = g * f3[b];
#pragma unroll
                        for (int k2 = 0; k2 < K; ++k2) phi[k2][b] = fma(f2[k2], gf3, phi[k2][b]);
                    }
                }
            }
        }
        cp_async_wait_all();
        __syncwarp();

        // K^3 step from the shared copy of R_t: element (k1,k2,k3) at rb[k3*SL + k2*K + k1]
        if constexpr (EXACT) {
            // the reference sums k3 = 0..K-1 (outer), k2 (inner) sequentially: half 0 sums its columns,
            // hands the partial to half 1, which continues with its columns
            double sp[K];
            if (part == 0) {
#pragma unroll
                for (int k1 = 0; k1 < K; ++k1) {
                    double sacc = 0.0;
#pragma unroll
                    for (int b = 0; b < KC; ++b)
#pragma unroll
                        for (int k2 = 0; k2 < K; ++k2) sacc = __dadd_rn(sacc, __dmul_rn(rb[b * SL + k2 * K + k1], phi[k2][b]));
                    sp[k1] = sacc;
                }
            }
#pragma unroll
            for (int k1 = 0; k1 < K; ++k1) sp[k1] = __shfl_up_sync(0xffffffffu, sp[k1], 16);
            if (part == 1) {
#pragma unroll
                for (int k1 = 0; k1 < K; ++k1) {
                    double sacc = sp[k1];
#pragma unroll
                    for (int b = 0; b < KC; ++b)
#pragma unroll
                        for (int k2 = 0; k2 < K; ++k2)
                            sacc = __dadd_rn(sacc, __dmul_rn(rb[(KC + b) * SL + k2 * K + k1], phi[k2][b]));
                    acc[k1] = __dadd_rn(acc[k1], sacc);
                }
            }
        } else {
            const double* __restrict__ rk = rb + k3b * SL;
#pragma unroll
            for (int b = 0; b < KC; ++b) {
#pragma unroll
                for (int k2 = 0; k2 < K; ++k2) {
                    const double2* r2v = reinterpret_cast<const double2*>(rk + b * SL + k2 * K);
#pragma unroll
                    for (int h = 0; h < K / 2; ++h) {
                        const double2 r = r2v[h];
                        acc[2 * h] = fma(r.x, phi[k2][b], acc[2 * h]);
                        acc[2 * h + 1] = fma(r.y, phi[k2][b], acc[2 * h + 1]);
                    }
                }
            }
        }
    }

    if constexpr (!EXACT) {
#pragma unroll
        for (int k1 = 0; k1 < K; ++k1) acc[k1] += __shfl_xor_sync(0xffffffffu, acc[k1], 16);
    }
    if (part == owner && live) {
#pragma unroll
        for (int k1 = 0; k1 < K; ++k1) qtc[q_off<K, CELL_MAJOR>(q1, k1, op.n_q)] = acc[k1];
    }
}

template <int K, int W, bool EXACT, bool JV>
__global__ void __launch_bounds__(W * 32, 1)
    af_tile_kernel(DevOp op, TileSched sc, const double* __restrict__ fT, const double* __restrict__ vT,
                   double* __restrict__ QT) {
    static_assert(K % 2 == 0, "the tile kernel splits Phi into two column halves");
    extern __shared__ __align__(16) double smem[];
    __shared__ int s_unit, s_next;
    const int M = op.n_q * K;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    double* fs = smem;
    double* vs = JV ? smem + (size_t)M * kTileCells : nullptr;
    double* rb = smem + (size_t)(JV ? 2 : 1) * M * kTileCells + (size_t)warp * RBuf<K>::SIZE;
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
            // rows of 16 cells (128 B) from the tiled global layout, 8 x 16-byte copies per row
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
            tile_q1<K, EXACT, JV>(op, sc.bin_q1[b0 + i], fs, vs, rb, qtc, lane);
        }
        __syncthreads();
    }
}

template <int K>
constexpr size_t tile_smem_bytes(int M, int W, bool jv) {
    return sizeof(double) * ((size_t)(jv ? 2 : 1) * M * kTileCells + (size_t)W * RBuf<K>::SIZE);
}

// ------------------------------------------------------------------------------------------
// Quarter-tile kernels: 8 cells of f (and, for J.v, of v) resident per CTA, 4 lanes per cell that
// split the K x K Phi accumulator by k3 quarter -- for the shapes whose 16-cell tile does not fit in
// shared memory (at K = 8: Q from L = 12 on, J.v from L = 10 on).  The routine is the tile routine's
// with 4 lane groups instead of 2; fast forms only.  An 8-cell row is 64 bytes, half of the banks,
// so rows are stored pairwise swapped (row r at r ^ ((r >> 1) & 1)): the four lane groups' f(q3)
// rows r, r + 2, r + 4, r + 6 then fall into both halves and cost 2 wavefronts, not 4.
// ------------------------------------------------------------------------------------------
constexpr int kQuarterCells = 8;

__device__ __forceinline__ int qrow(int r) { return r ^ ((r >> 1) & 1); }

template <int K, bool JV>
__device__ __forceinline__ void tile4_q1(const DevOp& op, int q1, const double* __restrict__ fs,
                                         const double* __restrict__ vs, double* rb, double* qtc, int lane) {
    static_assert(K % 4 == 0, "the quarter-tile routine splits Phi into four column quarters");
    constexpr int KC = K / 4;
    constexpr int SL = RBuf<K>::SL;
    constexpr int QC = kQuarterCells;
    const int c = lane & 7;
    const int part = lane >> 3;
    const int k3b = part * KC;

    double acc[K];
#pragma unroll
    for (int k1 = 0; k1 < K; ++k1) acc[k1] = part == 0 ? qtc[(size_t)(q1 * K + k1) * CF_TILE] : 0.0;

    const int s0 = op.q1_begin[q1], s1 = op.q1_begin[q1 + 1];
    for (int s = s0; s < s1; ++s) {
        const int t = op.slice_t[s];
        const int e0 = op.slice_e[s], e1 = op.slice_e[s + 1];
        __syncwarp();
        const double* __restrict__ Rt = op.R + (size_t)t * K * K * K;
        for (int i = lane; i < K * K * K / 2; i += 32) {
            const int j = (2 * i) / (K * K), w = (2 * i) % (K * K);
            cp_async16(rb + j * SL + w, Rt + 2 * i);
        }
        cp_async_commit();

        double phi[K][KC];
#pragma unroll
        for (int a = 0; a < K; ++a)
#pragma unroll
            for (int b = 0; b < KC; ++b) phi[a][b] = 0.0;

        const bool grouped = op.grouped & (JV ? 2 : 1);
        double hf[KC], hv[KC];
#pragma unroll
        for (int b = 0; b < KC; ++b) hf[b] = hv[b] = 0.0;
        int cur = -1;
        auto flush = [&]() {
#pragma unroll
            for (int k2 = 0; k2 < K; ++k2) {
                const double f2 = fs[qrow(cur * K + k2) * QC + c];
                if constexpr (JV) {
                    const double v2 = vs[qrow(cur * K + k2) * QC + c];
#pragma unroll
                    for (int b = 0; b < KC; ++b) phi[k2][b] = fma(v2, hf[b], fma(f2, hv[b], phi[k2][b]));
                } else {
#pragma unroll
                    for (int b = 0; b < KC; ++b) phi[k2][b] = fma(f2, hf[b], phi[k2][b]);
                }
            }
#pragma unroll
            for (int b = 0; b < KC; ++b) hf[b] = hv[b] = 0.0;
        };
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
                const int q2 = (int)(q23 & 0xffffu), r3 = (int)(q23 >> 16) * K + k3b;
                double f3[KC], v3[KC];
#pragma unroll
                for (int b = 0; b < KC; ++b) {
                    f3[b] = fs[qrow(r3 + b) * QC + c];
                    if constexpr (JV) v3[b] = vs[qrow(r3 + b) * QC + c];
                }
                if (grouped) {
                    // entries sorted by q2: sum G f(q3) (and G v(q3)) over the run, one outer product per run
                    if (q2 != cur) {
                        if (cur >= 0) flush();
                        cur = q2;
                    }
#pragma unroll
                    for (int b = 0; b < KC; ++b) {
                        hf[b] = fma(g, f3[b], hf[b]);
                        if constexpr (JV) hv[b] = fma(g, v3[b], hv[b]);
                    }
                } else {
                    const int r2 = q2 * K;
#pragma unroll
                    for (int k2 = 0; k2 < K; ++k2) {
                        const double f2 = fs[qrow(r2 + k2) * QC + c];
                        if constexpr (JV) {
                            const double v2 = vs[qrow(r2 + k2) * QC + c];
#pragma unroll
                            for (int b = 0; b < KC; ++b) phi[k2][b] = fma(v2, g * f3[b], fma(f2, g * v3[b], phi[k2][b]));
                        } else {
#pragma unroll
                            for (int b = 0; b < KC; ++b) phi[k2][b] = fma(f2, g * f3[b], phi[k2][b]);
                        }
                    }
                }
            }
        }
        if (grouped && cur >= 0) flush();
        cp_async_wait_all();
        __syncwarp();

        // K^3 step: this lane's k3 quarter; element (k1,k2,k3) at rb[k3*SL + k2*K + k1]
        const double* __restrict__ rk = rb + k3b * SL;
#pragma unroll
        for (int b = 0; b < KC; ++b) {
#pragma unroll
            for (int k2 = 0; k2 < K; ++k2) {
                const double2* r2v = reinterpret_cast<const double2*>(rk + b * SL + k2 * K);
#pragma unroll
                for (int h = 0; h < K / 2; ++h) {
                    const double2 r = r2v[h];
                    acc[2 * h] = fma(r.x, phi[k2][b], acc[2 * h]);
                    acc[2 * h + 1] = fma(r.y, phi[k2][b], acc[2 * h + 1]);
                }
            }
        }
    }
#pragma unroll
    for (int k1 = 0; k1 < K; ++k1) {
        acc[k1] += __shfl_xor_sync(0xffffffffu, acc[k1], 8);
        acc[k1] += __shfl_xor_sync(0xffffffffu, acc[k1], 16);
    }
    if (part == 0) {
#pragma unroll
        for (int k1 = 0; k1 < K; ++k1) qtc[(size_t)(q1 * K + k1) * CF_TILE] = acc[k1];
    }
}

template <int K, int W, bool JV>
__global__ void __launch_bounds__(W * 32, 1)
    af_tile4_kernel(DevOp op, TileSched sc, const double* __restrict__ fT, const double* __restrict__ vT,
                    double* __restrict__ QT) {
    extern __shared__ __align__(16) double smem[];
    __shared__ int s_unit, s_next;
    constexpr int QC = kQuarterCells;
    const int M = op.n_q * K;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    double* fs = smem;
    double* vs = JV ? smem + (size_t)M * QC : nullptr;
    double* rb = smem + (size_t)(JV ? 2 : 1) * M * QC + (size_t)warp * RBuf<K>::SIZE;
    int staged = -1;
    for (;;) {
        if (tid == 0) s_unit = atomicAdd(sc.counter, 1);
        __syncthreads();
        const int u = s_unit;
        if (u >= sc.n_units) break;
        int qt, bin;
        if (u < sc.n_whole) {
            qt = u;
            bin = 0;
        } else {
            const int v = u - sc.n_whole;
            qt = sc.n_whole + v / sc.split;
            bin = bin_base(sc.split) + v % sc.split;
        }
        // quarter qt of the tiled layout: tile qt / 4, cells 8 (qt % 4) .. + 7
        const size_t tile_base = (size_t)(qt >> 2) * M * CF_TILE + (size_t)(qt & 3) * QC;
        if (qt != staged) {
            // rows of 8 cells (64 B), 4 x 16-byte copies per row, to the row's swapped slot
            for (int i = tid; i < M * 4; i += W * 32) {
                const int r = i >> 2, w = (i & 3) * 2;
                cp_async16(fs + qrow(r) * QC + w, fT + tile_base + (size_t)r * CF_TILE + w);
                if constexpr (JV) cp_async16(vs + qrow(r) * QC + w, vT + tile_base + (size_t)r * CF_TILE + w);
            }
            cp_async_commit();
            cp_async_wait_all();
            staged = qt;
        }
        if (tid == 0) s_next = 0;
        __syncthreads();
        const int b0 = sc.bin_begin[bin], nb = sc.bin_begin[bin + 1] - b0;
        double* qtc = QT + tile_base + (lane & 7);
        for (;;) {
            int i = 0;
            if (lane == 0) i = atomicAdd(&s_next, 1);
            i = __shfl_sync(0xffffffffu, i, 0);
            if (i >= nb) break;
            tile4_q1<K, JV>(op, sc.bin_q1[b0 + i], fs, vs, rb, qtc, lane);
        }
        __syncthreads();
    }
}

template <int K>
constexpr size_t tile4_smem_bytes(int M, int W, bool jv) {
    return sizeof(double) * ((size_t)(jv ? 2 : 1) * M * kQuarterCells + (size_t)W * RBuf<K>::SIZE);
}

// ------------------------------------------------------------------------------------------
// Tile kernel on the caller's cell-major f and Q.  Resident (ss.ready == null): the device entry
// points, no layout passes, the tile kernel's schedule.  Streamed (host entry points): one launch
// over the whole batch while the batch is still being copied in and the results copied out.
//
// f and Q stay in the caller's cell-major layout [N_Q x K x B] in device memory.  The host cuts
// the batch into chunks of whole half-tiles and queues, on a copy stream, each chunk's f and Q
// uploads followed by a 4-byte copy that sets ready[c] = epoch.  Every half-tile is split into
// `split` q1 bins, so the first chunk already gives work to every CTA.  A CTA waits for its
// chunk's flag (bounded by wait_cycles of the SM clock; past that it records err and abort, and
// every later wait returns at once),
// stages the 16 cells from the cell-major rows, and contracts its bin with the same per-row code
// as the tile kernel, reading Q_in and writing Q_out in place: the same operations in the same
// order as the tiled kernel, hence the same bits.  After a unit every thread fences and the CTA
// counts the unit in done[c]; the CTA that completes chunk c fences at system scope and writes
// epoch into host_done[c], a word of mapped pinned host memory the host polls before queueing the
// chunk's download.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <int K, int W>
__global__ void __launch_bounds__(W * 32, 1)
    af_tile_stream_kernel(DevOp op, TileSched sc, StreamSync ss, const double* __restrict__ f, double* q,
                          long long n_cells) {
    static_assert(K % 2 == 0, "the tile kernel splits Phi into two column halves");
    extern __shared__ __align__(16) double smem[];
    __shared__ int s_unit, s_next;
    const int M = op.n_q * K;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    double* fs = smem;
    double* rb = smem + (size_t)M * kTileCells + (size_t)warp * RBuf<K>::SIZE;
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
        const int chunk = ht / ss.ht_per_chunk;
        const long long cell0 = (long long)ht * kTileCells;
        if (ht != staged) {
            if (tid == 0 && ss.ready) {
                const long long t0 = clock64();
                while (ld_acquire(ss.ready + chunk) != ss.epoch) {
                    if (*reinterpret_cast<volatile int*>(ss.abort) == ss.epoch) break;
                    if (clock64() - t0 > ss.wait_cycles) {
                        *reinterpret_cast<volatile int*>(ss.abort) = ss.epoch;
                        *reinterpret_cast<volatile int*>(ss.err) = 1;
                        break;
                    }
                    __nanosleep(256);
                }
            }
            __syncthreads();
            // element j = q + N_Q k of cell c (cell-major) goes to row q K + k of the tile; a warp
            // reads two consecutive j of 16 cells and writes two 16-cell rows of shared memory
            for (int i = tid; i < M * kTileCells; i += W * 32) {
                const int c = i & 15, j = i >> 4;
                const int r = (j % op.n_q) * K + j / op.n_q;
                if (cell0 + c < n_cells)
                    cp_async8(fs + r * kTileCells + c, f + (size_t)(cell0 + c) * M + j);
                else
                    fs[r * kTileCells + c] = 0.0;
            }
            cp_async_commit();
            cp_async_wait_all();
            staged = ht;
        }
        if (tid == 0) s_next = 0;
        __syncthreads();
        const int b0 = sc.bin_begin[bin], nb = sc.bin_begin[bin + 1] - b0;
        const long long cell = cell0 + (lane & 15);
        const bool live = cell < n_cells;
        double* qc = q + (size_t)(live ? cell : 0) * M;
        for (;;) {
            int i = 0;
            if (lane == 0) i = atomicAdd(&s_next, 1);
            i = __shfl_sync(0xffffffffu, i, 0);
            if (i >= nb) break;
            tile_q1<K, false, false, true>(op, sc.bin_q1[b0 + i], fs, nullptr, rb, qc, lane, live);
        }
        if (ss.done) __threadfence();
        __syncthreads();
        if (tid == 0 && ss.done) {
            // units of this chunk: its half-tiles below n_whole are one unit each, the rest `split`
            const int h0 = chunk * ss.ht_per_chunk;
            const int c_ht = min(ss.ht_per_chunk, sc.n_ht - h0);
            const int c_whole = max(0, min(c_ht, sc.n_whole - h0));
            const int c_units = c_whole + (c_ht - c_whole) * sc.split;
            if (atomicAdd(ss.done + chunk, 1) == c_units - 1) {
                __threadfence_system();
                *reinterpret_cast<volatile int*>(ss.host_done + chunk) = ss.epoch;
            }
        }
    }
}

}  // namespace cf
