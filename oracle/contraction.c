/*
 * oracle/contraction.c -- CPU restatement of the reference collision contraction.
 *
 * TEST INFRASTRUCTURE.  This file is the oracle the CUDA path is checked
 * against; it is linked only by the tests, by __graft_entry__.smoke() and by the
 * CPU-baseline leg of bench.py, never by the product library.
 *
 * Conventions (all from the reference):
 *   f, Q     column-major [N_Q x K]: element (q,k) at q + k*N_Q
 *            (src/mex/angular_first_collision_kernel_mex.cpp:53,68)
 *   labels   column-major [N_G x 3] of 1-based (q1,q2,q3) stored as double
 *            (src/mex/angular_first_collision_kernel_mex.cpp:37,48-49)
 *   ic_map   [N_G] 1-based l-triplet index stored as double
 *   R        column-major [K x K x K x N_L]: R[k1 + K*k2 + K^2*k3 + K^3*t]
 *            (src/mex/angular_first_collision_kernel_mex.cpp:65)
 *   Batched arrays are [N_Q x K x B] (cell b at offset b*N_Q*K).
 *
 * Every kernel ACCUMULATES into Q (Q += ...), as the reference does.
 * The arithmetic order inside each function follows the reference function it
 * cites, so that, compiled with the same flags and without FMA contraction, the
 * results agree bit for bit with the compiled reference sources.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define LAB(col, z) ((int)labels[(size_t)(z) + (size_t)(col) * (size_t)NG] - 1)
#define TIDX(z) ((int)ic_map[(z)] - 1)

/* End of the run of equal l-triplet index starting at z. */
static int64_t run_end_t(const double* ic_map, int64_t z, int64_t end) {
    const int t = TIDX(z);
    while (z < end && TIDX(z) == t) ++z;
    return z;
}

/* End of the run of equal q1 starting at z (inside [z, end)). */
static int64_t run_end_q1(const double* labels, int64_t NG, int64_t z, int64_t end) {
    const int q1 = LAB(0, z);
    while (z < end && LAB(0, z) == q1) ++z;
    return z;
}

/*
 * Angular-first contraction.
 * Follows src/mex/angular_first_collision_kernel_mex.cpp:6-75:
 *   per run of equal t (:24-32), per run of equal q1 (:35-43):
 *     Phi[k2 + K*k3] = sum_z g_z * f[q2,k2] * f[q3,k3]           (:45-58)
 *     Q[q1,k1]      += sum_{k3,k2} R_t[k1,k2,k3] * Phi[k2,k3]   (:60-69)
 */
int orc_af(double* Q, const double* f, const double* labels, const double* vals,
           const double* ic_map, const double* R, int64_t NG, int NQ, int K) {
    const int K2 = K * K, K3 = K2 * K;
    double* phi = (double*)malloc(sizeof(double) * (size_t)K2);
    if (!phi) return 1;
    int64_t z = 0;
    while (z < NG) {
        const int t = TIDX(z);
        const int64_t zt = run_end_t(ic_map, z, NG);
        int64_t s = z;
        while (s < zt) {
            const int q1 = LAB(0, s);
            const int64_t se = run_end_q1(labels, NG, s, zt);
            memset(phi, 0, sizeof(double) * (size_t)K2);
            for (int64_t i = s; i < se; ++i) {
                const int q2 = LAB(1, i), q3 = LAB(2, i);
                const double g = vals[i];
                for (int k3 = 0; k3 < K; ++k3) {
                    const double f3 = f[q3 + (size_t)k3 * NQ];
                    for (int k2 = 0; k2 < K; ++k2)
                        phi[k2 + k3 * K] += g * f[q2 + (size_t)k2 * NQ] * f3;
                }
            }
            const double* Rt = R + (size_t)t * K3;
            for (int k1 = 0; k1 < K; ++k1) {
                double acc = 0.0;
                for (int k3 = 0; k3 < K; ++k3)
                    for (int k2 = 0; k2 < K; ++k2)
                        acc += Rt[k1 + k2 * K + k3 * K2] * phi[k2 + k3 * K];
                Q[q1 + (size_t)k1 * NQ] += acc;
            }
            s = se;
        }
        z = zt;
    }
    free(phi);
    return 0;
}

/*
 * Radial-first contraction.
 * Follows src/mex/radial_first_collision_kernel_mex.cpp:5-76:
 *   per run of equal t (:27-35):
 *     Psi[z,k1] = sum_{k3,k2} R_t[k1,k2,k3] * f[q2,k2] * f[q3,k3]   (:41-59)
 *     Q[q1,k1] += g_z * Psi[z,k1]                                  (:64-72)
 */
int orc_rf(double* Q, const double* f, const double* labels, const double* vals,
           const double* ic_map, const double* R, int64_t NG, int NQ, int K) {
    const int K2 = K * K, K3 = K2 * K;
    double* psi = (double*)malloc(sizeof(double) * (size_t)(NG > 0 ? NG : 1) * (size_t)K);
    if (!psi) return 1;
    int64_t z0 = 0;
    while (z0 < NG) {
        const int t = TIDX(z0);
        const int64_t ze = run_end_t(ic_map, z0, NG);
        const double* Rt = R + (size_t)t * K3;
        for (int64_t z = z0; z < ze; ++z) {
            const int q2 = LAB(1, z), q3 = LAB(2, z);
            for (int k1 = 0; k1 < K; ++k1) {
                double acc = 0.0;
                for (int k3 = 0; k3 < K; ++k3) {
                    const double f3 = f[q3 + (size_t)k3 * NQ];
                    for (int k2 = 0; k2 < K; ++k2) {
                        const double f2 = f[q2 + (size_t)k2 * NQ];
                        acc += Rt[k1 + k2 * K + k3 * K2] * f2 * f3;
                    }
                }
                psi[(z - z0) * K + k1] = acc;
            }
        }
        for (int64_t z = z0; z < ze; ++z) {
            const int q1 = LAB(0, z);
            const double g = vals[z];
            for (int k1 = 0; k1 < K; ++k1) Q[q1 + (size_t)k1 * NQ] += g * psi[(z - z0) * K + k1];
        }
        z0 = ze;
    }
    free(psi);
    return 0;
}

/*
 * Naive sparse contraction over an unsorted COO list.
 * Follows src/mex/naive_collision_kernel_mex.cpp:3-46:
 *   Q[q1,k1] += g * R_t[k1,k2,k3] * (f[q2,k2] * f[q3,k3])   (:23-45)
 */
int orc_naive(double* Q, const double* f, const double* labels, const double* vals,
              const double* ic_map, const double* R, int64_t NG, int NQ, int K) {
    const int K2 = K * K, K3 = K2 * K;
    for (int64_t z = 0; z < NG; ++z) {
        const int q1 = LAB(0, z), q2 = LAB(1, z), q3 = LAB(2, z), t = TIDX(z);
        const double g = vals[z];
        for (int k2 = 0; k2 < K; ++k2)
            for (int k3 = 0; k3 < K; ++k3) {
                const double f23 = f[q2 + (size_t)k2 * NQ] * f[q3 + (size_t)k3 * NQ];
                for (int k1 = 0; k1 < K; ++k1)
                    Q[q1 + (size_t)k1 * NQ] += g * R[k1 + k2 * K + k3 * K2 + (size_t)t * K3] * f23;
            }
    }
    return 0;
}

/*
 * Dense contraction Q[i] += C[i + j*N + k*N^2] * f[j] * f[k].
 * Follows src/mex/dense_tensor_kernel_mex.cpp:3-30.
 */
int orc_dense(double* Q, const double* f, const double* C, int64_t N) {
    for (int64_t k = 0; k < N; ++k) {
        const double fk = f[k];
        for (int64_t j = 0; j < N; ++j) {
            const double fjk = f[j] * fk;
            const double* col = C + (size_t)(j + k * N) * (size_t)N;
            for (int64_t i = 0; i < N; ++i) Q[i] += col[i] * fjk;
        }
    }
    return 0;
}

/*
 * Jacobian apply J(f).v = Q(v,f) + Q(f,v), accumulated into out.
 * No reference counterpart: this is the bilinear form of the angular-first
 * contraction above (src/mex/angular_first_collision_kernel_mex.cpp:45-69) with
 * Phi = sum_z g_z (v[q2] (x) f[q3] + f[q2] (x) v[q3]).  With v = f it equals
 * 2*Q(f) up to rounding.  The linearisation J = C(:,:,f) + C(:,f,:) is the one
 * the reference forms densely at equilibrium
 * (tutorial_collisions_spectral_properties.m:43).
 */
int orc_jv(double* out, const double* f, const double* v, const double* labels,
           const double* vals, const double* ic_map, const double* R, int64_t NG, int NQ, int K) {
    const int K2 = K * K, K3 = K2 * K;
    double* phi = (double*)malloc(sizeof(double) * (size_t)K2);
    if (!phi) return 1;
    int64_t z = 0;
    while (z < NG) {
        const int t = TIDX(z);
        const int64_t zt = run_end_t(ic_map, z, NG);
        int64_t s = z;
        while (s < zt) {
            const int q1 = LAB(0, s);
            const int64_t se = run_end_q1(labels, NG, s, zt);
            memset(phi, 0, sizeof(double) * (size_t)K2);
            for (int64_t i = s; i < se; ++i) {
                const int q2 = LAB(1, i), q3 = LAB(2, i);
                const double g = vals[i];
                for (int k3 = 0; k3 < K; ++k3) {
                    const double f3 = f[q3 + (size_t)k3 * NQ];
                    const double v3 = v[q3 + (size_t)k3 * NQ];
                    for (int k2 = 0; k2 < K; ++k2)
                        phi[k2 + k3 * K] += g * (v[q2 + (size_t)k2 * NQ] * f3 + f[q2 + (size_t)k2 * NQ] * v3);
                }
            }
            const double* Rt = R + (size_t)t * K3;
            for (int k1 = 0; k1 < K; ++k1) {
                double acc = 0.0;
                for (int k3 = 0; k3 < K; ++k3)
                    for (int k2 = 0; k2 < K; ++k2)
                        acc += Rt[k1 + k2 * K + k3 * K2] * phi[k2 + k3 * K];
                out[q1 + (size_t)k1 * NQ] += acc;
            }
            s = se;
        }
        z = zt;
    }
    free(phi);
    return 0;
}

/* ---------------- batched drivers (cells are independent; OpenMP over cells) ---------------- */

typedef int (*orc_single_fn)(double*, const double*, const double*, const double*, const double*,
                             const double*, int64_t, int, int);

static int batch(orc_single_fn fn, double* Q, const double* f, int64_t B, const double* labels,
                 const double* vals, const double* ic_map, const double* R, int64_t NG, int NQ, int K,
                 int nthreads) {
    const size_t M = (size_t)NQ * (size_t)K;
    int err = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads) reduction(| : err)
#endif
    for (int64_t b = 0; b < B; ++b)
        err |= fn(Q + (size_t)b * M, f + (size_t)b * M, labels, vals, ic_map, R, NG, NQ, K);
    (void)nthreads;
    return err;
}

int orc_af_batch(double* Q, const double* f, int64_t B, const double* labels, const double* vals,
                 const double* ic_map, const double* R, int64_t NG, int NQ, int K, int nthreads) {
    return batch(orc_af, Q, f, B, labels, vals, ic_map, R, NG, NQ, K, nthreads);
}

int orc_rf_batch(double* Q, const double* f, int64_t B, const double* labels, const double* vals,
                 const double* ic_map, const double* R, int64_t NG, int NQ, int K, int nthreads) {
    return batch(orc_rf, Q, f, B, labels, vals, ic_map, R, NG, NQ, K, nthreads);
}

int orc_jv_batch(double* out, const double* f, const double* v, int64_t B, const double* labels,
                 const double* vals, const double* ic_map, const double* R, int64_t NG, int NQ, int K,
                 int nthreads) {
    const size_t M = (size_t)NQ * (size_t)K;
    int err = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads) reduction(| : err)
#endif
    for (int64_t b = 0; b < B; ++b)
        err |= orc_jv(out + (size_t)b * M, f + (size_t)b * M, v + (size_t)b * M, labels, vals, ic_map,
                      R, NG, NQ, K);
    (void)nthreads;
    return err;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
