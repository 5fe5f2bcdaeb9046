// rtensor.cu -- the reduced radial tensor R on the GPU.
//
// R_t[k1,k2,k3] is the reference's sum-factorised 5-D quadrature (compute_rtensor_sumfac_mex.cpp,
// 26 inputs prepared by GeneralCollisionTensor.m:43-181).  Its structure, restated:
//
//   for every radial node x and every "item" -- patch 1: (x, u) with an inner t loop; patch 2:
//   (x, y, t) -- the pre-collision speeds vL, vS and a Jacobian J fix the item; every inner point
//   (t, chi, eps) gives two post-collision velocities vp1, vp2, and for every channel t (an
//   l-triplet) the item accumulates
//     gain_s[k1] += W (sum_q Y_q(vp_s) P_gain[q]) * phi_{k1,l1}(|vp_s|)          (s = 1, 2)
//     loss_s[k1] += W' P_loss * phi_{k1,l1}(v_s)                                  (v_1 = vL, v_2 = vS)
//   and then contributes the rank-2 update
//     R_t[k1,k2,k3] += J (gain_1 - loss_1)[k1] phi_{k2,l2}(vL) phi_{k3,l3}(vS)
//                    + J (gain_2 - loss_2)[k1] phi_{k2,l2}(vS) phi_{k3,l3}(vL)
//   (phi_{k,l}(v) = norm_{k,l} L_k^{(l+1/2)}(v^2) v^l, Y the real spherical harmonics).
//
// On the device this is two kernels over chunks of items:
//   k_items     one CTA per (item, channel group): the warps evaluate the harmonics and radial
//               functions of 16 inner points at a time (8 when L > 15: one velocity per half-warp
//               or per warp) into shared memory, then each thread owns
//               channels and accumulates their gain/loss vectors; the CTA writes the item's
//               "net" vectors J (gain - loss) and its radial values at vL and vS;
//   k_contract  one CTA per channel: every thread owns entries of R_t and sums the rank-2 updates
//               of the chunk's items in item order.
// Every R entry is summed in a fixed order, so the result is deterministic (the reference's
// OpenMP reduction order is not); it agrees with the reference to rounding.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cf_b200.h"

void cf_set_last_error(const char* msg);

namespace {

constexpr int kItemWarps = 16;          // warps per k_items CTA
// velocity slots per round: one per warp, or one per half-warp when L <= 15 (a lane per m or l
// fits in 16 lanes); each point has two post-collision velocities
constexpr int kMaxSlots = 2 * kItemWarps;
constexpr int kMaxPointsPerRound = kMaxSlots / 2;
constexpr int kMaxL = 31;               // one lane per m (harmonics) and per l (radial functions)
constexpr int kMaxNK = 12;              // radial functions per l (k_contract's per-thread entries too)
constexpr double kEpsSafe = 1e-15;      // the reference's floor under square roots
constexpr double kPi = 3.14159265358979323846;

struct Dev {
    int NK, NL, NQ, L;
    double alpha;
    const double *x, *Wx;
    int Nx;
    const double *u1, *Wu1;
    int Nu1;
    const double *t1, *Wt1;
    int Nt1;
    const double *y2, *Wy2;
    int Ny2;
    const double *t2, *Wt2;
    int Nt2;
    const double *chi, *Wchi;
    int Nchi;
    const double *eps_c, *eps_s, *Weps;  // cos and sin of the eps nodes (host libm), weights
    int Neps;
    const double* rnorm;   // [NK x (L+1)]
    const double* shnorm;  // [NQ]
    const int *l1, *l2, *l3;
    const int* vq_begin;   // [NL+1] valid q of each channel (CSR over the reference's qi lists)
    const int* vq_q;       // 0-based q
    int nnz;
    const double* ploss1;  // [Nt1 x Nu1 x NL] as given
    const double* pgain1;  // [Nu1][Nt1][nnz] compressed from [Nt1 x Nu1 x NQ x NL]
    const double* ploss2;  // [Ny2 x NL] as given
    const double* pgain2;  // [Ny2][nnz] compressed from [Ny2 x NQ x NL]
};

// norm * L_k^{(l+1/2)}(v^2) * v^l for k = 0..NK-1 (three-term recurrence in k), into out[k]
__device__ void radial_all(int NK, int l, double v, const double* rnorm, double* out) {
    const double v2 = v * v, al = (double)l + 0.5;
    const double vl = pow(v, (double)l);
    double Lm = 1.0, Lc = 1.0 + al - v2;
    for (int k = 0; k < NK; ++k) {
        double Lk;
        if (k == 0) {
            Lk = 1.0;
        } else if (k == 1) {
            Lk = Lc;
        } else {
            Lk = ((2.0 * (k - 1) + 1.0 + al - v2) * Lc - ((k - 1) + al) * Lm) / (double)k;
            Lm = Lc;
            Lc = Lk;
        }
        out[k] = rnorm[k + NK * l] * Lk * vl;
    }
}

// Real harmonics of one direction (cos theta = xc, azimuth phi), lane m = 0..L writes every l >= m.
__device__ void harmonics_lane(int L, int m, double xc, double phi, const double* shnorm, double* Y) {
    double pmm = 1.0;
    if (m > 0) {
        const double somx2 = sqrt(fmax((1.0 - xc) * (1.0 + xc), 0.0));
        double fact = 1.0;
        for (int i = 1; i <= m; ++i) {
            pmm *= -fact * somx2;
            fact += 2.0;
        }
    }
    double cs = 1.0, sn = 0.0;
    if (m > 0) {
        cs = cos(m * phi);
        sn = sin(m * phi);
    }
    double p_prev = 0.0, p_cur = pmm;
    for (int l = m; l <= L; ++l) {
        double P;
        if (l == m) {
            P = pmm;
        } else if (l == m + 1) {
            P = xc * (2 * m + 1) * pmm;
            p_prev = pmm;
            p_cur = P;
        } else {
            P = (xc * (2 * l - 1) * p_cur - (l + m - 1) * p_prev) / (double)(l - m);
            p_prev = p_cur;
            p_cur = P;
        }
        const int q0 = l * l + l;
        if (m == 0) {
            Y[q0] = shnorm[q0] * P;
        } else {
            Y[q0 + m] = shnorm[q0 + m] * P * cs;
            Y[q0 - m] = shnorm[q0 - m] * P * sn;
        }
    }
}

// Gain and loss accumulation of one item for channels [c0, c1); writes the item's net vectors and
// (group 0) its radial values at vL and vS.
__global__ void __launch_bounds__(kItemWarps * 32, 1)
    k_items(Dev d, int64_t item0, int64_t n_items_chunk, int G, double* __restrict__ net,
            double* __restrict__ radv) {
    extern __shared__ __align__(16) double sm[];
    const int NK = d.NK, L = d.L, NQ = d.NQ, NR = (L + 1) * NK;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t itl = blockIdx.x;
    const int64_t it = item0 + itl;
    const int c0 = blockIdx.y * G, c1 = min(d.NL, c0 + G);
    const int j0 = d.vq_begin[c0], j1 = d.vq_begin[c1];
    // shared layout
    // accumulators [NK][G]: consecutive channels (consecutive threads) in consecutive words
    double* gG1 = sm;                          // [NK][G] gains
    double* gG2 = gG1 + (size_t)G * NK;
    double* gL1 = gG2 + (size_t)G * NK;        // [NK][G] losses
    double* gL2 = gL1 + (size_t)G * NK;
    double* Y = gL2 + (size_t)G * NK;          // [kMaxSlots][NQ]: harmonics of the round's velocities
    double* RV = Y + (size_t)kMaxSlots * NQ;   // [kMaxSlots][NR]: radial values at |vp|
    double* RVL = RV + (size_t)kMaxSlots * NR;   // [NR] at vL
    double* RVS = RVL + NR;                      // [NR] at vS
    double* wgt = RVS + NR;                      // [kMaxPointsPerRound]
    double* pg = wgt + kMaxPointsPerRound;       // [j1 - j0] this (t, u) or y slice of P_gain
    const int sub = L <= 15 ? 2 : 1;             // velocity slots per warp
    const int slot = sub == 2 ? 2 * warp + (lane >> 4) : warp;
    const int m_lane = sub == 2 ? (lane & 15) : lane;
    const int ppr = kItemWarps * sub / 2;        // points per round

    // decode the item
    const int64_t n1 = (int64_t)d.Nx * d.Nu1;
    int patch, i, o, tfix = 0;
    if (it < n1) {
        patch = 1;
        i = (int)(it / d.Nu1);
        o = (int)(it % d.Nu1);
    } else {
        patch = 2;
        const int64_t j = it - n1;
        i = (int)(j / ((int64_t)d.Ny2 * d.Nt2));
        const int64_t r = j % ((int64_t)d.Ny2 * d.Nt2);
        o = (int)(r / d.Nt2);
        tfix = (int)(r % d.Nt2);
    }
    const double xi = d.x[i];
    const double a = sqrt(xi / 2.0);
    double u_item = 0.0, vL = 0.0, vS = 0.0, Jo = 0.0;
    if (patch == 1) {
        u_item = d.u1[o];
        vL = a * (1.0 + u_item);
        vS = a * (1.0 - u_item);
        Jo = 0.5 * d.Wx[i] * d.Wu1[o] * u_item * exp(-xi * u_item * u_item) * (vL * vL * vS * vS);
    } else {
        const double y = d.y2[o];
        const double u = y * d.t2[tfix];
        vL = a * (1.0 + u);
        vS = a * (1.0 - u);
        Jo = 0.5 * d.Wx[i] * d.Wy2[o] * y * (4.0 * y);
    }
    for (int e = tid; e < 4 * G * NK; e += blockDim.x) gG1[e] = 0.0;  // all four accumulators
    if (warp == 0 && lane <= L) radial_all(NK, lane, vL, d.rnorm, RVL + lane * NK);
    if (warp == 1 && lane <= L) radial_all(NK, lane, vS, d.rnorm, RVS + lane * NK);
    __syncthreads();

    const int n_t = patch == 1 ? d.Nt1 : 1;
    const int n_pts = d.Nchi * d.Neps;
    for (int tt = 0; tt < n_t; ++tt) {
        // the point's scalars (every thread computes them; they are a few flops)
        double Jt, cb, umag, y;
        if (patch == 1) {
            const double t = d.t1[tt];
            y = u_item * t;
            Jt = d.Wt1[tt] * (4.0 * u_item * t);
            cb = 1.0 - 2.0 * y * y;
            umag = sqrt(2.0 * xi) * u_item * sqrt(1.0 + (1.0 - u_item * u_item) * t * t);
        } else {
            y = d.y2[o];
            const double t = d.t2[tfix];
            const double u = y * t;
            Jt = d.Wt2[tfix] * exp(-xi * u * u) * (vL * vL * vS * vS);
            cb = 1.0 - 2.0 * y * y;
            umag = sqrt(2.0 * xi) * y * sqrt(t * t + 1.0 - y * y * t * t);
        }
        const double sb = sqrt(fmax(1.0 - cb * cb, kEpsSafe));
        const double B = pow(umag * sqrt(2.0), d.alpha) / pow(xi, d.alpha / 2.0);
        const double lw = B * 2.0 * kPi * 2.0 * Jt;
        const double Ux1 = vS * sb, Uz1 = vL + vS * cb, ux1 = -vS * sb, uz1 = vL - vS * cb;
        const double um1 = sqrt(fmax(ux1 * ux1 + uz1 * uz1, kEpsSafe));
        const double zx1 = ux1 / um1, zz1 = uz1 / um1;
        const double Ux2 = vL * sb, Uz2 = vS + vL * cb, ux2 = -vL * sb, uz2 = vS - vL * cb;
        const double um2 = sqrt(fmax(ux2 * ux2 + uz2 * uz2, kEpsSafe));
        const double zx2 = ux2 / um2, zz2 = uz2 / um2;

        // this slice of P_gain, and the losses
        const double* pgs = patch == 1 ? d.pgain1 + ((size_t)o * d.Nt1 + tt) * d.nnz : d.pgain2 + (size_t)o * d.nnz;
        for (int j = j0 + tid; j < j1; j += blockDim.x) pg[j - j0] = pgs[j];
        for (int ch = c0 + tid; ch < c1; ch += blockDim.x) {
            const double pl = patch == 1 ? d.ploss1[tt + (size_t)d.Nt1 * (o + (size_t)d.Nu1 * ch)]
                                         : d.ploss2[o + (size_t)d.Ny2 * ch];
            const double li = lw * pl;
            const int l1 = d.l1[ch];
            double* a1 = gL1 + (ch - c0);
            double* a2 = gL2 + (ch - c0);
            for (int k = 0; k < NK; ++k) {
                a1[(size_t)k * G] += RVL[l1 * NK + k] * li;
                a2[(size_t)k * G] += RVS[l1 * NK + k] * li;
            }
        }
        __syncthreads();

        for (int p0 = 0; p0 < n_pts; p0 += ppr) {
            // slot s (a warp, or a half-warp) evaluates velocity (s & 1) of point p0 + (s >> 1)
            const int p = p0 + (slot >> 1), side = slot & 1;
            if (p < n_pts) {
                const int n = p / d.Neps, e = p % d.Neps;
                const double cc = d.chi[n];
                const double sc = sqrt(fmax(1.0 - cc * cc, 0.0));
                const double upx = sc * d.eps_c[e], upy = sc * d.eps_s[e], upz = cc;
                double vpx, vpy, vpz;
                if (side == 0) {
                    const double upx1 = upx * zz1 + upz * zx1, upz1 = -upx * zx1 + upz * zz1;
                    vpx = 0.5 * (Ux1 + um1 * upx1);
                    vpy = 0.5 * (um1 * upy);
                    vpz = 0.5 * (Uz1 + um1 * upz1);
                } else {
                    const double upx2 = upx * zz2 + upz * zx2, upz2 = -upx * zx2 + upz * zz2;
                    vpx = 0.5 * (Ux2 + um2 * upx2);
                    vpy = 0.5 * (um2 * upy);
                    vpz = 0.5 * (Uz2 + um2 * upz2);
                }
                const double vm = sqrt(fmax(vpx * vpx + vpy * vpy + vpz * vpz, kEpsSafe));
                const double xc = fmax(fmin(vpz / vm, 1.0), -1.0);
                const double phi = atan2(vpy, vpx);
                if (m_lane <= L) {
                    harmonics_lane(L, m_lane, xc, phi, d.shnorm, Y + (size_t)slot * NQ);
                    radial_all(NK, m_lane, vm, d.rnorm, RV + (size_t)slot * NR + m_lane * NK);
                }
                if (m_lane == 0 && side == 0) wgt[slot >> 1] = d.Wchi[n] * B * Jt * d.Weps[e];
            }
            __syncthreads();
            const int np = min(ppr, n_pts - p0);
            for (int ch = c0 + tid; ch < c1; ch += blockDim.x) {
                const int l1 = d.l1[ch], jb = d.vq_begin[ch], je = d.vq_begin[ch + 1];
                double* a1 = gG1 + (ch - c0);
                double* a2 = gG2 + (ch - c0);
                // the round's points summed in registers, then added to the item's accumulators
                double s1[kMaxNK], s2[kMaxNK];
#pragma unroll
                for (int k = 0; k < kMaxNK; ++k) {
                    s1[k] = 0.0;
                    s2[k] = 0.0;
                }
                for (int pp = 0; pp < np; ++pp) {
                    const double* Y1 = Y + (size_t)(2 * pp) * NQ;
                    const double* Y2 = Y1 + NQ;
                    double g1 = 0.0, g2 = 0.0;
                    for (int j = jb; j < je; ++j) {
                        const int q = d.vq_q[j];
                        const double w = pg[j - j0];
                        g1 += Y1[q] * w;
                        g2 += Y2[q] * w;
                    }
                    const double w1 = g1 * wgt[pp], w2 = g2 * wgt[pp];
                    const double* r1 = RV + (size_t)(2 * pp) * NR + l1 * NK;
                    const double* r2 = r1 + NR;
#pragma unroll
                    for (int k = 0; k < kMaxNK; ++k)
                        if (k < NK) {
                            s1[k] += w1 * r1[k];
                            s2[k] += w2 * r2[k];
                        }
                }
#pragma unroll
                for (int k = 0; k < kMaxNK; ++k)
                    if (k < NK) {
                        a1[(size_t)k * G] += s1[k];
                        a2[(size_t)k * G] += s2[k];
                    }
            }
            __syncthreads();
        }
    }
    // net vectors J (gain - loss), [channel][item][2][NK]
    for (int ch = c0 + tid; ch < c1; ch += blockDim.x) {
        double* dst = net + ((size_t)ch * n_items_chunk + itl) * 2 * NK;
        const size_t b = (size_t)(ch - c0);
        for (int k = 0; k < NK; ++k) {
            dst[k] = Jo * (gG1[b + (size_t)k * G] - gL1[b + (size_t)k * G]);
            dst[NK + k] = Jo * (gG2[b + (size_t)k * G] - gL2[b + (size_t)k * G]);
        }
    }
    if (blockIdx.y == 0)
        for (int e = tid; e < 2 * NR; e += blockDim.x) radv[(size_t)itl * 2 * NR + e] = e < NR ? RVL[e] : RVS[e - NR];
}

// R_t[k1,k2,k3] += sum over the chunk's items, in item order, of the rank-2 updates.
constexpr int kContractThreads = 256;
constexpr int kContractBlock = 32;  // items staged per round
__global__ void __launch_bounds__(kContractThreads) k_contract(Dev d, const double* __restrict__ net,
                                                               const double* __restrict__ radv,
                                                               int64_t n_items_chunk, double* __restrict__ R) {
    extern __shared__ __align__(16) double sm[];
    const int NK = d.NK, NR = (d.L + 1) * NK, K3 = NK * NK * NK;
    const int ch = blockIdx.x, tid = threadIdx.x;
    const int l2 = d.l2[ch], l3 = d.l3[ch];
    double* sn = sm;                                    // [block][2 NK] net vectors
    double* sr = sn + (size_t)kContractBlock * 2 * NK;  // [block][4 NK]: vL at l2, vS at l3, vS at l2, vL at l3
    constexpr int kMaxPer = 8;                          // entries of R per thread (NK <= 12: 1728 / 256 < 8)
    double acc[kMaxPer];
#pragma unroll
    for (int e = 0; e < kMaxPer; ++e) acc[e] = 0.0;
    for (int64_t b0 = 0; b0 < n_items_chunk; b0 += kContractBlock) {
        const int nb = (int)(n_items_chunk - b0 < kContractBlock ? n_items_chunk - b0 : kContractBlock);
        __syncthreads();
        for (int e = tid; e < nb * 2 * NK; e += kContractThreads)
            sn[e] = net[((size_t)ch * n_items_chunk + b0) * 2 * NK + e];
        for (int e = tid; e < nb * 4 * NK; e += kContractThreads) {
            const int itb = e / (4 * NK), r = e % (4 * NK), w = r / NK, k = r % NK;
            const double* rv = radv + (size_t)(b0 + itb) * 2 * NR;
            // w = 0: phi(vL) at l2; 1: phi(vS) at l3; 2: phi(vS) at l2; 3: phi(vL) at l3
            const int l = (w == 0 || w == 2) ? l2 : l3;
            const int side = (w == 0 || w == 3) ? 0 : 1;
            sr[e] = rv[side * NR + l * NK + k];
        }
        __syncthreads();
        for (int ib = 0; ib < nb; ++ib) {
            const double* n1 = sn + (size_t)ib * 2 * NK;
            const double* n2 = n1 + NK;
            const double* rL2 = sr + (size_t)ib * 4 * NK;
            const double* rS3 = rL2 + NK;
            const double* rS2 = rS3 + NK;
            const double* rL3 = rS2 + NK;
#pragma unroll
            for (int e = 0; e < kMaxPer; ++e) {
                const int idx = tid + e * kContractThreads;
                if (idx < K3) {
                    const int k1 = idx % NK, k2 = (idx / NK) % NK, k3 = idx / (NK * NK);
                    acc[e] += n1[k1] * rL2[k2] * rS3[k3] + n2[k1] * rS2[k2] * rL3[k3];
                }
            }
        }
    }
#pragma unroll
    for (int e = 0; e < kMaxPer; ++e) {
        const int idx = tid + e * kContractThreads;
        if (idx < K3) R[(size_t)ch * K3 + idx] += acc[e];
    }
}

#define RT_CHECK(expr)                                                                                  \
    do {                                                                                                \
        cudaError_t e_ = (expr);                                                                        \
        if (e_ != cudaSuccess) {                                                                        \
            char m_[256];                                                                               \
            snprintf(m_, sizeof(m_), "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
            cf_set_last_error(m_);                                                                      \
            st = e_ == cudaErrorMemoryAllocation ? CF_ENOMEM : CF_ECUDA;                                \
            goto done;                                                                                  \
        }                                                                                               \
    } while (0)

template <typename S>
cudaError_t upload(const S** dst, const S* src, size_t n, std::vector<void*>& owned) {
    S* p = nullptr;
    *dst = nullptr;
    cudaError_t e = cudaMalloc((void**)&p, std::max<size_t>(n, 1) * sizeof(S));
    if (e != cudaSuccess) return e;
    owned.push_back(p);
    *dst = p;
    return n ? cudaMemcpy(p, src, n * sizeof(S), cudaMemcpyHostToDevice) : cudaSuccess;
}

// The channels (l-triplets) and the CSR of their valid q_i (the reference stops each list at its
// first -1), after checking the sizes and indices of the inputs.
struct Channels {
    std::vector<int> l1, l2, l3, vq_begin, vq_q;
};

int sumfac_channels(const char* fn, double* R_out, const cf_sumfac_inputs* in, int32_t device, Channels& chn) {
    char msg[160];
    if (!R_out || !in) {
        snprintf(msg, sizeof(msg), "%s: null argument", fn);
        cf_set_last_error(msg);
        return CF_EINVAL;
    }
    const int NK = in->k_max + 1, NL = in->n_l, NQ = in->n_q;
    const int L = (int)std::lround(std::sqrt((double)NQ)) - 1;
    if (in->k_max < 0 || NK > 12 || NL < 1 || NQ < 1 || (L + 1) * (L + 1) != NQ || L > kMaxL || in->n_x < 1 ||
        in->n_u1 < 0 || in->n_t1 < 0 || in->n_y2 < 0 || in->n_t2 < 0 || in->n_chi < 0 || in->n_eps < 0) {
        snprintf(msg, sizeof(msg), "%s: sizes out of range (K_max+1 <= 12, N_Q = (L+1)^2 with L <= 31)", fn);
        cf_set_last_error(msg);
        return CF_ESHAPE;
    }
    const double* arrays[] = {in->x_nodes, in->w_x, in->radial_norm, in->sh_norm, in->l_triplets, in->qi_valid};
    for (const double* p : arrays)
        if (!p) {
            snprintf(msg, sizeof(msg), "%s: null input array", fn);
            cf_set_last_error(msg);
            return CF_EINVAL;
        }
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0) {
        snprintf(msg, sizeof(msg), "%s: no CUDA device", fn);
        cf_set_last_error(msg);
        return CF_ENODEVICE;
    }
    if (device < 0 || device >= n_dev) return CF_EINVAL;

    std::vector<int>&l1 = chn.l1, &l2 = chn.l2, &l3 = chn.l3, &vq_begin = chn.vq_begin, &vq_q = chn.vq_q;
    l1.assign(NL, 0);
    l2.assign(NL, 0);
    l3.assign(NL, 0);
    vq_begin.assign(NL + 1, 0);
    vq_q.clear();
    for (int ch = 0; ch < NL; ++ch) {
        l1[ch] = (int)in->l_triplets[ch];
        l2[ch] = (int)in->l_triplets[ch + NL];
        l3[ch] = (int)in->l_triplets[ch + 2 * NL];
        if (l1[ch] < 0 || l1[ch] > L || l2[ch] < 0 || l2[ch] > L || l3[ch] < 0 || l3[ch] > L) {
            snprintf(msg, sizeof(msg), "%s: an l-triplet is outside 0..L", fn);
            cf_set_last_error(msg);
            return CF_EBADIDX;
        }
        for (int idx = 0; idx < NQ; ++idx) {
            const int q = (int)in->qi_valid[idx + (size_t)NQ * ch];
            if (q == -1) break;
            if (q < 1 || q > NQ) {
                snprintf(msg, sizeof(msg), "%s: qi_valid holds an index outside 1..N_Q", fn);
                cf_set_last_error(msg);
                return CF_EBADIDX;
            }
            vq_q.push_back(q - 1);
        }
        vq_begin[ch + 1] = (int)vq_q.size();
    }
    return CF_OK;
}

// The quadrature proper, from the channel lists and the gain tables compressed to the valid
// (q, channel) pairs: pg1[(u * n_t1 + t) * nnz + j], pg2[y * nnz + j], j running over the pairs in
// channel order and, within a channel, in qi_valid order.
int sumfac_run(double* R_out, const cf_sumfac_inputs* in, const Channels& chn, const double* pg1_h,
               const double* pg2_h, int32_t device, double* device_seconds) {
    const int NK = in->k_max + 1, NL = in->n_l, NQ = in->n_q;
    const int L = (int)std::lround(std::sqrt((double)NQ)) - 1;
    const std::vector<int>&l1 = chn.l1, &l2 = chn.l2, &l3 = chn.l3, &vq_begin = chn.vq_begin, &vq_q = chn.vq_q;
    const int nnz = (int)vq_q.size();
    std::vector<double> eps_c(in->n_eps), eps_s(in->n_eps);
    for (int e = 0; e < in->n_eps; ++e) {
        eps_c[e] = std::cos(in->eps[e]);
        eps_s[e] = std::sin(in->eps[e]);
    }

    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    int st = CF_OK;
    std::vector<void*> owned;
    Dev d{};
    double *net = nullptr, *radv = nullptr, *dR = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    const int NR = (L + 1) * NK;
    const int64_t n_items = (int64_t)in->n_x * in->n_u1 + (int64_t)in->n_x * in->n_y2 * in->n_t2;
    int max_smem = 0;
    // channel group: the four accumulators, the round's harmonics and radial values, and the
    // group's P_gain slice fit in shared memory
    int G = NL, max_nnz_g = nnz;
    size_t smem = 0;
    int n_groups = 1;
    int64_t chunk = 0;
    d.NK = NK;
    d.NL = NL;
    d.NQ = NQ;
    d.L = L;
    d.alpha = in->alpha;
    d.Nx = in->n_x;
    d.Nu1 = in->n_u1;
    d.Nt1 = in->n_t1;
    d.Ny2 = in->n_y2;
    d.Nt2 = in->n_t2;
    d.Nchi = in->n_chi;
    d.Neps = in->n_eps;
    d.nnz = nnz;
    RT_CHECK(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    for (;;) {
        n_groups = (NL + G - 1) / G;
        max_nnz_g = 0;
        for (int g = 0; g < n_groups; ++g)
            max_nnz_g = std::max(max_nnz_g, vq_begin[std::min(NL, (g + 1) * G)] - vq_begin[g * G]);
        smem = sizeof(double) * ((size_t)4 * G * NK + (size_t)kMaxSlots * (NQ + NR) + 2 * NR + kMaxPointsPerRound +
                                 max_nnz_g);
        if (smem + 1024 <= (size_t)max_smem || G == 1) break;
        G = (G + 1) / 2;
    }
    if (smem + 1024 > (size_t)max_smem) {
        cf_set_last_error("cf_rtensor_sumfac: N_Q too large for the shared-memory layout");
        st = CF_EUNSUPPORTED;
        goto done;
    }
    RT_CHECK(upload(&d.x, in->x_nodes, in->n_x, owned));
    RT_CHECK(upload(&d.Wx, in->w_x, in->n_x, owned));
    RT_CHECK(upload(&d.u1, in->u1_nodes, in->n_u1, owned));
    RT_CHECK(upload(&d.Wu1, in->w_u1, in->n_u1, owned));
    RT_CHECK(upload(&d.t1, in->t1_nodes, in->n_t1, owned));
    RT_CHECK(upload(&d.Wt1, in->w_t1, in->n_t1, owned));
    RT_CHECK(upload(&d.y2, in->y2_nodes, in->n_y2, owned));
    RT_CHECK(upload(&d.Wy2, in->w_y2, in->n_y2, owned));
    RT_CHECK(upload(&d.t2, in->t2_nodes, in->n_t2, owned));
    RT_CHECK(upload(&d.Wt2, in->w_t2, in->n_t2, owned));
    RT_CHECK(upload(&d.chi, in->mu_chi, in->n_chi, owned));
    RT_CHECK(upload(&d.Wchi, in->w_chi, in->n_chi, owned));
    RT_CHECK(upload(&d.eps_c, eps_c.data(), eps_c.size(), owned));
    RT_CHECK(upload(&d.eps_s, eps_s.data(), eps_s.size(), owned));
    RT_CHECK(upload(&d.Weps, in->w_eps, in->n_eps, owned));
    RT_CHECK(upload(&d.rnorm, in->radial_norm, (size_t)NK * (L + 1), owned));
    RT_CHECK(upload(&d.shnorm, in->sh_norm, (size_t)NQ, owned));
    RT_CHECK(upload(&d.l1, l1.data(), l1.size(), owned));
    RT_CHECK(upload(&d.l2, l2.data(), l2.size(), owned));
    RT_CHECK(upload(&d.l3, l3.data(), l3.size(), owned));
    RT_CHECK(upload(&d.vq_begin, vq_begin.data(), vq_begin.size(), owned));
    RT_CHECK(upload(&d.vq_q, vq_q.data(), vq_q.size(), owned));
    RT_CHECK(upload(&d.ploss1, in->p_loss_p1, (size_t)in->n_t1 * in->n_u1 * NL, owned));
    RT_CHECK(upload(&d.pgain1, pg1_h, (size_t)in->n_u1 * in->n_t1 * nnz, owned));
    RT_CHECK(upload(&d.ploss2, in->p_loss_p2, (size_t)in->n_y2 * NL, owned));
    RT_CHECK(upload(&d.pgain2, pg2_h, (size_t)in->n_y2 * nnz, owned));
    // chunk of items: the net vectors of a chunk (written by k_items, read once by k_contract) stay
    // within 48 MB, so they live in the 126 MB L2 between the two kernels instead of crossing HBM
    chunk = std::max<int64_t>(1, std::min<int64_t>(n_items, ((int64_t)48 << 20) / ((int64_t)NL * 2 * NK * 8)));
    chunk = std::min<int64_t>(chunk, 65535);  // grid x of k_items
    RT_CHECK(cudaMalloc((void**)&net, (size_t)chunk * NL * 2 * NK * sizeof(double)));
    owned.push_back(net);
    RT_CHECK(cudaMalloc((void**)&radv, (size_t)chunk * 2 * NR * sizeof(double)));
    owned.push_back(radv);
    RT_CHECK(cudaMalloc((void**)&dR, (size_t)NK * NK * NK * NL * sizeof(double)));
    owned.push_back(dR);
    RT_CHECK(cudaMemset(dR, 0, (size_t)NK * NK * NK * NL * sizeof(double)));
    RT_CHECK(cudaFuncSetAttribute(k_items, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    RT_CHECK(cudaEventCreate(&ev0));
    RT_CHECK(cudaEventCreate(&ev1));
    RT_CHECK(cudaEventRecord(ev0));
    for (int64_t i0 = 0; i0 < n_items; i0 += chunk) {
        const int64_t nc = std::min(chunk, n_items - i0);
        k_items<<<dim3((unsigned)nc, (unsigned)n_groups), kItemWarps * 32, smem>>>(d, i0, nc, G, net, radv);
        RT_CHECK(cudaGetLastError());
        const size_t smem_c = sizeof(double) * (size_t)kContractBlock * 6 * NK;
        k_contract<<<NL, kContractThreads, smem_c>>>(d, net, radv, nc, dR);
        RT_CHECK(cudaGetLastError());
    }
    RT_CHECK(cudaEventRecord(ev1));
    RT_CHECK(cudaEventSynchronize(ev1));
    if (device_seconds) {
        float ms = 0.f;
        RT_CHECK(cudaEventElapsedTime(&ms, ev0, ev1));
        *device_seconds = ms * 1e-3;
    }
    RT_CHECK(cudaMemcpy(R_out, dR, (size_t)NK * NK * NK * NL * sizeof(double), cudaMemcpyDeviceToHost));
done:
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    for (void* p : owned) cudaFree(p);
    cudaSetDevice(prev);
    return st;
}


}  // namespace

extern "C" {

int cf_rtensor_sumfac(double* R_out, const cf_sumfac_inputs* in, int32_t device, double* device_seconds) {
    Channels chn;
    int st = sumfac_channels("cf_rtensor_sumfac", R_out, in, device, chn);
    if (st != CF_OK) return st;
    if (!in->p_gain_p1 || !in->p_gain_p2) {
        cf_set_last_error("cf_rtensor_sumfac: null input array");
        return CF_EINVAL;
    }
    const int NQ = in->n_q;
    const std::vector<int>&vq_begin = chn.vq_begin, &vq_q = chn.vq_q;
    const int NL = in->n_l;
    const int nnz = (int)vq_q.size();
    // P_gain compressed to the valid (q, channel) pairs, slice-major
    std::vector<double> pg1((size_t)in->n_u1 * in->n_t1 * nnz), pg2((size_t)in->n_y2 * nnz);
    for (int ch = 0; ch < NL; ++ch)
        for (int j = vq_begin[ch]; j < vq_begin[ch + 1]; ++j) {
            const size_t q = (size_t)vq_q[j];
            for (int u = 0; u < in->n_u1; ++u)
                for (int t = 0; t < in->n_t1; ++t)
                    pg1[((size_t)u * in->n_t1 + t) * nnz + j] =
                        in->p_gain_p1[t + (size_t)in->n_t1 * (u + (size_t)in->n_u1 * (q + (size_t)NQ * ch))];
            for (int y = 0; y < in->n_y2; ++y)
                pg2[(size_t)y * nnz + j] = in->p_gain_p2[y + (size_t)in->n_y2 * (q + (size_t)NQ * ch)];
        }
    return sumfac_run(R_out, in, chn, pg1.data(), pg2.data(), device, device_seconds);
}

int cf_rtensor_sumfac_packed(double* R_out, const cf_sumfac_inputs* in, const double* p_gain_p1_packed,
                             const double* p_gain_p2_packed, int32_t device, double* device_seconds) {
    Channels chn;
    int st = sumfac_channels("cf_rtensor_sumfac_packed", R_out, in, device, chn);
    if (st != CF_OK) return st;
    if (!p_gain_p1_packed || !p_gain_p2_packed) {
        cf_set_last_error("cf_rtensor_sumfac_packed: null packed gain table");
        return CF_EINVAL;
    }
    return sumfac_run(R_out, in, chn, p_gain_p1_packed, p_gain_p2_packed, device, device_seconds);
}

}  // extern "C"
