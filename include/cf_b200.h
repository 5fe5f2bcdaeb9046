/*
 * cf_b200.h -- C ABI of the B200 collision-contraction library (libcf_b200.so).
 *
 * The operator is the Wigner-Eckart-factorised spectral Boltzmann contraction
 *
 *   Q(f)[q1,k1] = sum_{z : q1(z) = q1} G_z sum_{k2,k3} R_{t(z)}[k1,k2,k3] f[q2(z),k2] f[q3(z),k3]
 *
 * routed through the COO Gaunt lists of the reference (labels, vals, ic_map) and
 * its reduced radial tensor R.  All arrays use the reference's MEX conventions:
 *
 *   f, Q    column-major double [N_Q x K] per cell; batched [N_Q x K x B]
 *           (element (q,k) of cell b at q + k*N_Q + b*N_Q*K)
 *   labels  column-major double [N_G x 3], 1-based (q1, q2, q3)
 *   vals    double [N_G]       real Gaunt values
 *   ic_map  double [N_G]       1-based l-triplet index t
 *   R       column-major double [K x K x K x N_L]: R[k1 + K*k2 + K^2*k3 + K^3*t]
 *
 * Every contraction ACCUMULATES into its output (out += ...), exactly as the
 * reference kernels write into their first argument.  The entries may be in any
 * order; Q is summed run by run of equal (ic_map, q1), as the reference does.
 *
 * Every function returns a cf_status.  Nothing here falls back to the CPU: without
 * a usable CUDA device the calls return CF_ENODEVICE.
 */
#ifndef CF_B200_H
#define CF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum cf_status {
    CF_OK = 0,
    CF_EINVAL = 1,        /* a null pointer or an out-of-range scalar argument      */
    CF_ESHAPE = 2,        /* sizes that do not fit together (N_G, K, N_L, B ...)     */
    CF_EBADIDX = 3,       /* a label outside [1, N_Q] or an ic_map outside [1, N_L] */
    CF_ENONFINITE = 4,    /* NaN or Inf in vals or R                                  */
    CF_ECUDA = 5,         /* a CUDA runtime error (message in cf_last_error())       */
    CF_ENOMEM = 6,        /* device or host allocation failed                         */
    CF_ENODEVICE = 7,     /* no CUDA device, or the library was not built for it      */
    CF_EUNSUPPORTED = 8,  /* a form / K combination this build does not provide       */
    CF_ETIMEOUT = 9       /* a bounded device-side wait gave up                       */
} cf_status;

/* Contraction forms.  All compute in FP64 unless stated otherwise. */
typedef enum cf_form {
    CF_FORM_AF = 0,        /* angular first: Phi = sum G f2 (x) f3 per (t,q1) run, then R_t . Phi      */
    CF_FORM_RF = 1,        /* radial first: Psi_z = R_t . (f2 (x) f3) per entry, then Q += G Psi       */
    CF_FORM_AF_EXACT = 2,  /* angular first in the reference's exact operation order (no FMA):
                              reproduces angular_first_collision_kernel_mex bit for bit (K <= 8)        */
    CF_FORM_RF_EXACT = 3,  /* radial first in the reference's exact operation order (no FMA)           */
    CF_FORM_AF_SYM = 4,    /* angular first on the q2 <-> q3 folded operator: the entries (q1,q2,q3) and
                              (q1,q3,q2) share one outer product against R_t + R_t'^T (half the work);
                              needs a COO list that is symmetric in its last two indices (the real
                              Gaunt lists are) and returns CF_EUNSUPPORTED otherwise                   */
    CF_FORM_AF_F32 = 5,    /* angular first in FP32 (f, R, Phi and the row sums rounded to FP32; result
                              added to the FP64 Q): ~1e-7 relative error, the invariant rows stay exactly
                              zero because R's conservation rows are exactly zero in FP32 too          */
    CF_FORM_AF_SYM_F32 = 6, /* the FP32 form on the folded operator                                      */
    CF_FORM_AF_BF16 = 7,   /* angular first with the K^3 step on the BF16 tensor cores as a two-term
                              split: R_t = R_hi + R_lo and Phi = Phi_hi + Phi_lo in BF16, products
                              accumulated in FP32 (the Phi step in FP32); ~1e-5 relative error; K = 8 */
    CF_FORM_AF_SYM_BF16 = 8, /* the BF16-split form on the folded operator                            */
    CF_FORM_AF_SYM_I8 = 9  /* the folded operator with Phi in FP64 and the K^3 step on the int8 tensor
                              cores (tcgen05): Phi and R_t as 47-bit fixed-point integers split into six
                              bytes each, byte products summed exactly in int32 tensor memory, recombined
                              in FP64; ~1e-11 of max|Q|; K = 4, 8 or 12; Q only, cell-major arrays
                              (cf_q_device, cf_contract_host); no counterpart in the reference */,
    CF_FORM_RF_DENSE = 10  /* radial first with the radial step factored out of the entries: per
                              (l-triplet t, q2) a dense [K^2 x K] x [K x cells] product
                              C = R_t x_2 f(q2) over the batch's cells, then K^2 per entry
                              (radial_first_collision_kernel_mex.cpp:41-59 computes K^3 per entry);
                              FP64, on the q2 <-> q3 folded operator where the operator folds; Q only,
                              cell-major arrays (cf_q_device, cf_contract_host); allocates its scratch
                              on first use at a batch size */
} cf_form;

typedef struct cf_plan cf_plan;

typedef struct cf_plan_info {
    int64_t n_g;          /* COO entries                                        */
    int64_t n_slices;     /* runs of equal (ic_map, q1): the S of the K^3 step  */
    int32_t n_l;          /* l-triplets (R channels)                            */
    int32_t n_q;          /* angular modes (L+1)^2                              */
    int32_t k;            /* radial functions per l                             */
    int32_t device;       /* CUDA device the plan lives on                      */
    double  flops_q;      /* algorithmic FLOP per cell for Q:  N_G(2K^2+K) + S 2K^3 */
    double  flops_jv;     /* algorithmic FLOP per cell for J.v: N_G(4K^2+2K) + S 2K^3 */
    int64_t device_bytes; /* device memory held by the plan (COO, R, buffers)   */
    int32_t last_path;    /* kernel family of the plan's last angular-first or J.v launch
                             (1 gather, 2 tile, 3 pair, 4 pair R via L1, 5 split pair; 0 none yet;
                             launches of the folded form count for the plan they fold) */
    int32_t reserved;
} cf_plan_info;

/* ------------------------------------------------------------------------------------------
 * MEX-compatible entry points: host pointers, one call = one contraction, synchronous.
 * The COO/R upload and re-bucketing is cached per content, so repeated calls with the same
 * operator pay only for f and Q.
 * ------------------------------------------------------------------------------------------ */

/* Replaces angular_first_collision_kernel_mex (src/mex/angular_first_collision_kernel_mex.cpp:6-75):
 * Q(N_Q x K) += AF contraction of f(N_Q x K).  N_L is what the MEX implies by numel(R)/K^3. */
int cf_angular_first(double* Q, const double* f, const double* labels, const double* vals,
                     const double* ic_map, const double* R, int64_t n_g, int32_t n_l, int32_t n_q,
                     int32_t k);

/* Replaces radial_first_collision_kernel_mex (src/mex/radial_first_collision_kernel_mex.cpp:5-76). */
int cf_radial_first(double* Q, const double* f, const double* labels, const double* vals,
                    const double* ic_map, const double* R, int64_t n_g, int32_t n_l, int32_t n_q,
                    int32_t k);

/* Batched host-pointer form of both (Q, f: [N_Q x K x B]); form is a cf_form.  The host-side
 * counterpart of calling the reference MEX once per cell (benchmark_collision_contraction_scaling.m:96-108).
 * From 512 cells up, the fast FP64 forms that run on the tile kernel (CF_FORM_AF_SYM with the
 * automatic kernel order; either fast form with kernel path 2) are streamed: one launch over the
 * whole batch starts as soon as the first chunk of cells is on the device and hands each chunk back
 * as soon as it is final, with the same result bits as the device entry points.  Other forms cut
 * the batch into chunks that go up, are contracted and come back on three streams.  Up to 8 cells
 * (one f per call, as the reference's MEX is called), the fast forms CF_FORM_AF, CF_FORM_AF_SYM and
 * CF_FORM_RF (K <= 8 for RF) are one launch of the few-cell kernel, with f and Q_in passed in the
 * launch's parameter block when they fit (2 B N_Q K <= 3968 doubles); cf_angular_first and
 * cf_radial_first take the same route. */
int cf_contract_host(double* Q, const double* f, int64_t b, const double* labels, const double* vals,
                     const double* ic_map, const double* R, int64_t n_g, int32_t n_l, int32_t n_q,
                     int32_t k, int32_t form);

/* n_calls back-to-back calls of cf_contract_host with these arguments (each adds into Q), timed on
 * the host clock in C: *seconds = their total wall time.  A latency benchmark of the host entry point
 * without a foreign-function caller's own per-call cost; stops at the first failing call. */
int cf_time_contract_host(int64_t n_calls, double* seconds, double* Q, const double* f, int64_t b,
                          const double* labels, const double* vals, const double* ic_map, const double* R,
                          int64_t n_g, int32_t n_l, int32_t n_q, int32_t k, int32_t form);

/* J(f).v = Q(v,f) + Q(f,v), accumulated into out; no counterpart in the reference (the reference
 * linearises only densely at equilibrium, tutorial_collisions_spectral_properties.m:43).  Host pointers,
 * [N_Q x K x B].  `exact` is the J.v mode, as for cf_jv_device. */
int cf_jacobian_apply_host(double* out, const double* f, const double* v, int64_t b,
                           const double* labels, const double* vals, const double* ic_map,
                           const double* R, int64_t n_g, int32_t n_l, int32_t n_q, int32_t k,
                           int32_t exact);

/* ------------------------------------------------------------------------------------------
 * Plan API: a device-resident operator and batched contractions on device buffers.
 * Device arrays are in the MEX-native layout [N_Q x K x B].  stream is a cudaStream_t
 * (NULL = the legacy default stream).  Calls are asynchronous on that stream.
 * ------------------------------------------------------------------------------------------ */

/* Validate and upload an operator (host arrays, same conventions as above) to device `device`
 * (-1 = the current device).  The same inputs the reference's GeneralCollisionTensor holds
 * (src/GeneralCollisionTensor.m:9-12). */
int cf_plan_create(cf_plan** plan, const double* labels, const double* vals, const double* ic_map,
                   const double* R, int64_t n_g, int32_t n_l, int32_t n_q, int32_t k,
                   int32_t device);
int cf_plan_destroy(cf_plan* plan);
int cf_plan_get_info(const cf_plan* plan, cf_plan_info* info);

/* Bytes of device scratch the batched calls need for B cells (the tiled copies of the inputs
 * and of the output).  Passing a workspace of at least this size to the *_ws calls makes
 * them allocation-free; the other calls allocate it inside the plan on first use. */
int cf_plan_workspace_size(const cf_plan* plan, int64_t b, int32_t jacobian, size_t* bytes);

/* Q_dev += Q(f_dev) for B cells. */
int cf_q_device(cf_plan* plan, double* q_dev, const double* f_dev, int64_t b, int32_t form,
                void* stream);
int cf_q_device_ws(cf_plan* plan, double* q_dev, const double* f_dev, int64_t b, int32_t form,
                   void* workspace, size_t workspace_bytes, void* stream);

/* out_dev += J(f_dev).v_dev for B cells.  `exact` selects the mode of every J.v call:
 * 0 = fast, 1 = exact operation order (every K; above K = 8 on the row kernel, at most 65535 cells
 * per call), 2 = the q2 <-> q3 folded operator (as CF_FORM_AF_SYM),
 * 3 = FP32 (f, v, R, Phi and the row sums in FP32, added into the FP64 out, as CF_FORM_AF_F32; even
 * K <= 12), 4 = FP32 on the folded operator.  cf_jv_tiled takes modes 0-2 (its tiles are FP64). */
int cf_jv_device(cf_plan* plan, double* out_dev, const double* f_dev, const double* v_dev,
                 int64_t b, int32_t exact, void* stream);

/* Tiled cell layout: [ceil(B/32)][N_Q][K][32] (32 cells per tile, cell index fastest).  Callers
 * that keep their cells resident (time steppers, Krylov solvers) use it directly and skip the
 * two layout passes.  cf_pack_cells / cf_unpack_cells convert from / to [N_Q x K x B]; pack fills
 * the padding cells of the last tile with zeros, unpack overwrites the B cells of dst.  The exact
 * forms above K = 8 (Q and J.v) run on cell-major arrays only: the tiled entries refuse them with
 * CF_EUNSUPPORTED. */
int cf_pack_cells(const cf_plan* plan, double* dst_tiled, const double* src_cells, int64_t b, void* stream);
int cf_unpack_cells(const cf_plan* plan, double* dst_cells, const double* src_tiled, int64_t b, void* stream);
int cf_q_tiled(cf_plan* plan, double* q_tiled, const double* f_tiled, int64_t b, int32_t form, void* stream);
int cf_jv_tiled(cf_plan* plan, double* out_tiled, const double* f_tiled, const double* v_tiled, int64_t b,
                int32_t exact, void* stream);

/* Kernel family of a plan's angular-first and Jacobian contractions: 0 = automatic (the first of
 * pair, tile, gather that fits; tile before pair for the fast Q form of the folded operator, whose
 * lighter Phi step favours the tile kernel's higher occupancy; the l-block kernel for the fast Q
 * forms, plain and folded, at K = 12), 1 = the gather kernel (warp per row and 32-cell tile,
 * f read through L1/L2), 2 = the tile-resident kernel (16 cells in shared memory, Phi split over
 * two lanes per cell), 3 = the pair kernel (16 cells in shared memory, the mirrored rows (l,+m) and
 * (l,-m) on the two half-warps), 4 = the pair kernel reading R through L1 instead of shared
 * memory, 5 = the split pair kernel (both mirrored rows in every lane, the k3 range split over the
 * half-warps; fast Q forms with even K <= 8, the pair kernel otherwise), 6 = the tile kernel with
 * its K^3 step on the FP64 tensor cores (warp-level MMA; fast Q form at K = 8, the tile kernel
 * otherwise), 11 = the band kernel (fast FP64 Q forms on l1-band work units, K = 4, 8, 12), 14 = the
 * l-block kernel (one CTA per l1 band and 8 cells, R_t plus the f rows of bands l2 and l3 staged per
 * l-triplet by bulk copies, the band's slices taken by the warps one at a time; fast FP64 Q forms,
 * K = 8 and 12).  2-6, 11 and 14 return
 * CF_EUNSUPPORTED where they do not fit.  All families agree to rounding, and bit for bit in the
 * exact forms. */
int cf_plan_set_kernel_path(cf_plan* plan, int32_t path);

/* Measured FP64 FMA throughput of `device` in TFLOP/s (independent DFMA chains on every SM, timed
 * with CUDA events): the peak the FP64 forms are compared against. */
int cf_fp64_fma_peak(int32_t device, double* tflops);

/* Q_dev += Q(f_dev) for B cells without allocating anything: no cudaMalloc, cudaFree or other
 * allocating routine runs inside this call.  No counterpart in the reference (its MEX kernels
 * run on the host).  It is for callers that cannot let a library allocate device memory -- a
 * host whose device memory is all owned by its own allocator, or code about to record work into
 * a stream capture -- which cf_q_device does on its first use of a batch size.  The scratch (the
 * tiled copies of f and Q) lives in a fixed array of CF_NOALLOC_SCRATCH_BYTES inside the library,
 * which each device holds from the first call on that device until the process exits; batches
 * whose 2 * ceil(B/32) * 32 * N_Q * K doubles do not fit are rejected with CF_ESHAPE (about 4300
 * cells at N_Q*K = 968), whichever kernel route the batch would take, including the routes that
 * leave the array unused.  The first call on a device looks up the array's device address with
 * that device current; make that first call before any stream capture.  All calls share the one
 * array, so calls that overlap on the GPU (other streams, other host threads) race on it.  The
 * plan itself is created beforehand with cf_plan_create, which does allocate, and so is its folded
 * operator: the folded forms (CF_FORM_AF_SYM and its FP32 / BF16 variants) return CF_EINVAL until
 * one cf_q_device or cf_q_tiled call in a folded form has built it.  The same holds for the tables
 * of the band kernels (kernel paths 11 and 14, the BF16-split forms at K = 4 and 12, and the fast
 * forms at K = 12, which run on the l-block kernel): one cf_q_device call in the form
 * builds them. */
#define CF_NOALLOC_SCRATCH_BYTES ((size_t)64 << 20)
int cf_q_device_noalloc(cf_plan* plan, double* q_dev, const double* f_dev, int64_t b, int32_t form,
                        void* stream);

/* Self-test of the streamed host path's bounded wait (no counterpart in the reference): launches
 * the streamed tile kernel of `plan` (even K <= 8) over 64 cells whose data and ready flags are
 * never sent, so every CTA's wait runs out after wait_seconds (0 < wait_seconds <= 10) and the
 * kernel returns.  Returns CF_ETIMEOUT when the wait gave up and reported it, as it should; the
 * plan's device scratch then holds garbage, nothing else is touched. */
int cf_plan_stream_selftest(cf_plan* plan, double wait_seconds);

/* Self-test of the l-block kernel's bounded waits (no counterpart in the reference): launches the
 * FP64 l-block kernel of `plan` (K = 8 or 12; builds the plan's band tables on first use) over 16
 * zero cells with no stage of R_t and f ever copied in, so every CTA's wait runs out after
 * wait_seconds (0 < wait_seconds <= 10) and the kernel returns through its normal exit.  Returns
 * CF_ETIMEOUT when the waits gave up and reported it, as they should; the plan's device scratch
 * then holds garbage, nothing else is touched. */
int cf_plan_lblock_selftest(cf_plan* plan, double wait_seconds);

/* ------------------------------------------------------------------------------------------
 * Ragged batches: cells of several resolutions (one plan per (L, K) bucket) contracted in ONE
 * persistent launch.  cells[b] is bucket b's cell count; q_dev[b], f_dev[b] are its
 * [N_Q x K x cells[b]] device arrays.  forms[b] (NULL: all CF_FORM_AF) is the FP64 form of bucket b:
 * buckets in CF_FORM_AF or CF_FORM_AF_SYM with K <= 8 share the fused launch, any other bucket runs
 * its own plan's kernels in the same step.  family picks the routine of the fused launch: 0 the
 * pair routine (8 warps per CTA), 1 the tile routine (16 warps per CTA; buckets of odd K then run
 * on their own).  tail_split (0, 4 or 16) is how many bins each of the last half-tiles of the fused
 * work table is cut into, so that the launch ends evenly.
 * cf_ragged_q enqueues pack, fused launch, the separate buckets and unpack on the stream (when every
 * non-empty bucket is fused on the tile routine: one launch on the cell-major arrays instead);
 * cf_ragged_graph_launch records that sequence into a CUDA graph on first use (per set of buffers)
 * and replays it.  No counterpart in the reference (it contracts one f at a time).
 * ------------------------------------------------------------------------------------------ */
typedef struct cf_ragged cf_ragged;
int cf_ragged_create(cf_ragged** ragged, cf_plan* const* plans, const int64_t* cells, const int32_t* forms,
                     int32_t n_buckets, int32_t tail_split, int32_t family);
int cf_ragged_destroy(cf_ragged* ragged);
int cf_ragged_q(cf_ragged* ragged, double* const* q_dev, const double* const* f_dev, void* stream);
int cf_ragged_graph_launch(cf_ragged* ragged, double* const* q_dev, const double* const* f_dev, void* stream);
/* The contraction alone on the handle's resident tiled buffers, as the last cf_ragged_q or
 * cf_ragged_graph_launch left them (Q_tiled += Q(f_tiled)): the step without its layout passes. */
int cf_ragged_q_resident(cf_ragged* ragged, void* stream);
/* q_host[b] += Q(f_host[b]) for every bucket, with host arrays [N_Q x K x cells[b]]; synchronous.
 * No counterpart in the reference.  When every non-empty bucket runs in the fused launch on the tile
 * routine (family 1), the batch is streamed: each bucket goes up in chunks of whole half-tiles in the
 * order the fused launch takes them, one launch starts on the first chunk, and each chunk comes back
 * as soon as it is final, with the same result bits as cf_ragged_q.  Any other handle copies every
 * bucket up, runs the cf_ragged_q step and copies back.  The first call allocates the handle's
 * device copies of the buckets; pinned host memory makes the copies asynchronous. */
int cf_ragged_q_host(cf_ragged* ragged, double* const* q_host, const double* const* f_host);
/* Work units of the fused table, CTAs of the fused launch, its dynamic shared memory and the number
 * of buckets it contracts (the others run their own kernels). */
int cf_ragged_info(const cf_ragged* ragged, int32_t* n_units, int32_t* ctas, int64_t* smem_bytes, int32_t* n_fused);

/* ------------------------------------------------------------------------------------------
 * The reduced radial tensor R on the GPU: replaces compute_rtensor_sumfac_mex
 * (src/mex/compute_rtensor_sumfac_mex.cpp:80-397), whose 26 inputs GeneralCollisionTensor.m:177-181
 * prepares; the fields below are those inputs in order (arrays column-major doubles as MATLAB
 * passes them, sizes taken from their lengths).  R_out (host, N_K^3 x N_L doubles with
 * N_K = k_max + 1) receives the quadrature, before the conservation rows are zeroed (the driver
 * does that, GeneralCollisionTensor.m:184-191).  k_max + 1 <= 12, N_Q = (L+1)^2 with L <= 31.
 * ------------------------------------------------------------------------------------------ */
typedef struct cf_sumfac_inputs {
    int32_t k_max, n_l, n_q;
    double alpha;                                   /* gamma: B = |u|^gamma                       */
    const double *x_nodes, *w_x;   int32_t n_x;     /* generalised Laguerre nodes and weights     */
    const double *u1_nodes, *w_u1; int32_t n_u1;    /* patch 1: u outer                           */
    const double *t1_nodes, *w_t1; int32_t n_t1;    /* patch 1: t inner                           */
    const double *y2_nodes, *w_y2; int32_t n_y2;    /* patch 2: y outer                           */
    const double *t2_nodes, *w_t2; int32_t n_t2;    /* patch 2: t inner                           */
    const double *mu_chi, *w_chi;  int32_t n_chi;   /* scattering angle cosines                   */
    const double *eps, *w_eps;     int32_t n_eps;   /* azimuths                                   */
    const double *radial_norm;                      /* [N_K x (L+1)]                               */
    const double *sh_norm;                          /* [N_Q]                                       */
    const double *l_triplets;                       /* [N_L x 3]                                   */
    const double *qi_valid;                         /* [N_Q x N_L], 1-based, -1 terminated         */
    const double *p_loss_p1;                        /* [n_t1 x n_u1 x N_L]                         */
    const double *p_gain_p1;                        /* [n_t1 x n_u1 x N_Q x N_L]                   */
    const double *p_loss_p2;                        /* [n_y2 x N_L]                                */
    const double *p_gain_p2;                        /* [n_y2 x N_Q x N_L]                          */
} cf_sumfac_inputs;
/* device_seconds (may be NULL) receives the device time of the quadrature kernels. */
int cf_rtensor_sumfac(double* R_out, const cf_sumfac_inputs* inputs, int32_t device, double* device_seconds);
/* The same quadrature with the two gain tables passed already compressed to the valid (q_i, channel)
 * pairs, so that the dense [n_t1 x n_u1 x N_Q x N_L] table (20 GB at L = 16, K_max = 11, pad 20)
 * never exists; inputs->p_gain_p1 / p_gain_p2 are ignored.  The pairs j = 0..nnz-1 run over the
 * channels in order and, within a channel, over its qi_valid list up to the first -1; the tables are
 * p_gain_p1_packed[(u * n_t1 + t) * nnz + j] = P_gain_p1[t, u, q_j, ch_j] and
 * p_gain_p2_packed[y * nnz + j] = P_gain_p2[y, q_j, ch_j].  Results equal cf_rtensor_sumfac's bit for
 * bit on the same tables.  No counterpart in the reference (compute_rtensor_sumfac_mex.cpp:80-397
 * takes the dense tables). */
int cf_rtensor_sumfac_packed(double* R_out, const cf_sumfac_inputs* inputs, const double* p_gain_p1_packed,
                             const double* p_gain_p2_packed, int32_t device, double* device_seconds);

/* ------------------------------------------------------------------------------------------
 * Explicit time stepping df/dt = Q(f) for a batch of cells, Heun's method (RK2):
 * f <- f + dt/2 (Q(f) + Q(f + dt Q(f))), n_steps times, in the tiled layout (cf_pack_cells), with
 * the contraction in `form` (any FP64 form).  The reference steps one cell with its dense tensor
 * (tutorial_stress_relaxation.m:77-91, tutorial_collisions_bwu_solution.m:77-92).  The workspace
 * (cf_rk2_workspace_size bytes) holds the two stage values and the intermediate state; a step
 * allocates nothing and never synchronises, so n steps can be recorded into a CUDA graph.
 * ------------------------------------------------------------------------------------------ */
int cf_rk2_workspace_size(const cf_plan* plan, int64_t b, size_t* bytes);
int cf_rk2_steps_tiled(cf_plan* plan, double* f_tiled, int64_t b, double dt, int32_t n_steps, int32_t form,
                       void* workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------------------------------
 * Implicit solves: (I - dt J(f)) x = b per cell with restarted GMRES, FP64.  No counterpart in
 * the reference (it steps only explicitly, with a dense tensor: tutorial_stress_relaxation.m:77-91).
 * All vectors are device arrays in the tiled layout (cf_pack_cells).  x holds the initial guess on
 * entry.  Preconditioning is on the right with block-Jacobi over the angular modes: `precond` is
 * NULL (none), N_Q blocks of K x K shared by all cells (precond_per_cell = 0), or B sets of N_Q
 * blocks (precond_per_cell = 1); block q maps rows q*K..q*K+K-1 (row-major, [out][in]).  A cell
 * is done when |b - A x| <= tol |b| in FP64.  J(f) u runs on the q2 <-> q3 folded operator when
 * the operator folds (the same bilinear form on half the entries), else on the plain one.
 * iters_out[B] (host, may be NULL) receives the
 * Arnoldi steps each cell used, relres_out[B] (host, may be NULL) the final relative residuals.
 * Returns CF_ETIMEOUT if some cell is still above tol after max_iters steps.
 * ------------------------------------------------------------------------------------------ */
int cf_gmres_workspace_size(const cf_plan* plan, int64_t b, int32_t restart, size_t* bytes);
int cf_gmres_solve_tiled(cf_plan* plan, const double* f_tiled, double dt, const double* b_tiled,
                         double* x_tiled, int64_t b, int32_t restart, int32_t max_iters, double tol,
                         const double* precond, int32_t precond_per_cell, int32_t* iters_out,
                         double* relres_out, void* workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------------------------------
 * Learned block preconditioner (no counterpart in the reference).  A small FP32 network maps a
 * cell's features (its coefficients and log10(dt nu)) to a correction Delta of the Maxwellian
 * blocks: P_q = P_eq,q + scale * Delta_q.  x -> Linear -> GELU -> Linear -> GELU -> Linear,
 * weights [out][in]; all products are this library's SGEMM kernels; Adam trains it.
 * ------------------------------------------------------------------------------------------ */
typedef struct cf_mlp cf_mlp;
int cf_mlp_create(cf_mlp** mlp, int32_t n_in, int32_t n_hidden, int32_t n_out, int32_t max_batch,
                  uint64_t seed, int32_t device);
int cf_mlp_destroy(cf_mlp* mlp);
int cf_mlp_num_params(const cf_mlp* mlp, int64_t* n);
/* dir 0: parameters device -> host, 1: host -> device, 2: gradients device -> host (flat layout
 * W1, b1, W2, b2, W3, b3, each padded to a multiple of 64 floats). */
int cf_mlp_copy(cf_mlp* mlp, float* host, int32_t dir);
/* y[n][n_out] = net(x[n][n_in]) (device arrays); train != 0 keeps the activations for backward. */
int cf_mlp_forward(cf_mlp* mlp, const float* x, float* y, int64_t n, int32_t train, void* stream);
/* Parameter gradients of sum(dy .* y) for the last training forward pass on the same x. */
int cf_mlp_backward(cf_mlp* mlp, const float* x, const float* dy, int64_t n, void* stream);
int cf_mlp_adam_step(cf_mlp* mlp, float lr, float beta1, float beta2, float eps, float weight_decay,
                     void* stream);
/* Probe loss of P = P_eq + scale * Delta for n cells: with probe pairs v_p and a_p = A v_p
 * (av, v: [n][n_probes][N_Q*K] FP32, block q at q*K; vnorm2: [n][n_probes] = |v_p|^2),
 * L = mean over cells of (1/n_p) sum_p sum_q |P_q a_pq - v_pq|^2 / |v_p|^2, accumulated into
 * *loss_dev (device), and dL/dDelta into grad [n][N_Q][K][K]. */
int cf_precond_probe_loss(const float* delta, const double* peq, const float* av, const float* v,
                          const float* vnorm2, float scale, int64_t n, int32_t n_probes, int32_t n_q,
                          int32_t k, float* grad, double* loss_dev, void* stream);
/* P [n][N_Q][K][K] (FP64) = P_eq + scale * Delta: the per-cell blocks cf_gmres_solve_tiled applies. */
int cf_precond_assemble(const float* delta, const double* peq, double* P, float scale, int64_t n,
                        int32_t n_q, int32_t k, void* stream);

/* ------------------------------------------------------------------------------------------
 * Status and introspection
 * ------------------------------------------------------------------------------------------ */
const char* cf_status_string(int status);
/* Detail of the last failing call on this host thread ("" if none). */
const char* cf_last_error(void);
/* Number of CUDA kernel launches this library has issued in this process. */
int64_t cf_launch_count(void);
/* How the last host call of at most 8 cells on this thread moved its data: 0 it did not take the
 * few-cell kernel, 1 f and Q_in in the launch's parameter block (Q_out written to mapped pinned
 * memory), 2 copies through pinned staging and a device buffer. */
int cf_few_route_last(void);
/* Library version string. */
const char* cf_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CF_B200_H */
