// common.cuh -- device-side operator layout shared by the contraction kernels.
//
// HBM layout of one uploaded operator (built on the host by plan.cu):
//
//   slices     runs of equal (t, q1) of the caller's COO list, grouped by q1 (each q1's runs
//              keep the caller's order, so Q[q1] receives its contributions in the same
//              order as in the reference's angular-first loop).
//   q1_begin   [N_Q+1]  slice range of each q1
//   slice_t    [S]      l-triplet of each slice (0-based)
//   slice_e    [S+1]    entry range of each slice
//   e_q23      [N_G]    packed 0-based (q2 | q3 << 16) of each entry, in slice order
//   e_g        [N_G]    Gaunt value of each entry, in slice order
//   R          [K^3 N_L] reduced radial tensor, R[k1 + K k2 + K^2 k3 + K^3 t]
//   item_q1    [n_items] the q1 values that have slices, heaviest first
//
// Cell data is kept in a tiled "cell-fastest" layout: 32 cells per tile, one per lane,
//   X_tiled[tile][q][k][lane]   (row r = q*K + k, 32 doubles = 256 B per row)
// so a warp that handles 32 cells reads one contiguous 256-byte line per (q, k) and every
// COO entry is uniform across the warp.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define CF_TILE 32

struct DevOp {
    const int* q1_begin;
    const int* slice_t;
    const int* slice_e;
    const uint32_t* e_q23;
    const double* e_g;
    const double* R;
    const float* R32;  // FP32 copy of R for the FP32 form
    const double* RT;  // K = 8 only: R_t transposed to [k1][kk = K k2 + k3] (A operands of the MMA kernel)
    const unsigned short* RTbf;  // K = 8 only: R_t^T split in BF16, [t][hi, lo][k1][kk] (BF16-split form)
    const int* item_q1;
    int grouped;  // each slice's entries sorted by q2 (the folded operator); bit 0: the fast Q tile
                  // routine sums G f(q3) over each run of equal q2 before one outer product with
                  // f(q2), bit 1: the fast J.v tile routine does the same with f and v
    int n_items;  // number of q1 with at least one slice
    int n_q;
    int k;
    int n_l;
};

// Batches of at most this many cells take the few-cell kernel (few_kernels.cuh).
constexpr int kFewCells = 8;

// Synchronisation words of the streamed tile kernel (tile_kernels.cuh, af_tile_stream_kernel).
struct StreamSync {
    const int* ready;  // [n_chunks] device; == epoch once chunk c's f and Q are in
    int* done;         // [n_chunks] device; units finished (zeroed before the launch)
    int* host_done;    // [n_chunks] mapped host memory; set to epoch once chunk c is final
    int* err;          // mapped host memory; set to 1 if a wait gave up
    int* abort;        // device; == epoch once a wait gave up (the other CTAs then stop waiting)
    int epoch;
    int ht_per_chunk;
    long long wait_cycles;
};

// Lanes per cell used by the angular-first kernels: the K x K Phi accumulator of one cell
// is split over P lanes (by k3 column) once it no longer fits one lane's registers.
__host__ __device__ constexpr int af_lanes_per_cell(int K) { return K <= 8 ? 1 : (K <= 12 ? 2 : 4); }
