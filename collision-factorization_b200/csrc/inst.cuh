// inst.cuh -- the body of one per-K translation unit (included by inst_k<K>.cu with CF_K defined).
#pragma once
#include "kernels.cuh"
#include "launch.cuh"

namespace cf {

template <int K, int P, bool EXACT, bool JV>
static LaunchResult launch_af(const LaunchArgs& a) {
    const int64_t warps = (int64_t)a.op.n_items * a.n_tiles * P;
    if (warps == 0) return {0, 0, cudaSuccess};
    const int64_t blocks = (warps + 3) / 4;
    if (blocks > INT32_MAX) return {2, 0, cudaSuccess};
    af_kernel<K, P, EXACT, JV><<<(unsigned)blocks, 128, 0, a.stream>>>(a.op, a.fT, a.vT, a.QT, (int)a.n_tiles);
    const cudaError_t e = cudaGetLastError();
    return {e == cudaSuccess ? 0 : 5, 1, e};
}

template <int K, bool EXACT>
static LaunchResult launch_rf(const LaunchArgs& a) {
    const int64_t warps = (int64_t)a.op.n_items * a.n_tiles;
    if (warps == 0) return {0, 0, cudaSuccess};
    const int64_t blocks = (warps + 3) / 4;
    if (blocks > INT32_MAX) return {2, 0, cudaSuccess};
    rf_kernel<K, EXACT><<<(unsigned)blocks, 128, 0, a.stream>>>(a.op, a.fT, a.QT, (int)a.n_tiles);
    const cudaError_t e = cudaGetLastError();
    return {e == cudaSuccess ? 0 : 5, 1, e};
}

template <int K>
static LaunchResult launch_for_k(const LaunchArgs& a) {
    if (a.what == OP_RF) return a.exact ? launch_rf<K, true>(a) : launch_rf<K, false>(a);
    if constexpr (K <= 8) {
        if (a.exact)
            return a.what == OP_JV ? launch_af<K, 1, true, true>(a) : launch_af<K, 1, true, false>(a);
    } else {
        if (a.exact) return {8, 0, cudaSuccess};
    }
    return a.what == OP_JV ? launch_af<K, jv_P(K), false, true>(a) : launch_af<K, af_P(K), false, false>(a);
}

}  // namespace cf

#define CF_CAT2(a, b) a##b
#define CF_CAT(a, b) CF_CAT2(a, b)
namespace cf {
LaunchResult CF_CAT(launch_k, CF_K)(const LaunchArgs& a) { return launch_for_k<CF_K>(a); }
}  // namespace cf
