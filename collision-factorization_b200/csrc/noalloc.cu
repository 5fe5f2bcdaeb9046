// noalloc.cu -- the allocation-free variant of the batched Q(f) contraction.
//
// cf_q_device needs device scratch (the tiled copies of f and Q) and allocates it inside the plan
// on first use.  Some callers cannot let a library call cudaMalloc: a host that owns every byte of
// device memory through its own allocator, or a caller about to record its work into a stream
// capture.  For them, cf_q_device_noalloc runs the same contraction with its scratch in the
// file-scope array below instead.  The array is a fixed CF_NOALLOC_SCRATCH_BYTES on every device
// that loads this module and stays allocated until the process exits.
//
// Host code may not pass g_noalloc_scratch to a kernel directly: on the host the symbol is a
// host-side stand-in, not a device address.  The device address is looked up once per device,
// with that device current, by cudaGetSymbolAddress on the first call made on that device.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/cf_b200.h"

// Sets the message cf_last_error() returns (plan.cu; not part of the C ABI).
void cf_set_last_error(const char* msg);
bool cf_plan_folded_built(cf_plan* plan);
bool cf_plan_band_pending(cf_plan* plan, int form);

namespace {

constexpr size_t kScratchBytes = CF_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

int scratch_for_device(int device, void** out) {
    if (device < 0 || device >= kMaxDevices) {
        cf_set_last_error("cf_q_device_noalloc: device index out of range");
        return CF_ENODEVICE;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_scratch_ptr[device] == nullptr) {
        int prev = -1;
        cudaError_t e = cudaGetDevice(&prev);
        if (e != cudaSuccess) {
            cf_set_last_error((std::string("cf_q_device_noalloc: cannot read the current device: ") +
                               cudaGetErrorString(e)).c_str());
            return CF_ECUDA;
        }
        if (prev != device && (e = cudaSetDevice(device)) != cudaSuccess) {
            cf_set_last_error((std::string("cf_q_device_noalloc: cannot select device ") + std::to_string(device) +
                               ": " + cudaGetErrorString(e)).c_str());
            return CF_ENODEVICE;
        }
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (prev != device) cudaSetDevice(prev);
        if (e != cudaSuccess || p == nullptr) {
            cf_set_last_error((std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e)).c_str());
            return CF_ECUDA;
        }
        g_scratch_ptr[device] = p;
    }
    *out = g_scratch_ptr[device];
    return CF_OK;
}

}  // namespace

extern "C" int cf_q_device_noalloc(cf_plan* plan, double* q_dev, const double* f_dev, int64_t b, int32_t form,
                                   void* stream) {
    if (!plan) return CF_EINVAL;
    cf_plan_info info;
    int st = cf_plan_get_info(plan, &info);
    if (st != CF_OK) return st;
    // The split form builds its own device tables on first use (and keeps an error word): refused.
    if (form == CF_FORM_RF_DENSE) {
        cf_set_last_error("cf_q_device_noalloc: the radial-first dense form (CF_FORM_RF_DENSE) allocates its scratch; "
                          "use cf_q_device");
        return CF_EUNSUPPORTED;
    }
    if (form == CF_FORM_AF_SYM_I8) {
        cf_set_last_error("cf_q_device_noalloc: the split form (CF_FORM_AF_SYM_I8) is not available without "
                          "allocation; use cf_q_device");
        return CF_EUNSUPPORTED;
    }
    // The folded forms run on the plan's folded twin, which its first use builds, with allocations.
    const bool folded = form == CF_FORM_AF_SYM || form == CF_FORM_AF_SYM_F32 || form == CF_FORM_AF_SYM_BF16;
    if (folded && !cf_plan_folded_built(plan)) {
        cf_set_last_error("cf_q_device_noalloc: this plan's folded operator is not built yet, and building it "
                          "allocates; make one cf_q_device or cf_q_tiled call in a folded form first");
        return CF_EINVAL;
    }
    // The band kernels' tables (BF16-split forms at K = 4 and 12; path 'band') are built on first use.
    if (cf_plan_band_pending(plan, form)) {
        cf_set_last_error("cf_q_device_noalloc: this plan's band-kernel tables are not built yet, and building "
                          "them allocates; make one cf_q_device call in this form first");
        return CF_EINVAL;
    }
    // The limit is checked for every batch, also where the route taken (the streamed tile kernel,
    // the few-cell kernel) would leave the array unused: the size a call may pass does not depend
    // on the route the library picks for it.
    size_t need = 0;
    st = cf_plan_workspace_size(plan, b, 0, &need);
    if (st != CF_OK) return st;
    if (need > kScratchBytes) {
        char msg[256];
        snprintf(msg, sizeof(msg),
                 "cf_q_device_noalloc: B = %lld cells of N_Q*K = %d need %zu bytes of scratch, more than the "
                 "fixed %zu (use cf_q_device or cf_q_device_ws for larger batches)",
                 (long long)b, info.n_q * info.k, need, kScratchBytes);
        cf_set_last_error(msg);
        return CF_ESHAPE;
    }
    void* scratch = nullptr;
    st = scratch_for_device(info.device, &scratch);
    if (st != CF_OK) return st;
    return cf_q_device_ws(plan, q_dev, f_dev, b, form, scratch, kScratchBytes, stream);
}

