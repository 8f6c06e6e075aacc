// Field operator apply that allocates nothing (mpm_field_apply_noalloc).
//
// Some callers cannot call cudaMalloc while they solve: a process whose
// device memory has been handed to another allocator (a framework's caching
// pool that owns nearly all of the GPU), or a real-time loop that must not
// hit the driver's allocator between steps.  For them the reciprocal-space
// grid -- the only scratch the operator needs beyond the field object's own
// per-frame data -- lives in the file-scope device array below instead of a
// cudaMalloc'd buffer.  Every GPU that loads this library holds these
// kNoAllocScratchBytes until the process exits.
#include "../../include/cumpm_b200.h"

#include <mutex>
#include <string>

#include "mpm_capi_internal.h"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;  // 16 MiB per device
constexpr int kMaxDevices = 64;

// Shared by every call: the last call's grid stays here.  Calls that overlap
// on the GPU (different streams, different threads) race on it.
static __device__ __align__(256) unsigned char g_noalloc_grid[kNoAllocScratchBytes];

std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

// Device address of the array on the current device, looked up once per
// device with that device current.  A host-side reference to the symbol is
// not a device address, so kernels only ever receive this pointer.
void* scratch_on_current_device() {
    int dev = -1;
    MPM_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw std::runtime_error("device ordinal out of range");
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        MPM_CUDA(cudaGetSymbolAddress(&p, g_noalloc_grid));
        g_addr[dev] = p;
    }
    return g_addr[dev];
}

}  // namespace

extern "C" {

size_t mpm_noalloc_scratch_bytes(void) { return kNoAllocScratchBytes; }

int mpm_field_apply_noalloc(mpm_field* f, const void* X, void* Y, int M, const void* self_coef, int jacobi,
                            int recip_fp32, int real_fp32, void* stream) {
    return mpm::capi_guard([&] {
        if (!f) throw std::invalid_argument("field must not be NULL");
        if (!X || !Y) throw std::invalid_argument("X and Y must not be NULL");
        if (M < 1) throw std::invalid_argument("M must be >= 1");
        if (jacobi && !self_coef) throw std::invalid_argument("jacobi scaling needs self coefficients");
        if (f->impl->spec().kind == mpm::FIELD_MONO) {
            const size_t need = f->impl->grid_bytes(M, recip_fp32 == 0);
            if (need > kNoAllocScratchBytes)
                throw std::invalid_argument("mpm_field_apply_noalloc: reciprocal grid of " + std::to_string(need) +
                                            " bytes exceeds the " + std::to_string(kNoAllocScratchBytes) +
                                            "-byte static scratch; use fewer right-hand sides or mpm_field_apply");
        }
        void* scratch = scratch_on_current_device();
        f->impl->apply_scratch(static_cast<const double2*>(X), static_cast<double2*>(Y), M,
                               static_cast<const double2*>(self_coef), jacobi != 0, recip_fp32 != 0, real_fp32 != 0,
                               scratch, kNoAllocScratchBytes, static_cast<cudaStream_t>(stream));
    });
}

}  // extern "C"
