// zm_static.cu -- inverse transform without any device allocation.
//
// zm_fft_inverse needs one field of intermediate storage: either the caller's input
// (which it then overwrites) or a caller-provided workspace.  Callers that own no
// spare device memory and may not allocate any -- a plugin whose host application
// controls every device allocation, or a loop under a fixed memory budget that must
// not grow or wait on an allocator -- and that also need their input kept intact, get
// this variant: the intermediate lives in a scratch array that is part of the library
// image, so the call allocates nothing.
#include <cuda_runtime.h>

#include <mutex>

#include "zm_internal.h"
#include "zmodel_b200.h"

// One per device that loads this library; held until the process exits.
static __device__ __align__(256) unsigned char zm_static_scratch[ZM_STATIC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void *g_scratch_addr[kMaxDevices] = {nullptr};
}  // namespace

extern "C" int zm_fft_inverse_static(zm_plan plan, const void *in, void *out, double scale_re,
                                     double scale_im, void *stream) {
    zm_plan_info info;
    int rc = zm_plan_get_info(plan, &info);
    if (rc != ZM_OK) return rc;
    if (info.field_bytes > (size_t)ZM_STATIC_SCRATCH_BYTES)
        return zm::report_error(ZM_ERR_WORKSPACE,
                                "zm_fft_inverse_static: field of %zu bytes exceeds the %zu-byte "
                                "static scratch; use zm_fft_inverse with a workspace",
                                info.field_bytes, (size_t)ZM_STATIC_SCRATCH_BYTES);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return zm::report_error(ZM_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return zm::report_error(ZM_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
    void *scratch = nullptr;
    {
        // First call on this device: the symbol's device address, looked up with this
        // device current.  The host-side name of the array is not a device address.
        // It is cached for the process's life; a cudaDeviceReset would make it stale
        // (the header tells callers not to use this function after one).
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        if (!g_scratch_addr[dev]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, zm_static_scratch);
            if (e != cudaSuccess || !p)
                return zm::report_error(ZM_ERR_CUDA, "cudaGetSymbolAddress(static scratch): %s",
                                        cudaGetErrorString(e));
            g_scratch_addr[dev] = p;
        }
        scratch = g_scratch_addr[dev];
    }
    return zm_fft_inverse(plan, in, out, scratch, scale_re, scale_im, stream);
}
