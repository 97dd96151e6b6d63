// Allocation-free variant of the half-step pair (tipt_rk2_fused_table).
//
// Some callers cannot call cudaMalloc: code running while another library
// captures a CUDA graph on the stream (allocation is illegal during capture),
// hosts embedding the stepper without a device allocator of their own, and
// real-time loops that must not allocate.  The half-step pair needs the
// intermediate state between its two halves; this entry point keeps that
// state in a file-scope device array instead of caller memory.
//
// The array is kNoAllocBytes (8 MiB) and every GPU that loads the library
// holds it until the process exits.  It is shared by every call: calls whose
// work overlaps on the GPU (different streams, or different host threads on
// one device) race on it and must be serialised by the caller.  Its contents
// are whatever the last call left there; each call overwrites the part it
// uses before reading it, so nothing needs clearing.
//
// In host code the array's name is only a host-side stand-in, never a device
// address: the device address is obtained once per device, with that device
// current, through cudaGetSymbolAddress on the first call, so the first call
// on each device should come before any stream capture.
#include <mutex>

#include "tipt_internal.h"

namespace tipt {

constexpr size_t kNoAllocBytes = 8u << 20;
static __device__ __align__(256) unsigned char g_mid_state[kNoAllocBytes];

constexpr int kMaxDevices = 64;
static std::mutex g_mid_mu;
static void* g_mid_addr[kMaxDevices] = {};

// Device address of g_mid_state on the current device (looked up once per device).
static int mid_state_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail_cuda(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices)
        return fail(TIPT_ERR_UNSUPPORTED, "device ordinal %d beyond %d", dev, kMaxDevices);
    std::lock_guard<std::mutex> lock(g_mid_mu);
    if (!g_mid_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_mid_state);
        if (e != cudaSuccess) return fail_cuda(e, "cudaGetSymbolAddress(intermediate state)");
        g_mid_addr[dev] = p;
    }
    *out = g_mid_addr[dev];
    return TIPT_OK;
}

}  // namespace tipt

using namespace tipt;

extern "C" int tipt_rk2_fused_table_noalloc(int storage, const void* phi, const void* pi,
                                            void* phi_out, void* pi_out, int64_t nx, int64_t ny,
                                            int64_t nz, const tipt_step_params* sp,
                                            const tipt_vsource* vp_T, const tipt_vsource* vp_Tm,
                                            const void* noise, void* stream) {
    int rc;
    if ((rc = check_storage(storage)) || (rc = check_dims(nx, ny, nz))) return rc;
    // intermediate phi and pi, the second block 256-byte aligned
    const size_t field = (size_t)(nx * ny * nz) * (size_t)elem_bytes(storage);
    const size_t off = (field + 255) & ~(size_t)255;
    if (off + field > kNoAllocBytes)
        return fail(TIPT_ERR_UNSUPPORTED,
                    "lattice of %lld sites needs %zu bytes of intermediate state; the "
                    "allocation-free entry point holds at most %zu bytes (use "
                    "tipt_rk2_fused_table with caller scratch)",
                    (long long)(nx * ny * nz), off + field, kNoAllocBytes);
    void* base = nullptr;
    if ((rc = mid_state_address(&base))) return rc;
    unsigned char* b = static_cast<unsigned char*>(base);
    return tipt_rk2_fused_table(storage, phi, pi, phi_out, pi_out, b, b + off, nx, ny, nz, sp,
                                vp_T, vp_Tm, noise, stream);
}
