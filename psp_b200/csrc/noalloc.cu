// B := A B without any device allocation (psp_cu_multiply_device_noalloc).
//
// The in-place operator apply needs a full-size temporary for A B before it
// can overwrite B.  psp_cu_multiply_device allocates that temporary on every
// call; this variant keeps it in a file-scope device array instead, so the
// call itself never allocates.  It serves callers that cannot allocate device
// memory at the time they call: code that runs while one of its own streams
// is being captured into a CUDA graph (an allocation there invalidates or
// breaks the capture), and services that reserve all device memory at
// start-up and treat any later allocation as an error.
//
// The caller's current device is current again when the call returns.
//
// Limits and sharing: the array holds kNoAllocMaxEntries complex doubles
// (16 MiB); every GPU that loads this library holds it until the process
// exits.  All calls on a device share the one array and it keeps the last
// call's contents; the apply overwrites every entry it later reads, so
// nothing needs clearing between calls.  Calls whose work overlaps on the GPU
// (other handles, other streams or threads) race on the array and must be
// ordered by the caller.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/psp_b200.h"
#include "handle.hpp"

namespace {

constexpr long long kNoAllocMaxEntries = 1LL << 20;  // complex doubles: 16 MiB

static __device__ __align__(256) psp_b200::z64 g_multiplyScratch[kNoAllocMaxEntries];

constexpr int kMaxDevices = 64;
std::mutex g_setupMutex;
void* g_scratchAddress[kMaxDevices] = {};

// Device address of the scratch array on `device` (which must be current).
// Resolved once per device, on the first call made on that device.
psp_b200::z64* ScratchOnDevice(int device) {
    std::lock_guard<std::mutex> lock(g_setupMutex);
    if (!g_scratchAddress[device]) {
        void* ptr = nullptr;
        CUDA_CHECK(cudaGetSymbolAddress(&ptr, g_multiplyScratch));
        g_scratchAddress[device] = ptr;
    }
    return static_cast<psp_b200::z64*>(g_scratchAddress[device]);
}

}  // namespace

namespace psp_b200 {
void SetLastError(const std::string& msg);  // capi.cu: text returned by psp_cu_last_error
}

namespace {
// Makes the caller's current device current again when the call returns.
struct RestoreDevice {
    int device = -1;
    RestoreDevice() {
        if (cudaGetDevice(&device) != cudaSuccess) device = -1;
    }
    ~RestoreDevice() {
        if (device >= 0) cudaSetDevice(device);
    }
};
}  // namespace

extern "C" int psp_cu_multiply_device_noalloc(psp_cu_handle* h, double* d_B, int k) {
    RestoreDevice restore;
    try {
        if (!h || !h->solver || !d_B) throw psp_b200::PspError(PSP_CU_LOGIC_ERROR, "null argument");
        psp_b200::Helmholtz& s = *h->solver;
        if (!s.dVel_.p) throw psp_b200::PspError(PSP_CU_NOT_INITIALIZED, "DistHelmholtz is not initialized");
        if (k < 1) throw psp_b200::PspError(PSP_CU_LOGIC_ERROR, "need at least one right-hand side");
        const long long entries = (long long)s.NumUnknowns() * k;
        if (entries > kNoAllocMaxEntries)
            throw psp_b200::PspError(PSP_CU_LOGIC_ERROR,
                                     "grid too large for the allocation-free multiply: nx*ny*nz*k = " +
                                         std::to_string(entries) + " exceeds " +
                                         std::to_string(kNoAllocMaxEntries));
        if (restore.device != s.device_) CUDA_CHECK(cudaSetDevice(s.device_));
        if (s.device_ >= kMaxDevices) throw psp_b200::PspError(PSP_CU_LOGIC_ERROR, "device index too large");
        psp_b200::z64* scratch = ScratchOnDevice(s.device_);
        psp_b200::z64* B = reinterpret_cast<psp_b200::z64*>(d_B);
        psp_b200::LaunchHelmholtzApply(B, scratch, nullptr, s.dVel_.as<double>(), s.sp_, k, s.stream());
        CUDA_CHECK(cudaMemcpyAsync(B, scratch, entries * sizeof(psp_b200::z64), cudaMemcpyDeviceToDevice,
                                   s.stream()));
        CUDA_CHECK(cudaStreamSynchronize(s.stream()));
        psp_b200::SetLastError("");
        return PSP_CU_OK;
    } catch (const psp_b200::PspError& e) {
        psp_b200::SetLastError(e.what());
        return e.code;
    } catch (const std::exception& e) {
        psp_b200::SetLastError(e.what());
        return PSP_CU_RUNTIME_ERROR;
    }
}
