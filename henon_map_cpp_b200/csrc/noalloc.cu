// Tracking entry point for callers that cannot allocate device memory.
//
// Some hosts of this library may not call cudaMalloc/cudaFree at all: a
// control or data-acquisition application that reserves all of its device
// memory at start-up and must never fail with out-of-memory mid-run, a
// framework whose allocator owns every device byte (a raw cudaMalloc
// fragments its pool or fails under its budget), or a latency-bound loop
// that cannot afford the device-wide synchronisation cudaFree implies.
// For them this file keeps the chunked tracker's survivor lists in a fixed
// device array that exists from the moment the library is loaded.
//
// The array is a file-scope __device__ variable of HM_NOALLOC_MAX_PARTICLES
// particles' worth of scratch (about 9 MiB); every GPU that loads the
// library's device code holds it until the process exits.  Its name in host
// code is only a host-side stand-in, so the device address is fetched once
// per device with cudaGetSymbolAddress (with that device current) and
// cached.  With CUDA's lazy module loading that first lookup is also what
// loads the device code, and so what takes the array's device memory: a
// caller that reserves all device memory must make one early call first
// (n = 0 does the set-up and nothing else).
#include <cuda_runtime.h>

#include <mutex>

#include "hm_internal.h"

namespace hm {
namespace {

constexpr size_t kNoAllocScratchBytes = track_workspace_bytes(HM_NOALLOC_MAX_PARTICLES);

// Shared by every call on a device; the last call's survivor lists stay in
// it.  The tracker clears its list counters before each launch.
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void *g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device (set-up on the
// first call per device).
hm_status scratch_address(void **out) {
    int dev = 0;
    HM_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return fail(HM_ERR_INVALID_ARG, "device ordinal out of range for the no-allocation scratch");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_scratch_addr[dev] == nullptr) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-allocation scratch)");
        if (p == nullptr) return fail(HM_ERR_CUDA, "no-allocation scratch has no device address");
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return ok();
}

}  // namespace
}  // namespace hm

extern "C" hm_status hm_track_device_noalloc(double *x, double *px, double *y, double *py,
                                             uint32_t *steps, size_t n, const double *tables,
                                             uint64_t table_len, uint32_t start_step,
                                             uint32_t n_turns, double mu, double barrier,
                                             int inverse, hm_arith arith, void *stream) {
    if (n > HM_NOALLOC_MAX_PARTICLES)
        return hm::fail(HM_ERR_INVALID_ARG,
                        "hm_track_device_noalloc: n exceeds the fixed scratch of " +
                            std::to_string(HM_NOALLOC_MAX_PARTICLES) +
                            " particles; use hm_track_device with a caller workspace");
    // The scratch address is the current device's: a stream of another
    // device would run the kernels there against this device's array.
    int cur = 0, sdev = 0;
    HM_CUDA_TRY(cudaGetDevice(&cur));
    HM_CUDA_TRY(cudaStreamGetDevice(static_cast<cudaStream_t>(stream), &sdev));
    if (sdev != cur)
        return hm::fail(HM_ERR_INVALID_ARG,
                        "hm_track_device_noalloc: the stream belongs to another device than the "
                        "current one");
    void *scratch = nullptr;
    HM_TRY(hm::scratch_address(&scratch));
    uint32_t done = 0;
    return hm::track_driver(x, px, y, py, steps, n, tables, table_len, start_step, n_turns, mu,
                            barrier, inverse != 0, arith, scratch,
                            static_cast<cudaStream_t>(stream), &done);
}
