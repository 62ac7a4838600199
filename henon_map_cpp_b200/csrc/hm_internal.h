// Internal declarations shared by the host side of libhenon_b200.so.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/henon_b200.h"

namespace hm {

// ---- error plumbing -------------------------------------------------------

// Records `msg` as the calling thread's last error and returns `code`.
hm_status fail(hm_status code, const std::string &msg);
// Clears the calling thread's last error and returns HM_OK.
hm_status ok();
// Converts a CUDA error into HM_ERR_CUDA / HM_ERR_OOM with context.
hm_status cuda_fail(cudaError_t err, const char *what);

#define HM_CUDA_TRY(expr)                                                   \
    do {                                                                     \
        cudaError_t hm_e_ = (expr);                                          \
        if (hm_e_ != cudaSuccess) return ::hm::cuda_fail(hm_e_, #expr);      \
    } while (0)

#define HM_TRY(expr)                                                        \
    do {                                                                     \
        hm_status hm_s_ = (expr);                                            \
        if (hm_s_ != HM_OK) return hm_s_;                                    \
    } while (0)

// True when the registered cancel callback asks to stop.
bool cancel_requested();

// ---- modulation (host, bit-identical to the reference) ---------------------

hm_status modulation(const std::string &kind, uint32_t n_turns, double omega_x,
                     double omega_y, double omega_0, double epsilon,
                     uint32_t offset, std::vector<double> &wx,
                     std::vector<double> &wy);
std::vector<double> birkhoff_weights(uint32_t n);

// ---- device buffers ---------------------------------------------------------

// Owning device allocation (cudaMalloc / cudaFree), move-only.
struct DeviceBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
    DeviceBuffer(DeviceBuffer &&o) noexcept : ptr(o.ptr), bytes(o.bytes) {
        o.ptr = nullptr;
        o.bytes = 0;
    }
    DeviceBuffer &operator=(DeviceBuffer &&o) noexcept;
    ~DeviceBuffer();
    hm_status alloc(size_t nbytes);    // frees any previous allocation
    hm_status ensure(size_t nbytes);   // grows (never shrinks)
    void release();
    template <class T> T *as() const { return static_cast<T *>(ptr); }
};

// ---- kernel launchers (defined in the .cu files) ---------------------------

// Parameters of one fused multi-turn chunk launch over a list of particles.
struct TrackChunk {
    // Caller state, indexed by the original particle index.
    double *ux, *upx, *uy, *upy;
    uint32_t *usteps;
    uint32_t n_user;
    // Input list; in_idx == nullptr means "all user particles, identity
    // order" (NaN particles are skipped, as check_nan does).
    const uint32_t *in_idx;
    const double *in_x, *in_px, *in_y, *in_py;
    const uint32_t *in_count;   // device count of the input list (or null)
    // Output list; out_idx == nullptr means "write survivors back to the
    // caller arrays" (last chunk).
    uint32_t *out_idx;
    double *out_x, *out_px, *out_y, *out_py;
    uint32_t *out_count;
    // Turn records and the table index of this chunk's first turn.
    const double *table;
    uint32_t turn0;        // forward: steps before the chunk; reverse: same
    uint32_t n_turns;      // turns in this chunk
    uint32_t steps_final;  // steps written for survivors of the last chunk
    double mu;
    long long b2bits;      // bit pattern of barrier^2 (0 when NaN)
};

struct TrackLaunch {
    int arith;      // hm_arith
    bool octupole;  // mu != 0
    bool reverse;
    int per_thread; // particles per thread (1, 2 or 4)
    int threads;    // threads per block
};

// Launches one chunk; grid sized from `n_in_upper` (an upper bound of the
// input count; blocks past the real count exit at once).
cudaError_t launch_track_chunk(const TrackChunk &c, const TrackLaunch &l,
                               uint32_t n_in_upper, cudaStream_t s);

// Scratch layout of the chunked tracker for n particles: 256 bytes of
// counters, then two survivor lists of {uint32 idx, double x, px, y, py}.
constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }
constexpr size_t track_workspace_bytes(size_t n) {
    return 256 + 2 * (align256(n * sizeof(uint32_t)) + 4 * align256(n * sizeof(double)));
}

// Host driver of the chunked tracking launches (capi.cpp).  `workspace`
// holds track_workspace_bytes(n) bytes of device memory (may be null when
// n_turns fits one chunk); *turns_done receives the turns applied.
hm_status track_driver(double *x, double *px, double *y, double *py,
                       uint32_t *steps, size_t n, const double *table,
                       uint64_t table_len, uint32_t s0, uint32_t n_turns,
                       double mu, double barrier, bool inverse, hm_arith arith,
                       void *workspace, cudaStream_t stream,
                       uint32_t *turns_done);

// Elementwise observable kernel launcher.
cudaError_t launch_observable(const double *x, const double *px,
                              const double *y, const double *py, double *out,
                              size_t n, int kind, cudaStream_t s);

// FP64 FMA-chain microbenchmark launcher; returns flops per launch.
cudaError_t launch_fp64_peak(double *sink, int blocks, int threads,
                             int iters, cudaStream_t s, double *flops);

}  // namespace hm
