// Internal declarations shared by the host side of libhenon_b200.so.
#pragma once

#include <cstddef>
#include <cstdint>
#include <mutex>
#include <random>
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
hm_status modulation_ripple(const std::string &kind, uint32_t n_turns, double omega_0,
                            uint32_t offset, std::vector<double> &ripple);

// ---- device buffers ---------------------------------------------------------

// Owning device allocation, move-only.  Blocks come from a per-device
// memory pool that keeps freed blocks for reuse (capi.cpp), so creating
// and destroying particle sets, trackers and scratch in a loop makes no
// allocation or unmapping call into the driver once the pool has grown.
// release() waits for the device like cudaFree before the block is reused.
struct DeviceBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    int device = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
    DeviceBuffer(DeviceBuffer &&o) noexcept : ptr(o.ptr), bytes(o.bytes), device(o.device) {
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

// Free device memory of the current device, counting the blocks that the
// library's pool holds but does not use (capi.cpp).
hm_status device_free_bytes(size_t *free_bytes);

}  // namespace hm

// ---- handles ------------------------------------------------------------------

// Particle ensemble on the device (particles_4d_gpu, src/henon.h:119-193).
struct hm_particles {
    size_t n_total = 0;      // base particles + ghosts
    size_t n_particles = 0;  // base particles
    size_t n_ghosts = 0;     // ghosts per base particle
    uint32_t global_steps = 0;
    // steps value shared by every live (non-NaN) particle: all particles
    // start at 0, survivors advance together and lost ones are frozen as NaN,
    // so the table index of a whole track() call is uniform.
    uint32_t live_step = 0;
    // Device state, and the initial conditions on the device (reset
    // restarts from them).  The device copies are authoritative.
    hm::DeviceBuffer x, px, y, py, steps, dvalid, dghost, didx, didx_base;
    hm::DeviceBuffer x0d, px0d, y0d, py0d;
    // Host mirrors of what the reference keeps on the host side (initial
    // conditions, valid, ghost, idx, idx_base).  Built from the device
    // copies on first use (add_ghost, tangent matrices), so that creating
    // and tracking a set never touches host memory beyond the caller's.
    mutable bool host_ready = false;
    mutable std::vector<double> x0, px0, y0, py0;
    mutable std::vector<uint8_t> valid, ghost;
    mutable std::vector<uint64_t> idx, idx_base;
    hm::DeviceBuffer work;  // survivor lists of the chunked tracker
    // Generator of "random" ghost directions: default-seeded, one per
    // particle set, as the reference's particles_4d::rng.
    std::mt19937_64 rng;
    // Key of the counter-based random kicks of hm_track (0 by default).
    unsigned long long kick_seed = 0;
};

// Modulation tables on the device (henon_tracker_gpu, src/henon.h:212-228).
struct hm_tracker {
    uint64_t allowed_steps = 0;
    std::vector<double> sx, cx, sy, cy;  // host copies
    hm::DeviceBuffer table;              // {sx, cx, sy, cy} per turn
    hm_arith arith = HM_ARITH_EXACT;
    // Modulation parameters the tables were built from (for derivatives).
    std::string kind = "sps";
    double omega_x = 0.0, omega_y = 0.0, omega_0 = 0.0, epsilon = 0.0;
    uint32_t offset = 0;
    // Birkhoff weights and modulation ripple of the last hm_adjoint turn
    // count, kept on the device between calls (rebuilt when the turn count
    // or the tables change); the mutex serialises adjoint calls.
    mutable std::mutex adjoint_mutex;
    mutable hm::DeviceBuffer adjoint_w, adjoint_S;
    mutable uint32_t adjoint_turns = 0;
    mutable bool adjoint_cached = false, adjoint_has_ripple = false;
};

namespace hm {

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
    // 0: turn records read from global memory; otherwise records are
    // staged through shared memory by bulk copies, this many turns a stage
    // (a power of two in [16, 512]; needs a 16-byte aligned table).
    uint32_t stage_turns;
    uint32_t *fault;       // set to nonzero when a staged copy timed out
    // Random kick of this module per turn (NaN: none), direction keyed by
    // (kick_seed, caller's particle index, table index of the turn).
    double kick_module;
    unsigned long long kick_seed;
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
// kick_module NaN means no random kicks.
hm_status track_driver(double *x, double *px, double *y, double *py,
                       uint32_t *steps, size_t n, const double *table,
                       uint64_t table_len, uint32_t s0, uint32_t n_turns,
                       double mu, double barrier, bool inverse, hm_arith arith,
                       void *workspace, cudaStream_t stream,
                       uint32_t *turns_done, double kick_module = __builtin_nan(""),
                       unsigned long long kick_seed = 0ull);

// Elementwise observable kernel launcher.
cudaError_t launch_observable(const double *x, const double *px,
                              const double *y, const double *py, double *out,
                              size_t n, int kind, cudaStream_t s);

// FP64 FMA-chain microbenchmark launcher; returns flops per launch.
cudaError_t launch_fp64_peak(double *sink, int blocks, int threads,
                             int iters, cudaStream_t s, double *flops);

// Tangent-map and indicator kernels (tangent.cu).
cudaError_t launch_matrices_step(double *M, const double *x, const double *px, const double *y,
                                 const double *py, const double *table, uint32_t idx, double mu,
                                 size_t n, bool set, cudaStream_t s);
cudaError_t launch_matrices_identity(double *M, size_t n, cudaStream_t s);
cudaError_t launch_matrices_apply(const double *M, const double *rv, double *out, size_t n,
                                  cudaStream_t s);
cudaError_t launch_vectors_multiply(const double *M, double *V, size_t n, cudaStream_t s);
cudaError_t launch_vectors_normalize(double *V, size_t n, cudaStream_t s);
cudaError_t launch_lyapunov(double *raw, double *bsum, const double *V, const double *weights,
                            const uint64_t *w_off, const uint64_t *w_len, int n_windows,
                            size_t idx, size_t n, cudaStream_t s);
cudaError_t launch_megno(double *l1, double *l2, double *l3, const double *A, const double *B,
                         size_t idx, size_t n, cudaStream_t s);
cudaError_t launch_megno_birkhoff(double *l1, double *l2, const double *weights,
                                  const uint64_t *w_off, const uint64_t *T, int n_windows,
                                  const double *A, const double *B, size_t idx, size_t n,
                                  cudaStream_t s);
cudaError_t launch_tune_init(const double *x, const double *px, const double *y, const double *py,
                             double *store_x, double *store_y, size_t n, cudaStream_t s);
cudaError_t launch_tune_add(const double *x, const double *px, const double *y, const double *py,
                            double *store_x, double *store_y, double *t1x, double *t1y,
                            double *t2x, double *t2y, const double *weights,
                            const uint64_t *w_off, const uint64_t *T, int n_windows, size_t idx,
                            size_t n, cudaStream_t s);

// Arguments of the fused tracking + indicator kernel (fused.cu).  Null
// pointers switch parts off: M (tangent matrix, MEGNO), V (tangent vectors,
// Lyapunov), store_x (Birkhoff tunes).  Window tables are on the device.
struct FusedArgs {
    double *x, *px, *y, *py;
    uint32_t *steps;
    uint32_t n;
    const double *table;
    uint32_t live_step;    // table index of the map for the first turn
    uint32_t global_step;  // global_steps before the first turn
    uint32_t n_turns;
    double mu;
    long long b2bits;
    int df_before;  // 1: DF at the point before the turn, table[live_step + k]
    // tangent matrix and MEGNO
    double *M;
    double *megno_l1, *megno_l2, *megno_l3;
    uint64_t megno_idx;
    double *snap;
    const uint64_t *snap_turns;
    int n_snap;
    double *mb_l1, *mb_l2;
    uint64_t mb_idx;
    const uint64_t *mb_T, *mb_off;
    const double *mb_w;
    int n_mb;
    // tangent vectors and Lyapunov windows
    double *V;
    double *ly_raw, *ly_b;
    uint64_t ly_idx;
    const uint64_t *ly_len, *ly_off;
    const double *ly_w;
    int n_ly;
    // Birkhoff tunes
    double *store_x, *store_y, *t1x, *t1y, *t2x, *t2y;
    uint64_t tu_idx;
    const uint64_t *tu_T, *tu_off;
    const double *tu_w;
    int n_tu;
    // Whole-orbit MEGNO only (tangent matrix alone, df_before): the
    // tracker's reproducible kicks (NaN: none; keyed by kick_seed, particle
    // index and table index) and backward turns (table[live_step - 1 - k],
    // steps decreasing, the Jacobian of the backward turn).
    double kick_module;
    unsigned long long kick_seed;
    int inverse;
};

cudaError_t launch_indicators(const FusedArgs &a, cudaStream_t s);
// Largest number of per-thread window accumulators the fused kernel takes
// (n_megno_birkhoff + 2 n_lyapunov + 4 n_tune).
size_t fused_max_slots();

// ---- batched heterogeneous tracking (batch.cu / batch.cpp) -------------------

constexpr int kBatchMaxSets = 1024;  // one planning thread per set

struct BatchSetDev {
    const double *table;   // this set's turn records
    uint64_t list_offset;  // start of the set's region in each survivor list
    uint32_t n_particles;
    uint32_t n_turns;      // turn budget
    double mu;
    long long b2bits;      // bit pattern of barrier^2 (0 when NaN)
};

struct BatchStateDev {
    uint32_t live;        // particles in the set's current list
    uint32_t next;        // survivors appended to the next list (atomic)
    uint32_t done;        // turns done
    uint32_t turns;       // turns of the current chunk
    uint32_t first_tile;  // first work item of the set in the current chunk
};

struct BatchDev {
    double *x, *px, *y, *py;
    uint32_t *steps;
    const uint32_t *particle_set;
    uint64_t n_total;
    const BatchSetDev *sets;
    BatchStateDev *state;
    int n_sets;
    uint64_t *list_idx[2];
    double *list_x[2], *list_px[2], *list_y[2], *list_py[2];
    uint32_t *tile_set;
    uint32_t *n_tiles, *next_item, *parity;
    int arith;
    int per_thread;
};

cudaError_t launch_batch_init(const BatchDev &b, cudaStream_t s);
cudaError_t launch_batch_plan(const BatchDev &b, uint32_t done_len, uint32_t next_len,
                              cudaStream_t s);
cudaError_t launch_batch_chunk(const BatchDev &b, int blocks, cudaStream_t s);
int batch_chunk_blocks_per_sm(int arith, int per_thread);

// ---- adjoint (adjoint.cu / adjoint.cpp) ---------------------------------------

struct AdjointArgs {
    const double *x0, *px0, *y0, *py0;
    size_t n;
    const double *table;  // tracker turn records
    const double *S;      // modulation ripple S_k (omega(k) = omega0 (1 + eps S_k))
    const double *w;      // Birkhoff weights of n_turns
    uint32_t n_turns, ckpt;
    double mu, epsilon, omega_x0, omega_y0;
    long long b2bits;
    int arith;
    double *ckpt_buf;  // [ceil(n_turns / ckpt)][4][n]
    double *seg_buf;   // [ckpt][4][n]
    double *loss;      // [n] per-particle loss (0 when lost)
    uint8_t *survived; // [n]
    uint32_t *steps;   // [n] turns survived
    double *g_ic;      // [4][n]
    double *g_th;      // [4][n] per-particle dL_i/d(omega_x0, omega_y0, eps, mu)
};

// mode 0: loss + reverse-mode gradients; 1: loss + forward-mode initial-
// condition gradient (tangent map); 2: loss only.
cudaError_t launch_adjoint(const AdjointArgs &a, int mode, cudaStream_t s);
// Particles per thread of the inverse-sweep adjoint kernel (1 or 2).
void set_adjoint_per_thread(int p);
int get_adjoint_per_thread();

// ---- orbit tunes (tunes.cu / tunes.cpp) -----------------------------------------

struct OrbitRecordArgs {
    double *x, *px, *y, *py;  // particle state (updated)
    uint32_t *steps;
    size_t n;
    const double *table;
    uint32_t live_step, n_turns;
    double mu;
    long long b2bits;
    int arith;
    double *ox, *opx, *oy, *opy;  // orbit [n][n_turns + 1] (each particle's samples contiguous)
    // Optional (null when unused): each coordinate's sum over the samples,
    // from 0.0 in sample order ([4][n]), and the first sample holding NaN
    // (n_turns + 1 when none).
    double *sums;
    uint32_t *first_nan;
    // Backward turns (table index live_step - 1 - k) and reproducible kicks
    // (kick_module NaN: none) of particle index id0 + i.
    int inverse;
    double kick_module;
    unsigned long long kick_seed;
    size_t id0;
};

cudaError_t launch_orbit_record(const OrbitRecordArgs &a, cudaStream_t s);

// Birkhoff tunes of the tracker's orbit in segments of turns
// (tunes.cu): one thread per (segment, plane, particle) sums the weighted
// phase advances of its segment for every window; a second kernel adds the
// segments in order.  Coordinates have means[c * n + i] subtracted first
// when means is not null.
struct BirkhoffSegArgs {
    const double *x, *px, *y, *py;  // orbit [n][S]
    const double *means;            // [4][n] or null
    const uint32_t *first_nan;      // [n]
    size_t n, S;
    uint32_t seg_len, n_seg;
    const uint32_t *from, *to;  // window sample bounds (inclusive)
    const uint64_t *w_off;
    const double *w;
    int n_win;
    const uint8_t *check_nan;  // per window: NaN tune when it holds a NaN sample
    double *partial;           // [n_win][2][n_seg][n]
    const int *out_col;        // per window: output column pair index
    double *out;               // [n][cols]
    size_t cols;
};
cudaError_t launch_birkhoff_segments(const BirkhoffSegArgs &a, cudaStream_t s);

// FFT tunes of one window of the tracker's orbit, both planes in one
// batch: gather (mean removed, Hann window) into rows z[plane n + i][k],
// cuFFT, then one warp per row finds the peak.
cudaError_t launch_hann_table(double *h, uint32_t len, cudaStream_t s);
cudaError_t launch_fft_gather2(const double *x, const double *px, const double *y,
                               const double *py, const double *means, size_t n, uint32_t from,
                               uint32_t len, const double *h, double2 *z, size_t S,
                               cudaStream_t s);
cudaError_t launch_fft_peak2(const double2 *z, uint32_t len, size_t n, uint32_t last_sample,
                             const uint32_t *first_nan, double *out, size_t cols, int col,
                             cudaStream_t s);
// FFT tunes of one window computed whole in one block's shared memory
// (tunes.cu; plans in fft_plan.cpp): the DFT of the window's L samples is
// an in-place mixed-radix network of length M (radices 2, 3, 4, 5, 8) when L
// has no other prime factor (M = L), else Bluestein's chirp convolution
// with M >= 2L - 1.  M is at most kFftMaxLen (the row fills at most 200 KB
// of shared memory); longer windows take the library path above.
constexpr int kFftMaxStages = 24;
constexpr uint32_t kFftMaxLen = 12800;
struct FftPlanDev {
    uint32_t L = 0, M = 0;
    int bluestein = 0;
    int swizzle = 0;  // shared-memory slots XOR-swizzled (M a multiple of 8)
    int n_stages = 0;
    uint8_t radix[kFftMaxStages] = {};
    uint32_t stage_len[kFftMaxStages] = {};   // span of the stage's butterflies
    uint32_t stage_prod[kFftMaxStages] = {};  // product of the earlier radices
    uint32_t n_coarse = 0;
    const double2 *tw_coarse = nullptr;  // exp(-2 pi i 64 u / M), u < n_coarse
    const double2 *tw_fine = nullptr;    // exp(-2 pi i v / M), v < 64
    const uint32_t *pos = nullptr;       // direct: where X_k lies after the network
    const double2 *chirp = nullptr;      // Bluestein: exp(-i pi n^2 / L), n < L
    const double2 *bhat = nullptr;       // Bluestein: the network's output for b
};
// The plan of windows of L samples on the current device (built once, kept
// until exit); *plan is null when L needs the library path.
hm_status fft_plan(uint32_t L, const FftPlanDev **plan);
// Shared-memory bytes of one block of fft_tune_kernel.
size_t fft_tune_smem_bytes(const FftPlanDev &plan);

struct FftTuneArgs {
    const double *x, *px, *y, *py;  // orbit: sample s of particle i at i stride_i + s stride_s
    const double *means;            // [4][n] sums, or null
    // [n] first NaN sample of each particle; null: the block scans its
    // window instead (NaN tune when any of its samples is NaN)
    const uint32_t *first_nan;
    size_t n, S;
    size_t stride_i, stride_s;      // (S, 1): the tracker's orbit; (1, n): stored orbits
    uint32_t from, last_sample;     // window samples from .. from + L - 1
    const double *hann;             // [L]
    double *out;                    // [n][cols]
    size_t cols;
    const int *out_cols;            // column pairs this window fills
    int n_out_cols;
    FftPlanDev plan;
    uint32_t prefetch_ahead;        // set by launch_fft_tunes
};
cudaError_t launch_fft_tunes(const FftTuneArgs &a, cudaStream_t s);

cudaError_t launch_mean_remove(double *x, double *px, double *y, double *py, size_t n, size_t S,
                               cudaStream_t s);
cudaError_t launch_birkhoff_tunes(const double *x, const double *px, const double *y,
                                  const double *py, size_t n, const uint32_t *from,
                                  const uint32_t *to, const uint64_t *w_off, const double *w,
                                  int n_win, double *out, cudaStream_t s);
cudaError_t launch_hann_gather(const double *q, const double *p, size_t n, uint32_t from,
                               uint32_t len, size_t first, size_t count, double2 *buf,
                               int *nan_flags, cudaStream_t s);
cudaError_t launch_fft_peak(const double2 *buf, uint32_t len, size_t count, const int *nan_flags,
                            double *out, size_t out_stride, size_t first, cudaStream_t s);

// (Re)allocates the device arrays of p's n_total particles and starts them
// at the given host coordinates, which become the initial conditions:
// steps = 0 and valid = 1; ghost, idx and idx_base from the host mirrors
// when they are built, else those of a set without ghosts (capi.cpp).
hm_status particles_upload(hm_particles *p, const double *x, const double *px, const double *y,
                           const double *py);
// Builds p's host mirrors from the device copies, once (capi.cpp).
hm_status particles_host_mirror(const hm_particles *p);

// Ghost particles and particle indices (ghosts.cu).
// Fused ghost Lyapunov loop (ghosts.cu): n_steps steps of `every` turns,
// each followed by the displacement log and the renormalisation of every
// ghost, for one base particle and its ghosts per thread.  Particle j of
// base b sits at b + n_base * j (j = 0 the base, 1..n_ghosts its ghosts).
struct GhostLyapunovArgs {
    double *x, *px, *y, *py;
    uint32_t *steps;
    size_t n_base;
    int n_ghosts;
    const double *table;
    uint32_t turn0;    // table index of the first turn (the live particles' steps)
    uint32_t every;    // turns per step
    uint32_t n_steps;  // steps of this launch
    double mu;
    long long b2bits;
    double module;
    double *lyap;  // [n_ghosts][n_base] running sums of log(d / module)
};
cudaError_t launch_ghost_lyapunov(const GhostLyapunovArgs &a, int arith, cudaStream_t s);
int ghost_lyapunov_max_ghosts();

cudaError_t launch_particle_indices(uint64_t *idx, uint64_t *idx_base, size_t n, cudaStream_t s);
cudaError_t launch_renormalize(double *x, double *px, double *y, double *py,
                               const uint64_t *idx_base, const uint8_t *ghost, size_t n,
                               double module, cudaStream_t s);
cudaError_t launch_displacement(const double *x, const double *px, const double *y,
                                const double *py, const uint64_t *idx, const uint64_t *idx_base,
                                const uint8_t *ghost, size_t n, size_t n_base, double *module,
                                double *dx, double *dpx, double *dy, double *dpy, cudaStream_t s);

// Uploads a host vector to a fresh device buffer.
template <class T>
hm_status upload(DeviceBuffer &dst, const std::vector<T> &src) {
    HM_TRY(dst.alloc(src.size() * sizeof(T)));
    if (!src.empty())
        HM_CUDA_TRY(cudaMemcpy(dst.ptr, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
    return ok();
}

}  // namespace hm
