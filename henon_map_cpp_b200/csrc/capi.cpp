// C ABI of libhenon_b200.so: handles, validation, error reporting and the
// host driver of the chunked tracking launches.
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "hm_internal.h"

namespace hm {

// ---- errors ---------------------------------------------------------------------

namespace {
thread_local std::string g_last_error;
std::atomic<hm_cancel_fn> g_cancel_fn{nullptr};
std::atomic<void *> g_cancel_ctx{nullptr};

// Launch shape of the tracking kernels (set by the autotuner).
struct TrackConfig {
    int threads = 128;
    int per_thread = 2;
    uint32_t chunk0 = 512;      // turns of the first chunk
    uint32_t chunk_max = 16384; // chunk length cap (chunks double up to it)
    // Turn records per staged bulk copy (0: direct reads).  Staging measured
    // 2-4 % faster than direct reads on the DA scan (1024^2 grid, 1e5 turns:
    // 17.7 vs 17.1 FP64 TFLOP/s at 256 turns a stage).
    uint32_t stage_turns = 256;
};
std::mutex g_cfg_mutex;
TrackConfig g_cfg;

TrackConfig track_config() {
    std::lock_guard<std::mutex> lock(g_cfg_mutex);
    return g_cfg;
}

// Kernel timing of the tracking launches (CUDA events on the launch stream).
struct Profile {
    std::atomic<bool> enabled{false};
    std::mutex mutex;
    double kernel_ms = 0.0;
    uint64_t launches = 0;
    uint64_t list_particles = 0;  // particles of the input lists, summed over launches
    uint64_t chunk_turns = 0;     // turns of the launches, summed
};
Profile g_profile;

// Event pair around one launch; elapsed time is added once the stream has
// been synchronised.
struct LaunchTimer {
    cudaEvent_t start = nullptr, stop = nullptr;
    bool armed = false;
    ~LaunchTimer() {
        if (start) cudaEventDestroy(start);
        if (stop) cudaEventDestroy(stop);
    }
    void begin(cudaStream_t s) {
        if (!g_profile.enabled.load()) return;
        if (!start) {
            cudaEventCreate(&start);
            cudaEventCreate(&stop);
        }
        cudaEventRecord(start, s);
        armed = true;
    }
    void end(cudaStream_t s) {
        if (armed) cudaEventRecord(stop, s);
    }
    uint64_t particles = 0, turns = 0;  // work of the armed launch
    void collect() {  // call after the stream has been synchronised
        if (!armed) return;
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, start, stop) == cudaSuccess) {
            std::lock_guard<std::mutex> lock(g_profile.mutex);
            g_profile.kernel_ms += ms;
            g_profile.launches += 1;
            g_profile.list_particles += particles;
            g_profile.chunk_turns += turns;
        }
        armed = false;
    }
};
}  // namespace

hm_status fail(hm_status code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

hm_status ok() {
    g_last_error.clear();
    return HM_OK;
}

hm_status cuda_fail(cudaError_t err, const char *what) {
    const hm_status code =
        err == cudaErrorMemoryAllocation ? HM_ERR_OOM
        : (err == cudaErrorNoDevice || err == cudaErrorInsufficientDriver) ? HM_ERR_NO_DEVICE
                                                                           : HM_ERR_CUDA;
    return fail(code, std::string("CUDA error: ") + cudaGetErrorString(err) + " (" + what + ")");
}

bool cancel_requested() {
    hm_cancel_fn fn = g_cancel_fn.load();
    return fn != nullptr && fn(g_cancel_ctx.load()) != 0;
}

// ---- device buffers ---------------------------------------------------------------

namespace {

// One pool per device, created on first use.  Its release threshold is
// unlimited: blocks freed into it stay mapped and are handed out again,
// until hm_release_cached_memory trims it.
struct PoolTable {
    std::mutex mutex;
    std::vector<cudaMemPool_t> pools;  // by device ordinal; null until first use
};

PoolTable &pool_table() {
    static PoolTable t;
    return t;
}

hm_status device_pool(int dev, cudaMemPool_t *out) {
    PoolTable &t = pool_table();
    std::lock_guard<std::mutex> lock(t.mutex);
    if (t.pools.size() <= size_t(dev)) t.pools.resize(size_t(dev) + 1, nullptr);
    if (!t.pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        HM_CUDA_TRY(cudaMemPoolCreate(&pool, &props));
        uint64_t keep_all = UINT64_MAX;
        const cudaError_t e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep_all);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(pool);
            return cuda_fail(e, "cudaMemPoolSetAttribute");
        }
        t.pools[dev] = pool;
    }
    *out = t.pools[dev];
    return ok();
}

// Makes dev current for the lifetime of the guard.
struct DeviceGuard {
    int saved = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&saved) == cudaSuccess && saved != dev) cudaSetDevice(dev);
        else saved = -1;
    }
    ~DeviceGuard() {
        if (saved >= 0) cudaSetDevice(saved);
    }
};

}  // namespace

DeviceBuffer &DeviceBuffer::operator=(DeviceBuffer &&o) noexcept {
    if (this != &o) {
        release();
        ptr = o.ptr;
        bytes = o.bytes;
        device = o.device;
        o.ptr = nullptr;
        o.bytes = 0;
    }
    return *this;
}

DeviceBuffer::~DeviceBuffer() { release(); }

void DeviceBuffer::release() {
    if (ptr) {
        // As cudaFree: every use of the block, on any stream, ends before
        // the pool may hand it out again.
        DeviceGuard guard(device);
        cudaDeviceSynchronize();
        cudaFreeAsync(ptr, 0);
    }
    ptr = nullptr;
    bytes = 0;
}

hm_status DeviceBuffer::alloc(size_t nbytes) {
    release();
    if (nbytes == 0) return ok();
    int dev = 0;
    HM_CUDA_TRY(cudaGetDevice(&dev));
    cudaMemPool_t pool = nullptr;
    HM_TRY(device_pool(dev, &pool));
    void *p = nullptr;
    cudaError_t got = cudaMallocFromPoolAsync(&p, nbytes, pool, 0);
    if (got == cudaErrorMemoryAllocation) {
        // Blocks the pool keeps but does not use may be what is missing:
        // hand them back to the device and try once more.
        cudaGetLastError();
        HM_CUDA_TRY(cudaDeviceSynchronize());
        HM_CUDA_TRY(cudaMemPoolTrimTo(pool, 0));
        got = cudaMallocFromPoolAsync(&p, nbytes, pool, 0);
    }
    if (got != cudaSuccess) return cuda_fail(got, "cudaMallocFromPoolAsync");
    // The block is ordered on the legacy stream; waiting for it makes it
    // usable from every stream, like a cudaMalloc block.
    const cudaError_t e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) {
        cudaFreeAsync(p, 0);
        return cuda_fail(e, "cudaStreamSynchronize after pool allocation");
    }
    ptr = p;
    bytes = nbytes;
    device = dev;
    return ok();
}

hm_status device_free_bytes(size_t *free_bytes) {
    size_t free_b = 0, total_b = 0;
    HM_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    int dev = 0;
    HM_CUDA_TRY(cudaGetDevice(&dev));
    cudaMemPool_t pool = nullptr;
    HM_TRY(device_pool(dev, &pool));
    uint64_t reserved = 0, used = 0;
    HM_CUDA_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
    HM_CUDA_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used));
    *free_bytes = free_b + size_t(reserved > used ? reserved - used : 0);
    return ok();
}

hm_status release_cached_memory() {
    PoolTable &t = pool_table();
    std::lock_guard<std::mutex> lock(t.mutex);
    for (size_t d = 0; d < t.pools.size(); ++d) {
        if (!t.pools[d]) continue;
        DeviceGuard guard(static_cast<int>(d));
        HM_CUDA_TRY(cudaDeviceSynchronize());
        HM_CUDA_TRY(cudaMemPoolTrimTo(t.pools[d], 0));
    }
    return ok();
}

hm_status DeviceBuffer::ensure(size_t nbytes) {
    if (nbytes <= bytes) return ok();
    return alloc(nbytes);
}

// ---- chunked tracking driver --------------------------------------------------------

namespace {

struct Workspace {
    uint32_t *count[2];
    uint32_t *fault;  // staged-copy timeouts of this call
    uint32_t *idx[2];
    double *x[2], *px[2], *y[2], *py[2];
};

Workspace carve(void *base, size_t n) {
    Workspace w{};
    char *p = static_cast<char *>(base);
    w.count[0] = reinterpret_cast<uint32_t *>(p);
    w.count[1] = w.count[0] + 1;
    w.fault = w.count[0] + 2;
    p += 256;
    for (int b = 0; b < 2; ++b) {
        w.idx[b] = reinterpret_cast<uint32_t *>(p);
        p += align256(n * sizeof(uint32_t));
        double **fields[4] = {&w.x[b], &w.px[b], &w.y[b], &w.py[b]};
        for (double **f : fields) {
            *f = reinterpret_cast<double *>(p);
            p += align256(n * sizeof(double));
        }
    }
    return w;
}

}  // namespace

// Advances n particles by n_turns turns of the map; *turns_done receives
// the turns actually applied (less than n_turns only when cancelled).
hm_status track_driver(double *x, double *px, double *y, double *py,
                       uint32_t *steps, size_t n, const double *table,
                       uint64_t table_len, uint32_t s0, uint32_t n_turns,
                       double mu, double barrier, bool inverse, hm_arith arith,
                       void *workspace, cudaStream_t stream,
                       uint32_t *turns_done, double kick_module, unsigned long long kick_seed) {
    *turns_done = 0;
    if (n == 0 || n_turns == 0) {
        *turns_done = n_turns;  // nothing to move; the turn counter still advances
        return ok();
    }
    if (n > 0xffffffffULL)
        return fail(HM_ERR_INVALID_ARG, "too many particles for one launch list (max 2^32-1)");
    if (!x || !px || !y || !py || !steps || !table)
        return fail(HM_ERR_INVALID_ARG, "null device pointer");
    if (arith != HM_ARITH_EXACT && arith != HM_ARITH_FAST)
        return fail(HM_ERR_INVALID_ARG, "unknown arithmetic mode");
    if (!inverse && uint64_t(s0) + n_turns > table_len)
        return fail(HM_ERR_BUDGET, "The number of turns is too large.");
    if (inverse && (n_turns > s0 || s0 > table_len))
        return fail(HM_ERR_BUDGET, "The number of turns is too large.");

    const TrackConfig cfg = track_config();
    const double b2 = barrier * barrier;
    long long b2bits = 0;
    if (!std::isnan(b2)) std::memcpy(&b2bits, &b2, sizeof(b2));

    TrackChunk c{};
    c.ux = x;
    c.upx = px;
    c.uy = y;
    c.upy = py;
    c.usteps = steps;
    c.n_user = uint32_t(n);
    c.table = table;
    c.mu = mu;
    c.b2bits = b2bits;
    c.kick_module = kick_module;
    c.kick_seed = kick_seed;
    TrackLaunch l{int(arith), mu != 0.0, inverse, cfg.per_thread, cfg.threads};

    const bool one_chunk = n_turns <= cfg.chunk0;
    if (!one_chunk && workspace == nullptr)
        return fail(HM_ERR_INVALID_ARG, "workspace required for more than one chunk of turns");
    Workspace w{};
    if (!one_chunk) w = carve(workspace, n);
    // Staged turn records need the workspace's fault word and a table that
    // bulk copies can read (16-byte aligned).
    const bool staged = cfg.stage_turns != 0 && !one_chunk &&
                        (reinterpret_cast<uintptr_t>(table) & 15u) == 0;
    c.stage_turns = staged ? cfg.stage_turns : 0u;
    c.fault = staged ? w.fault : nullptr;
    if (staged) HM_CUDA_TRY(cudaMemsetAsync(w.fault, 0, sizeof(uint32_t), stream));

    uint32_t done = 0;
    uint32_t chunk = cfg.chunk0;
    uint32_t n_in = uint32_t(n);
    int cur = -1;  // -1: the caller's arrays in identity order
    LaunchTimer timer;
    while (done < n_turns) {
        const uint32_t len = std::min(chunk, n_turns - done);
        const bool last = done + len == n_turns;
        c.turn0 = inverse ? s0 - done : s0 + done;
        c.n_turns = len;
        c.steps_final = inverse ? s0 - (done + len) : s0 + (done + len);
        if (cur < 0) {
            c.in_idx = nullptr;
            c.in_x = c.in_px = c.in_y = c.in_py = nullptr;
            c.in_count = nullptr;
        } else {
            c.in_idx = w.idx[cur];
            c.in_x = w.x[cur];
            c.in_px = w.px[cur];
            c.in_y = w.y[cur];
            c.in_py = w.py[cur];
            c.in_count = w.count[cur];
        }
        const int nxt = cur < 0 ? 0 : 1 - cur;
        if (last) {
            c.out_idx = nullptr;
            c.out_count = nullptr;
        } else {
            c.out_idx = w.idx[nxt];
            c.out_x = w.x[nxt];
            c.out_px = w.px[nxt];
            c.out_y = w.y[nxt];
            c.out_py = w.py[nxt];
            c.out_count = w.count[nxt];
            HM_CUDA_TRY(cudaMemsetAsync(w.count[nxt], 0, sizeof(uint32_t), stream));
        }
        timer.begin(stream);
        HM_CUDA_TRY(launch_track_chunk(c, l, n_in, stream));
        timer.end(stream);
        timer.particles = n_in;
        timer.turns = len;
        done += len;
        chunk = std::min<uint32_t>(chunk * 2u, cfg.chunk_max);
        if (last) break;
        uint32_t counters[3];  // count[0], count[1], fault
        HM_CUDA_TRY(cudaMemcpyAsync(counters, w.count[0], sizeof(counters),
                                    cudaMemcpyDeviceToHost, stream));
        HM_CUDA_TRY(cudaStreamSynchronize(stream));
        timer.collect();
        if (staged && counters[2] != 0u)
            return fail(HM_ERR_TIMEOUT, "turn-record copy into shared memory timed out");
        n_in = counters[nxt];
        cur = nxt;
        if (n_in == 0) {
            done = n_turns;  // every particle is lost; nothing left to write
            break;
        }
        if (cancel_requested()) {
            // Flush the survivors with their current steps and stop.
            c.turn0 = inverse ? s0 - done : s0 + done;
            c.n_turns = 0;
            c.steps_final = c.turn0;
            c.in_idx = w.idx[cur];
            c.in_x = w.x[cur];
            c.in_px = w.px[cur];
            c.in_y = w.y[cur];
            c.in_py = w.py[cur];
            c.in_count = w.count[cur];
            c.out_idx = nullptr;
            c.out_count = nullptr;
            HM_CUDA_TRY(launch_track_chunk(c, l, n_in, stream));
            HM_CUDA_TRY(cudaStreamSynchronize(stream));
            *turns_done = done;
            return fail(HM_ERR_CANCELLED, "tracking cancelled");
        }
    }
    uint32_t fault = 0u;
    if (staged)
        HM_CUDA_TRY(cudaMemcpyAsync(&fault, w.fault, sizeof(fault), cudaMemcpyDeviceToHost, stream));
    HM_CUDA_TRY(cudaStreamSynchronize(stream));
    timer.collect();
    if (fault != 0u) return fail(HM_ERR_TIMEOUT, "turn-record copy into shared memory timed out");
    *turns_done = n_turns;
    return ok();
}

hm_status set_profiling(int on) {
    std::lock_guard<std::mutex> lock(g_profile.mutex);
    g_profile.enabled.store(on != 0);
    g_profile.kernel_ms = 0.0;
    g_profile.launches = 0;
    g_profile.list_particles = 0;
    g_profile.chunk_turns = 0;
    return ok();
}

hm_status get_profile_work(uint64_t *list_particles, uint64_t *chunk_turns) {
    std::lock_guard<std::mutex> lock(g_profile.mutex);
    if (list_particles) *list_particles = g_profile.list_particles;
    if (chunk_turns) *chunk_turns = g_profile.chunk_turns;
    return ok();
}

hm_status get_profile(double *kernel_ms, uint64_t *launches) {
    std::lock_guard<std::mutex> lock(g_profile.mutex);
    if (kernel_ms) *kernel_ms = g_profile.kernel_ms;
    if (launches) *launches = g_profile.launches;
    return ok();
}

hm_status set_track_config(int threads, int per_thread, uint32_t chunk0, uint32_t chunk_max) {
    if (threads < 32 || threads > 256 || threads % 32 != 0)
        return fail(HM_ERR_INVALID_ARG, "threads must be 32..256 in steps of 32");
    if (per_thread != 1 && per_thread != 2 && per_thread != 4)
        return fail(HM_ERR_INVALID_ARG, "particles per thread must be 1, 2 or 4");
    if (chunk0 == 0 || chunk_max < chunk0)
        return fail(HM_ERR_INVALID_ARG, "need 0 < chunk0 <= chunk_max");
    std::lock_guard<std::mutex> lock(g_cfg_mutex);
    g_cfg.threads = threads;
    g_cfg.per_thread = per_thread;
    g_cfg.chunk0 = chunk0;
    g_cfg.chunk_max = chunk_max;
    return ok();
}

hm_status set_track_staging(uint32_t stage_turns) {
    if (stage_turns != 0 &&
        (stage_turns < 16 || stage_turns > 512 || (stage_turns & (stage_turns - 1)) != 0))
        return fail(HM_ERR_INVALID_ARG, "stage_turns must be 0 or a power of two in [16, 512]");
    std::lock_guard<std::mutex> lock(g_cfg_mutex);
    g_cfg.stage_turns = stage_turns;
    return ok();
}

hm_status get_track_config(int *threads, int *per_thread, uint32_t *chunk0, uint32_t *chunk_max) {
    const TrackConfig c = track_config();
    if (threads) *threads = c.threads;
    if (per_thread) *per_thread = c.per_thread;
    if (chunk0) *chunk0 = c.chunk0;
    if (chunk_max) *chunk_max = c.chunk_max;
    return ok();
}

}  // namespace hm

using hm::fail;
using hm::ok;

namespace {

hm_status upload_tables(hm_tracker *t, const std::vector<double> &wx,
                        const std::vector<double> &wy) {
    const size_t n = wx.size();
    t->sx.resize(n);
    t->cx.resize(n);
    t->sy.resize(n);
    t->cy.resize(n);
    // sin/cos of omega(n) with the host libm (src/henon.cu:2672-2686).
    for (size_t i = 0; i < n; ++i) {
        t->sx[i] = std::sin(wx[i]);
        t->cx[i] = std::cos(wx[i]);
        t->sy[i] = std::sin(wy[i]);
        t->cy[i] = std::cos(wy[i]);
    }
    std::vector<double> rec(4 * n);
    for (size_t i = 0; i < n; ++i) {
        rec[4 * i + 0] = t->sx[i];
        rec[4 * i + 1] = t->cx[i];
        rec[4 * i + 2] = t->sy[i];
        rec[4 * i + 3] = t->cy[i];
    }
    HM_TRY(t->table.alloc(rec.size() * sizeof(double)));
    if (n) HM_CUDA_TRY(cudaMemcpy(t->table.ptr, rec.data(), rec.size() * sizeof(double),
                                  cudaMemcpyHostToDevice));
    t->allowed_steps = n;
    return ok();
}

hm_status compute_tables(hm_tracker *t, uint32_t n_turns, double omega_x, double omega_y,
                         const char *kind, double omega_0, double epsilon, uint32_t offset) {
    if (!kind) return fail(HM_ERR_INVALID_ARG, "null modulation kind");
    std::vector<double> wx, wy;
    HM_TRY(hm::modulation(kind, n_turns, omega_x, omega_y, omega_0, epsilon, offset, wx, wy));
    HM_TRY(upload_tables(t, wx, wy));
    {
        // the adjoint's ripple follows the modulation
        std::lock_guard<std::mutex> lock(t->adjoint_mutex);
        t->adjoint_cached = false;
    }
    t->kind = kind;
    t->omega_x = omega_x;
    t->omega_y = omega_y;
    t->omega_0 = omega_0;
    t->epsilon = epsilon;
    t->offset = offset;
    return ok();
}

}  // namespace

namespace hm {

// (Re)allocates the device arrays of p for p->n_total particles and uploads
// coordinates, steps and the host-side bookkeeping vectors.
hm_status particles_upload(hm_particles *p, const double *x, const double *px,
                           const double *y, const double *py) {
    const size_t n = p->n_total;
    hm::DeviceBuffer *cur[4] = {&p->x, &p->px, &p->y, &p->py};
    hm::DeviceBuffer *ini[4] = {&p->x0d, &p->px0d, &p->y0d, &p->py0d};
    const double *src[4] = {x, px, y, py};
    for (int f = 0; f < 4; ++f) {
        HM_TRY(cur[f]->alloc(n * sizeof(double)));
        HM_TRY(ini[f]->alloc(n * sizeof(double)));
    }
    HM_TRY(p->steps.alloc(n * sizeof(uint32_t)));
    HM_TRY(p->dvalid.alloc(n));
    HM_TRY(p->dghost.alloc(n));
    HM_TRY(p->didx.alloc(n * sizeof(uint64_t)));
    HM_TRY(p->didx_base.alloc(n * sizeof(uint64_t)));
    if (n == 0) return ok();
    const cudaStream_t s = 0;
    for (int f = 0; f < 4; ++f) {
        HM_CUDA_TRY(cudaMemcpyAsync(cur[f]->ptr, src[f], n * sizeof(double), cudaMemcpyHostToDevice, s));
        HM_CUDA_TRY(cudaMemcpyAsync(ini[f]->ptr, cur[f]->ptr, n * sizeof(double),
                                    cudaMemcpyDeviceToDevice, s));
    }
    HM_CUDA_TRY(cudaMemsetAsync(p->steps.ptr, 0, n * sizeof(uint32_t), s));
    if (p->host_ready) {
        HM_CUDA_TRY(cudaMemcpyAsync(p->dvalid.ptr, p->valid.data(), n, cudaMemcpyHostToDevice, s));
        HM_CUDA_TRY(cudaMemcpyAsync(p->dghost.ptr, p->ghost.data(), n, cudaMemcpyHostToDevice, s));
        HM_CUDA_TRY(cudaMemcpyAsync(p->didx.ptr, p->idx.data(), n * sizeof(uint64_t),
                                    cudaMemcpyHostToDevice, s));
        HM_CUDA_TRY(cudaMemcpyAsync(p->didx_base.ptr, p->idx_base.data(), n * sizeof(uint64_t),
                                    cudaMemcpyHostToDevice, s));
    } else {
        HM_CUDA_TRY(cudaMemsetAsync(p->dvalid.ptr, 1, n, s));
        HM_CUDA_TRY(cudaMemsetAsync(p->dghost.ptr, 0, n, s));
        HM_CUDA_TRY(launch_particle_indices(p->didx.as<uint64_t>(), p->didx_base.as<uint64_t>(), n, s));
    }
    // The caller's (possibly pinned) arrays and the mirrors must outlive the copies.
    HM_CUDA_TRY(cudaStreamSynchronize(s));
    return ok();
}

hm_status particles_host_mirror(const hm_particles *p) {
    if (p->host_ready) return ok();
    const size_t n = p->n_total;
    p->x0.resize(n);
    p->px0.resize(n);
    p->y0.resize(n);
    p->py0.resize(n);
    p->valid.resize(n);
    p->ghost.resize(n);
    p->idx.resize(n);
    p->idx_base.resize(n);
    if (n) {
        const hm::DeviceBuffer *ini[4] = {&p->x0d, &p->px0d, &p->y0d, &p->py0d};
        std::vector<double> *dst[4] = {&p->x0, &p->px0, &p->y0, &p->py0};
        for (int f = 0; f < 4; ++f)
            HM_CUDA_TRY(cudaMemcpy(dst[f]->data(), ini[f]->ptr, n * sizeof(double), cudaMemcpyDeviceToHost));
        HM_CUDA_TRY(cudaMemcpy(p->valid.data(), p->dvalid.ptr, n, cudaMemcpyDeviceToHost));
        HM_CUDA_TRY(cudaMemcpy(p->ghost.data(), p->dghost.ptr, n, cudaMemcpyDeviceToHost));
        HM_CUDA_TRY(cudaMemcpy(p->idx.data(), p->didx.ptr, n * sizeof(uint64_t), cudaMemcpyDeviceToHost));
        HM_CUDA_TRY(cudaMemcpy(p->idx_base.data(), p->didx_base.ptr, n * sizeof(uint64_t),
                               cudaMemcpyDeviceToHost));
    }
    p->host_ready = true;
    return ok();
}

}  // namespace hm

using hm::particles_upload;

extern "C" {

const char *hm_last_error(void) { return hm::g_last_error.c_str(); }

int hm_version(void) { return 10000; }

int hm_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

hm_status hm_set_cancel_callback(hm_cancel_fn fn, void *ctx) {
    hm::g_cancel_ctx.store(ctx);
    hm::g_cancel_fn.store(fn);
    return ok();
}

hm_status hm_set_track_config(int threads, int per_thread, uint32_t chunk0, uint32_t chunk_max) {
    return hm::set_track_config(threads, per_thread, chunk0, chunk_max);
}

hm_status hm_set_track_staging(uint32_t stage_turns) { return hm::set_track_staging(stage_turns); }

hm_status hm_release_cached_memory(void) { return hm::release_cached_memory(); }

hm_status hm_get_track_staging(uint32_t *stage_turns) {
    if (!stage_turns) return fail(HM_ERR_INVALID_ARG, "null output");
    *stage_turns = hm::track_config().stage_turns;
    return ok();
}

hm_status hm_get_track_config(int *threads, int *per_thread, uint32_t *chunk0, uint32_t *chunk_max) {
    return hm::get_track_config(threads, per_thread, chunk0, chunk_max);
}

hm_status hm_set_profiling(int on) { return hm::set_profiling(on); }

hm_status hm_get_profile(double *kernel_ms, uint64_t *launches) {
    return hm::get_profile(kernel_ms, launches);
}

hm_status hm_get_profile_work(uint64_t *list_particles, uint64_t *chunk_turns) {
    return hm::get_profile_work(list_particles, chunk_turns);
}

// ---- host numerics ----------------------------------------------------------------

hm_status hm_modulation(const char *kind, uint32_t n_turns, double omega_x, double omega_y,
                        double omega_0, double epsilon, uint32_t offset, double *omega_x_out,
                        double *omega_y_out) {
    if (!kind || (n_turns && (!omega_x_out || !omega_y_out)))
        return fail(HM_ERR_INVALID_ARG, "null pointer");
    std::vector<double> wx, wy;
    HM_TRY(hm::modulation(kind, n_turns, omega_x, omega_y, omega_0, epsilon, offset, wx, wy));
    std::memcpy(omega_x_out, wx.data(), wx.size() * sizeof(double));
    std::memcpy(omega_y_out, wy.data(), wy.size() * sizeof(double));
    return ok();
}

}  // extern "C"

namespace hm {
std::vector<double> sps_modulation(double tune, double epsilon, int32_t start, int32_t end);
std::vector<double> basic_modulation(double tune, double omega, double epsilon, int32_t start,
                                     int32_t end);
}  // namespace hm

extern "C" {

hm_status hm_sps_modulation(double tune, double epsilon, int32_t start, int32_t end, double *out) {
    if (start >= end) return fail(HM_ERR_INVALID_ARG, "sps_modulation needs start < end");
    if (!out) return fail(HM_ERR_INVALID_ARG, "null pointer");
    auto v = hm::sps_modulation(tune, epsilon, start, end);
    std::memcpy(out, v.data(), v.size() * sizeof(double));
    return ok();
}

hm_status hm_basic_modulation(double tune, double omega, double epsilon, int32_t start,
                              int32_t end, double *out) {
    if (start >= end) return fail(HM_ERR_INVALID_ARG, "basic_modulation needs start < end");
    if (!out) return fail(HM_ERR_INVALID_ARG, "null pointer");
    auto v = hm::basic_modulation(tune, omega, epsilon, start, end);
    std::memcpy(out, v.data(), v.size() * sizeof(double));
    return ok();
}

hm_status hm_birkhoff_weights(uint32_t n_weights, double *out) {
    if (n_weights && !out) return fail(HM_ERR_INVALID_ARG, "null pointer");
    auto w = hm::birkhoff_weights(n_weights);
    std::memcpy(out, w.data(), w.size() * sizeof(double));
    return ok();
}

// ---- tracker ----------------------------------------------------------------------

hm_status hm_tracker_create(uint32_t n_turns, double omega_x, double omega_y,
                            const char *modulation_kind, double omega_0, double epsilon,
                            uint32_t offset, hm_tracker **out) {
    if (!out) return fail(HM_ERR_INVALID_ARG, "null output handle");
    *out = nullptr;
    auto *t = new hm_tracker();
    const hm_status s = compute_tables(t, n_turns, omega_x, omega_y, modulation_kind, omega_0,
                                       epsilon, offset);
    if (s != HM_OK) {
        delete t;
        return s;
    }
    *out = t;
    return ok();
}

hm_status hm_tracker_compute_a_modulation(hm_tracker *t, uint32_t n_turns, double omega_x,
                                          double omega_y, const char *modulation_kind,
                                          double omega_0, double epsilon, uint32_t offset) {
    if (!t) return fail(HM_ERR_INVALID_ARG, "null tracker");
    return compute_tables(t, n_turns, omega_x, omega_y, modulation_kind, omega_0, epsilon, offset);
}

hm_status hm_tracker_destroy(hm_tracker *t) {
    delete t;
    return ok();
}

hm_status hm_tracker_allowed_steps(const hm_tracker *t, uint64_t *out) {
    if (!t || !out) return fail(HM_ERR_INVALID_ARG, "null pointer");
    *out = t->allowed_steps;
    return ok();
}

hm_status hm_tracker_get_tables(const hm_tracker *t, double *sin_x, double *cos_x, double *sin_y,
                                double *cos_y) {
    if (!t) return fail(HM_ERR_INVALID_ARG, "null tracker");
    const size_t n = t->sx.size();
    if (n && (!sin_x || !cos_x || !sin_y || !cos_y)) return fail(HM_ERR_INVALID_ARG, "null pointer");
    std::memcpy(sin_x, t->sx.data(), n * sizeof(double));
    std::memcpy(cos_x, t->cx.data(), n * sizeof(double));
    std::memcpy(sin_y, t->sy.data(), n * sizeof(double));
    std::memcpy(cos_y, t->cy.data(), n * sizeof(double));
    return ok();
}

hm_status hm_tracker_device_tables(const hm_tracker *t, const double **out) {
    if (!t || !out) return fail(HM_ERR_INVALID_ARG, "null pointer");
    *out = t->table.as<const double>();
    return ok();
}

hm_status hm_tracker_set_arith(hm_tracker *t, hm_arith arith) {
    if (!t) return fail(HM_ERR_INVALID_ARG, "null tracker");
    if (arith != HM_ARITH_EXACT && arith != HM_ARITH_FAST)
        return fail(HM_ERR_INVALID_ARG, "unknown arithmetic mode");
    t->arith = arith;
    return ok();
}

hm_status hm_tracker_get_arith(const hm_tracker *t, hm_arith *out) {
    if (!t || !out) return fail(HM_ERR_INVALID_ARG, "null pointer");
    *out = t->arith;
    return ok();
}

// ---- particles --------------------------------------------------------------------

hm_status hm_particles_create(const double *x, const double *px, const double *y,
                              const double *py, size_t n, hm_particles **out) {
    if (!out) return fail(HM_ERR_INVALID_ARG, "null output handle");
    *out = nullptr;
    if (n && (!x || !px || !y || !py)) return fail(HM_ERR_INVALID_ARG, "null coordinate array");
    if (n > 0xffffffffULL) return fail(HM_ERR_INVALID_ARG, "too many particles (max 2^32-1)");
    auto *p = new hm_particles();
    p->n_total = p->n_particles = n;
    const hm_status s = particles_upload(p, x, px, y, py);
    if (s != HM_OK) {
        delete p;
        return s;
    }
    *out = p;
    return ok();
}

hm_status hm_particles_destroy(hm_particles *p) {
    delete p;
    return ok();
}

hm_status hm_particles_reset(hm_particles *p) {
    if (!p) return fail(HM_ERR_INVALID_ARG, "null particles");
    // Restart from the initial conditions with steps = 0 and valid = 1
    // (particles_4d::reset and particles_4d_gpu::reset,
    // src/henon.cu:727-735, 1238-1244); ghosts and indices
    // are unchanged.
    if (p->host_ready) std::fill(p->valid.begin(), p->valid.end(), uint8_t(1));
    p->live_step = 0;
    const size_t n = p->n_total;
    if (n == 0) return ok();
    const cudaStream_t s = 0;
    const hm::DeviceBuffer *ini[4] = {&p->x0d, &p->px0d, &p->y0d, &p->py0d};
    hm::DeviceBuffer *cur[4] = {&p->x, &p->px, &p->y, &p->py};
    for (int f = 0; f < 4; ++f)
        HM_CUDA_TRY(cudaMemcpyAsync(cur[f]->ptr, ini[f]->ptr, n * sizeof(double),
                                    cudaMemcpyDeviceToDevice, s));
    HM_CUDA_TRY(cudaMemsetAsync(p->steps.ptr, 0, n * sizeof(uint32_t), s));
    HM_CUDA_TRY(cudaMemsetAsync(p->dvalid.ptr, 1, n, s));
    HM_CUDA_TRY(cudaStreamSynchronize(s));
    return ok();
}

hm_status hm_particles_size(const hm_particles *p, size_t *n_total, size_t *n_particles,
                            size_t *n_ghosts) {
    if (!p) return fail(HM_ERR_INVALID_ARG, "null particles");
    if (n_total) *n_total = p->n_total;
    if (n_particles) *n_particles = p->n_particles;
    if (n_ghosts) *n_ghosts = p->n_ghosts;
    return ok();
}

hm_status hm_particles_global_steps(const hm_particles *p, uint32_t *out) {
    if (!p || !out) return fail(HM_ERR_INVALID_ARG, "null pointer");
    *out = p->global_steps;
    return ok();
}

hm_status hm_particles_device_ptr(const hm_particles *p, hm_field field, void **out) {
    if (!p || !out) return fail(HM_ERR_INVALID_ARG, "null pointer");
    switch (field) {
        case HM_FIELD_X: *out = p->x.ptr; break;
        case HM_FIELD_PX: *out = p->px.ptr; break;
        case HM_FIELD_Y: *out = p->y.ptr; break;
        case HM_FIELD_PY: *out = p->py.ptr; break;
        case HM_FIELD_STEPS: *out = p->steps.ptr; break;
        case HM_FIELD_VALID: *out = p->dvalid.ptr; break;
        case HM_FIELD_GHOST: *out = p->dghost.ptr; break;
        case HM_FIELD_IDX: *out = p->didx.ptr; break;
        case HM_FIELD_IDX_BASE: *out = p->didx_base.ptr; break;
        default: return fail(HM_ERR_INVALID_ARG, "unknown field");
    }
    return ok();
}

hm_status hm_particles_get(const hm_particles *p, hm_field field, void *host_out) {
    if (!p) return fail(HM_ERR_INVALID_ARG, "null particles");
    void *src = nullptr;
    HM_TRY(hm_particles_device_ptr(p, field, &src));
    size_t elem = 8;
    if (field == HM_FIELD_STEPS) elem = 4;
    if (field == HM_FIELD_VALID || field == HM_FIELD_GHOST) elem = 1;
    const size_t bytes = p->n_total * elem;
    if (bytes == 0) return ok();
    if (!host_out) return fail(HM_ERR_INVALID_ARG, "null output");
    HM_CUDA_TRY(cudaMemcpy(host_out, src, bytes, cudaMemcpyDeviceToHost));
    return ok();
}

hm_status hm_particles_observable(const hm_particles *p, hm_observable kind, double *host_out) {
    if (!p) return fail(HM_ERR_INVALID_ARG, "null particles");
    if (kind < HM_OBS_RADIUS || kind > HM_OBS_ANGLE_Y) return fail(HM_ERR_INVALID_ARG, "unknown observable");
    const size_t n = p->n_total;
    if (n == 0) return ok();
    if (!host_out) return fail(HM_ERR_INVALID_ARG, "null output");
    hm::DeviceBuffer out;
    HM_TRY(out.alloc(n * sizeof(double)));
    HM_CUDA_TRY(hm::launch_observable(p->x.as<double>(), p->px.as<double>(), p->y.as<double>(),
                                      p->py.as<double>(), out.as<double>(), n, int(kind), 0));
    HM_CUDA_TRY(cudaMemcpy(host_out, out.ptr, n * sizeof(double), cudaMemcpyDeviceToHost));
    return ok();
}

hm_status hm_particles_set_kick_seed(hm_particles *p, uint64_t seed) {
    if (!p) return fail(HM_ERR_INVALID_ARG, "null particles");
    p->kick_seed = seed;
    return ok();
}

hm_status hm_particles_get_kick_seed(const hm_particles *p, uint64_t *seed) {
    if (!p || !seed) return fail(HM_ERR_INVALID_ARG, "null particles or output");
    *seed = p->kick_seed;
    return ok();
}

// ---- tracking ---------------------------------------------------------------------

size_t hm_track_workspace_bytes(size_t n) { return hm::track_workspace_bytes(n); }

hm_status hm_track_device(double *x, double *px, double *y, double *py, uint32_t *steps, size_t n,
                          const double *tables, uint64_t table_len, uint32_t start_step,
                          uint32_t n_turns, double mu, double barrier, int inverse,
                          hm_arith arith, void *workspace, void *stream) {
    uint32_t done = 0;
    return hm::track_driver(x, px, y, py, steps, n, tables, table_len, start_step, n_turns, mu,
                            barrier, inverse != 0, arith, workspace,
                            static_cast<cudaStream_t>(stream), &done);
}

hm_status hm_track(hm_tracker *t, hm_particles *p, uint32_t n_turns, double mu, double barrier,
                   double kick_module, int inverse) {
    if (!t || !p) return fail(HM_ERR_INVALID_ARG, "null tracker or particles");
    // Turn budget (src/henon.cu:3158-3167), in 64-bit arithmetic.
    if (inverse) {
        if (n_turns > p->global_steps) return fail(HM_ERR_BUDGET, "The number of turns is too large.");
    } else {
        if (uint64_t(n_turns) + p->global_steps > t->allowed_steps)
            return fail(HM_ERR_BUDGET, "The number of turns is too large.");
    }
    if (inverse && n_turns > p->live_step)
        return fail(HM_ERR_BUDGET,
                    "The number of turns is too large. (inverse tracking past the particles' steps)");
    void *ws = nullptr;
    if (p->n_total) {
        HM_TRY(p->work.ensure(hm::track_workspace_bytes(p->n_total)));
        ws = p->work.ptr;
    }
    uint32_t done = 0;
    const hm_status s = hm::track_driver(
        p->x.as<double>(), p->px.as<double>(), p->y.as<double>(), p->py.as<double>(),
        p->steps.as<uint32_t>(), p->n_total, t->table.as<const double>(), t->allowed_steps,
        p->live_step, n_turns, mu, barrier, inverse != 0, t->arith, ws, 0, &done, kick_module,
        p->kick_seed);
    if (s != HM_OK && s != HM_ERR_CANCELLED) return s;
    // global_steps follows the turns applied (src/henon.cu:3181-3184).
    if (inverse) {
        p->global_steps -= done;
        p->live_step -= done;
    } else {
        p->global_steps += done;
        p->live_step += done;
    }
    return s;
}

// ---- measurement -------------------------------------------------------------------

hm_status hm_fp64_peak(double seconds_target, double *tflops, double *ms) {
    if (!tflops) return fail(HM_ERR_INVALID_ARG, "null output");
    int dev = 0, sms = 0;
    HM_CUDA_TRY(cudaGetDevice(&dev));
    HM_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    hm::DeviceBuffer sink;
    HM_TRY(sink.alloc(size_t(sms) * 64 * sizeof(double)));
    // Destroyed on every return path, the early error returns included.
    struct EventPair {
        cudaEvent_t a = nullptr, b = nullptr;
        ~EventPair() {
            if (a) cudaEventDestroy(a);
            if (b) cudaEventDestroy(b);
        }
    } ev;
    HM_CUDA_TRY(cudaEventCreate(&ev.a));
    HM_CUDA_TRY(cudaEventCreate(&ev.b));
    cudaEvent_t a = ev.a, b = ev.b;
    const int blocks = sms * 8, threads = 256;
    int iters = 256;
    double flops = 0.0;
    float elapsed = 0.f;
    // Warm up, then grow the launch until it lasts about seconds_target.
    for (int round = 0; round < 12; ++round) {
        HM_CUDA_TRY(cudaEventRecord(a, 0));
        HM_CUDA_TRY(hm::launch_fp64_peak(sink.as<double>(), blocks, threads, iters, 0, &flops));
        HM_CUDA_TRY(cudaEventRecord(b, 0));
        HM_CUDA_TRY(cudaEventSynchronize(b));
        HM_CUDA_TRY(cudaEventElapsedTime(&elapsed, a, b));
        if (round > 0 && elapsed * 1e-3 >= seconds_target) break;
        if (elapsed * 1e-3 < seconds_target) {
            const double scale = elapsed > 0.f ? seconds_target / (elapsed * 1e-3) : 8.0;
            iters = int(std::min(double(iters) * std::min(scale * 1.1, 8.0), 1e8));
        }
    }
    *tflops = flops / (double(elapsed) * 1e-3) / 1e12;
    if (ms) *ms = elapsed;
    return ok();
}

}  // extern "C"
