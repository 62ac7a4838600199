// C ABI of the tune estimates (hm_orbit_tunes, hm_tracker_orbit_tunes,
// hm_storage_tunes): window validation, Birkhoff weight tables, cuFFT
// plans, and particle slicing so orbit buffers fit device memory.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <cufft.h>

#include "hm_internal.h"

using hm::DeviceBuffer;
using hm::fail;
using hm::ok;

struct hm_storage;  // defined in indicators.cpp
extern "C" hm_status hm_storage_device_ptr(const hm_storage *h, hm_field field, const double **out);
extern "C" hm_status hm_storage_size(const hm_storage *h, size_t *n, size_t *batch, size_t *stored);

#define HM_CUFFT_TRY_STREAM(plan)                                           \
    do {                                                                    \
        const cufftResult _r = cufftSetStream((plan), 0);                   \
        if (_r != CUFFT_SUCCESS) return cufft_fail(_r, "set stream");       \
    } while (0)

namespace {

hm_status cufft_fail(cufftResult r, const char *what) {
    if (r == CUFFT_ALLOC_FAILED) return fail(HM_ERR_OOM, std::string("cuFFT: allocation failed (") + what + ")");
    return fail(HM_ERR_CUDA, std::string("cuFFT error ") + std::to_string(int(r)) + " (" + what + ")");
}

// Birkhoff tunes of the windows (from, to) plus the full orbit [0, S-1].
hm_status birkhoff_device(const double *x, const double *px, const double *y, const double *py,
                          size_t n, size_t S, const std::vector<uint32_t> &from,
                          const std::vector<uint32_t> &to, double *dev_out) {
    std::vector<uint32_t> f(from), t(to);
    f.push_back(0);
    t.push_back(uint32_t(S - 1));
    std::vector<double> w;
    std::vector<uint64_t> off;
    for (size_t j = 0; j < f.size(); ++j) {
        off.push_back(w.size());
        auto ww = hm::birkhoff_weights(t[j] - f[j]);
        w.insert(w.end(), ww.begin(), ww.end());
    }
    DeviceBuffer df, dt, doff, dw;
    HM_TRY(hm::upload(df, f));
    HM_TRY(hm::upload(dt, t));
    HM_TRY(hm::upload(doff, off));
    HM_TRY(hm::upload(dw, w));
    HM_CUDA_TRY(hm::launch_birkhoff_tunes(x, px, y, py, n, df.as<uint32_t>(), dt.as<uint32_t>(),
                                          doff.as<uint64_t>(), dw.as<double>(), int(f.size()),
                                          dev_out, 0));
    return ok();
}

// FFT tunes of the windows (from, to) plus the full orbit [1, S-1]: in
// shared memory (fft_tune_kernel) where the window fits one block, else in
// particle slices bounded by the spectrum buffer through cuFFT.
hm_status fft_device(const double *x, const double *px, const double *y, const double *py,
                     size_t n, size_t S, const std::vector<uint32_t> &from,
                     const std::vector<uint32_t> &to, double *dev_out) {
    std::vector<uint32_t> f(from), len;
    for (size_t j = 0; j < from.size(); ++j) len.push_back(to[j] - from[j] + 1);
    f.push_back(1);
    len.push_back(uint32_t(S - 1));
    const size_t cols = 2 * f.size();
    const size_t budget = size_t(1) << 31;  // bytes of complex spectrum per slice
    for (size_t j = 0; j < f.size(); ++j) {
        const uint32_t L = len[j];
        if (L == 0) continue;
        // Windows one block holds: transformed in shared memory, every
        // particle in one launch, the window's own samples deciding NaN.
        const hm::FftPlanDev *plan = nullptr;
        HM_TRY(hm::fft_plan(L, &plan));
        if (plan) {
            DeviceBuffer hann, col;
            HM_TRY(hann.alloc(size_t(L) * sizeof(double)));
            HM_CUDA_TRY(hm::launch_hann_table(hann.as<double>(), L, 0));
            HM_TRY(hm::upload(col, std::vector<int>{int(j)}));
            hm::FftTuneArgs a{};
            a.x = x;
            a.px = px;
            a.y = y;
            a.py = py;
            a.n = n;
            a.S = S;
            a.stride_i = 1;
            a.stride_s = n;
            a.from = f[j];
            a.last_sample = f[j] + L - 1;
            a.hann = hann.as<double>();
            a.out = dev_out;
            a.cols = cols;
            a.out_cols = col.as<int>();
            a.n_out_cols = 1;
            a.plan = *plan;
            HM_CUDA_TRY(hm::launch_fft_tunes(a, 0));
            continue;
        }
        const size_t slice = std::max<size_t>(1, std::min(n, budget / (size_t(L) * sizeof(double2))));
        DeviceBuffer buf, flags;
        HM_TRY(buf.alloc(slice * L * sizeof(double2)));
        HM_TRY(flags.alloc(slice * sizeof(int)));
        std::map<size_t, cufftHandle> plans;
        hm_status status = ok();
        for (size_t first = 0; first < n && status == HM_OK; first += slice) {
            const size_t count = std::min(slice, n - first);
            cufftHandle &plan = plans[count];
            if (plan == 0) {
                int nl = int(L);
                const cufftResult r = cufftPlanMany(&plan, 1, &nl, nullptr, 1, nl, nullptr, 1, nl,
                                                    CUFFT_Z2Z, int(count));
                if (r != CUFFT_SUCCESS) {
                    status = cufft_fail(r, "plan");
                    break;
                }
            }
            for (int plane = 0; plane < 2 && status == HM_OK; ++plane) {
                const double *q = plane ? y : x, *p = plane ? py : px;
                cudaError_t e = cudaMemset(flags.ptr, 0, count * sizeof(int));
                if (e == cudaSuccess)
                    e = hm::launch_hann_gather(q, p, n, f[j], L, first, count, buf.as<double2>(),
                                               flags.as<int>(), 0);
                if (e != cudaSuccess) {
                    status = hm::cuda_fail(e, "hann gather");
                    break;
                }
                auto *z = reinterpret_cast<cufftDoubleComplex *>(buf.ptr);
                const cufftResult r = cufftExecZ2Z(plan, z, z, CUFFT_FORWARD);
                if (r != CUFFT_SUCCESS) {
                    status = cufft_fail(r, "exec");
                    break;
                }
                e = hm::launch_fft_peak(buf.as<double2>(), L, count, flags.as<int>(),
                                        dev_out + 2 * j + plane, cols, first, 0);
                if (e != cudaSuccess) status = hm::cuda_fail(e, "fft peak");
            }
        }
        for (auto &kv : plans)
            if (kv.second) cufftDestroy(kv.second);
        HM_TRY(status);
    }
    return ok();
}

hm_status check_windows(size_t S, const uint32_t *from, const uint32_t *to, size_t w) {
    if (w && (!from || !to)) return fail(HM_ERR_INVALID_ARG, "null window bounds");
    for (size_t j = 0; j < w; ++j) {
        if (from[j] >= S || to[j] >= S)
            return fail(HM_ERR_INVALID_ARG, "compute_tune: from and to must be valid indices");
        if (from[j] > to[j]) return fail(HM_ERR_INVALID_ARG, "compute_tune: from[i] > to[i]");
    }
    return ok();
}

}  // namespace

extern "C" {

hm_status hm_orbit_tunes(const double *x, const double *px, const double *y, const double *py,
                         size_t n, size_t n_samples, const uint32_t *from, const uint32_t *to,
                         size_t n_windows, int method, double *host_out) {
    if (method != 0 && method != 1) return fail(HM_ERR_INVALID_ARG, "method must be 0 (Birkhoff) or 1 (FFT)");
    if (n_samples < 2) return fail(HM_ERR_INVALID_ARG, "need at least two samples");
    HM_TRY(check_windows(n_samples, from, to, n_windows));
    if (n == 0) return ok();
    if (!x || !px || !y || !py || !host_out) return fail(HM_ERR_INVALID_ARG, "null pointer");
    const std::vector<uint32_t> f(from, from + n_windows), t(to, to + n_windows);
    const size_t cols = 2 * (n_windows + 1);
    DeviceBuffer out;
    HM_TRY(out.alloc(n * cols * sizeof(double)));
    if (method == 0) HM_TRY(birkhoff_device(x, px, y, py, n, n_samples, f, t, out.as<double>()));
    else HM_TRY(fft_device(x, px, y, py, n, n_samples, f, t, out.as<double>()));
    HM_CUDA_TRY(cudaMemcpy(host_out, out.ptr, n * cols * sizeof(double), cudaMemcpyDeviceToHost));
    return ok();
}

// hm_orbit_tunes on host arrays [n_samples][n] (uploaded first).
hm_status hm_orbit_tunes_host(const double *x, const double *px, const double *y,
                              const double *py, size_t n, size_t n_samples, const uint32_t *from,
                              const uint32_t *to, size_t n_windows, int method, double *host_out) {
    if (n == 0) return hm_orbit_tunes(nullptr, nullptr, nullptr, nullptr, 0, n_samples, from, to,
                                      n_windows, method, host_out);
    if (!x || !px || !y || !py) return fail(HM_ERR_INVALID_ARG, "null orbit");
    const size_t bytes = n * n_samples * sizeof(double);
    DeviceBuffer d[4];
    const double *src[4] = {x, px, y, py};
    for (int k = 0; k < 4; ++k) {
        HM_TRY(d[k].alloc(bytes));
        HM_CUDA_TRY(cudaMemcpy(d[k].ptr, src[k], bytes, cudaMemcpyHostToDevice));
    }
    return hm_orbit_tunes(d[0].as<double>(), d[1].as<double>(), d[2].as<double>(),
                          d[3].as<double>(), n, n_samples, from, to, n_windows, method, host_out);
}

}  // extern "C"

namespace {

// cuFFT plans of the tracker's tune path (windows too long for the
// shared-memory transform), kept across calls: one per (device, length,
// batch), rows of `length` contiguous values (fft_gather2 writes both
// planes' rows, batch = 2 particles).  Creating a plan costs more than
// running it at these sizes.  Plans hold no work area of their own: each
// call lends one from the library's pool (released with the call), so a
// cached plan keeps no device memory between calls.
// Process-wide cap on the particles of one tune slice (0: none).
std::atomic<size_t> g_tune_slice_limit{0};

struct CachedPlan {
    cufftHandle plan = 0;
    size_t work = 0;  // bytes of work area an execution needs
};
struct PlanCache {
    std::mutex mutex;
    std::map<std::tuple<int, uint32_t, size_t>, CachedPlan> plans;
};

// Never destroyed: at process exit the CUDA context may already be gone,
// and the driver reclaims the plans' memory with it.
PlanCache &plan_cache() {
    static PlanCache *c = new PlanCache;
    return *c;
}

hm_status strided_plan(uint32_t len, size_t batch, CachedPlan *out) {
    int dev = 0;
    HM_CUDA_TRY(cudaGetDevice(&dev));
    PlanCache &c = plan_cache();
    std::lock_guard<std::mutex> lock(c.mutex);
    const auto key = std::make_tuple(dev, len, batch);
    auto it = c.plans.find(key);
    if (it != c.plans.end()) {
        *out = it->second;
        return ok();
    }
    if (c.plans.size() >= 16) {  // bounded: drop the whole cache
        for (auto &kv : c.plans) cufftDestroy(kv.second.plan);
        c.plans.clear();
    }
    CachedPlan cp;
    cufftResult r = cufftCreate(&cp.plan);
    if (r != CUFFT_SUCCESS) return cufft_fail(r, "create");
    int nl = int(len);
    r = cufftSetAutoAllocation(cp.plan, 0);
    if (r == CUFFT_SUCCESS)
        r = cufftMakePlanMany(cp.plan, 1, &nl, nullptr, 1, nl, nullptr, 1, nl, CUFFT_Z2Z,
                              int(batch), &cp.work);
    if (r != CUFFT_SUCCESS) {
        cufftDestroy(cp.plan);
        return cufft_fail(r, "plan");
    }
    c.plans[key] = cp;
    *out = cp;
    return ok();
}

// Forward transform of `batch` rows of `len` values in place on the
// default stream, with `work` (at least the plan's work area) lent to it.
hm_status exec_strided(uint32_t len, size_t batch, double2 *z, DeviceBuffer &work) {
    CachedPlan cp;
    HM_TRY(strided_plan(len, batch, &cp));
    HM_TRY(work.ensure(std::max<size_t>(cp.work, 1)));
    PlanCache &c = plan_cache();
    std::lock_guard<std::mutex> lock(c.mutex);  // stream and work area are per plan
    HM_CUFFT_TRY_STREAM(cp.plan);
    cufftResult r = cufftSetWorkArea(cp.plan, work.ptr);
    if (r != CUFFT_SUCCESS) return cufft_fail(r, "work area");
    auto *zc = reinterpret_cast<cufftDoubleComplex *>(z);
    r = cufftExecZ2Z(cp.plan, zc, zc, CUFFT_FORWARD);
    if (r != CUFFT_SUCCESS) return cufft_fail(r, "exec");
    return ok();
}

// Work area per row of a library transform of `len` values (an estimate
// over a batch of 1024 rows, doubled for margin).
size_t fft_work_per_row(uint32_t len) {
    size_t est = 0;
    int nl = int(len);
    if (cufftEstimateMany(1, &nl, nullptr, 1, nl, nullptr, 1, nl, CUFFT_Z2Z, 1024, &est) !=
        CUFFT_SUCCESS)
        return 8u * size_t(len) * sizeof(double2);
    return 2u * (est / 1024u + 1u);
}

// One tune window of the tracker path: inclusive sample bounds, the NaN
// rule, and the output column pair it fills.
struct Window {
    uint32_t from, to;
    bool check_nan;
    std::vector<int> cols;
};

// Equal windows are computed once and written to every column pair they
// serve (the engine appends [0, n_turns], which equals the full orbit).
void add_window(std::vector<Window> &ws, uint32_t from, uint32_t to, bool check_nan, int col) {
    for (Window &w : ws)
        if (w.from == from && w.to == to && w.check_nan == check_nan) {
            w.cols.push_back(col);
            return;
        }
    ws.push_back(Window{from, to, check_nan, {col}});
}

}  // namespace

extern "C" {

// Tracks n_turns turns recording the orbit (sample 0 = the current state),
// optionally removes each orbit's mean, and returns Birkhoff tunes (and FFT
// tunes when fft_out) of the windows plus the full orbit:
// henon_tracker::birkhoff_tunes (remove_mean = 0) and ::all_tunes
// (remove_mean = 1), src/henon.cu:2890-3078, with their kick_module and
// inverse options.  Outputs host double[n_total][2 (n_windows + 1)].
hm_status hm_tracker_orbit_tunes(hm_tracker *t, hm_particles *p, uint32_t n_turns, double mu,
                                 double barrier, double kick_module, int inverse,
                                 const uint32_t *from, const uint32_t *to, size_t n_windows,
                                 int remove_mean, double *birkhoff_out, double *fft_out) {
    if (!t || !p) return fail(HM_ERR_INVALID_ARG, "null tracker or particles");
    if (inverse) {
        if (n_turns > p->global_steps || n_turns > p->live_step)
            return fail(HM_ERR_BUDGET, "The number of turns is too large.");
    } else if (uint64_t(n_turns) + p->global_steps > t->allowed_steps) {
        return fail(HM_ERR_BUDGET, "The number of turns is too large.");
    }
    if (n_turns == 0) return fail(HM_ERR_INVALID_ARG, "need at least one turn");
    const size_t S = size_t(n_turns) + 1;
    HM_TRY(check_windows(S, from, to, n_windows));
    const size_t n = p->n_total;
    if (n && !birkhoff_out) return fail(HM_ERR_INVALID_ARG, "null output");
    const size_t cols = 2 * (n_windows + 1);
    // Birkhoff windows: the caller's (NaN when they hold a NaN sample) and
    // the full orbit [0, S-1] (no check: NaN propagates through the sums).
    // FFT windows: the caller's, and the full orbit's samples 1..S-1 (NaN
    // when any sample is).
    std::vector<Window> bw, fw;
    for (size_t j = 0; j < n_windows; ++j) {
        add_window(bw, from[j], to[j], true, int(j));
        add_window(fw, from[j], to[j], true, int(j));
    }
    add_window(bw, 0, uint32_t(S - 1), false, int(n_windows));
    add_window(fw, 1, uint32_t(S - 1), true, int(n_windows));
    // Expanded per column pair for the Birkhoff finish kernel.
    std::vector<uint32_t> bf, bt;
    std::vector<uint8_t> bchk;
    std::vector<int> bcol;
    std::vector<uint64_t> boff;
    std::vector<double> bwts;
    for (const Window &w : bw) {
        auto ww = hm::birkhoff_weights(w.to - w.from);
        for (int c : w.cols) {
            bf.push_back(w.from);
            bt.push_back(w.to);
            bchk.push_back(w.check_nan ? 1 : 0);
            bcol.push_back(c);
            boff.push_back(bwts.size());
            bwts.insert(bwts.end(), ww.begin(), ww.end());
        }
    }
    DeviceBuffer d_bf, d_bt, d_bchk, d_bcol, d_boff, d_bw;
    HM_TRY(hm::upload(d_bf, bf));
    HM_TRY(hm::upload(d_bt, bt));
    HM_TRY(hm::upload(d_bchk, bchk));
    HM_TRY(hm::upload(d_bcol, bcol));
    HM_TRY(hm::upload(d_boff, boff));
    HM_TRY(hm::upload(d_bw, bwts));
    // Hann tables of the FFT windows, and each window's transform: whole
    // in shared memory when a plan exists for its length (fft_tune_kernel),
    // else a library transform of rows gathered in global memory.
    uint32_t max_len = 0;  // longest window of the library path
    std::vector<DeviceBuffer> hann(fw.size()), fcols(fw.size());
    std::vector<const hm::FftPlanDev *> fplan(fw.size(), nullptr);
    if (fft_out) {
        for (size_t j = 0; j < fw.size(); ++j) {
            const uint32_t L = fw[j].to - fw[j].from + 1;
            HM_TRY(hann[j].alloc(size_t(L) * sizeof(double)));
            HM_CUDA_TRY(hm::launch_hann_table(hann[j].as<double>(), L, 0));
            HM_TRY(hm::fft_plan(L, &fplan[j]));
            if (fplan[j]) HM_TRY(hm::upload(fcols[j], fw[j].cols));
            else max_len = std::max(max_len, L);
        }
    }
    // Particle slice: the orbit (32 B per sample) plus, for the library
    // path's longest window, both planes' rows (32 B per sample) and the
    // transform's work area, in at most two thirds of the free device
    // memory.
    size_t free_b = 0;
    HM_TRY(hm::device_free_bytes(&free_b));
    const size_t per_particle = S * 4 * sizeof(double) +
                                (max_len ? 2 * (size_t(max_len) * sizeof(double2) +
                                                fft_work_per_row(max_len))
                                         : 0u);
    size_t slice = std::max<size_t>(1, std::min<size_t>(n, (free_b / 3 * 2) / per_particle));
    if (const size_t cap = g_tune_slice_limit.load(); cap > 0) slice = std::min(slice, cap);
    const size_t m0 = std::min(n, slice);
    // Segments of the Birkhoff sums: enough threads to fill the device.
    const uint32_t seg_len = std::max<uint32_t>(64u, uint32_t(std::min<size_t>(
                                                         S, (S * m0 * 2 + 262143) / 262144)));
    const uint32_t n_seg = uint32_t((S - 1 + seg_len - 1) / seg_len);
    DeviceBuffer orbit, out, sums, first_nan, partial, z, fft_work;
    HM_TRY(orbit.alloc(m0 * S * 4 * sizeof(double)));
    HM_TRY(out.alloc(cols * m0 * sizeof(double)));
    if (remove_mean) HM_TRY(sums.alloc(4 * m0 * sizeof(double)));
    HM_TRY(first_nan.alloc(m0 * sizeof(uint32_t)));
    HM_TRY(partial.alloc(bf.size() * 2 * size_t(std::max<uint32_t>(n_seg, 1)) * m0 * sizeof(double)));
    if (fft_out && max_len) HM_TRY(z.alloc(size_t(max_len) * 2 * m0 * sizeof(double2)));
    const double b2 = barrier * barrier;
    long long b2bits = 0;
    if (!std::isnan(b2)) std::memcpy(&b2bits, &b2, sizeof(b2));
    for (size_t first = 0; first < n; first += slice) {
        const size_t m = std::min(slice, n - first);
        double *o = orbit.as<double>();
        hm::OrbitRecordArgs a{};
        a.x = p->x.as<double>() + first;
        a.px = p->px.as<double>() + first;
        a.y = p->y.as<double>() + first;
        a.py = p->py.as<double>() + first;
        a.steps = p->steps.as<uint32_t>() + first;
        a.n = m;
        a.table = t->table.as<double>();
        a.live_step = p->live_step;
        a.n_turns = n_turns;
        a.mu = mu;
        a.b2bits = b2bits;
        a.arith = t->arith;
        a.ox = o;
        a.opx = o + S * m;
        a.oy = o + 2 * S * m;
        a.opy = o + 3 * S * m;
        a.sums = remove_mean ? sums.as<double>() : nullptr;
        a.first_nan = first_nan.as<uint32_t>();
        a.inverse = inverse != 0;
        a.kick_module = kick_module;
        a.kick_seed = p->kick_seed;
        a.id0 = first;
        HM_CUDA_TRY(hm::launch_orbit_record(a, 0));
        const double *means = remove_mean ? sums.as<double>() : nullptr;

        hm::BirkhoffSegArgs g{};
        g.x = a.ox;
        g.px = a.opx;
        g.y = a.oy;
        g.py = a.opy;
        g.means = means;
        g.first_nan = a.first_nan;
        g.n = m;
        g.S = S;
        g.seg_len = seg_len;
        g.n_seg = n_seg;
        g.from = d_bf.as<uint32_t>();
        g.to = d_bt.as<uint32_t>();
        g.w_off = d_boff.as<uint64_t>();
        g.w = d_bw.as<double>();
        g.n_win = int(bf.size());
        g.check_nan = d_bchk.as<uint8_t>();
        g.partial = partial.as<double>();
        g.out_col = d_bcol.as<int>();
        g.out = out.as<double>();
        g.cols = cols;
        HM_CUDA_TRY(hm::launch_birkhoff_segments(g, 0));
        HM_CUDA_TRY(cudaMemcpy(birkhoff_out + first * cols, out.ptr, m * cols * sizeof(double),
                               cudaMemcpyDeviceToHost));
        if (fft_out) {
            for (size_t j = 0; j < fw.size(); ++j) {
                const uint32_t L = fw[j].to - fw[j].from + 1;
                if (fplan[j]) {
                    hm::FftTuneArgs f{};
                    f.x = a.ox;
                    f.px = a.opx;
                    f.y = a.oy;
                    f.py = a.opy;
                    f.means = means;
                    f.first_nan = a.first_nan;
                    f.n = m;
                    f.S = S;
                    f.stride_i = S;
                    f.stride_s = 1;
                    f.from = fw[j].from;
                    f.last_sample = fw[j].to;
                    f.hann = hann[j].as<double>();
                    f.out = out.as<double>();
                    f.cols = cols;
                    f.out_cols = fcols[j].as<int>();
                    f.n_out_cols = int(fw[j].cols.size());
                    f.plan = *fplan[j];
                    HM_CUDA_TRY(hm::launch_fft_tunes(f, 0));
                    continue;
                }
                auto *zz = z.as<double2>();
                HM_CUDA_TRY(hm::launch_fft_gather2(a.ox, a.opx, a.oy, a.opy, means, m, fw[j].from,
                                                   L, hann[j].as<double>(), zz, S, 0));
                HM_TRY(exec_strided(L, 2 * m, zz, fft_work));
                for (int c : fw[j].cols)
                    HM_CUDA_TRY(hm::launch_fft_peak2(zz, L, m, fw[j].to, a.first_nan,
                                                     out.as<double>(), cols, c, 0));
            }
            HM_CUDA_TRY(cudaMemcpy(fft_out + first * cols, out.ptr, m * cols * sizeof(double),
                                   cudaMemcpyDeviceToHost));
        }
    }
    if (inverse) {
        p->global_steps -= n_turns;
        p->live_step -= n_turns;
    } else {
        p->global_steps += n_turns;
        p->live_step += n_turns;
    }
    return ok();
}

hm_status hm_set_tune_slice_limit(size_t max_particles) {
    g_tune_slice_limit.store(max_particles);
    return ok();
}

hm_status hm_get_tune_slice_limit(size_t *max_particles) {
    if (!max_particles) return fail(HM_ERR_INVALID_ARG, "null output");
    *max_particles = g_tune_slice_limit.load();
    return ok();
}

// storage tunes (storage_4d::tune_birkhoff / tune_fft, src/henon.cu:3261-3329)
// over the stored snapshots.
hm_status hm_storage_tunes(const hm_storage *s, const uint32_t *from, const uint32_t *to,
                           size_t n_windows, int method, double *host_out) {
    if (!s) return fail(HM_ERR_INVALID_ARG, "null storage");
    size_t n = 0, batch = 0, stored = 0;
    HM_TRY(hm_storage_size(s, &n, &batch, &stored));
    const double *c[4];
    for (int k = 0; k < 4; ++k) HM_TRY(hm_storage_device_ptr(s, hm_field(HM_FIELD_X + k), &c[k]));
    return hm_orbit_tunes(c[0], c[1], c[2], c[3], n, stored, from, to, n_windows, method, host_out);
}

}  // extern "C"
