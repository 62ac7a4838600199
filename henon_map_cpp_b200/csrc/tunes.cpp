// C ABI of the tune estimates (hm_orbit_tunes, hm_tracker_orbit_tunes,
// hm_storage_tunes): window validation, Birkhoff weight tables, cuFFT
// plans, and particle slicing so orbit buffers fit device memory.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
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

// FFT tunes of the windows (from, to) plus the full orbit [1, S-1], in
// particle slices bounded by the spectrum buffer.
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

// Tracks n_turns turns recording the orbit (sample 0 = the current state),
// optionally removes each orbit's mean, and returns Birkhoff tunes (and FFT
// tunes when fft_out) of the windows plus the full orbit:
// henon_tracker::birkhoff_tunes (remove_mean = 0) and ::all_tunes
// (remove_mean = 1), src/henon.cu:2890-3078.  Outputs host
// double[n_total][2 (n_windows + 1)].
hm_status hm_tracker_orbit_tunes(hm_tracker *t, hm_particles *p, uint32_t n_turns, double mu,
                                 double barrier, const uint32_t *from, const uint32_t *to,
                                 size_t n_windows, int remove_mean, double *birkhoff_out,
                                 double *fft_out) {
    if (!t || !p) return fail(HM_ERR_INVALID_ARG, "null tracker or particles");
    if (uint64_t(n_turns) + p->global_steps > t->allowed_steps)
        return fail(HM_ERR_BUDGET, "The number of turns is too large.");
    if (n_turns == 0) return fail(HM_ERR_INVALID_ARG, "need at least one turn");
    const size_t S = size_t(n_turns) + 1;
    HM_TRY(check_windows(S, from, to, n_windows));
    const size_t n = p->n_total;
    if (n && !birkhoff_out) return fail(HM_ERR_INVALID_ARG, "null output");
    const std::vector<uint32_t> f(from, from + n_windows), tt(to, to + n_windows);
    const size_t cols = 2 * (n_windows + 1);
    // Orbit slice: at most half the free device memory.
    size_t free_b = 0;
    HM_TRY(hm::device_free_bytes(&free_b));
    const size_t per_particle = S * 4 * sizeof(double);
    const size_t slice = std::max<size_t>(1, std::min<size_t>(n, (free_b / 2) / per_particle));
    DeviceBuffer orbit, out;
    HM_TRY(orbit.alloc(std::min(n, slice) * per_particle));
    HM_TRY(out.alloc(cols * std::min(n, slice) * sizeof(double)));
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
        HM_CUDA_TRY(hm::launch_orbit_record(a, 0));
        if (remove_mean) HM_CUDA_TRY(hm::launch_mean_remove(a.ox, a.opx, a.oy, a.opy, m, S, 0));
        HM_TRY(birkhoff_device(a.ox, a.opx, a.oy, a.opy, m, S, f, tt, out.as<double>()));
        HM_CUDA_TRY(cudaMemcpy(birkhoff_out + first * cols, out.ptr, m * cols * sizeof(double),
                               cudaMemcpyDeviceToHost));
        if (fft_out) {
            HM_TRY(fft_device(a.ox, a.opx, a.oy, a.opy, m, S, f, tt, out.as<double>()));
            HM_CUDA_TRY(cudaMemcpy(fft_out + first * cols, out.ptr, m * cols * sizeof(double),
                                   cudaMemcpyDeviceToHost));
        }
    }
    p->global_steps += n_turns;
    p->live_step += n_turns;
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
