// C ABI of the tangent-map containers and indicator constructs
// (matrix_4d_vector_gpu, vector_4d_gpu, lyapunov_birkhoff_construct[_multi],
// megno_construct, megno_birkhoff_construct, tune_birkhoff_construct,
// storage_4d_gpu: src/henon.h:265-447, src/henon.cu:1789-2655, 3351-3462).
//
// Every operation is one elementwise launch on the legacy default stream,
// as in the reference; the fused multi-turn path is hm_track_indicators.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "hm_internal.h"

using hm::DeviceBuffer;
using hm::fail;
using hm::ok;

struct hm_matrices {
    size_t n = 0;
    DeviceBuffer m;  // double[n][16]
};

struct hm_vectors {
    size_t n = 0;
    DeviceBuffer v;  // double[n][4]
};

// Birkhoff weight tables of several windows, concatenated on the device.
struct WeightSet {
    std::vector<uint64_t> len;
    DeviceBuffer weights, off, dlen;
    hm_status build(const std::vector<uint64_t> &lengths) {
        len = lengths;
        std::vector<double> all;
        std::vector<uint64_t> offs;
        for (uint64_t l : lengths) {
            offs.push_back(all.size());
            auto w = hm::birkhoff_weights(uint32_t(l));
            all.insert(all.end(), w.begin(), w.end());
        }
        HM_TRY(hm::upload(weights, all));
        HM_TRY(hm::upload(off, offs));
        return hm::upload(dlen, lengths);
    }
};

struct hm_lyapunov {
    size_t n = 0;
    size_t idx = 0;
    WeightSet w;
    DeviceBuffer raw, bsum;  // double[n_windows][n]
};

struct hm_megno {
    size_t n = 0;
    size_t idx = 1;
    DeviceBuffer l1, l2, l3;
};

struct hm_megno_birkhoff {
    size_t n = 0;
    size_t idx = 1;
    WeightSet w;
    DeviceBuffer l1, l2;  // l2: double[n_windows][n]
};

struct hm_tune_birkhoff {
    size_t n = 0;
    size_t idx = 1;
    bool first_done = false;
    WeightSet w;
    DeviceBuffer store_x, store_y, t1x, t1y, t2x, t2y;
};

struct hm_storage {
    size_t n = 0, batch = 0, idx = 0;
    DeviceBuffer x, px, y, py;  // double[batch][n]
};

namespace {

hm_status zeros(DeviceBuffer &b, size_t bytes) {
    HM_TRY(b.alloc(bytes));
    if (bytes) HM_CUDA_TRY(cudaMemset(b.ptr, 0, bytes));
    return ok();
}

hm_status to_host(void *dst, const DeviceBuffer &src, size_t bytes) {
    if (bytes == 0) return ok();
    if (!dst) return fail(HM_ERR_INVALID_ARG, "null output");
    HM_CUDA_TRY(cudaMemcpy(dst, src.ptr, bytes, cudaMemcpyDeviceToHost));
    return ok();
}

hm_status check_particles(size_t n, const hm_particles *p) {
    if (!p) return fail(HM_ERR_INVALID_ARG, "null particles");
    if (p->n_total < n)
        return fail(HM_ERR_INVALID_ARG, "construct is larger than the particle ensemble");
    return ok();
}

template <class H>
hm_status make(H **out, H *h, hm_status s) {
    if (s != HM_OK) {
        delete h;
        return s;
    }
    *out = h;
    return ok();
}

// Table index of the tangent matrix: the particles' global_steps, as in
// matrix_4d_vector_gpu::structured_multiply (src/henon.cu:1827-1845).
hm_status matrices_step(hm_matrices *m, const hm_tracker *t, const hm_particles *p, double mu,
                        bool set) {
    if (!m || !t) return fail(HM_ERR_INVALID_ARG, "null matrices or tracker");
    HM_TRY(check_particles(m->n, p));
    if (m->n && p->global_steps >= t->allowed_steps)
        return fail(HM_ERR_BUDGET,
                    "The number of turns is too large. (tangent matrix past the table end)");
    HM_CUDA_TRY(hm::launch_matrices_step(m->m.as<double>(), p->x.as<double>(), p->px.as<double>(),
                                         p->y.as<double>(), p->py.as<double>(),
                                         t->table.as<double>(), p->global_steps, mu, m->n, set, 0));
    return ok();
}

}  // namespace

extern "C" {

// ---- matrix_4d_vector_gpu ---------------------------------------------------------

hm_status hm_matrices_create(size_t n, hm_matrices **out) {
    if (!out) return fail(HM_ERR_INVALID_ARG, "null output handle");
    *out = nullptr;
    auto *m = new hm_matrices();
    m->n = n;
    hm_status s = m->m.alloc(n * 16 * sizeof(double));
    if (s == HM_OK && n) {
        cudaError_t e = hm::launch_matrices_identity(m->m.as<double>(), n, 0);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) s = hm::cuda_fail(e, "identity matrices");
    }
    return make(out, m, s);
}

hm_status hm_matrices_destroy(hm_matrices *m) {
    delete m;
    return ok();
}

hm_status hm_matrices_size(const hm_matrices *m, size_t *n) {
    if (!m || !n) return fail(HM_ERR_INVALID_ARG, "null pointer");
    *n = m->n;
    return ok();
}

hm_status hm_matrices_reset(hm_matrices *m) {
    if (!m) return fail(HM_ERR_INVALID_ARG, "null matrices");
    HM_CUDA_TRY(hm::launch_matrices_identity(m->m.as<double>(), m->n, 0));
    return ok();
}

hm_status hm_matrices_structured_multiply(hm_matrices *m, const hm_tracker *t,
                                          const hm_particles *p, double mu) {
    return matrices_step(m, t, p, mu, false);
}

hm_status hm_matrices_set_with_tracker(hm_matrices *m, const hm_tracker *t, const hm_particles *p,
                                       double mu) {
    return matrices_step(m, t, p, mu, true);
}

hm_status hm_matrices_copy(hm_matrices *dst, const hm_matrices *src) {
    if (!dst || !src) return fail(HM_ERR_INVALID_ARG, "null matrices");
    if (dst->n != src->n) return fail(HM_ERR_INVALID_ARG, "matrix sets differ in size");
    if (dst->n)
        HM_CUDA_TRY(cudaMemcpy(dst->m.ptr, src->m.ptr, dst->n * 16 * sizeof(double),
                               cudaMemcpyDeviceToDevice));
    return ok();
}

hm_status hm_matrices_get(const hm_matrices *m, double *host_out) {
    if (!m) return fail(HM_ERR_INVALID_ARG, "null matrices");
    return to_host(host_out, m->m, m->n * 16 * sizeof(double));
}

hm_status hm_matrices_get_vector(const hm_matrices *m, const double *host_rv, double *host_out) {
    if (!m) return fail(HM_ERR_INVALID_ARG, "null matrices");
    if (m->n == 0) return ok();
    if (!host_rv || !host_out) return fail(HM_ERR_INVALID_ARG, "null vector");
    DeviceBuffer rv, out;
    HM_TRY(rv.alloc(m->n * 4 * sizeof(double)));
    HM_TRY(out.alloc(m->n * 4 * sizeof(double)));
    HM_CUDA_TRY(cudaMemcpy(rv.ptr, host_rv, m->n * 4 * sizeof(double), cudaMemcpyHostToDevice));
    HM_CUDA_TRY(hm::launch_matrices_apply(m->m.as<double>(), rv.as<double>(), out.as<double>(),
                                          m->n, 0));
    return to_host(host_out, out, m->n * 4 * sizeof(double));
}

// ---- vector_4d_gpu ------------------------------------------------------------------

hm_status hm_vectors_create(const double *host, size_t n, hm_vectors **out) {
    if (!out) return fail(HM_ERR_INVALID_ARG, "null output handle");
    *out = nullptr;
    if (n && !host) return fail(HM_ERR_INVALID_ARG, "null vectors");
    auto *v = new hm_vectors();
    v->n = n;
    hm_status s = v->v.alloc(n * 4 * sizeof(double));
    if (s == HM_OK && n) {
        const cudaError_t e =
            cudaMemcpy(v->v.ptr, host, n * 4 * sizeof(double), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) s = hm::cuda_fail(e, "vectors upload");
    }
    return make(out, v, s);
}

hm_status hm_vectors_destroy(hm_vectors *v) {
    delete v;
    return ok();
}

hm_status hm_vectors_set(hm_vectors *v, const double *host, int broadcast) {
    if (!v) return fail(HM_ERR_INVALID_ARG, "null vectors");
    if (v->n == 0) return ok();
    if (!host) return fail(HM_ERR_INVALID_ARG, "null data");
    if (broadcast) {
        std::vector<double> rep(v->n * 4);
        for (size_t i = 0; i < v->n; ++i) std::memcpy(&rep[4 * i], host, 4 * sizeof(double));
        HM_CUDA_TRY(cudaMemcpy(v->v.ptr, rep.data(), rep.size() * sizeof(double),
                               cudaMemcpyHostToDevice));
    } else {
        HM_CUDA_TRY(cudaMemcpy(v->v.ptr, host, v->n * 4 * sizeof(double), cudaMemcpyHostToDevice));
    }
    return ok();
}

hm_status hm_vectors_multiply(hm_vectors *v, const hm_matrices *m) {
    if (!v || !m) return fail(HM_ERR_INVALID_ARG, "null vectors or matrices");
    if (m->n < v->n) return fail(HM_ERR_INVALID_ARG, "fewer matrices than vectors");
    HM_CUDA_TRY(hm::launch_vectors_multiply(m->m.as<double>(), v->v.as<double>(), v->n, 0));
    return ok();
}

hm_status hm_vectors_normalize(hm_vectors *v) {
    if (!v) return fail(HM_ERR_INVALID_ARG, "null vectors");
    HM_CUDA_TRY(hm::launch_vectors_normalize(v->v.as<double>(), v->n, 0));
    return ok();
}

hm_status hm_vectors_get(const hm_vectors *v, double *host_out) {
    if (!v) return fail(HM_ERR_INVALID_ARG, "null vectors");
    return to_host(host_out, v->v, v->n * 4 * sizeof(double));
}

// ---- lyapunov_birkhoff_construct[_multi] ----------------------------------------------

hm_status hm_lyapunov_create(size_t n, const uint64_t *n_weights, size_t n_windows,
                             hm_lyapunov **out) {
    if (!out) return fail(HM_ERR_INVALID_ARG, "null output handle");
    *out = nullptr;
    if (n_windows && !n_weights) return fail(HM_ERR_INVALID_ARG, "null window list");
    for (size_t i = 0; i < n_windows; ++i)
        if (n_weights[i] == 0 || n_weights[i] > 0xffffffffULL)
            return fail(HM_ERR_INVALID_ARG, "window lengths must be in [1, 2^32)");
    auto *h = new hm_lyapunov();
    h->n = n;
    hm_status s = h->w.build(std::vector<uint64_t>(n_weights, n_weights + n_windows));
    if (s == HM_OK) s = zeros(h->raw, n_windows * n * sizeof(double));
    if (s == HM_OK) s = zeros(h->bsum, n_windows * n * sizeof(double));
    return make(out, h, s);
}

hm_status hm_lyapunov_destroy(hm_lyapunov *h) {
    delete h;
    return ok();
}

hm_status hm_lyapunov_reset(hm_lyapunov *h) {
    if (!h) return fail(HM_ERR_INVALID_ARG, "null construct");
    h->idx = 0;
    const size_t bytes = h->w.len.size() * h->n * sizeof(double);
    if (bytes) {
        HM_CUDA_TRY(cudaMemset(h->raw.ptr, 0, bytes));
        HM_CUDA_TRY(cudaMemset(h->bsum.ptr, 0, bytes));
    }
    return ok();
}

hm_status hm_lyapunov_change_weights(hm_lyapunov *h, uint64_t n_weights) {
    if (!h) return fail(HM_ERR_INVALID_ARG, "null construct");
    if (h->w.len.size() != 1)
        return fail(HM_ERR_INVALID_ARG, "change_weights needs a single-window construct");
    if (n_weights == 0 || n_weights > 0xffffffffULL)
        return fail(HM_ERR_INVALID_ARG, "window length must be in [1, 2^32)");
    return h->w.build({n_weights});
}

hm_status hm_lyapunov_add(hm_lyapunov *h, const hm_vectors *v) {
    if (!h || !v) return fail(HM_ERR_INVALID_ARG, "null construct or vectors");
    if (v->n < h->n) return fail(HM_ERR_INVALID_ARG, "fewer vectors than the construct");
    HM_CUDA_TRY(hm::launch_lyapunov(h->raw.as<double>(), h->bsum.as<double>(), v->v.as<double>(),
                                    h->w.weights.as<double>(), h->w.off.as<uint64_t>(),
                                    h->w.dlen.as<uint64_t>(), int(h->w.len.size()), h->idx, h->n,
                                    0));
    h->idx += 1;
    return ok();
}

hm_status hm_lyapunov_windows(const hm_lyapunov *h, size_t *n_windows) {
    if (!h || !n_windows) return fail(HM_ERR_INVALID_ARG, "null pointer");
    *n_windows = h->w.len.size();
    return ok();
}

hm_status hm_lyapunov_get_weights(const hm_lyapunov *h, size_t window, double *host_out) {
    if (!h) return fail(HM_ERR_INVALID_ARG, "null construct");
    if (window >= h->w.len.size()) return fail(HM_ERR_INVALID_ARG, "window out of range");
    std::vector<uint64_t> off(h->w.len.size());
    HM_CUDA_TRY(cudaMemcpy(off.data(), h->w.off.ptr, off.size() * sizeof(uint64_t),
                           cudaMemcpyDeviceToHost));
    if (!host_out) return fail(HM_ERR_INVALID_ARG, "null output");
    HM_CUDA_TRY(cudaMemcpy(host_out, h->w.weights.as<double>() + off[window],
                           h->w.len[window] * sizeof(double), cudaMemcpyDeviceToHost));
    return ok();
}

// birkhoff == 0: raw averages (get_values_raw); 1: weighted (get_values_b).
// Output: double[n_windows][n].
hm_status hm_lyapunov_get(const hm_lyapunov *h, int birkhoff, double *host_out) {
    if (!h) return fail(HM_ERR_INVALID_ARG, "null construct");
    return to_host(host_out, birkhoff ? h->bsum : h->raw, h->w.len.size() * h->n * sizeof(double));
}

// ---- megno_construct --------------------------------------------------------------------

hm_status hm_megno_create(size_t n, hm_megno **out) {
    if (!out) return fail(HM_ERR_INVALID_ARG, "null output handle");
    *out = nullptr;
    auto *h = new hm_megno();
    h->n = n;
    hm_status s = zeros(h->l1, n * sizeof(double));
    if (s == HM_OK) s = zeros(h->l2, n * sizeof(double));
    if (s == HM_OK) s = zeros(h->l3, n * sizeof(double));
    return make(out, h, s);
}

hm_status hm_megno_destroy(hm_megno *h) {
    delete h;
    return ok();
}

hm_status hm_megno_reset(hm_megno *h) {
    if (!h) return fail(HM_ERR_INVALID_ARG, "null construct");
    h->idx = 1;
    if (h->n) {
        HM_CUDA_TRY(cudaMemset(h->l1.ptr, 0, h->n * sizeof(double)));
        HM_CUDA_TRY(cudaMemset(h->l2.ptr, 0, h->n * sizeof(double)));
        HM_CUDA_TRY(cudaMemset(h->l3.ptr, 0, h->n * sizeof(double)));
    }
    return ok();
}

hm_status hm_megno_add(hm_megno *h, const hm_matrices *a, const hm_matrices *b) {
    if (!h || !a || !b) return fail(HM_ERR_INVALID_ARG, "null construct or matrices");
    if (a->n < h->n || b->n < h->n) return fail(HM_ERR_INVALID_ARG, "fewer matrices than the construct");
    HM_CUDA_TRY(hm::launch_megno(h->l1.as<double>(), h->l2.as<double>(), h->l3.as<double>(),
                                 a->m.as<double>(), b->m.as<double>(), h->idx, h->n, 0));
    h->idx += 1;
    return ok();
}

hm_status hm_megno_get(const hm_megno *h, double *host_out) {
    if (!h) return fail(HM_ERR_INVALID_ARG, "null construct");
    return to_host(host_out, h->l3, h->n * sizeof(double));
}

// ---- megno_birkhoff_construct ------------------------------------------------------------

hm_status hm_megno_birkhoff_create(size_t n, const uint64_t *turn_samples, size_t n_samples,
                                   hm_megno_birkhoff **out) {
    if (!out) return fail(HM_ERR_INVALID_ARG, "null output handle");
    *out = nullptr;
    if (n_samples && !turn_samples) return fail(HM_ERR_INVALID_ARG, "null turn samples");
    for (size_t i = 0; i < n_samples; ++i)
        if (turn_samples[i] == 0 || turn_samples[i] > 0xffffffffULL)
            return fail(HM_ERR_INVALID_ARG, "turn samples must be in [1, 2^32)");
    auto *h = new hm_megno_birkhoff();
    h->n = n;
    hm_status s = h->w.build(std::vector<uint64_t>(turn_samples, turn_samples + n_samples));
    if (s == HM_OK) s = zeros(h->l1, n * sizeof(double));
    if (s == HM_OK) s = zeros(h->l2, n_samples * n * sizeof(double));
    return make(out, h, s);
}

hm_status hm_megno_birkhoff_destroy(hm_megno_birkhoff *h) {
    delete h;
    return ok();
}

hm_status hm_megno_birkhoff_reset(hm_megno_birkhoff *h) {
    if (!h) return fail(HM_ERR_INVALID_ARG, "null construct");
    h->idx = 1;
    if (h->n) HM_CUDA_TRY(cudaMemset(h->l1.ptr, 0, h->n * sizeof(double)));
    if (h->n && !h->w.len.empty())
        HM_CUDA_TRY(cudaMemset(h->l2.ptr, 0, h->w.len.size() * h->n * sizeof(double)));
    return ok();
}

hm_status hm_megno_birkhoff_add(hm_megno_birkhoff *h, const hm_matrices *a, const hm_matrices *b) {
    if (!h || !a || !b) return fail(HM_ERR_INVALID_ARG, "null construct or matrices");
    if (a->n < h->n || b->n < h->n) return fail(HM_ERR_INVALID_ARG, "fewer matrices than the construct");
    HM_CUDA_TRY(hm::launch_megno_birkhoff(h->l1.as<double>(), h->l2.as<double>(),
                                          h->w.weights.as<double>(), h->w.off.as<uint64_t>(),
                                          h->w.dlen.as<uint64_t>(), int(h->w.len.size()),
                                          a->m.as<double>(), b->m.as<double>(), h->idx, h->n, 0));
    h->idx += 1;
    return ok();
}

// Output: double[n_samples][n].
hm_status hm_megno_birkhoff_get(const hm_megno_birkhoff *h, double *host_out) {
    if (!h) return fail(HM_ERR_INVALID_ARG, "null construct");
    return to_host(host_out, h->l2, h->w.len.size() * h->n * sizeof(double));
}

// ---- tune_birkhoff_construct ---------------------------------------------------------------

hm_status hm_tune_birkhoff_create(size_t n, const uint64_t *turn_samples, size_t n_samples,
                                  hm_tune_birkhoff **out) {
    if (!out) return fail(HM_ERR_INVALID_ARG, "null output handle");
    *out = nullptr;
    if (n_samples && !turn_samples) return fail(HM_ERR_INVALID_ARG, "null turn samples");
    for (size_t i = 0; i < n_samples; ++i)
        if (turn_samples[i] == 0 || turn_samples[i] > 0x7fffffffULL)
            return fail(HM_ERR_INVALID_ARG, "turn samples must be in [1, 2^31)");
    auto *h = new hm_tune_birkhoff();
    h->n = n;
    hm_status s = h->w.build(std::vector<uint64_t>(turn_samples, turn_samples + n_samples));
    const size_t acc = n_samples * n * sizeof(double);
    if (s == HM_OK) s = zeros(h->store_x, n * sizeof(double));
    if (s == HM_OK) s = zeros(h->store_y, n * sizeof(double));
    if (s == HM_OK) s = zeros(h->t1x, acc);
    if (s == HM_OK) s = zeros(h->t1y, acc);
    if (s == HM_OK) s = zeros(h->t2x, acc);
    if (s == HM_OK) s = zeros(h->t2y, acc);
    return make(out, h, s);
}

hm_status hm_tune_birkhoff_destroy(hm_tune_birkhoff *h) {
    delete h;
    return ok();
}

hm_status hm_tune_birkhoff_reset(hm_tune_birkhoff *h) {
    if (!h) return fail(HM_ERR_INVALID_ARG, "null construct");
    h->idx = 1;
    const size_t acc = h->w.len.size() * h->n * sizeof(double);
    if (acc) {
        HM_CUDA_TRY(cudaMemset(h->t1x.ptr, 0, acc));
        HM_CUDA_TRY(cudaMemset(h->t1y.ptr, 0, acc));
        HM_CUDA_TRY(cudaMemset(h->t2x.ptr, 0, acc));
        HM_CUDA_TRY(cudaMemset(h->t2y.ptr, 0, acc));
    }
    return ok();
}

hm_status hm_tune_birkhoff_first_add(hm_tune_birkhoff *h, const hm_particles *p) {
    if (!h) return fail(HM_ERR_INVALID_ARG, "null construct");
    HM_TRY(check_particles(h->n, p));
    HM_CUDA_TRY(hm::launch_tune_init(p->x.as<double>(), p->px.as<double>(), p->y.as<double>(),
                                     p->py.as<double>(), h->store_x.as<double>(),
                                     h->store_y.as<double>(), h->n, 0));
    h->first_done = true;
    return ok();
}

hm_status hm_tune_birkhoff_add(hm_tune_birkhoff *h, const hm_particles *p) {
    if (!h) return fail(HM_ERR_INVALID_ARG, "null construct");
    HM_TRY(check_particles(h->n, p));
    if (!h->first_done) return fail(HM_ERR_INVALID_ARG, "First call add_first");
    HM_CUDA_TRY(hm::launch_tune_add(p->x.as<double>(), p->px.as<double>(), p->y.as<double>(),
                                    p->py.as<double>(), h->store_x.as<double>(),
                                    h->store_y.as<double>(), h->t1x.as<double>(),
                                    h->t1y.as<double>(), h->t2x.as<double>(), h->t2y.as<double>(),
                                    h->w.weights.as<double>(), h->w.off.as<uint64_t>(),
                                    h->w.dlen.as<uint64_t>(), int(h->w.len.size()), h->idx, h->n,
                                    0));
    h->idx += 1;
    return ok();
}

// which: 0 tune1_x, 1 tune1_y, 2 tune2_x, 3 tune2_y.  Output double[n_samples][n].
hm_status hm_tune_birkhoff_get(const hm_tune_birkhoff *h, int which, double *host_out) {
    if (!h) return fail(HM_ERR_INVALID_ARG, "null construct");
    const DeviceBuffer *b[4] = {&h->t1x, &h->t1y, &h->t2x, &h->t2y};
    if (which < 0 || which > 3) return fail(HM_ERR_INVALID_ARG, "which must be 0..3");
    return to_host(host_out, *b[which], h->w.len.size() * h->n * sizeof(double));
}

// ---- storage_4d_gpu -------------------------------------------------------------------------

hm_status hm_storage_create(size_t n, size_t batch, hm_storage **out) {
    if (!out) return fail(HM_ERR_INVALID_ARG, "null output handle");
    *out = nullptr;
    auto *h = new hm_storage();
    h->n = n;
    h->batch = batch;
    const size_t bytes = n * batch * sizeof(double);
    hm_status s = zeros(h->x, bytes);
    if (s == HM_OK) s = zeros(h->px, bytes);
    if (s == HM_OK) s = zeros(h->y, bytes);
    if (s == HM_OK) s = zeros(h->py, bytes);
    return make(out, h, s);
}

hm_status hm_storage_destroy(hm_storage *h) {
    delete h;
    return ok();
}

hm_status hm_storage_store(hm_storage *h, const hm_particles *p) {
    if (!h) return fail(HM_ERR_INVALID_ARG, "null storage");
    HM_TRY(check_particles(h->n, p));
    if (h->idx >= h->batch) return fail(HM_ERR_INVALID_ARG, "storage is full (batch_size reached)");
    const size_t bytes = h->n * sizeof(double);
    const size_t off = h->idx * h->n;
    if (bytes) {
        HM_CUDA_TRY(cudaMemcpy(h->x.as<double>() + off, p->x.ptr, bytes, cudaMemcpyDeviceToDevice));
        HM_CUDA_TRY(cudaMemcpy(h->px.as<double>() + off, p->px.ptr, bytes, cudaMemcpyDeviceToDevice));
        HM_CUDA_TRY(cudaMemcpy(h->y.as<double>() + off, p->y.ptr, bytes, cudaMemcpyDeviceToDevice));
        HM_CUDA_TRY(cudaMemcpy(h->py.as<double>() + off, p->py.ptr, bytes, cudaMemcpyDeviceToDevice));
    }
    h->idx += 1;
    return ok();
}

hm_status hm_storage_reset(hm_storage *h) {
    if (!h) return fail(HM_ERR_INVALID_ARG, "null storage");
    h->idx = 0;
    const size_t bytes = h->n * h->batch * sizeof(double);
    if (bytes) {
        HM_CUDA_TRY(cudaMemset(h->x.ptr, 0, bytes));
        HM_CUDA_TRY(cudaMemset(h->px.ptr, 0, bytes));
        HM_CUDA_TRY(cudaMemset(h->y.ptr, 0, bytes));
        HM_CUDA_TRY(cudaMemset(h->py.ptr, 0, bytes));
    }
    return ok();
}

hm_status hm_storage_size(const hm_storage *h, size_t *n, size_t *batch, size_t *stored) {
    if (!h) return fail(HM_ERR_INVALID_ARG, "null storage");
    if (n) *n = h->n;
    if (batch) *batch = h->batch;
    if (stored) *stored = h->idx;
    return ok();
}

// field: HM_FIELD_X..HM_FIELD_PY.  Output double[batch][n].
hm_status hm_storage_get(const hm_storage *h, hm_field field, double *host_out) {
    if (!h) return fail(HM_ERR_INVALID_ARG, "null storage");
    const DeviceBuffer *b[4] = {&h->x, &h->px, &h->y, &h->py};
    if (field < HM_FIELD_X || field > HM_FIELD_PY) return fail(HM_ERR_INVALID_ARG, "field must be x, px, y or py");
    return to_host(host_out, *b[field], h->n * h->batch * sizeof(double));
}

// ---- fused tracking + indicators ----------------------------------------------------------

}  // extern "C"

namespace {

// The fused construct loop; kick_module (NaN: none) and inverse only for
// whole-orbit MEGNO (hm_tracker_megno).
hm_status track_indicators(hm_tracker *t, hm_particles *p, uint32_t n_turns, double mu,
                           double barrier, const hm_indicator_set *set, double kick_module,
                           bool inverse) {
    if (!t || !p || !set) return fail(HM_ERR_INVALID_ARG, "null tracker, particles or set");
    const size_t n = p->n_total;
    const hm_indicator_set &s = *set;
    if ((s.megno || s.megno_birkhoff || s.matrix_old) && !s.matrix)
        return fail(HM_ERR_INVALID_ARG, "MEGNO needs the tangent matrix (set.matrix)");
    if (s.lyapunov && !s.vectors)
        return fail(HM_ERR_INVALID_ARG, "the Lyapunov construct needs tangent vectors (set.vectors)");
    if (s.n_megno_samples && !s.megno)
        return fail(HM_ERR_INVALID_ARG, "MEGNO samples need set.megno");
    auto size_ok = [n](size_t m) { return m == n; };
    if ((s.matrix && !size_ok(s.matrix->n)) || (s.matrix_old && !size_ok(s.matrix_old->n)) ||
        (s.megno && !size_ok(s.megno->n)) || (s.megno_birkhoff && !size_ok(s.megno_birkhoff->n)) ||
        (s.vectors && !size_ok(s.vectors->n)) || (s.lyapunov && !size_ok(s.lyapunov->n)) ||
        (s.tune && !size_ok(s.tune->n)))
        return fail(HM_ERR_INVALID_ARG, "every construct must have the particle count as size");
    if (s.tune && !s.tune->first_done) return fail(HM_ERR_INVALID_ARG, "First call add_first");
    const size_t slots = (s.megno_birkhoff ? s.megno_birkhoff->w.len.size() : 0) +
                         2 * (s.lyapunov ? s.lyapunov->w.len.size() : 0) +
                         4 * (s.tune ? s.tune->w.len.size() : 0);
    if (slots > hm::fused_max_slots())
        return fail(HM_ERR_INVALID_ARG, "too many indicator windows for the fused kernel (max "
                                        "n_megno_birkhoff + 2 n_lyapunov + 4 n_tune = 96)");
    // Turn budget (src/henon.cu:3158-3167) and the table read of
    // structured_multiply after the last turn.
    const bool tangent = (s.matrix || s.vectors) && !s.jacobian_of_turn;
    if (inverse) {
        if (n_turns > p->global_steps || n_turns > p->live_step)
            return fail(HM_ERR_BUDGET, "The number of turns is too large.");
    } else if (uint64_t(n_turns) + p->global_steps + (tangent ? 1 : 0) > t->allowed_steps) {
        return fail(HM_ERR_BUDGET, "The number of turns is too large.");
    }
    if (n_turns == 0) return ok();

    hm::DeviceBuffer snap_turns, snap;
    if (s.n_megno_samples) {
        if (!s.megno_sample_turns) return fail(HM_ERR_INVALID_ARG, "null MEGNO sample turns");
        HM_TRY(hm::upload(snap_turns, std::vector<uint64_t>(s.megno_sample_turns,
                                                            s.megno_sample_turns + s.n_megno_samples)));
        HM_TRY(snap.alloc(s.n_megno_samples * n * sizeof(double)));
        if (s.megno_samples_out)
            HM_CUDA_TRY(cudaMemcpy(snap.ptr, s.megno_samples_out, s.n_megno_samples * n * sizeof(double),
                                   cudaMemcpyHostToDevice));
        else
            HM_CUDA_TRY(cudaMemset(snap.ptr, 0xff, s.n_megno_samples * n * sizeof(double)));
    }

    hm::FusedArgs a{};
    a.x = p->x.as<double>();
    a.px = p->px.as<double>();
    a.y = p->y.as<double>();
    a.py = p->py.as<double>();
    a.steps = p->steps.as<uint32_t>();
    a.n = uint32_t(n);
    a.table = t->table.as<double>();
    a.mu = mu;
    const double b2 = barrier * barrier;
    a.b2bits = 0;
    if (!std::isnan(b2)) std::memcpy(&a.b2bits, &b2, sizeof(b2));
    a.df_before = s.jacobian_of_turn ? 1 : 0;
    a.kick_module = kick_module;
    a.kick_seed = p->kick_seed;
    a.inverse = inverse ? 1 : 0;
    if (s.matrix) a.M = s.matrix->m.as<double>();
    if (s.megno) {
        a.megno_l1 = s.megno->l1.as<double>();
        a.megno_l2 = s.megno->l2.as<double>();
        a.megno_l3 = s.megno->l3.as<double>();
        a.snap = snap.as<double>();
        a.snap_turns = snap_turns.as<uint64_t>();
        a.n_snap = int(s.n_megno_samples);
    }
    if (s.megno_birkhoff) {
        a.mb_l1 = s.megno_birkhoff->l1.as<double>();
        a.mb_l2 = s.megno_birkhoff->l2.as<double>();
        a.mb_T = s.megno_birkhoff->w.dlen.as<uint64_t>();
        a.mb_off = s.megno_birkhoff->w.off.as<uint64_t>();
        a.mb_w = s.megno_birkhoff->w.weights.as<double>();
        a.n_mb = int(s.megno_birkhoff->w.len.size());
    }
    if (s.vectors) a.V = s.vectors->v.as<double>();
    if (s.lyapunov) {
        a.ly_raw = s.lyapunov->raw.as<double>();
        a.ly_b = s.lyapunov->bsum.as<double>();
        a.ly_len = s.lyapunov->w.dlen.as<uint64_t>();
        a.ly_off = s.lyapunov->w.off.as<uint64_t>();
        a.ly_w = s.lyapunov->w.weights.as<double>();
        a.n_ly = int(s.lyapunov->w.len.size());
    }
    if (s.tune) {
        a.store_x = s.tune->store_x.as<double>();
        a.store_y = s.tune->store_y.as<double>();
        a.t1x = s.tune->t1x.as<double>();
        a.t1y = s.tune->t1y.as<double>();
        a.t2x = s.tune->t2x.as<double>();
        a.t2y = s.tune->t2y.as<double>();
        a.tu_T = s.tune->w.dlen.as<uint64_t>();
        a.tu_off = s.tune->w.off.as<uint64_t>();
        a.tu_w = s.tune->w.weights.as<double>();
        a.n_tu = int(s.tune->w.len.size());
    }

    // Chunks of turns (cancellation points); matrix_old is refreshed from
    // the matrix right before the last turn.
    const uint32_t chunk = 4096;
    uint32_t done = 0;
    hm_status status = ok();
    while (done < n_turns) {
        uint32_t len = std::min(chunk, n_turns - done);
        const bool old_needed = s.matrix_old != nullptr;
        if (old_needed && done + len == n_turns) {
            if (len > 1) len -= 1;  // stop one turn short, copy, then the last turn
            else HM_TRY(hm_matrices_copy(s.matrix_old, s.matrix));
        }
        a.live_step = p->live_step;
        a.global_step = p->global_steps;
        a.n_turns = len;
        a.megno_idx = s.megno ? s.megno->idx : 0;
        a.mb_idx = s.megno_birkhoff ? s.megno_birkhoff->idx : 0;
        a.ly_idx = s.lyapunov ? s.lyapunov->idx : 0;
        a.tu_idx = s.tune ? s.tune->idx : 0;
        HM_CUDA_TRY(hm::launch_indicators(a, 0));
        HM_CUDA_TRY(cudaDeviceSynchronize());
        if (inverse) {
            p->live_step -= len;
            p->global_steps -= len;
        } else {
            p->live_step += len;
            p->global_steps += len;
        }
        if (s.megno) s.megno->idx += len;
        if (s.megno_birkhoff) s.megno_birkhoff->idx += len;
        if (s.lyapunov) s.lyapunov->idx += len;
        if (s.tune) s.tune->idx += len;
        done += len;
        if (done < n_turns && hm::cancel_requested()) {
            status = fail(HM_ERR_CANCELLED, "tracking cancelled");
            break;
        }
    }
    if (s.n_megno_samples && s.megno_samples_out)
        HM_CUDA_TRY(cudaMemcpy(s.megno_samples_out, snap.ptr, s.n_megno_samples * n * sizeof(double),
                               cudaMemcpyDeviceToHost));
    return status;
}

}  // namespace

extern "C" {

hm_status hm_track_indicators(hm_tracker *t, hm_particles *p, uint32_t n_turns, double mu,
                              double barrier, const hm_indicator_set *set) {
    return track_indicators(t, p, n_turns, mu, barrier, set, std::nan(""), false);
}

// henon_tracker::megno (src/henon.cu:2755-2887) on the GPU, with the
// megno_construct definition (Frobenius norm, src/henon.cu:2253-2284) of
// the tangent map of the orbit (the Jacobian of each turn at the point
// before it), its kick_module and inverse options included.
hm_status hm_tracker_megno(hm_tracker *t, hm_particles *p, uint32_t n_turns, double mu,
                           double barrier, double kick_module, int inverse,
                           const uint64_t *turn_samples, size_t n_samples, double *host_out) {
    if (!t || !p) return fail(HM_ERR_INVALID_ARG, "null tracker or particles");
    if (n_samples && (!turn_samples || !host_out)) return fail(HM_ERR_INVALID_ARG, "null samples");
    const size_t n = p->n_total;
    hm_matrices *M = nullptr;
    hm_megno *g = nullptr;
    HM_TRY(hm_matrices_create(n, &M));
    hm_status st = hm_megno_create(n, &g);
    if (st == HM_OK) {
        std::vector<double> snap(n_samples * n, std::nan(""));
        hm_indicator_set s{};
        s.matrix = M;
        s.megno = g;
        s.megno_sample_turns = turn_samples;
        s.n_megno_samples = n_samples;
        s.megno_samples_out = snap.data();
        s.jacobian_of_turn = 1;
        st = track_indicators(t, p, n_turns, mu, barrier, &s, kick_module, inverse != 0);
        if (st == HM_OK)
            for (size_t i = 0; i < n; ++i)
                for (size_t j = 0; j < n_samples; ++j)
                    host_out[i * n_samples + j] = snap[j * n + i];
    }
    hm_megno_destroy(g);
    hm_matrices_destroy(M);
    return st;
}

hm_status hm_storage_device_ptr(const hm_storage *h, hm_field field, const double **out) {
    if (!h || !out) return fail(HM_ERR_INVALID_ARG, "null pointer");
    const DeviceBuffer *b[4] = {&h->x, &h->px, &h->y, &h->py};
    if (field < HM_FIELD_X || field > HM_FIELD_PY) return fail(HM_ERR_INVALID_ARG, "field must be x, px, y or py");
    *out = b[field]->as<const double>();
    return ok();
}

}  // extern "C"
