// C ABI of the orbit-loss adjoint (hm_adjoint*): host set-up of the ripple
// and weight tables and of the checkpoint buffers.
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "hm_internal.h"

using hm::DeviceBuffer;
using hm::fail;
using hm::ok;

namespace {

size_t ckpt_count(uint32_t n_turns, uint32_t every) { return (size_t(n_turns) + every - 1) / every; }

}  // namespace

extern "C" {

size_t hm_adjoint_workspace_bytes(size_t n, uint32_t n_turns, uint32_t checkpoint_every) {
    if (checkpoint_every == 0) return 0;
    return hm::align256((ckpt_count(n_turns, checkpoint_every) + checkpoint_every) * 4 * n *
                        sizeof(double));
}

hm_status hm_set_adjoint_config(int per_thread) {
    if (per_thread != 1 && per_thread != 2)
        return fail(HM_ERR_INVALID_ARG, "particles per thread must be 1 or 2");
    hm::set_adjoint_per_thread(per_thread);
    return ok();
}

hm_status hm_get_adjoint_config(int *per_thread) {
    if (!per_thread) return fail(HM_ERR_INVALID_ARG, "null output");
    *per_thread = hm::get_adjoint_per_thread();
    return ok();
}

hm_status hm_adjoint(const hm_tracker *t, const double *x0, const double *px0, const double *y0,
                     const double *py0, size_t n, double mu, double barrier, uint32_t n_turns,
                     uint32_t checkpoint_every, int mode, double *loss, uint8_t *survived,
                     uint32_t *steps, double *grad_ic, double *grad_theta, void *workspace,
                     void *stream) {
    if (!t) return fail(HM_ERR_INVALID_ARG, "null tracker");
    if (mode < 0 || mode > 3) return fail(HM_ERR_INVALID_ARG, "mode must be 0, 1, 2 or 3");
    if (n_turns > t->allowed_steps) return fail(HM_ERR_BUDGET, "The number of turns is too large.");
    if (n == 0) return ok();
    if (!x0 || !px0 || !y0 || !py0 || !loss || !survived || !steps)
        return fail(HM_ERR_INVALID_ARG, "null device array");
    const bool reverse = mode == 0 || mode == 3;
    if (reverse && (checkpoint_every == 0 || !workspace || !grad_ic || !grad_theta))
        return fail(HM_ERR_INVALID_ARG, "the adjoint needs checkpoint_every > 0, a workspace and "
                                        "gradient outputs");
    if (mode == 1 && !grad_ic) return fail(HM_ERR_INVALID_ARG, "null gradient output");
    std::lock_guard<std::mutex> lock(t->adjoint_mutex);
    if (!t->adjoint_cached || t->adjoint_turns != n_turns) {
        HM_TRY(hm::upload(t->adjoint_w, hm::birkhoff_weights(n_turns)));
        t->adjoint_S.release();
        t->adjoint_turns = n_turns;
        t->adjoint_cached = true;
        t->adjoint_has_ripple = false;
    }
    const bool need_ripple = reverse || (mode == 1 && grad_theta != nullptr);
    if (need_ripple && !t->adjoint_has_ripple) {
        // Only the theta gradients need d omega / d theta (and an "sps" or
        // "basic" modulation).
        std::vector<double> ripple;
        HM_TRY(hm::modulation_ripple(t->kind, n_turns, t->omega_0, t->offset, ripple));
        HM_TRY(hm::upload(t->adjoint_S, ripple));
        t->adjoint_has_ripple = true;
    }
    hm::AdjointArgs a{};
    a.x0 = x0;
    a.px0 = px0;
    a.y0 = y0;
    a.py0 = py0;
    a.n = n;
    a.table = t->table.as<double>();
    a.S = t->adjoint_S.as<double>();
    a.w = t->adjoint_w.as<double>();
    a.n_turns = n_turns;
    a.ckpt = checkpoint_every ? checkpoint_every : 1;
    a.mu = mu;
    a.epsilon = t->epsilon;
    a.omega_x0 = 2 * M_PI * t->omega_x;
    a.omega_y0 = 2 * M_PI * t->omega_y;
    const double b2 = barrier * barrier;
    a.b2bits = 0;
    if (!std::isnan(b2)) std::memcpy(&a.b2bits, &b2, sizeof(b2));
    a.arith = t->arith;
    if (reverse) {
        a.ckpt_buf = static_cast<double *>(workspace);
        a.seg_buf = a.ckpt_buf + ckpt_count(n_turns, checkpoint_every) * 4 * n;
    }
    a.loss = loss;
    a.survived = survived;
    a.steps = steps;
    a.g_ic = grad_ic;
    a.g_th = mode == 2 ? nullptr : grad_theta;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    HM_CUDA_TRY(hm::launch_adjoint(a, mode, s));
    HM_CUDA_TRY(cudaStreamSynchronize(s));
    return ok();
}

}  // extern "C"
