// Ghost particles and host-side tangent matrices of the particle API
// (particles_4d[_gpu]::add_ghost / renormalize / get_displacement_*,
// henon_tracker_gpu::get_tangent_matrix).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "hm_internal.h"

using hm::DeviceBuffer;
using hm::fail;
using hm::ok;

namespace {

// Isotropic 4D displacement of modulus `module` from four standard normal
// draws of a fresh distribution (random_4d_kick, host form,
// src/henon.cu:362-385).
void random_kick(double &x, double &px, double &y, double &py, double module,
                 std::mt19937_64 &gen) {
    std::normal_distribution<double> normal(0.0, 1.0);
    double k[4];
    for (double &v : k) v = normal(gen);
    const double mod = std::sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2] + k[3] * k[3]);
    x += k[0] * module / mod;
    px += k[1] * module / mod;
    y += k[2] * module / mod;
    py += k[3] * module / mod;
}

// tangent_matrix, host form (src/henon.cu:198-222), row-major.
void tangent_host(double x, double y, double sx, double cx, double sy, double cy, double mu,
                  double *m) {
    m[0] = cx + sx * (2 * x + mu * 3 * x * x - mu * 3 * y * y);
    m[1] = sx;
    m[2] = sx * (-2 * y - mu * 6 * x * y);
    m[3] = 0.0;
    m[4] = -sx + cx * (2 * x + mu * 3 * x * x - mu * 3 * y * y);
    m[5] = cx;
    m[6] = cx * (-2 * y - mu * 6 * x * y);
    m[7] = 0.0;
    m[8] = sy * (-2 * y - mu * 6 * x * y);
    m[9] = 0.0;
    m[10] = cy + sy * (-2 * x - mu * 3 * x * x + mu * 3 * y * y);
    m[11] = sy;
    m[12] = cy * (-2 * y - mu * 6 * x * y);
    m[13] = 0.0;
    m[14] = -sy + cy * (-2 * x - mu * 3 * x * x + mu * 3 * y * y);
    m[15] = cy;
}

// inverse_tangent_matrix (src/henon.cu:224-249), row-major.
void inverse_tangent_host(double x, double px, double y, double py, double sx, double cx,
                          double sy, double cy, double mu, double *m) {
    const double u = cx * x - px * sx;  // x after the inverse rotation
    const double w = cy * y - py * sy;
    m[0] = cx;
    m[1] = -sx;
    m[2] = 0;
    m[3] = 0;
    m[4] = -3 * cx * mu * (std::pow(u, 2) - std::pow(w, 2)) - 2 * cx * u + sx;
    m[5] = cx + 3 * mu * sx * (std::pow(u, 2) - std::pow(w, 2)) + 2 * sx * u;
    m[6] = 2 * cy * w * (3 * mu * u + 1);
    m[7] = 2 * sy * w * (-3 * mu * u - 1);
    m[8] = 0;
    m[9] = 0;
    m[10] = cy;
    m[11] = -sy;
    m[12] = 2 * cx * w * (3 * mu * u + 1);
    m[13] = 2 * sx * w * (-3 * mu * u - 1);
    m[14] = 3 * cy * mu * (std::pow(u, 2) - std::pow(w, 2)) + 2 * cy * u + sy;
    m[15] = cy - 3 * mu * sy * (std::pow(u, 2) - std::pow(w, 2)) - 2 * sy * u;
}

}  // namespace

extern "C" {

// particles_4d::add_ghost (src/henon.cu:737-818) as used by
// particles_4d_gpu::add_ghost (:1247-1255): ghosts are built from the
// host-side coordinates (the initial conditions) and the whole set is
// uploaded again, so the device state restarts from the initial conditions
// with steps = 0, as in the reference.
hm_status hm_particles_add_ghost(hm_particles *p, double module, const char *direction) {
    if (!p || !direction) return fail(HM_ERR_INVALID_ARG, "null particles or direction");
    const std::string dir(direction);
    if (dir != "x" && dir != "px" && dir != "y" && dir != "py" && dir != "random")
        return fail(HM_ERR_INVALID_ARG, "Invalid direction.");
    HM_TRY(hm::particles_host_mirror(p));
    const size_t n = p->n_total;
    std::vector<double> gx, gpx, gy, gpy;
    std::vector<uint8_t> gvalid;
    std::vector<uint64_t> gidx, gbase;
    for (size_t i = 0; i < n; ++i) {
        if (p->ghost[i]) continue;
        double x = p->x0[i], px = p->px0[i], y = p->y0[i], py = p->py0[i];
        if (dir == "x") x = x + module;
        else if (dir == "y") y = y + module;
        else if (dir == "px") px = px + module;
        else if (dir == "py") py = py + module;
        else random_kick(x, px, y, py, module, p->rng);
        gx.push_back(x);
        gpx.push_back(px);
        gy.push_back(y);
        gpy.push_back(py);
        gvalid.push_back(p->valid[i]);
        gidx.push_back(p->n_ghosts);
        gbase.push_back(i);
    }
    p->x0.insert(p->x0.end(), gx.begin(), gx.end());
    p->px0.insert(p->px0.end(), gpx.begin(), gpx.end());
    p->y0.insert(p->y0.end(), gy.begin(), gy.end());
    p->py0.insert(p->py0.end(), gpy.begin(), gpy.end());
    p->valid.insert(p->valid.end(), gvalid.begin(), gvalid.end());
    p->ghost.insert(p->ghost.end(), gx.size(), uint8_t(1));
    p->idx.insert(p->idx.end(), gidx.begin(), gidx.end());
    p->idx_base.insert(p->idx_base.end(), gbase.begin(), gbase.end());
    p->n_total += gx.size();
    p->n_ghosts += 1;
    p->live_step = 0;
    p->work.release();
    return hm::particles_upload(p, p->x0.data(), p->px0.data(), p->y0.data(), p->py0.data());
}

// renormalize (src/henon.cu:1257-1282): every ghost moved along its
// displacement to distance `module` from its base particle.
hm_status hm_particles_renormalize(hm_particles *p, double module) {
    if (!p) return fail(HM_ERR_INVALID_ARG, "null particles");
    HM_CUDA_TRY(hm::launch_renormalize(p->x.as<double>(), p->px.as<double>(), p->y.as<double>(),
                                       p->py.as<double>(), p->didx_base.as<uint64_t>(),
                                       p->dghost.as<uint8_t>(), p->n_total, module, 0));
    return ok();
}

// get_displacement_module (src/henon.cu:1284-1343): host
// double[n_particles][n_ghosts], NaN when ghost or base is lost.
hm_status hm_particles_displacement_module(const hm_particles *p, double *host_out) {
    if (!p) return fail(HM_ERR_INVALID_ARG, "null particles");
    const size_t nb = p->n_particles, ng = p->n_ghosts;
    if (nb * ng == 0) return ok();
    if (!host_out) return fail(HM_ERR_INVALID_ARG, "null output");
    DeviceBuffer out;
    HM_TRY(out.alloc(nb * ng * sizeof(double)));
    HM_CUDA_TRY(hm::launch_displacement(p->x.as<double>(), p->px.as<double>(), p->y.as<double>(),
                                        p->py.as<double>(), p->didx.as<uint64_t>(),
                                        p->didx_base.as<uint64_t>(), p->dghost.as<uint8_t>(),
                                        p->n_total, nb, out.as<double>(), nullptr, nullptr,
                                        nullptr, nullptr, 0));
    std::vector<double> g(nb * ng);  // [ghost][base]
    HM_CUDA_TRY(cudaMemcpy(g.data(), out.ptr, g.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (size_t b = 0; b < nb; ++b)
        for (size_t k = 0; k < ng; ++k) host_out[b * ng + k] = g[k * nb + b];
    return ok();
}

// The ghost Lyapunov loop of tests/test_new_standard.ipynb:477-479 (track
// `every` turns, accumulate log(displacement / module), renormalize) in
// fused launches (ghosts.cu).  host_out: double[n_particles][n_ghosts],
// the sums over this call's steps.
hm_status hm_track_ghost_lyapunov(hm_tracker *t, hm_particles *p, uint32_t n_steps,
                                  uint32_t every, double mu, double barrier, double module,
                                  double *host_out) {
    if (!t || !p) return fail(HM_ERR_INVALID_ARG, "null tracker or particles");
    const size_t nb = p->n_particles, ng = p->n_ghosts;
    if (ng == 0) return fail(HM_ERR_INVALID_ARG, "the particles have no ghosts (add_ghost first)");
    if (ng > size_t(hm::ghost_lyapunov_max_ghosts()))
        return fail(HM_ERR_NOT_SUPPORTED, "at most " +
                                              std::to_string(hm::ghost_lyapunov_max_ghosts()) +
                                              " ghosts per particle in the fused ghost loop");
    if (every == 0) return fail(HM_ERR_INVALID_ARG, "every must be positive");
    if (p->n_total != nb * (1 + ng)) return fail(HM_ERR_INVALID_ARG, "inconsistent ghost layout");
    const uint64_t turns = uint64_t(n_steps) * every;
    if (turns + p->global_steps > t->allowed_steps || turns > 0xffffffffull)
        return fail(HM_ERR_BUDGET, "The number of turns is too large.");
    if (nb == 0 || n_steps == 0) return ok();
    if (!host_out) return fail(HM_ERR_INVALID_ARG, "null output");
    DeviceBuffer lyap;
    HM_TRY(lyap.alloc(nb * ng * sizeof(double)));
    HM_CUDA_TRY(cudaMemsetAsync(lyap.ptr, 0, nb * ng * sizeof(double), 0));
    hm::GhostLyapunovArgs a{};
    a.x = p->x.as<double>();
    a.px = p->px.as<double>();
    a.y = p->y.as<double>();
    a.py = p->py.as<double>();
    a.steps = p->steps.as<uint32_t>();
    a.n_base = nb;
    a.n_ghosts = int(ng);
    a.table = t->table.as<const double>();
    a.every = every;
    a.mu = mu;
    const double b2 = barrier * barrier;
    a.b2bits = 0;
    if (!std::isnan(b2)) std::memcpy(&a.b2bits, &b2, sizeof(b2));
    a.module = module;
    a.lyap = lyap.as<double>();
    // Launches of whole steps, about 4096 turns each (cancellation is
    // checked between them).
    const uint32_t per_launch = std::max<uint32_t>(1u, 4096u / every);
    uint32_t done = 0;
    hm_status status = HM_OK;
    while (done < n_steps) {
        a.turn0 = p->live_step;
        a.n_steps = std::min(per_launch, n_steps - done);
        HM_CUDA_TRY(hm::launch_ghost_lyapunov(a, t->arith, 0));
        HM_CUDA_TRY(cudaStreamSynchronize(0));
        done += a.n_steps;
        p->global_steps += a.n_steps * every;
        p->live_step += a.n_steps * every;
        if (done < n_steps && hm::cancel_requested()) {
            status = fail(HM_ERR_CANCELLED, "ghost loop cancelled");
            break;
        }
    }
    std::vector<double> g(nb * ng);  // [ghost][base]
    HM_CUDA_TRY(cudaMemcpy(g.data(), lyap.ptr, g.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (size_t b = 0; b < nb; ++b)
        for (size_t k = 0; k < ng; ++k) host_out[b * ng + k] = g[k * nb + b];
    return status == HM_OK ? ok() : status;
}

// get_displacement_direction (src/henon.cu:1345-1442): host
// double[4][n_particles][n_ghosts] (x, px, y, py components).
hm_status hm_particles_displacement_direction(const hm_particles *p, double *host_out) {
    if (!p) return fail(HM_ERR_INVALID_ARG, "null particles");
    const size_t nb = p->n_particles, ng = p->n_ghosts;
    if (nb * ng == 0) return ok();
    if (!host_out) return fail(HM_ERR_INVALID_ARG, "null output");
    DeviceBuffer out;
    HM_TRY(out.alloc(4 * nb * ng * sizeof(double)));
    double *o = out.as<double>();
    HM_CUDA_TRY(hm::launch_displacement(p->x.as<double>(), p->px.as<double>(), p->y.as<double>(),
                                        p->py.as<double>(), p->didx.as<uint64_t>(),
                                        p->didx_base.as<uint64_t>(), p->dghost.as<uint8_t>(),
                                        p->n_total, nb, nullptr, o, o + nb * ng, o + 2 * nb * ng,
                                        o + 3 * nb * ng, 0));
    std::vector<double> g(4 * nb * ng);  // [component][ghost][base]
    HM_CUDA_TRY(cudaMemcpy(g.data(), out.ptr, g.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (size_t c = 0; c < 4; ++c)
        for (size_t b = 0; b < nb; ++b)
            for (size_t k = 0; k < ng; ++k)
                host_out[(c * nb + b) * ng + k] = g[(c * ng + k) * nb + b];
    return ok();
}

// henon_tracker_gpu::get_tangent_matrix (src/henon.cu:3187-3219): on the
// host, from the current coordinates and table[global_steps]; the inverse
// form when reverse; NaN matrices for particles not marked valid.
// Output double[n_total][16].
hm_status hm_tracker_tangent_matrices(const hm_tracker *t, const hm_particles *p, double mu,
                                      int reverse, double *host_out) {
    if (!t || !p) return fail(HM_ERR_INVALID_ARG, "null tracker or particles");
    const size_t n = p->n_total;
    if (n == 0) return ok();
    if (!host_out) return fail(HM_ERR_INVALID_ARG, "null output");
    const uint32_t s = p->global_steps;
    if (s >= t->allowed_steps)
        return fail(HM_ERR_BUDGET, "The number of turns is too large. (tangent matrix past the table end)");
    HM_TRY(hm::particles_host_mirror(p));
    std::vector<double> x(n), px(n), y(n), py(n);
    HM_CUDA_TRY(cudaMemcpy(x.data(), p->x.ptr, n * sizeof(double), cudaMemcpyDeviceToHost));
    HM_CUDA_TRY(cudaMemcpy(px.data(), p->px.ptr, n * sizeof(double), cudaMemcpyDeviceToHost));
    HM_CUDA_TRY(cudaMemcpy(y.data(), p->y.ptr, n * sizeof(double), cudaMemcpyDeviceToHost));
    HM_CUDA_TRY(cudaMemcpy(py.data(), p->py.ptr, n * sizeof(double), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i) {
        double *m = host_out + 16 * i;
        if (!p->valid[i]) {
            for (int k = 0; k < 16; ++k) m[k] = std::nan("");
        } else if (!reverse) {
            tangent_host(x[i], y[i], t->sx[s], t->cx[s], t->sy[s], t->cy[s], mu, m);
        } else {
            inverse_tangent_host(x[i], px[i], y[i], py[i], t->sx[s], t->cx[s], t->sy[s],
                                 t->cy[s], mu, m);
        }
    }
    return ok();
}

}  // extern "C"
