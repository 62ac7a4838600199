// Ghost-particle kernels: shadow particles displaced from their base
// particle, used for displacement-based Lyapunov estimates
// (src/henon.cu:1257-1442; usage tests/test_new_standard.ipynb:477-479).
#include <cuda_runtime.h>

#include <cstdint>

#include "hm_device.cuh"
#include "hm_internal.h"

namespace hm {
namespace {

using dev::Rn;

// |a - b| with the differences squared and summed left to right
// (displacement, src/henon.cu:407-410).
__device__ __forceinline__ double displacement(double x1, double px1, double y1, double py1,
                                               double x2, double px2, double y2, double py2) {
    const double dx = Rn::sub(x1, x2), dpx = Rn::sub(px1, px2);
    const double dy = Rn::sub(y1, y2), dpy = Rn::sub(py1, py2);
    return sqrt(Rn::add(Rn::add(Rn::add(Rn::mul(dx, dx), Rn::mul(dpx, dpx)), Rn::mul(dy, dy)),
                        Rn::mul(dpy, dpy)));
}

// c + (v - c) * (final / initial) (realign, src/henon.cu:412-418).
__device__ __forceinline__ double realign(double v, double c, double ratio) {
    return Rn::add(c, Rn::mul(Rn::sub(v, c), ratio));
}

__global__ void renormalize_kernel(double *x, double *px, double *y, double *py,
                                   const uint64_t *idx_base, const uint8_t *ghost, size_t n,
                                   double module) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n || !ghost[i]) return;
    const size_t b = idx_base[i];
    const double bx = x[b], bpx = px[b], by = y[b], bpy = py[b];
    const double init = displacement(x[i], px[i], y[i], py[i], bx, bpx, by, bpy);
    const double ratio = Rn::div(module, init);
    x[i] = realign(x[i], bx, ratio);
    px[i] = realign(px[i], bpx, ratio);
    y[i] = realign(y[i], by, ratio);
    py[i] = realign(py[i], bpy, ratio);
}

// Module (dir == nullptr) or unit direction of every ghost relative to its
// base particle, written to [ghost index][base index] slots.
__global__ void displacement_kernel(const double *x, const double *px, const double *y,
                                    const double *py, const uint64_t *idx,
                                    const uint64_t *idx_base, const uint8_t *ghost, size_t n,
                                    size_t n_base, double *module, double *dx, double *dpx,
                                    double *dy, double *dpy) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n || !ghost[i]) return;
    const size_t b = idx_base[i];
    const size_t o = b + n_base * idx[i];
    const double gx = x[i], gpx = px[i], gy = y[i], gpy = py[i];
    const double bx = x[b], bpx = px[b], by = y[b], bpy = py[b];
    const bool lost = dev::is_lost(gx, gpx, gy, gpy) || dev::is_lost(bx, bpx, by, bpy);
    if (module) {
        module[o] = lost ? dev::quiet_nan() : displacement(gx, gpx, gy, gpy, bx, bpx, by, bpy);
        return;
    }
    if (lost) {
        dx[o] = dpx[o] = dy[o] = dpy[o] = dev::quiet_nan();
        return;
    }
    const double ratio = Rn::div(1.0, displacement(gx, gpx, gy, gpy, bx, bpx, by, bpy));
    dx[o] = Rn::sub(realign(gx, bx, ratio), bx);
    dpx[o] = Rn::sub(realign(gpx, bpx, ratio), bpx);
    dy[o] = Rn::sub(realign(gy, by, ratio), by);
    dpy[o] = Rn::sub(realign(gpy, bpy, ratio), bpy);
}

// ---- the ghost Lyapunov loop, fused ---------------------------------------------
// The displacement Lyapunov estimate of tests/test_new_standard.ipynb:477-479
// is a host loop of steps, each
//     tracker.track(p, every, mu)                       (every particle)
//     lyap += log(p.get_displacement_module() / module) (per ghost)
//     p.renormalize(module)                             (ghosts back to module)
// This kernel runs whole steps for one base particle and its G ghosts per
// thread, all in registers: the same turn arithmetic and barrier test as
// the tracker, the same displacement (src/henon.cu:407-410) and realign
// (:412-418) as the per-call kernels above, so coordinates and steps are
// those of the loop bit for bit, and lyap sums log(d / module) per step in
// step order (CUDA's log).  A particle lost to the barrier keeps its steps
// and becomes NaN; a ghost whose base is lost becomes NaN at the next
// renormalisation, as the per-call kernel leaves it (its displacement is
// NaN, and so are the sums of both from then on).
constexpr int kGhostMax = 4;

template <int ARITH, bool OCT, int G>
__global__ void __launch_bounds__(128) ghost_lyapunov_kernel(const GhostLyapunovArgs a) {
    constexpr int K = 1 + G;
    const size_t b = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool in_range = b < a.n_base;
    const size_t bb = in_range ? b : 0;
    dev::Particle p[K];
    bool live[K], entry_live[K];
    uint32_t steps[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const size_t i = bb + a.n_base * size_t(j);
        double x = a.x[i], px = a.px[i], y = a.y[i], py = a.py[i];
        entry_live[j] = in_range && !dev::is_lost(x, px, y, py);
        live[j] = entry_live[j];
        steps[j] = a.steps[i];
        // Slots without a live particle hold zeros, a fixed point of the map.
        if (!live[j]) x = px = y = py = 0.0;
        p[j] = dev::make_particle(x, px, y, py);
    }
    double lyap[G];
#pragma unroll
    for (int g = 0; g < G; ++g) lyap[g] = in_range ? a.lyap[size_t(g) * a.n_base + bb] : 0.0;
    const dev::Barrier bar = dev::make_barrier<ARITH>(a.b2bits);
    const double mu = a.mu, module = a.module;
    uint32_t turn = a.turn0;
    const uint32_t end = a.turn0 + a.n_steps * a.every;
    // The next turn's record is loaded a turn ahead, off the orbits' chains.
    dev::Turn t_next = a.n_steps ? dev::load_turn(a.table, turn) : dev::Turn{};
    for (uint32_t st = 0; st < a.n_steps; ++st) {
        for (uint32_t k = 0; k < a.every; ++k, ++turn) {
            const dev::Turn t = t_next;
            if (turn + 1 < end) t_next = dev::load_turn(a.table, turn + 1);
            uint32_t ored = 0u;
#pragma unroll
            for (int j = 0; j < K; ++j) {
                dev::turn<ARITH, OCT, false>(p[j], t, mu);
                ored |= dev::hi_or(p[j]);
            }
            if (!dev::small_or(ored, bar)) {
#pragma unroll
                for (int j = 0; j < K; ++j)
                    if (live[j] && !dev::inside_after_turn<ARITH>(p[j], bar)) {
                        live[j] = false;
                        steps[j] = turn;  // turns survived: frozen
                        p[j] = dev::make_particle(0.0, 0.0, 0.0, 0.0);
                    }
            }
        }
        // End of a step: displacement, lyap, renormalisation of each ghost.
#pragma unroll
        for (int g = 0; g < G; ++g) {
            dev::Particle &q = p[1 + g];
            const dev::Particle &c = p[0];
            if (!live[1 + g] || !live[0]) {
                // the per-call displacement is NaN; a live ghost of a lost
                // base is realigned on NaN and becomes NaN
                lyap[g] = Rn::add(lyap[g], dev::quiet_nan());
                if (live[1 + g]) {
                    live[1 + g] = false;
                    steps[1 + g] = turn;
                    q = dev::make_particle(0.0, 0.0, 0.0, 0.0);
                }
                continue;
            }
            const double d = displacement(q.x, q.px, q.y, q.py, c.x, c.px, c.y, c.py);
            lyap[g] = Rn::add(lyap[g], log(Rn::div(d, module)));
            const double ratio = Rn::div(module, d);
            const double x = realign(q.x, c.x, ratio), px = realign(q.px, c.px, ratio);
            const double y = realign(q.y, c.y, ratio), py = realign(q.py, c.py, ratio);
            if (dev::is_lost(x, px, y, py)) {  // d = 0 or overflow: NaN, as the loop
                live[1 + g] = false;
                steps[1 + g] = turn;
                q = dev::make_particle(0.0, 0.0, 0.0, 0.0);
            } else {
                q = dev::make_particle(x, px, y, py);
            }
        }
    }
    if (!in_range) return;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        if (!entry_live[j]) continue;  // NaN before this call: untouched
        const size_t i = b + a.n_base * size_t(j);
        if (live[j]) {
            a.x[i] = p[j].x;
            a.px[i] = p[j].px;
            a.y[i] = p[j].y;
            a.py[i] = p[j].py;
            a.steps[i] = turn;
        } else {
            a.x[i] = a.px[i] = a.y[i] = a.py[i] = dev::quiet_nan();
            a.steps[i] = steps[j];
        }
    }
#pragma unroll
    for (int g = 0; g < G; ++g) a.lyap[size_t(g) * a.n_base + b] = lyap[g];
}

template <int ARITH, bool OCT>
cudaError_t launch_ghosts_g(const GhostLyapunovArgs &a, cudaStream_t s) {
    const unsigned blocks = unsigned((a.n_base + 127) / 128);
    switch (a.n_ghosts) {
        case 1: ghost_lyapunov_kernel<ARITH, OCT, 1><<<blocks, 128, 0, s>>>(a); break;
        case 2: ghost_lyapunov_kernel<ARITH, OCT, 2><<<blocks, 128, 0, s>>>(a); break;
        case 3: ghost_lyapunov_kernel<ARITH, OCT, 3><<<blocks, 128, 0, s>>>(a); break;
        case 4: ghost_lyapunov_kernel<ARITH, OCT, 4><<<blocks, 128, 0, s>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// idx = idx_base = i: the indices of a set without ghosts (particles_4d
// constructor, src/henon.cu:713-719).
__global__ void particle_indices_kernel(uint64_t *idx, uint64_t *idx_base, size_t n) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) {
        idx[i] = i;
        idx_base[i] = i;
    }
}

}  // namespace

cudaError_t launch_particle_indices(uint64_t *idx, uint64_t *idx_base, size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    particle_indices_kernel<<<unsigned((n + 255) / 256), 256, 0, s>>>(idx, idx_base, n);
    return cudaGetLastError();
}

int ghost_lyapunov_max_ghosts() { return kGhostMax; }

cudaError_t launch_ghost_lyapunov(const GhostLyapunovArgs &a, int arith, cudaStream_t s) {
    if (a.n_base == 0 || a.n_steps == 0) return cudaSuccess;
    if (a.n_ghosts < 1 || a.n_ghosts > kGhostMax) return cudaErrorInvalidValue;
    const bool oct = a.mu != 0.0;
    if (arith == HM_ARITH_FAST)
        return oct ? launch_ghosts_g<HM_ARITH_FAST, true>(a, s)
                   : launch_ghosts_g<HM_ARITH_FAST, false>(a, s);
    return oct ? launch_ghosts_g<HM_ARITH_EXACT, true>(a, s)
               : launch_ghosts_g<HM_ARITH_EXACT, false>(a, s);
}

cudaError_t launch_renormalize(double *x, double *px, double *y, double *py,
                               const uint64_t *idx_base, const uint8_t *ghost, size_t n,
                               double module, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    renormalize_kernel<<<unsigned((n + 255) / 256), 256, 0, s>>>(x, px, y, py, idx_base, ghost, n,
                                                                 module);
    return cudaGetLastError();
}

cudaError_t launch_displacement(const double *x, const double *px, const double *y,
                                const double *py, const uint64_t *idx, const uint64_t *idx_base,
                                const uint8_t *ghost, size_t n, size_t n_base, double *module,
                                double *dx, double *dpx, double *dy, double *dpy, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    displacement_kernel<<<unsigned((n + 255) / 256), 256, 0, s>>>(
        x, px, y, py, idx, idx_base, ghost, n, n_base, module, dx, dpx, dy, dpy);
    return cudaGetLastError();
}

}  // namespace hm
