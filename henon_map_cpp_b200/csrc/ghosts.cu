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
