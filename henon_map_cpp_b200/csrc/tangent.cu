// Tangent-map and indicator kernels with the reference's per-call semantics.
//
// These are the elementwise operations behind the drop-in classes
// matrix_4d_vector_gpu, vector_4d_gpu and the indicator "constructs"
// (src/henon.cu:267-359, 2042-2655).  Every arithmetic step is separately
// rounded in the reference's order, and the transcendental functions are
// CUDA's own log/log10/atan2/sqrt, so results are bit-identical to the
// reference CUDA build with --fmad=false.  The fused multi-turn kernel that
// replaces the per-turn Python loop over these calls lives in fused.cu.
#include <cuda_runtime.h>

#include <cstdint>

#include "hm_device.cuh"
#include "hm_internal.h"

namespace hm {
namespace {

using dev::Rn;

constexpr int kThreads = 256;

unsigned blocks_for(size_t n) { return unsigned((n + kThreads - 1) / kThreads); }

// M <- DF(x; table[idx]) * M, or M <- DF when set (get_matrices_and_multiply
// / get_matrices_and_set, src/henon.cu:267-313).
__global__ void matrices_step_kernel(double *M, const double *x, const double *px,
                                     const double *y, const double *py, const double *table,
                                     uint32_t idx, double mu, size_t n, int set) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const dev::Turn t = dev::load_turn(table, idx);
    double df[16];
    dev::tangent_matrix_exact(x[i], y[i], t, mu, df);
    double *m = M + i * 16;
    if (set) {
#pragma unroll
        for (int k = 0; k < 16; ++k) m[k] = df[k];
        return;
    }
    double cur[16], out[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) cur[k] = m[k];
    dev::matmul4_exact(df, cur, out);
#pragma unroll
    for (int k = 0; k < 16; ++k) m[k] = out[k];
    (void)px;
    (void)py;
}

__global__ void matrices_identity_kernel(double *M, size_t n) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n * 16) return;
    const int k = int(i % 16);
    M[i] = (k == 0 || k == 5 || k == 10 || k == 15) ? 1.0 : 0.0;
}

// out[i] = M[i] * rv[i] with each row summed left to right
// (matrix_4d_vector_gpu::get_vector, src/henon.cu:1892-1905).
__global__ void matrices_apply_kernel(const double *M, const double *rv, double *out, size_t n) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double *m = M + i * 16;
    const double *v = rv + i * 4;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        double s = Rn::mul(m[r * 4 + 0], v[0]);
        s = Rn::add(s, Rn::mul(m[r * 4 + 1], v[1]));
        s = Rn::add(s, Rn::mul(m[r * 4 + 2], v[2]));
        s = Rn::add(s, Rn::mul(m[r * 4 + 3], v[3]));
        out[i * 4 + r] = s;
    }
}

// v <- M v, rows summed from 0.0 (matrix_vector_multiply, :316-338).
__global__ void vectors_multiply_kernel(const double *M, double *V, size_t n) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double *m = M + i * 16;
    double v[4], t[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = V[i * 4 + k];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        double s = 0.0;
#pragma unroll
        for (int c = 0; c < 4; ++c) s = Rn::add(s, Rn::mul(m[r * 4 + c], v[c]));
        t[r] = s;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) V[i * 4 + k] = t[k];
}

// v <- v / |v| (normalize_vectors, :341-359).
__global__ void vectors_normalize_kernel(double *V, size_t n) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double *v = V + i * 4;
    const double norm = dev::norm_exact<4>(v);
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = Rn::div(v[k], norm);
}

// For every window w with idx < n_w: raw_w += log|v| / n_w and
// b_w += log|v| * weights_w[idx] (kernel_lyap_birk, :2083-2098; windows as
// lyapunov_birkhoff_construct_multi::add, :2171-2183).
__global__ void lyapunov_kernel(double *raw, double *bsum, const double *V, const double *weights,
                                const uint64_t *w_off, const uint64_t *w_len, int n_windows,
                                size_t idx, size_t n) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double l = log(dev::norm_exact<4>(V + i * 4));
    for (int w = 0; w < n_windows; ++w) {
        const uint64_t len = w_len[w];
        if (idx >= len) continue;
        raw[size_t(w) * n + i] = Rn::add(raw[size_t(w) * n + i], Rn::div(l, double(len)));
        bsum[size_t(w) * n + i] =
            Rn::add(bsum[size_t(w) * n + i], Rn::mul(l, weights[w_off[w] + idx]));
    }
}

// MEGNO layers from the Frobenius norms of A (new) and B (old)
// (kernel_megno, :2253-2284).
__global__ void megno_kernel(double *l1, double *l2, double *l3, const double *A, const double *B,
                             size_t idx, size_t n) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double ta = dev::norm_exact<16>(A + i * 16);
    const double tb = dev::norm_exact<16>(B + i * 16);
    const double di = double(idx);
    const double a1 = Rn::add(l1[i], Rn::mul(log10(Rn::div(ta, tb)), di));
    const double a2 = Rn::add(l2[i], Rn::mul(Rn::div(1.0, di), a1));
    l1[i] = a1;
    l2[i] = a2;
    l3[i] = Rn::mul(Rn::div(1.0, di), a2);
}

// Birkhoff-weighted MEGNO per window (kernel_megno_birkhoff, :2366-2402).
__global__ void megno_birkhoff_kernel(double *l1, double *l2, const double *weights,
                                      const uint64_t *w_off, const uint64_t *T, int n_windows,
                                      const double *A, const double *B, size_t idx, size_t n) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double ta = dev::norm_exact<16>(A + i * 16);
    const double tb = dev::norm_exact<16>(B + i * 16);
    const double di = double(idx);
    const double a1 = Rn::add(l1[i], Rn::mul(log10(Rn::div(ta, tb)), di));
    l1[i] = a1;
    for (int w = 0; w < n_windows; ++w) {
        if (idx <= T[w]) {
            double &acc = l2[size_t(w) * n + i];
            acc = Rn::add(acc, Rn::div(Rn::mul(a1, weights[w_off[w] + idx - 1]), di));
        }
    }
}

// First angles (kernel_tune_birkhoff_init, :2533-2546).
__global__ void tune_init_kernel(const double *x, const double *px, const double *y,
                                 const double *py, double *store_x, double *store_y, size_t n) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    store_x[i] = atan2(px[i], x[i]);
    store_y[i] = atan2(py[i], y[i]);
}

// Phase advance wrapped to (0, 2pi], weighted into window 1 [0, T) or
// window 2 [T, 2T) (kernel_tune_birkhoff, :2548-2584).
__global__ void tune_add_kernel(const double *x, const double *px, const double *y,
                                const double *py, double *store_x, double *store_y, double *t1x,
                                double *t1y, double *t2x, double *t2y, const double *weights,
                                const uint64_t *w_off, const uint64_t *T, int n_windows,
                                size_t idx, size_t n) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double ax = atan2(px[i], x[i]);
    const double ay = atan2(py[i], y[i]);
    double dx = Rn::sub(ax, store_x[i]);
    double dy = Rn::sub(ay, store_y[i]);
    const double two_pi = 2 * M_PI;
    dx = dx > 0 ? dx : Rn::add(dx, two_pi);
    dy = dy > 0 ? dy : Rn::add(dy, two_pi);
    store_x[i] = ax;
    store_y[i] = ay;
    for (int w = 0; w < n_windows; ++w) {
        const uint64_t len = T[w];
        const size_t o = size_t(w) * n + i;
        if (idx < len) {
            const double wt = weights[w_off[w] + idx];
            t1x[o] = Rn::add(t1x[o], Rn::mul(dx, wt));
            t1y[o] = Rn::add(t1y[o], Rn::mul(dy, wt));
        } else if (idx < 2 * len) {
            const double wt = weights[w_off[w] + idx - len];
            t2x[o] = Rn::add(t2x[o], Rn::mul(dx, wt));
            t2y[o] = Rn::add(t2y[o], Rn::mul(dy, wt));
        }
    }
}

}  // namespace

cudaError_t launch_matrices_step(double *M, const double *x, const double *px, const double *y,
                                 const double *py, const double *table, uint32_t idx, double mu,
                                 size_t n, bool set, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    matrices_step_kernel<<<blocks_for(n), kThreads, 0, s>>>(M, x, px, y, py, table, idx, mu, n,
                                                            set ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_matrices_identity(double *M, size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    matrices_identity_kernel<<<blocks_for(n * 16), kThreads, 0, s>>>(M, n);
    return cudaGetLastError();
}

cudaError_t launch_matrices_apply(const double *M, const double *rv, double *out, size_t n,
                                  cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    matrices_apply_kernel<<<blocks_for(n), kThreads, 0, s>>>(M, rv, out, n);
    return cudaGetLastError();
}

cudaError_t launch_vectors_multiply(const double *M, double *V, size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    vectors_multiply_kernel<<<blocks_for(n), kThreads, 0, s>>>(M, V, n);
    return cudaGetLastError();
}

cudaError_t launch_vectors_normalize(double *V, size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    vectors_normalize_kernel<<<blocks_for(n), kThreads, 0, s>>>(V, n);
    return cudaGetLastError();
}

cudaError_t launch_lyapunov(double *raw, double *bsum, const double *V, const double *weights,
                            const uint64_t *w_off, const uint64_t *w_len, int n_windows,
                            size_t idx, size_t n, cudaStream_t s) {
    if (n == 0 || n_windows == 0) return cudaSuccess;
    lyapunov_kernel<<<blocks_for(n), kThreads, 0, s>>>(raw, bsum, V, weights, w_off, w_len,
                                                       n_windows, idx, n);
    return cudaGetLastError();
}

cudaError_t launch_megno(double *l1, double *l2, double *l3, const double *A, const double *B,
                         size_t idx, size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    megno_kernel<<<blocks_for(n), kThreads, 0, s>>>(l1, l2, l3, A, B, idx, n);
    return cudaGetLastError();
}

cudaError_t launch_megno_birkhoff(double *l1, double *l2, const double *weights,
                                  const uint64_t *w_off, const uint64_t *T, int n_windows,
                                  const double *A, const double *B, size_t idx, size_t n,
                                  cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    megno_birkhoff_kernel<<<blocks_for(n), kThreads, 0, s>>>(l1, l2, weights, w_off, T, n_windows,
                                                             A, B, idx, n);
    return cudaGetLastError();
}

cudaError_t launch_tune_init(const double *x, const double *px, const double *y, const double *py,
                             double *store_x, double *store_y, size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    tune_init_kernel<<<blocks_for(n), kThreads, 0, s>>>(x, px, y, py, store_x, store_y, n);
    return cudaGetLastError();
}

cudaError_t launch_tune_add(const double *x, const double *px, const double *y, const double *py,
                            double *store_x, double *store_y, double *t1x, double *t1y,
                            double *t2x, double *t2y, const double *weights,
                            const uint64_t *w_off, const uint64_t *T, int n_windows, size_t idx,
                            size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    tune_add_kernel<<<blocks_for(n), kThreads, 0, s>>>(x, px, y, py, store_x, store_y, t1x, t1y,
                                                       t2x, t2y, weights, w_off, T, n_windows,
                                                       idx, n);
    return cudaGetLastError();
}

}  // namespace hm
