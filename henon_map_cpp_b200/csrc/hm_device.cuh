// Device helpers shared by the kernels of libhenon_b200.so.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace hm {
namespace dev {

constexpr unsigned kFullMask = 0xffffffffu;

__device__ __forceinline__ double quiet_nan() {
    return __longlong_as_double(0x7ff8000000000000LL);  // glibc NAN
}

// Separately rounded binary64 operations: the __d*_rn intrinsics are never
// contracted into fused multiply-adds, so a sequence of them reproduces the
// host's SSE2 arithmetic (and nvcc --fmad=false device code) bit for bit.
struct Rn {
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
};

// One turn record {sin wx, cos wx, sin wy, cos wy}.
struct Turn {
    double sx, cx, sy, cy;
};

__device__ __forceinline__ Turn load_turn(const double *table, uint32_t i) {
    const double2 *p = reinterpret_cast<const double2 *>(table) + 2 * size_t(i);
    const double2 a = __ldg(p);
    const double2 b = __ldg(p + 1);
    return Turn{a.x, a.y, b.x, b.y};
}

__device__ __forceinline__ bool is_lost(double x, double px, double y, double py) {
    return isnan(x) || isnan(px) || isnan(y) || isnan(py);
}

// Jacobian of one turn, row-major, in the reference's expression order
// (tangent_matrix, src/henon.cu:175-196): every entry is evaluated from the
// same sub-expressions, so sharing them is exact.
__device__ __forceinline__ void tangent_matrix_exact(double x, double y, const Turn &t, double mu,
                                                     double m[16]) {
    using R = Rn;
    const double mu3 = R::mul(mu, 3.0);
    const double mu6 = R::mul(mu, 6.0);
    const double mu3xx = R::mul(R::mul(mu3, x), x);
    const double mu3yy = R::mul(R::mul(mu3, y), y);
    // 2*x + mu*3*x*x - mu*3*y*y
    const double a = R::sub(R::add(R::mul(2.0, x), mu3xx), mu3yy);
    // -2*y - mu*6*x*y
    const double b = R::sub(R::mul(-2.0, y), R::mul(R::mul(mu6, x), y));
    // -2*x - mu*3*x*x + mu*3*y*y
    const double d = R::add(R::sub(R::mul(-2.0, x), mu3xx), mu3yy);
    m[0] = R::add(t.cx, R::mul(t.sx, a));
    m[1] = t.sx;
    m[2] = R::mul(t.sx, b);
    m[3] = 0.0;
    m[4] = R::add(-t.sx, R::mul(t.cx, a));
    m[5] = t.cx;
    m[6] = R::mul(t.cx, b);
    m[7] = 0.0;
    m[8] = R::mul(t.sy, b);
    m[9] = 0.0;
    m[10] = R::add(t.cy, R::mul(t.sy, d));
    m[11] = t.sy;
    m[12] = R::mul(t.cy, b);
    m[13] = 0.0;
    m[14] = R::add(-t.sy, R::mul(t.cy, d));
    m[15] = t.cy;
}

// out = a * b for row-major 4x4, every sum started from 0.0 and accumulated
// in k order (get_matrices_and_multiply, src/henon.cu:279-288).
__device__ __forceinline__ void matmul4_exact(const double a[16], const double b[16],
                                              double out[16]) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < 4; ++k) s = Rn::add(s, Rn::mul(a[i * 4 + k], b[k * 4 + j]));
            out[i * 4 + j] = s;
        }
    }
}

// sqrt of the sum of squares from 0.0 in index order (the Frobenius norm of
// kernel_megno, src/henon.cu:2258-2277; the vector norm of kernel_lyap_birk
// and normalize_vectors, :2089-2094, :349-354).
template <int N>
__device__ __forceinline__ double norm_exact(const double *v) {
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < N; ++i) s = Rn::add(s, Rn::mul(v[i], v[i]));
    return sqrt(s);
}

}  // namespace dev
}  // namespace hm
