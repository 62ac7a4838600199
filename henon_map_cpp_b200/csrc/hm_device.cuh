// Device helpers shared by the kernels of libhenon_b200.so.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/henon_b200.h"

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

// ---- bulk copies into shared memory ---------------------------------------------
// cp.async.bulk (the untiled TMA copy, no multicast) from this GPU's global
// memory into the CTA's shared memory, completed on an mbarrier by
// transaction count.  Source, destination and size must be multiples of 16
// bytes.
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

// Makes mbarrier initialisation visible to the async proxy (TMA).
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this CTA's earlier shared-memory accesses before later async-proxy
// writes (a bulk copy refilling a buffer that threads have read).
__device__ __forceinline__ void async_proxy_fence() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes,
                                          uint64_t *bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0u;
}

// Waits for the phase with the given parity to complete; gives up (returns
// false) after kWaitPolls polls or about two seconds, whichever comes first,
// so that a copy that never lands cannot hang the GPU.
constexpr uint32_t kWaitPolls = 1u << 24;
constexpr long long kWaitCycles = 4000000000ll;

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    const long long t0 = clock64();
    for (uint32_t i = 0; i < kWaitPolls; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if (clock64() - t0 > kWaitCycles) break;
    }
    return false;
}

// ---- the map ------------------------------------------------------------------
// Particle in registers; xx = x*x and yy = y*y of the current coordinates
// are carried from one turn's barrier test into the next turn's kicks (the
// reference computes the same products twice).
struct Particle {
    double x, px, y, py, xx, yy;
};

__device__ __forceinline__ Particle make_particle(double x, double px, double y, double py) {
    return Particle{x, px, y, py, Rn::mul(x, x), Rn::mul(y, y)};
}

// x^2+px^2+y^2+py^2 grouped as (x*x + px*px) + (y*y + py*py), separately
// rounded: the radius of check_barrier, src/henon.cu:113-116.
__device__ __forceinline__ double radius_exact(const Particle &p) {
    return Rn::add(Rn::add(p.xx, Rn::mul(p.px, p.px)), Rn::add(p.yy, Rn::mul(p.py, p.py)));
}

// The same sum with two fused multiply-adds: three FP64 instructions
// instead of five, within 2 ulp of the exact sum (all terms are >= 0).
__device__ __forceinline__ double radius_fma(const Particle &p) {
    return fma(p.px, p.px, p.xx) + fma(p.py, p.py, p.yy);
}

// Forward turn in the reference order: sextupole, [octupole], rotate x then
// y with table[steps] (henon_step, src/henon.cu:493-508, primitives
// :131-173).
template <bool OCT>
__device__ __forceinline__ void turn_exact_fwd(Particle &p, const Turn &t, double mu) {
    // px += x*x - y*y ; py += (-2*x)*y          (sextupole, :131-143)
    double px = Rn::add(p.px, Rn::sub(p.xx, p.yy));
    double py = Rn::add(p.py, Rn::mul(Rn::mul(-2.0, p.x), p.y));
    if (OCT) {
        // px += mu*((x*x*x) - ((3*y)*y)*x), py likewise   (octupole, :145-157)
        px = Rn::add(px, Rn::mul(mu, Rn::sub(Rn::mul(p.xx, p.x),
                                             Rn::mul(Rn::mul(Rn::mul(3.0, p.y), p.y), p.x))));
        py = Rn::add(py, Rn::mul(mu, Rn::sub(Rn::mul(p.yy, p.y),
                                             Rn::mul(Rn::mul(Rn::mul(3.0, p.x), p.x), p.y))));
    }
    // x' = x*c + px*s ; px' = (-x)*s + px*c       (rotation, :159-173)
    const double x = Rn::add(Rn::mul(p.x, t.cx), Rn::mul(px, t.sx));
    px = Rn::add(Rn::mul(-p.x, t.sx), Rn::mul(px, t.cx));
    const double y = Rn::add(Rn::mul(p.y, t.cy), Rn::mul(py, t.sy));
    py = Rn::add(Rn::mul(-p.y, t.sy), Rn::mul(py, t.cy));
    p = Particle{x, px, y, py, Rn::mul(x, x), Rn::mul(y, y)};
}

// Reverse turn: rotate x then y backwards with table[steps-1], subtract the
// octupole, subtract the sextupole (src/henon.cu:510-528).
template <bool OCT>
__device__ __forceinline__ void turn_exact_rev(Particle &p, const Turn &t, double mu) {
    const double x = Rn::sub(Rn::mul(p.x, t.cx), Rn::mul(p.px, t.sx));
    double px = Rn::add(Rn::mul(p.x, t.sx), Rn::mul(p.px, t.cx));
    const double y = Rn::sub(Rn::mul(p.y, t.cy), Rn::mul(p.py, t.sy));
    double py = Rn::add(Rn::mul(p.y, t.sy), Rn::mul(p.py, t.cy));
    const double xx = Rn::mul(x, x);
    const double yy = Rn::mul(y, y);
    if (OCT) {
        px = Rn::sub(px, Rn::mul(mu, Rn::sub(Rn::mul(xx, x),
                                             Rn::mul(Rn::mul(Rn::mul(3.0, y), y), x))));
        py = Rn::sub(py, Rn::mul(mu, Rn::sub(Rn::mul(yy, y),
                                             Rn::mul(Rn::mul(Rn::mul(3.0, x), x), y))));
    }
    px = Rn::sub(px, Rn::sub(xx, yy));
    py = Rn::sub(py, Rn::mul(Rn::mul(-2.0, x), y));
    p = Particle{x, px, y, py, xx, yy};
}

// The same map with fused multiply-adds and x^3-3xy^2 = x(x^2-3y^2): 14
// (mu = 0) / 20 (mu != 0) FP64 instructions per particle-turn, against
// 19 / 33 for the exact turn (the barrier test adds none in the common case).
template <bool OCT>
__device__ __forceinline__ void turn_fast_fwd(Particle &p, const Turn &t, double mu) {
    double px = p.px + (p.xx - p.yy);
    double py = fma(-2.0 * p.x, p.y, p.py);
    if (OCT) {
        px = fma(mu * p.x, fma(-3.0, p.yy, p.xx), px);
        py = fma(mu * p.y, fma(-3.0, p.xx, p.yy), py);
    }
    const double x = fma(p.x, t.cx, px * t.sx);
    px = fma(px, t.cx, -p.x * t.sx);
    const double y = fma(p.y, t.cy, py * t.sy);
    py = fma(py, t.cy, -p.y * t.sy);
    p = Particle{x, px, y, py, x * x, y * y};
}

template <bool OCT>
__device__ __forceinline__ void turn_fast_rev(Particle &p, const Turn &t, double mu) {
    const double x = fma(p.x, t.cx, -p.px * t.sx);
    double px = fma(p.x, t.sx, p.px * t.cx);
    const double y = fma(p.y, t.cy, -p.py * t.sy);
    double py = fma(p.y, t.sy, p.py * t.cy);
    const double xx = x * x;
    const double yy = y * y;
    if (OCT) {
        px = fma(-mu * x, fma(-3.0, yy, xx), px);
        py = fma(-mu * y, fma(-3.0, xx, yy), py);
    }
    px = px - (xx - yy);
    py = fma(2.0 * x, y, py);
    p = Particle{x, px, y, py, xx, yy};
}

// One turn of the map; the barrier test is separate (inside_after_turn).
template <int ARITH, bool OCT, bool REV>
__device__ __forceinline__ void turn(Particle &p, const Turn &t, double mu) {
    if (ARITH == HM_ARITH_EXACT) {
        if (REV) turn_exact_rev<OCT>(p, t, mu);
        else turn_exact_fwd<OCT>(p, t, mu);
    } else {
        if (REV) turn_fast_rev<OCT>(p, t, mu);
        else turn_fast_fwd<OCT>(p, t, mu);
    }
}

// ---- reproducible random kicks ---------------------------------------------------
// The reference kicks a particle by kick_module along a random direction
// before the sextupole (random_4d_kick, src/henon.cu:387-405, from a
// clock()-seeded curand stream).  Here the direction comes from a
// counter-based generator keyed by (seed, particle index, table index of
// the turn): the same run gives the same kicks however it is split into
// launches, chunks and compacted lists.
//   Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
//   easy as 1, 2, 3", SC'11): counter {turn, attempt, idx_lo, idx_hi}, key
//   {seed_lo, seed_hi}.
//   Direction uniform on the unit 3-sphere by Marsaglia's method (Ann. Math.
//   Statist. 43 (1972) 645-646): (u1, u2), (u3, u4) uniform in the unit
//   disc, s1 = u1^2+u2^2, s2 = u3^2+u4^2, direction (u1, u2, u3 f, u4 f),
//   f = sqrt((1 - s1) / s2).
// One Philox block gives a candidate point for each disc
// (u = (int32(r) + 0.5) * 2^-31, exact); each disc keeps its first
// accepted point.  After kKickAttempts attempts (probability < 1e-42) a
// disc without a point takes (0, 0) (first) or (1, 0) (second).  Every
// operation is a correctly rounded IEEE one, so a host restatement gives
// the same bits.
constexpr uint32_t kKickAttempts = 64u;

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

__device__ __forceinline__ double kick_uniform(uint32_t r) {
    return Rn::mul(Rn::add(double(int32_t(r)), 0.5), 0x1p-31);
}

struct KickDirection {
    double d0, d1, d2, d3;
};

__device__ __forceinline__ KickDirection kick_direction(unsigned long long seed,
                                                        unsigned long long idx, uint32_t turn) {
    const uint32_t k0 = uint32_t(seed), k1 = uint32_t(seed >> 32);
    double u1 = 0.0, u2 = 0.0, u3 = 1.0, u4 = 0.0, s1 = 0.0, s2 = 1.0;
    bool got1 = false, got2 = false;
    for (uint32_t a = 0; a < kKickAttempts && !(got1 && got2); ++a) {
        const uint4 r = philox4x32_10(make_uint4(turn, a, uint32_t(idx), uint32_t(idx >> 32)), k0, k1);
        if (!got1) {
            const double a1 = kick_uniform(r.x), a2 = kick_uniform(r.y);
            const double s = Rn::add(Rn::mul(a1, a1), Rn::mul(a2, a2));
            if (s < 1.0) {
                u1 = a1;
                u2 = a2;
                s1 = s;
                got1 = true;
            }
        }
        if (!got2) {
            const double a3 = kick_uniform(r.z), a4 = kick_uniform(r.w);
            const double s = Rn::add(Rn::mul(a3, a3), Rn::mul(a4, a4));
            if (s < 1.0 && s > 0.0) {
                u3 = a3;
                u4 = a4;
                s2 = s;
                got2 = true;
            }
        }
    }
    const double f = __dsqrt_rn(Rn::div(Rn::sub(1.0, s1), s2));
    return KickDirection{u1, u2, Rn::mul(u3, f), Rn::mul(u4, f)};
}

// Adds (forward) or subtracts (backward) the kick of module km along d and
// refreshes the carried squares.
template <bool SUB>
__device__ __forceinline__ void apply_kick(Particle &p, const KickDirection &d, double km) {
    if (SUB) {
        p.x = Rn::sub(p.x, Rn::mul(d.d0, km));
        p.px = Rn::sub(p.px, Rn::mul(d.d1, km));
        p.y = Rn::sub(p.y, Rn::mul(d.d2, km));
        p.py = Rn::sub(p.py, Rn::mul(d.d3, km));
    } else {
        p.x = Rn::add(p.x, Rn::mul(d.d0, km));
        p.px = Rn::add(p.px, Rn::mul(d.d1, km));
        p.y = Rn::add(p.y, Rn::mul(d.d2, km));
        p.py = Rn::add(p.py, Rn::mul(d.d3, km));
    }
    p.xx = Rn::mul(p.x, p.x);
    p.yy = Rn::mul(p.y, p.y);
}

// ---- the barrier test ------------------------------------------------------------
// A particle is kept while r < barrier^2 (check_barrier, src/henon.cu:
// 113-116).  r is a sum of squares, so it is +0, positive, +inf or NaN, and
// the comparison is an unsigned compare of bit patterns: non-negative
// doubles order like their patterns and every NaN pattern, of either sign,
// lies above +inf's, so NaN particles are lost exactly when
// `r < barrier_pow_2` is false.  The test stays off the FP64 pipe.
//
// In exact arithmetic the decision must be the one the separately rounded
// sum radius_exact gives.  It is taken from radius_fma instead whenever
// radius_fma lies more than kBarrierMargin patterns below barrier^2: the
// two sums are within 2 + 3 rounding errors of the same non-negative real
// sum, i.e. within ~6 representable doubles of each other (subnormal and
// overflowing sums included), so a margin of 64 decides the same way.
// Inside the margin (or above it, where the particle may be lost) the
// caller settles the test with radius_exact.  Fast arithmetic uses
// radius_fma itself (margin 0).
constexpr unsigned long long kBarrierMargin = 64ull;

// Before any of that, a test on the coordinates alone, on the integer pipe:
// if |x|, |px|, |y|, |py| are all below T = sqrt(barrier^2)/2 (1 - 2^-20),
// every computed sum of their squares (either grouping, with or without
// FMAs: at most four roundings of non-negative terms, each below T^2) is
// below 4 T^2 (1 + 2^-50) < barrier^2, so the particle is inside in both
// arithmetic modes.  The test compares the high words of |c|'s bit
// patterns with that of T (a smaller high word means a smaller value; NaN
// and infinities lie above every finite T).  barrier^2 = +inf takes
// T = sqrt(DBL_MAX)/2 (1 - 2^-20), so that the bound stays finite; a NaN
// barrier arrives as pattern 0 and disables the test, as does a tiny one.
// In a stable orbit every coordinate stays far below the barrier, so the
// common case spends no FP64 instruction on the barrier at all.
struct Barrier {
    unsigned long long b2;  // pattern of barrier^2 (0 for a NaN barrier)
    unsigned long long lo;  // patterns below lo: inside for certain
    unsigned long long hi;  // exact arithmetic: patterns above hi are outside
    uint32_t small_hi;      // high word of T: all |c| high words below it: inside
};

__device__ __forceinline__ uint32_t small_threshold_hi(unsigned long long b2) {
    const double r2 = fmin(__longlong_as_double(static_cast<long long>(b2)), 1.7976931348623157e308);
    // Near the subnormal range rounding errors are absolute, not relative:
    // a barrier^2 below 2^-900 disables the test (above it the margin
    // r2 2^-19 always exceeds four subnormal rounding errors of 2^-1075).
    if (!(r2 >= 0x1p-900)) return 0u;
    const double t = Rn::mul(Rn::mul(__dsqrt_rn(r2), 0.5), 1.0 - 0x1p-20);
    return static_cast<uint32_t>(__double2hiint(t));
}

template <int ARITH>
__device__ __forceinline__ Barrier make_barrier(long long b2bits) {
    const unsigned long long b2 = static_cast<unsigned long long>(b2bits);
    const uint32_t small_hi = small_threshold_hi(b2);
    if (ARITH != HM_ARITH_EXACT) return Barrier{b2, b2, b2, small_hi};
    const unsigned long long lo = b2 > kBarrierMargin ? b2 - kBarrierMargin : 0ull;
    const unsigned long long hi = b2 < ~0ull - kBarrierMargin ? b2 + kBarrierMargin : ~0ull;
    return Barrier{b2, lo, hi, small_hi};
}

__device__ __forceinline__ unsigned long long pattern(double r) {
    return static_cast<unsigned long long>(__double_as_longlong(r));
}

__device__ __forceinline__ uint32_t abs_hi(double v) {
    return static_cast<uint32_t>(__double2hiint(v)) & 0x7fffffffu;
}

// OR of the high words of the four coordinates.  With the sign bit masked
// off, an OR of high words is at least each of them, so an OR below
// small_hi passes small_inside for every coordinate it covers: a thread
// ORs all its particles and compares once (three-input LOP3s, no FP64).
__device__ __forceinline__ uint32_t hi_or(const Particle &p) {
    return static_cast<uint32_t>(__double2hiint(p.x)) | static_cast<uint32_t>(__double2hiint(p.px)) |
           static_cast<uint32_t>(__double2hiint(p.y)) | static_cast<uint32_t>(__double2hiint(p.py));
}

__device__ __forceinline__ bool small_or(uint32_t ored, const Barrier &b) {
    return (ored & 0x7fffffffu) < b.small_hi;
}

// Every coordinate is small (no FP64 instruction).
__device__ __forceinline__ bool small_inside(const Particle &p, const Barrier &b) {
    const uint32_t m = max(max(abs_hi(p.x), abs_hi(p.px)), max(abs_hi(p.y), abs_hi(p.py)));
    return m < b.small_hi;
}

// Next case: r_fma decides "inside" on its own.
__device__ __forceinline__ bool surely_inside(double r_fma, const Barrier &b) {
    return pattern(r_fma) < b.lo;
}

// The rest: the reference's decision for a particle whose r_fma did not
// pass surely_inside.
template <int ARITH>
__device__ __forceinline__ bool settle_inside(double r_fma, const Particle &p, const Barrier &b) {
    if (ARITH != HM_ARITH_EXACT) return false;
    return pattern(r_fma) <= b.hi && pattern(radius_exact(p)) < b.b2;
}

template <int ARITH>
__device__ __forceinline__ bool inside(double r_fma, const Particle &p, const Barrier &b) {
    return surely_inside(r_fma, b) || settle_inside<ARITH>(r_fma, p, b);
}

// The whole decision for a particle after a turn: the coordinate test,
// then the FMA sum, then (exact arithmetic, near the barrier) the
// reference's sum.
template <int ARITH>
__device__ __forceinline__ bool inside_after_turn(const Particle &p, const Barrier &b) {
    return small_inside(p, b) || inside<ARITH>(radius_fma(p), p, b);
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

// Jacobian of one backward turn at the point (x, px, y, py) before it, in
// the expression order of the reference's inverse_tangent_matrix
// (src/henon.cu:224-249, where u and w are the coordinates after the
// inverse rotations and pow(v, 2) is v * v).
__device__ __forceinline__ void inverse_tangent_matrix_exact(double x, double px, double y,
                                                             double py, const Turn &t, double mu,
                                                             double m[16]) {
    using R = Rn;
    const double u = R::sub(R::mul(t.cx, x), R::mul(px, t.sx));
    const double w = R::sub(R::mul(t.cy, y), R::mul(py, t.sy));
    const double d2 = R::sub(R::mul(u, u), R::mul(w, w));
    const double mu3u = R::mul(R::mul(3.0, mu), u);
    const double gp = R::add(mu3u, 1.0);                       // 3 mu u + 1
    const double gm = R::sub(R::mul(R::mul(-3.0, mu), u), 1.0);  // -3 mu u - 1
    m[0] = t.cx;
    m[1] = -t.sx;
    m[2] = 0.0;
    m[3] = 0.0;
    m[4] = R::add(R::sub(R::mul(R::mul(R::mul(-3.0, t.cx), mu), d2), R::mul(R::mul(2.0, t.cx), u)),
                  t.sx);
    m[5] = R::add(R::add(t.cx, R::mul(R::mul(R::mul(3.0, mu), t.sx), d2)),
                  R::mul(R::mul(2.0, t.sx), u));
    m[6] = R::mul(R::mul(R::mul(2.0, t.cy), w), gp);
    m[7] = R::mul(R::mul(R::mul(2.0, t.sy), w), gm);
    m[8] = 0.0;
    m[9] = 0.0;
    m[10] = t.cy;
    m[11] = -t.sy;
    m[12] = R::mul(R::mul(R::mul(2.0, t.cx), w), gp);
    m[13] = R::mul(R::mul(R::mul(2.0, t.sx), w), gm);
    m[14] = R::add(R::add(R::mul(R::mul(R::mul(3.0, t.cy), mu), d2), R::mul(R::mul(2.0, t.cy), u)),
                   t.sy);
    m[15] = R::sub(R::sub(t.cy, R::mul(R::mul(R::mul(3.0, mu), t.sy), d2)),
                   R::mul(R::mul(2.0, t.sy), u));
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

// The same product for a = a turn's Jacobian (tangent_matrix_exact), whose
// rows have one structural zero each: entry 3 of rows 0 and 1, entry 1 of
// rows 2 and 3.  With every entry of b finite, a skipped term is 0 * b = +-0
// and adding +-0 to a running sum that started from +0.0 never changes it
// (the sum is never -0: x + y rounds to -0 only when both are -0), so the
// three remaining terms, added in k order to 0.0, give the dense product's
// bits.  The caller must fall back to matmul4_exact when b has an infinite
// or NaN entry (0 * inf is NaN in the dense sum).
__device__ __forceinline__ void jacobian_matmul4_exact(const double a[16], const double b[16],
                                                       double out[16]) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const double b0 = b[j], b1 = b[4 + j], b2 = b[8 + j], b3 = b[12 + j];
        out[j] = Rn::add(Rn::add(Rn::add(0.0, Rn::mul(a[0], b0)), Rn::mul(a[1], b1)),
                         Rn::mul(a[2], b2));
        out[4 + j] = Rn::add(Rn::add(Rn::add(0.0, Rn::mul(a[4], b0)), Rn::mul(a[5], b1)),
                             Rn::mul(a[6], b2));
        out[8 + j] = Rn::add(Rn::add(Rn::add(0.0, Rn::mul(a[8], b0)), Rn::mul(a[10], b2)),
                             Rn::mul(a[11], b3));
        out[12 + j] = Rn::add(Rn::add(Rn::add(0.0, Rn::mul(a[12], b0)), Rn::mul(a[14], b2)),
                              Rn::mul(a[15], b3));
    }
}

// The Jacobian applied to a vector, likewise (v finite).
__device__ __forceinline__ void jacobian_matvec4_exact(const double a[16], const double v[4],
                                                       double out[4]) {
    out[0] = Rn::add(Rn::add(Rn::add(0.0, Rn::mul(a[0], v[0])), Rn::mul(a[1], v[1])),
                     Rn::mul(a[2], v[2]));
    out[1] = Rn::add(Rn::add(Rn::add(0.0, Rn::mul(a[4], v[0])), Rn::mul(a[5], v[1])),
                     Rn::mul(a[6], v[2]));
    out[2] = Rn::add(Rn::add(Rn::add(0.0, Rn::mul(a[8], v[0])), Rn::mul(a[10], v[2])),
                     Rn::mul(a[11], v[3]));
    out[3] = Rn::add(Rn::add(Rn::add(0.0, Rn::mul(a[12], v[0])), Rn::mul(a[14], v[2])),
                     Rn::mul(a[15], v[3]));
}

// True when the double is neither infinite nor NaN (exponent field not all
// ones), tested on the integer pipe.
__device__ __forceinline__ bool finite_bits(double v) {
    return (static_cast<uint32_t>(__double2hiint(v)) & 0x7ff00000u) != 0x7ff00000u;
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
