// Fused multi-turn tracking kernels for the 4D modulated Henon map (sm_100a).
//
// One launch advances a list of live particles by a chunk of turns with the
// particle state held in registers (several particles per thread for
// instruction-level parallelism).  The per-turn rotation record
// {sin wx, cos wx, sin wy, cos wy} is the same for every live particle (all
// live particles share the same `steps`), so each warp reads one broadcast
// record per turn.  Losses are detected per turn; a lost particle is written
// out at once (NaN coordinates, frozen steps) and survivors are re-compacted
// into a dense list at the end of the chunk so that the next chunk's warps
// are full.
//
// Reference semantics: henon_step, src/henon.cu:420-542, built from the
// primitives of src/henon.cu:113-173; launch loop of
// henon_tracker_gpu::track, src/henon.cu:3155-3185.
#include <cuda_runtime.h>

#include <cstdint>

#include "hm_internal.h"

namespace hm {
namespace {

constexpr unsigned kFullMask = 0xffffffffu;

__device__ __forceinline__ double quiet_nan() {
    return __longlong_as_double(0x7ff8000000000000LL);  // glibc NAN
}

// Separately rounded binary64 operations; the __d*_rn intrinsics are never
// contracted into fused multiply-adds, so a sequence of them reproduces the
// host's SSE2 arithmetic bit for bit.
struct Rn {
    static __device__ __forceinline__ double mul(double a, double b) {
        return __dmul_rn(a, b);
    }
    static __device__ __forceinline__ double add(double a, double b) {
        return __dadd_rn(a, b);
    }
    static __device__ __forceinline__ double sub(double a, double b) {
        return __dsub_rn(a, b);
    }
};

struct Turn {
    double sx, cx, sy, cy;
};

__device__ __forceinline__ Turn load_turn(const double *table, uint32_t i) {
    const double2 *p = reinterpret_cast<const double2 *>(table) + 2 * size_t(i);
    const double2 a = __ldg(p);
    const double2 b = __ldg(p + 1);
    return Turn{a.x, a.y, b.x, b.y};
}

// Particle in registers; xx = x*x and yy = y*y of the current coordinates
// are carried from the barrier test of one turn into the kicks of the next
// (the reference computes the same products twice).
struct Particle {
    double x, px, y, py, xx, yy;
};

// ---- one turn, reference order ---------------------------------------------
// Forward: sextupole, [octupole], rotate x then y with table[steps]
// (src/henon.cu:493-508).  Returns x^2+px^2+y^2+py^2 grouped as
// (x*x + px*px) + (y*y + py*py) (check_barrier, src/henon.cu:113-116).
template <bool OCT>
__device__ __forceinline__ double turn_exact_fwd(Particle &p, const Turn &t,
                                                 double mu) {
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
    p.xx = Rn::mul(x, x);
    p.yy = Rn::mul(y, y);
    p.x = x;
    p.px = px;
    p.y = y;
    p.py = py;
    return Rn::add(Rn::add(p.xx, Rn::mul(px, px)), Rn::add(p.yy, Rn::mul(py, py)));
}

// Reverse: rotate x then y backwards with table[steps-1], subtract the
// octupole, subtract the sextupole (src/henon.cu:510-528).
template <bool OCT>
__device__ __forceinline__ double turn_exact_rev(Particle &p, const Turn &t,
                                                 double mu) {
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
    p.x = x;
    p.px = px;
    p.y = y;
    p.py = py;
    p.xx = xx;
    p.yy = yy;
    return Rn::add(Rn::add(xx, Rn::mul(px, px)), Rn::add(yy, Rn::mul(py, py)));
}

// ---- one turn, fused multiply-adds ----------------------------------------
// The same map with FMAs and x^3-3xy^2 = x(x^2-3y^2); 17 (mu=0) / 23 (mu!=0)
// FP64 instructions per particle-turn instead of 24 / 38.
template <bool OCT>
__device__ __forceinline__ double turn_fast_fwd(Particle &p, const Turn &t,
                                                double mu) {
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
    p.xx = x * x;
    p.yy = y * y;
    p.x = x;
    p.px = px;
    p.y = y;
    p.py = py;
    return fma(px, px, p.xx) + fma(py, py, p.yy);
}

template <bool OCT>
__device__ __forceinline__ double turn_fast_rev(Particle &p, const Turn &t,
                                                double mu) {
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
    p.x = x;
    p.px = px;
    p.y = y;
    p.py = py;
    p.xx = xx;
    p.yy = yy;
    return fma(px, px, xx) + fma(py, py, yy);
}

template <int ARITH, bool OCT, bool REV>
__device__ __forceinline__ double turn(Particle &p, const Turn &t, double mu) {
    if (ARITH == HM_ARITH_EXACT)
        return REV ? turn_exact_rev<OCT>(p, t, mu) : turn_exact_fwd<OCT>(p, t, mu);
    return REV ? turn_fast_rev<OCT>(p, t, mu) : turn_fast_fwd<OCT>(p, t, mu);
}

// r < barrier^2 for r = +0, positive finite, +inf or NaN (r is a sum of
// squares, never -0), as an unsigned 64-bit compare of the bit patterns:
// non-negative doubles order like their bit patterns and every NaN pattern,
// of either sign, lies above the pattern of +inf, so NaN/overflowed
// particles are lost exactly when `(...) < barrier_pow_2` is false.  Keeps
// the per-turn test off the FP64 pipe.
__device__ __forceinline__ bool inside(double r, long long b2bits) {
    return static_cast<unsigned long long>(__double_as_longlong(r)) <
           static_cast<unsigned long long>(b2bits);
}

// One chunk of turns for the particles of one block (K per thread).
template <int ARITH, bool OCT, bool REV, int K>
__global__ void __launch_bounds__(256)
track_chunk_kernel(const TrackChunk c) {
    const uint32_t n_in = c.in_count ? *c.in_count : c.n_user;
    const uint32_t base = blockIdx.x * (blockDim.x * K);
    if (base >= n_in) return;  // whole block past the list

    Particle p[K];
    uint32_t id[K];
    bool live[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const uint32_t e = base + j * blockDim.x + threadIdx.x;
        double x = 0.0, px = 0.0, y = 0.0, py = 0.0;
        live[j] = e < n_in;
        id[j] = e;
        if (live[j]) {
            if (c.in_idx) {
                id[j] = c.in_idx[e];
                x = c.in_x[e];
                px = c.in_px[e];
                y = c.in_y[e];
                py = c.in_py[e];
            } else {
                x = c.ux[e];
                px = c.upx[e];
                y = c.uy[e];
                py = c.upy[e];
                // check_nan (src/henon.cu:118-121): a NaN particle is left
                // untouched, steps included.
                live[j] = !(isnan(x) || isnan(px) || isnan(y) || isnan(py));
            }
        }
        p[j] = Particle{x, px, y, py, Rn::mul(x, x), Rn::mul(y, y)};
    }

    const double mu = c.mu;
    const long long b2 = c.b2bits;
    const uint32_t nt = c.n_turns;
    Turn t = nt ? load_turn(c.table, REV ? c.turn0 - 1u : c.turn0) : Turn{0.0, 0.0, 0.0, 0.0};
    bool thread_live = false;
#pragma unroll
    for (int j = 0; j < K; ++j) thread_live |= live[j];
    bool warp_live = __any_sync(kFullMask, thread_live);
    for (uint32_t k = 0; warp_live && k < nt; ++k) {
        // Prefetch the next turn's record (clamped to this chunk).
        const uint32_t kn = (k + 1 < nt) ? k + 1 : k;
        const Turn tn = load_turn(c.table, REV ? c.turn0 - 1u - kn : c.turn0 + kn);
        bool lost[K];
        bool any_lost = false;
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const double r = turn<ARITH, OCT, REV>(p[j], t, mu);
            lost[j] = live[j] && !inside(r, b2);
            any_lost |= lost[j];
        }
        if (__any_sync(kFullMask, any_lost)) {
            // Rare path: freeze lost particles (set_to_nan, :123-129); their
            // steps count the turns survived so far.
            const uint32_t s = REV ? c.turn0 - k : c.turn0 + k;
            bool any_live = false;
#pragma unroll
            for (int j = 0; j < K; ++j) {
                if (lost[j]) {
                    const uint32_t i = id[j];
                    c.ux[i] = quiet_nan();
                    c.upx[i] = quiet_nan();
                    c.uy[i] = quiet_nan();
                    c.upy[i] = quiet_nan();
                    c.usteps[i] = s;
                    live[j] = false;
                }
                any_live |= live[j];
            }
            warp_live = __any_sync(kFullMask, any_live);
        }
        t = tn;
    }

    if (c.out_idx == nullptr) {
        // Last chunk: survivors go back to the caller's arrays.
#pragma unroll
        for (int j = 0; j < K; ++j) {
            if (live[j]) {
                const uint32_t i = id[j];
                c.ux[i] = p[j].x;
                c.upx[i] = p[j].px;
                c.uy[i] = p[j].y;
                c.upy[i] = p[j].py;
                c.usteps[i] = c.steps_final;
            }
        }
        return;
    }
    // Re-compaction: each warp appends its survivors to the next list with
    // one atomic per slot; order inside a warp is preserved.
    const unsigned lane = threadIdx.x & 31u;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const unsigned m = __ballot_sync(kFullMask, live[j]);
        if (m == 0u) continue;
        const int leader = __ffs(m) - 1;
        uint32_t off = 0;
        if (lane == unsigned(leader)) off = atomicAdd(c.out_count, uint32_t(__popc(m)));
        off = __shfl_sync(kFullMask, off, leader);
        if (live[j]) {
            const uint32_t o = off + __popc(m & ((1u << lane) - 1u));
            c.out_idx[o] = id[j];
            c.out_x[o] = p[j].x;
            c.out_px[o] = p[j].px;
            c.out_y[o] = p[j].y;
            c.out_py[o] = p[j].py;
        }
    }
}

template <int ARITH, bool OCT, bool REV>
cudaError_t launch_k(const TrackChunk &c, const TrackLaunch &l, uint32_t n_upper,
                     cudaStream_t s) {
    const int threads = l.threads;
    const int K = l.per_thread;
    const uint64_t per_block = uint64_t(threads) * uint64_t(K);
    const unsigned blocks = unsigned((uint64_t(n_upper) + per_block - 1) / per_block);
    if (blocks == 0) return cudaSuccess;
    switch (K) {
        case 1: track_chunk_kernel<ARITH, OCT, REV, 1><<<blocks, threads, 0, s>>>(c); break;
        case 2: track_chunk_kernel<ARITH, OCT, REV, 2><<<blocks, threads, 0, s>>>(c); break;
        case 4: track_chunk_kernel<ARITH, OCT, REV, 4><<<blocks, threads, 0, s>>>(c); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <int ARITH>
cudaError_t launch_a(const TrackChunk &c, const TrackLaunch &l, uint32_t n, cudaStream_t s) {
    if (l.octupole)
        return l.reverse ? launch_k<ARITH, true, true>(c, l, n, s)
                         : launch_k<ARITH, true, false>(c, l, n, s);
    return l.reverse ? launch_k<ARITH, false, true>(c, l, n, s)
                     : launch_k<ARITH, false, false>(c, l, n, s);
}

// ---- observables ------------------------------------------------------------
// GPU getters of particles_4d_gpu (src/henon.cu:67-111): computed for every
// entry, NaN particles give NaN.  Sums are left to right, separately rounded.
__global__ void observable_kernel(const double *x, const double *px,
                                  const double *y, const double *py, double *out,
                                  size_t n, int kind) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double a = x[i], b = px[i], c = y[i], d = py[i];
    double v;
    switch (kind) {
        case HM_OBS_RADIUS:
            v = sqrt(Rn::add(Rn::add(Rn::add(Rn::mul(a, a), Rn::mul(b, b)), Rn::mul(c, c)),
                             Rn::mul(d, d)));
            break;
        case HM_OBS_ACTION:
            v = Rn::add(Rn::add(Rn::add(Rn::mul(a, a), Rn::mul(b, b)), Rn::mul(c, c)),
                        Rn::mul(d, d));
            break;
        case HM_OBS_ACTION_X: v = Rn::add(Rn::mul(a, a), Rn::mul(b, b)); break;
        case HM_OBS_ACTION_Y: v = Rn::add(Rn::mul(c, c), Rn::mul(d, d)); break;
        case HM_OBS_ANGLE_X: v = atan2(b, a); break;
        default: v = atan2(d, c); break;
    }
    out[i] = v;
}

// ---- FP64 peak ---------------------------------------------------------------
// Eight independent FMA chains per thread; the denominator of the FP64
// roofline (an FMA counts as two flops).
__global__ void __launch_bounds__(256) fp64_peak_kernel(double *sink, int iters,
                                                         double m, double a) {
    double v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = 1.0 + 1e-3 * (threadIdx.x + j);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = fma(v[j], m, a);
        }
    }
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += v[j];
    if (s == 12345.678) sink[blockIdx.x] = s;  // never true; keeps the chains live
}

}  // namespace

cudaError_t launch_track_chunk(const TrackChunk &c, const TrackLaunch &l,
                               uint32_t n_in_upper, cudaStream_t s) {
    if (l.threads <= 0 || l.threads > 256 || (l.threads & 31) != 0)
        return cudaErrorInvalidValue;
    return l.arith == HM_ARITH_FAST ? launch_a<HM_ARITH_FAST>(c, l, n_in_upper, s)
                                    : launch_a<HM_ARITH_EXACT>(c, l, n_in_upper, s);
}

cudaError_t launch_observable(const double *x, const double *px, const double *y,
                              const double *py, double *out, size_t n, int kind,
                              cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const unsigned blocks = unsigned((n + 255) / 256);
    observable_kernel<<<blocks, 256, 0, s>>>(x, px, y, py, out, n, kind);
    return cudaGetLastError();
}

cudaError_t launch_fp64_peak(double *sink, int blocks, int threads, int iters,
                             cudaStream_t s, double *flops) {
    fp64_peak_kernel<<<blocks, threads, 0, s>>>(sink, iters, 0.9999999, 1e-7);
    *flops = double(blocks) * threads * double(iters) * 16.0 * 8.0 * 2.0;
    return cudaGetLastError();
}

}  // namespace hm
