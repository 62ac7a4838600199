// Reverse-mode adjoint of the modulated Henon map (sm_100a).
//
// Per particle i the orbit loss is the Birkhoff-weighted average
//     L_i = sum_{k=0}^{N-1} w_k A(x_{k+1}),   A = x^2 + px^2 + y^2 + py^2,
// w = birkhoff_weights(N), x_{k+1} the state after turn k.  Lost particles
// (outside the barrier before turn N) contribute nothing.
//
// Parameters theta = (omega_x0, omega_y0, epsilon, mu) with
//     omega_{x,y}(k) = omega_{x,y}0 (1 + epsilon S_k),
//     S_k = sum_j c_j cos(Omega_j (k + offset))   (SPS ripple, host table).
//
// One thread per particle: the forward pass stores a checkpoint every C
// turns; the reverse sweep recomputes each segment from its checkpoint into
// a scratch buffer and propagates the adjoint lambda_k = J_k^T lambda_{k+1}
// + w_{k-1} grad A(x_k) through it, accumulating dL_i/dtheta.  The forward
// arithmetic is the tracker's (exact or FMA), so the orbit is the one
// hm_track computes.  A forward-mode kernel (tangent map M_k propagated
// along the orbit, g = sum_k w_k M_{k+1}^T grad A(x_{k+1})) gives an
// independent J^T v for the initial conditions.
#include <cuda_runtime.h>

#include <cstdint>

#include "hm_device.cuh"
#include "hm_internal.h"

namespace hm {
namespace {

using dev::Rn;

struct S4 {
    double x, px, y, py;
};

// The inverse-sweep kernel walks the turns in step across its block, so it
// stages each turn's records -- the rotation record, w_k and S_k -- through
// shared memory: while the block runs the kStage turns of one stage, each
// thread holds kPerThread doubles of the next stage in registers (plain
// loads, issued a whole stage ahead of use) and stores them into the other
// buffer at the end of the stage.  The launch often holds few warps per
// SM, too few to hide per-turn L2 latency otherwise.  (Blocks of 64 threads
// balance a small launch better over the SMs but measured 2.6 % slower:
// twice the staging registers per thread.)
constexpr int kThreads = 128;
constexpr uint32_t kStage = 64u;
constexpr int kRec = 6;  // doubles per turn: sin wx, cos wx, sin wy, cos wy, w_k, S_k
constexpr int kPerThread = int(kStage) * kRec / kThreads;
static_assert(kPerThread * kThreads == int(kStage) * kRec, "stage must split evenly");

// Records of turns [lo, lo + kn) into registers, element e = 6 (turn - lo) + field.
__device__ __forceinline__ void rec_load(double (&r)[kPerThread], const AdjointArgs &a,
                                         uint32_t lo, uint32_t kn) {
#pragma unroll
    for (int q = 0; q < kPerThread; ++q) {
        const uint32_t e = threadIdx.x + uint32_t(kThreads * q);
        const uint32_t t = e / uint32_t(kRec), f = e % uint32_t(kRec);
        double v = 0.0;
        if (t < kn) {
            const size_t k = size_t(lo) + t;
            v = f < 4u ? a.table[4u * k + f] : (f == 4u ? a.w[k] : a.S[k]);
        }
        r[q] = v;
    }
}

__device__ __forceinline__ void rec_store(double *buf, const double (&r)[kPerThread]) {
#pragma unroll
    for (int q = 0; q < kPerThread; ++q) buf[threadIdx.x + uint32_t(kThreads * q)] = r[q];
}

// One forward turn of a particle held with its squares (dev::Particle, so
// that x*x and y*y are not recomputed).  Sets `in` to the tracker's survival
// decision (the same barrier test, bit for bit) and returns the radius the
// loss uses: x^2+px^2+y^2+py^2 with two FMAs, within 2 ulp of the
// separately rounded sum.
template <int ARITH, bool OCT>
__device__ __forceinline__ double fwd(dev::Particle &p, const dev::Turn &t, double mu,
                                      const dev::Barrier &bar, bool &in) {
    dev::turn<ARITH, OCT, false>(p, t, mu);
    const double r = dev::radius_fma(p);
    in = dev::small_inside(p, bar) || dev::inside<ARITH>(r, p, bar);
    return r;
}

__device__ __forceinline__ S4 coords(const dev::Particle &p) { return S4{p.x, p.px, p.y, p.py}; }

__device__ __forceinline__ void store4(double *buf, size_t slot, size_t n, size_t i, const S4 &s) {
    double *b = buf + slot * 4 * n;
    b[i] = s.x;
    b[n + i] = s.px;
    b[2 * n + i] = s.y;
    b[3 * n + i] = s.py;
}

__device__ __forceinline__ S4 load4(const double *buf, size_t slot, size_t n, size_t i) {
    const double *b = buf + slot * 4 * n;
    return S4{b[i], b[n + i], b[2 * n + i], b[3 * n + i]};
}

template <int ARITH, bool OCT>
__global__ void __launch_bounds__(128) adjoint_kernel(const AdjointArgs a) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const size_t n = a.n;
    const uint32_t N = a.n_turns, C = a.ckpt;
    dev::Particle s = dev::make_particle(a.x0[i], a.px0[i], a.y0[i], a.py0[i]);
    const dev::Barrier bar = dev::make_barrier<ARITH>(a.b2bits);
    bool alive = !dev::is_lost(s.x, s.px, s.y, s.py);
    double loss = 0.0;
    uint32_t k = 0;
    for (; alive && k < N; ++k) {
        if (k % C == 0) store4(a.ckpt_buf, k / C, n, i, coords(s));
        bool in;
        const double r = fwd<ARITH, OCT>(s, dev::load_turn(a.table, k), a.mu, bar, in);
        if (!in) {
            alive = false;
            break;
        }
        loss = fma(a.w[k], r, loss);
    }
    a.steps[i] = alive ? N : k;
    if (!alive) {
        a.loss[i] = 0.0;
        a.survived[i] = 0;
        a.g_ic[i] = a.g_ic[n + i] = a.g_ic[2 * n + i] = a.g_ic[3 * n + i] = 0.0;
        a.g_th[i] = a.g_th[n + i] = a.g_th[2 * n + i] = a.g_th[3 * n + i] = 0.0;
        return;
    }
    a.loss[i] = loss;
    a.survived[i] = 1;

    // Reverse sweep, segment by segment.
    double lx = 0.0, lpx = 0.0, ly = 0.0, lpy = 0.0;
    double g_wx = 0.0, g_wy = 0.0, g_eps = 0.0, g_mu = 0.0;
    const double mu = a.mu;
    const uint32_t n_seg = (N + C - 1) / C;
    for (int seg = int(n_seg) - 1; seg >= 0; --seg) {
        const uint32_t k0 = uint32_t(seg) * C;
        const uint32_t len = min(C, N - k0);
        const S4 c = load4(a.ckpt_buf, uint32_t(seg), n, i);
        dev::Particle q = dev::make_particle(c.x, c.px, c.y, c.py);
        for (uint32_t j = 0; j < len; ++j) {
            store4(a.seg_buf, j, n, i, coords(q));
            dev::turn<ARITH, OCT, false>(q, dev::load_turn(a.table, k0 + j), mu);
        }
        for (int j = int(len) - 1; j >= 0; --j) {
            const uint32_t kk = k0 + uint32_t(j);
            const S4 p = load4(a.seg_buf, uint32_t(j), n, i);
            const dev::Turn t = dev::load_turn(a.table, kk);
            // forward intermediates of turn kk
            const double x = p.x, y = p.y;
            const double xx = x * x, yy = y * y;
            const double qx = (xx - yy) + mu * x * (xx - 3.0 * yy);
            const double qy = -2.0 * x * y + mu * y * (yy - 3.0 * xx);
            const double px1 = p.px + qx, py1 = p.py + qy;
            const double X = t.cx * x + t.sx * px1, PX = -t.sx * x + t.cx * px1;
            const double Y = t.cy * y + t.sy * py1, PY = -t.sy * y + t.cy * py1;
            // dL/d(state after turn kk): lambda + w_kk grad A
            const double w2 = 2.0 * a.w[kk];
            const double aX = fma(w2, X, lx), aPX = fma(w2, PX, lpx);
            const double aY = fma(w2, Y, ly), aPY = fma(w2, PY, lpy);
            // rotation angle derivatives: d(X, PX)/d omega = (PX, -X)
            const double gwx = aX * PX - aPX * X;
            const double gwy = aY * PY - aPY * Y;
            const double Sk = a.S[kk];
            const double f = fma(a.epsilon, Sk, 1.0);
            g_wx = fma(gwx, f, g_wx);
            g_wy = fma(gwy, f, g_wy);
            g_eps = fma(Sk, a.omega_x0 * gwx + a.omega_y0 * gwy, g_eps);
            // through the rotations (transpose)
            const double rx = t.cx * aX - t.sx * aPX, rpx = t.sx * aX + t.cx * aPX;
            const double ry = t.cy * aY - t.sy * aPY, rpy = t.sy * aY + t.cy * aPY;
            // through the kicks
            const double da = 2.0 * x + 3.0 * mu * (xx - yy);     // dqx/dx
            const double db = -2.0 * y - 6.0 * mu * x * y;       // dqx/dy = dqy/dx
            const double dd = -2.0 * x + 3.0 * mu * (yy - xx);    // dqy/dy
            g_mu = fma(rpx, x * (xx - 3.0 * yy), fma(rpy, y * (yy - 3.0 * xx), g_mu));
            lx = rx + rpx * da + rpy * db;
            ly = ry + rpx * db + rpy * dd;
            lpx = rpx;
            lpy = rpy;
        }
    }
    a.g_ic[i] = lx;
    a.g_ic[n + i] = lpx;
    a.g_ic[2 * n + i] = ly;
    a.g_ic[3 * n + i] = lpy;
    a.g_th[i] = g_wx;
    a.g_th[n + i] = g_wy;
    a.g_th[2 * n + i] = g_eps;
    a.g_th[3 * n + i] = g_mu;
}

// Reverse sweep without a segment buffer: inside each segment the pre-turn
// states are rebuilt backwards with the map's exact inverse (inverse
// rotations, then the kicks subtracted), starting from the stored state at
// the segment's end (the next checkpoint, or the final state).  Rounding
// errors of the reconstruction can grow only across one segment, and the
// per-turn memory traffic of the replay variant disappears.
// P particles per thread (particle index blockIdx.x * P * kThreads +
// j * kThreads + threadIdx.x): P independent chains per thread hide the
// latency of each turn's dependent FP64 operations.
template <int ARITH, bool OCT, int P>
__global__ void __launch_bounds__(kThreads) adjoint_inverse_kernel(const AdjointArgs a) {
    __shared__ __align__(16) double recs[2][kStage * kRec];
    const size_t n = a.n;
    const uint32_t N = a.n_turns, C = a.ckpt;
    const uint32_t n_stages = (N + kStage - 1) / kStage;
    const dev::Barrier bar = dev::make_barrier<ARITH>(a.b2bits);
    size_t idx[P];
    bool in_range[P], alive[P];
    dev::Particle s[P];
#pragma unroll
    for (int j = 0; j < P; ++j) {
        idx[j] = (size_t(blockIdx.x) * P + j) * kThreads + threadIdx.x;
        in_range[j] = idx[j] < n;
        const size_t ii = in_range[j] ? idx[j] : 0;
        s[j] = dev::make_particle(a.x0[ii], a.px0[ii], a.y0[ii], a.py0[ii]);
        alive[j] = in_range[j] && !dev::is_lost(s[j].x, s[j].px, s[j].y, s[j].py);
        // Particles out of the game hold zeros, a fixed point of the map.
        if (!alive[j]) s[j] = dev::make_particle(0.0, 0.0, 0.0, 0.0);
    }
    double next[kPerThread];

    // ---- forward sweep: loss and checkpoints ----------------------------------
    double loss[P];
    uint32_t lost_at[P];
#pragma unroll
    for (int j = 0; j < P; ++j) {
        loss[j] = 0.0;
        lost_at[j] = N;
    }
    uint32_t next_ckpt = 0;  // turn of the next checkpoint store
    if (n_stages > 0) {
        rec_load(next, a, 0u, min(kStage, N));
        rec_store(recs[0], next);
    }
    __syncthreads();
    for (uint32_t sg = 0; sg < n_stages; ++sg) {
        const uint32_t k0 = sg * kStage, kn = min(kStage, N - k0);
        const bool more = sg + 1 < n_stages;
        if (more) rec_load(next, a, k0 + kStage, min(kStage, N - k0 - kStage));
        const double *R = recs[sg & 1u];
        // The stage's turns with no branch on their results (the tracking
        // kernel's scheme, track.cu turns_staged): the loss accumulates and
        // every coordinate's high word is ORed; one warp vote at the end.
        // Only a warp with a coordinate at or above the bound of
        // dev::small_or (so possibly a loss) restores the stage's start and
        // redoes it with the per-turn test, which finds the loss turn.
        dev::Particle s0[P];
        double loss0[P];
#pragma unroll
        for (int j = 0; j < P; ++j) {
            s0[j] = s[j];
            loss0[j] = loss[j];
        }
        const uint32_t ckpt0 = next_ckpt;
        uint32_t ored = 0u;
        for (uint32_t kk = 0; kk < kn; ++kk) {
            const uint32_t k = k0 + kk;
            if (k == next_ckpt) {
#pragma unroll
                for (int j = 0; j < P; ++j)
                    if (alive[j]) store4(a.ckpt_buf, k / C, n, idx[j], coords(s[j]));
                next_ckpt += C;
            }
            const double *rr = R + kRec * kk;
            const dev::Turn t{rr[0], rr[1], rr[2], rr[3]};
#pragma unroll
            for (int j = 0; j < P; ++j) {
                dev::turn<ARITH, OCT, false>(s[j], t, a.mu);
                loss[j] = fma(rr[4], dev::radius_fma(s[j]), loss[j]);
                ored |= dev::hi_or(s[j]);
            }
        }
        if (__any_sync(dev::kFullMask, !dev::small_or(ored, bar))) {
#pragma unroll
            for (int j = 0; j < P; ++j) {
                s[j] = s0[j];
                loss[j] = loss0[j];
            }
            next_ckpt = ckpt0;
            for (uint32_t kk = 0; kk < kn; ++kk) {
                const uint32_t k = k0 + kk;
                if (k == next_ckpt) {
#pragma unroll
                    for (int j = 0; j < P; ++j)
                        if (alive[j]) store4(a.ckpt_buf, k / C, n, idx[j], coords(s[j]));
                    next_ckpt += C;
                }
                const double *rr = R + kRec * kk;
                const dev::Turn t{rr[0], rr[1], rr[2], rr[3]};
#pragma unroll
                for (int j = 0; j < P; ++j) {
                    bool in;
                    const double r = fwd<ARITH, OCT>(s[j], t, a.mu, bar, in);
                    loss[j] = fma(rr[4], r, loss[j]);
                    if (alive[j] && !in) {
                        lost_at[j] = k;
                        alive[j] = false;
                        s[j] = dev::make_particle(0.0, 0.0, 0.0, 0.0);
                    }
                }
            }
        }
        // The other buffer was last read in the previous stage, which the
        // whole block has finished; the barrier publishes the stores.
        if (more) rec_store(recs[(sg + 1u) & 1u], next);
        bool any = false;
#pragma unroll
        for (int j = 0; j < P; ++j) any |= alive[j];
        if (!__syncthreads_or(any)) break;
    }
#pragma unroll
    for (int j = 0; j < P; ++j)
        if (in_range[j]) {
            a.steps[idx[j]] = alive[j] ? N : lost_at[j];
            a.loss[idx[j]] = alive[j] ? loss[j] : 0.0;
            a.survived[idx[j]] = alive[j] ? 1 : 0;
        }

    // ---- reverse sweep: turns N-1 .. 0 --------------------------------------------
    // The sweep carries half the adjoint (lambda / 2, with w_k in place of
    // 2 w_k in grad A); every quantity is linear in it, so the results are
    // doubled, exactly, at the end.
    const double mu = a.mu, mu6 = -6.0 * a.mu;
    double lx[P], lpx[P], ly[P], lpy[P];
    // sum_k gw_k and sum_k S_k gw_k per plane: the parameter gradients are
    // combined from them at the end.
    double Gx[P], Gy[P], Hx[P], Hy[P], g_mu[P];
    S4 post[P], pre[P];
    const uint32_t n_seg = (N + C - 1) / C;
    bool any_alive = false;
#pragma unroll
    for (int j = 0; j < P; ++j) {
        lx[j] = lpx[j] = ly[j] = lpy[j] = 0.0;
        Gx[j] = Gy[j] = Hx[j] = Hy[j] = g_mu[j] = 0.0;
        post[j] = coords(s[j]);  // the state after turn N-1
        // The end state of the next (earlier) segment, loaded one segment
        // ahead of its use.
        pre[j] = S4{0.0, 0.0, 0.0, 0.0};
        if (alive[j] && n_seg > 1u) pre[j] = load4(a.ckpt_buf, n_seg - 1u, n, idx[j]);
        any_alive |= alive[j];
    }
    // Turns left in the current segment; at 0 the next (earlier) segment
    // starts from its stored end state, the checkpoint after it.
    uint32_t seg_left = N - (n_seg ? n_seg - 1u : 0u) * C;
    if (__syncthreads_or(any_alive) && n_stages > 0) {
        rec_load(next, a, N - min(kStage, N), min(kStage, N));
        rec_store(recs[0], next);
        __syncthreads();
        for (uint32_t sg = 0; sg < n_stages; ++sg) {
            const uint32_t k0 = sg * kStage, kn = min(kStage, N - k0);
            const bool more = sg + 1 < n_stages;
            if (more) {
                const uint32_t kn2 = min(kStage, N - k0 - kStage);
                rec_load(next, a, N - k0 - kStage - kn2, kn2);
            }
            // records of the table span [N - k0 - kn, N - k0), ascending
            const double *R = recs[sg & 1u];
            for (uint32_t jt = 0; any_alive && jt < kn; ++jt) {
                const uint32_t kk = N - 1u - (k0 + jt);  // turn index, descending
                if (seg_left == 0u) {
                    const uint32_t ci = (kk + 1u) / C;
#pragma unroll
                    for (int j = 0; j < P; ++j) {
                        post[j] = pre[j];
                        if (alive[j] && ci > 1u) pre[j] = load4(a.ckpt_buf, ci - 1u, n, idx[j]);
                    }
                    seg_left = C;
                }
                --seg_left;
                const double *rr = R + kRec * (kn - 1u - jt);
                const dev::Turn t{rr[0], rr[1], rr[2], rr[3]};
                const double w = rr[4], Sk = rr[5];
#pragma unroll
                for (int j = 0; j < P; ++j) {
                    const double X = post[j].x, PX = post[j].px, Y = post[j].y, PY = post[j].py;
                    // inverse turn (henon_step reverse order, src/henon.cu:510-528)
                    const double x = fma(t.cx, X, -t.sx * PX), px1 = fma(t.sx, X, t.cx * PX);
                    const double y = fma(t.cy, Y, -t.sy * PY), py1 = fma(t.sy, Y, t.cy * PY);
                    const double xx = x * x, yy = y * y, xy = x * y;
                    const double dxy = xx - yy;
                    // x (x^2 - 3y^2), y (y^2 - 3x^2): the octupole kicks over mu
                    const double xa = x * fma(-3.0, yy, xx), ya = y * fma(-3.0, xx, yy);
                    double qx = dxy, qy = -2.0 * xy;
                    if (OCT) {
                        qx = fma(mu, xa, qx);
                        qy = fma(mu, ya, qy);
                    }
                    post[j] = S4{x, px1 - qx, y, py1 - qy};
                    // adjoint of the post-turn state: (lambda + 2 w_k grad A) / 2
                    const double aX = fma(w, X, lx[j]), aPX = fma(w, PX, lpx[j]);
                    const double aY = fma(w, Y, ly[j]), aPY = fma(w, PY, lpy[j]);
                    const double gwx = fma(aX, PX, -aPX * X);
                    const double gwy = fma(aY, PY, -aPY * Y);
                    Gx[j] += gwx;
                    Gy[j] += gwy;
                    Hx[j] = fma(Sk, gwx, Hx[j]);
                    Hy[j] = fma(Sk, gwy, Hy[j]);
                    const double rx = fma(t.cx, aX, -t.sx * aPX), rpx = fma(t.sx, aX, t.cx * aPX);
                    const double ry = fma(t.cy, aY, -t.sy * aPY), rpy = fma(t.sy, aY, t.cy * aPY);
                    double da = 2.0 * x, db = -2.0 * y;
                    if (OCT) {
                        da = fma(3.0 * mu, dxy, da);
                        db = fma(mu6, xy, db);
                    }
                    // d(py1)/dy = -2x (- 3 mu (x^2 - y^2)) = -da exactly, since
                    // fma(-a, b, -c) = -fma(a, b, c).
                    const double dd = -da;
                    // d(px1, py1)/d mu = (x (x^2 - 3y^2), y (y^2 - 3x^2)), also at mu = 0
                    g_mu[j] = fma(rpx, xa, fma(rpy, ya, g_mu[j]));
                    lx[j] = fma(rpx, da, fma(rpy, db, rx));
                    ly[j] = fma(rpx, db, fma(rpy, dd, ry));
                    lpx[j] = rpx;
                    lpy[j] = rpy;
                }
            }
            if (more) rec_store(recs[(sg + 1u) & 1u], next);
            __syncthreads();
        }
    }
#pragma unroll
    for (int j = 0; j < P; ++j) {
        if (!in_range[j]) continue;
        const size_t i = idx[j];
        if (!alive[j]) {
            a.g_ic[i] = a.g_ic[n + i] = a.g_ic[2 * n + i] = a.g_ic[3 * n + i] = 0.0;
            a.g_th[i] = a.g_th[n + i] = a.g_th[2 * n + i] = a.g_th[3 * n + i] = 0.0;
            continue;
        }
        a.g_ic[i] = 2.0 * lx[j];
        a.g_ic[n + i] = 2.0 * lpx[j];
        a.g_ic[2 * n + i] = 2.0 * ly[j];
        a.g_ic[3 * n + i] = 2.0 * lpy[j];
        // omega(k) = omega0 (1 + eps S_k): d/d omega0 = 1 + eps S_k, d/d eps = omega0 S_k
        a.g_th[i] = 2.0 * fma(a.epsilon, Hx[j], Gx[j]);
        a.g_th[n + i] = 2.0 * fma(a.epsilon, Hy[j], Gy[j]);
        a.g_th[2 * n + i] = 2.0 * fma(a.omega_x0, Hx[j], a.omega_y0 * Hy[j]);
        a.g_th[3 * n + i] = 2.0 * g_mu[j];
    }
}

// Forward mode: loss and, with TANGENT, g = sum_k w_k M_{k+1}^T grad A(x_{k+1})
// with M_{k+1} = DF_k ... DF_0 (DF_k = tangent_matrix at x_k, table[k]).
// When a.g_th is given it also carries P_{k+1} = d x_{k+1} / d theta
// (4 x 4: state by theta = (omega_x0, omega_y0, epsilon, mu)),
//     P_{k+1} = DF_k P_k + E_k,
// E_k the explicit derivative of turn k: the rotation by omega(k) gives
// d(x', px')/d omega = (px', -x') (and likewise in y), with
// d omega(k)/d omega0 = 1 + epsilon S_k and d omega(k)/d epsilon = omega0 S_k;
// the octupole gives d(px1, py1)/d mu = (x^3 - 3 x y^2, y^3 - 3 x^2 y) at the
// turn's entry point, rotated with the turn.  Then
//     dL/dtheta_j = sum_k w_k grad A(x_{k+1}) . P_{k+1}[:, j],
// an independent check of the reverse sweep's theta gradient.
template <int ARITH, bool OCT, bool TANGENT>
__global__ void __launch_bounds__(128) forward_loss_kernel(const AdjointArgs a) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const size_t n = a.n;
    const bool theta = TANGENT && a.g_th != nullptr;
    dev::Particle s = dev::make_particle(a.x0[i], a.px0[i], a.y0[i], a.py0[i]);
    const dev::Barrier bar = dev::make_barrier<ARITH>(a.b2bits);
    bool alive = !dev::is_lost(s.x, s.px, s.y, s.py);
    double M[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    double P[16] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    double g[4] = {0, 0, 0, 0};
    double gt[4] = {0, 0, 0, 0};
    double loss = 0.0;
    uint32_t k = 0;
    for (; alive && k < a.n_turns; ++k) {
        const dev::Turn t = dev::load_turn(a.table, k);
        double df[16];
        double u = 0.0, v = 0.0;
        if (TANGENT) {
            dev::tangent_matrix_exact(s.x, s.y, t, a.mu, df);
            if (theta) {
                u = s.x * fma(-3.0, s.yy, s.xx);  // x^3 - 3 x y^2
                v = s.y * fma(-3.0, s.xx, s.yy);  // y^3 - 3 x^2 y
            }
        }
        bool in;
        const double r = fwd<ARITH, OCT>(s, t, a.mu, bar, in);
        if (!in) {
            alive = false;
            break;
        }
        loss = fma(a.w[k], r, loss);
        if (TANGENT) {
            double out[16];
#pragma unroll
            for (int rr = 0; rr < 4; ++rr)
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    double acc = 0.0;
#pragma unroll
                    for (int q = 0; q < 4; ++q) acc = fma(df[rr * 4 + q], M[q * 4 + c], acc);
                    out[rr * 4 + c] = acc;
                }
#pragma unroll
            for (int q = 0; q < 16; ++q) M[q] = out[q];
            const double w2 = 2.0 * a.w[k];
            const double vv[4] = {w2 * s.x, w2 * s.px, w2 * s.y, w2 * s.py};
#pragma unroll
            for (int c = 0; c < 4; ++c)
                g[c] = fma(M[c], vv[0], fma(M[4 + c], vv[1], fma(M[8 + c], vv[2], fma(M[12 + c], vv[3], g[c]))));
            if (theta) {
#pragma unroll
                for (int rr = 0; rr < 4; ++rr)
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        double acc = 0.0;
#pragma unroll
                        for (int q = 0; q < 4; ++q) acc = fma(df[rr * 4 + q], P[q * 4 + c], acc);
                        out[rr * 4 + c] = acc;
                    }
                const double Sk = a.S[k];
                const double f0 = fma(a.epsilon, Sk, 1.0);  // d omega(k) / d omega0
                const double ex = a.omega_x0 * Sk, ey = a.omega_y0 * Sk;  // d omega / d eps
                // columns: 0 omega_x0, 1 omega_y0, 2 epsilon, 3 mu
                out[0 * 4 + 0] = fma(s.px, f0, out[0 * 4 + 0]);
                out[1 * 4 + 0] = fma(-s.x, f0, out[1 * 4 + 0]);
                out[2 * 4 + 1] = fma(s.py, f0, out[2 * 4 + 1]);
                out[3 * 4 + 1] = fma(-s.y, f0, out[3 * 4 + 1]);
                out[0 * 4 + 2] = fma(s.px, ex, out[0 * 4 + 2]);
                out[1 * 4 + 2] = fma(-s.x, ex, out[1 * 4 + 2]);
                out[2 * 4 + 2] = fma(s.py, ey, out[2 * 4 + 2]);
                out[3 * 4 + 2] = fma(-s.y, ey, out[3 * 4 + 2]);
                out[0 * 4 + 3] = fma(t.sx, u, out[0 * 4 + 3]);
                out[1 * 4 + 3] = fma(t.cx, u, out[1 * 4 + 3]);
                out[2 * 4 + 3] = fma(t.sy, v, out[2 * 4 + 3]);
                out[3 * 4 + 3] = fma(t.cy, v, out[3 * 4 + 3]);
#pragma unroll
                for (int q = 0; q < 16; ++q) P[q] = out[q];
#pragma unroll
                for (int c = 0; c < 4; ++c)
                    gt[c] = fma(P[c], vv[0], fma(P[4 + c], vv[1], fma(P[8 + c], vv[2], fma(P[12 + c], vv[3], gt[c]))));
            }
        }
    }
    a.steps[i] = alive ? a.n_turns : k;
    a.survived[i] = alive ? 1 : 0;
    a.loss[i] = alive ? loss : 0.0;
    if (TANGENT) {
#pragma unroll
        for (int c = 0; c < 4; ++c) a.g_ic[size_t(c) * n + i] = alive ? g[c] : 0.0;
        if (theta) {
#pragma unroll
            for (int c = 0; c < 4; ++c) a.g_th[size_t(c) * n + i] = alive ? gt[c] : 0.0;
        }
    }
}

// Particles per thread of the inverse-sweep kernel (1 or 2; results do not
// depend on it).  Two chains per thread hide more of each turn's FP64
// latency: 4.92 ms against 5.20 ms on 65,536 particles x 1e4 turns.
int g_adjoint_per_thread = 2;

template <int ARITH>
cudaError_t launch_a(const AdjointArgs &a, int mode, cudaStream_t s) {
    const unsigned blocks = unsigned((a.n + 127) / 128);
    const bool oct = a.mu != 0.0;
    if (mode == 0) {
        if (oct) adjoint_kernel<ARITH, true><<<blocks, 128, 0, s>>>(a);
        else adjoint_kernel<ARITH, false><<<blocks, 128, 0, s>>>(a);
    } else if (mode == 3) {
        if (g_adjoint_per_thread == 2) {
            const unsigned b = unsigned((a.n + 2 * kThreads - 1) / (2 * kThreads));
            if (oct) adjoint_inverse_kernel<ARITH, true, 2><<<b, kThreads, 0, s>>>(a);
            else adjoint_inverse_kernel<ARITH, false, 2><<<b, kThreads, 0, s>>>(a);
        } else {
            const unsigned b = unsigned((a.n + kThreads - 1) / kThreads);
            if (oct) adjoint_inverse_kernel<ARITH, true, 1><<<b, kThreads, 0, s>>>(a);
            else adjoint_inverse_kernel<ARITH, false, 1><<<b, kThreads, 0, s>>>(a);
        }
    } else if (mode == 1) {
        if (oct) forward_loss_kernel<ARITH, true, true><<<blocks, 128, 0, s>>>(a);
        else forward_loss_kernel<ARITH, false, true><<<blocks, 128, 0, s>>>(a);
    } else {
        if (oct) forward_loss_kernel<ARITH, true, false><<<blocks, 128, 0, s>>>(a);
        else forward_loss_kernel<ARITH, false, false><<<blocks, 128, 0, s>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace

void set_adjoint_per_thread(int p) { g_adjoint_per_thread = p == 2 ? 2 : 1; }
int get_adjoint_per_thread() { return g_adjoint_per_thread; }

cudaError_t launch_adjoint(const AdjointArgs &a, int mode, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    return a.arith == HM_ARITH_FAST ? launch_a<HM_ARITH_FAST>(a, mode, s)
                                    : launch_a<HM_ARITH_EXACT>(a, mode, s);
}

}  // namespace hm
