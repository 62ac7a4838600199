// Fused multi-turn tracking + tangent map + indicators (sm_100a).
//
// The reference computes indicators from Python, one turn at a time, with
// 3-6 launches per turn (tests/test_construct.ipynb, test_new_standard.ipynb):
//
//     M_old.explicit_copy(M)                  (when MEGNO is accumulated)
//     tracker.track(p, 1, mu, barrier)
//     M.structured_multiply(tracker, p, mu)   DF(x_{n+1}; table[global_steps])
//     megno.add(M, M_old); megno_b.add(M, M_old)
//     J.set_with_tracker(tracker, p, mu); v.multiply(J); lyap.add(v); v.normalize()
//     tune.add(p)
//
// This kernel runs that loop for a chunk of turns in one launch, one
// particle per thread, with the orbit, M, v and the MEGNO layers in
// registers and the per-window accumulators in shared memory.  Every step
// uses the same separately rounded arithmetic and the same CUDA libm calls
// as the per-call kernels (tangent.cu), so the results are bit-identical to
// running the loop with the per-call API or with the reference CUDA build
// compiled with --fmad=false.
#include <cuda_runtime.h>

#include <cstdint>

#include "hm_device.cuh"
#include "hm_internal.h"

namespace hm {
namespace {

using dev::Rn;

// Windows of one kind, sorted by the sample index at which they stop taking
// samples (every window starts at the construct's first sample, so at any
// index the open windows are a suffix of this order).  Built per block in
// shared memory: a turn then walks its open windows with a counter, reading
// each one's bound and weight pointer as a broadcast, instead of loading
// bounds and offsets from global memory per window and turn.
struct WinEntry {
    const double *w;  // the window's weights
    uint64_t len;     // MEGNO-Birkhoff: T; Lyapunov: length; tunes: T
    uint64_t lim;     // first index at which the window is closed
    double dlen;      // double(len) (Lyapunov's divisor)
    int orig;         // the window's index in the construct
    int pad;
};

template <int KIND>  // 0: MEGNO-Birkhoff (open while idx <= T), 1: Lyapunov
                     // (idx < length), 2: tunes (two windows, idx < 2 T)
__device__ __forceinline__ uint64_t window_limit(uint64_t b) {
    return KIND == 0 ? b + 1u : (KIND == 1 ? b : 2u * b);
}

// Every thread of the block takes part; ties keep the construct's order.
template <int KIND>
__device__ __forceinline__ void build_windows(WinEntry *tab, const uint64_t *bound,
                                              const uint64_t *off, const double *w, int n) {
    for (int v = int(threadIdx.x); v < n; v += int(blockDim.x)) {
        const uint64_t lim = window_limit<KIND>(bound[v]);
        int rank = 0;
        for (int u = 0; u < n; ++u) {
            const uint64_t lu = window_limit<KIND>(bound[u]);
            rank += (lu < lim || (lu == lim && u < v)) ? 1 : 0;
        }
        WinEntry e;
        e.w = w + off[v];
        e.len = bound[v];
        e.lim = lim;
        e.dlen = double(bound[v]);
        e.orig = v;
        e.pad = 0;
        tab[rank] = e;
    }
}

// First open window at index idx, from a previous first open window.
__device__ __forceinline__ int first_open(const WinEntry *tab, int n, int s, uint64_t idx) {
    while (s < n && tab[s].lim <= idx) ++s;
    return s;
}

// Next sample turn of MEGNO at or after idx (~0 when none).
__device__ __forceinline__ uint64_t next_sample(const uint64_t *turns, int n, uint64_t idx) {
    uint64_t best = ~0ull;
    for (int j = 0; j < n; ++j) {
        const uint64_t s = turns[j];
        if (s >= idx && s < best) best = s;
    }
    return best;
}

// SPLIT: every particle is followed by two warps.  Both track it (the
// same operations, so the same orbit); the even warp of a pair also carries
// the tangent matrix, MEGNO and the MEGNO-Birkhoff windows, the odd one the
// tangent vector, the Lyapunov windows and the tunes.  Each thread then
// holds about half of a particle's window accumulators, so the same shared
// memory holds twice the threads: the loop is a long chain of dependent
// FP64 operations, and more warps per SM hide its latency.
// EXT: kicks and backward turns (whole-orbit MEGNO: DO_M alone, the
// Jacobian of each turn at the point before it).
template <bool OCT, bool DO_M, bool DO_V, bool DO_T, bool SPLIT, bool EXT = false>
__global__ void __launch_bounds__(128, SPLIT ? 4 : 1) indicators_kernel(const FusedArgs a) {
    extern __shared__ double smem[];
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    // Role of this warp: with SPLIT, even warps do the matrix work and odd
    // warps the vector and tune work; without it, every warp does all.
    const bool role_m = !SPLIT || (warp & 1u) == 0u;
    const bool role_v = !SPLIT || (warp & 1u) == 1u;
    const bool do_m = DO_M && role_m, do_v = DO_V && role_v, do_t = DO_T && role_v;
    // Threads (per role) of a block, and this thread's index among them.
    const int T = SPLIT ? int(blockDim.x) / 2 : int(blockDim.x);
    const int tid = SPLIT ? int((warp >> 1) * 32u + lane) : int(threadIdx.x);
    const uint32_t i = blockIdx.x * uint32_t(T) + uint32_t(tid);
    const bool in_range = i < a.n;
    const uint32_t ii = in_range ? i : 0;
    // Per-thread window accumulators in shared memory, laid out [slot][thread]
    // so that a warp touches 32 consecutive doubles.  With SPLIT the matrix
    // role's slots come first, then the vector role's, each T threads wide.
    double *mb_l2 = smem;                                  // [n_mb][T]
    double *ly_raw = mb_l2 + size_t(a.n_mb) * T;           // [n_ly][T]
    double *ly_b = ly_raw + size_t(a.n_ly) * T;            // [n_ly][T]
    double *t1x = ly_b + size_t(a.n_ly) * T;               // [n_tu][T]
    double *t1y = t1x + size_t(a.n_tu) * T;
    double *t2x = t1y + size_t(a.n_tu) * T;
    double *t2y = t2x + size_t(a.n_tu) * T;
    // then the window tables of the three kinds (sorted by closing index);
    // the accumulators above are kept in table order.
    WinEntry *tab_mb = reinterpret_cast<WinEntry *>(t2y + size_t(a.n_tu) * T);
    WinEntry *tab_ly = tab_mb + a.n_mb;
    WinEntry *tab_tu = tab_ly + a.n_ly;
    const size_t n = a.n;
    if (DO_M && a.mb_l1) build_windows<0>(tab_mb, a.mb_T, a.mb_off, a.mb_w, a.n_mb);
    if (DO_V) build_windows<1>(tab_ly, a.ly_len, a.ly_off, a.ly_w, a.n_ly);
    if (DO_T) build_windows<2>(tab_tu, a.tu_T, a.tu_off, a.tu_w, a.n_tu);
    __syncthreads();

    // ---- load state ---------------------------------------------------------
    double x = a.x[ii], px = a.px[ii], y = a.y[ii], py = a.py[ii];
    uint32_t steps = a.steps[ii];
    bool alive = in_range && !dev::is_lost(x, px, y, py);
    double M[16];
    double old_norm = 0.0, m_l1 = 0.0, m_l2 = 0.0, m_l3 = 0.0, b_l1 = 0.0;
    if (do_m) {
#pragma unroll
        for (int k = 0; k < 16; ++k) M[k] = a.M[size_t(ii) * 16 + k];
        old_norm = dev::norm_exact<16>(M);
        if (a.megno_l1) {
            m_l1 = a.megno_l1[ii];
            m_l2 = a.megno_l2[ii];
            m_l3 = a.megno_l3[ii];
        }
        if (a.mb_l1) b_l1 = a.mb_l1[ii];
        for (int w = 0; w < a.n_mb; ++w) mb_l2[w * T + tid] = a.mb_l2[tab_mb[w].orig * n + ii];
    }
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (do_v) {
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = a.V[size_t(ii) * 4 + k];
        for (int w = 0; w < a.n_ly; ++w) {
            const size_t g = size_t(tab_ly[w].orig) * n + ii;
            ly_raw[w * T + tid] = a.ly_raw[g];
            ly_b[w * T + tid] = a.ly_b[g];
        }
    }
    double store_x = 0.0, store_y = 0.0;
    if (do_t) {
        store_x = a.store_x[ii];
        store_y = a.store_y[ii];
        for (int w = 0; w < a.n_tu; ++w) {
            const size_t g = size_t(tab_tu[w].orig) * n + ii;
            t1x[w * T + tid] = a.t1x[g];
            t1y[w * T + tid] = a.t1y[g];
            t2x[w * T + tid] = a.t2x[g];
            t2y[w * T + tid] = a.t2y[g];
        }
    }

    const double mu = a.mu;
    const dev::Barrier bar = dev::make_barrier<HM_ARITH_EXACT>(a.b2bits);
    bool warp_live = __any_sync(dev::kFullMask, alive);
    // First open window of each kind, and the next MEGNO sample turn.
    const bool snaps = do_m && a.megno_l1 && a.n_snap > 0;
    uint64_t next_snap = snaps ? next_sample(a.snap_turns, a.n_snap, a.megno_idx) : ~0ull;
    int s_mb = first_open(tab_mb, a.mb_l1 ? a.n_mb : 0, 0, a.mb_idx);
    int s_ly = first_open(tab_ly, a.n_ly, 0, a.ly_idx);
    int s_tu = first_open(tab_tu, a.n_tu, 0, a.tu_idx);
    uint32_t k = 0;
    for (; k < a.n_turns && warp_live; ++k) {
        double df[16];
        const bool rev = EXT && a.inverse;
        const uint32_t tidx = rev ? a.live_step - 1u - k : a.live_step + k;
        // ---- Jacobian of the turn, at the point before it (option) ------------
        if ((do_m || do_v) && a.df_before) {
            const dev::Turn td = dev::load_turn(a.table, tidx);
            if (rev) dev::inverse_tangent_matrix_exact(x, px, y, py, td, mu, df);
            else dev::tangent_matrix_exact(x, y, td, mu, df);
        }
        // ---- track(p, 1) ------------------------------------------------------
        if (alive) {
            const dev::Turn t = dev::load_turn(a.table, tidx);
            dev::Particle q = dev::make_particle(x, px, y, py);
            if (EXT) {
                // kicks as hm_track: before the forward turn, subtracted
                // after the backward one, keyed by the particle's index
                const bool kick = !isnan(a.kick_module);
                if (kick && !rev)
                    dev::apply_kick<false>(q, dev::kick_direction(a.kick_seed, ii, tidx),
                                           a.kick_module);
                if (rev) dev::turn<HM_ARITH_EXACT, OCT, true>(q, t, mu);
                else dev::turn<HM_ARITH_EXACT, OCT, false>(q, t, mu);
                if (kick && rev)
                    dev::apply_kick<true>(q, dev::kick_direction(a.kick_seed, ii, tidx),
                                          a.kick_module);
            } else {
                dev::turn<HM_ARITH_EXACT, OCT, false>(q, t, mu);
            }
            if (dev::inside_after_turn<HM_ARITH_EXACT>(q, bar)) {
                steps = rev ? steps - 1u : steps + 1u;
                x = q.x;
                px = q.px;
                y = q.y;
                py = q.py;
            } else {
                x = px = y = py = dev::quiet_nan();
                alive = false;
            }
        }
        // ---- tangent matrix at the new point, table[global_steps] -------------
        if ((do_m || do_v) && !a.df_before) {
            const dev::Turn td = dev::load_turn(a.table, a.global_step + k + 1u);
            dev::tangent_matrix_exact(x, y, td, mu, df);
        }
        if (do_m) {
            // old_norm is the norm of M: finite exactly when every entry is
            // (an overflowing sum of finite squares also takes the dense
            // product, which is then equally right).
            double out[16];
            // (the backward turn's Jacobian has other structural zeros)
            if (!rev && dev::finite_bits(old_norm)) dev::jacobian_matmul4_exact(df, M, out);
            else dev::matmul4_exact(df, M, out);
#pragma unroll
            for (int q = 0; q < 16; ++q) M[q] = out[q];
            const double new_norm = dev::norm_exact<16>(M);
            const double lr = log10(Rn::div(new_norm, old_norm));
            if (a.megno_l1) {
                const double di = double(a.megno_idx + k);
                const double inv = Rn::div(1.0, di);  // 1.0/idx, used twice
                m_l1 = Rn::add(m_l1, Rn::mul(lr, di));
                m_l2 = Rn::add(m_l2, Rn::mul(inv, m_l1));
                m_l3 = Rn::mul(inv, m_l2);
                const uint64_t cur = a.megno_idx + k;
                if (cur == next_snap) {  // a sample turn: every slot that asks
                    for (int j = 0; j < a.n_snap; ++j)
                        if (a.snap_turns[j] == cur && in_range) a.snap[size_t(j) * n + ii] = m_l3;
                    next_snap = next_sample(a.snap_turns, a.n_snap, cur + 1u);
                }
            }
            if (a.mb_l1) {
                const uint64_t idx = a.mb_idx + k;
                const double di = double(idx);
                b_l1 = Rn::add(b_l1, Rn::mul(lr, di));
                s_mb = first_open(tab_mb, a.n_mb, s_mb, idx);
                for (int w = s_mb; w < a.n_mb; ++w) {
                    double &acc = mb_l2[w * T + tid];
                    acc = Rn::add(acc, Rn::div(Rn::mul(b_l1, tab_mb[w].w[idx - 1]), di));
                }
            }
            old_norm = new_norm;
        }
        if (do_v) {
            double t4[4];
            if (dev::finite_bits(v[0]) && dev::finite_bits(v[1]) && dev::finite_bits(v[2]) &&
                dev::finite_bits(v[3])) {
                dev::jacobian_matvec4_exact(df, v, t4);
            } else {
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    double s = 0.0;
#pragma unroll
                    for (int c = 0; c < 4; ++c) s = Rn::add(s, Rn::mul(df[r * 4 + c], v[c]));
                    t4[r] = s;
                }
            }
            const double nv = dev::norm_exact<4>(t4);
            if (a.n_ly) {
                const double l = log(nv);
                const uint64_t idx = a.ly_idx + k;
                s_ly = first_open(tab_ly, a.n_ly, s_ly, idx);
                for (int w = s_ly; w < a.n_ly; ++w) {
                    const WinEntry &e = tab_ly[w];
                    ly_raw[w * T + tid] = Rn::add(ly_raw[w * T + tid], Rn::div(l, e.dlen));
                    ly_b[w * T + tid] = Rn::add(ly_b[w * T + tid], Rn::mul(l, e.w[idx]));
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) v[q] = Rn::div(t4[q], nv);
        }
        if (do_t) {
            const double ax = atan2(px, x), ay = atan2(py, y);
            double dx = Rn::sub(ax, store_x), dy = Rn::sub(ay, store_y);
            const double two_pi = 2 * M_PI;
            dx = dx > 0 ? dx : Rn::add(dx, two_pi);
            dy = dy > 0 ? dy : Rn::add(dy, two_pi);
            store_x = ax;
            store_y = ay;
            const uint64_t idx = a.tu_idx + k;
            s_tu = first_open(tab_tu, a.n_tu, s_tu, idx);
            for (int w = s_tu; w < a.n_tu; ++w) {
                const WinEntry &e = tab_tu[w];
                if (idx < e.len) {  // first window [0, T)
                    const double wt = e.w[idx];
                    t1x[w * T + tid] = Rn::add(t1x[w * T + tid], Rn::mul(dx, wt));
                    t1y[w * T + tid] = Rn::add(t1y[w * T + tid], Rn::mul(dy, wt));
                } else {  // second window [T, 2 T)
                    const double wt = e.w[idx - e.len];
                    t2x[w * T + tid] = Rn::add(t2x[w * T + tid], Rn::mul(dx, wt));
                    t2y[w * T + tid] = Rn::add(t2y[w * T + tid], Rn::mul(dy, wt));
                }
            }
        }
        // A warp whose particles are all lost stops: every later update
        // would only add NaN to windows that are still open (fixed below).
        if (!alive) warp_live = __any_sync(dev::kFullMask, alive);
    }

    // ---- windows a stopped warp would still have touched become NaN --------
    if (k < a.n_turns) {
        const double nan = dev::quiet_nan();
        const uint64_t left = a.n_turns - k;  // turns skipped
        if (do_m && a.megno_l1)
            for (int j = 0; j < a.n_snap; ++j) {
                const uint64_t s = a.snap_turns[j];
                if (s >= a.megno_idx + k && s < a.megno_idx + a.n_turns && in_range)
                    a.snap[size_t(j) * n + ii] = nan;
            }
        if (do_m && a.mb_l1) {
            const uint64_t idx = a.mb_idx + k;
            for (int w = 0; w < a.n_mb; ++w)
                if (idx <= tab_mb[w].len) mb_l2[w * T + tid] = nan;
        }
        if (do_v) {
            const uint64_t idx = a.ly_idx + k;
            for (int w = 0; w < a.n_ly; ++w)
                if (idx < tab_ly[w].len) {
                    ly_raw[w * T + tid] = nan;
                    ly_b[w * T + tid] = nan;
                }
        }
        if (do_t) {
            const uint64_t first = a.tu_idx + k, last = a.tu_idx + k + left - 1;
            for (int w = 0; w < a.n_tu; ++w) {
                const uint64_t len = tab_tu[w].len;
                if (first < len) {
                    t1x[w * T + tid] = nan;
                    t1y[w * T + tid] = nan;
                }
                // window 2 is [len, 2 len): touched if it meets [first, last]
                if (first < 2 * len && last >= len) {
                    t2x[w * T + tid] = nan;
                    t2y[w * T + tid] = nan;
                }
            }
        }
    }

    if (!in_range) return;
    // ---- store state (both roles hold the same orbit; one writes it) ---------
    if (role_m) {
        a.x[i] = x;
        a.px[i] = px;
        a.y[i] = y;
        a.py[i] = py;
        a.steps[i] = steps;
    }
    if (do_m) {
#pragma unroll
        for (int q = 0; q < 16; ++q) a.M[size_t(i) * 16 + q] = M[q];
        if (a.megno_l1) {
            a.megno_l1[i] = m_l1;
            a.megno_l2[i] = m_l2;
            a.megno_l3[i] = m_l3;
        }
        if (a.mb_l1) a.mb_l1[i] = b_l1;
        for (int w = 0; w < a.n_mb; ++w) a.mb_l2[tab_mb[w].orig * n + i] = mb_l2[w * T + tid];
    }
    if (do_v) {
#pragma unroll
        for (int q = 0; q < 4; ++q) a.V[size_t(i) * 4 + q] = v[q];
        for (int w = 0; w < a.n_ly; ++w) {
            const size_t g = size_t(tab_ly[w].orig) * n + i;
            a.ly_raw[g] = ly_raw[w * T + tid];
            a.ly_b[g] = ly_b[w * T + tid];
        }
    }
    if (do_t) {
        a.store_x[i] = store_x;
        a.store_y[i] = store_y;
        for (int w = 0; w < a.n_tu; ++w) {
            const size_t g = size_t(tab_tu[w].orig) * n + i;
            a.t1x[g] = t1x[w * T + tid];
            a.t1y[g] = t1y[w * T + tid];
            a.t2x[g] = t2x[w * T + tid];
            a.t2y[g] = t2y[w * T + tid];
        }
    }
}

// The matrix and the vector/tune work are split over two warps per particle
// when both are requested (64 particles per block of 128 threads).
template <bool OCT, bool DO_M, bool DO_V, bool DO_T>
cudaError_t launch4(const FusedArgs &a, cudaStream_t s) {
    constexpr int threads = 128;
    constexpr bool split = DO_M && (DO_V || DO_T);
    constexpr int per_block = split ? threads / 2 : threads;  // particles
    const size_t slots = size_t(a.n_mb) + 2 * size_t(a.n_ly) + 4 * size_t(a.n_tu);
    const size_t tables = (size_t(a.n_mb) + a.n_ly + a.n_tu) * sizeof(WinEntry);
    const size_t smem = slots * per_block * sizeof(double) + tables;
    auto k = indicators_kernel<OCT, DO_M, DO_V, DO_T, split>;
    if (smem > 48 * 1024) {
        const cudaError_t e =
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
    }
    const unsigned blocks = unsigned((a.n + per_block - 1) / per_block);
    k<<<blocks, threads, smem, s>>>(a);
    return cudaGetLastError();
}

template <bool OCT>
cudaError_t launch_oct(const FusedArgs &a, cudaStream_t s) {
    const bool m = a.M != nullptr, v = a.V != nullptr, t = a.store_x != nullptr;
    if (m && v && t) return launch4<OCT, true, true, true>(a, s);
    if (m && v) return launch4<OCT, true, true, false>(a, s);
    if (m && t) return launch4<OCT, true, false, true>(a, s);
    if (v && t) return launch4<OCT, false, true, true>(a, s);
    if (m) return launch4<OCT, true, false, false>(a, s);
    if (v) return launch4<OCT, false, true, false>(a, s);
    if (t) return launch4<OCT, false, false, true>(a, s);
    return launch4<OCT, false, false, false>(a, s);
}

}  // namespace

size_t fused_max_slots() { return 96; }

cudaError_t launch_indicators(const FusedArgs &a, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    if (!isnan(a.kick_module) || a.inverse) {
        // whole-orbit MEGNO with kicks or backward turns
        if (a.M == nullptr || a.V != nullptr || a.store_x != nullptr || a.n_mb != 0 ||
            !a.df_before)
            return cudaErrorInvalidValue;
        const unsigned blocks = unsigned((a.n + 127) / 128);
        if (a.mu != 0.0)
            indicators_kernel<true, true, false, false, false, true><<<blocks, 128, 0, s>>>(a);
        else
            indicators_kernel<false, true, false, false, false, true><<<blocks, 128, 0, s>>>(a);
        return cudaGetLastError();
    }
    return a.mu != 0.0 ? launch_oct<true>(a, s) : launch_oct<false>(a, s);
}

}  // namespace hm
