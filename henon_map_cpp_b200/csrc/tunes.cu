// Tune estimates from turn-by-turn orbits (sm_100a).
//
// Orbits the caller stored (storage tunes) hold S snapshots of n particles
// per coordinate, laid out [sample][particle] (storage_4d_gpu's layout), so
// a warp reads 32 particles of one sample in one coalesced access:
// * mean_remove_kernel: subtracts each coordinate's orbit mean
//   (src/henon.cu:3040-3051);
// * birkhoff_kernel: Birkhoff-weighted phase advance over sample windows
//   (birkhoff_tune / birkhoff_tune_vec, src/dynamic_indicator.cpp:81-131,
//   198-253);
// * hann_gather_kernel + cuFFT + fft_peak_kernel: Hann-windowed spectrum of
//   x + i px and the interpolated peak (compute_fft, interpolation, A,
//   fft_tune_vec, src/dynamic_indicator.cpp:32-61, 134-196, 255-330).
// The tracker's own tune path (birkhoff_tunes / all_tunes,
// src/henon.cu:2890-3078) records the orbit itself, particle-major
// ([particle][sample] per coordinate: each particle's samples contiguous),
// with each coordinate's running sum and the first NaN sample, and then
// never rewrites it; the mean is subtracted as samples are read:
// * orbit_record_kernel: tracks n_turns turns and writes every state
//   (sample 0 = the start);
// * birkhoff_seg_kernel / birkhoff_finish_kernel: Birkhoff sums in segments
//   of turns over many threads;
// * fft_tune_kernel: one window's spectrum computed whole in one block's
//   shared memory, and its peak; windows too long for one block take
//   fft_gather2_kernel + cuFFT + fft_peak2_kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "hm_device.cuh"
#include "hm_internal.h"

namespace hm {
namespace {

using dev::Rn;

// Tracks n_turns turns and writes every state (sample 0 = the start).  The
// turn is the tracker's: forward with table[live_step + k], or backward with
// table[live_step - 1 - k] (REV), with the tracker's reproducible kicks
// (KICK: added before the forward turn, subtracted after the backward
// one).  Optionally each coordinate's sum over the samples (from 0.0, in
// sample order: the reference's std::accumulate for all_tunes' mean,
// src/henon.cu:3040-3051) and the first NaN sample.
// The orbit is particle-major, so a warp's samples of one turn would land
// in 32 different rows: each lane collects kRecGroup samples in shared
// memory and the warp then writes them out as whole 128-byte lines (lanes
// 0-15 one particle's run, lanes 16-31 the next).  Lanes past the last
// particle run the loop on zeros (a fixed point) and write nothing.
constexpr uint32_t kRecGroup = 16;

__host__ __device__ constexpr size_t record_smem_bytes(int threads) {
    return size_t(threads) * 4u * (kRecGroup + 1u) * sizeof(double);  // +1: bank padding
}

template <int ARITH, bool OCT, bool REV, bool KICK>
__global__ void orbit_record_kernel(OrbitRecordArgs a) {
    extern __shared__ double rec_stage[];  // [warp][coordinate][lane (kRecGroup + 1)]
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool valid = i < a.n;
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const size_t n = a.n, S = size_t(a.n_turns) + 1u;
    const size_t first_of_warp = i - lane;
    constexpr uint32_t G = kRecGroup, W = G + 1u;
    double *st = rec_stage + size_t(warp) * 4u * 32u * W;
    double x = 0.0, px = 0.0, y = 0.0, py = 0.0;
    uint32_t steps = 0;
    if (valid) {
        x = a.x[i];
        px = a.px[i];
        y = a.y[i];
        py = a.py[i];
        steps = a.steps[i];
    }
    bool alive = valid && !dev::is_lost(x, px, y, py);
    uint32_t first_nan = alive ? a.n_turns + 1u : 0u;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    const bool sums = a.sums != nullptr;
    // Sample s of this lane into the stage; the warp writes a full group
    // (or the last, partial one) out.
    auto put = [&](uint32_t s) {
        const uint32_t g = s % G;
        st[0 * 32u * W + lane * W + g] = x;
        st[1 * 32u * W + lane * W + g] = px;
        st[2 * 32u * W + lane * W + g] = y;
        st[3 * 32u * W + lane * W + g] = py;
        if (sums) {
            s0 = Rn::add(s0, x);
            s1 = Rn::add(s1, px);
            s2 = Rn::add(s2, y);
            s3 = Rn::add(s3, py);
        }
        if (g == G - 1u || s == a.n_turns) {
            __syncwarp();
            const uint32_t base = s - g, cnt = g + 1u;
#pragma unroll
            for (uint32_t v = lane; v < 32u * G; v += 32u) {
                const uint32_t pl = v / G, gg = v % G;
                const size_t ip = first_of_warp + pl;
                if (gg < cnt && ip < n) {
                    const size_t o = ip * S + base + gg;
                    a.ox[o] = st[0 * 32u * W + pl * W + gg];
                    a.opx[o] = st[1 * 32u * W + pl * W + gg];
                    a.oy[o] = st[2 * 32u * W + pl * W + gg];
                    a.opy[o] = st[3 * 32u * W + pl * W + gg];
                }
            }
            __syncwarp();
        }
    };
    put(0);
    dev::Particle p = dev::make_particle(x, px, y, py);
    const dev::Barrier bar = dev::make_barrier<ARITH>(a.b2bits);
    const unsigned long long id = a.id0 + i;
    // The next turn's record is loaded a turn ahead, off the orbit's chain.
    auto table_index = [&](uint32_t k) { return REV ? a.live_step - 1u - k : a.live_step + k; };
    dev::Turn t_next = a.n_turns ? dev::load_turn(a.table, table_index(0)) : dev::Turn{};
    for (uint32_t k = 0; k < a.n_turns; ++k) {
        const dev::Turn t = t_next;
        if (k + 1 < a.n_turns) t_next = dev::load_turn(a.table, table_index(k + 1));
        if (alive) {
            const uint32_t idx = table_index(k);
            if (KICK && !REV)
                dev::apply_kick<false>(p, dev::kick_direction(a.kick_seed, id, idx), a.kick_module);
            dev::turn<ARITH, OCT, REV>(p, t, a.mu);
            if (KICK && REV)
                dev::apply_kick<true>(p, dev::kick_direction(a.kick_seed, id, idx), a.kick_module);
            if (dev::inside_after_turn<ARITH>(p, bar)) {
                steps = REV ? steps - 1u : steps + 1u;
                x = p.x;
                px = p.px;
                y = p.y;
                py = p.py;
            } else {
                x = px = y = py = dev::quiet_nan();
                alive = false;
                first_nan = k + 1u;
            }
        }
        put(k + 1u);
    }
    if (!valid) return;
    a.x[i] = x;
    a.px[i] = px;
    a.y[i] = y;
    a.py[i] = py;
    a.steps[i] = steps;
    if (sums) {
        a.sums[i] = s0;
        a.sums[n + i] = s1;
        a.sums[2 * n + i] = s2;
        a.sums[3 * n + i] = s3;
    }
    // With the mean removed, one NaN sample makes the mean, and so every
    // sample, NaN.
    if (sums && first_nan <= a.n_turns) first_nan = 0u;
    if (a.first_nan) a.first_nan[i] = first_nan;
}

__device__ double interp_a(double a, double b, double c);

// mean = sum / samples, as the reference divides std::accumulate's result.
__device__ __forceinline__ double mean_of(const double *means, size_t n, size_t i, int c,
                                          size_t S) {
    return means ? Rn::div(means[size_t(c) * n + i], double(S)) : 0.0;
}

// v - mean, separately rounded (the reference subtracts the mean from every
// stored sample); without a mean the sample itself.
__device__ __forceinline__ double centred(double v, const double *means, double m) {
    return means ? Rn::sub(v, m) : v;
}

// Birkhoff phase-advance sums of one segment of turns [s0, s1) for one plane
// of one particle, every window at once: the transition s -> s+1 adds
// w_j[s - from_j] dtheta_s to window j when from_j <= s < to_j, dtheta
// wrapped by +2 pi when negative (birkhoff_tune,
// src/dynamic_indicator.cpp:81-131).  Windows in groups of kWinGroup
// (blockIdx.y) so that the sums stay in registers.
constexpr int kWinGroup = 8;

__global__ void birkhoff_seg_kernel(const BirkhoffSegArgs a) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t n = a.n;
    const size_t sp = t / n;  // segment * 2 + plane
    if (sp >= 2u * size_t(a.n_seg)) return;
    const size_t i = t - sp * n;
    const uint32_t seg = uint32_t(sp >> 1);
    const int plane = int(sp & 1u);
    const int w0 = int(blockIdx.y) * kWinGroup;
    const int nw = min(kWinGroup, a.n_win - w0);
    const double *q = plane ? a.y : a.x, *p = plane ? a.py : a.px;
    const double mq = mean_of(a.means, n, i, 2 * plane, a.S);
    const double mp = mean_of(a.means, n, i, 2 * plane + 1, a.S);
    const uint32_t s0 = seg * a.seg_len;
    const uint32_t s1 = min(uint32_t(a.S - 1), s0 + a.seg_len);
    uint32_t lo[kWinGroup], hi[kWinGroup];
    long long wb[kWinGroup];  // weight of transition s: w[wb + s]
    double acc[kWinGroup];
#pragma unroll
    for (int j = 0; j < kWinGroup; ++j) {
        acc[j] = 0.0;
        lo[j] = 1u;  // empty window
        hi[j] = 0u;
        wb[j] = 0;
        if (j < nw) {
            lo[j] = a.from[w0 + j];
            hi[j] = a.to[w0 + j];
            wb[j] = (long long)a.w_off[w0 + j] - (long long)lo[j];
        }
    }
    const size_t row = i * a.S;  // this particle's samples
    double prev = atan2(centred(p[row + s0], a.means, mp), centred(q[row + s0], a.means, mq));
    for (uint32_t s = s0; s < s1; ++s) {
        const size_t o = row + s + 1u;
        const double th = atan2(centred(p[o], a.means, mp), centred(q[o], a.means, mq));
        double d = Rn::sub(th, prev);
        if (d < 0.0) d = Rn::add(d, 2.0 * M_PI);
        prev = th;
#pragma unroll
        for (int j = 0; j < kWinGroup; ++j)
            if (s >= lo[j] && s < hi[j]) acc[j] = Rn::add(acc[j], Rn::mul(a.w[wb[j] + s], d));
    }
#pragma unroll
    for (int j = 0; j < kWinGroup; ++j)
        if (j < nw)
            a.partial[((size_t(w0 + j) * 2 + plane) * a.n_seg + seg) * n + i] = acc[j];
}

// 1 - (sum of the segments' sums, in segment order) / (2 pi); NaN for a
// window marked check_nan that holds a NaN sample (birkhoff_tune_vec checks
// the caller's windows, not the appended full orbit).
__global__ void birkhoff_finish_kernel(const BirkhoffSegArgs a) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t n = a.n;
    const size_t wp = t / n;  // window * 2 + plane
    if (wp >= 2u * size_t(a.n_win)) return;
    const size_t i = t - wp * n;
    const int j = int(wp >> 1), plane = int(wp & 1u);
    const double *part = a.partial + (size_t(j) * 2 + plane) * a.n_seg * n + i;
    double sum = 0.0;
    for (uint32_t g = 0; g < a.n_seg; ++g) sum = Rn::add(sum, part[size_t(g) * n]);
    double tune = Rn::sub(1.0, Rn::div(sum, Rn::mul(2.0, M_PI)));
    if (a.check_nan[j] && a.first_nan[i] <= a.to[j]) tune = dev::quiet_nan();
    a.out[i * a.cols + 2 * size_t(a.out_col[j]) + plane] = tune;
}

// Hann window 2 sin^2(pi k / len) (compute_fft, src/dynamic_indicator.cpp:
// 32-61), the same expression as hann_gather_kernel's.
__global__ void hann_table_kernel(double *h, uint32_t len) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= len) return;
    const double s = sin(M_PI * double(k) / double(len));
    h[k] = 2 * pow(s, 2);
}

// z[plane n + i][k] = ((q - mean) + i (p - mean)) h_k over the window's
// samples from .. from + len - 1: one row of len values per column (plane,
// particle), cuFFT's native batch layout.  The orbit's samples are
// contiguous per particle, so rows are read and written along samples.
__global__ void __launch_bounds__(256) fft_gather2_kernel(const double *x, const double *px,
                                                          const double *y, const double *py,
                                                          const double *means, size_t n,
                                                          uint32_t from, uint32_t len,
                                                          const double *h, double2 *z, size_t S,
                                                          int plane) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n * len) return;
    const size_t i = t / len;
    const uint32_t k = uint32_t(t - i * len);
    const double *q = plane ? y : x, *p = plane ? py : px;
    const double mq = mean_of(means, n, i, 2 * plane, S);
    const double mp = mean_of(means, n, i, 2 * plane + 1, S);
    const size_t o = i * S + from + k;
    const double re = centred(q[o], means, mq), im = centred(p[o], means, mp);
    const double hk = h[k];
    z[(size_t(plane) * n + i) * len + k] = make_double2(re * hk, im * hk);
}

// One warp per column (plane, particle): first maximum of |z_k| over k
// (lanes stride the row, then a shuffle reduction keeping the smallest k
// among equal maxima), then the interpolation of
// src/dynamic_indicator.cpp:139-176 -> |1 - v|; NaN when the window's
// samples from .. last_sample hold a NaN.
__global__ void fft_peak2_kernel(const double2 *z, uint32_t len, size_t n, uint32_t last_sample,
                                 const uint32_t *first_nan, double *out, size_t out_cols,
                                 int col) {
    const size_t c = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32;
    const unsigned lane = threadIdx.x & 31u;
    if (c >= 2 * n) return;
    const int plane = c >= n ? 1 : 0;
    const size_t i = c - size_t(plane) * n;
    const double2 *row = z + c * len;
    auto mag = [&](uint32_t k) {
        const double2 v = row[k];
        return sqrt(v.x * v.x + v.y * v.y);
    };
    const bool nan = first_nan[i] <= last_sample;
    double best = -1.0;
    uint32_t best_k = 0xffffffffu;
    if (!nan) {
        for (uint32_t k = lane; k < len; k += 32) {
            const double m = mag(k);
            if (m > best) {  // k grows within a lane: the first maximum is kept
                best = m;
                best_k = k;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(dev::kFullMask, best, o);
        const uint32_t ok = __shfl_down_sync(dev::kFullMask, best_k, o);
        if (ob > best || (ob == best && ok < best_k)) {
            best = ob;
            best_k = ok;
        }
    }
    if (lane != 0) return;
    double value;
    if (nan) {
        value = dev::quiet_nan();
    } else {
        uint32_t index = best_k;
        const double N = double(len);
        if (index == 0) {
            value = 1.0;
        } else if (index == len - 1) {
            value = 0.0;
        } else {
            uint32_t i1, i2;
            if (mag(index - 1) > mag(index + 1)) {
                i1 = index - 1;
                i2 = index;
                index = index - 1;
            } else {
                i1 = index;
                i2 = index + 1;
            }
            const double v = (double(index) / N) +
                             (1.0 / (2.0 * M_PI)) *
                                 asin(interp_a(mag(i1), mag(i2), cos(2.0 * M_PI / N)) *
                                      sin(2.0 * M_PI / N));
            value = fabs(1.0 - v);
        }
    }
    out[i * out_cols + 2 * size_t(col) + plane] = value;
}

// v -= mean(v) per particle and coordinate, one thread per (coordinate,
// particle), particles fastest; the mean is the left-to-right sum from 0.0
// divided by the sample count (std::accumulate / size).
__global__ void mean_remove_kernel(double *x, double *px, double *y, double *py, size_t n,
                                   size_t S) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t q = t / n;  // coordinate
    if (q >= 4u) return;
    const size_t i = t - q * n;
    double *c = q == 0u ? x : q == 1u ? px : q == 2u ? y : py;
    double s = 0.0;
#pragma unroll 8
    for (size_t k = 0; k < S; ++k) s = Rn::add(s, c[k * n + i]);
    const double m = Rn::div(s, double(S));
#pragma unroll 8
    for (size_t k = 0; k < S; ++k) c[k * n + i] = Rn::sub(c[k * n + i], m);
}

// Birkhoff tune over samples [from, to] of (q, p): 1 - sum_i w_i dtheta_i /
// (2 pi), dtheta wrapped by +2pi when negative, w = birkhoff_weights(to -
// from); NaN when check_nan and any sample of the window is NaN.
// Birkhoff tune of one plane over samples [from, to] of particle i; *has_nan
// reports a NaN in any of the four coordinates of the window (q, p of this
// plane and o1, o2 of the other).  The sample loads do not depend on the
// running sum, so the loop is unrolled to keep several in flight.
__device__ double birkhoff_window(const double *q, const double *p, const double *o1,
                                  const double *o2, size_t n, size_t i, uint32_t from,
                                  uint32_t to, const double *w, bool *has_nan) {
    double sum = 0.0;
    bool nan_seen = false;
    const size_t f = size_t(from) * n + i;
    double prev = atan2(p[f], q[f]);
    nan_seen |= isnan(q[f]) || isnan(p[f]) || isnan(o1[f]) || isnan(o2[f]);
#pragma unroll 4
    for (uint32_t s = from; s < to; ++s) {
        const size_t o = size_t(s + 1) * n + i;
        const double qq = q[o], pp = p[o];
        nan_seen |= isnan(qq) || isnan(pp) || isnan(o1[o]) || isnan(o2[o]);
        const double th = atan2(pp, qq);
        double d = Rn::sub(th, prev);
        if (d < 0.0) d = Rn::add(d, 2.0 * M_PI);
        sum = Rn::add(sum, Rn::mul(w[s - from], d));
        prev = th;
    }
    *has_nan = nan_seen;
    return Rn::sub(1.0, Rn::div(sum, Rn::mul(2.0, M_PI)));
}

// One thread per (window, plane, particle), particles fastest: a warp
// walks one window of one plane for 32 consecutive particles (coalesced
// loads, no divergence between windows of different lengths), and for few
// particles the windows and planes supply the parallelism.
__global__ void birkhoff_kernel(const double *x, const double *px, const double *y,
                                const double *py, size_t n, const uint32_t *from,
                                const uint32_t *to, const uint64_t *w_off, const double *w,
                                int n_win, double *out) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t wp = t / n;  // window * 2 + plane
    if (wp >= 2u * size_t(n_win)) return;
    const size_t i = t - wp * n;
    const int j = int(wp >> 1);
    const bool plane_y = (wp & 1u) != 0u;
    bool nan_seen = false;
    double tune = plane_y ? birkhoff_window(y, py, x, px, n, i, from[j], to[j], w + w_off[j], &nan_seen)
                          : birkhoff_window(x, px, y, py, n, i, from[j], to[j], w + w_off[j], &nan_seen);
    // birkhoff_tune_vec checks all four coordinates of the window for the
    // windows it was given, not for the appended full orbit.
    const bool is_full = j == n_win - 1;
    if (!is_full && nan_seen) tune = dev::quiet_nan();
    out[i * size_t(2 * n_win) + 2 * size_t(j) + (plane_y ? 1u : 0u)] = tune;
}

// z_k = (x + i px)[from + k] * 2 sin^2(pi k / len) for one window, one row
// of len complex values per particle; nan_flags[i] set when any sample of
// the window is NaN.
__global__ void hann_gather_kernel(const double *q, const double *p, size_t n, uint32_t from,
                                   uint32_t len, size_t first, size_t count, double2 *buf,
                                   int *nan_flags) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= count * len) return;
    const size_t r = t / len, k = t % len;
    const size_t i = first + r;
    const double re = q[size_t(from + k) * n + i], im = p[size_t(from + k) * n + i];
    if (isnan(re) || isnan(im)) nan_flags[r] = 1;
    const double s = sin(M_PI * double(k) / double(len));
    const double h = 2 * pow(s, 2);
    buf[r * len + k] = make_double2(re * h, im * h);
}

// A(a, b, c) of the peak interpolation (src/dynamic_indicator.cpp:134-137).
__device__ double interp_a(double a, double b, double c) {
    return (-(a + b * c) * (a - b) +
            b * sqrt(pow(c, 2) * pow((a + b), 2) - 2 * a * b * (2 * pow(c, 2) - c - 1))) /
           (pow(a, 2) + pow(b, 2) + 2 * a * b * c);
}

// One warp per particle: argmax of |FFT| (first maximum), then the
// interpolation of src/dynamic_indicator.cpp:139-176 -> |1 - value|.
__global__ void fft_peak_kernel(const double2 *buf, uint32_t len, size_t count,
                                const int *nan_flags, double *out, size_t out_stride,
                                size_t first) {
    const size_t warp = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32;
    const unsigned lane = threadIdx.x & 31u;
    if (warp >= count) return;
    const double2 *row = buf + warp * len;
    double best = -1.0;
    uint32_t best_k = 0xffffffffu;
    for (uint32_t k = lane; k < len; k += 32) {
        const double2 z = row[k];
        const double m = sqrt(z.x * z.x + z.y * z.y);
        if (m > best || (m == best && k < best_k)) {
            best = m;
            best_k = k;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(dev::kFullMask, best, o);
        const uint32_t ok = __shfl_down_sync(dev::kFullMask, best_k, o);
        if (ob > best || (ob == best && ok < best_k)) {
            best = ob;
            best_k = ok;
        }
    }
    if (lane != 0) return;
    double value;
    if (nan_flags[warp]) {
        value = dev::quiet_nan();
    } else {
        uint32_t index = best_k;
        const double N = double(len);
        auto mag = [&](uint32_t k) {
            const double2 z = row[k];
            return sqrt(z.x * z.x + z.y * z.y);
        };
        if (index == 0) {
            value = 1.0;
        } else if (index == len - 1) {
            value = 0.0;
        } else {
            uint32_t i1, i2;
            if (mag(index - 1) > mag(index + 1)) {
                i1 = index - 1;
                i2 = index;
                index = index - 1;
            } else {
                i1 = index;
                i2 = index + 1;
            }
            const double v = (double(index) / N) +
                             (1.0 / (2.0 * M_PI)) *
                                 asin(interp_a(mag(i1), mag(i2), cos(2.0 * M_PI / N)) *
                                      sin(2.0 * M_PI / N));
            value = fabs(1.0 - v);
        }
    }
    out[(first + warp) * out_stride] = value;
}

// ---- FFT tunes in shared memory --------------------------------------------------
// One block per row (plane, particle) of one window: the samples are read
// from the orbit (mean subtracted, Hann window applied) into shared memory,
// transformed there, and the block writes the interpolated peak.  The
// transform of length M is an in-place mixed-radix network of radices 2, 3,
// 4, 5 and 8.  Forward, decimation in frequency: stage s splits each block of
// N = r * span values (radix r) into r butterflies of stride `span`,
//     y_k = sum_q x_q w_r^{qk},  stored times w_N^{jk} (j: offset in the span),
// which takes natural order in and leaves X_k at a digit-reversed position
// (FftPlanDev::pos).  The inverse network runs the stages backwards with
// conjugate twiddles applied before each butterfly (decimation in time),
// which takes that order back to natural order (times M).  A window whose
// length has no prime factor above 5 is transformed directly (M = L): its
// samples, conjugated, are loaded at the forward network's positions, and
// the inverse network returns conj(X_k) in natural order.  Other lengths
// take Bluestein's convolution (L. Bluestein, "A linear filtering approach to the
// computation of the discrete Fourier transform", IEEE Trans. Audio
// Electroacoust. 18 (1970) 451-455), which uses both networks:
//     X_k = c_k sum_n (z_n c_n) conj(c_{k-n}),  c_n = exp(-i pi n^2 / L),
// the cyclic convolution of length M >= 2L - 1 being the inverse network of
// the pointwise product of the forward network's outputs (that of b_m =
// conj(c_m) is precomputed, in the same order).  |c_k| = 1 and the peak
// interpolation depends on magnitude ratios only, so the peak is taken on
// |conv_k| directly.

__device__ __forceinline__ double2 c_add(double2 a, double2 b) {
    return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 c_sub(double2 a, double2 b) {
    return make_double2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ double2 c_mul(double2 a, double2 b) {  // a b
    return make_double2(fma(a.x, b.x, -(a.y * b.y)), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 c_mulc(double2 a, double2 b) {  // a conj(b)
    return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -(a.x * b.y)));
}
__device__ __forceinline__ double2 c_i(double2 a) {  // i a
    return make_double2(-a.y, a.x);
}

// Shared-memory slots of a row: M rounded up to a multiple of 8.
__host__ __device__ __forceinline__ uint32_t fft_row_slots(const FftPlanDev &pl) {
    return (pl.M + 7u) & ~7u;
}

// exp(-2 pi i t / M) from the two shared-memory tables (t < M).
__device__ __forceinline__ double2 fft_twiddle(const double2 *coarse, const double2 *fine,
                                               uint32_t t) {
    return c_mul(coarse[t >> 6], fine[t & 63u]);
}

// The DFT of R values in registers (R = 2, 3, 4, 5, 8), forward
// (w = exp(-2 pi i / R)) or inverse (conjugate w).
template <bool INV>
__device__ __forceinline__ void dft4(double2 &x0, double2 &x1, double2 &x2, double2 &x3) {
    const double2 t0 = c_add(x0, x2), t1 = c_sub(x0, x2);
    const double2 t2 = c_add(x1, x3), t3 = c_sub(x1, x3);
    const double2 it3 = c_i(t3);
    x0 = c_add(t0, t2);
    x2 = c_sub(t0, t2);
    x1 = INV ? c_add(t1, it3) : c_sub(t1, it3);
    x3 = INV ? c_sub(t1, it3) : c_add(t1, it3);
}

template <int R, bool INV>
__device__ __forceinline__ void dft_small(double2 (&v)[R]) {
    if constexpr (R == 2) {
        const double2 a = v[0], b = v[1];
        v[0] = c_add(a, b);
        v[1] = c_sub(a, b);
    } else if constexpr (R == 4) {
        dft4<INV>(v[0], v[1], v[2], v[3]);
    } else if constexpr (R == 8) {
        // even and odd halves, then X_k = E_k + w8^k O_k, X_{k+4} = E_k - w8^k O_k
        double2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
        double2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
        dft4<INV>(e0, e1, e2, e3);
        dft4<INV>(o0, o1, o2, o3);
        constexpr double h = 0.70710678118654752440;  // sqrt(2) / 2
        // w8 o1, w8^2 o2, w8^3 o3 (forward w8 = h (1 - i); inverse h (1 + i))
        const double2 p1 = INV ? make_double2(h * (o1.x - o1.y), h * (o1.x + o1.y))
                               : make_double2(h * (o1.x + o1.y), h * (o1.y - o1.x));
        const double2 p2 = INV ? c_i(o2) : make_double2(o2.y, -o2.x);
        const double2 p3 = INV ? make_double2(-h * (o3.x + o3.y), h * (o3.x - o3.y))
                               : make_double2(h * (o3.y - o3.x), -h * (o3.x + o3.y));
        v[0] = c_add(e0, o0);
        v[4] = c_sub(e0, o0);
        v[1] = c_add(e1, p1);
        v[5] = c_sub(e1, p1);
        v[2] = c_add(e2, p2);
        v[6] = c_sub(e2, p2);
        v[3] = c_add(e3, p3);
        v[7] = c_sub(e3, p3);
    } else if constexpr (R == 5) {
        // cos(2 pi / 5), cos(4 pi / 5), sin(2 pi / 5), sin(4 pi / 5)
        constexpr double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
        constexpr double s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;
        const double2 x0 = v[0];
        const double2 t1 = c_add(v[1], v[4]), t2 = c_add(v[2], v[3]);
        const double2 u1 = c_sub(v[1], v[4]), u2 = c_sub(v[2], v[3]);
        v[0] = c_add(x0, c_add(t1, t2));
        const double2 a1 = make_double2(fma(c2, t2.x, fma(c1, t1.x, x0.x)),
                                        fma(c2, t2.y, fma(c1, t1.y, x0.y)));
        const double2 a2 = make_double2(fma(c1, t2.x, fma(c2, t1.x, x0.x)),
                                        fma(c1, t2.y, fma(c2, t1.y, x0.y)));
        const double2 ib1 = c_i(make_double2(fma(s1, u1.x, s2 * u2.x), fma(s1, u1.y, s2 * u2.y)));
        const double2 ib2 = c_i(make_double2(fma(s2, u1.x, -(s1 * u2.x)),
                                             fma(s2, u1.y, -(s1 * u2.y))));
        v[1] = INV ? c_add(a1, ib1) : c_sub(a1, ib1);
        v[4] = INV ? c_sub(a1, ib1) : c_add(a1, ib1);
        v[2] = INV ? c_add(a2, ib2) : c_sub(a2, ib2);
        v[3] = INV ? c_sub(a2, ib2) : c_add(a2, ib2);
    } else {
        static_assert(R == 3, "radix");
        constexpr double s = 0.86602540378443864676;  // sin(2 pi / 3)
        const double2 x0 = v[0];
        const double2 t = c_add(v[1], v[2]), u = c_sub(v[1], v[2]);
        v[0] = c_add(x0, t);
        const double2 a = make_double2(fma(-0.5, t.x, x0.x), fma(-0.5, t.y, x0.y));
        const double2 ib = c_i(make_double2(s * u.x, s * u.y));
        v[1] = INV ? c_add(a, ib) : c_sub(a, ib);
        v[2] = INV ? c_sub(a, ib) : c_add(a, ib);
    }
}

// Shared-memory slot of row value i: with SWZ the low three bits of i (its
// place among 8 consecutive values, one 128-byte bank row of double2) are
// XORed with the next three, so that the small strides of the last stages
// (radices 8, 4, 2 run last) fall into different banks.  A bijection on
// every aligned group of 8, so rows of a multiple of 8 values stay in place.
template <bool SWZ>
__device__ __forceinline__ uint32_t slot(uint32_t i) {
    return SWZ ? (i ^ ((i >> 3) & 7u)) : i;
}

// w^k for k < 8 from w, w^2 and w^4 (at most two products deep).
__device__ __forceinline__ double2 twiddle_pow(int k, double2 w1, double2 w2, double2 w4) {
    switch (k) {
        case 1: return w1;
        case 2: return w2;
        case 3: return c_mul(w1, w2);
        case 4: return w4;
        case 5: return c_mul(w1, w4);
        case 6: return c_mul(w2, w4);
        default: return c_mul(c_mul(w1, w2), w4);
    }
}

// One stage of radix R over row[0, M): butterfly b (b < M / R) covers
// block b / span at offset j = b % span; the twiddles w_N^{jk}, N = R span,
// are exp(-2 pi i j k prod / M) = w^k with w from the tables.  Forward:
// butterfly, then twiddles; inverse: conjugate twiddles, then the inverse
// butterfly.  A stage of span 1 has j = 0 and no twiddles (TW false).
template <int R, bool INV, bool SWZ, bool TW>
__device__ __forceinline__ void fft_stage(double2 *row, uint32_t M, uint32_t span, uint32_t prod,
                                          const double2 *tc, const double2 *tf) {
    const uint32_t nb = M / R, T = blockDim.x;
    uint32_t blk = threadIdx.x / span, j = threadIdx.x - blk * span;
    const uint32_t dq = T / span, dr = T - dq * span;
    constexpr int kUnroll = R >= 8 ? 1 : 2;  // radix 8 fills the registers alone
#pragma unroll kUnroll
    for (uint32_t b = threadIdx.x; b < nb; b += T) {
        const uint32_t base = blk * span * R + j;
        double2 w1 = make_double2(1.0, 0.0), w2 = w1, w4 = w1;
        if (TW) {
            w1 = fft_twiddle(tc, tf, j * prod);
            w2 = c_mul(w1, w1);
            w4 = c_mul(w2, w2);
        }
        double2 v[R];
        if (!INV) {
#pragma unroll
            for (int q = 0; q < R; ++q) v[q] = row[slot<SWZ>(base + q * span)];
            dft_small<R, false>(v);
#pragma unroll
            for (int k = 0; k < R; ++k)
                row[slot<SWZ>(base + k * span)] =
                    (TW && k > 0) ? c_mul(v[k], twiddle_pow(k, w1, w2, w4)) : v[k];
        } else {
#pragma unroll
            for (int q = 0; q < R; ++q) {
                const double2 x = row[slot<SWZ>(base + q * span)];
                v[q] = (TW && q > 0) ? c_mulc(x, twiddle_pow(q, w1, w2, w4)) : x;
            }
            dft_small<R, true>(v);
#pragma unroll
            for (int k = 0; k < R; ++k) row[slot<SWZ>(base + k * span)] = v[k];
        }
        blk += dq;
        j += dr;
        if (j >= span) {
            j -= span;
            ++blk;
        }
    }
}

template <int R, bool INV, bool SWZ>
__device__ __forceinline__ void fft_stage_any(double2 *row, uint32_t M, uint32_t span,
                                              uint32_t prod, const double2 *tc,
                                              const double2 *tf) {
    if (span == 1) fft_stage<R, INV, SWZ, false>(row, M, span, prod, tc, tf);
    else fft_stage<R, INV, SWZ, true>(row, M, span, prod, tc, tf);
}

// The forward (decimation in frequency) or inverse (decimation in time)
// network in place over the row; the caller synchronises before.
template <bool INV, bool SWZ>
__device__ void fft_network(double2 *row, const FftPlanDev &pl, const double2 *tc,
                            const double2 *tf) {
    for (int t = 0; t < pl.n_stages; ++t) {
        const int s = INV ? pl.n_stages - 1 - t : t;
        const uint32_t span = pl.stage_len[s], prod = pl.stage_prod[s];
        switch (pl.radix[s]) {
            case 8: fft_stage_any<8, INV, SWZ>(row, pl.M, span, prod, tc, tf); break;
            case 4: fft_stage_any<4, INV, SWZ>(row, pl.M, span, prod, tc, tf); break;
            case 2: fft_stage_any<2, INV, SWZ>(row, pl.M, span, prod, tc, tf); break;
            case 5: fft_stage_any<5, INV, SWZ>(row, pl.M, span, prod, tc, tf); break;
            default: fft_stage_any<3, INV, SWZ>(row, pl.M, span, prod, tc, tf); break;
        }
        __syncthreads();
    }
}

constexpr int kFftThreadsMax = 1024;

template <bool SWZ>
__global__ void __launch_bounds__(kFftThreadsMax) fft_tune_kernel(const FftTuneArgs a) {
    extern __shared__ __align__(16) double2 fft_sm[];
    __shared__ double red_m[kFftThreadsMax / 32];
    __shared__ uint32_t red_k[kFftThreadsMax / 32];
    const FftPlanDev &pl = a.plan;
    double2 *row = fft_sm;
    double2 *tc = row + fft_row_slots(pl);
    double2 *tf = tc + pl.n_coarse;
    const size_t rix = blockIdx.x;  // plane * n + particle
    const int plane = rix >= a.n ? 1 : 0;
    const size_t i = rix - size_t(plane) * a.n;
    // Only one or a few rows fit in an SM's shared memory, so a block's
    // reads would not overlap other rows' transforms: each block asks L2 for
    // the window of the row that starts about one wave of resident blocks
    // later (prefetch.global.L2, one per 128-byte line, addresses within
    // the row).
    if (a.stride_s == 1) {  // rows contiguous
        const size_t r2 = rix + a.prefetch_ahead;
        if (r2 < 2 * a.n) {
            const int plane2 = r2 >= a.n ? 1 : 0;
            const size_t i2 = r2 - size_t(plane2) * a.n;
            const size_t bytes = size_t(pl.L) * sizeof(double);
            const size_t o2 = i2 * a.stride_i + a.from;
            const char *rq = reinterpret_cast<const char *>((plane2 ? a.y : a.x) + o2);
            const char *rp = reinterpret_cast<const char *>((plane2 ? a.py : a.px) + o2);
            const uint32_t lines = uint32_t((bytes + 127u) / 128u) + 1u;
            for (uint32_t l = threadIdx.x; l < 2u * lines; l += blockDim.x) {
                const size_t off = min(size_t(l % lines) * 128u, bytes - sizeof(double));
                const char *ptr = (l < lines ? rq : rp) + off;
                asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr));
            }
        }
    }
    if (a.first_nan && a.first_nan[i] <= a.last_sample) {  // a NaN sample in the window: NaN tune
        if (threadIdx.x == 0)
            for (int c = 0; c < a.n_out_cols; ++c)
                a.out[i * a.cols + 2 * size_t(a.out_cols[c]) + plane] = dev::quiet_nan();
        return;
    }
    for (uint32_t t = threadIdx.x; t < pl.n_coarse; t += blockDim.x) tc[t] = pl.tw_coarse[t];
    for (uint32_t t = threadIdx.x; t < 64u; t += blockDim.x) tf[t] = pl.tw_fine[t];
    const double *q = plane ? a.y : a.x, *p = plane ? a.py : a.px;
    const double mq = mean_of(a.means, a.n, i, 2 * plane, a.S);
    const double mp = mean_of(a.means, a.n, i, 2 * plane + 1, a.S);
    // z_k = ((q - mean) + i (p - mean)) h_k.  Bluestein: z_k c_k in natural
    // order (zeros up to M) for the forward network.  Direct: conj(z_k) at
    // the forward network's position of k, so that the inverse network
    // gives conj(X_k) in natural order (the magnitudes are those of X_k).
    const size_t o0 = i * a.stride_i + size_t(a.from) * a.stride_s;
    int nan_seen = 0;
#pragma unroll 4
    for (uint32_t k = threadIdx.x; k < pl.M; k += blockDim.x) {
        double2 v = make_double2(0.0, 0.0);
        if (k < pl.L) {
            const size_t o = o0 + size_t(k) * a.stride_s;
            const double re = centred(q[o], a.means, mq), im = centred(p[o], a.means, mp);
            nan_seen |= isnan(re) || isnan(im);
            const double hk = a.hann[k];
            v = make_double2(re * hk, im * hk);
            if (pl.bluestein) v = c_mul(v, pl.chirp[k]);
            else v.y = -v.y;
        }
        row[slot<SWZ>(pl.bluestein ? k : pl.pos[k])] = v;
    }
    // Without first-NaN records the window's own samples decide
    // (fft_tune_vec's rule, scanning the window).
    if (__syncthreads_or(a.first_nan == nullptr && nan_seen)) {
        if (threadIdx.x == 0)
            for (int c = 0; c < a.n_out_cols; ++c)
                a.out[i * a.cols + 2 * size_t(a.out_cols[c]) + plane] = dev::quiet_nan();
        return;
    }
    if (pl.bluestein) {
        fft_network<false, SWZ>(row, pl, tc, tf);
        for (uint32_t k = threadIdx.x; k < pl.M; k += blockDim.x)
            row[slot<SWZ>(k)] = c_mul(row[slot<SWZ>(k)], pl.bhat[k]);
        __syncthreads();
    }
    fft_network<true, SWZ>(row, pl, tc, tf);
    auto at = [&](uint32_t k) { return row[slot<SWZ>(k)]; };
    // First maximum of |X_k| (squared, monotone) over k < L; k grows within
    // a thread, and ties across threads keep the smallest k.
    double best = -1.0;
    uint32_t best_k = 0xffffffffu;
    for (uint32_t k = threadIdx.x; k < pl.L; k += blockDim.x) {
        const double2 v = at(k);
        const double m2 = v.x * v.x + v.y * v.y;
        if (m2 > best) {
            best = m2;
            best_k = k;
        }
    }
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(dev::kFullMask, best, o);
        const uint32_t ok = __shfl_down_sync(dev::kFullMask, best_k, o);
        if (ob > best || (ob == best && ok < best_k)) {
            best = ob;
            best_k = ok;
        }
    }
    if (lane == 0) {
        red_m[warp] = best;
        red_k[warp] = best_k;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (unsigned w = 1; w < blockDim.x / 32u; ++w)
        if (red_m[w] > best || (red_m[w] == best && red_k[w] < best_k)) {
            best = red_m[w];
            best_k = red_k[w];
        }
    auto mag = [&](uint32_t k) {
        const double2 v = at(k);
        return sqrt(v.x * v.x + v.y * v.y);
    };
    // interpolation (src/dynamic_indicator.cpp:139-176), as fft_peak2_kernel
    const uint32_t len = pl.L;
    double value;
    uint32_t index = best_k;
    const double N = double(len);
    if (index == 0 || index >= len) {
        value = 1.0;
    } else if (index == len - 1) {
        value = 0.0;
    } else {
        uint32_t i1, i2;
        if (mag(index - 1) > mag(index + 1)) {
            i1 = index - 1;
            i2 = index;
            index = index - 1;
        } else {
            i1 = index;
            i2 = index + 1;
        }
        const double v = (double(index) / N) +
                         (1.0 / (2.0 * M_PI)) *
                             asin(interp_a(mag(i1), mag(i2), cos(2.0 * M_PI / N)) *
                                  sin(2.0 * M_PI / N));
        value = fabs(1.0 - v);
    }
    for (int c = 0; c < a.n_out_cols; ++c)
        a.out[i * a.cols + 2 * size_t(a.out_cols[c]) + plane] = value;
}

template <int ARITH, bool OCT>
void launch_record_ok(const OrbitRecordArgs &a, unsigned blocks, int threads, cudaStream_t s) {
    const bool kick = !isnan(a.kick_module);
    const size_t smem = record_smem_bytes(threads);
    if (a.inverse) {
        if (kick) orbit_record_kernel<ARITH, OCT, true, true><<<blocks, threads, smem, s>>>(a);
        else orbit_record_kernel<ARITH, OCT, true, false><<<blocks, threads, smem, s>>>(a);
    } else {
        if (kick) orbit_record_kernel<ARITH, OCT, false, true><<<blocks, threads, smem, s>>>(a);
        else orbit_record_kernel<ARITH, OCT, false, false><<<blocks, threads, smem, s>>>(a);
    }
}

}  // namespace

cudaError_t launch_orbit_record(const OrbitRecordArgs &a, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    // One warp per block: the orbit of few particles is a long serial chain,
    // spread over as many SMs as possible, and the staging buffer (17 KB a
    // warp) sets the residency, not the block size.
    const int threads = 32;
    const unsigned blocks = unsigned((a.n + threads - 1) / threads);
    const bool oct = a.mu != 0.0;
    if (a.arith == HM_ARITH_FAST) {
        if (oct) launch_record_ok<HM_ARITH_FAST, true>(a, blocks, threads, s);
        else launch_record_ok<HM_ARITH_FAST, false>(a, blocks, threads, s);
    } else {
        if (oct) launch_record_ok<HM_ARITH_EXACT, true>(a, blocks, threads, s);
        else launch_record_ok<HM_ARITH_EXACT, false>(a, blocks, threads, s);
    }
    return cudaGetLastError();
}

cudaError_t launch_birkhoff_segments(const BirkhoffSegArgs &a, cudaStream_t s) {
    if (a.n == 0 || a.n_win == 0) return cudaSuccess;
    const size_t threads = 2u * size_t(a.n_seg) * a.n;
    const dim3 grid(unsigned((threads + 127) / 128), unsigned((a.n_win + kWinGroup - 1) / kWinGroup));
    birkhoff_seg_kernel<<<grid, 128, 0, s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const size_t t2 = 2u * size_t(a.n_win) * a.n;
    birkhoff_finish_kernel<<<unsigned((t2 + 127) / 128), 128, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_hann_table(double *h, uint32_t len, cudaStream_t s) {
    if (len == 0) return cudaSuccess;
    hann_table_kernel<<<(len + 255) / 256, 256, 0, s>>>(h, len);
    return cudaGetLastError();
}

cudaError_t launch_fft_gather2(const double *x, const double *px, const double *y,
                               const double *py, const double *means, size_t n, uint32_t from,
                               uint32_t len, const double *h, double2 *z, size_t S,
                               cudaStream_t s) {
    if (n == 0 || len == 0) return cudaSuccess;
    const unsigned grid = unsigned((n * len + 255) / 256);
    for (int plane = 0; plane < 2; ++plane) {
        fft_gather2_kernel<<<grid, 256, 0, s>>>(x, px, y, py, means, n, from, len, h, z, S, plane);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_fft_peak2(const double2 *z, uint32_t len, size_t n, uint32_t last_sample,
                             const uint32_t *first_nan, double *out, size_t cols, int col,
                             cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const size_t threads = 2 * n * 32;
    fft_peak2_kernel<<<unsigned((threads + 255) / 256), 256, 0, s>>>(z, len, n, last_sample,
                                                                    first_nan, out, cols, col);
    return cudaGetLastError();
}

size_t fft_tune_smem_bytes(const FftPlanDev &plan) {
    return (size_t(fft_row_slots(plan)) + plan.n_coarse + 64u) * sizeof(double2);
}

cudaError_t launch_fft_tunes(const FftTuneArgs &a, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    if (a.plan.M == 0 || a.plan.M > kFftMaxLen || a.plan.L == 0) return cudaErrorInvalidValue;
    const size_t smem = fft_tune_smem_bytes(a.plan);
    auto kernel = a.plan.swizzle ? fft_tune_kernel<true> : fft_tune_kernel<false>;
    if (smem > 40u * 1024u) {
        const cudaError_t e =
            cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
    }
    // About one radix-8 butterfly per thread and stage.  A row of 6144
    // values or more fills most of an SM's shared memory, so its block takes
    // up to 1024 threads; shorter rows take 256, so that several blocks share
    // an SM.
    const uint32_t want = (a.plan.M / 8u + 31u) / 32u * 32u;
    const uint32_t cap = a.plan.M >= 6144u ? uint32_t(kFftThreadsMax) : 256u;
    const int threads = int(std::min<uint32_t>(cap, std::max<uint32_t>(64u, want)));
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    if (e != cudaSuccess) return e;
    FftTuneArgs b = a;
    b.prefetch_ahead = uint32_t(std::max(1, sms * std::max(1, per_sm)));
    kernel<<<unsigned(2 * a.n), threads, smem, s>>>(b);
    return cudaGetLastError();
}

cudaError_t launch_mean_remove(double *x, double *px, double *y, double *py, size_t n, size_t S,
                               cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    mean_remove_kernel<<<unsigned((4u * n + 127) / 128), 128, 0, s>>>(x, px, y, py, n, S);
    return cudaGetLastError();
}

cudaError_t launch_birkhoff_tunes(const double *x, const double *px, const double *y,
                                  const double *py, size_t n, const uint32_t *from,
                                  const uint32_t *to, const uint64_t *w_off, const double *w,
                                  int n_win, double *out, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const size_t threads = n * 2u * size_t(n_win);
    birkhoff_kernel<<<unsigned((threads + 127) / 128), 128, 0, s>>>(x, px, y, py, n, from, to,
                                                                    w_off, w, n_win, out);
    return cudaGetLastError();
}

cudaError_t launch_hann_gather(const double *q, const double *p, size_t n, uint32_t from,
                               uint32_t len, size_t first, size_t count, double2 *buf,
                               int *nan_flags, cudaStream_t s) {
    const size_t total = count * len;
    if (total == 0) return cudaSuccess;
    hann_gather_kernel<<<unsigned((total + 255) / 256), 256, 0, s>>>(q, p, n, from, len, first,
                                                                      count, buf, nan_flags);
    return cudaGetLastError();
}

cudaError_t launch_fft_peak(const double2 *buf, uint32_t len, size_t count, const int *nan_flags,
                            double *out, size_t out_stride, size_t first, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    const size_t threads = count * 32;
    fft_peak_kernel<<<unsigned((threads + 255) / 256), 256, 0, s>>>(buf, len, count, nan_flags,
                                                                    out, out_stride, first);
    return cudaGetLastError();
}

}  // namespace hm
