// Tune estimates from turn-by-turn orbits (sm_100a).
//
// An orbit buffer holds S snapshots of n particles per coordinate, laid
// out [sample][particle] (storage_4d_gpu's layout), so a warp reads 32
// particles of one sample in one coalesced access.
//
// * orbit_record_kernel: tracks n_turns turns and writes every state
//   (sample 0 = the start), like the reference's CPU tune routines that
//   store the orbit before computing tunes (src/henon.cu:2890-3078);
// * mean_remove_kernel: subtracts each coordinate's orbit mean
//   (src/henon.cu:3040-3051);
// * birkhoff_kernel: Birkhoff-weighted phase advance over sample windows
//   (birkhoff_tune / birkhoff_tune_vec, src/dynamic_indicator.cpp:81-131,
//   198-253);
// * hann_gather_kernel + cuFFT + fft_peak_kernel: Hann-windowed spectrum of
//   x + i px and the interpolated peak (compute_fft, interpolation, A,
//   fft_tune_vec, src/dynamic_indicator.cpp:32-61, 134-196, 255-330).
// Those serve orbits the caller stored (storage tunes).  The tracker's own
// tune path records the orbit with each coordinate's running sum and the
// first NaN sample, and then never rewrites it: the mean is subtracted as
// samples are read, Birkhoff sums run in segments of turns over many
// threads (birkhoff_seg_kernel / birkhoff_finish_kernel), and the FFT
// gather writes both planes of a window as one batch of rows through
// shared-memory tiles (fft_gather2_kernel, fft_peak2_kernel).
#include <cuda_runtime.h>

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
template <int ARITH, bool OCT, bool REV, bool KICK>
__global__ void orbit_record_kernel(OrbitRecordArgs a) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const size_t n = a.n;
    double x = a.x[i], px = a.px[i], y = a.y[i], py = a.py[i];
    uint32_t steps = a.steps[i];
    bool alive = !dev::is_lost(x, px, y, py);
    uint32_t first_nan = alive ? a.n_turns + 1u : 0u;
    a.ox[i] = x;
    a.opx[i] = px;
    a.oy[i] = y;
    a.opy[i] = py;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    const bool sums = a.sums != nullptr;
    if (sums) {
        s0 = Rn::add(s0, x);
        s1 = Rn::add(s1, px);
        s2 = Rn::add(s2, y);
        s3 = Rn::add(s3, py);
    }
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
        const size_t o = size_t(k + 1) * n + i;
        a.ox[o] = x;
        a.opx[o] = px;
        a.oy[o] = y;
        a.opy[o] = py;
        if (sums) {
            s0 = Rn::add(s0, x);
            s1 = Rn::add(s1, px);
            s2 = Rn::add(s2, y);
            s3 = Rn::add(s3, py);
        }
    }
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
    double prev = atan2(centred(p[size_t(s0) * n + i], a.means, mp),
                        centred(q[size_t(s0) * n + i], a.means, mq));
    for (uint32_t s = s0; s < s1; ++s) {
        const size_t o = size_t(s + 1) * n + i;
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
// particle), cuFFT's native batch layout.  A block moves a tile of 32
// samples x 32 columns through shared memory, so that the orbit is read
// along particles and the rows are written along samples, both coalesced.
constexpr int kTile = 32;

__global__ void __launch_bounds__(256) fft_gather2_kernel(const double *x, const double *px,
                                                          const double *y, const double *py,
                                                          const double *means, size_t n,
                                                          uint32_t from, uint32_t len,
                                                          const double *h, double2 *z, size_t S,
                                                          int plane) {
    __shared__ double2 tile[kTile][kTile + 1];
    const size_t i0 = size_t(blockIdx.x) * kTile;  // first particle of the tile
    const uint32_t k0 = blockIdx.y * kTile;        // first sample of the tile
    const double *q = plane ? y : x, *p = plane ? py : px;
    const unsigned tx = threadIdx.x & 31u, ty = threadIdx.x >> 5;  // 8 warps
    // read: lane tx takes particle i0 + tx; warp ty samples k0 + ty, + 8, ...
    {
        const size_t i = i0 + tx;
        const bool ok_i = i < n;
        const double mq = ok_i ? mean_of(means, n, i, 2 * plane, S) : 0.0;
        const double mp = ok_i ? mean_of(means, n, i, 2 * plane + 1, S) : 0.0;
        for (unsigned r = ty; r < unsigned(kTile); r += 8u) {
            const uint32_t k = k0 + r;
            double2 v = make_double2(0.0, 0.0);
            if (ok_i && k < len) {
                const size_t o = size_t(from + k) * n + i;
                const double re = centred(q[o], means, mq), im = centred(p[o], means, mp);
                const double hk = h[k];
                v = make_double2(re * hk, im * hk);
            }
            tile[r][tx] = v;
        }
    }
    __syncthreads();
    // write: warp ty takes particles i0 + ty, + 8, ...; lane tx sample k0 + tx
    for (unsigned ii = ty; ii < unsigned(kTile); ii += 8u) {
        const size_t i = i0 + ii;
        const uint32_t k = k0 + tx;
        if (i < n && k < len) z[(size_t(plane) * n + i) * len + k] = tile[tx][ii];
    }
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

template <int ARITH, bool OCT>
void launch_record_ok(const OrbitRecordArgs &a, unsigned blocks, int threads, cudaStream_t s) {
    const bool kick = !isnan(a.kick_module);
    if (a.inverse) {
        if (kick) orbit_record_kernel<ARITH, OCT, true, true><<<blocks, threads, 0, s>>>(a);
        else orbit_record_kernel<ARITH, OCT, true, false><<<blocks, threads, 0, s>>>(a);
    } else {
        if (kick) orbit_record_kernel<ARITH, OCT, false, true><<<blocks, threads, 0, s>>>(a);
        else orbit_record_kernel<ARITH, OCT, false, false><<<blocks, threads, 0, s>>>(a);
    }
}

}  // namespace

cudaError_t launch_orbit_record(const OrbitRecordArgs &a, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    // Small blocks: the orbit of few particles is a long serial chain, so
    // spread the threads over as many SMs as possible.
    const int threads = a.n < 148u * 128u ? 32 : 128;
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
    const dim3 grid(unsigned((n + kTile - 1) / kTile), (len + kTile - 1) / kTile);
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
