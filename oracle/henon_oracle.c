/*
 * henon_oracle.c -- CPU restatement of the reference's Henon-map arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests, the
 * smoke test and the CPU-baseline leg of bench.py call it.  The library
 * (henon_map_cpp_b200) never links, loads or calls it.
 *
 * Build (no FMA contraction, no -march, no fast-math):
 *   gcc -O2 -std=gnu11 -fPIC -shared -ffp-contract=off -fno-fast-math -fopenmp \
 *       oracle/henon_oracle.c -o oracle/liboracle.so -lm
 *
 * Every function cites the reference code (carlidel/henon_map_cpp) whose
 * arithmetic it restates; expressions keep the reference's association
 * order so that results are bit-identical to its CPU path.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---- modulation (src/modulation.cpp:3-60) ------------------------------- */

static const double kCoeff[7] = {1.000e-4, 0.218e-4, 0.708e-4, 0.254e-4,
                                 0.100e-4, 0.078e-4, 0.218e-4};
static const int kMult[7] = {1, 2, 3, 6, 7, 10, 12};

/* sps_modulation: omega(n) = 2*pi*tune*(1 + eps*sum_j c_j cos(W_j * n)) */
void or_sps_modulation(double tune, double epsilon, int32_t start,
                       int32_t end, double *out) {
    double w[7];
    for (int j = 0; j < 7; ++j) w[j] = (double)kMult[j] * (2 * M_PI / 868.12);
    for (uint32_t i = 0; i < (uint32_t)(end - start); ++i) {
        double sum = 0.0;
        const double n = (double)(uint32_t)(i + (uint32_t)start);
        for (int j = 0; j < 7; ++j) sum += kCoeff[j] * cos(w[j] * n);
        out[i] = 2 * M_PI * tune * (1 + epsilon * sum);
    }
}

/* basic_modulation: omega(i) = 2*pi*tune*(1 + eps*cos(2*pi*omega*i)) */
void or_basic_modulation(double tune, double omega, double epsilon,
                         int32_t start, int32_t end, double *out) {
    for (int i = 0; i < end - start; ++i)
        out[i] = 2 * M_PI * tune * (1 + epsilon * cos(2 * M_PI * omega * i));
}

/* sin/cos tables of omega (src/henon.cu:2679-2682). */
void or_tables(const double *omega, size_t n, double *s, double *c) {
    for (size_t i = 0; i < n; ++i) {
        s[i] = sin(omega[i]);
        c[i] = cos(omega[i]);
    }
}

/* birkhoff_weights (src/dynamic_indicator.cpp:63-79). */
void or_birkhoff_weights(uint32_t n, double *w) {
    double sum = 0.0;
    for (uint32_t i = 0; i < n; ++i) {
        double t = (double)i / (double)n;
        w[i] = exp(-1 / (t * (1.0 - t)));
    }
    for (uint32_t i = 0; i < n; ++i) sum += w[i];
    for (uint32_t i = 0; i < n; ++i) w[i] = w[i] / sum;
}

/* ---- one turn (src/henon.cu:113-173, host henon_step 420-480) ------------ */

static int is_lost(double x, double px, double y, double py) {
    return isnan(x) || isnan(px) || isnan(y) || isnan(py);
}

static void turn(double *x, double *px, double *y, double *py, uint32_t *steps,
                 const double *sinx, const double *cosx, const double *siny,
                 const double *cosy, double barrier_pow_2, double mu,
                 int reverse) {
    double X = *x, PX = *px, Y = *y, PY = *py;
    if (is_lost(X, PX, Y, PY)) return;
    if (!reverse) {
        /* sextupole */
        PX += X * X - Y * Y;
        PY += -2.0 * X * Y;
        /* octupole */
        if (mu != 0.0) {
            PX += mu * (X * X * X - 3.0 * Y * Y * X);
            PY += mu * (Y * Y * Y - 3.0 * X * X * Y);
        }
        /* rotations with table[steps] */
        const uint32_t s = *steps;
        double xt = X, pt = PX;
        X = xt * cosx[s] + pt * sinx[s];
        PX = -xt * sinx[s] + pt * cosx[s];
        xt = Y;
        pt = PY;
        Y = xt * cosy[s] + pt * siny[s];
        PY = -xt * siny[s] + pt * cosy[s];
    } else {
        const uint32_t s = *steps - 1;
        double xt = X, pt = PX;
        X = xt * cosx[s] - pt * sinx[s];
        PX = xt * sinx[s] + pt * cosx[s];
        xt = Y;
        pt = PY;
        Y = xt * cosy[s] - pt * siny[s];
        PY = xt * siny[s] + pt * cosy[s];
        if (mu != 0.0) {
            PX -= mu * (X * X * X - 3.0 * Y * Y * X);
            PY -= mu * (Y * Y * Y - 3.0 * X * X * Y);
        }
        PX -= X * X - Y * Y;
        PY -= -2.0 * X * Y;
    }
    if ((X * X + PX * PX) + (Y * Y + PY * PY) < barrier_pow_2) {
        *steps += reverse ? (uint32_t)-1 : 1u;
        *x = X;
        *px = PX;
        *y = Y;
        *py = PY;
    } else {
        *x = NAN;
        *px = NAN;
        *y = NAN;
        *py = NAN;
    }
}

/* ---- reproducible random kicks --------------------------------------------
 * The reference kicks every particle by kick_module along a random direction
 * before the sextupole (random_4d_kick, src/henon.cu:362-405, called from
 * henon_step :438-441 and :465-468 in reverse), from a clock()-seeded curand
 * stream on the GPU.  This library draws the direction from a counter-based
 * generator keyed by (seed, particle index, table index of the turn), so
 * that a run is reproducible and independent of how it is split into
 * launches.  The restatement here is bit-identical to the device code:
 *   Philox4x32-10 (J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw,
 *   "Parallel random numbers: as easy as 1, 2, 3", SC'11): counter
 *   {turn, attempt, idx_lo, idx_hi}, key {seed_lo, seed_hi};
 *   a direction uniform on the unit 3-sphere by Marsaglia's method
 *   (Ann. Math. Statist. 43 (1972) 645-646): (u1, u2) and (u3, u4) uniform
 *   in the unit disc, s1 = u1^2+u2^2, s2 = u3^2+u4^2, then
 *   (u1, u2, u3 f, u4 f) with f = sqrt((1 - s1) / s2).
 * Each attempt turns one Philox block into candidate points for both discs
 * (u = (int32(r) + 0.5) * 2^-31, exact); a disc keeps its first accepted
 * point.  After 64 attempts (probability of getting there < 1e-42) a disc
 * without a point takes (0, 0) for the first disc and (1, 0) for the
 * second. */
void or_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

static double kick_uniform(uint32_t r) { return ((double)(int32_t)r + 0.5) * 0x1p-31; }

void or_kick_direction(uint64_t seed, uint64_t idx, uint32_t turn, double d[4]) {
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    double u1 = 0.0, u2 = 0.0, u3 = 1.0, u4 = 0.0, s1 = 0.0, s2 = 1.0;
    int got1 = 0, got2 = 0;
    for (uint32_t a = 0; a < 64u && !(got1 && got2); ++a) {
        const uint32_t ctr[4] = {turn, a, (uint32_t)idx, (uint32_t)(idx >> 32)};
        uint32_t r[4];
        or_philox4x32_10(ctr, key, r);
        if (!got1) {
            const double a1 = kick_uniform(r[0]), a2 = kick_uniform(r[1]);
            const double s = a1 * a1 + a2 * a2;
            if (s < 1.0) {
                u1 = a1;
                u2 = a2;
                s1 = s;
                got1 = 1;
            }
        }
        if (!got2) {
            const double a3 = kick_uniform(r[2]), a4 = kick_uniform(r[3]);
            const double s = a3 * a3 + a4 * a4;
            if (s < 1.0 && s > 0.0) {
                u3 = a3;
                u4 = a4;
                s2 = s;
                got2 = 1;
            }
        }
    }
    const double f = sqrt((1.0 - s1) / s2);
    d[0] = u1;
    d[1] = u2;
    d[2] = u3 * f;
    d[3] = u4 * f;
}

/* One turn with a kick of module km along the direction of (seed, j, table
 * index): added before the sextupole going forward; going backward,
 * subtracted after the inverse sextupole (undoing the forward turn's kick),
 * then the barrier test. */
static void turn_kicked(double *x, double *px, double *y, double *py, uint32_t *steps,
                        const double *sinx, const double *cosx, const double *siny,
                        const double *cosy, double barrier_pow_2, double mu, int reverse,
                        double km, uint64_t seed, uint64_t j) {
    if (is_lost(*x, *px, *y, *py)) return;
    double d[4];
    if (!reverse) {
        or_kick_direction(seed, j, *steps, d);
        *x += d[0] * km;
        *px += d[1] * km;
        *y += d[2] * km;
        *py += d[3] * km;
        turn(x, px, y, py, steps, sinx, cosx, siny, cosy, barrier_pow_2, mu, 0);
        return;
    }
    or_kick_direction(seed, j, *steps - 1, d);
    /* the inverse turn without its barrier test (an overflowed state is
     * lost either way), then the kick, then the test */
    turn(x, px, y, py, steps, sinx, cosx, siny, cosy, INFINITY, mu, 1);
    if (is_lost(*x, *px, *y, *py)) return;
    *x -= d[0] * km;
    *px -= d[1] * km;
    *y -= d[2] * km;
    *py -= d[3] * km;
    const double X = *x, PX = *px, Y = *y, PY = *py;
    if (!((X * X + PX * PX) + (Y * Y + PY * PY) < barrier_pow_2)) {
        *steps += 1u; /* the inverse turn counted a step that was not survived */
        *x = NAN;
        *px = NAN;
        *y = NAN;
        *py = NAN;
    }
}

/* henon_tracker::track with random kicks (kick_module not NaN). */
void or_track_kicked(double *x, double *px, double *y, double *py, uint32_t *steps, size_t n,
                     const double *sinx, const double *cosx, const double *siny,
                     const double *cosy, uint32_t n_turns, double mu, double barrier,
                     int reverse, double kick_module, uint64_t seed, int n_threads) {
    const double b2 = barrier * barrier;
#ifdef _OPENMP
    if (n_threads <= 0) n_threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(n_threads)
#endif
    for (long long j = 0; j < (long long)n; ++j)
        for (uint32_t k = 0; k < n_turns; ++k)
            turn_kicked(&x[j], &px[j], &y[j], &py[j], &steps[j], sinx, cosx, siny, cosy, b2, mu,
                        reverse, kick_module, seed, (uint64_t)j);
    (void)n_threads;
}

/* henon_tracker::track (src/henon.cu:2701-2752): n_turns turns of every
 * particle, particles spread over n_threads OpenMP threads (<=0: all). */
void or_track(double *x, double *px, double *y, double *py, uint32_t *steps,
              size_t n, const double *sinx, const double *cosx,
              const double *siny, const double *cosy, uint32_t n_turns,
              double mu, double barrier, int reverse, int n_threads) {
    const double b2 = barrier * barrier;
#ifdef _OPENMP
    if (n_threads <= 0) n_threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(n_threads)
#endif
    for (long long j = 0; j < (long long)n; ++j)
        for (uint32_t k = 0; k < n_turns; ++k)
            turn(&x[j], &px[j], &y[j], &py[j], &steps[j], sinx, cosx, siny, cosy,
                 b2, mu, reverse);
    (void)n_threads;
}

int or_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ---- tangent map (src/henon.cu:175-265) --------------------------------- */

/* tangent_matrix (device form :175-196, host form :198-222), row-major. */
void or_tangent_matrix(double x, double px, double y, double py, double sx,
                       double cx, double sy, double cy, double mu,
                       double *out) {
    (void)px;
    (void)py;
    out[0] = cx + sx * (2 * x + mu * 3 * x * x - mu * 3 * y * y);
    out[1] = sx;
    out[2] = sx * (-2 * y - mu * 6 * x * y);
    out[3] = 0.0;
    out[4] = -sx + cx * (2 * x + mu * 3 * x * x - mu * 3 * y * y);
    out[5] = cx;
    out[6] = cx * (-2 * y - mu * 6 * x * y);
    out[7] = 0.0;
    out[8] = sy * (-2 * y - mu * 6 * x * y);
    out[9] = 0.0;
    out[10] = cy + sy * (-2 * x - mu * 3 * x * x + mu * 3 * y * y);
    out[11] = sy;
    out[12] = cy * (-2 * y - mu * 6 * x * y);
    out[13] = 0.0;
    out[14] = -sy + cy * (-2 * x - mu * 3 * x * x + mu * 3 * y * y);
    out[15] = cy;
}

/* result = a * b, 4x4 row-major, sums started from 0.0 and accumulated in
 * k order (get_matrices_and_multiply, :267-295; multiply_matrices :251-265) */
void or_matmul4(const double *a, const double *b, double *out) {
    double r[16];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double s = 0.0;
            for (int k = 0; k < 4; ++k) s += a[i * 4 + k] * b[k * 4 + j];
            r[i * 4 + j] = s;
        }
    memcpy(out, r, sizeof(r));
}
