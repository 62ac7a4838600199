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
