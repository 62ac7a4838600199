// Host-side tune-modulation tables and Birkhoff weights.
//
// The per-turn rotation angles omega(n) and their sin/cos are computed on the
// host with the C library's libm, exactly as the reference does
// (src/modulation.cpp:3-134, src/henon.cu:2657-2694): the device only reads
// the resulting tables, so the expression order below is chosen to give
// bit-identical doubles to the reference on the same host.
#include <cmath>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "hm_internal.h"

namespace hm {
namespace {

// Harmonics of the SPS power-converter ripple: coefficient c_j and angular
// frequency k_j * 2*pi/868.12 (src/modulation.cpp:13-29).  The constants
// are the physical model; they have to be the reference's values.
constexpr int kSpsHarmonics = 7;
constexpr double kSpsCoefficient[kSpsHarmonics] = {
    1.000e-4, 0.218e-4, 0.708e-4, 0.254e-4, 0.100e-4, 0.078e-4, 0.218e-4};
constexpr int kSpsMultiple[kSpsHarmonics] = {1, 2, 3, 6, 7, 10, 12};

// Runs body(i) for i in [0, n) on all host threads, interleaved.
template <class F> void parallel_for(size_t n, F body) {
    unsigned n_threads = std::thread::hardware_concurrency();
    if (n_threads == 0) n_threads = 1;
    if (n < 4096 || n_threads == 1) {
        for (size_t i = 0; i < n; ++i) body(i);
        return;
    }
    std::vector<std::thread> pool;
    pool.reserve(n_threads);
    for (unsigned t = 0; t < n_threads; ++t)
        pool.emplace_back([=, &body] {
            for (size_t i = t; i < n; i += n_threads) body(i);
        });
    for (auto &th : pool) th.join();
}

}  // namespace

// omega(n) = 2*pi*tune * (1 + eps * sum_j c_j cos(Omega_j * n)),
// n = start .. end-1, harmonics summed in ascending j
// (sps_modulation, src/modulation.cpp:31-60).
std::vector<double> sps_modulation(double tune, double epsilon, int32_t start,
                                   int32_t end) {
    std::vector<double> out(end > start ? size_t(end - start) : 0);
    double omega_k[kSpsHarmonics];
    const double fundamental = 2 * M_PI / 868.12;
    for (int j = 0; j < kSpsHarmonics; ++j)
        omega_k[j] = double(kSpsMultiple[j]) * fundamental;
    const double two_pi_tune = 2 * M_PI * tune;
    parallel_for(out.size(), [&](size_t i) {
        // The reference adds an unsigned index to the int start: the turn
        // number is formed in 32-bit unsigned arithmetic.
        const double turn = double(uint32_t(uint32_t(i) + uint32_t(start)));
        double ripple = 0.0;
        for (int j = 0; j < kSpsHarmonics; ++j)
            ripple += kSpsCoefficient[j] * std::cos(omega_k[j] * turn);
        out[i] = two_pi_tune * (1 + epsilon * ripple);
    });
    return out;
}

// omega(i) = 2*pi*tune * (1 + eps * cos(2*pi*omega*i)), i counted from 0
// (basic_modulation, src/modulation.cpp:3-11).
std::vector<double> basic_modulation(double tune, double omega, double epsilon,
                                     int32_t start, int32_t end) {
    std::vector<double> out(end > start ? size_t(end - start) : 0);
    const double two_pi_tune = 2 * M_PI * tune;
    const double two_pi_omega = 2 * M_PI * omega;
    for (size_t i = 0; i < out.size(); ++i)
        out[i] = two_pi_tune * (1 + epsilon * std::cos(two_pi_omega * int(i)));
    return out;
}

hm_status modulation(const std::string &kind, uint32_t n_turns, double omega_x,
                     double omega_y, double omega_0, double epsilon,
                     uint32_t offset, std::vector<double> &wx,
                     std::vector<double> &wy) {
    const int32_t start = int32_t(offset);
    const int32_t end = int32_t(offset + n_turns);
    if (kind == "sps") {
        wx = sps_modulation(omega_x, epsilon, start, end);
        wy = sps_modulation(omega_y, epsilon, start, end);
    } else if (kind == "basic") {
        if (std::isnan(omega_0))
            return fail(HM_ERR_INVALID_ARG,
                        "basic modulation needs a finite omega_0");
        wx = basic_modulation(omega_x, omega_0, epsilon, start, end);
        wy = basic_modulation(omega_y, omega_0, epsilon, start, end);
    } else if (kind == "none") {
        // The reference fills empty vectors (src/modulation.cpp:119-123) and
        // then reads past them; here the tables hold the constant angles.
        wx.assign(n_turns, omega_x);
        wy.assign(n_turns, omega_y);
    } else if (kind == "gaussian" || kind == "uniform") {
        // Random tunes drawn per turn (src/modulation.cpp:62-99): angle =
        // 2*pi*sample with sample ~ N(omega, eps) or U(omega, eps).
        std::random_device rd;
        auto draw = [&](double a, std::vector<double> &out) {
            std::mt19937 gen(rd());
            out.resize(n_turns);
            if (kind == "gaussian") {
                std::normal_distribution<double> dist(a, epsilon);
                for (auto &v : out) v = 2 * M_PI * dist(gen);
            } else {
                std::uniform_real_distribution<double> dist(a, epsilon);
                for (auto &v : out) v = 2 * M_PI * dist(gen);
            }
        };
        draw(omega_x, wx);
        draw(omega_y, wy);
    } else {
        return fail(HM_ERR_UNKNOWN_MODULATION, "Unknown modulation kind");
    }
    return ok();
}

// The ripple S_n of omega(n) = 2*pi*tune*(1 + eps*S_n) for the kinds whose
// angle is differentiable in (tune, eps): "sps" (the harmonic sum above) and
// "basic" (cos(2*pi*omega_0*i)).
hm_status modulation_ripple(const std::string &kind, uint32_t n_turns, double omega_0,
                            uint32_t offset, std::vector<double> &ripple) {
    ripple.assign(n_turns, 0.0);
    if (kind == "sps") {
        double omega_k[kSpsHarmonics];
        const double fundamental = 2 * M_PI / 868.12;
        for (int j = 0; j < kSpsHarmonics; ++j)
            omega_k[j] = double(kSpsMultiple[j]) * fundamental;
        parallel_for(n_turns, [&](size_t i) {
            const double turn = double(uint32_t(uint32_t(i) + offset));
            double s = 0.0;
            for (int j = 0; j < kSpsHarmonics; ++j) s += kSpsCoefficient[j] * std::cos(omega_k[j] * turn);
            ripple[i] = s;
        });
        return ok();
    }
    if (kind == "basic") {
        const double two_pi_omega = 2 * M_PI * omega_0;
        for (uint32_t i = 0; i < n_turns; ++i) ripple[i] = std::cos(two_pi_omega * int(i));
        return ok();
    }
    return fail(HM_ERR_NOT_SUPPORTED,
                "derivatives need an 'sps' or 'basic' modulation (random tunes have none)");
}

// w_i = exp(-1/(t(1-t))), t = i/n, normalised by the left-to-right sum
// (birkhoff_weights, src/dynamic_indicator.cpp:63-79).
std::vector<double> birkhoff_weights(uint32_t n) {
    std::vector<double> w(n);
    for (uint32_t i = 0; i < n; ++i) {
        const double t = double(i) / double(n);
        w[i] = std::exp(-1 / (t * (1.0 - t)));
    }
    double sum = 0.0;
    for (double v : w) sum += v;
    for (double &v : w) v = v / sum;
    return w;
}

}  // namespace hm
