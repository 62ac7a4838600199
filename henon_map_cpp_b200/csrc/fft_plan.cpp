// Plans of the shared-memory FFT tunes (fft_tune_kernel, tunes.cu).
//
// A plan holds, for windows of L samples, the factorisation of the
// transform length M into radices 5, 3, 8, 4 and 2, the twiddles
// exp(-2 pi i t / M) as two tables whose product gives any t < M (64-step
// coarse values and the 64 fine ones; both fit in shared memory), and
// either the position of each X_k after the forward network (M = L) or,
// for Bluestein's convolution (M >= 2L - 1), the chirp
// c_n = exp(-i pi n^2 / L) and the forward network's output for the
// convolution kernel b_m = conj(c_m) (m in (-L, L), cyclic).  Tables are
// computed on the host in long double and rounded once.  Plans are built on
// first use per (device, L) and kept until exit: a plan is at most a few
// hundred KB of device memory, and a kernel of another thread may still
// read it.
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <map>
#include <memory>
#include <mutex>
#include <utility>
#include <vector>

#include "hm_internal.h"

namespace hm {
namespace {

using cld = std::complex<long double>;

// Radices of M: fives and threes first (the early stages, whose spans are
// long), then eights and a four or a two (the late stages, short spans,
// which the shared-memory swizzle spreads over the banks); false when M has
// another prime factor.
bool factor(uint32_t M, std::vector<uint8_t> *rad) {
    rad->clear();
    uint32_t m = M;
    for (uint32_t r : {5u, 3u, 8u, 4u, 2u})
        while (m % r == 0) {
            rad->push_back(uint8_t(r));
            m /= r;
        }
    return m == 1 && rad->size() <= size_t(kFftMaxStages);
}

// exp(-2 pi i t / D), the angle reduced to (-pi, pi] exactly first.
cld cis(uint64_t t, uint64_t D) {
    const long double pi = 3.141592653589793238462643383279502884L;
    t %= D;
    const long double tt = 2 * t > D ? (long double)t - (long double)D : (long double)t;
    const long double a = -2.0L * pi * tt / (long double)D;
    return cld(std::cos(a), std::sin(a));
}

// The forward network of fft_tune_kernel (decimation in frequency, natural
// order in, the plan's positions out) with exact twiddles.
void network_forward(std::vector<cld> &x, const std::vector<uint8_t> &rad) {
    const uint32_t M = uint32_t(x.size());
    std::vector<cld> w(M);
    for (uint32_t t = 0; t < M; ++t) w[t] = cis(t, M);
    uint32_t N = M, prod = 1;
    for (uint8_t r : rad) {
        const uint32_t span = N / r;
        for (uint32_t b0 = 0; b0 < M; b0 += N)
            for (uint32_t j = 0; j < span; ++j) {
                cld v[8], y[8];
                for (uint32_t q = 0; q < r; ++q) v[q] = x[b0 + j + q * span];
                for (uint32_t k = 0; k < r; ++k) {
                    y[k] = 0;
                    for (uint32_t q = 0; q < r; ++q) y[k] += v[q] * w[(uint64_t(q) * k * (M / r)) % M];
                }
                for (uint32_t k = 0; k < r; ++k)
                    x[b0 + j + k * span] = y[k] * w[(uint64_t(j) * k * prod) % M];
            }
        N = span;
        prod *= r;
    }
}

std::vector<double2> to_double2(const std::vector<cld> &v) {
    std::vector<double2> out(v.size());
    for (size_t i = 0; i < v.size(); ++i) out[i] = make_double2(double(v[i].real()), double(v[i].imag()));
    return out;
}

struct PlanEntry {
    FftPlanDev dev;
    DeviceBuffer coarse, fine, pos, chirp, bhat;
};

struct FftPlans {
    std::mutex mutex;
    std::map<std::pair<int, uint32_t>, std::unique_ptr<PlanEntry>> plans;
};

// Never destroyed: at process exit the CUDA context may already be gone.
FftPlans &fft_plans() {
    static FftPlans *p = new FftPlans;
    return *p;
}

hm_status build_plan(uint32_t L, PlanEntry *e, bool *supported) {
    *supported = false;
    std::vector<uint8_t> rad;
    uint32_t M = 0;
    bool blue = false;
    if (L <= kFftMaxLen && factor(L, &rad)) {
        M = L;
    } else {
        // The shortest convolution length of radices 2, 3, 5 that is a
        // multiple of 8 (bank-conflict free), else the shortest.
        const uint64_t need = 2ull * L - 1ull;
        for (int pass = 0; pass < 2 && M == 0; ++pass)
            for (uint64_t m = need; m <= kFftMaxLen; ++m)
                if ((pass == 1 || m % 8 == 0) && factor(uint32_t(m), &rad)) {
                    M = uint32_t(m);
                    break;
                }
        if (M == 0) return ok();  // too long for one block: the library path
        factor(M, &rad);
        blue = true;
    }
    FftPlanDev &d = e->dev;
    d.L = L;
    d.M = M;
    d.bluestein = blue ? 1 : 0;
    d.swizzle = M % 8 == 0 ? 1 : 0;
    d.n_stages = int(rad.size());
    uint32_t N = M, prod = 1;
    for (size_t s = 0; s < rad.size(); ++s) {
        d.radix[s] = rad[s];
        d.stage_len[s] = N / rad[s];
        d.stage_prod[s] = prod;
        N /= rad[s];
        prod *= rad[s];
    }
    d.n_coarse = (M + 63u) / 64u;
    std::vector<cld> coarse(d.n_coarse), fine(64);
    for (uint32_t u = 0; u < d.n_coarse; ++u) coarse[u] = cis(64ull * u, M);
    for (uint32_t v = 0; v < 64u; ++v) fine[v] = cis(v, M);
    HM_TRY(upload(e->coarse, to_double2(coarse)));
    HM_TRY(upload(e->fine, to_double2(fine)));
    d.tw_coarse = e->coarse.as<double2>();
    d.tw_fine = e->fine.as<double2>();
    if (!blue) {
        // X_k with k = d1 + r1 d2 + r1 r2 d3 + ... lies at d1 M/r1 + d2 M/(r1 r2) + ...
        std::vector<uint32_t> pos(M);
        for (uint32_t k = 0; k < M; ++k) {
            uint32_t kk = k, p = 0, span = M;
            for (uint8_t r : rad) {
                const uint32_t dig = kk % r;
                kk /= r;
                span /= r;
                p += dig * span;
            }
            pos[k] = p;
        }
        HM_TRY(upload(e->pos, pos));
        d.pos = e->pos.as<uint32_t>();
    } else {
        std::vector<cld> c(L), b(M, cld(0));
        for (uint64_t n = 0; n < L; ++n) c[n] = cis((n * n) % (2ull * L), 2ull * L);
        b[0] = std::conj(c[0]);
        for (uint32_t m = 1; m < L; ++m) {
            b[m] = std::conj(c[m]);
            b[M - m] = std::conj(c[m]);
        }
        network_forward(b, rad);
        HM_TRY(upload(e->chirp, to_double2(c)));
        HM_TRY(upload(e->bhat, to_double2(b)));
        d.chirp = e->chirp.as<double2>();
        d.bhat = e->bhat.as<double2>();
    }
    *supported = true;
    return ok();
}

}  // namespace

hm_status fft_plan(uint32_t L, const FftPlanDev **plan) {
    *plan = nullptr;
    if (L == 0) return ok();
    int dev = 0;
    HM_CUDA_TRY(cudaGetDevice(&dev));
    FftPlans &c = fft_plans();
    std::lock_guard<std::mutex> lock(c.mutex);
    const auto key = std::make_pair(dev, L);
    auto it = c.plans.find(key);
    if (it == c.plans.end()) {
        auto e = std::make_unique<PlanEntry>();
        bool supported = false;
        HM_TRY(build_plan(L, e.get(), &supported));
        if (!supported) e.reset();
        it = c.plans.emplace(key, std::move(e)).first;
    }
    if (it->second) *plan = &it->second->dev;
    return ok();
}

}  // namespace hm
