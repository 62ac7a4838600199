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

#include <atomic>
#include <cstdint>

#include "hm_device.cuh"
#include "hm_internal.h"

namespace hm {
namespace {

using dev::Barrier;
using dev::kFullMask;
using dev::Particle;
using dev::quiet_nan;
using dev::Rn;
using dev::Turn;

// One turn of the K particles of a thread.  The common case costs the map
// and, per thread, an OR of the coordinates' high words and one integer
// compare (dev::small_or); a warp with a thread whose coordinates are not
// all small takes the rare path, which settles the barrier test per
// particle and freezes lost particles (set_to_nan, src/henon.cu:123-129)
// with steps = the turns they survived.  A lost particle's registers are
// set to zero, a fixed point of the map, so that it never trips the OR
// again.
template <int ARITH, bool OCT, bool REV, int K, bool KICK>
__device__ __forceinline__ void turn_all(const TrackChunk &c, const Barrier &bar, double mu,
                                         const Turn &t, uint32_t k, Particle (&p)[K],
                                         const uint32_t (&id)[K], bool (&live)[K],
                                         bool &warp_live) {
    uint32_t ored = 0u;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        // Random kick: before the sextupole going forward (table index
        // turn0 + k); going backward, subtracted after the inverse
        // sextupole (table index turn0 - 1 - k), undoing the forward kick.
        if (KICK && !REV)
            dev::apply_kick<false>(p[j], dev::kick_direction(c.kick_seed, id[j], c.turn0 + k),
                                   c.kick_module);
        dev::turn<ARITH, OCT, REV>(p[j], t, mu);
        if (KICK && REV)
            dev::apply_kick<true>(p[j], dev::kick_direction(c.kick_seed, id[j], c.turn0 - 1u - k),
                                  c.kick_module);
        if (!KICK || live[j]) ored |= dev::hi_or(p[j]);
    }
    if (__any_sync(kFullMask, !dev::small_or(ored, bar))) {
        const uint32_t s = REV ? c.turn0 - k : c.turn0 + k;
        bool any_live = false;
#pragma unroll
        for (int j = 0; j < K; ++j) {
            if (live[j] && !dev::small_inside(p[j], bar) &&
                !dev::inside<ARITH>(dev::radius_fma(p[j]), p[j], bar)) {
                const uint32_t i = id[j];
                c.ux[i] = quiet_nan();
                c.upx[i] = quiet_nan();
                c.uy[i] = quiet_nan();
                c.upy[i] = quiet_nan();
                c.usteps[i] = s;
                live[j] = false;
                p[j] = dev::make_particle(0.0, 0.0, 0.0, 0.0);
            }
            any_live |= live[j];
        }
        warp_live = __any_sync(kFullMask, any_live);
    }
}

// The chunk's turns with the turn records read from global memory: every
// lane of a warp loads the same 32-byte record (one broadcast transaction,
// an L1 hit after the first warp), prefetched one turn ahead.
template <int ARITH, bool OCT, bool REV, int K, bool KICK>
__device__ __forceinline__ void turns_direct(const TrackChunk &c, const Barrier &bar,
                                             Particle (&p)[K], const uint32_t (&id)[K],
                                             bool (&live)[K], bool warp_live) {
    const double mu = c.mu;
    const uint32_t nt = c.n_turns;
    Turn t = nt ? dev::load_turn(c.table, REV ? c.turn0 - 1u : c.turn0) : Turn{0.0, 0.0, 0.0, 0.0};
    for (uint32_t k = 0; warp_live && k < nt; ++k) {
        const uint32_t kn = (k + 1 < nt) ? k + 1 : k;
        const Turn tn = dev::load_turn(c.table, REV ? c.turn0 - 1u - kn : c.turn0 + kn);
        turn_all<ARITH, OCT, REV, K, KICK>(c, bar, mu, t, k, p, id, live, warp_live);
        t = tn;
    }
}

// Turns between two barrier votes of the staged kernel (see turns_staged).
constexpr uint32_t kCheckTurns = 32;

// Shared memory of a staged launch: two stage buffers of turn records and,
// without kicks, one checkpoint {x, px, y, py} per particle.
__host__ __device__ constexpr size_t staged_smem_bytes(uint32_t stage_turns, uint32_t threads,
                                                       int per_thread, bool kick) {
    return size_t(stage_turns) * 2u * 32u + (kick ? 0u : size_t(threads) * per_thread * 32u);
}

__device__ __forceinline__ Turn staged_record(const double *rec, uint32_t kn, uint32_t kk,
                                              bool rev) {
    const double2 *q = reinterpret_cast<const double2 *>(rec + 4u * (rev ? kn - 1u - kk : kk));
    const double2 a = q[0], b = q[1];
    return Turn{a.x, a.y, b.x, b.y};
}

// The chunk's turns with the turn records staged in shared memory: the
// chunk is cut into stages of c.stage_turns turns whose records (a
// contiguous span of the table) one thread brings in with a bulk copy,
// double-buffered, so that the copy of stage s+1 overlaps the turns of
// stage s.  Every warp then reads each record from shared memory as a
// broadcast.  Warps whose particles are all lost keep taking part in the
// per-stage barriers; the block stops when none of its warps is live.
//
// Without kicks, a stage runs in runs of kCheckTurns turns with no
// per-turn control flow: the thread saves its particles to shared memory,
// applies the turns while ORing every coordinate's high word, and the warp
// votes once at the end.  If no coordinate of any turn reached the bound
// of dev::small_or, no particle can have been lost in the run, which is
// then exactly what the per-turn test would have produced.  Otherwise the
// warp restores the saved particles and redoes the run with the per-turn
// test (turn_all), which finds the loss turn.  A per-turn vote made each
// turn wait for the tail of the previous one; a redo costs one run per
// loss event of a warp.
// Returns false when a copy did not land within the bounded wait (the
// chunk's results are then invalid and c.fault is set).
template <int ARITH, bool OCT, bool REV, int K, bool KICK>
__device__ __forceinline__ bool turns_staged(const TrackChunk &c, const Barrier &bar,
                                             Particle (&p)[K], const uint32_t (&id)[K],
                                             bool (&live)[K], bool warp_live) {
    // [2][S][4] turn records, then (no kicks) [K][blockDim.x] checkpoints.
    extern __shared__ __align__(128) double stage_buf[];
    __shared__ __align__(8) uint64_t full[2];
    const double mu = c.mu;
    const uint32_t nt = c.n_turns, S = c.stage_turns;
    const uint32_t n_stages = (nt + S - 1) / S;
    double2 *const ckpt = reinterpret_cast<double2 *>(stage_buf + size_t(S) * 8u);
    const bool leader = threadIdx.x == 0;
    auto issue = [&](uint32_t st) {
        const uint32_t k0 = st * S;
        const uint32_t kn = min(S, nt - k0);
        const uint32_t lo = REV ? c.turn0 - k0 - kn : c.turn0 + k0;
        dev::bulk_load(stage_buf + size_t(st & 1u) * S * 4u, c.table + size_t(lo) * 4u,
                       kn * 32u, &full[st & 1u]);
    };
    if (leader) {
        dev::mbar_init(&full[0], 1);
        dev::mbar_init(&full[1], 1);
        dev::mbar_init_fence();
    }
    __syncthreads();
    if (leader) {
        if (n_stages > 0) issue(0);
        if (n_stages > 1) issue(1);
    }
    bool timed_out = false;
    uint32_t st = 0;
    for (; st < n_stages; ++st) {
        const uint32_t buf = st & 1u;
        // Warp-uniform, so that the turn loop's warp votes see every lane.
        const bool landed = dev::mbar_wait(&full[buf], (st >> 1) & 1u);
        if (!__all_sync(kFullMask, landed)) timed_out = true;
        const uint32_t k0 = st * S;
        const uint32_t kn = min(S, nt - k0);
        const double *rec = stage_buf + size_t(buf) * S * 4u;
        if (!timed_out && KICK) {
#pragma unroll 2
            for (uint32_t kk = 0; warp_live && kk < kn; ++kk)
                turn_all<ARITH, OCT, REV, K, KICK>(c, bar, mu, staged_record(rec, kn, kk, REV),
                                                   k0 + kk, p, id, live, warp_live);
        } else if (!timed_out) {
            for (uint32_t j0 = 0; warp_live && j0 < kn; j0 += kCheckTurns) {
                const uint32_t j1 = min(j0 + kCheckTurns, kn);
#pragma unroll
                for (int j = 0; j < K; ++j) {
                    ckpt[2u * (j * blockDim.x + threadIdx.x)] = make_double2(p[j].x, p[j].px);
                    ckpt[2u * (j * blockDim.x + threadIdx.x) + 1u] = make_double2(p[j].y, p[j].py);
                }
                uint32_t ored = 0u;
#pragma unroll 2
                for (uint32_t kk = j0; kk < j1; ++kk) {
                    const Turn t = staged_record(rec, kn, kk, REV);
#pragma unroll
                    for (int j = 0; j < K; ++j) {
                        dev::turn<ARITH, OCT, REV>(p[j], t, mu);
                        ored |= dev::hi_or(p[j]);
                    }
                }
                if (__any_sync(kFullMask, !dev::small_or(ored, bar))) {
#pragma unroll
                    for (int j = 0; j < K; ++j) {
                        const double2 a = ckpt[2u * (j * blockDim.x + threadIdx.x)];
                        const double2 b = ckpt[2u * (j * blockDim.x + threadIdx.x) + 1u];
                        p[j] = dev::make_particle(a.x, a.y, b.x, b.y);
                    }
                    for (uint32_t kk = j0; warp_live && kk < j1; ++kk)
                        turn_all<ARITH, OCT, REV, K, KICK>(c, bar, mu,
                                                           staged_record(rec, kn, kk, REV),
                                                           k0 + kk, p, id, live, warp_live);
                }
            }
        }
        // Every warp is done with this buffer (and knows whether any warp of
        // the block is still live or has given up waiting).
        const bool block_fault = __syncthreads_or(timed_out);
        const bool block_live = __syncthreads_or(warp_live);
        if (block_fault || !block_live) break;
        if (leader && st + 2 < n_stages) {
            dev::async_proxy_fence();
            issue(st + 2);
        }
    }
    // Copies still in flight must land before the block's shared memory is
    // released: the one issued for stage st + 1 and, after a wait that gave
    // up, the one of stage st itself.  These waits are bounded too.
    const bool gave_up = __syncthreads_or(timed_out);
    if (gave_up && st < n_stages) dev::mbar_wait(&full[st & 1u], (st >> 1) & 1u);
    if (st + 1 < n_stages) {
        const uint32_t nx = st + 1;
        if (!dev::mbar_wait(&full[nx & 1u], (nx >> 1) & 1u)) timed_out = true;
    }
    const bool fault = __syncthreads_or(timed_out);
    if (fault && leader && c.fault) atomicOr(c.fault, 1u);
    return !fault;
}

// One chunk of turns for the particles of one block (K per thread).
template <int ARITH, bool OCT, bool REV, int K, bool STAGED, bool KICK>
__device__ __forceinline__ void track_chunk(const TrackChunk &c) {
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
        // Slots without a live particle hold zeros, a fixed point of the map.
        if (!live[j]) x = px = y = py = 0.0;
        p[j] = dev::make_particle(x, px, y, py);
    }

    const Barrier bar = dev::make_barrier<ARITH>(c.b2bits);
    bool thread_live = false;
#pragma unroll
    for (int j = 0; j < K; ++j) thread_live |= live[j];
    const bool warp_live = __any_sync(kFullMask, thread_live);
    if (STAGED) {
        if (!turns_staged<ARITH, OCT, REV, K, KICK>(c, bar, p, id, live, warp_live)) return;
    } else {
        turns_direct<ARITH, OCT, REV, K, KICK>(c, bar, p, id, live, warp_live);
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

// At most two particles per thread the kernel fits 64 registers without
// spills, i.e. 8 blocks of 128 threads per SM; four per thread need more.
template <int ARITH, bool OCT, bool REV, int K, bool STAGED, bool KICK>
__global__ void __launch_bounds__(256, K <= 2 ? 4 : 1) track_chunk_kernel(const TrackChunk c) {
    track_chunk<ARITH, OCT, REV, K, STAGED, KICK>(c);
}

// Staged fast arithmetic with two particles per thread, capped at 56
// registers (9 blocks of 128 threads per SM): 76.5 % of the FP64 peak on
// the DA scan against 74.5 % at 64.  Exact arithmetic gains nothing there.
template <int ARITH, bool OCT, bool REV>
__global__ void __maxnreg__(56) track_chunk_kernel_r56(const TrackChunk c) {
    track_chunk<ARITH, OCT, REV, 2, true, false>(c);
}

template <int ARITH, bool OCT, bool REV, int K, bool KICK>
cudaError_t launch_s(const TrackChunk &c, unsigned blocks, int threads, cudaStream_t s) {
    if (c.stage_turns == 0) {
        track_chunk_kernel<ARITH, OCT, REV, K, false, KICK><<<blocks, threads, 0, s>>>(c);
    } else {
        const size_t smem = staged_smem_bytes(c.stage_turns, uint32_t(threads), K, KICK);
        auto kernel = track_chunk_kernel<ARITH, OCT, REV, K, true, KICK>;
        if constexpr (ARITH == HM_ARITH_FAST && K == 2 && !KICK)
            kernel = track_chunk_kernel_r56<ARITH, OCT, REV>;
        // Dynamic plus static shared memory above 48 KB needs the opt-in
        // (the kernel's static part is its two mbarriers): 256 threads with
        // four particles each and 256-turn stages take exactly 48 KB dynamic.
        if (smem > 40u * 1024u) {
            const cudaError_t e =
                cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
            if (e != cudaSuccess) return e;
        }
        kernel<<<blocks, threads, smem, s>>>(c);
    }
    return cudaGetLastError();
}

// Multiprocessors of the current device (cached per device ordinal).
int sm_count() {
    constexpr int kMaxDevices = 64;
    static std::atomic<int> cache[kMaxDevices];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 1;
    int v = cache[dev].load(std::memory_order_relaxed);
    if (v <= 0) {
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
            return 1;
        cache[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

template <int ARITH, bool OCT, bool REV>
cudaError_t launch_k(const TrackChunk &c, const TrackLaunch &l, uint32_t n_upper,
                     cudaStream_t s) {
    const int threads = l.threads;
    if (!isnan(c.kick_module)) {
        // Kicked turns are dominated by the integer work of the generator:
        // one particle per thread.
        const unsigned blocks = unsigned((uint64_t(n_upper) + threads - 1) / threads);
        if (blocks == 0) return cudaSuccess;
        return launch_s<ARITH, OCT, REV, 1, true>(c, blocks, threads, s);
    }
    // Several particles per thread add instruction-level parallelism once
    // the device is full; a short list would instead leave SMs idle (a
    // particle is one serial chain of turns whatever its thread holds), so
    // K is halved while the grid would give fewer than two blocks per SM.
    int K = l.per_thread;
    const uint64_t min_blocks = 2u * uint64_t(sm_count());
    while (K > 1 && (uint64_t(n_upper) + uint64_t(threads) * K - 1) / (uint64_t(threads) * K) <
                        min_blocks)
        K /= 2;
    const uint64_t per_block = uint64_t(threads) * uint64_t(K);
    const unsigned blocks = unsigned((uint64_t(n_upper) + per_block - 1) / per_block);
    if (blocks == 0) return cudaSuccess;
    switch (K) {
        case 1: return launch_s<ARITH, OCT, REV, 1, false>(c, blocks, threads, s);
        case 2: return launch_s<ARITH, OCT, REV, 2, false>(c, blocks, threads, s);
        case 4: return launch_s<ARITH, OCT, REV, 4, false>(c, blocks, threads, s);
        default: return cudaErrorInvalidValue;
    }
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
