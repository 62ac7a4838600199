// Batched heterogeneous tracking: many parameter sets (tunes, epsilon, mu,
// barrier), each with its own particle count and turn budget, advanced
// together chunk by chunk with no host round trip in between.
//
// Per chunk:
//   * batch_chunk_kernel -- a persistent grid; every warp pops warp-tiles
//     (32*K live particles of ONE set, so the turn record, mu and barrier
//     are warp-uniform) from a device work queue, runs the set's turns of
//     this chunk with the particles in registers, writes lost particles out
//     at once and appends survivors to its set's next list;
//   * batch_plan_kernel -- one block: per-set survivor counts -> next tile
//     table (prefix sum), counters reset, ping-pong parity flipped.
// The sets are split into groups, each with its own chain of (plan, chunk)
// launches and its own tile table and counters; the chains run on separate
// streams.  The whole sequence has a fixed shape, so the host captures it
// once in a CUDA graph and replays it.
//
// The per-particle arithmetic is the tracking kernel's (track.cu), so every
// set's result is bit-identical to a plain hm_track of that set.
#include <cuda_runtime.h>

#include <cstdint>

#include "hm_device.cuh"
#include "hm_internal.h"

namespace hm {
namespace {

using dev::Particle;

// Each warp of the persistent chunk kernel works on tiles of different
// sets, so every warp stages its own set's turn records through shared
// memory: while the warp runs the kStageTurns turns of one stage, each lane
// holds kPerLane doubles of the next stage in registers (one coalesced
// 256-byte load per kPerLane), and stores them into the warp's other buffer
// at the end of the stage.  Without it, a warp whose set has few particles
// left waits on an L2 round trip every few turns.
constexpr uint32_t kStageTurns = 32u;
constexpr int kThreads = 128;
constexpr int kWarps = kThreads / 32;
constexpr int kPerLane = int(kStageTurns) * 4 / 32;

// Records [lo, lo + kn) of a table; element e of the stage = table[4 lo + e].
__device__ __forceinline__ void stage_load(double (&r)[kPerLane], const double *table, uint32_t lo,
                                           uint32_t kn, unsigned lane) {
#pragma unroll
    for (int q = 0; q < kPerLane; ++q) {
        const uint32_t e = lane + 32u * uint32_t(q);
        r[q] = e < 4u * kn ? __ldg(table + 4u * size_t(lo) + e) : 0.0;
    }
}

__device__ __forceinline__ void stage_store(double *buf, const double (&r)[kPerLane],
                                            unsigned lane) {
#pragma unroll
    for (int q = 0; q < kPerLane; ++q) buf[lane + 32u * uint32_t(q)] = r[q];
}

// Copies every non-NaN particle of every set into list 0 of its set and
// counts them (check_nan: NaN particles are never touched).
__global__ void batch_init_kernel(BatchDev b) {
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= b.n_total) return;
    const uint32_t s = b.particle_set[i];
    const double x = b.x[i], px = b.px[i], y = b.y[i], py = b.py[i];
    if (dev::is_lost(x, px, y, py)) return;
    const BatchSetDev &set = b.sets[s];
    const uint32_t o = atomicAdd(&b.state[s].next, 1u);
    const uint64_t slot = set.list_offset + o;
    b.list_idx[0][slot] = i;
    b.list_x[0][slot] = x;
    b.list_px[0][slot] = px;
    b.list_y[0][slot] = y;
    b.list_py[0][slot] = py;
}

// Between chunks: survivors -> live counts, next tile table.  One block.
__global__ void batch_plan_kernel(BatchDev b, uint32_t chunk_len_done, uint32_t chunk_len_next) {
    __shared__ uint32_t tiles_of[kBatchMaxSets];
    const int s = threadIdx.x;
    const uint32_t tile = 32u * uint32_t(b.per_thread);
    if (s < b.n_sets) {
        BatchStateDev &st = b.state[s];
        const uint32_t budget = b.sets[s].n_turns;
        const uint32_t ran = min(chunk_len_done, budget - st.done);
        st.done += ran;
        st.live = (st.done < budget) ? st.next : 0u;
        st.next = 0u;
        st.turns = min(chunk_len_next, budget - st.done);
        tiles_of[s] = st.turns ? (st.live + tile - 1) / tile : 0u;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t total = 0;
        for (int k = 0; k < b.n_sets; ++k) {
            b.state[k].first_tile = total;
            total += tiles_of[k];
        }
        *b.n_tiles = total;
        *b.next_item = 0u;
        // The first plan of a chain reads list 0, where the collection put
        // every particle; each later one swaps the lists.
        *b.parity = chunk_len_done == 0u ? 0u : (*b.parity ^ 1u);
    }
    __syncthreads();
    if (s < b.n_sets) {
        const uint32_t first = b.state[s].first_tile;
        for (uint32_t t = 0; t < tiles_of[s]; ++t) b.tile_set[first + t] = uint32_t(s);
    }
}

template <int ARITH, bool OCT, int K>
__device__ __forceinline__ void run_tile(const BatchDev &b, const BatchSetDev &set,
                                         const BatchStateDev &st, uint32_t s, uint32_t start,
                                         int in, int out, double *bufs, double2 *ckpt) {
    const unsigned lane = threadIdx.x & 31u;
    Particle p[K];
    uint64_t id[K];
    bool live[K];
    bool any = false;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const uint32_t e = start + uint32_t(j) * 32u + lane;
        live[j] = e < st.live;
        const uint64_t slot = set.list_offset + (live[j] ? e : 0u);
        id[j] = b.list_idx[in][slot];
        p[j] = dev::make_particle(b.list_x[in][slot], b.list_px[in][slot], b.list_y[in][slot],
                                  b.list_py[in][slot]);
        // Slots without a live particle hold zeros, a fixed point of the map.
        if (!live[j]) p[j] = dev::make_particle(0.0, 0.0, 0.0, 0.0);
        any |= live[j];
    }
    const uint32_t turn0 = st.done, nt = st.turns;
    const double mu = set.mu;
    const dev::Barrier bar = dev::make_barrier<ARITH>(set.b2bits);
    bool warp_live = __any_sync(dev::kFullMask, any);
    const uint32_t n_stages = (nt + kStageTurns - 1) / kStageTurns;
    double next[kPerLane];
    if (warp_live && n_stages > 0) {
        stage_load(next, set.table, turn0, min(kStageTurns, nt), lane);
        stage_store(bufs, next, lane);
    }
    __syncwarp();
    for (uint32_t sg = 0; warp_live && sg < n_stages; ++sg) {
        const uint32_t k0 = sg * kStageTurns, kn_stage = min(kStageTurns, nt - k0);
        const bool more = sg + 1 < n_stages;
        if (more)
            stage_load(next, set.table, turn0 + k0 + kStageTurns,
                       min(kStageTurns, nt - k0 - kStageTurns), lane);
        const double *rec = bufs + (sg & 1u) * kStageTurns * 4u;
        // The stage's turns with no per-turn control flow, ORing every
        // coordinate's high word; one vote at the end.  Only a warp with a
        // coordinate at or above the bound of dev::small_or restores the
        // saved particles and redoes the stage with the per-turn test
        // (the scheme of the tracking kernel, track.cu turns_staged).
#pragma unroll
        for (int j = 0; j < K; ++j) {
            ckpt[2 * (j * 32 + int(lane))] = make_double2(p[j].x, p[j].px);
            ckpt[2 * (j * 32 + int(lane)) + 1] = make_double2(p[j].y, p[j].py);
        }
        uint32_t ored_stage = 0u;
        for (uint32_t kk = 0; kk < kn_stage; ++kk) {
            const double2 *q = reinterpret_cast<const double2 *>(rec + 4u * kk);
            const double2 q0 = q[0], q1 = q[1];
            const dev::Turn t{q0.x, q0.y, q1.x, q1.y};
#pragma unroll
            for (int j = 0; j < K; ++j) {
                dev::turn<ARITH, OCT, false>(p[j], t, mu);
                ored_stage |= dev::hi_or(p[j]);
            }
        }
        const bool redo = __any_sync(dev::kFullMask, !dev::small_or(ored_stage, bar));
        if (redo) {
#pragma unroll
            for (int j = 0; j < K; ++j) {
                const double2 a = ckpt[2 * (j * 32 + int(lane))];
                const double2 c = ckpt[2 * (j * 32 + int(lane)) + 1];
                p[j] = dev::make_particle(a.x, a.y, c.x, c.y);
            }
        }
        for (uint32_t kk = 0; redo && warp_live && kk < kn_stage; ++kk) {
            const uint32_t k = k0 + kk;
            const double2 *q = reinterpret_cast<const double2 *>(rec + 4u * kk);
            const double2 q0 = q[0], q1 = q[1];
            const dev::Turn t{q0.x, q0.y, q1.x, q1.y};
            // Per thread one OR of the coordinates' high words and one
            // compare; lost particles hold zeros (see track.cu turn_all).
            uint32_t ored = 0u;
#pragma unroll
            for (int j = 0; j < K; ++j) {
                dev::turn<ARITH, OCT, false>(p[j], t, mu);
                ored |= dev::hi_or(p[j]);
            }
            if (__any_sync(dev::kFullMask, !dev::small_or(ored, bar))) {
                bool still = false;
#pragma unroll
                for (int j = 0; j < K; ++j) {
                    if (live[j] && !dev::small_inside(p[j], bar) &&
                        !dev::inside<ARITH>(dev::radius_fma(p[j]), p[j], bar)) {
                        b.x[id[j]] = b.px[id[j]] = b.y[id[j]] = b.py[id[j]] = dev::quiet_nan();
                        b.steps[id[j]] = turn0 + k;
                        live[j] = false;
                        p[j] = dev::make_particle(0.0, 0.0, 0.0, 0.0);
                    }
                    still |= live[j];
                }
                warp_live = __any_sync(dev::kFullMask, still);
            }
        }
        // The other buffer was last read in the previous stage, which every
        // lane has finished.
        if (more) stage_store(bufs + ((sg + 1u) & 1u) * kStageTurns * 4u, next, lane);
        __syncwarp();
    }
    const bool final_chunk = turn0 + nt == set.n_turns;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        if (final_chunk) {
            if (live[j]) {
                b.x[id[j]] = p[j].x;
                b.px[id[j]] = p[j].px;
                b.y[id[j]] = p[j].y;
                b.py[id[j]] = p[j].py;
                b.steps[id[j]] = set.n_turns;
            }
            continue;
        }
        const unsigned m = __ballot_sync(dev::kFullMask, live[j]);
        if (m == 0u) continue;
        const int leader = __ffs(m) - 1;
        uint32_t off = 0;
        if (lane == unsigned(leader)) off = atomicAdd(&b.state[s].next, uint32_t(__popc(m)));
        off = __shfl_sync(dev::kFullMask, off, leader);
        if (live[j]) {
            const uint64_t slot = set.list_offset + off + __popc(m & ((1u << lane) - 1u));
            b.list_idx[out][slot] = id[j];
            b.list_x[out][slot] = p[j].x;
            b.list_px[out][slot] = p[j].px;
            b.list_y[out][slot] = p[j].y;
            b.list_py[out][slot] = p[j].py;
        }
    }
}

// Persistent: warps pop warp-tiles until the chunk's queue is empty.  One
// particle per thread fits 72 registers without spills: 7 blocks per SM.
template <int ARITH, int K>
__global__ void __launch_bounds__(kThreads, K == 1 ? 7 : 1) batch_chunk_kernel(BatchDev b) {
    __shared__ __align__(16) double stage_bufs[kWarps][2 * kStageTurns * 4];
    // Per warp, the particles {x, px}, {y, py} at the start of a stage.
    __shared__ __align__(16) double2 checkpoints[kWarps][2 * 32 * K];
    const unsigned lane = threadIdx.x & 31u;
    double *bufs = stage_bufs[threadIdx.x >> 5];
    double2 *ckpt = checkpoints[threadIdx.x >> 5];
    const uint32_t n_tiles = *b.n_tiles;
    const int in = int(*b.parity), out = 1 - in;
    while (true) {
        uint32_t item = 0;
        if (lane == 0) item = atomicAdd(b.next_item, 1u);
        item = __shfl_sync(dev::kFullMask, item, 0);
        if (item >= n_tiles) return;
        const uint32_t s = b.tile_set[item];
        const BatchStateDev st = b.state[s];
        const BatchSetDev &set = b.sets[s];
        const uint32_t start = (item - st.first_tile) * 32u * uint32_t(K);
        if (set.mu != 0.0)
            run_tile<ARITH, true, K>(b, set, st, s, start, in, out, bufs, ckpt);
        else
            run_tile<ARITH, false, K>(b, set, st, s, start, in, out, bufs, ckpt);
    }
}

}  // namespace

cudaError_t launch_batch_init(const BatchDev &b, cudaStream_t s) {
    if (b.n_total == 0) return cudaSuccess;
    batch_init_kernel<<<unsigned((b.n_total + 255) / 256), 256, 0, s>>>(b);
    return cudaGetLastError();
}

cudaError_t launch_batch_plan(const BatchDev &b, uint32_t done_len, uint32_t next_len,
                              cudaStream_t s) {
    batch_plan_kernel<<<1, kBatchMaxSets, 0, s>>>(b, done_len, next_len);
    return cudaGetLastError();
}

cudaError_t launch_batch_chunk(const BatchDev &b, int blocks, cudaStream_t s) {
    const int a = b.arith, k = b.per_thread;
#define HM_BATCH_LAUNCH(A, KK) batch_chunk_kernel<A, KK><<<blocks, kThreads, 0, s>>>(b)
    if (a == HM_ARITH_FAST) {
        if (k == 1) HM_BATCH_LAUNCH(HM_ARITH_FAST, 1);
        else if (k == 2) HM_BATCH_LAUNCH(HM_ARITH_FAST, 2);
        else HM_BATCH_LAUNCH(HM_ARITH_FAST, 4);
    } else {
        if (k == 1) HM_BATCH_LAUNCH(HM_ARITH_EXACT, 1);
        else if (k == 2) HM_BATCH_LAUNCH(HM_ARITH_EXACT, 2);
        else HM_BATCH_LAUNCH(HM_ARITH_EXACT, 4);
    }
#undef HM_BATCH_LAUNCH
    return cudaGetLastError();
}

int batch_chunk_blocks_per_sm(int arith, int per_thread) {
    int n = 0;
    cudaError_t e;
    if (arith == HM_ARITH_FAST)
        e = per_thread == 1   ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_chunk_kernel<HM_ARITH_FAST, 1>, kThreads, 0)
            : per_thread == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_chunk_kernel<HM_ARITH_FAST, 2>, kThreads, 0)
                              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_chunk_kernel<HM_ARITH_FAST, 4>, kThreads, 0);
    else
        e = per_thread == 1   ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_chunk_kernel<HM_ARITH_EXACT, 1>, kThreads, 0)
            : per_thread == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_chunk_kernel<HM_ARITH_EXACT, 2>, kThreads, 0)
                              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_chunk_kernel<HM_ARITH_EXACT, 4>, kThreads, 0);
    return e == cudaSuccess && n > 0 ? n : 1;
}

}  // namespace hm
