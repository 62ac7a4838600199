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

// Records [lo, lo + kn) of a table into a warp's stage buffer with
// asynchronous 16-byte copies (cp.async, no registers held): chunk c of the
// stage (two doubles) is table[4 lo + 2c ..]; chunks past the kn records
// are zero-filled without reading.  Sources are 16-byte aligned (32-byte
// records of a 256-byte-aligned table), and so is the buffer.
constexpr int kChunksPerLane = int(kStageTurns) * 4 / 2 / 32;
static_assert(kChunksPerLane * 32 * 2 == int(kStageTurns) * 4, "stage must split evenly");

__device__ __forceinline__ void stage_async(double *buf, const double *table, uint32_t lo,
                                            uint32_t kn, unsigned lane) {
#pragma unroll
    for (int q = 0; q < kChunksPerLane; ++q) {
        const uint32_t c = lane + 32u * uint32_t(q);
        const bool in = c < 2u * kn;
        const double *src = table + (in ? 4u * size_t(lo) + 2u * c : 0u);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(dev::smem_addr(buf + 2u * c)),
                     "l"(src), "r"(in ? 16u : 0u)
                     : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// This lane's copies have landed; with the __syncwarp after it, every
// lane's.
__device__ __forceinline__ void stage_wait() {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
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
    // A particle's slot in the input list is recomputed from the tile, and
    // its 64-bit index read back from the list only when it is written out
    // (lost, final chunk) or appended to the next list: fewer registers.
    auto slot_of = [&](int j) {
        return set.list_offset + start + uint32_t(j) * 32u + lane;
    };
    Particle p[K];
    bool live[K];
    bool any = false;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const uint32_t e = start + uint32_t(j) * 32u + lane;
        live[j] = e < st.live;
        const uint64_t slot = live[j] ? slot_of(j) : set.list_offset;
        p[j] = dev::make_particle(b.list_x[in][slot], b.list_px[in][slot], b.list_y[in][slot],
                                  b.list_py[in][slot]);
        // Slots without a live particle hold zeros, a fixed point of the map.
        if (!live[j]) p[j] = dev::make_particle(0.0, 0.0, 0.0, 0.0);
        any |= live[j];
    }
    const uint32_t turn0 = st.done, nt = st.turns;
    const double mu = set.mu;
    // The common path needs only the coordinate bound of the barrier test;
    // the rare per-turn redo rebuilds the whole test from b2bits.
    const uint32_t small_hi = dev::make_barrier<ARITH>(set.b2bits).small_hi;
    bool warp_live = __any_sync(dev::kFullMask, any);
    const uint32_t n_stages = (nt + kStageTurns - 1) / kStageTurns;
    if (warp_live && n_stages > 0) stage_async(bufs, set.table, turn0, min(kStageTurns, nt), lane);
    stage_wait();
    __syncwarp();
    for (uint32_t sg = 0; warp_live && sg < n_stages; ++sg) {
        const uint32_t k0 = sg * kStageTurns, kn_stage = min(kStageTurns, nt - k0);
        const bool more = sg + 1 < n_stages;
        // The other buffer was last read in the previous stage, which every
        // lane has finished.
        if (more)
            stage_async(bufs + ((sg + 1u) & 1u) * kStageTurns * 4u, set.table,
                        turn0 + k0 + kStageTurns, min(kStageTurns, nt - k0 - kStageTurns), lane);
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
        // (small_or with the bound alone: the OR of the high words, sign
        // masked, against the coordinate bound)
        const bool redo = __any_sync(dev::kFullMask, (ored_stage & 0x7fffffffu) >= small_hi);
        if (redo) {
#pragma unroll
            for (int j = 0; j < K; ++j) {
                const double2 a = ckpt[2 * (j * 32 + int(lane))];
                const double2 c = ckpt[2 * (j * 32 + int(lane)) + 1];
                p[j] = dev::make_particle(a.x, a.y, c.x, c.y);
            }
        }
        const dev::Barrier bar = dev::make_barrier<ARITH>(set.b2bits);
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
                        const uint64_t id = b.list_idx[in][slot_of(j)];
                        b.x[id] = b.px[id] = b.y[id] = b.py[id] = dev::quiet_nan();
                        b.steps[id] = turn0 + k;
                        live[j] = false;
                        p[j] = dev::make_particle(0.0, 0.0, 0.0, 0.0);
                    }
                    still |= live[j];
                }
                warp_live = __any_sync(dev::kFullMask, still);
            }
        }
        // The next stage's copies have landed.
        stage_wait();
        __syncwarp();
    }
    // No copy may still be in flight when the warp moves to its next tile
    // (a stage left early by an all-lost warp).
    stage_wait();
    __syncwarp();
    const bool final_chunk = turn0 + nt == set.n_turns;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        if (final_chunk) {
            if (live[j]) {
                const uint64_t id = b.list_idx[in][slot_of(j)];
                b.x[id] = p[j].x;
                b.px[id] = p[j].px;
                b.y[id] = p[j].y;
                b.py[id] = p[j].py;
                b.steps[id] = set.n_turns;
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
            b.list_idx[out][slot] = b.list_idx[in][slot_of(j)];
            b.list_x[out][slot] = p[j].x;
            b.list_px[out][slot] = p[j].px;
            b.list_y[out][slot] = p[j].y;
            b.list_py[out][slot] = p[j].py;
        }
    }
}

// Persistent: warps pop warp-tiles until the chunk's queue is empty.  With
// the turn records copied by cp.async (no staging registers), particle
// slots recomputed from the tile and only the barrier's coordinate bound in
// registers, one particle per thread fits 64 registers (8 blocks per SM)
// and two fit 90 (5 blocks per SM).
template <int ARITH, int K>
__global__ void __launch_bounds__(kThreads, K == 1 ? 8 : (K == 2 ? 5 : 1))
    batch_chunk_kernel(BatchDev b) {
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
