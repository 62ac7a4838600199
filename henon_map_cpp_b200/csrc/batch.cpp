// C ABI of batched heterogeneous tracking (hm_batch_*): host set-up, the
// chunk schedule and the CUDA graph that replays the whole batch.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "hm_internal.h"

using hm::DeviceBuffer;
using hm::fail;
using hm::ok;

// The sets are split into `n_groups` groups of about equal work (particles
// x turns), each tracked by its own chain of chunk launches on its own
// stream.  A chunk launch ends with a ramp-down in which its last tiles
// run while SMs empty; the chains run concurrently, so one group's
// ramp-down is filled by another group's tiles instead of idling until the
// next chunk.  The set metadata is stored group by group (position order);
// particles keep the caller's order.
//
// Each group's persistent chunk kernel gets a share of the device's resident
// blocks in proportion to the group's work, grid_share x (its particles x
// turns) / (all of them), at most the whole device.  Several groups'
// kernels then run side by side, each with more rounds of tiles per launch
// than one kernel spread over the whole device, so less of each launch is
// spent in its last, partly empty round; a group heavier than the others
// (one large set) still gets a proportionally larger grid.
struct hm_batch {
    std::vector<hm_batch_set> params;  // caller's order
    std::vector<std::string> kinds;
    std::vector<uint64_t> offsets;    // particle offset of each set (n_sets + 1), caller's order
    std::vector<uint64_t> table_off;  // offset of each set's records in `tables`
    uint64_t n_total = 0;
    uint32_t max_turns = 0;
    DeviceBuffer x0, px0, y0, py0, x, px, y, py, steps, particle_set;
    DeviceBuffer sets, state, tables, tile_set, counters;
    DeviceBuffer lists[2][5];
    hm::BatchDev dev{};  // all sets (reset and collection)
    int arith = HM_ARITH_EXACT;
    int per_thread = 1;
    uint32_t chunk0 = 512, chunk_max = 4096;
    double grid_share = 1.5;  // 0: every group's kernel spans the device
    int n_groups = 1;
    std::vector<uint32_t> order;        // position -> caller's set index
    std::vector<uint32_t> group_first;  // sets of group g: positions [first[g], first[g+1])
    std::vector<uint32_t> tile_first;   // tile-table region of each group
    int blocks = 0;
    bool loaded = false;
    cudaStream_t stream = nullptr;
    std::vector<cudaStream_t> group_streams;
    std::vector<cudaEvent_t> events;  // fork + one join per group
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~hm_batch() {
        drop_graph();
        drop_groups();
        if (stream) cudaStreamDestroy(stream);
    }
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    void drop_groups() {
        for (cudaEvent_t e : events) cudaEventDestroy(e);
        for (cudaStream_t g : group_streams) cudaStreamDestroy(g);
        events.clear();
        group_streams.clear();
    }
    std::vector<uint32_t> schedule(uint32_t turns) const {
        std::vector<uint32_t> lens;
        uint32_t done = 0, len = chunk0;
        while (done < turns) {
            const uint32_t l = std::min(len, turns - done);
            lens.push_back(l);
            done += l;
            len = std::min<uint32_t>(len * 2u, chunk_max);
        }
        return lens;
    }
    uint32_t group_turns(int g) const {
        uint32_t t = 0;
        for (uint32_t q = group_first[g]; q < group_first[g + 1]; ++q)
            t = std::max(t, params[order[q]].n_turns);
        return t;
    }
    // The chunk/plan view of group g: its sets, its tile table and counters.
    hm::BatchDev group_dev(int g) const {
        hm::BatchDev d = dev;
        d.sets = dev.sets + group_first[g];
        d.state = dev.state + group_first[g];
        d.n_sets = int(group_first[g + 1] - group_first[g]);
        d.tile_set = dev.tile_set + tile_first[g];
        d.n_tiles = counters.as<uint32_t>() + 4 * g;
        d.next_item = d.n_tiles + 1;
        d.parity = d.n_tiles + 2;
        return d;
    }
};

namespace {

constexpr int kMaxGroups = 16;

// Enqueues the whole batch on b->stream: reset from the initial
// conditions, collect, then one chain of plans and chunks per group,
// forked from and joined back into the main stream.
hm_status enqueue(hm_batch *b) {
    const cudaStream_t s = b->stream;
    const size_t nb = b->n_total * sizeof(double);
    HM_CUDA_TRY(cudaMemcpyAsync(b->x.ptr, b->x0.ptr, nb, cudaMemcpyDeviceToDevice, s));
    HM_CUDA_TRY(cudaMemcpyAsync(b->px.ptr, b->px0.ptr, nb, cudaMemcpyDeviceToDevice, s));
    HM_CUDA_TRY(cudaMemcpyAsync(b->y.ptr, b->y0.ptr, nb, cudaMemcpyDeviceToDevice, s));
    HM_CUDA_TRY(cudaMemcpyAsync(b->py.ptr, b->py0.ptr, nb, cudaMemcpyDeviceToDevice, s));
    HM_CUDA_TRY(cudaMemsetAsync(b->steps.ptr, 0, b->n_total * sizeof(uint32_t), s));
    HM_CUDA_TRY(cudaMemsetAsync(b->state.ptr, 0, b->params.size() * sizeof(hm::BatchStateDev), s));
    HM_CUDA_TRY(hm::launch_batch_init(b->dev, s));
    HM_CUDA_TRY(cudaEventRecord(b->events[0], s));
    std::vector<double> work(size_t(b->n_groups), 0.0);
    double total = 0.0;
    for (int g = 0; g < b->n_groups; ++g) {
        for (uint32_t q = b->group_first[g]; q < b->group_first[g + 1]; ++q) {
            const hm_batch_set &p = b->params[b->order[q]];
            work[size_t(g)] += double(p.n_particles) * double(p.n_turns);
        }
        total += work[size_t(g)];
    }
    for (int g = 0; g < b->n_groups; ++g) {
        const cudaStream_t gs = b->group_streams[size_t(g)];
        const hm::BatchDev d = b->group_dev(g);
        int blocks = b->blocks;
        if (b->grid_share > 0.0 && total > 0.0) {
            const double share = b->grid_share * work[size_t(g)] / total;
            blocks = std::max(1, std::min(b->blocks, int(std::ceil(share * b->blocks))));
        }
        HM_CUDA_TRY(cudaStreamWaitEvent(gs, b->events[0], 0));
        uint32_t prev = 0;
        for (uint32_t len : b->schedule(b->group_turns(g))) {
            HM_CUDA_TRY(hm::launch_batch_plan(d, prev, len, gs));
            HM_CUDA_TRY(hm::launch_batch_chunk(d, blocks, gs));
            prev = len;
        }
        HM_CUDA_TRY(hm::launch_batch_plan(d, prev, 0, gs));
        HM_CUDA_TRY(cudaEventRecord(b->events[size_t(g) + 1], gs));
        HM_CUDA_TRY(cudaStreamWaitEvent(s, b->events[size_t(g) + 1], 0));
    }
    return ok();
}

// Splits the sets into n groups of about equal work (longest processing
// time first); group g is the position range [group_first[g],
// group_first[g + 1]).
void assign_groups(hm_batch *b, int n) {
    const size_t n_sets = b->params.size();
    n = std::max(1, std::min<int>(n, int(n_sets)));
    std::vector<uint32_t> by_work(n_sets);
    for (size_t k = 0; k < n_sets; ++k) by_work[k] = uint32_t(k);
    auto work = [b](uint32_t k) {
        return double(b->params[k].n_particles) * double(b->params[k].n_turns);
    };
    std::stable_sort(by_work.begin(), by_work.end(),
                     [&](uint32_t p, uint32_t q) { return work(p) > work(q); });
    const size_t groups = size_t(n);
    std::vector<double> load(groups, 0.0);
    std::vector<std::vector<uint32_t>> members(groups);
    for (uint32_t k : by_work) {
        const size_t g = size_t(std::min_element(load.begin(), load.end()) - load.begin());
        load[g] += work(k);
        members[g].push_back(k);
    }
    b->n_groups = n;
    b->order.clear();
    b->group_first.assign(1, 0);
    for (auto &m : members) {
        std::sort(m.begin(), m.end());
        b->order.insert(b->order.end(), m.begin(), m.end());
        b->group_first.push_back(uint32_t(b->order.size()));
    }
}

// Groups the sets and uploads what depends on the grouping: set metadata
// in position order, each particle's position, the groups' tile tables,
// one stream per group.
hm_status layout(hm_batch *b, int groups) {
    b->drop_graph();
    b->drop_groups();
    assign_groups(b, std::min(groups, kMaxGroups));
    const size_t n_sets = b->params.size();
    std::vector<hm::BatchSetDev> sd(n_sets);
    std::vector<uint32_t> set_of(b->n_total);
    for (size_t q = 0; q < n_sets; ++q) {
        const size_t k = b->order[q];
        const hm_batch_set &p = b->params[k];
        sd[q].table = b->tables.as<double>() + b->table_off[k];
        sd[q].list_offset = b->offsets[k];
        sd[q].n_particles = uint32_t(p.n_particles);
        sd[q].n_turns = p.n_turns;
        sd[q].mu = p.mu;
        const double b2 = p.barrier * p.barrier;
        sd[q].b2bits = 0;
        if (!std::isnan(b2)) std::memcpy(&sd[q].b2bits, &b2, sizeof(b2));
        std::fill(set_of.begin() + b->offsets[k], set_of.begin() + b->offsets[k + 1], uint32_t(q));
    }
    // Tile-table capacity of each group: one warp-tile per 32 particles at
    // most, plus a partial tile per set.
    b->tile_first.assign(1, 0);
    for (int g = 0; g < b->n_groups; ++g) {
        uint64_t cap = 1;
        for (uint32_t q = b->group_first[g]; q < b->group_first[g + 1]; ++q)
            cap += b->params[b->order[q]].n_particles / 32 + 1;
        b->tile_first.push_back(uint32_t(b->tile_first.back() + cap));
    }
    HM_TRY(hm::upload(b->sets, sd));
    HM_TRY(hm::upload(b->particle_set, set_of));
    HM_TRY(b->tile_set.alloc(size_t(b->tile_first.back()) * sizeof(uint32_t)));
    for (int g = 0; g < b->n_groups; ++g) {
        cudaStream_t gs = nullptr;
        HM_CUDA_TRY(cudaStreamCreateWithFlags(&gs, cudaStreamNonBlocking));
        b->group_streams.push_back(gs);
    }
    for (int q = 0; q <= b->n_groups; ++q) {
        cudaEvent_t ev = nullptr;
        HM_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        b->events.push_back(ev);
    }
    b->dev.sets = b->sets.as<hm::BatchSetDev>();
    b->dev.particle_set = b->particle_set.as<uint32_t>();
    b->dev.tile_set = b->tile_set.as<uint32_t>();
    return ok();
}

}  // namespace

extern "C" {

hm_status hm_batch_create(size_t n_sets, const hm_batch_set *sets, hm_batch **out) {
    if (!out) return fail(HM_ERR_INVALID_ARG, "null output handle");
    *out = nullptr;
    if (n_sets == 0 || !sets) return fail(HM_ERR_INVALID_ARG, "a batch needs at least one set");
    if (n_sets > size_t(hm::kBatchMaxSets))
        return fail(HM_ERR_INVALID_ARG, "too many parameter sets (max 1024)");
    auto *b = new hm_batch();
    b->params.assign(sets, sets + n_sets);
    b->offsets.assign(1, 0);
    std::vector<double> records;
    std::vector<uint64_t> table_off;
    for (size_t k = 0; k < n_sets; ++k) {
        const hm_batch_set &p = sets[k];
        b->kinds.emplace_back(p.modulation_kind ? p.modulation_kind : "sps");
        std::vector<double> wx, wy;
        hm_status s = hm::modulation(b->kinds.back(), p.n_turns, p.omega_x, p.omega_y, p.omega_0,
                                     p.epsilon, p.offset, wx, wy);
        if (s != HM_OK) {
            delete b;
            return s;
        }
        table_off.push_back(records.size());
        for (size_t i = 0; i < wx.size(); ++i) {
            // sin/cos of omega(n) with the host libm (src/henon.cu:2679-2682)
            records.push_back(std::sin(wx[i]));
            records.push_back(std::cos(wx[i]));
            records.push_back(std::sin(wy[i]));
            records.push_back(std::cos(wy[i]));
        }
        b->offsets.push_back(b->offsets.back() + p.n_particles);
        b->max_turns = std::max(b->max_turns, p.n_turns);
    }
    b->n_total = b->offsets.back();
    if (b->n_total > 0xffffffffULL) {
        delete b;
        return fail(HM_ERR_INVALID_ARG, "too many particles in the batch (max 2^32-1)");
    }
    b->table_off = table_off;
    auto s = hm::upload(b->tables, records);
    const size_t n = b->n_total;
    DeviceBuffer *dbl[8] = {&b->x0, &b->px0, &b->y0, &b->py0, &b->x, &b->px, &b->y, &b->py};
    for (auto *d : dbl)
        if (s == HM_OK) s = d->alloc(n * sizeof(double));
    if (s == HM_OK) s = b->steps.alloc(n * sizeof(uint32_t));
    for (int l = 0; l < 2 && s == HM_OK; ++l) {
        s = b->lists[l][0].alloc(n * sizeof(uint64_t));
        for (int f = 1; f < 5 && s == HM_OK; ++f) s = b->lists[l][f].alloc(n * sizeof(double));
    }
    if (s == HM_OK) s = b->state.alloc(n_sets * sizeof(hm::BatchStateDev));
    if (s == HM_OK) s = b->counters.alloc(size_t(4 * kMaxGroups) * sizeof(uint32_t));
    if (s == HM_OK) {
        const cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) s = hm::cuda_fail(e, "cudaStreamCreate");
    }
    if (s == HM_OK) s = layout(b, kMaxGroups);
    if (s != HM_OK) {
        delete b;
        return s;
    }
    hm::BatchDev &d = b->dev;
    d.x = b->x.as<double>();
    d.px = b->px.as<double>();
    d.y = b->y.as<double>();
    d.py = b->py.as<double>();
    d.steps = b->steps.as<uint32_t>();
    d.n_total = n;
    d.state = b->state.as<hm::BatchStateDev>();
    d.n_sets = int(n_sets);
    for (int l = 0; l < 2; ++l) {
        d.list_idx[l] = b->lists[l][0].as<uint64_t>();
        d.list_x[l] = b->lists[l][1].as<double>();
        d.list_px[l] = b->lists[l][2].as<double>();
        d.list_y[l] = b->lists[l][3].as<double>();
        d.list_py[l] = b->lists[l][4].as<double>();
    }
    // sets, particle_set and tile_set were set by layout(); the counters of
    // `dev` are group 0's (the groups' chains use group_dev).
    d.n_tiles = b->counters.as<uint32_t>();
    d.next_item = d.n_tiles + 1;
    d.parity = d.n_tiles + 2;
    d.arith = b->arith;
    d.per_thread = b->per_thread;
    *out = b;
    return ok();
}

hm_status hm_batch_destroy(hm_batch *b) {
    delete b;
    return ok();
}

hm_status hm_batch_configure(hm_batch *b, hm_arith arith, int per_thread, uint32_t chunk0,
                             uint32_t chunk_max) {
    if (!b) return fail(HM_ERR_INVALID_ARG, "null batch");
    if (arith != HM_ARITH_EXACT && arith != HM_ARITH_FAST)
        return fail(HM_ERR_INVALID_ARG, "unknown arithmetic mode");
    if (per_thread != 1 && per_thread != 2 && per_thread != 4)
        return fail(HM_ERR_INVALID_ARG, "particles per thread must be 1, 2 or 4");
    if (chunk0 == 0 || chunk_max < chunk0) return fail(HM_ERR_INVALID_ARG, "need 0 < chunk0 <= chunk_max");
    b->arith = arith;
    b->per_thread = per_thread;
    b->chunk0 = chunk0;
    b->chunk_max = chunk_max;
    b->dev.arith = arith;
    b->dev.per_thread = per_thread;
    b->blocks = 0;  // the resident-block count depends on the kernel variant
    b->drop_graph();
    return ok();
}

hm_status hm_batch_set_grid_share(hm_batch *b, double share) {
    if (!b) return fail(HM_ERR_INVALID_ARG, "null batch");
    if (!(share >= 0.0) || std::isinf(share))
        return fail(HM_ERR_INVALID_ARG, "grid share must be finite and >= 0");
    b->grid_share = share;
    b->drop_graph();
    return ok();
}

hm_status hm_batch_set_groups(hm_batch *b, int groups) {
    if (!b) return fail(HM_ERR_INVALID_ARG, "null batch");
    if (groups < 1 || groups > kMaxGroups)
        return fail(HM_ERR_INVALID_ARG, "groups must be 1.." + std::to_string(kMaxGroups));
    return layout(b, groups);
}

hm_status hm_batch_size(const hm_batch *b, uint64_t *n_total, uint32_t *n_chunks) {
    if (!b) return fail(HM_ERR_INVALID_ARG, "null batch");
    if (n_total) *n_total = b->n_total;
    if (n_chunks) *n_chunks = uint32_t(b->schedule(b->max_turns).size());
    return ok();
}

hm_status hm_batch_load(hm_batch *b, const double *x, const double *px, const double *y,
                        const double *py) {
    if (!b) return fail(HM_ERR_INVALID_ARG, "null batch");
    const size_t nb = b->n_total * sizeof(double);
    if (nb && (!x || !px || !y || !py)) return fail(HM_ERR_INVALID_ARG, "null coordinates");
    if (nb) {
        HM_CUDA_TRY(cudaMemcpy(b->x0.ptr, x, nb, cudaMemcpyHostToDevice));
        HM_CUDA_TRY(cudaMemcpy(b->px0.ptr, px, nb, cudaMemcpyHostToDevice));
        HM_CUDA_TRY(cudaMemcpy(b->y0.ptr, y, nb, cudaMemcpyHostToDevice));
        HM_CUDA_TRY(cudaMemcpy(b->py0.ptr, py, nb, cudaMemcpyHostToDevice));
    }
    b->loaded = true;
    return ok();
}

hm_status hm_batch_run(hm_batch *b, int use_graph) {
    if (!b) return fail(HM_ERR_INVALID_ARG, "null batch");
    if (!b->loaded) return fail(HM_ERR_INVALID_ARG, "load the initial conditions first");
    if (b->n_total == 0) return ok();
    if (b->blocks == 0) {
        int dev = 0, sms = 0;
        HM_CUDA_TRY(cudaGetDevice(&dev));
        HM_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        b->blocks = sms * hm::batch_chunk_blocks_per_sm(b->arith, b->per_thread);
    }
    if (!use_graph) {
        HM_TRY(enqueue(b));
        HM_CUDA_TRY(cudaStreamSynchronize(b->stream));
        return ok();
    }
    if (!b->exec) {
        HM_CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        const hm_status s = enqueue(b);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (s != HM_OK) {
            if (g) cudaGraphDestroy(g);
            return s;
        }
        HM_CUDA_TRY(e);
        b->graph = g;
        HM_CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
    }
    HM_CUDA_TRY(cudaGraphLaunch(b->exec, b->stream));
    HM_CUDA_TRY(cudaStreamSynchronize(b->stream));
    return ok();
}

hm_status hm_batch_get(const hm_batch *b, hm_field field, void *host_out) {
    if (!b) return fail(HM_ERR_INVALID_ARG, "null batch");
    const DeviceBuffer *src = nullptr;
    size_t elem = 8;
    switch (field) {
        case HM_FIELD_X: src = &b->x; break;
        case HM_FIELD_PX: src = &b->px; break;
        case HM_FIELD_Y: src = &b->y; break;
        case HM_FIELD_PY: src = &b->py; break;
        case HM_FIELD_STEPS: src = &b->steps; elem = 4; break;
        default: return fail(HM_ERR_INVALID_ARG, "field must be x, px, y, py or steps");
    }
    if (b->n_total == 0) return ok();
    if (!host_out) return fail(HM_ERR_INVALID_ARG, "null output");
    HM_CUDA_TRY(cudaMemcpy(host_out, src->ptr, b->n_total * elem, cudaMemcpyDeviceToHost));
    return ok();
}

}  // extern "C"
