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

struct hm_batch {
    std::vector<hm_batch_set> params;
    std::vector<std::string> kinds;
    std::vector<uint64_t> offsets;  // particle offset of each set (n_sets + 1)
    uint64_t n_total = 0;
    uint32_t max_turns = 0;
    DeviceBuffer x0, px0, y0, py0, x, px, y, py, steps, particle_set;
    DeviceBuffer sets, state, tables, tile_set, counters;
    DeviceBuffer lists[2][5];
    hm::BatchDev dev{};
    int arith = HM_ARITH_EXACT;
    int per_thread = 2;
    uint32_t chunk0 = 512, chunk_max = 16384;
    int blocks = 0;
    bool loaded = false;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~hm_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (stream) cudaStreamDestroy(stream);
    }
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    std::vector<uint32_t> schedule() const {
        std::vector<uint32_t> lens;
        uint32_t done = 0, len = chunk0;
        while (done < max_turns) {
            const uint32_t l = std::min(len, max_turns - done);
            lens.push_back(l);
            done += l;
            len = std::min<uint32_t>(len * 2u, chunk_max);
        }
        return lens;
    }
};

namespace {

// Enqueues the whole batch on b->stream: reset from the initial
// conditions, collect, then chunks and plans.
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
    const std::vector<uint32_t> lens = b->schedule();
    uint32_t prev = 0;
    for (uint32_t len : lens) {
        HM_CUDA_TRY(hm::launch_batch_plan(b->dev, prev, len, s));
        HM_CUDA_TRY(hm::launch_batch_chunk(b->dev, b->blocks, s));
        prev = len;
    }
    HM_CUDA_TRY(hm::launch_batch_plan(b->dev, prev, 0, s));
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
    auto s = hm::upload(b->tables, records);
    std::vector<hm::BatchSetDev> sd(n_sets);
    std::vector<uint32_t> set_of(b->n_total);
    for (size_t k = 0; k < n_sets; ++k) {
        const hm_batch_set &p = sets[k];
        sd[k].table = b->tables.as<double>() + table_off[k];
        sd[k].list_offset = b->offsets[k];
        sd[k].n_particles = uint32_t(p.n_particles);
        sd[k].n_turns = p.n_turns;
        sd[k].mu = p.mu;
        const double b2 = p.barrier * p.barrier;
        sd[k].b2bits = 0;
        if (!std::isnan(b2)) std::memcpy(&sd[k].b2bits, &b2, sizeof(b2));
        std::fill(set_of.begin() + b->offsets[k], set_of.begin() + b->offsets[k + 1], uint32_t(k));
    }
    if (s == HM_OK) s = hm::upload(b->sets, sd);
    if (s == HM_OK) s = hm::upload(b->particle_set, set_of);
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
    if (s == HM_OK) s = b->tile_set.alloc((n / 32 + n_sets + 1) * sizeof(uint32_t));
    if (s == HM_OK) s = b->counters.alloc(256);
    if (s == HM_OK) {
        const cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) s = hm::cuda_fail(e, "cudaStreamCreate");
    }
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
    d.particle_set = b->particle_set.as<uint32_t>();
    d.n_total = n;
    d.sets = b->sets.as<hm::BatchSetDev>();
    d.state = b->state.as<hm::BatchStateDev>();
    d.n_sets = int(n_sets);
    for (int l = 0; l < 2; ++l) {
        d.list_idx[l] = b->lists[l][0].as<uint64_t>();
        d.list_x[l] = b->lists[l][1].as<double>();
        d.list_px[l] = b->lists[l][2].as<double>();
        d.list_y[l] = b->lists[l][3].as<double>();
        d.list_py[l] = b->lists[l][4].as<double>();
    }
    d.tile_set = b->tile_set.as<uint32_t>();
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
    b->drop_graph();
    return ok();
}

hm_status hm_batch_size(const hm_batch *b, uint64_t *n_total, uint32_t *n_chunks) {
    if (!b) return fail(HM_ERR_INVALID_ARG, "null batch");
    if (n_total) *n_total = b->n_total;
    if (n_chunks) *n_chunks = uint32_t(b->schedule().size());
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
