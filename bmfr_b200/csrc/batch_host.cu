// batch_host.cu — the many-stream engine of include/bmfr_batch.h: stream
// slots with their HBM histories, the per-step description, the CUDA graph
// of a step, and the autotuner.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "batch.cuh"
#include "bmfr_batch.h"
#include "status.h"

using bmfr::cuda_fail;
using bmfr::fail;

namespace {

struct StreamSlot {
    bool used = false;    // taken (possibly still being allocated)
    bool ready = false;   // allocated: steps may name it
    int width = 0, height = 0;
    bmfr::Geometry g{};
    int frame = 0;
    bool own_inputs = false;
    size_t bytes = 0;
    void* base = nullptr;   // one pool allocation holds every buffer below
    // histories (HistT per the batch's half_history) and per-frame buffers
    void* noisy_acc[2] = {nullptr, nullptr};
    void* acc_filt[2] = {nullptr, nullptr};
    void* result[2] = {nullptr, nullptr};
    uint8_t* spp[2] = {nullptr, nullptr};
    float2* prev_pix = nullptr;
    uint8_t* accept = nullptr;
    float* tone_mapped = nullptr;
    float* result_f32 = nullptr;
    float* weights = nullptr;
    float* mins_maxs = nullptr;
    float* noise = nullptr;
    void* tmp = nullptr;   // staged pipeline: the stream's tmp_data
    // own input slots
    float* normals[2] = {nullptr, nullptr};
    float* positions[2] = {nullptr, nullptr};
    float* albedo = nullptr;
    float* noisy = nullptr;
};

// Lays the stream's buffers out from `base` (256-byte aligned pieces) and
// returns the total size; with base == nullptr only the size is computed.
size_t carve(StreamSlot& s, const bmfr_params& p, int w, int h, bool own_inputs, char* base) {
    const bmfr::Geometry g = bmfr::make_geometry(w, h);
    const size_t px = (size_t)w * h;
    const size_t hist = px * 3 * (p.half_history ? 2 : 4);
    size_t off = 0;
    auto take = [&](size_t n, auto** ptr) {
        *ptr = base ? reinterpret_cast<std::remove_pointer_t<decltype(ptr)>>(base + off) : nullptr;
        off += (n + 255) & ~size_t(255);
    };
    for (int i = 0; i < 2; ++i) {
        take(hist, &s.noisy_acc[i]);
        take(hist, &s.acc_filt[i]);
        take(hist, &s.result[i]);
        take(px, &s.spp[i]);
    }
    take(px * 8, &s.prev_pix);
    take(px, &s.accept);
    take(px * 12, &s.tone_mapped);
    take(px * 12, &s.result_f32);
    take((size_t)g.blocks * bmfr::kFeatures * 3 * 4, &s.weights);
    take((size_t)g.blocks * bmfr::kScaled * 2 * 4, &s.mins_maxs);
    take(bmfr::kNoiseTableBytes, &s.noise);
    if (p.pipeline == BMFR_PIPELINE_STAGED)
        take((size_t)g.MW * g.MH * bmfr::kBuffers * (p.use_half_precision_in_tmp_data ? 2 : 4), &s.tmp);
    if (own_inputs) {
        for (int i = 0; i < 2; ++i) {
            take(px * 12, &s.normals[i]);
            take(px * 12, &s.positions[i]);
        }
        take(px * 12, &s.albedo);
        take(px * 12, &s.noisy);
    }
    return off;
}

size_t stream_bytes(const bmfr_params& p, int w, int h, bool own_inputs) {
    StreamSlot tmp;
    return carve(tmp, p, w, h, own_inputs, nullptr);
}

}  // namespace

// Worker CUDA streams of the staged step: the listed streams' kernels are
// spread over them so that the kernels of small streams run side by side.
constexpr int kStepWorkers = 8;

struct bmfr_batch {
    // Guards the slot table, `used` and `last`: streams may be added and
    // removed from other threads while a step is being formed.
    mutable std::mutex mu;
    bmfr_params p{};
    int device = 0;
    int sms = 0;
    size_t budget = 0, used = 0;
    std::vector<StreamSlot> slots = std::vector<StreamSlot>(BMFR_BATCH_MAX_STREAMS);
    bmfr::BatchTuning tuning{0, 30, 32, 0, 0};
    int block_occupancy = 1;
    bmfr::BatchStepDesc* d_desc = nullptr;
    bmfr::BatchStepDesc* h_desc[2] = {nullptr, nullptr};
    int* d_counters = nullptr;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    bool graphs_valid = false;
    // Stream memory comes from a device pool in stream order on mem_stream,
    // so that streams join and leave without a device-wide synchronisation;
    // steps wait for mem_ready (the last allocation and its zeroing).
    cudaMemPool_t pool = nullptr;
    cudaStream_t mem_stream = nullptr;
    cudaEvent_t mem_ready = nullptr;
    int next = 0;
    int last = -1;
    // staged step: workers, the fork and join events, the fitter's status word
    cudaStream_t workers[kStepWorkers] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[kStepWorkers] = {};
    int* d_status = nullptr;
};

namespace {

int check_batch(const bmfr_batch* b) {
    if (!b) return fail(BMFR_E_INVALID, "batch is NULL");
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev != b->device)
        return fail(BMFR_E_STATE, "the current CUDA device is not the batch's device");
    return BMFR_OK;
}

int check_slot(const bmfr_batch* b, int slot) {
    if (slot < 0 || slot >= BMFR_BATCH_MAX_STREAMS || !b->slots[slot].used || !b->slots[slot].ready)
        return fail(BMFR_E_NOT_FOUND, "no stream in slot " + std::to_string(slot));
    return BMFR_OK;
}

// Returns the slot's memory to the pool once every step launched so far is
// done with it (steps run in order, so the last one is enough).
void free_slot(bmfr_batch* b, StreamSlot& s) {
    if (s.base) {
        if (b->last >= 0) cudaStreamWaitEvent(b->mem_stream, b->done[b->last], 0);
        cudaFreeAsync(s.base, b->mem_stream);
    }
    b->used -= s.bytes;
    s = StreamSlot();
}

void destroy_graphs(bmfr_batch* b) {
    for (int k = 0; k < 2; ++k) {
        if (b->graph[k]) cudaGraphExecDestroy(b->graph[k]);
        b->graph[k] = nullptr;
    }
    b->graphs_valid = false;
}

// Captures the fused step: description upload, queue reset, noise tables,
// the block queue and the TAA tiles.  One graph per pinned description
// buffer.
int build_graphs(bmfr_batch* b) {
    for (cudaEvent_t e : b->done)
        if (e) cudaEventSynchronize(e);
    destroy_graphs(b);
    cudaStream_t cs;
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "batch capture stream");
    const bool half_tmp = b->p.use_half_precision_in_tmp_data != 0;
    int ctas = b->tuning.block_ctas_per_sm > 0 ? std::min(b->tuning.block_ctas_per_sm, b->block_occupancy)
                                               : b->block_occupancy;
    ctas = std::max(ctas, 1);
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
        cudaGraph_t graph = nullptr;
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) break;
        e = cudaMemcpyAsync(b->d_desc, b->h_desc[k], sizeof(bmfr::BatchStepDesc), cudaMemcpyHostToDevice, cs);
        if (e == cudaSuccess) e = cudaMemsetAsync(b->d_counters, 0, 2 * sizeof(int), cs);
        if (e == cudaSuccess) e = bmfr::launch_batch_noise(b->d_desc, BMFR_BATCH_MAX_STREAMS, cs);
        const bool pixel_pass = b->tuning.pixel_pass != 0;
        if (e == cudaSuccess)
            e = bmfr::launch_batch_blocks(b->d_desc, b->d_counters, b->p.fp32_qr, half_tmp,
                                          b->p.half_history != 0, b->tuning.staging_depth, ctas * b->sms,
                                          !pixel_pass, cs);
        if (e == cudaSuccess && pixel_pass) e = bmfr::launch_batch_wsacc(b->d_desc, b->p.half_history != 0, b->sms, cs);
        if (e == cudaSuccess) e = bmfr::launch_batch_taa(b->d_desc, b->p.half_history != 0, b->tuning, b->sms, cs);
        cudaError_t e2 = cudaStreamEndCapture(cs, &graph);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&b->graph[k], graph, 0);
        if (graph) cudaGraphDestroy(graph);
    }
    cudaStreamDestroy(cs);
    if (e != cudaSuccess) {
        destroy_graphs(b);
        return cuda_fail(e, "batch graph capture");
    }
    b->graphs_valid = true;
    return BMFR_OK;
}

bmfr::AccumArgs step_args(const bmfr_batch* b, const float* m, const float* off, int frame) {
    bmfr::AccumArgs a;
    std::memcpy(a.m, m, sizeof a.m);
    a.off_x = off[0];
    a.off_y = off[1];
    a.pos_lim2 = b->p.position_limit_squared;
    a.nrm_lim2 = b->p.normal_limit_squared;
    a.blend_alpha = b->p.blend_alpha;
    a.frame = frame;
    a.use_half = b->p.use_half_precision_in_tmp_data ? 1 : 0;
    return a;
}

// Fills description buffer k for the listed streams.
int fill_desc(bmfr_batch* b, bmfr::BatchStepDesc* d, int n, const int* slots, const bmfr_frame_io* io,
              const float* matrices, const float* offsets) {
    const int tw = b->tuning.tile_w, th = b->tuning.tile_h;
    int blocks = 0, tiles = 0, px_tiles = 0;
    for (int i = 0; i < n; ++i) {
        StreamSlot& s = b->slots[slots[i]];
        const int f = s.frame, cur = f & 1, prv = cur ^ 1;
        const bmfr_frame_io* fi = io ? &io[i] : nullptr;
        const bool own = !fi || !fi->albedo;
        if (own && !s.own_inputs)
            return fail(BMFR_E_INVALID, "stream " + std::to_string(slots[i]) + " has no input slots; pass io");
        bmfr::BatchStreamJob& J = d->s[i];
        J.job.g = s.g;
        J.job.a = step_args(b, matrices + 16 * i, offsets + 2 * i, f);
        J.job.nc = bmfr::make_noise_const(b->p.noise_amount);
        J.job.second_alpha = b->p.second_blend_alpha;
        bmfr::FusedBuffers& fb = J.job.fb;
        fb.cur_n = own ? s.normals[cur] : fi->normals;
        fb.prev_n = own ? s.normals[prv] : fi->previous_normals;
        fb.cur_p = own ? s.positions[cur] : fi->positions;
        fb.prev_p = own ? s.positions[prv] : fi->previous_positions;
        fb.noisy_in = own ? s.noisy : fi->noisy;
        fb.albedo = own ? s.albedo : fi->albedo;
        if (!fb.cur_n || !fb.cur_p || !fb.noisy_in || !fb.albedo)
            return fail(BMFR_E_INVALID, "step: NULL input buffer");
        if (f > 0 && (!fb.prev_n || !fb.prev_p))
            return fail(BMFR_E_INVALID, "step: previous G-buffer missing");
        if (!fb.prev_n) fb.prev_n = fb.cur_n;   // frame 0 reads no history
        if (!fb.prev_p) fb.prev_p = fb.cur_p;
        fb.noisy_acc_cur = s.noisy_acc[cur];
        fb.noisy_acc_prev = s.noisy_acc[prv];
        fb.prev_spp = s.spp[prv];
        fb.cur_spp = s.spp[cur];
        fb.prev_pix = s.prev_pix;
        fb.accept = s.accept;
        fb.tone_mapped = s.tone_mapped;
        fb.acc_prev = s.acc_filt[prv];
        fb.acc_cur = s.acc_filt[cur];
        fb.weights = s.weights;
        fb.mins_maxs = s.mins_maxs;
        fb.noise = s.noise;
        J.block_start = blocks;
        J.tile_start = tiles;
        J.tiles_x = (s.width + tw - 1) / tw;
        J.px_tile_start = px_tiles;
        J.px_tiles_x = (s.width + 31) / 32;
        px_tiles += J.px_tiles_x * ((s.height + 7) / 8);
        J.taa_alpha = b->p.taa_blend_alpha;
        J.result_hist = s.result[cur];
        J.result_prev = s.result[prv];
        J.result_out = (fi && fi->result) ? fi->result : s.result_f32;
        J.tmp = s.tmp;
        blocks += s.g.blocks;
        tiles += J.tiles_x * ((s.height + th - 1) / th);
    }
    d->n_streams = n;
    d->n_blocks = blocks;
    d->n_tiles = tiles;
    d->n_px_tiles = px_tiles;
    d->tile_w = tw;
    return BMFR_OK;
}

// The staged step on the streams of description d (host copy): for each
// stream the plan's kernels — noise table, accumulation, fitter, weighted sum
// + filtered accumulation, TAA — with the stream's buffers, the same
// launches and arithmetic as a plan's frame, so each stream's output equals
// the plan's.  The streams are spread over the worker CUDA streams, largest
// first onto the least loaded worker, forked from and joined into `s`.
cudaError_t launch_staged_step(bmfr_batch* b, const bmfr::BatchStepDesc& d, cudaStream_t s) {
    const bool half_tmp = b->p.use_half_precision_in_tmp_data != 0;
    const bool half_hist = b->p.half_history != 0;
    std::vector<int> order(d.n_streams);
    for (int i = 0; i < d.n_streams; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int x, int y) {
        return d.s[x].job.g.blocks > d.s[y].job.g.blocks;
    });
    long long load[kStepWorkers] = {};
    bool used[kStepWorkers] = {};
    cudaError_t e = cudaEventRecord(b->fork, s);
    for (int i : order) {
        if (e != cudaSuccess) break;
        int w = 0;
        for (int k = 1; k < kStepWorkers; ++k)
            if (load[k] < load[w]) w = k;
        const bmfr::BatchStreamJob& J = d.s[i];
        const bmfr::FusedBuffers& fb = J.job.fb;
        const bmfr::Geometry& g = J.job.g;
        const int f = J.job.a.frame;
        cudaStream_t ws = b->workers[w];
        if (!used[w]) {
            e = cudaStreamWaitEvent(ws, b->fork, 0);
            used[w] = true;
        }
        load[w] += g.blocks;
        if (e == cudaSuccess) e = bmfr::launch_noise_table(f, const_cast<float*>(fb.noise), ws);
        if (e == cudaSuccess)
            e = bmfr::launch_accumulate_noisy(g, J.job.a, fb.prev_pix, fb.accept, fb.cur_n, fb.prev_n, fb.cur_p,
                                              fb.prev_p, fb.noisy_in, fb.noisy_acc_cur, fb.noisy_acc_prev, half_hist,
                                              fb.prev_spp, fb.cur_spp, J.tmp, ws);
        if (e == cudaSuccess)
            e = bmfr::launch_fitter(g, f, J.job.nc, J.tmp, half_tmp, b->p.fp32_qr, fb.weights, fb.mins_maxs,
                                    fb.noise, b->d_status, ws);
        if (e == cudaSuccess)
            e = bmfr::launch_weighted_sum_accumulate(g, f, J.job.second_alpha, fb.weights, fb.mins_maxs, fb.cur_n,
                                                     fb.cur_p, nullptr, fb.prev_pix, fb.accept, fb.albedo,
                                                     fb.tone_mapped, fb.cur_spp, fb.acc_prev, fb.acc_cur, half_hist,
                                                     ws);
        if (e == cudaSuccess)
            e = bmfr::launch_taa(g, f, J.taa_alpha, fb.prev_pix, fb.tone_mapped, J.result_hist, J.result_prev,
                                 J.result_out, half_hist, ws);
    }
    // Every worker that took work joins back to `s`, after an error too, so
    // what was queued stays ordered before the caller's later work; the
    // first error is the one returned.
    for (int w = 0; w < kStepWorkers; ++w) {
        if (!used[w]) continue;
        cudaError_t ej = cudaEventRecord(b->join[w], b->workers[w]);
        if (ej == cudaSuccess) ej = cudaStreamWaitEvent(s, b->join[w], 0);
        if (e == cudaSuccess) e = ej;
    }
    return e;
}

}  // namespace

extern "C" {

int bmfr_batch_stream_bytes(const bmfr_params* params, int width, int height, int own_inputs, size_t* bytes) {
    if (!params || !bytes) return fail(BMFR_E_INVALID, "NULL argument");
    *bytes = stream_bytes(*params, width, height, own_inputs != 0);
    return BMFR_OK;
}

int bmfr_batch_create(const bmfr_params* params, size_t memory_budget_bytes, bmfr_batch** out) {
    if (!params || !out) return fail(BMFR_E_INVALID, "NULL argument");
    *out = nullptr;
    if (!params->cache_tmp_data) return fail(BMFR_E_UNSUPPORTED, "cache_tmp_data = 0 is not served");
    if (params->fp32_qr < 0 || params->fp32_qr > 2) return fail(BMFR_E_INVALID, "fp32_qr must be 0, 1 or 2");
    if (params->pipeline != BMFR_PIPELINE_STAGED && params->pipeline != BMFR_PIPELINE_FUSED)
        return fail(BMFR_E_INVALID, "unknown pipeline");
    int dev = -1;
    if (cudaError_t e = cudaGetDevice(&dev); e != cudaSuccess) {
        cudaGetLastError();
        return cuda_fail(e, "no CUDA device");
    }
    bmfr_batch* b = new bmfr_batch;
    b->p = *params;
    b->device = dev;
    b->budget = memory_budget_bytes;
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
    const bool half_tmp = params->use_half_precision_in_tmp_data != 0;
    b->block_occupancy =
        std::max(1, params->pipeline == BMFR_PIPELINE_STAGED
                        ? 1
                        : bmfr::batch_block_occupancy(params->fp32_qr, half_tmp, params->half_history != 0));
    cudaError_t e = cudaMalloc(&b->d_desc, sizeof(bmfr::BatchStepDesc));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_status, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(b->d_status, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    for (int w = 0; w < kStepWorkers && e == cudaSuccess; ++w) {
        e = cudaStreamCreateWithFlags(&b->workers[w], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join[w], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaMalloc(&b->d_counters, 2 * sizeof(int));
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
        e = cudaMallocHost(&b->h_desc[k], sizeof(bmfr::BatchStepDesc));
        if (e == cudaSuccess) std::memset(b->h_desc[k], 0, sizeof(bmfr::BatchStepDesc));
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done[k], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        e = cudaMemPoolCreate(&b->pool, &props);
    }
    if (e == cudaSuccess) {
        // Freed stream memory stays with the pool for the next stream.
        uint64_t keep = ~uint64_t(0);
        e = cudaMemPoolSetAttribute(b->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->mem_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->mem_ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(b->mem_ready, b->mem_stream);
    if (e != cudaSuccess) {
        bmfr_batch_destroy(b);
        return cuda_fail(e, "batch allocation");
    }
    *out = b;
    return BMFR_OK;
}

int bmfr_batch_destroy(bmfr_batch* b) {
    if (!b) return BMFR_OK;
    for (cudaEvent_t e : b->done)
        if (e) cudaEventSynchronize(e);
    destroy_graphs(b);
    for (StreamSlot& s : b->slots)
        if (s.used) free_slot(b, s);
    for (int k = 0; k < 2; ++k) {
        if (b->h_desc[k]) cudaFreeHost(b->h_desc[k]);
        if (b->done[k]) cudaEventDestroy(b->done[k]);
    }
    if (b->mem_stream) cudaStreamSynchronize(b->mem_stream);
    if (b->mem_ready) cudaEventDestroy(b->mem_ready);
    if (b->mem_stream) cudaStreamDestroy(b->mem_stream);
    if (b->pool) cudaMemPoolDestroy(b->pool);
    for (int w = 0; w < kStepWorkers; ++w) {
        if (b->workers[w]) cudaStreamSynchronize(b->workers[w]);
        if (b->workers[w]) cudaStreamDestroy(b->workers[w]);
        if (b->join[w]) cudaEventDestroy(b->join[w]);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->d_status) cudaFree(b->d_status);
    if (b->d_desc) cudaFree(b->d_desc);
    if (b->d_counters) cudaFree(b->d_counters);
    delete b;
    return BMFR_OK;
}

int bmfr_batch_add_stream(bmfr_batch* b, int width, int height, int own_inputs, int* slot) {
    if (int st = check_batch(b)) return st;
    if (!slot) return fail(BMFR_E_INVALID, "slot is NULL");
    if (width < 32 || height < 32 || width > 16384 || height > 16384)
        return fail(BMFR_E_INVALID, "image size must be within [32, 16384]");
    const bmfr::Geometry g = bmfr::make_geometry(width, height);
    if (g.MW - 3 > 2 * width - 1 || g.MH - 3 > 2 * height - 1)
        return fail(BMFR_E_UNSUPPORTED, "image too small for the mirrored 16-pixel margin");
    const size_t bytes = stream_bytes(b->p, width, height, own_inputs != 0);
    int k = 0;
    {
        std::lock_guard<std::mutex> lk(b->mu);
        while (k < BMFR_BATCH_MAX_STREAMS && b->slots[k].used) ++k;
        if (k == BMFR_BATCH_MAX_STREAMS) return fail(BMFR_E_TOO_LARGE, "all stream slots are in use");
        if (b->budget && b->used + bytes > b->budget)
            return fail(BMFR_E_BUDGET, "stream needs " + std::to_string(bytes) + " bytes, " +
                                           std::to_string(b->budget - b->used) + " left in the budget");
        b->slots[k].used = true;   // reserved; steps cannot name it until ready
        b->slots[k].bytes = bytes;
        b->used += bytes;
    }
    // The allocation may have to grow the pool, which can take a while:
    // steps of the other streams go on meanwhile.
    void* base = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&base, bytes, b->pool, b->mem_stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(base, 0, bytes, b->mem_stream);
    if (e == cudaSuccess) e = cudaEventRecord(b->mem_ready, b->mem_stream);
    std::lock_guard<std::mutex> lk(b->mu);
    StreamSlot& s = b->slots[k];
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (base) cudaFreeAsync(base, b->mem_stream);
        b->used -= bytes;
        s = StreamSlot();
        return fail(BMFR_E_NOMEM, "device allocation for the stream failed: " + std::string(cudaGetErrorString(e)));
    }
    s.width = width;
    s.height = height;
    s.g = g;
    s.frame = 0;
    s.own_inputs = own_inputs != 0;
    s.base = base;
    carve(s, b->p, width, height, s.own_inputs, static_cast<char*>(base));
    s.ready = true;
    *slot = k;
    return BMFR_OK;
}

int bmfr_batch_remove_stream(bmfr_batch* b, int slot) {
    if (int st = check_batch(b)) return st;
    std::lock_guard<std::mutex> lk(b->mu);
    if (int st = check_slot(b, slot)) return st;
    free_slot(b, b->slots[slot]);   // in stream order after the steps that use it
    return BMFR_OK;
}

int bmfr_batch_reset_stream(bmfr_batch* b, int slot) {
    if (!b) return fail(BMFR_E_INVALID, "batch is NULL");
    std::lock_guard<std::mutex> lk(b->mu);
    if (int st = check_slot(b, slot)) return st;
    b->slots[slot].frame = 0;
    return BMFR_OK;
}

int bmfr_batch_stream_frame(const bmfr_batch* b, int slot) {
    if (!b) return fail(BMFR_E_INVALID, "batch is NULL");
    std::lock_guard<std::mutex> lk(b->mu);
    if (int st = check_slot(b, slot)) return st;
    return b->slots[slot].frame;
}

int bmfr_batch_reserve(bmfr_batch* b, size_t bytes) {
    if (int st = check_batch(b)) return st;
    if (bytes == 0) return BMFR_OK;
    void* p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, b->pool, b->mem_stream);
    if (e == cudaSuccess) e = cudaFreeAsync(p, b->mem_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->mem_stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(BMFR_E_NOMEM, "reserving stream memory failed: " + std::string(cudaGetErrorString(e)));
    }
    return BMFR_OK;
}

size_t bmfr_batch_bytes_in_use(const bmfr_batch* b) {
    if (!b) return 0;
    std::lock_guard<std::mutex> lk(b->mu);
    return b->used;
}

int bmfr_batch_stream_inputs(bmfr_batch* b, int slot, bmfr_frame_inputs* in) {
    if (!b || !in) return fail(BMFR_E_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(b->mu);
    if (int st = check_slot(b, slot)) return st;
    StreamSlot& s = b->slots[slot];
    if (!s.own_inputs) return fail(BMFR_E_STATE, "stream was added without input slots");
    // The caller writes these on its own streams: the allocation must exist.
    if (cudaError_t e = cudaEventSynchronize(b->mem_ready); e != cudaSuccess) return cuda_fail(e, "stream memory");
    const int cur = s.frame & 1;
    in->albedo = s.albedo;
    in->normals = s.normals[cur];
    in->positions = s.positions[cur];
    in->noisy = s.noisy;
    return BMFR_OK;
}

int bmfr_batch_step(bmfr_batch* b, int n, const int* slots, const bmfr_frame_io* io, const float* matrices,
                    const float* offsets, void* stream) {
    if (int st = check_batch(b)) return st;
    if (n <= 0 || n > BMFR_BATCH_MAX_STREAMS || !slots || !matrices || !offsets)
        return fail(BMFR_E_INVALID, "step: bad stream list");
    const bool staged = b->p.pipeline == BMFR_PIPELINE_STAGED;
    if (!staged && !b->graphs_valid)
        if (int st = build_graphs(b)) return st;
    const int k = b->next;
    cudaError_t e = cudaEventSynchronize(b->done[k]);   // description buffer k is free again
    if (e != cudaSuccess) return cuda_fail(e, "step: waiting for an earlier step");
    std::lock_guard<std::mutex> lk(b->mu);
    for (int i = 0; i < n; ++i) {
        if (int st = check_slot(b, slots[i])) return st;
        for (int j = 0; j < i; ++j)
            if (slots[j] == slots[i]) return fail(BMFR_E_INVALID, "step: a stream is listed twice");
    }
    if (int st = fill_desc(b, b->h_desc[k], n, slots, io, matrices, offsets)) return st;
    cudaStream_t s = (cudaStream_t)stream;
    if (b->last >= 0) {
        e = cudaStreamWaitEvent(s, b->done[b->last], 0);
        if (e != cudaSuccess) return cuda_fail(e, "step: ordering after the previous step");
    }
    e = cudaStreamWaitEvent(s, b->mem_ready, 0);   // streams added since are allocated and zeroed
    if (e != cudaSuccess) return cuda_fail(e, "step: ordering after stream allocation");
    e = staged ? launch_staged_step(b, *b->h_desc[k], s) : cudaGraphLaunch(b->graph[k], s);
    if (e == cudaSuccess) e = cudaEventRecord(b->done[k], s);
    if (e != cudaSuccess) return cuda_fail(e, staged ? "step: launches" : "step: graph launch");
    b->last = k;
    b->next = k ^ 1;
    for (int i = 0; i < n; ++i) b->slots[slots[i]].frame += 1;
    return BMFR_OK;
}

}  // extern "C"

namespace {

// Layout of a stream snapshot: this header, then the histories the next
// frame reads (those written by the stream's last frame): accumulated noisy
// colour, accumulated filtered colour, TAA result, spp, and with own input
// slots the previous normals and positions.
struct SnapshotHeader {
    char magic[8];   // "BMFRSNP1"
    int32_t width, height, frame, own_inputs;
    int32_t half_history, use_half, pipeline, fp32_qr;
    uint64_t payload_bytes;
};

struct HistoryPart {
    void* ptr;
    size_t bytes;
};

// The slot's history buffers that frame `frame` reads, in snapshot order.
std::vector<HistoryPart> history_parts(const bmfr_batch* b, const StreamSlot& s, int frame) {
    const size_t px = (size_t)s.width * s.height;
    const size_t hist = px * 3 * (b->p.half_history ? 2 : 4);
    const int prv = (frame & 1) ^ 1;
    std::vector<HistoryPart> parts = {{s.noisy_acc[prv], hist}, {s.acc_filt[prv], hist}, {s.result[prv], hist},
                                      {s.spp[prv], px}};
    if (s.own_inputs) {
        parts.push_back({s.normals[prv], px * 12});
        parts.push_back({s.positions[prv], px * 12});
    }
    return parts;
}

size_t payload_bytes(const std::vector<HistoryPart>& parts) {
    size_t n = 0;
    for (const HistoryPart& h : parts) n += h.bytes;
    return n;
}

}  // namespace

extern "C" {

int bmfr_batch_snapshot_bytes(const bmfr_batch* b, int slot, size_t* bytes) {
    if (!b || !bytes) return fail(BMFR_E_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(b->mu);
    if (int st = check_slot(b, slot)) return st;
    const StreamSlot& s = b->slots[slot];
    *bytes = sizeof(SnapshotHeader) + payload_bytes(history_parts(b, s, s.frame));
    return BMFR_OK;
}

int bmfr_batch_snapshot(bmfr_batch* b, int slot, void* dst, void* stream) {
    if (int st = check_batch(b)) return st;
    if (!dst) return fail(BMFR_E_INVALID, "snapshot: NULL destination");
    cudaStream_t cs = (cudaStream_t)stream;
    std::lock_guard<std::mutex> lk(b->mu);
    if (int st = check_slot(b, slot)) return st;
    const StreamSlot& s = b->slots[slot];
    const std::vector<HistoryPart> parts = history_parts(b, s, s.frame);
    SnapshotHeader h{};
    std::memcpy(h.magic, "BMFRSNP1", 8);
    h.width = s.width;
    h.height = s.height;
    h.frame = s.frame;
    h.own_inputs = s.own_inputs ? 1 : 0;
    h.half_history = b->p.half_history ? 1 : 0;
    h.use_half = b->p.use_half_precision_in_tmp_data ? 1 : 0;
    h.pipeline = b->p.pipeline;
    h.fp32_qr = b->p.fp32_qr;
    h.payload_bytes = payload_bytes(parts);
    cudaError_t e = cudaSuccess;
    if (b->last >= 0) e = cudaStreamWaitEvent(cs, b->done[b->last], 0);   // after the stream's last step
    if (e == cudaSuccess) e = cudaMemcpyAsync(dst, &h, sizeof h, cudaMemcpyDefault, cs);
    char* out = static_cast<char*>(dst) + sizeof h;
    for (const HistoryPart& part : parts) {
        if (e != cudaSuccess) break;
        e = cudaMemcpyAsync(out, part.ptr, part.bytes, cudaMemcpyDefault, cs);
        out += part.bytes;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
    return e == cudaSuccess ? BMFR_OK : cuda_fail(e, "snapshot copies");
}

int bmfr_batch_restore(bmfr_batch* b, const void* src, void* stream, int* slot) {
    if (int st = check_batch(b)) return st;
    if (!src || !slot) return fail(BMFR_E_INVALID, "restore: NULL argument");
    cudaStream_t cs = (cudaStream_t)stream;
    SnapshotHeader h{};
    cudaError_t e = cudaMemcpy(&h, src, sizeof h, cudaMemcpyDefault);
    if (e != cudaSuccess) return cuda_fail(e, "restore: reading the header");
    if (std::memcmp(h.magic, "BMFRSNP1", 8) != 0) return fail(BMFR_E_INVALID, "restore: not a stream snapshot");
    if (h.half_history != (b->p.half_history ? 1 : 0) || h.use_half != (b->p.use_half_precision_in_tmp_data ? 1 : 0))
        return fail(BMFR_E_INVALID, "restore: the snapshot's history format differs from the batch's");
    if (h.frame < 0) return fail(BMFR_E_INVALID, "restore: bad frame counter");
    int k = -1;
    if (int st = bmfr_batch_add_stream(b, h.width, h.height, h.own_inputs, &k)) return st;
    std::vector<HistoryPart> parts;
    {
        std::lock_guard<std::mutex> lk(b->mu);
        StreamSlot& s = b->slots[k];
        parts = history_parts(b, s, h.frame);
        if (payload_bytes(parts) != h.payload_bytes) {
            free_slot(b, s);
            return fail(BMFR_E_INVALID, "restore: snapshot size does not match the stream");
        }
        s.frame = h.frame;
    }
    e = cudaStreamWaitEvent(cs, b->mem_ready, 0);   // the slot's memory is allocated and zeroed
    const char* in = static_cast<const char*>(src) + sizeof h;
    for (const HistoryPart& part : parts) {
        if (e != cudaSuccess) break;
        e = cudaMemcpyAsync(part.ptr, in, part.bytes, cudaMemcpyDefault, cs);
        in += part.bytes;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
    if (e != cudaSuccess) {
        bmfr_batch_remove_stream(b, k);
        return cuda_fail(e, "restore copies");
    }
    *slot = k;
    return BMFR_OK;
}

int bmfr_batch_stream_result(const bmfr_batch* b, int slot, const float** result) {
    if (!b || !result) return fail(BMFR_E_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(b->mu);
    if (int st = check_slot(b, slot)) return st;
    *result = b->slots[slot].result_f32;
    return BMFR_OK;
}

int bmfr_batch_get_tuning(const bmfr_batch* b, bmfr_batch_tuning* t) {
    if (!b || !t) return fail(BMFR_E_INVALID, "NULL argument");
    t->block_ctas_per_sm = b->tuning.block_ctas_per_sm;
    t->taa_tile_w = b->tuning.tile_w;
    t->taa_tile_h = b->tuning.tile_h;
    t->staging_depth = b->tuning.staging_depth;
    t->pixel_pass = b->tuning.pixel_pass;
    return BMFR_OK;
}

int bmfr_batch_set_tuning(bmfr_batch* b, const bmfr_batch_tuning* t) {
    if (int st = check_batch(b)) return st;
    if (!t) return fail(BMFR_E_INVALID, "tuning is NULL");
    const bool shape_ok = t->taa_tile_w == 30 && (t->taa_tile_h == 8 || t->taa_tile_h == 16 || t->taa_tile_h == 32 ||
                                                  t->taa_tile_h == 64);
    if (!shape_ok) return fail(BMFR_E_INVALID, "TAA tile shape must be 30x8, 30x16, 30x32 or 30x64");
    if (t->block_ctas_per_sm < 0 || t->staging_depth < 0 || t->staging_depth > 4)
        return fail(BMFR_E_INVALID, "bad block CTAs per SM or staging depth");
    if (t->pixel_pass != 0 && t->pixel_pass != 1) return fail(BMFR_E_INVALID, "pixel_pass must be 0 or 1");
    b->tuning.block_ctas_per_sm = t->block_ctas_per_sm;
    b->tuning.tile_w = t->taa_tile_w;
    b->tuning.tile_h = t->taa_tile_h;
    b->tuning.staging_depth = t->staging_depth;
    b->tuning.pixel_pass = t->pixel_pass;
    return b->p.pipeline == BMFR_PIPELINE_STAGED ? BMFR_OK : build_graphs(b);   // the staged step has no graph
}

int bmfr_batch_autotune(bmfr_batch* b, int n, const int* slots, const bmfr_frame_io* io, const float* matrices,
                        const float* offsets, int steps, void* stream, bmfr_batch_tuning* chosen, float* best_ms) {
    if (int st = check_batch(b)) return st;
    if (steps < 1) return fail(BMFR_E_INVALID, "autotune needs at least one step");
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    auto time_tuning = [&](const bmfr_batch_tuning& t, float* ms) -> int {
        if (int st = bmfr_batch_set_tuning(b, &t)) return st;
        if (int st = bmfr_batch_step(b, n, slots, io, matrices, offsets, stream)) return st;   // warm-up
        cudaEventRecord(t0, s);
        for (int i = 0; i < steps; ++i)
            if (int st = bmfr_batch_step(b, n, slots, io, matrices, offsets, stream)) return st;
        cudaEventRecord(t1, s);
        cudaError_t e = cudaEventSynchronize(t1);
        if (e != cudaSuccess) return cuda_fail(e, "autotune timing");
        cudaEventElapsedTime(ms, t0, t1);
        *ms /= steps;
        return BMFR_OK;
    };
    bmfr_batch_tuning best{0, 30, 32, 0, 0};
    float best_t = 1e30f;
    int status = BMFR_OK;
    if (b->p.pipeline == BMFR_PIPELINE_STAGED) {
        // The staged step launches the plan's kernels, whose shapes are
        // fixed: only its time is reported.
        status = time_tuning(best, &best_t);
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        if (status != BMFR_OK) return status;
        if (chosen) *chosen = best;
        if (best_ms) *best_ms = best_t;
        return BMFR_OK;
    }
    // Blocks per SM and staging depth together, then the TAA CTA shape.
    for (int ctas = 1; ctas <= b->block_occupancy && status == BMFR_OK; ++ctas) {
        const int max_depth = b->p.pipeline == BMFR_PIPELINE_STAGED ? 0 : 2;   // staging: fused step only
        for (int depth = 0; depth <= max_depth && status == BMFR_OK; ++depth) {
            bmfr_batch_tuning t{ctas, 30, 32, depth, 0};
            float ms = 0.f;
            status = time_tuning(t, &ms);
            if (status == BMFR_OK && ms < best_t) {
                best_t = ms;
                best = t;
            }
        }
    }
    const int shapes[3][2] = {{30, 8}, {30, 16}, {30, 64}};
    for (int i = 0; i < 3 && status == BMFR_OK; ++i) {
        bmfr_batch_tuning t = best;
        t.taa_tile_w = shapes[i][0];
        t.taa_tile_h = shapes[i][1];
        float ms = 0.f;
        status = time_tuning(t, &ms);
        if (status == BMFR_OK && ms < best_t) {
            best_t = ms;
            best = t;
        }
    }
    // Then the per-pixel stages as their own pass over image tiles.
    if (status == BMFR_OK) {
        bmfr_batch_tuning t = best;
        t.pixel_pass = 1;
        float ms = 0.f;
        status = time_tuning(t, &ms);
        if (status == BMFR_OK && ms < best_t) {
            best_t = ms;
            best = t;
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (status != BMFR_OK) return status;
    if (int st = bmfr_batch_set_tuning(b, &best)) return st;
    if (chosen) *chosen = best;
    if (best_ms) *best_ms = best_t;
    return BMFR_OK;
}

}  // extern "C"
