// server.cu — continuous batching of frame requests over the many-stream
// engine (include/bmfr_batch.h): per-stream request queues, a scheduling
// thread that turns whatever is ready into the next step while earlier steps
// run on the GPU, a completion thread that stamps each request's latency, and
// admission of streams against the memory budget.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "bmfr_batch.h"
#include "status.h"

using bmfr::cuda_fail;
using bmfr::fail;

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id;
    int stream;
    bmfr_frame_io io;
    bool has_io;
    float matrix[16];
    float offset[2];
    Clock::time_point arrival;
};

struct StepRecord {
    cudaEvent_t done = nullptr;   // null if the step's event could not be made
    bool last = false;            // the scheduler's final record: the completion thread ends
    std::vector<uint64_t> requests;
    std::vector<int> streams;
    std::vector<Clock::time_point> arrivals;
    Clock::time_point launched;
};

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

struct bmfr_server {
    bmfr_params params{};
    bmfr_server_config cfg{};
    int device = 0;
    bmfr_batch* batch = nullptr;
    cudaStream_t stream = nullptr;

    std::mutex mu;                       // queues, request states, statistics
    std::mutex batch_mu;                 // steps and tuning of the batch (its slot table has its own lock)
    std::condition_variable cv_sched;    // work for the scheduler
    std::condition_variable cv_done;     // a request completed
    std::unordered_map<int, std::deque<Request>> pending;   // per open stream
    std::map<int, int> open;             // stream id -> frames submitted and not completed
    uint64_t next_id = 1;
    std::unordered_map<uint64_t, double> finished;   // request id -> latency ms
    std::unordered_map<uint64_t, bool> in_flight;
    bool stop = false;

    std::mutex step_mu;
    std::condition_variable cv_steps;
    std::deque<StepRecord> steps_in_flight;

    // statistics
    std::vector<double> latencies;
    uint64_t submitted = 0, completed = 0, n_steps = 0, n_frames = 0, admitted = 0, rejected = 0;
    double busy = 0.0;
    Clock::time_point stats_start = Clock::now();
    Clock::time_point busy_since{};
    int steps_outstanding = 0;
    std::string thread_error;

    std::thread scheduler, completer;
};

namespace {

// Scheduling thread: one step per round with the oldest pending frame of
// every stream that has one.  Steps run in launch order on the GPU, so a
// stream's frames stay sequential across steps.
void schedule_loop(bmfr_server* s) {
    cudaSetDevice(s->device);
    for (;;) {
        std::vector<Request> take;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            const int max_in_flight = s->cfg.max_steps_in_flight > 0 ? s->cfg.max_steps_in_flight : 2;
            s->cv_sched.wait(lk, [&] {
                if (s->steps_outstanding >= max_in_flight) return false;   // requests gather meanwhile
                if (s->stop) return true;
                for (auto& kv : s->pending)
                    if (!kv.second.empty()) return true;
                return false;
            });
            bool any = false;
            for (auto& kv : s->pending) any = any || !kv.second.empty();
            if (s->stop && !any) break;
            std::vector<std::pair<Clock::time_point, int>> ready;
            for (auto& kv : s->pending)
                if (!kv.second.empty()) ready.push_back({kv.second.front().arrival, kv.first});
            std::sort(ready.begin(), ready.end());
            const int cap = s->cfg.max_streams_per_step > 0 ? s->cfg.max_streams_per_step : BMFR_BATCH_MAX_STREAMS;
            for (auto& r : ready) {
                if ((int)take.size() >= cap) break;
                take.push_back(s->pending[r.second].front());
                s->pending[r.second].pop_front();
            }
        }
        const int n = (int)take.size();
        std::vector<int> slots(n);
        std::vector<bmfr_frame_io> io(n);
        std::vector<float> mats(16 * n), offs(2 * n);
        for (int i = 0; i < n; ++i) {
            slots[i] = take[i].stream;
            if (take[i].has_io) io[i] = take[i].io;
            else std::memset(&io[i], 0, sizeof(bmfr_frame_io));
            std::memcpy(&mats[16 * i], take[i].matrix, sizeof take[i].matrix);
            std::memcpy(&offs[2 * i], take[i].offset, sizeof take[i].offset);
        }
        StepRecord rec;
        int st = BMFR_OK;
        if (cudaEventCreateWithFlags(&rec.done, cudaEventDisableTiming) != cudaSuccess) {
            rec.done = nullptr;
            st = fail(BMFR_E_CUDA, "server: creating a step's event failed");
        }
        if (st == BMFR_OK) {
            std::lock_guard<std::mutex> blk(s->batch_mu);
            st = bmfr_batch_step(s->batch, n, slots.data(), io.data(), mats.data(), offs.data(), s->stream);
        }
        if (st == BMFR_OK) st = cudaEventRecord(rec.done, s->stream) == cudaSuccess ? BMFR_OK : BMFR_E_CUDA;
        if (st != BMFR_OK) {
            std::lock_guard<std::mutex> lk(s->mu);
            s->thread_error = bmfr_last_error();
        }
        rec.launched = Clock::now();
        for (auto& r : take) {
            rec.requests.push_back(r.id);
            rec.streams.push_back(r.stream);
            rec.arrivals.push_back(r.arrival);
        }
        {
            std::lock_guard<std::mutex> lk(s->step_mu);
            s->steps_in_flight.push_back(std::move(rec));
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->steps_outstanding++ == 0) s->busy_since = Clock::now();
            s->n_steps += 1;
            s->n_frames += n;
        }
        s->cv_steps.notify_one();
    }
    {
        std::lock_guard<std::mutex> lk(s->step_mu);
        StepRecord sentinel;
        sentinel.last = true;
        s->steps_in_flight.push_back(std::move(sentinel));
    }
    s->cv_steps.notify_one();
}

// Completion thread: waits for each step in launch order and stamps its
// requests.
void complete_loop(bmfr_server* s) {
    cudaSetDevice(s->device);
    for (;;) {
        StepRecord rec;
        {
            std::unique_lock<std::mutex> lk(s->step_mu);
            s->cv_steps.wait(lk, [&] { return !s->steps_in_flight.empty(); });
            rec = std::move(s->steps_in_flight.front());
            s->steps_in_flight.pop_front();
        }
        if (rec.last) break;
        if (rec.done) {
            cudaEventSynchronize(rec.done);
        } else {
            cudaStreamSynchronize(s->stream);   // no event: wait for everything queued so far
        }
        const Clock::time_point t = Clock::now();
        if (rec.done) cudaEventDestroy(rec.done);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            for (size_t i = 0; i < rec.requests.size(); ++i) {
                const double ms = ms_between(rec.arrivals[i], t);
                s->finished[rec.requests[i]] = ms;
                s->in_flight.erase(rec.requests[i]);
                s->latencies.push_back(ms);
                s->completed += 1;
                auto it = s->open.find(rec.streams[i]);
                if (it != s->open.end()) it->second -= 1;
            }
            if (--s->steps_outstanding == 0) s->busy += ms_between(s->busy_since, t);
        }
        s->cv_done.notify_all();
        s->cv_sched.notify_one();   // room for the next step
    }
}

double percentile(std::vector<double> v, double p) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = p * (double)(v.size() - 1);
    const size_t i = (size_t)pos;
    const double f = pos - (double)i;
    return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

}  // namespace

extern "C" {

int bmfr_server_create(const bmfr_params* params, const bmfr_server_config* config, bmfr_server** out) {
    if (!params || !config || !out) return fail(BMFR_E_INVALID, "NULL argument");
    *out = nullptr;
    bmfr_server* s = new bmfr_server;
    s->params = *params;
    s->cfg = *config;
    cudaGetDevice(&s->device);
    if (int st = bmfr_batch_create(params, config->memory_budget_bytes, &s->batch)) {
        delete s;
        return st;
    }
    if (int st = bmfr_batch_reserve(s->batch, config->reserve_bytes)) {
        bmfr_batch_destroy(s->batch);
        delete s;
        return st;
    }
    if (cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking); e != cudaSuccess) {
        bmfr_batch_destroy(s->batch);
        delete s;
        return cuda_fail(e, "server stream");
    }
    s->scheduler = std::thread(schedule_loop, s);
    s->completer = std::thread(complete_loop, s);
    *out = s;
    return BMFR_OK;
}

int bmfr_server_destroy(bmfr_server* s) {
    if (!s) return BMFR_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_sched.notify_all();
    if (s->scheduler.joinable()) s->scheduler.join();
    if (s->completer.joinable()) s->completer.join();
    cudaStreamSynchronize(s->stream);
    bmfr_batch_destroy(s->batch);
    cudaStreamDestroy(s->stream);
    delete s;
    return BMFR_OK;
}

int bmfr_server_open_stream(bmfr_server* s, int width, int height, int* id) {
    if (!s || !id) return fail(BMFR_E_INVALID, "NULL argument");
    // Not under batch_mu: the batch guards its slot table itself, and an
    // allocation that grows the memory pool must not hold up the steps.
    const int st = bmfr_batch_add_stream(s->batch, width, height, s->cfg.own_inputs, id);
    std::lock_guard<std::mutex> lk(s->mu);
    if (st == BMFR_E_BUDGET) s->rejected += 1;
    if (st != BMFR_OK) return st;
    s->admitted += 1;
    s->pending[*id];
    s->open[*id] = 0;
    return BMFR_OK;
}

int bmfr_server_close_stream(bmfr_server* s, int id) {
    if (!s) return fail(BMFR_E_INVALID, "server is NULL");
    {
        std::unique_lock<std::mutex> lk(s->mu);
        if (!s->open.count(id)) return fail(BMFR_E_NOT_FOUND, "no open stream " + std::to_string(id));
        // Its submitted frames finish first.
        s->cv_done.wait(lk, [&] { return s->open[id] == 0 || !s->thread_error.empty(); });
        s->open.erase(id);
        s->pending.erase(id);
    }
    return bmfr_batch_remove_stream(s->batch, id);
}

int bmfr_server_snapshot_stream(bmfr_server* s, int id, void* dst, void* stream) {
    if (!s) return fail(BMFR_E_INVALID, "server is NULL");
    {
        std::unique_lock<std::mutex> lk(s->mu);
        if (!s->open.count(id)) return fail(BMFR_E_NOT_FOUND, "no open stream " + std::to_string(id));
        // Its submitted frames finish first.
        s->cv_done.wait(lk, [&] { return s->open[id] == 0 || !s->thread_error.empty(); });
        if (!s->thread_error.empty()) return fail(BMFR_E_STATE, "server step failed: " + s->thread_error);
    }
    return bmfr_batch_snapshot(s->batch, id, dst, stream);
}

int bmfr_server_restore_stream(bmfr_server* s, const void* src, void* stream, int* id) {
    if (!s || !id) return fail(BMFR_E_INVALID, "NULL argument");
    const int st = bmfr_batch_restore(s->batch, src, stream, id);
    std::lock_guard<std::mutex> lk(s->mu);
    if (st == BMFR_E_BUDGET) s->rejected += 1;
    if (st != BMFR_OK) return st;
    s->admitted += 1;
    s->pending[*id];
    s->open[*id] = 0;
    return BMFR_OK;
}

int bmfr_server_stream_inputs(bmfr_server* s, int id, bmfr_frame_inputs* in) {
    if (!s) return fail(BMFR_E_INVALID, "server is NULL");
    return bmfr_batch_stream_inputs(s->batch, id, in);
}

int bmfr_server_submit(bmfr_server* s, int id, const bmfr_frame_io* io, const float* matrix, const float* offset,
                       uint64_t* request_id) {
    if (!s || !matrix || !offset) return fail(BMFR_E_INVALID, "NULL argument");
    Request r;
    r.stream = id;
    r.has_io = io != nullptr;
    if (io) r.io = *io;
    std::memcpy(r.matrix, matrix, sizeof r.matrix);
    std::memcpy(r.offset, offset, sizeof r.offset);
    r.arrival = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (!s->open.count(id)) return fail(BMFR_E_NOT_FOUND, "no open stream " + std::to_string(id));
        if (!s->thread_error.empty()) return fail(BMFR_E_STATE, "server step failed: " + s->thread_error);
        r.id = s->next_id++;
        s->pending[id].push_back(r);
        s->in_flight[r.id] = true;
        s->open[id] += 1;
        s->submitted += 1;
    }
    s->cv_sched.notify_one();
    if (request_id) *request_id = r.id;
    return BMFR_OK;
}

int bmfr_server_poll(bmfr_server* s, uint64_t rid, int* done, double* latency_ms) {
    if (!s || !done) return fail(BMFR_E_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->finished.find(rid);
    if (it != s->finished.end()) {
        *done = 1;
        if (latency_ms) *latency_ms = it->second;
        return BMFR_OK;
    }
    if (!s->in_flight.count(rid)) return fail(BMFR_E_NOT_FOUND, "unknown request");
    *done = 0;
    return BMFR_OK;
}

int bmfr_server_drain(bmfr_server* s, double timeout_ms) {
    if (!s) return fail(BMFR_E_INVALID, "server is NULL");
    std::unique_lock<std::mutex> lk(s->mu);
    const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms),
                                        [&] { return s->in_flight.empty(); });
    if (!s->thread_error.empty()) return fail(BMFR_E_STATE, "server step failed: " + s->thread_error);
    return ok ? BMFR_OK : fail(BMFR_E_TIMEOUT, "requests still pending after the timeout");
}

int bmfr_server_stats_get(bmfr_server* s, bmfr_server_stats* o) {
    if (!s || !o) return fail(BMFR_E_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(o, 0, sizeof *o);
    o->requests_submitted = s->submitted;
    o->requests_completed = s->completed;
    o->steps = s->n_steps;
    o->frames = s->n_frames;
    o->streams_admitted = s->admitted;
    o->streams_rejected = s->rejected;
    o->p50_latency_ms = percentile(s->latencies, 0.50);
    o->p99_latency_ms = percentile(s->latencies, 0.99);
    double mx = 0.0, sum = 0.0;
    for (double v : s->latencies) {
        mx = std::max(mx, v);
        sum += v;
    }
    o->max_latency_ms = mx;
    o->mean_latency_ms = s->latencies.empty() ? 0.0 : sum / (double)s->latencies.size();
    o->mean_frames_per_step = s->n_steps ? (double)s->n_frames / (double)s->n_steps : 0.0;
    o->busy_seconds = s->busy / 1e3 + (s->steps_outstanding ? ms_between(s->busy_since, Clock::now()) / 1e3 : 0.0);
    o->elapsed_seconds = ms_between(s->stats_start, Clock::now()) / 1e3;
    return BMFR_OK;
}

int bmfr_server_stats_reset(bmfr_server* s) {
    if (!s) return fail(BMFR_E_INVALID, "server is NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    s->latencies.clear();
    s->submitted = s->completed = s->n_steps = s->n_frames = 0;
    s->busy = 0.0;
    s->stats_start = Clock::now();
    if (s->steps_outstanding) s->busy_since = s->stats_start;
    s->finished.clear();
    return BMFR_OK;
}

bmfr_batch* bmfr_server_batch(bmfr_server* s) { return s ? s->batch : nullptr; }

int bmfr_server_set_tuning(bmfr_server* s, const bmfr_batch_tuning* t) {
    if (!s) return fail(BMFR_E_INVALID, "server is NULL");
    std::lock_guard<std::mutex> blk(s->batch_mu);
    return bmfr_batch_set_tuning(s->batch, t);
}

}  // extern "C"
