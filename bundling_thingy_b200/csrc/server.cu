// server.cu — continuous batching of arriving bundling requests (bt_server_*).
//
// One worker thread owns one bt_batch and every device context, and never
// blocks on the device while there is work to move: it polls events.
//   - Requests whose arrival time has passed join the ready queue (arrival
//     order).
//   - A batch step starts as soon as the previous one has finished: every
//     running graph advances by `step` iterations (one CUDA graph launch per
//     iteration on the batch's stream), step = the smallest remaining
//     iteration count, at most `max_step` while other requests wait to join.
//   - Admission: while `max_active` and the device-memory budget allow, the
//     head of the queue takes an idle context of the same options (or a new
//     one) and starts its upload on the context's own stream. Each upload
//     phase (count; emit, density pass 0 and first binning; check and
//     search-cell shape) starts when the previous one is done, beside the
//     running step; a loaded graph joins the batch for the next step.
//   - After a step, every graph that reached its iteration count leaves the
//     batch and its positions are unsorted into records on its own stream;
//     the request is finished when they are ready. Its memory stays charged
//     until the client releases it; released contexts are kept idle for reuse
//     by the next request with the same options (and freed when memory is
//     short).
//
// Admission generalises Allocation::new (src/resampling.rs:321-397) from one
// graph to all resident graphs: each context charges its device allocations
// to one shared account before making them (bt::MemAccount). A phase refused
// by the account launches nothing, so the request goes back to the queue
// (idle contexts are freed first) and is retried when memory is released; it
// fails with BT_ERR_BUDGET only when nothing else holds memory.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "bt.h"
#include "context.h"

namespace {

enum class State { Pending, Counting, Loading, Running, Done, Failed };

struct Request {
    uint64_t id = 0;
    bt_options opt{};
    std::vector<float> xy;
    std::vector<uint32_t> starts;
    uint32_t iterations = 0;
    double arrival = 0.0;
    State state = State::Pending;
    bt_ctx* ctx = nullptr;
    uint32_t slot = 0;
    bool delivered = false;
    bool cancel = false;   // bt_server_cancel asked (guarded by bt_server::mu)
    bt_request_result result{};
};

thread_local std::string g_server_error;

bt_options normalized_options(const bt_options& in, int32_t device) {
    bt_options o = in;
    o.device = device;
    o.timing = 0;
    return o;
}

bool same_options(const bt_options& a, const bt_options& b) { return std::memcmp(&a, &b, sizeof(a)) == 0; }

}  // namespace

struct bt_server {
    bt_server_options opt{};
    bt::MemAccount account;
    bt_batch* batch = nullptr;
    cudaEvent_t step_done = nullptr;   // end of the batch step in flight
    std::chrono::steady_clock::time_point t0;
    std::thread worker;

    std::mutex mu;                    // guards everything below up to the worker-only part
    std::condition_variable work_cv;  // new submissions, releases, stop
    std::condition_variable done_cv;  // finished requests
    bool stop = false;
    std::string err;
    uint64_t next_id = 1;
    std::map<uint64_t, std::unique_ptr<Request>> requests;   // submitted and not released
    std::vector<Request*> incoming;                          // not yet seen by the worker
    std::vector<bt_ctx*> released;                           // contexts handed back by clients
    std::deque<uint64_t> finished;                           // completion order, undelivered
    bt_server_stats stats{};

    // Worker-only state.
    std::vector<Request*> future;    // arrival time not reached, sorted by (arrival, id)
    std::deque<Request*> ready;      // arrived, waiting for admission, sorted by (arrival, id)
    std::vector<Request*> uploading, running;   // uploading: Counting or Loading
    std::vector<Request*> finishing;   // out of the batch, records being unsorted
    std::vector<bt_ctx*> pool;       // idle contexts

    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace {

bool by_arrival(const Request* a, const Request* b) {
    return a->arrival < b->arrival || (a->arrival == b->arrival && a->id < b->id);
}

bt_status sfail(bt_server* s, bt_status code, const std::string& msg) {
    if (s) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->err = msg;
    }
    g_server_error = msg;
    return code;
}

void set_result(Request* r, bt_status status, const std::string& msg, double t) {
    r->result.id = r->id;
    r->result.status = status;
    r->result.iterations = r->ctx ? r->ctx->iterations : 0;
    r->result.samples = r->ctx ? r->ctx->samples : 0;
    r->result.arrival_s = r->arrival;
    r->result.finished_s = t;
    r->result.device_bytes = r->ctx ? r->ctx->device_bytes : 0;
    std::snprintf(r->result.message, sizeof(r->result.message), "%s", msg.c_str());
}

// Worker: publish a finished or failed request (the lock is not held).
void publish(bt_server* s, Request* r, bt_status status, const std::string& msg) {
    std::lock_guard<std::mutex> lk(s->mu);
    set_result(r, status, msg, s->now());
    r->state = status == BT_OK ? State::Done : State::Failed;
    if (status == BT_OK) {
        ++s->stats.finished;
        ++s->stats.resident_results;
    } else {
        ++s->stats.failed;
    }
    r->xy.clear();
    r->xy.shrink_to_fit();
    r->starts.clear();
    r->starts.shrink_to_fit();
    s->finished.push_back(r->id);
    s->done_cv.notify_all();
}

void fail_request(bt_server* s, Request* r, bt_status status, const std::string& msg) {
    if (r->ctx) {
        s->pool.push_back(r->ctx);   // its memory stays reusable
        r->ctx = nullptr;
    }
    publish(s, r, status, msg);
}

bool evict_idle(bt_server* s) {
    {
        // Contexts the client released since the turn began are idle too.
        std::lock_guard<std::mutex> lk(s->mu);
        for (bt_ctx* c : s->released) s->pool.push_back(c);
        s->released.clear();
    }
    if (s->pool.empty()) return false;
    bt_destroy(s->pool.front());
    s->pool.erase(s->pool.begin());
    std::lock_guard<std::mutex> lk(s->mu);
    ++s->stats.evictions;
    return true;
}

// The largest idle context with these options (the likeliest to need no
// further allocation).
bt_ctx* take_idle(bt_server* s, const bt_options& o) {
    size_t best = s->pool.size();
    for (size_t i = 0; i < s->pool.size(); ++i)
        if (same_options(s->pool[i]->opt, o) &&
            (best == s->pool.size() || s->pool[i]->device_bytes > s->pool[best]->device_bytes))
            best = i;
    if (best == s->pool.size()) return nullptr;
    bt_ctx* c = s->pool[best];
    s->pool.erase(s->pool.begin() + static_cast<std::ptrdiff_t>(best));
    return c;
}

// Memory that will come back without this request's help: running graphs and
// results the client still holds.
bool others_hold_memory(bt_server* s, const Request* self) {
    for (const Request* r : s->running)
        if (r != self) return true;
    for (const Request* r : s->uploading)
        if (r != self) return true;
    if (!s->finishing.empty()) return true;
    std::lock_guard<std::mutex> lk(s->mu);
    return s->stats.resident_results > 0;
}

// A phase was refused by the budget: free idle contexts and retry, defer the
// request while others hold memory, fail it when it cannot fit alone.
enum class Budget { Retry, Defer, Fail };
Budget on_budget(bt_server* s, const Request* r) {
    if (evict_idle(s)) return Budget::Retry;
    if (others_hold_memory(s, r)) {
        std::lock_guard<std::mutex> lk(s->mu);
        ++s->stats.budget_waits;
        return Budget::Defer;
    }
    return Budget::Fail;
}

size_t active_count(const bt_server* s) { return s->uploading.size() + s->running.size() + s->finishing.size(); }

// Samples from which a request iterates on its own (bt_server_options::solo_samples = 0).
constexpr uint32_t kSoloSamples = 32768;

// Records the end of the work queued so far on a context's stream.
bool mark(bt_ctx* c) { return cudaEventRecord(c->done, c->stream) == cudaSuccess; }

// 1 when the marked work is done, 0 while it runs, -1 on a device error.
int marked_done(bt_ctx* c) {
    const cudaError_t e = cudaEventQuery(c->done);
    if (e == cudaSuccess) return 1;
    if (e == cudaErrorNotReady) return 0;
    return -1;
}

// Back to the ready queue in arrival order; its context stays idle and
// evictable, so a graph that fits alone always progresses.
void requeue(bt_server* s, Request* r) {
    s->pool.push_back(r->ctx);
    r->ctx = nullptr;
    r->state = State::Pending;
    s->ready.insert(std::upper_bound(s->ready.begin(), s->ready.end(), r, by_arrival), r);
    std::lock_guard<std::mutex> lk(s->mu);
    ++s->stats.budget_waits;
}

// Starts the uploads of the head of the ready queue; returns whether any
// started (or failed).
bool admit(bt_server* s) {
    bool moved = false;
    while (!s->ready.empty()) {
        if (s->opt.max_active && active_count(s) >= s->opt.max_active) return moved;
        Request* r = s->ready.front();
        bt_ctx* c = take_idle(s, r->opt);
        if (!c) {
            const double t0 = s->now();
            bt_status st = bt::create_context(&r->opt, &s->account, &c);
            {
                std::lock_guard<std::mutex> lk(s->mu);
                s->stats.create_s += s->now() - t0;
                if (st == BT_OK) ++s->stats.contexts_created;
            }
            if (st == BT_ERR_BUDGET) {
                const Budget b = on_budget(s, r);
                if (b == Budget::Retry) continue;
                if (b == Budget::Defer) return moved;
            }
            if (st != BT_OK) {
                s->ready.pop_front();
                fail_request(s, r, st, bt_last_error(nullptr));
                moved = true;
                continue;
            }
        }
        r->ctx = c;
        bt_status st = bt::upload_begin(c, r->xy.data(), static_cast<uint32_t>(r->xy.size() / 2), r->starts.data(),
                                        static_cast<uint32_t>(r->starts.size()));
        if (st == BT_ERR_BUDGET) {
            s->pool.push_back(c);
            r->ctx = nullptr;
            const Budget b = on_budget(s, r);
            if (b == Budget::Retry) continue;
            if (b == Budget::Defer) return moved;
        }
        s->ready.pop_front();
        moved = true;
        if (st != BT_OK || !mark(c)) {
            const std::string msg = c->err;
            fail_request(s, r, st ? st : BT_ERR_CUDA, msg);
            continue;
        }
        r->state = State::Counting;
        r->result.admitted_s = s->now();
        s->uploading.push_back(r);
    }
    return moved;
}

// Uploads move on without blocking: each phase is launched when the previous
// one's work is done on the request's stream. Requests refused by the budget
// go back to the ready queue. Returns whether anything moved.
bool advance_uploads(bt_server* s) {
    bool moved = false;
    std::vector<Request*> still;
    for (size_t k = 0; k < s->uploading.size(); ++k) {
        Request* r = s->uploading[k];
        const int done = marked_done(r->ctx);
        if (done == 0) {
            still.push_back(r);
            continue;
        }
        moved = true;
        if (done < 0) {
            fail_request(s, r, BT_ERR_CUDA, std::string("device execution: ") + cudaGetErrorString(cudaGetLastError()));
            continue;
        }
        auto others = [&] {
            for (size_t q = k + 1; q < s->uploading.size(); ++q)
                if (s->uploading[q]->ctx) return true;
            return !still.empty() || others_hold_memory(s, r);
        };
        if (r->state == State::Counting) {
            bt_status st = bt::upload_finish(r->ctx);
            while (st == BT_ERR_BUDGET && evict_idle(s)) st = bt::upload_finish(r->ctx);
            if (st == BT_ERR_BUDGET && others()) {
                requeue(s, r);
                continue;
            }
            if (st != BT_OK || !mark(r->ctx)) {
                const std::string msg = r->ctx->err;
                fail_request(s, r, st ? st : BT_ERR_CUDA, msg);
                continue;
            }
            r->state = State::Loading;
            still.push_back(r);
            continue;
        }
        // Loaded: check, pick the search-cell shape, keep room for the records.
        uint32_t samples = 0;
        bt_status st = bt::upload_check(r->ctx, &samples);
        if (st == BT_OK) st = bt::upload_adapt(r->ctx);
        if (st == BT_OK) {
            st = bt::reserve_records(r->ctx);
            while (st == BT_ERR_BUDGET && evict_idle(s)) st = bt::reserve_records(r->ctx);
            if (st == BT_ERR_BUDGET && others()) {
                requeue(s, r);
                continue;
            }
        }
        if (st == BT_OK && r->iterations == 0) {
            // Nothing to iterate: the upload is the result.
            st = bt::prepare_records(r->ctx);
            if (st == BT_OK && mark(r->ctx)) {
                s->finishing.push_back(r);
                continue;
            }
        }
        if (st != BT_OK) {
            const std::string msg = r->ctx->err;
            fail_request(s, r, st, msg);
            continue;
        }
        const uint32_t solo = s->opt.solo_samples ? s->opt.solo_samples : kSoloSamples;
        if (samples >= solo) {
            // Large enough to fill the device by itself (a persistent batch
            // step would only slow it down): all its iterations and the
            // records on its own stream, beside the batch.
            st = bt_iterate_async(r->ctx, r->iterations);
            if (st == BT_OK) st = bt::prepare_records(r->ctx);
            if (st == BT_OK && mark(r->ctx)) {
                r->state = State::Running;
                s->finishing.push_back(r);
                continue;
            }
            const std::string msg = r->ctx->err;
            fail_request(s, r, st ? st : BT_ERR_CUDA, msg);
            continue;
        }
        if (bt_status ast = bt::batch_attach(s->batch, r->ctx, &r->slot)) {
            fail_request(s, r, ast, bt_batch_last_error(s->batch));
            continue;
        }
        r->state = State::Running;
        s->running.push_back(r);
    }
    s->uploading.swap(still);
    return moved;
}

// Graphs that reached their iteration count leave the batch after its step;
// their records are unsorted on their own streams.
void retire(bt_server* s) {
    std::vector<Request*> still;
    for (Request* r : s->running) {
        if (r->ctx->iterations < r->iterations) {
            still.push_back(r);
            continue;
        }
        bt_ctx* c = bt::batch_detach(s->batch, r->slot);
        if (!c) {
            r->ctx = nullptr;
            publish(s, r, BT_ERR_CUDA, "batch slot lost");
            continue;
        }
        if (bt_status st = bt::prepare_records(c)) {
            const std::string msg = c->err;
            fail_request(s, r, st, msg);
            continue;
        }
        if (!mark(c)) {
            fail_request(s, r, BT_ERR_CUDA, "cudaEventRecord");
            continue;
        }
        s->finishing.push_back(r);
    }
    s->running.swap(still);
}

// Requests whose records are ready are finished. Returns whether any was.
bool publish_ready(bt_server* s) {
    bool moved = false;
    std::vector<Request*> still;
    for (Request* r : s->finishing) {
        const int done = marked_done(r->ctx);
        if (done == 0) {
            still.push_back(r);
            continue;
        }
        moved = true;
        if (done < 0) {
            fail_request(s, r, BT_ERR_CUDA, std::string("device execution: ") + cudaGetErrorString(cudaGetLastError()));
            continue;
        }
        publish(s, r, BT_OK, "");
    }
    s->finishing.swap(still);
    return moved;
}

// Queued requests that were cancelled, or that waited past the admission
// deadline, finish with an error without touching the device. Returns
// whether any did.
bool drop_queued(bt_server* s) {
    const double t = s->now();
    const double limit = s->opt.queue_timeout_ms ? s->opt.queue_timeout_ms * 1e-3 : -1.0;
    std::vector<std::pair<Request*, bt_status>> dropped;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        std::vector<Request*> waiting;   // not arrived yet: only a cancellation drops them
        for (Request* r : s->future) {
            if (r->cancel) {
                dropped.emplace_back(r, BT_ERR_CANCELLED);
            } else {
                waiting.push_back(r);
            }
        }
        s->future.swap(waiting);
        std::deque<Request*> keep;
        for (Request* r : s->ready) {
            if (r->cancel) {
                dropped.emplace_back(r, BT_ERR_CANCELLED);
            } else if (limit >= 0.0 && t - r->arrival > limit) {
                dropped.emplace_back(r, BT_ERR_TIMEOUT);
            } else {
                keep.push_back(r);
            }
        }
        s->ready.swap(keep);
    }
    for (auto& d : dropped) {
        if (d.second == BT_ERR_CANCELLED) {
            publish(s, d.first, BT_ERR_CANCELLED, "cancelled before admission");
        } else {
            char msg[96];
            std::snprintf(msg, sizeof(msg), "not admitted within %u ms of its arrival", s->opt.queue_timeout_ms);
            publish(s, d.first, BT_ERR_TIMEOUT, msg);
        }
    }
    return !dropped.empty();
}

void fail_running(bt_server* s, bt_status st, const std::string& msg) {
    for (Request* r : s->running) {
        bt_ctx* c = bt::batch_detach(s->batch, r->slot);
        if (c) bt_destroy(c);
        r->ctx = nullptr;
        publish(s, r, st, msg);
    }
    s->running.clear();
}

void worker_main(bt_server* s) {
    cudaSetDevice(s->opt.device);
    double t_launch = 0, t_upload = 0, t_wait = 0, t_retire = 0, t_idle = 0;
    bool step_busy = false;
    for (;;) {
        // Arrivals and releases.
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (s->stop) break;
            for (Request* r : s->incoming)
                s->future.insert(std::upper_bound(s->future.begin(), s->future.end(), r, by_arrival), r);
            s->incoming.clear();
            for (bt_ctx* c : s->released) s->pool.push_back(c);
            s->released.clear();
        }
        const double t = s->now();
        size_t arrived = 0;
        while (arrived < s->future.size() && s->future[arrived]->arrival <= t) ++arrived;
        for (size_t i = 0; i < arrived; ++i)
            s->ready.insert(std::upper_bound(s->ready.begin(), s->ready.end(), s->future[i], by_arrival),
                            s->future[i]);
        s->future.erase(s->future.begin(), s->future.begin() + static_cast<std::ptrdiff_t>(arrived));

        const bool dropped = drop_queued(s);
        double mark_t = s->now();
        auto lap = [&](double& acc) {
            const double now = s->now();
            acc += now - mark_t;
            mark_t = now;
        };
        bool moved = dropped;
        // The next batch step as soon as the previous one is done.
        if (!step_busy && !s->running.empty()) {
            // Nothing waiting to join: run the running graphs up to the first
            // one's end in one launch sequence (no host turn per iteration).
            const bool joining = !s->ready.empty() || !s->uploading.empty();
            uint32_t step = joining ? std::max<uint32_t>(1, s->opt.max_step) : UINT32_MAX;
            for (const Request* r : s->running) step = std::min(step, r->iterations - r->ctx->iterations);
            if (bt_status st = bt_batch_iterate_async(s->batch, step)) {
                fail_running(s, st, bt_batch_last_error(s->batch));
            } else if (cudaEventRecord(s->step_done, bt::batch_stream(s->batch)) != cudaSuccess) {
                fail_running(s, BT_ERR_CUDA, "cudaEventRecord");
            } else {
                step_busy = true;
                std::lock_guard<std::mutex> lk(s->mu);
                ++s->stats.steps;
            }
            moved = true;
            lap(t_launch);
        }
        moved |= publish_ready(s);
        lap(t_retire);
        moved |= admit(s);
        moved |= advance_uploads(s);
        lap(t_upload);
        if (step_busy && cudaEventQuery(s->step_done) != cudaErrorNotReady) {
            step_busy = false;
            moved = true;
            if (bt_status st = bt_batch_synchronize(s->batch)) {
                fail_running(s, st, bt_batch_last_error(s->batch));
            } else {
                retire(s);
            }
            lap(t_retire);
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->stats.queued = static_cast<uint32_t>(s->ready.size() + s->future.size() + s->incoming.size());
            s->stats.active = static_cast<uint32_t>(active_count(s));
            s->stats.peak_active = std::max(s->stats.peak_active, s->stats.active);
            s->stats.device_bytes = s->account.used.load();
            s->stats.peak_device_bytes = std::max(s->stats.peak_device_bytes, s->stats.device_bytes);
            s->stats.launch_s = t_launch;
            s->stats.upload_s = t_upload;
            s->stats.wait_s = t_wait;
            s->stats.retire_s = t_retire;
            s->stats.idle_s = t_idle;
        }
        if (moved) continue;
        if (step_busy || !s->uploading.empty() || !s->finishing.empty()) {
            // Device work in flight: poll again shortly.
            std::this_thread::sleep_for(std::chrono::microseconds(20));
            lap(t_wait);
            continue;
        }
        // Idle: sleep until the next arrival, a submission or a release.
        std::unique_lock<std::mutex> lk(s->mu);
        if (s->stop) break;
        if (!s->incoming.empty() || !s->released.empty()) continue;
        if (!s->ready.empty()) {
            // Waiting on the budget: a release wakes us (or the admission
            // deadline of the oldest queued request).
            double wait_s = 0.05;
            if (s->opt.queue_timeout_ms)
                wait_s = std::min(wait_s, std::max(1e-4, s->ready.front()->arrival + s->opt.queue_timeout_ms * 1e-3 -
                                                             s->now()));
            s->work_cv.wait_for(lk, std::chrono::duration<double>(wait_s));
        } else if (!s->future.empty()) {
            const double wait_s = s->future.front()->arrival - s->now();
            if (wait_s > 0) s->work_cv.wait_for(lk, std::chrono::duration<double>(std::min(wait_s, 0.05)));
        } else {
            s->work_cv.wait_for(lk, std::chrono::milliseconds(50));
        }
        lk.unlock();
        lap(t_idle);
    }
    if (step_busy) bt_batch_synchronize(s->batch);   // bounded wait
}

}  // namespace

extern "C" {

void bt_server_options_init(bt_server_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->max_active = 32;
    o->budget_bytes = 120000000000ull;
    o->max_step = 1;
}

bt_status bt_server_create(const bt_server_options* options, bt_server** out) {
    if (!options || !out) return sfail(nullptr, BT_ERR_INVALID, "null argument");
    *out = nullptr;
    if (options->budget_bytes == 0) return sfail(nullptr, BT_ERR_INVALID, "server memory budget must be nonzero");
    auto* s = new bt_server();
    s->opt = *options;
    if (s->opt.max_step == 0) s->opt.max_step = 1;
    s->account.limit = options->budget_bytes;
    s->stats = bt_server_stats{};
    if (bt_status st = bt_batch_create(options->device, &s->batch)) {
        const std::string msg = bt_last_error(nullptr);
        delete s;
        return sfail(nullptr, st, msg);
    }
    // The server picks each request's lane itself (solo_samples): whatever
    // it attaches stays in the persistent step.
    bt_batch_set_solo_samples(s->batch, UINT32_MAX);
    if (cudaEventCreateWithFlags(&s->step_done, cudaEventDisableTiming) != cudaSuccess) {
        bt_batch_destroy(s->batch);
        delete s;
        return sfail(nullptr, BT_ERR_CUDA, "cudaEventCreate");
    }
    if (options->reserve_bytes) {
        // Map the reserve into the stream-ordered pool once: an allocation
        // that grows the pool while batch steps run stalls the worker.
        const uint64_t bytes = std::min(options->reserve_bytes, options->budget_bytes);
        cudaError_t e = bt::prepare_device_memory(options->device);
        const cudaStream_t st = bt::batch_stream(s->batch);
        void* p = nullptr;
        if (e == cudaSuccess) e = cudaMallocAsync(&p, bytes, st);
        if (e == cudaSuccess) e = cudaFreeAsync(p, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            cudaGetLastError();
            cudaEventDestroy(s->step_done);
            bt_batch_destroy(s->batch);
            delete s;
            return sfail(nullptr, e == cudaErrorMemoryAllocation ? BT_ERR_BUDGET : BT_ERR_CUDA,
                         std::string("device memory reserve: ") + cudaGetErrorString(e));
        }
    }
    s->t0 = std::chrono::steady_clock::now();
    s->worker = std::thread(worker_main, s);
    *out = s;
    return BT_OK;
}

void bt_server_destroy(bt_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->work_cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->opt.device);
    for (Request* r : s->running) {
        bt_ctx* c = bt::batch_detach(s->batch, r->slot);
        if (c) bt_destroy(c);
        r->ctx = nullptr;
    }
    for (auto& kv : s->requests)
        if (kv.second->ctx) bt_destroy(kv.second->ctx);
    for (bt_ctx* c : s->pool) bt_destroy(c);
    for (bt_ctx* c : s->released) bt_destroy(c);
    bt_batch_destroy(s->batch);
    if (s->step_done) cudaEventDestroy(s->step_done);
    delete s;
}

const char* bt_server_last_error(const bt_server* s) { return s ? s->err.c_str() : g_server_error.c_str(); }

double bt_server_clock(const bt_server* s) { return s ? s->now() : 0.0; }

bt_status bt_server_submit(bt_server* s, const bt_options* options, const float* xy, uint32_t n_points,
                           const uint32_t* starts, uint32_t n_starts, uint32_t iterations, double arrival_s,
                           uint64_t* id) {
    if (!s || !options || !xy || !starts || !id) return sfail(s, BT_ERR_INVALID, "null argument");
    if (options->neighbor_radius == 0) return sfail(s, BT_ERR_NOT_CONFIGURED, "neighbor radius is not configured");
    auto r = std::make_unique<Request>();
    r->opt = normalized_options(*options, s->opt.device);
    r->xy.assign(xy, xy + 2ull * n_points);
    r->starts.assign(starts, starts + n_starts);
    r->iterations = iterations;
    r->arrival = arrival_s < 0.0 ? s->now() : arrival_s;
    std::lock_guard<std::mutex> lk(s->mu);
    r->id = s->next_id++;
    *id = r->id;
    s->incoming.push_back(r.get());
    s->requests.emplace(r->id, std::move(r));
    ++s->stats.submitted;
    s->work_cv.notify_all();
    return BT_OK;
}

bt_status bt_server_next(bt_server* s, double timeout_s, bt_request_result* result) {
    if (!s || !result) return sfail(s, BT_ERR_INVALID, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(std::max(0.0, timeout_s));
    for (;;) {
        while (!s->finished.empty()) {
            const uint64_t id = s->finished.front();
            s->finished.pop_front();
            auto it = s->requests.find(id);
            if (it == s->requests.end() || it->second->delivered) continue;
            it->second->delivered = true;
            *result = it->second->result;
            return BT_OK;
        }
        if (s->done_cv.wait_until(lk, deadline) == std::cv_status::timeout && s->finished.empty()) {
            s->err = "no request finished in time";
            g_server_error = s->err;
            return BT_ERR_TIMEOUT;
        }
    }
}

bt_ctx* bt_server_result(bt_server* s, uint64_t id) {
    if (!s) return nullptr;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->requests.find(id);
    if (it == s->requests.end() || it->second->state != State::Done) return nullptr;
    return it->second->ctx;
}

bt_status bt_server_read_points(bt_server* s, uint64_t id, void* dst, size_t bytes) {
    bt_ctx* c = bt_server_result(s, id);
    if (!c) return sfail(s, BT_ERR_INVALID, "no finished request with this id");
    if (bt_status st = bt::copy_records(c, dst, bytes)) return sfail(s, st, c->err);
    return BT_OK;
}

bt_status bt_server_release(bt_server* s, uint64_t id) {
    if (!s) return sfail(nullptr, BT_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->requests.find(id);
    if (it == s->requests.end()) {
        s->err = "no such request";
        g_server_error = s->err;
        return BT_ERR_INVALID;
    }
    Request* r = it->second.get();
    if (r->state != State::Done && r->state != State::Failed) {
        s->err = "request has not finished";
        g_server_error = s->err;
        return BT_ERR_INVALID;
    }
    if (r->state == State::Done) {
        if (r->ctx) s->released.push_back(r->ctx);
        --s->stats.resident_results;
    }
    s->requests.erase(it);
    s->work_cv.notify_all();
    return BT_OK;
}

bt_status bt_server_cancel(bt_server* s, uint64_t id) {
    if (!s) return sfail(nullptr, BT_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->requests.find(id);
    if (it == s->requests.end() || it->second->state == State::Done || it->second->state == State::Failed) {
        s->err = "no unfinished request with this id";
        g_server_error = s->err;
        return BT_ERR_INVALID;
    }
    it->second->cancel = true;
    s->work_cv.notify_all();
    return BT_OK;
}

bt_status bt_server_stats_get(bt_server* s, bt_server_stats* out) {
    if (!s || !out) return sfail(s, BT_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->stats;
    out->device_bytes = s->account.used.load();
    return BT_OK;
}

}  // extern "C"
