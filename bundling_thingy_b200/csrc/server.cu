// server.cu — continuous batching of arriving bundling requests (bt_server_*).
//
// One worker thread owns one bt_batch and every device context. Each turn of
// its loop:
//   1. requests whose arrival time has passed join the ready queue (arrival
//      order);
//   2. admission: while `max_active` and the device-memory budget allow, the
//      head of the queue takes an idle context of the same options (or a new
//      one) and starts its upload — the count phase of Gpu::upload, on the
//      context's own stream;
//   3. the batch advances every running graph by `step` iterations (one CUDA
//      graph launch per iteration on the batch's stream), step = the smallest
//      remaining iteration count, at most `max_step`;
//   4. meanwhile the admitted uploads finish (emit, density pass 0, first
//      binning), are checked and join the batch for the next turn;
//   5. after the batch's step, every graph that reached its iteration count
//      leaves the batch: its positions are unsorted into records on its own
//      stream and the request is finished. Its memory stays charged until the
//      client releases it; released contexts are kept idle for reuse by the
//      next request with the same options (and freed when memory is short).
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
    bt_request_result result{};
};

thread_local std::string g_server_error;

bt_options normalized_options(const bt_options& in, int32_t device) {
    bt_options o = in;
    o.device = device;
    o.timing = 0;
    std::memset(o.reserved, 0, sizeof(o.reserved));
    return o;
}

bool same_options(const bt_options& a, const bt_options& b) { return std::memcmp(&a, &b, sizeof(a)) == 0; }

}  // namespace

struct bt_server {
    bt_server_options opt{};
    bt::MemAccount account;
    bt_batch* batch = nullptr;
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
    std::vector<Request*> counting, running;
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
    for (const Request* r : s->counting)
        if (r != self) return true;
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

size_t active_count(const bt_server* s) { return s->counting.size() + s->running.size(); }

// Step 2: start the uploads of the head of the ready queue.
void admit(bt_server* s) {
    while (!s->ready.empty()) {
        if (s->opt.max_active && active_count(s) >= s->opt.max_active) return;
        Request* r = s->ready.front();
        bt_ctx* c = take_idle(s, r->opt);
        if (!c) {
            bt_status st = bt::create_context(&r->opt, &s->account, &c);
            if (st == BT_ERR_BUDGET) {
                const Budget b = on_budget(s, r);
                if (b == Budget::Retry) continue;
                if (b == Budget::Defer) return;
            }
            if (st != BT_OK) {
                s->ready.pop_front();
                fail_request(s, r, st, bt_last_error(nullptr));
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
            if (b == Budget::Defer) return;
        }
        s->ready.pop_front();
        if (st != BT_OK) {
            const std::string msg = c->err;
            fail_request(s, r, st, msg);
            continue;
        }
        r->state = State::Counting;
        r->result.admitted_s = s->now();
        s->counting.push_back(r);
    }
}

// Step 4: finish the admitted uploads and join them to the batch. Requests
// refused by the budget go back to the ready queue.
void finish_uploads(bt_server* s) {
    if (s->counting.empty()) return;
    std::vector<Request*> batch_of(s->counting);
    s->counting.clear();
    std::vector<Request*> loading;
    for (Request* r : batch_of) {
        if (bt_status st = bt::upload_wait(r->ctx)) {
            const std::string msg = r->ctx->err;
            fail_request(s, r, st, msg);
            continue;
        }
        loading.push_back(r);
    }
    // Another graph of this turn that is still uploading or loaded holds
    // memory it will give back when it finishes.
    auto wave_holds = [&](const Request* self) {
        for (const Request* q : batch_of)
            if (q != self && q->ctx && (q->state == State::Counting || q->state == State::Loading)) return true;
        return false;
    };
    std::vector<Request*> loaded;
    for (Request* r : loading) {
        bt_status st = bt::upload_finish(r->ctx);
        while (st == BT_ERR_BUDGET && evict_idle(s)) st = bt::upload_finish(r->ctx);
        if (st == BT_ERR_BUDGET && (wave_holds(r) || others_hold_memory(s, r))) {
            // Graphs of this turn, running graphs or held results will give
            // memory back: requeue in arrival order (the context stays idle
            // and evictable, so a graph that fits alone always progresses).
            s->pool.push_back(r->ctx);
            r->ctx = nullptr;
            r->state = State::Pending;
            s->ready.insert(std::upper_bound(s->ready.begin(), s->ready.end(), r, by_arrival), r);
            std::lock_guard<std::mutex> lk(s->mu);
            ++s->stats.budget_waits;
            continue;
        }
        if (st != BT_OK) {
            const std::string msg = r->ctx->err;
            fail_request(s, r, st, msg);
            continue;
        }
        r->state = State::Loading;
        loaded.push_back(r);
    }
    for (Request* r : loaded) {
        uint32_t samples = 0;
        bt_status st = bt::upload_wait(r->ctx);
        if (st == BT_OK) st = bt::upload_check(r->ctx, &samples);
        if (st == BT_OK) st = bt::upload_adapt(r->ctx);
        if (st == BT_OK) st = bt::reserve_records(r->ctx);
        if (st == BT_OK && r->iterations == 0) {
            // Nothing to iterate: the upload is the result.
            st = bt::prepare_records(r->ctx);
            if (st == BT_OK) st = bt::upload_wait(r->ctx);
            if (st == BT_OK) {
                publish(s, r, BT_OK, "");
                continue;
            }
        }
        if (st == BT_OK) st = bt::batch_attach(s->batch, r->ctx, &r->slot);
        if (st != BT_OK) {
            const std::string msg = bt_batch_last_error(s->batch)[0] ? bt_batch_last_error(s->batch) : r->ctx->err;
            fail_request(s, r, st, msg);
            continue;
        }
        r->state = State::Running;
        s->running.push_back(r);
    }
}

// Step 5: graphs that reached their iteration count leave the batch.
void complete(bt_server* s) {
    std::vector<Request*> still, done;
    for (Request* r : s->running) (r->ctx->iterations >= r->iterations ? done : still).push_back(r);
    if (done.empty()) return;
    s->running.swap(still);
    for (Request* r : done) {
        bt_ctx* c = bt::batch_detach(s->batch, r->slot);
        bt_status st = c ? bt::prepare_records(c) : BT_ERR_CUDA;
        if (!c) {
            r->ctx = nullptr;
            publish(s, r, st, "batch slot lost");
            continue;
        }
        if (st != BT_OK) {
            const std::string msg = c->err;
            fail_request(s, r, st, msg);
        }
    }
    for (Request* r : done) {
        if (!r->ctx || r->state != State::Running) continue;
        bt_status st = bt::upload_wait(r->ctx);
        if (st != BT_OK) {
            const std::string msg = r->ctx->err;
            fail_request(s, r, st, msg);
            continue;
        }
        publish(s, r, BT_OK, "");
    }
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
    for (;;) {
        // 1. Arrivals and releases.
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

        // 2. Admission.
        admit(s);

        // 3. One batch step over the running graphs.
        uint32_t step = 0;
        if (!s->running.empty()) {
            step = std::max<uint32_t>(1, s->opt.max_step);
            for (const Request* r : s->running) step = std::min(step, r->iterations - r->ctx->iterations);
            if (bt_status st = bt_batch_iterate_async(s->batch, step)) {
                fail_running(s, st, bt_batch_last_error(s->batch));
                step = 0;
            }
        }

        // 4. Uploads finish while the batch iterates.
        finish_uploads(s);

        // 5. Completions.
        if (step) {
            if (bt_status st = bt_batch_synchronize(s->batch)) {
                fail_running(s, st, bt_batch_last_error(s->batch));
            } else {
                complete(s);
            }
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (step) ++s->stats.steps;
            s->stats.queued = static_cast<uint32_t>(s->ready.size() + s->future.size() + s->incoming.size());
            s->stats.active = static_cast<uint32_t>(active_count(s));
            s->stats.peak_active = std::max(s->stats.peak_active, s->stats.active);
            s->stats.device_bytes = s->account.used.load();
            s->stats.peak_device_bytes = std::max(s->stats.peak_device_bytes, s->stats.device_bytes);
        }

        // Idle: sleep until the next arrival, a submission or a release.
        if (s->running.empty() && s->counting.empty()) {
            std::unique_lock<std::mutex> lk(s->mu);
            if (s->stop) break;
            if (!s->incoming.empty() || !s->released.empty()) continue;
            if (!s->ready.empty()) {
                // Waiting on the budget: a release wakes us.
                s->work_cv.wait_for(lk, std::chrono::milliseconds(50));
            } else if (!s->future.empty()) {
                const double wait_s = s->future.front()->arrival - s->now();
                if (wait_s > 0)
                    s->work_cv.wait_for(lk, std::chrono::duration<double>(std::min(wait_s, 0.05)));
            } else {
                s->work_cv.wait_for(lk, std::chrono::milliseconds(50));
            }
        }
    }
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

bt_status bt_server_stats_get(bt_server* s, bt_server_stats* out) {
    if (!s || !out) return sfail(s, BT_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->stats;
    out->device_bytes = s->account.used.load();
    return BT_OK;
}

}  // extern "C"
