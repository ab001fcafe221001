// Request server: continuous admission of compress / decompress requests onto a fixed
// set of worker contexts (chain_server_*).
//
// Requests wait in one FIFO queue.  A worker thread (one per context; each context has
// its own stream and arenas, which stay resident between requests) takes the head
// request as soon as it is free and the request's estimated device working set fits in
// the server's memory budget next to the requests already running; a request larger
// than the whole budget runs alone.  The server stamps each request when it is
// submitted, started and finished (steady clock), so callers can read queueing and
// service times without waiting on it promptly.
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "ctx.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    int op = 0;                     // 0 compress, 1 decompress
    chain_batch_item* item = nullptr;
    size_t mem = 0;                 // estimated device working set
    bool done = false;
    chain_status status = CHAIN_OK;
    std::string message;
    Clock::time_point t_submit, t_start, t_end;
};

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

struct chain_server {
    int device = 0;
    size_t budget = 0;
    const chain_opts* opts = nullptr;
    chain_opts opts_copy{};
    std::vector<chain_ctx*> ctx;
    std::vector<std::thread> threads;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<uint64_t> queue;
    std::unordered_map<uint64_t, Request> reqs;
    size_t inflight = 0;
    int running = 0;
    int waiters = 0;                // threads inside chain_server_wait
    uint64_t next_ticket = 1;
    bool stop = false;
};

using namespace chain;

namespace {

// Device bytes a request is expected to hold while it runs: the arenas of this library
// need about 64 bytes per coordinate value to compress and 40 to decompress (the value
// count of a decompress request is read off its output capacity, since the container
// may be in device memory), plus the container.
size_t estimate_bytes(int op, const chain_batch_item& it) {
    if (op == 0) return static_cast<size_t>(it.n) * it.dims * 64 + (1u << 20);
    const size_t values = it.output_capacity / (it.dtype == CHAIN_F64 ? 8 : 4);
    return values * 40 + it.input_bytes + (1u << 20);
}

void worker(chain_server* s, size_t k) {
    chain_ctx* c = s->ctx[k];
    for (;;) {
        uint64_t ticket = 0;
        Request* r = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            // after stop, the queue is drained before the worker exits, so that every
            // submitted request finishes and its waiter is released
            s->cv_work.wait(lk, [&] {
                if (s->queue.empty()) return s->stop;
                const size_t mem = s->reqs.find(s->queue.front())->second.mem;
                return s->running == 0 || s->inflight + mem <= s->budget;
            });
            if (s->queue.empty()) return;
            ticket = s->queue.front();
            s->queue.pop_front();
            r = &s->reqs.find(ticket)->second;
            s->inflight += r->mem;
            ++s->running;
            r->t_start = Clock::now();
        }
        chain_batch_item& it = *r->item;
        chain_status st;
        it.output_bytes = 0;
        if (r->op == 0) {
            size_t len = 0;
            st = chain_compress(c, it.input, it.dtype, it.layout, it.n, it.dims, it.eb, it.p, it.threshold, s->opts,
                                &len);
            if (st == CHAIN_OK) {
                it.output_bytes = len;
                st = (!it.output || it.output_capacity < len)
                         ? set_err(CHAIN_ERR_BUFFER_TOO_SMALL, "output buffer smaller than the container")
                         : chain_result_copy(c, it.output, it.output_capacity);
            }
        } else {
            uint64_t n = 0;
            uint32_t d = 0;
            st = chain_decompress(c, it.input, it.input_bytes, it.dtype, it.layout, it.output, it.output_capacity, &n,
                                  &d);
            it.n = n;
            it.dims = d;
            if (st == CHAIN_OK) it.output_bytes = static_cast<size_t>(n) * d * (it.dtype == CHAIN_F64 ? 8 : 4);
        }
        it.status = st;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            r->t_end = Clock::now();
            r->status = st;
            if (st != CHAIN_OK) r->message = chain_last_error_message();
            r->done = true;
            s->inflight -= r->mem;
            --s->running;
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
}

}  // namespace

extern "C" {

chain_status chain_server_create(int device, int workers, size_t memory_budget_bytes, const chain_opts* opts,
                                 chain_server** out) {
    if (!out) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "out is null");
    *out = nullptr;
    if (workers < 1 || workers > 64) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "workers must be in 1..64");
    chain_server* s = new (std::nothrow) chain_server();
    if (!s) return set_err(CHAIN_ERR_OUT_OF_MEMORY, "server allocation failed");
    s->device = device;
    s->budget = memory_budget_bytes;
    if (opts) {
        s->opts_copy = *opts;
        s->opts = &s->opts_copy;
    }
    for (int k = 0; k < workers; ++k) {
        chain_ctx* c = nullptr;
        const chain_status st = chain_ctx_create(device, nullptr, &c);
        if (st != CHAIN_OK) {
            for (chain_ctx* x : s->ctx) chain_ctx_destroy(x);
            delete s;
            return st;
        }
        s->ctx.push_back(c);
    }
    for (size_t k = 0; k < s->ctx.size(); ++k) s->threads.emplace_back(worker, s, k);
    *out = s;
    return CHAIN_OK;
}

// Stops admission, lets the workers finish every queued request, then waits until no
// thread is left inside chain_server_wait before freeing the server.
void chain_server_destroy(chain_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->threads) t.join();
    {
        std::unique_lock<std::mutex> lk(s->mu);
        s->cv_done.notify_all();
        s->cv_done.wait(lk, [&] { return s->waiters == 0; });
    }
    for (chain_ctx* c : s->ctx) chain_ctx_destroy(c);
    delete s;
}

chain_status chain_server_submit(chain_server* s, int op, chain_batch_item* item, uint64_t* ticket) {
    if (!s || !item || !ticket) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "null argument");
    if (op != 0 && op != 1) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "op must be 0 (compress) or 1 (decompress)");
    const size_t mem = estimate_bytes(op, *item);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "server is stopping");
        const uint64_t t = s->next_ticket++;
        Request& r = s->reqs[t];
        r.op = op;
        r.item = item;
        r.mem = mem;
        r.t_submit = Clock::now();
        s->queue.push_back(t);
        *ticket = t;
    }
    s->cv_work.notify_one();
    return CHAIN_OK;
}

chain_status chain_server_wait(chain_server* s, uint64_t ticket, double* queue_ms, double* service_ms) {
    if (!s) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto f = s->reqs.find(ticket);
    if (f == s->reqs.end()) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "unknown ticket");
    Request* rp = &f->second;   // element references survive rehashing; iterators do not
    ++s->waiters;
    s->cv_done.wait(lk, [&] { return rp->done; });
    const Request r = *rp;
    s->reqs.erase(ticket);
    --s->waiters;
    if (s->stop) s->cv_done.notify_all();   // chain_server_destroy waits for the last waiter
    lk.unlock();
    if (queue_ms) *queue_ms = ms_between(r.t_submit, r.t_start);
    if (service_ms) *service_ms = ms_between(r.t_start, r.t_end);
    if (r.status != CHAIN_OK) return set_err(r.status, r.message);
    return CHAIN_OK;
}

}  // extern "C"
