// Batched compression and decompression of independent frames (chain_batch_*).
//
// A batch object owns `workers` library contexts on one device, each with its own
// non-blocking stream and its own arenas (kept warm between batches).  A batch call
// starts one host thread per context; the threads claim frames from a shared counter
// and run the ordinary per-frame path on their own context, so the launches, host
// round trips and small kernels of many frames overlap on the GPU.  Results are the
// same bytes (compress) and the same values (decompress) as one-frame calls.
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <string>
#include <thread>
#include <vector>

#include "ctx.h"

struct chain_batch {
    int device = 0;
    std::vector<chain_ctx*> ctx;
    size_t active = 0;          // contexts a call uses (0 = all)
    bool tuned = false;
    chain_opts tuned_opts{};    // used by chain_batch_compress when its opts are null
};

using namespace chain;

namespace {

// Runs fn(ctx, index) for every item on the batch's contexts; returns the first
// failing item's status and message (or CHAIN_OK).
template <typename Fn>
chain_status run_batch(chain_batch* b, size_t count, chain_batch_item* items, Fn fn) {
    std::atomic<size_t> next{0};
    std::vector<std::string> msg(count);
    const size_t nthreads = std::min(b->active ? b->active : b->ctx.size(), count);
    std::vector<std::thread> threads;
    threads.reserve(nthreads);
    for (size_t t = 0; t < nthreads; ++t) {
        threads.emplace_back([&, t]() {
            chain_ctx* c = b->ctx[t];
            for (;;) {
                const size_t i = next.fetch_add(1, std::memory_order_relaxed);
                if (i >= count) break;
                items[i].status = fn(c, items[i]);
                if (items[i].status != CHAIN_OK) msg[i] = chain_last_error_message();
            }
        });
    }
    for (auto& th : threads) th.join();
    for (size_t i = 0; i < count; ++i)
        if (items[i].status != CHAIN_OK)
            return set_err(items[i].status, "frame " + std::to_string(i) + ": " + msg[i]);
    return set_err(CHAIN_OK, std::string());
}

}  // namespace

extern "C" {

chain_status chain_batch_create(int device, int workers, chain_batch** out) {
    if (!out) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "out is null");
    *out = nullptr;
    if (workers < 1 || workers > 64) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "workers must be in 1..64");
    chain_batch* b = new (std::nothrow) chain_batch();
    if (!b) return set_err(CHAIN_ERR_OUT_OF_MEMORY, "batch allocation failed");
    b->device = device;
    for (int k = 0; k < workers; ++k) {
        chain_ctx* c = nullptr;
        const chain_status s = chain_ctx_create(device, nullptr, &c);
        if (s != CHAIN_OK) {
            chain_batch_destroy(b);
            return s;
        }
        b->ctx.push_back(c);
    }
    *out = b;
    return CHAIN_OK;
}

void chain_batch_destroy(chain_batch* b) {
    if (!b) return;
    for (chain_ctx* c : b->ctx) chain_ctx_destroy(c);
    delete b;
}

chain_status chain_batch_compress(chain_batch* b, chain_batch_item* items, size_t count, const chain_opts* opts) {
    if (!b || (count && !items)) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "null argument");
    if (!opts && b->tuned) opts = &b->tuned_opts;
    return run_batch(b, count, items, [opts](chain_ctx* c, chain_batch_item& it) -> chain_status {
        it.output_bytes = 0;
        size_t len = 0;
        chain_status s = chain_compress(c, it.input, it.dtype, it.layout, it.n, it.dims, it.eb, it.p, it.threshold,
                                        opts, &len);
        if (s != CHAIN_OK) return s;
        it.output_bytes = len;
        if (!it.output || it.output_capacity < len)
            return set_err(CHAIN_ERR_BUFFER_TOO_SMALL, "output holds " + std::to_string(it.output_capacity) +
                                                           " bytes, the container has " + std::to_string(len));
        return chain_result_copy(c, it.output, it.output_capacity);
    });
}

chain_status chain_batch_decompress(chain_batch* b, chain_batch_item* items, size_t count) {
    if (!b || (count && !items)) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "null argument");
    return run_batch(b, count, items, [](chain_ctx* c, chain_batch_item& it) -> chain_status {
        it.output_bytes = 0;
        uint64_t n = 0;
        uint32_t d = 0;
        const chain_status s = chain_decompress(c, it.input, it.input_bytes, it.dtype, it.layout, it.output,
                                                it.output_capacity, &n, &d);
        it.n = n;
        it.dims = d;
        if (s == CHAIN_OK) it.output_bytes = static_cast<size_t>(n) * d * (it.dtype == CHAIN_F64 ? 8 : 4);
        return s;
    });
}

chain_status chain_batch_tune(chain_batch* b, chain_batch_item* items, size_t count, chain_tune_result* result) {
    if (!b || !items || !count || !result) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "null or empty argument");
    using Clock = std::chrono::steady_clock;
    struct Cand {
        uint32_t steps;
        size_t workers;
    };
    const size_t all = b->ctx.size();
    std::vector<Cand> cands;
    for (uint32_t steps : {1024u, 512u, 256u})
        for (size_t w : {all, (all + 1) / 2, (all + 3) / 4})
            if (w >= 1 && (cands.empty() || cands.back().steps != steps || cands.back().workers != w))
                cands.push_back({steps, w});
    b->tuned = false;
    const size_t saved_active = b->active;
    double best_ms = 0, default_ms = 0;
    uint64_t best_bytes = 0, default_bytes = 0;
    Cand best{1024u, all};
    chain_status st = CHAIN_OK;
    for (size_t ci = 0; ci < cands.size() && st == CHAIN_OK; ++ci) {
        chain_opts o{};
        o.struct_size = sizeof(chain_opts);
        o.bl = o.l1 = o.l2 = 1;
        o.rans_max_steps = cands[ci].steps;
        b->active = cands[ci].workers;
        double ms = 0;
        uint64_t bytes = 0;
        for (int rep = 0; rep < 3 && st == CHAIN_OK; ++rep) {   // a warm-up, then the best of two
            const auto t0 = Clock::now();
            st = chain_batch_compress(b, items, count, &o);
            const double t = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
            if (rep == 1 || (rep == 2 && t < ms)) ms = t;
        }
        if (st != CHAIN_OK) break;
        for (size_t i = 0; i < count; ++i) bytes += items[i].output_bytes;
        if (ci == 0) {
            default_ms = best_ms = ms;
            default_bytes = best_bytes = bytes;
        } else if (ms < best_ms && static_cast<double>(bytes) <= 1.003 * static_cast<double>(default_bytes)) {
            best_ms = ms;
            best_bytes = bytes;
            best = cands[ci];
        }
    }
    b->active = saved_active;
    if (st != CHAIN_OK) return st;
    b->tuned_opts = chain_opts{};
    b->tuned_opts.struct_size = sizeof(chain_opts);
    b->tuned_opts.bl = b->tuned_opts.l1 = b->tuned_opts.l2 = 1;
    b->tuned_opts.rans_max_steps = best.steps;
    b->tuned = true;
    b->active = best.workers;
    result->rans_max_steps = best.steps;
    result->workers = static_cast<uint32_t>(best.workers);
    result->best_ms = best_ms;
    result->default_ms = default_ms;
    result->best_bytes = best_bytes;
    result->default_bytes = default_bytes;
    return set_err(CHAIN_OK, std::string());
}

}  // extern "C"
