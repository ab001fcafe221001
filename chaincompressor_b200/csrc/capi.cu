// C ABI of libchain_b200 (declared in include/chain_b200.h).
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "chain_format.h"
#include "ctx.h"

namespace chain {

static thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
uint64_t launch_count_total() { return g_launches.load(std::memory_order_relaxed); }
static std::atomic<uint64_t> g_allocs{0};
void count_alloc() { g_allocs.fetch_add(1, std::memory_order_relaxed); }
uint64_t alloc_count_total() { return g_allocs.load(std::memory_order_relaxed); }

chain_status set_err(chain_status st, const std::string& msg) {
    g_last_error = msg;
    return st;
}

chain_status cuda_err(cudaError_t e, const char* what) {
    const chain_status st = e == cudaErrorMemoryAllocation ? CHAIN_ERR_OUT_OF_MEMORY : CHAIN_ERR_DEVICE;
    cudaGetLastError();  // clear a sticky launch error so the context stays usable
    return set_err(st, std::string(what) + ": " + cudaGetErrorString(e));
}

bool is_device_ptr(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

chain_status ensure_state(chain_ctx* ctx, size_t bytes) {
    if (ctx->state_bytes >= bytes) return CHAIN_OK;
    if (ctx->state_dev) cudaFree(ctx->state_dev);
    if (ctx->state_host) cudaFreeHost(ctx->state_host);
    ctx->state_dev = nullptr;
    ctx->state_host = nullptr;
    ctx->state_bytes = 0;
    const size_t want = bytes < (64u << 10) ? (64u << 10) : bytes;
    count_alloc();
    CHAIN_CUDA(cudaMalloc(&ctx->state_dev, want));
    count_alloc();
    CHAIN_CUDA(cudaMallocHost(&ctx->state_host, want));
    ctx->state_bytes = want;
    return CHAIN_OK;
}

}  // namespace chain

using namespace chain;

namespace {
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};
}  // namespace

extern "C" {

const char* chain_last_error_message(void) { return g_last_error.c_str(); }

chain_status chain_ctx_create(int device, void* cuda_stream, chain_ctx** out) {
    if (!out) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "out is null");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        return set_err(CHAIN_ERR_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= count) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "invalid device ordinal");
    DeviceGuard g(device);
    chain_ctx* ctx = new (std::nothrow) chain_ctx();
    if (!ctx) return set_err(CHAIN_ERR_OUT_OF_MEMORY, "context allocation failed");
    ctx->device = device;
    if (cuda_stream) {
        ctx->stream = static_cast<cudaStream_t>(cuda_stream);
    } else {
        e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete ctx;
            return cuda_err(e, "cudaStreamCreate");
        }
        ctx->own_stream = true;
    }
    *out = ctx;
    return CHAIN_OK;
}

void chain_ctx_destroy(chain_ctx* ctx) {
    if (!ctx) return;
    DeviceGuard g(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    ctx->frame.release();
    ctx->keys.release();
    ctx->coded.release();
    ctx->dec.release();
    ctx->pinned.release();
    ctx->timer.release();
    if (ctx->state_dev) cudaFree(ctx->state_dev);
    if (ctx->state_host) cudaFreeHost(ctx->state_host);
    if (ctx->side) {
        cudaStreamSynchronize(ctx->side);
        cudaStreamDestroy(ctx->side);
    }
    if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
    if (ctx->join_ev) cudaEventDestroy(ctx->join_ev);
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

size_t chain_compress_bound(uint64_t n, uint32_t dims) {
    // header + 5 components (worst case: raw rANS with a full 2^18 table, 3 bytes per
    // symbol, one 132-byte chunk record per 32 symbols) + every value corrected.
    const uint64_t nd = n * dims;
    uint64_t b = header_bytes(dims) + 20 + 16 * nd;
    b += 5 * (12 + 13 + 1 + 9ull * dims + 8 + 64 + 3ull * kRansMaxAlphabet);
    b += 3 * (3 * nd + 132 * (nd / 32 + 1) + 4 * nd);
    b += 2 * (3 * n + 132 * (n / 32 + 1) + 4 * n);
    return static_cast<size_t>(b);
}

chain_status chain_compress(chain_ctx* ctx, const void* points, chain_dtype dtype, chain_layout layout, uint64_t n,
                            uint32_t dims, double eb, int64_t p, int64_t threshold, const chain_opts* opts,
                            size_t* out_len) {
    if (!ctx || !points || !out_len) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "null argument");
    if (dtype != CHAIN_F32 && dtype != CHAIN_F64) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "dtype must be f32 or f64");
    if (layout != CHAIN_SOA && layout != CHAIN_AOS) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "invalid layout");
    // lcps_cpp.cpp:2029-2036
    if (!(eb > 0.0) || !std::isfinite(2.0 * eb))
        return set_err(CHAIN_ERR_INVALID_ARGUMENT, "eb must be positive with finite 2*eb");
    if (p <= 0) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "p must be positive");
    if (n == 0) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "zero-size array to reduction operation minimum which has no identity");
    if (dims == 0) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "points must have at least one dimension");
    if (dims > static_cast<uint32_t>(kMaxDims))
        return set_err(CHAIN_ERR_UNSUPPORTED, "this build supports at most 16 dimensions");
    if (n >= (1ull << 31)) return set_err(CHAIN_ERR_UNSUPPORTED, "this build supports fewer than 2^31 points");
    int bl = 1, l1 = 1, l2 = 1;
    uint32_t bpl = 0, steps = 0;
    if (opts) {
        if (opts->struct_size < offsetof(chain_opts, reserved))
            return set_err(CHAIN_ERR_INVALID_ARGUMENT, "chain_opts.struct_size too small");
        if (opts->bl >= 0) bl = opts->bl != 0;
        if (opts->l1 >= 0) l1 = opts->l1 != 0;
        if (opts->l2 >= 0) l2 = opts->l2 != 0;
        bpl = opts->rans_bytes_per_lane;
        steps = opts->rans_max_steps;
    }
    DeviceGuard g(ctx->device);
    ctx->result = nullptr;
    ctx->result_len = 0;
    g_last_error.clear();
    return encode_frame(ctx, points, dtype, layout, n, dims, eb, p, threshold, bl, l1, l2, bpl, steps, out_len);
}

chain_status chain_result_copy(chain_ctx* ctx, void* dst, size_t capacity) {
    if (!ctx || !dst) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "null argument");
    if (!ctx->result) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "no compressed result in this context");
    if (capacity < ctx->result_len) return set_err(CHAIN_ERR_BUFFER_TOO_SMALL, "destination buffer too small");
    DeviceGuard g(ctx->device);
    CHAIN_CUDA(cudaMemcpyAsync(dst, ctx->result, ctx->result_len, cudaMemcpyDefault, ctx->stream));
    CHAIN_CUDA(cudaStreamSynchronize(ctx->stream));
    return CHAIN_OK;
}

const void* chain_result_device_ptr(const chain_ctx* ctx) { return ctx ? ctx->result : nullptr; }

chain_status chain_peek(const void* container, size_t len, uint64_t* n, uint32_t* dims, chain_dtype* input_dtype) {
    if (!container) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "null container");
    DecodePlan plan;
    if (!parse_container(static_cast<const uint8_t*>(container), len, &plan))
        return set_err(CHAIN_ERR_CORRUPT_STREAM, "LCG2: container failed validation (check at chain_format.h:" +
                                                     std::to_string(plan.why) + ")");
    if (n) *n = plan.N;
    if (dims) *dims = plan.D;
    if (input_dtype) *input_dtype = plan.input_dtype == 8 ? CHAIN_F64 : CHAIN_F32;
    return CHAIN_OK;
}

chain_status chain_decompress(chain_ctx* ctx, const void* container, size_t len, chain_dtype out_dtype,
                              chain_layout out_layout, void* out, size_t out_capacity_bytes, uint64_t* n,
                              uint32_t* dims) {
    if (!ctx || !container || !out) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "null argument");
    if (out_dtype != CHAIN_F32 && out_dtype != CHAIN_F64)
        return set_err(CHAIN_ERR_INVALID_ARGUMENT, "dtype must be f32 or f64");
    if (out_layout != CHAIN_SOA && out_layout != CHAIN_AOS) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "invalid layout");
    DeviceGuard g(ctx->device);
    g_last_error.clear();
    return decode_frame(ctx, container, len, out_dtype, out_layout, out, out_capacity_bytes, n, dims);
}

chain_status chain_debug_streams(chain_ctx* ctx, int64_t* idrel, int64_t* diff, uint64_t* ndiff, int64_t* keep,
                                 uint64_t* nkeep, int64_t* choice2, uint64_t* nblocks, int64_t* rel) {
    if (!ctx || !ctx->result) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "no compressed result in this context");
    DeviceGuard g(ctx->device);
    const EncodeDebug& d = ctx->dbg;
    if (ndiff) *ndiff = d.ndiff;
    if (nkeep) *nkeep = d.nkeep;
    if (nblocks) *nblocks = d.nblocks;
    // streams are stored with esz bytes per value (1, 2 or 4)
    auto fetch = [&](const void* src, uint32_t esz, uint64_t count, int64_t* dst) -> chain_status {
        if (!dst || count == 0) return CHAIN_OK;
        std::vector<uint8_t> tmp(count * esz);
        CHAIN_CUDA(cudaMemcpyAsync(tmp.data(), src, count * esz, cudaMemcpyDeviceToHost, ctx->stream));
        CHAIN_CUDA(cudaStreamSynchronize(ctx->stream));
        for (uint64_t i = 0; i < count; ++i) {
            if (esz == 1) {
                dst[i] = tmp[i];
            } else if (esz == 2) {
                uint16_t v;
                std::memcpy(&v, tmp.data() + 2 * i, 2);
                dst[i] = v;
            } else {
                uint32_t v;
                std::memcpy(&v, tmp.data() + 4 * i, 4);
                dst[i] = v;
            }
        }
        return CHAIN_OK;
    };
    chain_status s;
    if ((s = fetch(d.idrel, 4, d.n, idrel)) != CHAIN_OK) return s;
    if ((s = fetch(d.diff, d.kd_esz, d.ndiff * d.dims, diff)) != CHAIN_OK) return s;
    if ((s = fetch(d.keep, d.kd_esz, d.nkeep * d.dims, keep)) != CHAIN_OK) return s;
    if ((s = fetch(d.choice2, 1, d.nblocks, choice2)) != CHAIN_OK) return s;
    if ((s = fetch(d.rel, d.rel_esz, d.n * d.dims, rel)) != CHAIN_OK) return s;
    return CHAIN_OK;
}

uint64_t chain_launch_count(void) { return launch_count_total(); }
uint64_t chain_alloc_count(void) { return alloc_count_total(); }

chain_status chain_set_stage_timing(chain_ctx* ctx, int enabled) {
    if (!ctx) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "null context");
    ctx->timer.enabled = enabled != 0;
    return CHAIN_OK;
}

int chain_stage_times(const chain_ctx* ctx, const char** names, float* ms, int max) {
    if (!ctx) return 0;
    const int n = ctx->timer.ready > 0 ? ctx->timer.ready - 1 : 0;
    for (int i = 0; i < n && i < max; ++i) {
        if (names) names[i] = ctx->timer.names[i + 1];
        if (ms) ms[i] = ctx->timer.ms[i + 1];
    }
    return n;
}

}  // extern "C"
