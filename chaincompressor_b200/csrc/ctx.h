// Host-side context, device arena and error plumbing of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <string>

#include "../../include/chain_b200.h"

namespace chain {

void count_alloc();   // counts the library's own cudaMalloc / cudaMallocHost calls

// Bump allocator over one device allocation.  reserve() grows the allocation between
// calls (never while kernels of the current call are queued on it).  A `fixed` arena
// lies over memory it does not own: reserve() never allocates or frees, it only
// reports whether `bytes` fit (and records the request in `requested`).
struct Arena {
    uint8_t* base = nullptr;
    size_t cap = 0;
    size_t used = 0;
    bool fixed = false;
    size_t requested = 0;
    cudaError_t reserve(size_t bytes) {
        used = 0;
        if (fixed) {
            requested = bytes;
            return bytes <= cap ? cudaSuccess : cudaErrorMemoryAllocation;
        }
        if (bytes <= cap) return cudaSuccess;
        if (base) cudaFree(base);
        base = nullptr;
        cap = 0;
        size_t want = bytes + bytes / 8 + (1u << 20);
        count_alloc();
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&base), want);
        if (e != cudaSuccess) { base = nullptr; return e; }
        cap = want;
        return cudaSuccess;
    }
    template <typename T>
    T* take(size_t count) {
        const size_t off = (used + 255) & ~size_t(255);
        const size_t bytes = count * sizeof(T);
        if (off + bytes > cap) return nullptr;
        used = off + bytes;
        return reinterpret_cast<T*>(base + off);
    }
    static size_t need(size_t count, size_t elem) { return ((count * elem + 255) & ~size_t(255)); }
    void release() {
        if (base) cudaFree(base);
        base = nullptr;
        cap = used = 0;
    }
};

struct PinnedBuf {
    uint8_t* ptr = nullptr;
    size_t cap = 0;
    cudaError_t reserve(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        cap = 0;
        count_alloc();
        cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&ptr), bytes);
        if (e != cudaSuccess) { ptr = nullptr; return e; }
        cap = bytes;
        return cudaSuccess;
    }
    void release() {
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        cap = 0;
    }
};

// Optional per-stage timing with CUDA events on the library stream (enabled per
// context; used by bench.py for the per-kernel roofline and by tracing).
struct StageTimer {
    static constexpr int kMax = 48;
    bool enabled = false;
    int count = 0;
    const char* names[kMax];
    cudaEvent_t ev[kMax];
    bool created = false;
    float ms[kMax];
    int ready = 0;
    void begin(cudaStream_t s) {
        count = 0;
        ready = 0;
        if (!enabled) return;
        if (!created) {
            for (int i = 0; i < kMax; ++i) cudaEventCreate(&ev[i]);
            created = true;
        }
        mark("start", s);
    }
    void mark(const char* name, cudaStream_t s) {
        if (!enabled || count >= kMax) return;
        names[count] = name;
        cudaEventRecord(ev[count], s);
        ++count;
    }
    // Call after the stream was synchronised.
    void finish() {
        if (!enabled) return;
        for (int i = 1; i < count; ++i) cudaEventElapsedTime(&ms[i], ev[i - 1], ev[i]);
        ready = count;
    }
    void release() {
        if (created) for (int i = 0; i < kMax; ++i) cudaEventDestroy(ev[i]);
        created = false;
    }
};

// The encoder's integer streams of the last compress (device memory).  idrel is stored
// with four bytes per value, choice2 with one, diff and keep with kd_esz (1, 2 or 4),
// rel with rel_esz (1 when p <= 256, else 4).
struct EncodeDebug {
    const uint32_t* idrel = nullptr;
    const void* diff = nullptr;
    const void* keep = nullptr;
    uint32_t kd_esz = 4;
    const uint8_t* choice2 = nullptr;
    const void* rel = nullptr;
    uint32_t rel_esz = 4;
    uint64_t n = 0, ndiff = 0, nkeep = 0, nblocks = 0;
    uint32_t dims = 0;
};

}  // namespace chain

struct chain_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // The encoder's side stream (highest priority; created by the first compress) and the
    // events that fork work onto it after level 1 and join it back before planning.
    cudaStream_t side = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    chain::Arena frame;    // per-frame working buffers (encoder)
    chain::Arena keys;     // encoder block keys, sort buffers and record keys (sized once the key width is known)
    chain::Arena coded;    // encoder entropy/output buffers
    chain::Arena dec;      // decoder buffers
    chain::PinnedBuf pinned;
    void* state_dev = nullptr;    // device scratch scalars (EncState / DecState)
    // Host mirror of state_dev: pinned when the context allocated it (ensure_state).
    // chain_decompress_noalloc points it at a pageable static array instead; copies to
    // and from pageable memory are synchronous, which that entry point relies on no more
    // than decode_frame does (it synchronises the stream before reading the mirror).
    void* state_host = nullptr;
    size_t state_bytes = 0;
    const uint8_t* result = nullptr;  // device container of the last compress
    size_t result_len = 0;
    chain::EncodeDebug dbg;
    chain::StageTimer timer;
};

namespace chain {

chain_status set_err(chain_status st, const std::string& msg);
chain_status cuda_err(cudaError_t e, const char* what);
bool is_device_ptr(const void* p);

#define CHAIN_CUDA(expr)                                        \
    do {                                                        \
        cudaError_t _e = (expr);                                \
        if (_e != cudaSuccess) return ::chain::cuda_err(_e, #expr); \
    } while (0)

#define CHAIN_LAUNCH_CHECK(what)                                \
    do {                                                        \
        cudaError_t _e = cudaGetLastError();                    \
        if (_e != cudaSuccess) return ::chain::cuda_err(_e, what); \
    } while (0)

chain_status ensure_state(chain_ctx* ctx, size_t bytes);

chain_status encode_frame(chain_ctx* ctx, const void* points, chain_dtype dtype, chain_layout layout,
                          uint64_t n, uint32_t dims, double eb, int64_t p, int64_t threshold,
                          int bl, int l1, int l2, uint32_t bytes_per_lane, uint32_t max_steps, size_t* out_len);

chain_status decode_frame(chain_ctx* ctx, const void* container, size_t len, chain_dtype out_dtype,
                          chain_layout out_layout, void* out, size_t out_capacity, uint64_t* n,
                          uint32_t* dims);

// Bytes of device state (and of its host mirror) that decode_frame uses.
size_t decode_state_bytes();

}  // namespace chain
