// chain_decompress_noalloc: decompression that allocates no memory.
//
// Some callers cannot allocate at the moment they decode a frame: in-situ readers and
// analysis plug-ins that run inside a host application which owns the whole device
// memory pool (or runs under a hard per-process memory cap), and latency-critical loops
// that must not pay for cudaMalloc / cudaFree, which can synchronise the whole device.
// chain_decompress needs a context whose arena grows with the frame, so it is not usable
// there.  This entry point runs the same decoder (decode_frame, the same kernels and the
// same bit-exact output) with every working buffer carved out of one file-scope device
// array of fixed size, and its host mirror out of a file-scope host array.
//
// Limits and sharing:
//   * The device array holds kNoAllocScratchBytes (64 MiB).  A frame whose decoder
//     working set (the decoded integer streams, the rANS tables, a copy of a host
//     container, and a staging copy of host output) does not fit is rejected with
//     CHAIN_ERR_UNSUPPORTED and a message giving the bytes it needs.
//   * Every GPU on which this module is loaded holds the array until the process exits.
//   * Every call on a device shares the array, which keeps the last call's contents;
//     decode_frame clears everything that must start at zero (its state and counters)
//     at the start of each call.  Calls that overlapped on the GPU would race on the
//     array, so calls are serialised: each holds a process-wide lock and returns only
//     after its GPU work on `cuda_stream` has completed.
//   * The first call on a device (the current device of the calling thread) looks up
//     the array's device address with cudaGetSymbolAddress; make that first call before
//     any stream capture begins on that device.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "ctx.h"

namespace chain {

constexpr size_t kNoAllocScratchBytes = 64ull << 20;
constexpr size_t kNoAllocStateBytes = 64u << 10;   // decoder state at the front of the array
constexpr int kNoAllocMaxDevices = 64;

// The scratch array.  In host code this name is only a stand-in for the symbol; its
// device address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

static std::mutex g_noalloc_lock;
static uint8_t* g_noalloc_dev[kNoAllocMaxDevices];   // device address of the array, per device
alignas(256) static uint8_t g_noalloc_host_state[kNoAllocStateBytes];

// Set-up for the current device: the array's device address (first call only).
static chain_status noalloc_scratch(int dev, uint8_t** out) {
    if (!g_noalloc_dev[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return cuda_err(e != cudaSuccess ? e : cudaErrorInvalidSymbol,
                                                    "cudaGetSymbolAddress(decoder scratch)");
        g_noalloc_dev[dev] = static_cast<uint8_t*>(p);
    }
    *out = g_noalloc_dev[dev];
    return CHAIN_OK;
}

}  // namespace chain

using namespace chain;

extern "C" chain_status chain_decompress_noalloc(const void* container, size_t len, chain_dtype out_dtype,
                                                 chain_layout out_layout, void* out, size_t out_capacity_bytes,
                                                 uint64_t* n, uint32_t* dims, void* cuda_stream) {
    if (!container || !out) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "null argument");
    if (out_dtype != CHAIN_F32 && out_dtype != CHAIN_F64)
        return set_err(CHAIN_ERR_INVALID_ARGUMENT, "dtype must be f32 or f64");
    if (out_layout != CHAIN_SOA && out_layout != CHAIN_AOS) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "invalid layout");
    if (decode_state_bytes() > kNoAllocStateBytes)
        return set_err(CHAIN_ERR_UNSUPPORTED, "decoder state does not fit the no-allocation scratch");
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_err(e, "cudaGetDevice");
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        return set_err(CHAIN_ERR_UNSUPPORTED, "chain_decompress_noalloc supports device ordinals below 64");
    std::lock_guard<std::mutex> lock(g_noalloc_lock);
    set_err(CHAIN_OK, std::string());
    uint8_t* scratch = nullptr;
    chain_status s = noalloc_scratch(dev, &scratch);
    if (s != CHAIN_OK) return s;

    chain_ctx ctx;   // a view: nothing in it owns memory, nothing is released
    ctx.device = dev;
    ctx.stream = static_cast<cudaStream_t>(cuda_stream);
    ctx.state_dev = scratch;
    ctx.state_host = g_noalloc_host_state;
    ctx.state_bytes = kNoAllocStateBytes;
    ctx.dec.base = scratch + kNoAllocStateBytes;
    ctx.dec.cap = kNoAllocScratchBytes - kNoAllocStateBytes;
    ctx.dec.fixed = true;
    s = decode_frame(&ctx, container, len, out_dtype, out_layout, out, out_capacity_bytes, n, dims);
    // Early error returns can leave work queued; the array is free again only once the
    // stream is idle.
    e = cudaStreamSynchronize(ctx.stream);
    if (s == CHAIN_ERR_OUT_OF_MEMORY && ctx.dec.requested > ctx.dec.cap)
        return set_err(CHAIN_ERR_UNSUPPORTED,
                       "frame too large for chain_decompress_noalloc: its decoder working set is " +
                           std::to_string(ctx.dec.requested) + " bytes, the fixed scratch holds " +
                           std::to_string(ctx.dec.cap) + " (decode it with chain_decompress)");
    if (s == CHAIN_OK && e != cudaSuccess) return cuda_err(e, "cudaStreamSynchronize");
    return s;
}
