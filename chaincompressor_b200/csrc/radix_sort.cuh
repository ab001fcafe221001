// Stable LSD radix sort of (key, index) pairs over only the key bits in use.
//
// Used by the encoder to group points by block key: after sorting the Z-order block
// keys stably, the points of one block are adjacent and in increasing index order, so
// "the next point of the same block" is the sorted neighbour (lcps_cpp.cpp:2116-2138
// computes the same relation with a hash map).
//
// Each 8-bit pass is three launches: a per-tile digit histogram, a device-wide
// exclusive scan of the digit-major count table, and a stable scatter.  The scatter
// ranks keys inside a 4096-key tile with warp match_any + popc (each warp owns a
// contiguous 512-key slice, processed 32 keys per round in order), so equal digits
// keep their input order.
#pragma once

#include "chain_common.cuh"
#include "scan.cuh"

namespace chain {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortBins = 256;

template <typename KT>
__global__ void __launch_bounds__(kSortThreads)
radix_hist_kernel(const KT* __restrict__ keys, uint64_t n, int shift, uint32_t* __restrict__ counts,
                  uint32_t num_tiles) {
    __shared__ uint32_t hist[kSortBins];
    hist[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kSortTile;
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const uint64_t i = base + static_cast<uint64_t>(k) * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&hist[static_cast<uint32_t>(keys[i] >> shift) & 0xFFu], 1u);
    }
    __syncthreads();
    counts[static_cast<uint64_t>(threadIdx.x) * num_tiles + blockIdx.x] = hist[threadIdx.x];
}

template <typename KT>
__global__ void __launch_bounds__(kSortThreads)
radix_scatter_kernel(const KT* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                     KT* __restrict__ keys_out, uint32_t* __restrict__ vals_out, uint64_t n, int shift,
                     const uint32_t* __restrict__ offsets, uint32_t num_tiles) {
    __shared__ uint32_t whist[kSortWarps][kSortBins];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int t = threadIdx.x; t < kSortWarps * kSortBins; t += kSortThreads) (&whist[0][0])[t] = 0;
    __syncthreads();
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kSortTile + static_cast<uint64_t>(warp) * (kSortItems * 32);
    KT key[kSortItems];
    uint32_t rank[kSortItems];
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint64_t i = base + static_cast<uint64_t>(r) * 32 + lane;
        const bool valid = i < n;
        key[r] = valid ? keys_in[i] : KT(0);
        const uint32_t digit = static_cast<uint32_t>(key[r] >> shift) & 0xFFu;
        const uint32_t active = __ballot_sync(0xffffffffu, valid);
        uint32_t peers = 0;
        if (valid) peers = __match_any_sync(active, digit);
        const uint32_t prior = valid ? whist[warp][digit] : 0u;
        __syncwarp();
        rank[r] = prior + __popc(peers & lt);
        if (valid && (peers & lt) == 0) whist[warp][digit] = prior + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    {
        const int d = threadIdx.x;  // one thread per digit
        uint32_t run = offsets[static_cast<uint64_t>(d) * num_tiles + blockIdx.x];
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t c = whist[w][d];
            whist[w][d] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint64_t i = base + static_cast<uint64_t>(r) * 32 + lane;
        if (i < n) {
            const uint32_t digit = static_cast<uint32_t>(key[r] >> shift) & 0xFFu;
            const uint32_t pos = whist[warp][digit] + rank[r];
            keys_out[pos] = key[r];
            vals_out[pos] = vals_in ? vals_in[i] : static_cast<uint32_t>(i);
        }
    }
}

struct CountIn {
    const uint32_t* c;
    __device__ uint32_t operator()(uint64_t i) const { return c[i]; }
};
struct CountOut {
    uint32_t* c;
    __device__ void operator()(uint64_t i, uint32_t prefix, uint32_t) const { c[i] = prefix; }
};

inline uint32_t radix_tiles(uint64_t n) { return static_cast<uint32_t>((n + kSortTile - 1) / kSortTile); }

// Scratch requirement (bytes) of radix_sort_pairs for n keys.
inline size_t radix_counts_elems(uint64_t n) { return static_cast<size_t>(radix_tiles(n)) * kSortBins; }

// Sorts keys_in (values implicitly 0..n-1) by bits [0, key_bits), stably.  Ping-pongs
// between (keys_a, vals_a) and (keys_b, vals_b); keys_in is only read.  Returns true
// when the result is in the *_b buffers.  counts: radix_counts_elems(n) u32;
// scan_buf: scan_tiles(counts) u32.
template <typename KT>
bool radix_sort_pairs(const KT* keys_in, KT* keys_a, uint32_t* vals_a, KT* keys_b, uint32_t* vals_b, uint64_t n,
                      int key_bits, uint32_t* counts, uint32_t* scan_buf, cudaStream_t stream) {
    const uint32_t tiles = radix_tiles(n);
    int passes = (key_bits + 7) / 8;
    if (passes == 0) passes = 1;  // one pass produces the identity permutation
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        const KT* kin = p == 0 ? keys_in : (p % 2 == 1 ? keys_a : keys_b);
        const uint32_t* vin = p == 0 ? nullptr : (p % 2 == 1 ? vals_a : vals_b);
        KT* kout = p % 2 == 0 ? keys_a : keys_b;
        uint32_t* vout = p % 2 == 0 ? vals_a : vals_b;
        radix_hist_kernel<KT><<<tiles, kSortThreads, 0, stream>>>(kin, n, shift, counts, tiles);
        const uint64_t ncounts = static_cast<uint64_t>(tiles) * kSortBins;
        device_exclusive_scan<uint32_t>(CountIn{counts}, CountOut{counts}, ncounts, scan_buf,
                                        static_cast<uint32_t*>(nullptr), stream);
        radix_scatter_kernel<KT><<<tiles, kSortThreads, 0, stream>>>(kin, vin, kout, vout, n, shift, counts, tiles);
    }
    return passes % 2 == 0;
}

}  // namespace chain
