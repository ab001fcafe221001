// Stable LSD radix sort of (key, index) pairs over only the key bits in use.
//
// Used by the encoder to group points by block key: after sorting the Z-order block
// keys stably, the points of one block are adjacent and in increasing index order, so
// "the next point of the same block" is the sorted neighbour (lcps_cpp.cpp:2116-2138
// computes the same relation with a hash map).
//
// Each 8-bit pass is three launches: a per-tile digit histogram, a device-wide
// exclusive scan of the digit-major count table, and a stable scatter.  The scatter
// loads its whole tile at once (indices wait in shared memory in input order), ranks
// keys with 8 ballots per 32 keys (each warp owns a contiguous slice, processed 32 keys
// per round in order, so equal digits keep their input order), reorders the tile by
// digit in shared memory, and writes each digit's run to its global position with
// consecutive threads on consecutive addresses.
#pragma once

#include "chain_common.cuh"
#include "scan.cuh"

namespace chain {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortBins = 256;

template <typename KT>
struct SortShape {
    static constexpr int kItems = sizeof(KT) > 4 ? 8 : 12;
    static constexpr int kTile = kSortThreads * kItems;
};

template <typename KT>
__global__ void __launch_bounds__(kSortThreads)
radix_hist_kernel(const KT* __restrict__ keys, uint64_t n, int shift, uint32_t* __restrict__ counts,
                  uint32_t num_tiles) {
    constexpr int I = SortShape<KT>::kItems, TILE = SortShape<KT>::kTile;
    __shared__ uint32_t hist[kSortBins];
    hist[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * TILE;
    const uint32_t rem = base >= n ? 0u : static_cast<uint32_t>(min(n - base, static_cast<uint64_t>(TILE)));
    // all loads first (one round trip per thread), then the shared-memory counts
    KT k[I];
#pragma unroll
    for (int r = 0; r < I; ++r) {
        const uint32_t i = r * kSortThreads + threadIdx.x;
        k[r] = i < rem ? __ldg(keys + base + i) : KT(0);
    }
#pragma unroll
    for (int r = 0; r < I; ++r)
        if (static_cast<uint32_t>(r * kSortThreads + threadIdx.x) < rem)
            atomicAdd(&hist[static_cast<uint32_t>(k[r] >> shift) & 0xFFu], 1u);
    __syncthreads();
    counts[static_cast<uint64_t>(threadIdx.x) * num_tiles + blockIdx.x] = hist[threadIdx.x];
}

// Shared-memory staging of a tile's reordered pairs: one 8-byte word per pair for
// 32-bit keys, separate arrays for 64-bit keys.
template <typename KT>
struct ScatterStage {
    KT key[SortShape<KT>::kTile];
    uint32_t val[SortShape<KT>::kTile];
    __device__ __forceinline__ void put(uint32_t i, KT k, uint32_t v) { key[i] = k; val[i] = v; }
    __device__ __forceinline__ void get(uint32_t i, KT& k, uint32_t& v) const { k = key[i]; v = val[i]; }
};
template <>
struct ScatterStage<uint32_t> {
    uint2 kv[SortShape<uint32_t>::kTile];
    __device__ __forceinline__ void put(uint32_t i, uint32_t k, uint32_t v) { kv[i] = make_uint2(k, v); }
    __device__ __forceinline__ void get(uint32_t i, uint32_t& k, uint32_t& v) const {
        const uint2 t = kv[i];
        k = t.x;
        v = t.y;
    }
};

// Four CTAs per SM (63 registers, <= 46 KB of shared memory): the ranking loop is
// latency-bound, so resident warps matter more than registers.
template <typename KT>
__global__ void __launch_bounds__(kSortThreads, 4)
radix_scatter_kernel(const KT* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                     KT* __restrict__ keys_out, uint32_t* __restrict__ vals_out, uint64_t n, int shift,
                     const uint32_t* __restrict__ offsets, uint32_t num_tiles) {
    constexpr int I = SortShape<KT>::kItems;
    __shared__ uint32_t whist[kSortWarps][kSortBins];
    __shared__ int32_t delta[kSortBins];         // global position - tile-local position, per digit
    __shared__ uint32_t scratch[33];
    __shared__ ScatterStage<KT> stage;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int t = threadIdx.x; t < kSortWarps * kSortBins; t += kSortThreads) (&whist[0][0])[t] = 0;
    __syncthreads();
    const uint64_t tile0 = static_cast<uint64_t>(blockIdx.x) * SortShape<KT>::kTile;
    const uint64_t base = tile0 + static_cast<uint64_t>(warp) * (I * 32);
    // keys of this warp's slice that exist (the slice is [base, base + 32 I))
    const uint32_t rem = base >= n ? 0u : static_cast<uint32_t>(min(n - base, static_cast<uint64_t>(I * 32)));
    const KT* kin = keys_in + base;
    const uint32_t* vin = vals_in ? vals_in + base : nullptr;
    KT key[I];
    uint32_t rd[I];   // rank within the warp's digit run (bits 0..15) | digit << 16
    const uint32_t lt = lanemask_lt();
    // all loads first, so that they are in flight together (indices are implicit on
    // the first pass); the indices wait in shared memory, in input order, until the
    // tile's positions are known
    __shared__ uint32_t sval_in[SortShape<KT>::kTile];
    uint32_t* my_val = sval_in + warp * (I * 32) + lane;
    {
        uint32_t val[I];
#pragma unroll
        for (int r = 0; r < I; ++r) {
            const uint32_t i = r * 32 + lane;
            key[r] = i < rem ? kin[i] : KT(0);
            val[r] = i < rem ? (vin ? vin[i] : static_cast<uint32_t>(base) + i) : 0u;
        }
#pragma unroll
        for (int r = 0; r < I; ++r) my_val[r * 32] = val[r];
    }
    // stable rank within the warp: lanes with an equal digit found with 8 ballots
#pragma unroll
    for (int r = 0; r < I; ++r) {
        const bool valid = static_cast<uint32_t>(r * 32 + lane) < rem;
        const uint32_t digit = static_cast<uint32_t>(key[r] >> shift) & 0xFFu;
        uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const bool bit = (digit >> b) & 1u;
            const uint32_t bal = __ballot_sync(0xffffffffu, bit);
            peers &= bit ? bal : ~bal;
        }
        const uint32_t prior = valid ? whist[warp][digit] : 0u;
        __syncwarp();
        rd[r] = (prior + __popc(peers & lt)) | (digit << 16);
        if (valid && (peers & lt) == 0) whist[warp][digit] = prior + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    {
        // per digit: tile count, then per-warp offsets inside the tile
        const int d = threadIdx.x;
        uint32_t cnt = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) cnt += whist[w][d];
        uint32_t tot;
        const uint32_t start = block_exclusive_sum(cnt, scratch, &tot);
        delta[d] = static_cast<int32_t>(offsets[static_cast<uint64_t>(d) * num_tiles + blockIdx.x] - start);
        uint32_t run = start;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t c = whist[w][d];
            whist[w][d] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < I; ++r) {
        const uint32_t v = my_val[r * 32];
        if (static_cast<uint32_t>(r * 32 + lane) < rem) stage.put(whist[warp][rd[r] >> 16] + (rd[r] & 0xFFFFu), key[r], v);
    }
    __syncthreads();
    const uint32_t tile_n = static_cast<uint32_t>(min(static_cast<uint64_t>(SortShape<KT>::kTile), n - tile0));
    for (uint32_t j = threadIdx.x; j < tile_n; j += kSortThreads) {
        KT k;
        uint32_t v;
        stage.get(j, k, v);
        const uint32_t digit = static_cast<uint32_t>(k >> shift) & 0xFFu;
        const uint32_t pos = static_cast<uint32_t>(delta[digit] + static_cast<int32_t>(j));
        keys_out[pos] = k;
        vals_out[pos] = v;
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

template <typename KT>
inline uint32_t radix_tiles(uint64_t n) {
    return static_cast<uint32_t>((n + SortShape<KT>::kTile - 1) / SortShape<KT>::kTile);
}

// Count-table entries radix_sort_pairs needs for n keys of either key width.
inline size_t radix_counts_elems(uint64_t n) { return static_cast<size_t>(radix_tiles<uint64_t>(n)) * kSortBins; }

struct NoSortHook {
    void operator()(bool /*after_scatter*/) const {}
};

// Sorts keys_in (values implicitly 0..n-1) by bits [0, key_bits), stably.  Ping-pongs
// between (keys_a, vals_a) and (keys_b, vals_b); keys_in is only read.  Returns true
// when the result is in the *_b buffers.  counts: radix_counts_elems(n) u32;
// scan_buf: scan_scratch_bytes(counts) bytes.  hook(false) runs before each pass's
// scatter launch and hook(true) after it (stage timing).
template <typename KT, typename Hook = NoSortHook>
bool radix_sort_pairs(const KT* keys_in, KT* keys_a, uint32_t* vals_a, KT* keys_b, uint32_t* vals_b, uint64_t n,
                      int key_bits, uint32_t* counts, uint32_t* scan_buf, cudaStream_t stream,
                      const Hook& hook = Hook()) {
    const uint32_t tiles = radix_tiles<KT>(n);
    int passes = (key_bits + 7) / 8;
    if (passes == 0) passes = 1;  // one pass produces the identity permutation
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        const KT* kin = p == 0 ? keys_in : (p % 2 == 1 ? keys_a : keys_b);
        const uint32_t* vin = p == 0 ? nullptr : (p % 2 == 1 ? vals_a : vals_b);
        KT* kout = p % 2 == 0 ? keys_a : keys_b;
        uint32_t* vout = p % 2 == 0 ? vals_a : vals_b;
        radix_hist_kernel<KT><<<tiles, kSortThreads, 0, stream>>>(kin, n, shift, counts, tiles); count_launch();
        const uint64_t ncounts = static_cast<uint64_t>(tiles) * kSortBins;
        device_exclusive_scan<uint32_t>(CountIn{counts}, CountOut{counts}, ncounts, scan_buf,
                                        static_cast<uint32_t*>(nullptr), stream);
        hook(false);
        radix_scatter_kernel<KT><<<tiles, kSortThreads, 0, stream>>>(kin, vin, kout, vout, n, shift, counts, tiles); count_launch();
        hook(true);
    }
    return passes % 2 == 0;
}

// ------------------------------------------------------------- small sorts
// Up to kSmallSort (key, index) pairs sorted by one CTA: a bitonic sort in shared
// memory (keys padded with the largest value).  Not stable: used where keys are unique
// or where the order of equal keys does not matter.
constexpr uint32_t kSmallSort = 2048;
template <typename KT>
__global__ void __launch_bounds__(1024) small_sort_kernel(const KT* __restrict__ keys_in, KT* __restrict__ keys_out,
                                                          uint32_t* __restrict__ vals_out, uint32_t n) {
    __shared__ KT sk[kSmallSort];
    __shared__ uint32_t sv[kSmallSort];
    uint32_t n2 = 1;
    while (n2 < n) n2 <<= 1;
    for (uint32_t i = threadIdx.x; i < n2; i += blockDim.x) {
        sk[i] = i < n ? keys_in[i] : static_cast<KT>(~static_cast<KT>(0));
        sv[i] = i;
    }
    __syncthreads();
    for (uint32_t k = 2; k <= n2; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < n2; i += blockDim.x) {
                const uint32_t ixj = i ^ j;
                if (ixj > i) {
                    const bool up = (i & k) == 0;
                    const KT a = sk[i], b = sk[ixj];
                    if ((a > b) == up) {
                        sk[i] = b;
                        sk[ixj] = a;
                        const uint32_t t = sv[i];
                        sv[i] = sv[ixj];
                        sv[ixj] = t;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        keys_out[i] = sk[i];
        vals_out[i] = sv[i];
    }
}

// radix_sort_pairs for any n, except that up to kSmallSort keys are sorted by one CTA
// (not stable; the result is then in the *_a buffers).
template <typename KT>
bool sort_pairs(const KT* keys_in, KT* keys_a, uint32_t* vals_a, KT* keys_b, uint32_t* vals_b, uint64_t n,
                int key_bits, uint32_t* counts, uint32_t* scan_buf, cudaStream_t stream) {
    if (n <= kSmallSort) {
        small_sort_kernel<KT><<<1, 1024, 0, stream>>>(keys_in, keys_a, vals_a, static_cast<uint32_t>(n)); count_launch();
        return false;
    }
    return radix_sort_pairs<KT>(keys_in, keys_a, vals_a, keys_b, vals_b, n, key_bits, counts, scan_buf, stream);
}

}  // namespace chain
