// Stable LSD radix sort of (key, index) pairs over only the key bits in use.
//
// Used by the encoder to group points by block key: after sorting the Z-order block
// keys stably, the points of one block are adjacent and in increasing index order, so
// "the next point of the same block" is the sorted neighbour (lcps_cpp.cpp:2116-2138
// computes the same relation with a hash map).
//
// The key bits are split into ceil(key_bits / 8) passes of equal digit width (at most 8
// bits: a 21-bit key takes three 7-bit passes).  Each pass is three launches: a per-tile
// digit histogram (for the first pass the caller may have produced it already, as the
// quantizer does), a per-digit scan of that digit's row of tile counts (one CTA per
// digit; the rows' totals are scanned by each scatter CTA itself), and a stable scatter.
// The scatter loads its whole tile at once (indices wait in shared memory in input
// order), ranks keys with one ballot per digit bit per 32 keys (each warp owns a
// contiguous slice, processed 32 keys per round in order, so equal digits keep their
// input order), reorders the tile by digit in shared memory, and writes each digit's run
// to its global position with consecutive threads on consecutive addresses.
#pragma once

#include "chain_common.cuh"
#include "scan.cuh"

namespace chain {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortBins = 256;      // bins of the widest (8-bit) digit
constexpr int kSortMaxBits = 8;

template <typename KT>
struct SortShape {
    static constexpr int kItems = sizeof(KT) == 4 ? 12 : (sizeof(KT) == 8 ? 8 : 4);   // 16-byte keys: 4
    static constexpr int kTile = kSortThreads * kItems;
};

// Passes and digit width for a key of key_bits bits: as few passes of at most 8 bits
// as cover it, all of the same width (at least one pass: it yields the identity).  Keys
// stored in 8 or 16 bytes (key_sz) always take 8-bit digits.
struct RadixPlan {
    int passes;
    int bits;
};
inline RadixPlan radix_plan(int key_bits, int key_sz = 4) {
    RadixPlan r;
    r.passes = key_bits <= 0 ? 1 : (key_bits + kSortMaxBits - 1) / kSortMaxBits;
    r.bits = key_bits <= 0 ? 1 : (key_bits + r.passes - 1) / r.passes;
    if (key_sz > 4) r.bits = kSortMaxBits;
    return r;
}

// Per-tile histogram of digit (key >> shift) & (2^bits - 1) into counts[d * tiles + t].
template <typename KT>
__global__ void __launch_bounds__(kSortThreads)
radix_hist_kernel(const KT* __restrict__ keys, uint64_t n, int shift, int bits, uint32_t* __restrict__ counts,
                  uint32_t num_tiles) {
    constexpr int I = SortShape<KT>::kItems, TILE = SortShape<KT>::kTile;
    __shared__ uint32_t hist[kSortBins];
    const uint32_t bins = 1u << bits, mask = bins - 1;
    hist[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * TILE;
    const uint32_t rem = base >= n ? 0u : static_cast<uint32_t>(min(n - base, static_cast<uint64_t>(TILE)));
    // all loads first (one round trip per thread), then the shared-memory counts
    KT k[I];
#pragma unroll
    for (int r = 0; r < I; ++r) {
        const uint32_t i = r * kSortThreads + threadIdx.x;
        k[r] = i < rem ? ldg_key(keys + base + i) : KT(0);
    }
#pragma unroll
    for (int r = 0; r < I; ++r)
        if (static_cast<uint32_t>(r * kSortThreads + threadIdx.x) < rem)
            atomicAdd(&hist[static_cast<uint32_t>(k[r] >> shift) & mask], 1u);
    __syncthreads();
    if (threadIdx.x < bins) counts[static_cast<uint64_t>(threadIdx.x) * num_tiles + blockIdx.x] = hist[threadIdx.x];
}

// One CTA of kRowscanThreads per digit: exclusive scan, in place, of the digit's row of
// tile counts (counts[d * tiles .. d * tiles + tiles)); the row's total goes to
// row_total[d].  A round covers 8192 tiles (about 25M four-byte keys).
constexpr int kRowscanThreads = 1024;
__global__ void __launch_bounds__(kRowscanThreads)
radix_rowscan_kernel(uint32_t* __restrict__ counts, uint32_t num_tiles, uint32_t* __restrict__ row_total) {
    constexpr int kPer = 8;   // consecutive tiles per thread per round
    __shared__ uint32_t scratch[33];
    uint32_t* row = counts + static_cast<uint64_t>(blockIdx.x) * num_tiles;
    uint32_t carry = 0;
    for (uint32_t base = 0; base < num_tiles; base += kRowscanThreads * kPer) {
        const uint32_t t0 = base + threadIdx.x * kPer;
        uint32_t v[kPer];
        uint32_t sum = 0;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            v[k] = t0 + k < num_tiles ? row[t0 + k] : 0u;
            sum += v[k];
        }
        uint32_t tot;
        uint32_t ex = carry + block_exclusive_sum(sum, scratch, &tot);
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            if (t0 + k < num_tiles) row[t0 + k] = ex;
            ex += v[k];
        }
        carry += tot;
    }
    if (threadIdx.x == 0) row_total[blockIdx.x] = carry;
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
// offsets: the tile's row-exclusive prefix per digit (counts[d * tiles + t] after
// radix_rowscan_kernel); row_total: each digit's count over all tiles.
template <typename KT, int BITS>
__global__ void __launch_bounds__(kSortThreads, 4)
radix_scatter_kernel(const KT* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                     KT* __restrict__ keys_out, uint32_t* __restrict__ vals_out, uint64_t n, int shift,
                     const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ row_total,
                     uint32_t num_tiles) {
    constexpr int I = SortShape<KT>::kItems;
    constexpr int bits = BITS;
    __shared__ uint32_t whist[kSortWarps][kSortBins];
    __shared__ int32_t delta[kSortBins];         // global position - tile-local position, per digit
    __shared__ uint64_t scratch[33];
    __shared__ ScatterStage<KT> stage;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t bins = 1u << bits, mask = bins - 1;
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
        const uint32_t digit = static_cast<uint32_t>(key[r] >> shift) & mask;
        uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
        for (int b = 0; b < BITS; ++b) {
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
        // per digit: tile count, then per-warp offsets inside the tile; one scan gives
        // both the digit's start inside the tile (low word: the tile's counts) and its
        // start in the output (high word: the digits' totals over all tiles)
        const int d = threadIdx.x;
        uint32_t cnt = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) cnt += whist[w][d];
        const uint64_t total = static_cast<uint32_t>(d) < bins ? __ldg(row_total + d) : 0u;
        const uint64_t ex = block_exclusive_sum((total << 32) | cnt, scratch, static_cast<uint64_t*>(nullptr));
        const uint32_t start = static_cast<uint32_t>(ex);
        const uint32_t digit_base = static_cast<uint32_t>(ex >> 32);
        if (static_cast<uint32_t>(d) < bins)
            delta[d] = static_cast<int32_t>(digit_base + offsets[static_cast<uint64_t>(d) * num_tiles + blockIdx.x] -
                                            start);
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
        const uint32_t digit = static_cast<uint32_t>(k >> shift) & mask;
        const uint32_t pos = static_cast<uint32_t>(delta[digit] + static_cast<int32_t>(j));
        keys_out[pos] = k;
        vals_out[pos] = v;
    }
}

template <typename KT>
inline uint32_t radix_tiles(uint64_t n) {
    return static_cast<uint32_t>((n + SortShape<KT>::kTile - 1) / SortShape<KT>::kTile);
}

// Count-table entries radix_sort_pairs needs for n keys of any key width (the digit
// rows, then the rows' totals; 16-byte keys have the smallest tiles).
inline size_t radix_counts_elems(uint64_t n) {
    return static_cast<size_t>(radix_tiles<u128>(n)) * kSortBins + kSortBins;
}

// The scatter for a run-time digit width (instantiated per width, so that the ranking
// loop is fully unrolled).
template <typename KT>
inline void launch_radix_scatter(int bits, uint32_t tiles, cudaStream_t stream, const KT* kin, const uint32_t* vin,
                                 KT* kout, uint32_t* vout, uint64_t n, int shift, const uint32_t* counts,
                                 const uint32_t* row_total) {
#define CHAIN_SCATTER(B)                                                                                          \
    radix_scatter_kernel<KT, B><<<tiles, kSortThreads, 0, stream>>>(kin, vin, kout, vout, n, shift, counts, row_total, \
                                                                    tiles)
    if constexpr (sizeof(KT) > 4) {   // always 8-bit digits (radix_plan)
        CHAIN_SCATTER(8);
    } else {
        switch (bits) {
            case 1: CHAIN_SCATTER(1); break;
            case 2: CHAIN_SCATTER(2); break;
            case 3: CHAIN_SCATTER(3); break;
            case 4: CHAIN_SCATTER(4); break;
            case 5: CHAIN_SCATTER(5); break;
            case 6: CHAIN_SCATTER(6); break;
            case 7: CHAIN_SCATTER(7); break;
            default: CHAIN_SCATTER(8); break;
        }
    }
#undef CHAIN_SCATTER
    count_launch();
}

struct NoSortHook {
    void operator()(bool /*after_scatter*/) const {}
};

// Sorts keys_in (values implicitly 0..n-1) by bits [0, key_bits), stably.  Ping-pongs
// between (keys_a, vals_a) and (keys_b, vals_b); keys_in is only read.  Returns true
// when the result is in the *_b buffers.  counts: radix_counts_elems(n) u32.  When
// first_counts_ready, counts already holds the first pass's per-tile histogram (digit
// rows of radix_tiles<KT>(n) tiles, digit width radix_plan(key_bits).bits).  hook(false)
// runs before each pass's scatter launch and hook(true) after it (stage timing).
template <typename KT, typename Hook = NoSortHook>
bool radix_sort_pairs(const KT* keys_in, KT* keys_a, uint32_t* vals_a, KT* keys_b, uint32_t* vals_b, uint64_t n,
                      int key_bits, uint32_t* counts, cudaStream_t stream, const Hook& hook = Hook(),
                      bool first_counts_ready = false) {
    const uint32_t tiles = radix_tiles<KT>(n);
    const RadixPlan plan = radix_plan(key_bits, sizeof(KT));
    uint32_t* row_total = counts + static_cast<size_t>(tiles) * kSortBins;
    for (int p = 0; p < plan.passes; ++p) {
        const int shift = plan.bits * p;
        const KT* kin = p == 0 ? keys_in : (p % 2 == 1 ? keys_a : keys_b);
        const uint32_t* vin = p == 0 ? nullptr : (p % 2 == 1 ? vals_a : vals_b);
        KT* kout = p % 2 == 0 ? keys_a : keys_b;
        uint32_t* vout = p % 2 == 0 ? vals_a : vals_b;
        if (p > 0 || !first_counts_ready) {
            radix_hist_kernel<KT><<<tiles, kSortThreads, 0, stream>>>(kin, n, shift, plan.bits, counts, tiles); count_launch();
        }
        radix_rowscan_kernel<<<1u << plan.bits, kRowscanThreads, 0, stream>>>(counts, tiles, row_total); count_launch();
        hook(false);
        launch_radix_scatter<KT>(plan.bits, tiles, stream, kin, vin, kout, vout, n, shift, counts, row_total);
        hook(true);
    }
    return plan.passes % 2 == 0;
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
                int key_bits, uint32_t* counts, cudaStream_t stream) {
    if (n <= kSmallSort) {
        small_sort_kernel<KT><<<1, 1024, 0, stream>>>(keys_in, keys_a, vals_a, static_cast<uint32_t>(n)); count_launch();
        return false;
    }
    return radix_sort_pairs<KT>(keys_in, keys_a, vals_a, keys_b, vals_b, n, key_bits, counts, stream);
}

}  // namespace chain
