// Device-wide exclusive scan (reduce-then-scan) over a functor-produced sequence with
// an associative operator.
//
//   in(i)  -> T              value of element i (0 <= i < n), evaluated once
//   out(i, prefix, value)    called once per element with its exclusive prefix
//   Op: T operator()(T a, T b) (a precedes b), static T identity()
//
// Three launches: per-tile reduction, a one-CTA scan of the tile aggregates, and the
// per-tile scan seeded with the tile's prefix.  A tile is 256 threads x kItems<T>
// elements; elements are loaded in a coalesced (striped) order into shared memory,
// each thread scans a contiguous run, and out() is called from that run.
#pragma once

#include <type_traits>
#include <utility>

#include "chain_common.cuh"

namespace chain {

constexpr int kScanThreads = 256;

template <typename T>
struct ScanShape {
    static constexpr int kItems = sizeof(T) > 8 ? 8 : 16;
    static constexpr int kTile = kScanThreads * kItems;
};

template <typename T>
struct SumOp {
    __device__ __forceinline__ T operator()(T a, T b) const { return a + b; }
    __device__ __forceinline__ static T identity() { return T(0); }
};

// Warp shuffle of any trivially copyable type made of 32-bit words.
template <typename T>
__device__ __forceinline__ T shfl_up_any(T v, int o) {
    static_assert(sizeof(T) % 4 == 0, "scan types must be made of 32-bit words");
    union U {
        T t;
        uint32_t w[sizeof(T) / 4];
        __device__ U() {}
    } u;
    u.t = v;
#pragma unroll
    for (int k = 0; k < static_cast<int>(sizeof(T) / 4); ++k) u.w[k] = __shfl_up_sync(0xffffffffu, u.w[k], o);
    return u.t;
}

template <typename T>
__device__ __forceinline__ T shfl_idx_any(T v, int src) {
    static_assert(sizeof(T) % 4 == 0, "shuffled types must be made of 32-bit words");
    union U {
        T t;
        uint32_t w[sizeof(T) / 4];
        __device__ U() {}
    } u;
    u.t = v;
#pragma unroll
    for (int k = 0; k < static_cast<int>(sizeof(T) / 4); ++k) u.w[k] = __shfl_sync(0xffffffffu, u.w[k], src);
    return u.t;
}

template <typename T, typename Op>
__device__ __forceinline__ T warp_inclusive_scan_op(T v, Op op) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = shfl_up_any(v, o);
        if (lane >= o) v = op(t, v);
    }
    return v;
}

// Exclusive scan across the CTA; *total (may be null) receives the CTA aggregate.
template <typename T, typename Op>
__device__ __forceinline__ T block_exclusive_scan_op(T v, Op op, T* scratch, T* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
    T inc = warp_inclusive_scan_op(v, op);
    T exc = shfl_up_any(inc, 1);
    if (lane == 0) exc = Op::identity();
    if (lane == 31) scratch[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = lane < nwarps ? scratch[lane] : Op::identity();
        T wi = warp_inclusive_scan_op(w, op);
        T we = shfl_up_any(wi, 1);
        if (lane == 0) we = Op::identity();
        if (lane < nwarps) scratch[lane] = we;
        if (lane == nwarps - 1) scratch[32] = wi;
    }
    __syncthreads();
    T out = op(scratch[warp], exc);
    if (total) *total = scratch[32];
    __syncthreads();
    return out;
}

// Padded shared-memory index: one spare slot every 32 elements keeps the per-thread
// contiguous reads free of bank conflicts.
__device__ __forceinline__ int scan_pad(int j) { return j + (j >> 5); }

template <typename T, typename InF>
__device__ __forceinline__ void scan_stage(InF in, uint64_t n, uint64_t base, T* vals) {
    constexpr int I = ScanShape<T>::kItems;
#pragma unroll
    for (int k = 0; k < I; ++k) {
        const int j = k * kScanThreads + threadIdx.x;
        const uint64_t i = base + j;
        if (i < n) vals[scan_pad(j)] = in(i);
    }
}

template <typename T, typename InF, typename Op>
__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(InF in, uint64_t n, T* tile_aggr, Op op) {
    constexpr int I = ScanShape<T>::kItems, TILE = ScanShape<T>::kTile;
    __shared__ T vals[TILE + TILE / 32];
    __shared__ T scratch[33];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * TILE;
    scan_stage<T>(in, n, base, vals);
    __syncthreads();
    T acc = Op::identity();
#pragma unroll
    for (int k = 0; k < I; ++k) {
        const int j = threadIdx.x * I + k;
        if (base + j < n) acc = op(acc, vals[scan_pad(j)]);
    }
    T tot;
    block_exclusive_scan_op(acc, op, scratch, &tot);
    if (threadIdx.x == 0) tile_aggr[blockIdx.x] = tot;
}

// In-place exclusive scan of `count` tile aggregates by one CTA of 1024 threads; the
// grand total goes to *total (may be null).
template <typename T, typename Op>
__global__ void __launch_bounds__(1024) scan_tilesums_kernel(T* aggr, uint64_t count, T* total, Op op) {
    __shared__ T scratch[33];
    T carry = Op::identity();
    for (uint64_t base = 0; base < count; base += 1024) {
        const uint64_t i = base + threadIdx.x;
        T v = i < count ? aggr[i] : Op::identity();
        T tot;
        T ex = block_exclusive_scan_op(v, op, scratch, &tot);
        if (i < count) aggr[i] = op(carry, ex);
        carry = op(carry, tot);
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

// Scan-then-output kernel.  With Striped = true, out() is called in the coalesced
// (striped) element order, from prefixes and values staged in shared memory; use it
// when out() writes element-indexed arrays.  Striped needs two tiles of shared memory,
// so it is used for 4-byte element types.
template <typename T, typename InF, typename OutF, typename Op, bool Striped>
__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(InF in, OutF out, uint64_t n,
                                                                  const T* tile_prefix, Op op) {
    constexpr int I = ScanShape<T>::kItems, TILE = ScanShape<T>::kTile;
    constexpr int PADDED = TILE + TILE / 32;
    __shared__ T vals[Striped ? 2 * PADDED : PADDED];
    __shared__ T scratch[33];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * TILE;
    const T tp = tile_prefix[blockIdx.x];   // loaded with the tile, not after the scan's barriers
    scan_stage<T>(in, n, base, vals);
    __syncthreads();
    T local[I];
    T agg = Op::identity();
#pragma unroll
    for (int k = 0; k < I; ++k) {
        const int j = threadIdx.x * I + k;
        local[k] = base + j < n ? vals[scan_pad(j)] : Op::identity();
        agg = op(agg, local[k]);
    }
    T ex = op(tp, block_exclusive_scan_op(agg, op, scratch, static_cast<T*>(nullptr)));
    if constexpr (Striped) {
        T* pre = vals + PADDED;
#pragma unroll
        for (int k = 0; k < I; ++k) {
            pre[scan_pad(threadIdx.x * I + k)] = ex;
            ex = op(ex, local[k]);
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < I; ++k) {
            const int j = k * kScanThreads + threadIdx.x;
            const uint64_t i = base + j;
            if (i < n) out(i, pre[scan_pad(j)], vals[scan_pad(j)]);
        }
    } else {
#pragma unroll
        for (int k = 0; k < I; ++k) {
            const uint64_t i = base + threadIdx.x * I + k;
            if (i < n) out(i, ex, local[k]);
            ex = op(ex, local[k]);
        }
    }
}

template <typename T>
inline uint64_t scan_tiles(uint64_t n) {
    return (n + ScanShape<T>::kTile - 1) / ScanShape<T>::kTile;
}
// Bytes of tile-aggregate scratch that any scan over n elements of a type up to 16
// bytes needs.
inline uint64_t scan_scratch_bytes(uint64_t n) { return 16 * (n / 2048 + 16); }

// Scans of up to kScanSingleMax elements run as one CTA (one launch instead of three):
// thread t takes the 16 consecutive elements from 16 t, one block scan joins the runs.
constexpr uint64_t kScanSingleMax = 16384;
template <typename T, typename InF, typename OutF, typename Op>
__global__ void __launch_bounds__(1024) scan_single_kernel(InF in, OutF out, uint64_t n, T* total, Op op) {
    constexpr int kPer = static_cast<int>(kScanSingleMax / 1024);
    __shared__ T scratch[33];
    const uint64_t b = static_cast<uint64_t>(threadIdx.x) * kPer;
    T v[kPer];
    T agg = Op::identity();
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        v[k] = b + k < n ? in(b + k) : Op::identity();
        agg = op(agg, v[k]);
    }
    T tot;
    T ex = block_exclusive_scan_op(agg, op, scratch, &tot);
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        if (b + k < n) out(b + k, ex, v[k]);
        ex = op(ex, v[k]);
    }
    if (threadIdx.x == 0 && total) *total = tot;
}

// Launches the scan kernels on `stream`; `tile_buf` holds scan_tiles<T>(n) values.
// out() runs in striped (coalesced) element order for 4-byte element types (in thread
// runs for scans of up to kScanSingleMax elements).
template <typename T, typename InF, typename OutF, typename Op = SumOp<T>>
void device_exclusive_scan(InF in, OutF out, uint64_t n, T* tile_buf, T* total, cudaStream_t stream,
                           Op op = Op()) {
    constexpr bool kStriped = sizeof(T) <= 4;
    const uint64_t tiles = scan_tiles<T>(n);
    if (tiles == 0) {
        if (total) cudaMemsetAsync(total, 0, sizeof(T), stream);
        return;
    }
    if (n <= kScanSingleMax) {
        scan_single_kernel<T, InF, OutF, Op><<<1, 1024, 0, stream>>>(in, out, n, total, op); count_launch();
        return;
    }
    scan_reduce_kernel<T, InF, Op><<<static_cast<unsigned>(tiles), kScanThreads, 0, stream>>>(in, n, tile_buf, op); count_launch();
    scan_tilesums_kernel<T, Op><<<1, 1024, 0, stream>>>(tile_buf, tiles, total, op); count_launch();
    scan_apply_kernel<T, InF, OutF, Op, kStriped><<<static_cast<unsigned>(tiles), kScanThreads, 0, stream>>>(
        in, out, n, tile_buf, op); count_launch();
}

// ------------------------------------------------------------ flag scans
// Exclusive count of set flags: pred(i) -> bool for 0 <= i < n, and out(i, rank, flag)
// called once per element with rank = number of set flags before i.  A tile is
// kFlagThreads x kFlagItems elements; warp w of a tile handles 32 * kFlagItems
// consecutive elements in rounds of 32 (element = base + 32 k + lane), so ranks come
// from ballots and popcounts and every out() call is coalesced.  Three launches: tile
// counts, a one-CTA scan of the counts, and the ranked pass (pred is evaluated twice).
constexpr int kFlagThreads = 256;
constexpr int kFlagItems = 16;
constexpr int kFlagTile = kFlagThreads * kFlagItems;

// In-place exclusive scan of `count` u32 tile counts by one CTA (blockDim a multiple of
// 32, at most 1024), kPer consecutive counts per thread per round.  The counts are read
// with ld.global.cg: the other CTAs of the same launch wrote them.  *total (may be null)
// receives their sum.
__device__ inline void block_scan_counts(uint32_t* counts, uint64_t count, uint32_t* total) {
    constexpr int kPer = 8;
    __shared__ uint32_t scratch[33];
    uint32_t carry = 0;
    const uint64_t per_round = static_cast<uint64_t>(blockDim.x) * kPer;
    for (uint64_t base = 0; base < count; base += per_round) {
        const uint64_t i0 = base + static_cast<uint64_t>(threadIdx.x) * kPer;
        uint32_t v[kPer], sum = 0;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            v[k] = i0 + k < count ? __ldcg(counts + i0 + k) : 0u;
            sum += v[k];
        }
        uint32_t tot;
        uint32_t ex = carry + block_exclusive_sum(sum, scratch, &tot);
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            if (i0 + k < count) counts[i0 + k] = ex;
            ex += v[k];
        }
        carry += tot;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

// The CTA of a launch that finishes last (done: a counter that is zero at launch, and
// is zero again afterwards) turns the launch's tile counts into exclusive prefixes.
// Every CTA calls it after writing its count; it returns true in the CTA that scanned.
__device__ inline bool last_cta_scan_counts(uint32_t* counts, uint32_t* total, uint32_t* done) {
    __shared__ bool s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    block_scan_counts(counts, gridDim.x, total);
    if (threadIdx.x == 0) *done = 0;
    return true;
}

// done (may be null): see last_cta_scan_counts; the tile counts then leave as exclusive
// prefixes and *total receives their sum.
template <typename Pred>
__global__ void __launch_bounds__(kFlagThreads) flag_count_kernel(Pred pred, uint64_t n, uint32_t* tile_counts,
                                                                   uint32_t* total = nullptr, uint32_t* done = nullptr) {
    __shared__ uint32_t wsum[kFlagThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kFlagTile + static_cast<uint64_t>(warp) * 32 * kFlagItems;
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < kFlagItems; ++k) {
        const uint64_t i = base + 32 * k + lane;
        c += __popc(__ballot_sync(0xffffffffu, i < n && pred(i)));
    }
    if (lane == 0) wsum[warp] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kFlagThreads / 32; ++w) t += wsum[w];
        tile_counts[blockIdx.x] = t;
    }
    if (done) last_cta_scan_counts(tile_counts, total, done);
}

// flag_count_kernel for predicates that test a 4-byte word for zero (Pred::zero_words()
// returns the words): 16-byte loads and per-thread counts, no ballots (the counts need no
// element order within the tile).
static __global__ void __launch_bounds__(kFlagThreads) flag_count_zero_words_kernel(const uint32_t* __restrict__ w, uint64_t n,
                                                                             uint32_t* tile_counts, uint32_t* total,
                                                                             uint32_t* done) {
    static_assert(kFlagItems % 4 == 0, "whole 16-byte words per thread");
    __shared__ uint32_t wsum[kFlagThreads / 32];
    const uint64_t tile0 = static_cast<uint64_t>(blockIdx.x) * kFlagTile;
    uint32_t c = 0;
    if ((reinterpret_cast<uintptr_t>(w) & 15) == 0 && tile0 + kFlagTile <= n) {
        const uint4* v = reinterpret_cast<const uint4*>(w + tile0);
#pragma unroll
        for (int k = 0; k < kFlagItems / 4; ++k) {
            const uint4 q = __ldg(v + k * kFlagThreads + threadIdx.x);
            c += (q.x == 0u) + (q.y == 0u) + (q.z == 0u) + (q.w == 0u);
        }
    } else {
        for (int k = 0; k < kFlagItems; ++k) {
            const uint64_t i = tile0 + static_cast<uint64_t>(k) * kFlagThreads + threadIdx.x;
            c += (i < n && w[i] == 0u) ? 1u : 0u;
        }
    }
    c = warp_sum(c);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int k = 0; k < kFlagThreads / 32; ++k) t += wsum[k];
        tile_counts[blockIdx.x] = t;
    }
    if (done) last_cta_scan_counts(tile_counts, total, done);
}

template <typename P, typename = void>
struct HasZeroWords : std::false_type {};
template <typename P>
struct HasZeroWords<P, std::void_t<decltype(std::declval<const P&>().zero_words())>> : std::true_type {};

// The counting launch of a flag scan (flag_count_kernel, or its zero-word form).
template <typename Pred>
void launch_flag_count(Pred pred, uint64_t n, uint64_t tiles, uint32_t* tile_buf, uint32_t* total, uint32_t* done,
                       cudaStream_t stream) {
    if constexpr (HasZeroWords<Pred>::value)
        flag_count_zero_words_kernel<<<static_cast<unsigned>(tiles), kFlagThreads, 0, stream>>>(pred.zero_words(), n,
                                                                                                tile_buf, total, done);
    else
        flag_count_kernel<Pred><<<static_cast<unsigned>(tiles), kFlagThreads, 0, stream>>>(pred, n, tile_buf, total,
                                                                                          done);
    count_launch();
}

// kOutUnroll: rounds of out() calls unrolled together (more loads in flight against
// more registers; the best depth depends on out()).
template <typename Pred, typename OutF, int kOutUnroll = 4>
__global__ void __launch_bounds__(kFlagThreads) flag_apply_kernel(Pred pred, OutF out, uint64_t n,
                                                                   const uint32_t* tile_prefix) {
    __shared__ uint32_t wsum[kFlagThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kFlagTile + static_cast<uint64_t>(warp) * 32 * kFlagItems;
    const uint32_t tp = tile_prefix[blockIdx.x];   // in flight with the flags
    uint32_t m[kFlagItems];
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < kFlagItems; ++k) {
        const uint64_t i = base + 32 * k + lane;
        m[k] = __ballot_sync(0xffffffffu, i < n && pred(i));
        c += __popc(m[k]);
    }
    if (lane == 0) wsum[warp] = c;
    __syncthreads();
    uint32_t run = tp;
    for (int w = 0; w < warp; ++w) run += wsum[w];
    const uint32_t lt = lanemask_lt();
#pragma unroll kOutUnroll
    for (int k = 0; k < kFlagItems; ++k) {
        const uint64_t i = base + 32 * k + lane;
        if (i < n) out(i, run + __popc(m[k] & lt), (m[k] >> lane) & 1u);
        run += __popc(m[k]);
    }
}

// The ranked pass of a compaction, dst[rank] = src[i] for every flagged i: each thread
// loads its items' flags and (for values of at most eight bytes) source values before
// the ballots, so a warp waits on memory once per tile instead of once per round of
// stores.  Values are read for unflagged items too (the sectors are mostly shared).
template <typename Pred, typename T>
__global__ void __launch_bounds__(kFlagThreads) flag_gather_kernel(Pred pred, const T* __restrict__ src,
                                                                    T* __restrict__ dst, uint64_t n,
                                                                    const uint32_t* tile_prefix) {
    __shared__ uint32_t wsum[kFlagThreads / 32];
    constexpr bool kPre = sizeof(T) <= 8;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kFlagTile + static_cast<uint64_t>(warp) * 32 * kFlagItems;
    uint32_t m[kFlagItems];
    T v[kPre ? kFlagItems : 1];
#pragma unroll
    for (int k = 0; k < kFlagItems; ++k) {
        const uint64_t i = base + 32 * k + lane;
        m[k] = i < n ? pred(i) : 0u;
        if (kPre) v[k] = i < n ? src[i] : T(0);
    }
    const uint32_t tp = tile_prefix[blockIdx.x];
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < kFlagItems; ++k) {
        m[k] = __ballot_sync(0xffffffffu, m[k] != 0);
        c += __popc(m[k]);
    }
    if (lane == 0) wsum[warp] = c;
    __syncthreads();
    uint32_t run = tp;
    for (int w = 0; w < warp; ++w) run += wsum[w];
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < kFlagItems; ++k) {
        if ((m[k] >> lane) & 1u) {
            const uint64_t i = base + 32 * k + lane;
            dst[run + __popc(m[k] & lt)] = kPre ? v[k] : src[i];
        }
        run += __popc(m[k]);
    }
}

inline uint64_t flag_tiles(uint64_t n) { return (n + kFlagTile - 1) / kFlagTile; }

// `tile_buf` holds flag_tiles(n) u32 (scan_scratch_bytes(n) bytes suffice); *total
// (may be null) receives the number of set flags.  With `done` (a device counter that is
// zero, see last_cta_scan_counts) the counting launch also scans the tile counts: two
// launches instead of three.
template <typename Pred, typename OutF, int kOutUnroll = 4>
void device_flag_scan(Pred pred, OutF out, uint64_t n, uint32_t* tile_buf, uint32_t* total, cudaStream_t stream,
                      uint32_t* done = nullptr) {
    const uint64_t tiles = flag_tiles(n);
    if (tiles == 0) {
        if (total) cudaMemsetAsync(total, 0, sizeof(uint32_t), stream);
        return;
    }
    launch_flag_count(pred, n, tiles, tile_buf, total, done, stream);
    if (!done) {
        scan_tilesums_kernel<uint32_t, SumOp<uint32_t>><<<1, 1024, 0, stream>>>(tile_buf, tiles, total, SumOp<uint32_t>());
        count_launch();
    }
    flag_apply_kernel<Pred, OutF, kOutUnroll><<<static_cast<unsigned>(tiles), kFlagThreads, 0, stream>>>(pred, out, n,
                                                                                                    tile_buf); count_launch();
}

// device_flag_scan for a compaction (dst[rank] = src[i] for flagged i): the counting
// launch scans the tile counts (`done` as there), then flag_gather_kernel.
template <typename Pred, typename T>
void device_flag_gather(Pred pred, const T* src, T* dst, uint64_t n, uint32_t* tile_buf, uint32_t* total,
                        uint32_t* done, cudaStream_t stream) {
    const uint64_t tiles = flag_tiles(n);
    if (tiles == 0) {
        if (total) cudaMemsetAsync(total, 0, sizeof(uint32_t), stream);
        return;
    }
    launch_flag_count(pred, n, tiles, tile_buf, total, done, stream);
    flag_gather_kernel<Pred, T><<<static_cast<unsigned>(tiles), kFlagThreads, 0, stream>>>(pred, src, dst, n, tile_buf);
    count_launch();
}

// The same scan when the per-tile counts are already in `tile_buf` (a producer kernel
// that runs one CTA per kFlagTile elements wrote them).
template <typename Pred, typename OutF, int kOutUnroll = 4>
void device_flag_scan_counted(Pred pred, OutF out, uint64_t n, uint32_t* tile_buf, uint32_t* total,
                              cudaStream_t stream) {
    const uint64_t tiles = flag_tiles(n);
    if (tiles == 0) {
        if (total) cudaMemsetAsync(total, 0, sizeof(uint32_t), stream);
        return;
    }
    scan_tilesums_kernel<uint32_t, SumOp<uint32_t>><<<1, 1024, 0, stream>>>(tile_buf, tiles, total, SumOp<uint32_t>()); count_launch();
    flag_apply_kernel<Pred, OutF, kOutUnroll><<<static_cast<unsigned>(tiles), kFlagThreads, 0, stream>>>(pred, out, n,
                                                                                                    tile_buf); count_launch();
}

}  // namespace chain
