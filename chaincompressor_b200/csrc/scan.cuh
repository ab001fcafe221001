// Device-wide exclusive scan (reduce-then-scan) over a functor-produced sequence with
// an associative operator.
//
//   in(i)  -> T              value of element i (0 <= i < n)
//   out(i, prefix, value)    called once per element with its exclusive prefix
//   Op: T operator()(T a, T b) (a precedes b), static T identity()
//
// Three launches: per-tile reduction, a one-CTA scan of the tile aggregates, and the
// per-tile scan seeded with the tile's prefix.  Tiles are 4096 elements, read and
// written in a coalesced (striped) order and scanned through shared memory.
#pragma once

#include "chain_common.cuh"

namespace chain {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

template <typename T>
struct SumOp {
    __device__ __forceinline__ T operator()(T a, T b) const { return a + b; }
    __device__ __forceinline__ static T identity() { return T(0); }
};

template <typename T, typename Op>
__device__ __forceinline__ T warp_inclusive_scan_op(T v, Op op) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v = op(t, v);
    }
    return v;
}

// Exclusive scan across the CTA; *total receives the CTA aggregate.
template <typename T, typename Op>
__device__ __forceinline__ T block_exclusive_scan_op(T v, Op op, T* scratch, T* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
    T inc = warp_inclusive_scan_op(v, op);
    T exc = __shfl_up_sync(0xffffffffu, inc, 1);
    if (lane == 0) exc = Op::identity();
    if (lane == 31) scratch[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = lane < nwarps ? scratch[lane] : Op::identity();
        T wi = warp_inclusive_scan_op(w, op);
        T we = __shfl_up_sync(0xffffffffu, wi, 1);
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

template <typename T, typename InF, typename Op>
__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(InF in, uint64_t n, T* tile_aggr, Op op) {
    __shared__ T scratch[33];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kScanTile + static_cast<uint64_t>(threadIdx.x) * kScanItems;
    // each thread reduces a contiguous run (order matters for non-commutative ops)
    T acc = Op::identity();
#pragma unroll 4
    for (int k = 0; k < kScanItems; ++k) {
        const uint64_t i = base + k;
        if (i < n) acc = op(acc, in(i));
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

template <typename T, typename InF, typename OutF, typename Op>
__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(InF in, OutF out, uint64_t n,
                                                                  const T* tile_prefix, Op op) {
    __shared__ T vals[kScanTile + kScanTile / 32];
    __shared__ T scratch[33];
    // padded index: one extra slot every 32 elements avoids bank conflicts on the
    // per-thread contiguous reads below
#define CHAIN_SCAN_PAD(j) ((j) + ((j) >> 5))
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kScanTile;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int j = k * kScanThreads + threadIdx.x;
        const uint64_t i = base + j;
        vals[CHAIN_SCAN_PAD(j)] = i < n ? in(i) : Op::identity();
    }
    __syncthreads();
    T local[kScanItems];
    T agg = Op::identity();
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        local[k] = vals[CHAIN_SCAN_PAD(threadIdx.x * kScanItems + k)];
        agg = op(agg, local[k]);
    }
    T ex = op(tile_prefix[blockIdx.x], block_exclusive_scan_op(agg, op, scratch, static_cast<T*>(nullptr)));
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        vals[CHAIN_SCAN_PAD(threadIdx.x * kScanItems + k)] = ex;
        ex = op(ex, local[k]);
    }
    __syncthreads();
    // out() also receives the element's own value, re-read through the input functor.
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int j = k * kScanThreads + threadIdx.x;
        const uint64_t i = base + j;
        if (i < n) out(i, vals[CHAIN_SCAN_PAD(j)], in(i));
    }
#undef CHAIN_SCAN_PAD
}

inline uint64_t scan_tiles(uint64_t n) { return (n + kScanTile - 1) / kScanTile; }

// Launches the three scan kernels on `stream`; `tile_buf` holds scan_tiles(n) values.
template <typename T, typename InF, typename OutF, typename Op = SumOp<T>>
void device_exclusive_scan(InF in, OutF out, uint64_t n, T* tile_buf, T* total, cudaStream_t stream,
                           Op op = Op()) {
    const uint64_t tiles = scan_tiles(n);
    if (tiles == 0) {
        if (total) cudaMemsetAsync(total, 0, sizeof(T), stream);
        return;
    }
    scan_reduce_kernel<T, InF, Op><<<static_cast<unsigned>(tiles), kScanThreads, 0, stream>>>(in, n, tile_buf, op);
    scan_tilesums_kernel<T, Op><<<1, 1024, 0, stream>>>(tile_buf, tiles, total, op);
    scan_apply_kernel<T, InF, OutF, Op><<<static_cast<unsigned>(tiles), kScanThreads, 0, stream>>>(in, out, n,
                                                                                               tile_buf, op);
}

}  // namespace chain
