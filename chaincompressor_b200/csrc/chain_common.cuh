// Shared device/host definitions of the B200 Chain compressor.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstddef>

#if defined(__FAST_MATH__) || defined(__CUDA_FAST_MATH__)
#error "Chain FP64 quantization requires compilation without fast-math"
#endif

namespace chain {

constexpr int kMaxDims = 16;          // D limit of this build (the reference accepts any D)
constexpr int kStreams = 5;           // idrel, diff, keep, choice2, rel
constexpr uint32_t kRansMaxAlphabet = 1u << 18;  // lcps_cpp.cpp:539
constexpr int kRansMaxPrec = 20;
constexpr int kRansMinPrec = 12;
constexpr int kWarp = 32;

// Device error bits (OR-ed into a flag word; the host maps them to chain_status).
enum ErrBits : uint32_t {
    kErrNonFinite = 1u << 0,
    kErrQuantOverflow = 1u << 1,
    kErrCorrupt = 1u << 2,
    kErrInternal = 1u << 3,
    kErrCapacity = 1u << 4,
    kErrUnsupported = 1u << 5,
};

// Component encodings of the container (see chain_format.h).
enum Encoding : uint8_t { kEncEmpty = 0, kEncTagged = 1, kEncFixed = 2, kEncRaw = 3 };

// Host-side count of kernel launches issued by the library (tracing aid: every launch
// site calls count_launch()).
void count_launch();          // process-wide, thread-safe
uint64_t launch_count_total();
// Host-side count of the library's own memory allocations (every cudaMalloc and
// cudaMallocHost it issues; allocation sites call count_alloc()).
void count_alloc();           // process-wide, thread-safe
uint64_t alloc_count_total();

__host__ __device__ inline int bitlen32(uint32_t v) {
#ifdef __CUDA_ARCH__
    return 32 - __clz(v);
#else
    int b = 0;
    while (v) { ++b; v >>= 1; }
    return b;
#endif
}

__host__ __device__ inline int bitlen64(uint64_t v) {
#ifdef __CUDA_ARCH__
    return 64 - __clzll(static_cast<long long>(v));
#else
    int b = 0;
    while (v) { ++b; v >>= 1; }
    return b;
#endif
}

// Order-preserving map of an IEEE double onto uint64 (-0.0 sorts below +0.0).
__host__ __device__ inline uint64_t ordered_bits(double x) {
    uint64_t u;
    memcpy(&u, &x, 8);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__host__ __device__ inline double from_ordered_bits(uint64_t o) {
    uint64_t u = (o >> 63) ? (o & 0x7FFFFFFFFFFFFFFFull) : ~o;
    double x;
    memcpy(&x, &u, 8);
    return x;
}

__device__ inline void set_error(uint32_t* err, uint32_t bits) { atomicOr(err, bits); }

// Element i of an integer stream stored with esz bytes per value (1, 2 or 4).
__device__ __forceinline__ uint32_t load_elem(const void* p, uint64_t i, uint32_t esz) {
    if (esz == 1) return static_cast<const uint8_t*>(p)[i];
    if (esz == 2) return static_cast<const uint16_t*>(p)[i];
    return static_cast<const uint32_t*>(p)[i];
}

__device__ inline uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <typename T>
__device__ inline T warp_inclusive_sum(T v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

template <typename T>
__device__ inline T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T>
__device__ inline T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T t = __shfl_xor_sync(0xffffffffu, v, o);
        v = t > v ? t : v;
    }
    return v;
}

template <typename T>
__device__ inline T warp_min(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T t = __shfl_xor_sync(0xffffffffu, v, o);
        v = t < v ? t : v;
    }
    return v;
}

// Block-wide exclusive sum for blockDim.x <= 1024; `scratch` holds >= 33 values.
template <typename T>
__device__ inline T block_exclusive_sum(T v, T* scratch, T* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
    T inc = warp_inclusive_sum(v);
    if (lane == 31) scratch[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = lane < nwarps ? scratch[lane] : T(0);
        T wi = warp_inclusive_sum(w);
        if (lane < nwarps) scratch[lane] = wi - w;
        if (lane == nwarps - 1) scratch[32] = wi;
    }
    __syncthreads();
    T out = scratch[warp] + inc - v;
    if (total) *total = scratch[32];
    __syncthreads();
    return out;
}

template <typename T>
__device__ inline T block_reduce_sum(T v, T* scratch) {
    T tot;
    block_exclusive_sum(v, scratch, &tot);
    return tot;
}

// 3-D Morton spreading of 21 bits (bits i -> 3i).
__host__ __device__ inline uint64_t spread3(uint64_t n) {
    n &= 0x1FFFFFull;
    n = (n | (n << 32)) & 0x1F00000000FFFFull;
    n = (n | (n << 16)) & 0x1F0000FF0000FFull;
    n = (n | (n << 8)) & 0x100F00F00F00F00Full;
    n = (n | (n << 4)) & 0x10C30C30C30C30C3ull;
    n = (n | (n << 2)) & 0x1249249249249249ull;
    return n;
}
__host__ __device__ inline uint32_t compact3(uint64_t n) {
    n &= 0x1249249249249249ull;
    n = (n ^ (n >> 2)) & 0x10C30C30C30C30C3ull;
    n = (n ^ (n >> 4)) & 0x100F00F00F00F00Full;
    n = (n ^ (n >> 8)) & 0x1F0000FF0000FFull;
    n = (n ^ (n >> 16)) & 0x1F00000000FFFFull;
    n = (n ^ (n >> 32)) & 0x1FFFFFull;
    return static_cast<uint32_t>(n);
}
// 2-D Morton spreading of 32 bits (bit i -> 2i).
__host__ __device__ inline uint64_t spread2(uint64_t n) {
    n &= 0xFFFFFFFFull;
    n = (n | (n << 16)) & 0x0000FFFF0000FFFFull;
    n = (n | (n << 8)) & 0x00FF00FF00FF00FFull;
    n = (n | (n << 4)) & 0x0F0F0F0F0F0F0F0Full;
    n = (n | (n << 2)) & 0x3333333333333333ull;
    n = (n | (n << 1)) & 0x5555555555555555ull;
    return n;
}
__host__ __device__ inline uint32_t compact2(uint64_t n) {
    n &= 0x5555555555555555ull;
    n = (n ^ (n >> 1)) & 0x3333333333333333ull;
    n = (n ^ (n >> 2)) & 0x0F0F0F0F0F0F0F0Full;
    n = (n ^ (n >> 4)) & 0x00FF00FF00FF00FFull;
    n = (n ^ (n >> 8)) & 0x0000FFFF0000FFFFull;
    n = (n ^ (n >> 16)) & 0x00000000FFFFFFFFull;
    return static_cast<uint32_t>(n);
}

// Block key of a point: Z-order interleave of its D block coordinates, each kb bits
// wide (D*kb <= 64).  Injective on block tuples, so equal keys <=> same block.
__host__ __device__ inline uint64_t block_key(const uint32_t* b, int dims, int kb) {
    if (dims == 3 && kb <= 21) return spread3(b[0]) | (spread3(b[1]) << 1) | (spread3(b[2]) << 2);
    if (dims == 2) return spread2(b[0]) | (spread2(b[1]) << 1);
    if (dims == 1) return b[0];
    uint64_t k = 0;
    for (int bit = kb - 1; bit >= 0; --bit)
        for (int d = dims - 1; d >= 0; --d) k = (k << 1) | ((b[d] >> bit) & 1u);
    return k;
}
__host__ __device__ inline void block_unkey(uint64_t k, int dims, int kb, uint32_t* b) {
    if (dims == 3 && kb <= 21) {
        b[0] = compact3(k); b[1] = compact3(k >> 1); b[2] = compact3(k >> 2);
        return;
    }
    if (dims == 2) { b[0] = compact2(k); b[1] = compact2(k >> 1); return; }
    if (dims == 1) { b[0] = static_cast<uint32_t>(k); return; }
    for (int d = 0; d < dims; ++d) b[d] = 0;
    int pos = 0;
    for (int bit = 0; bit < kb; ++bit)
        for (int d = 0; d < dims; ++d, ++pos) b[d] |= static_cast<uint32_t>((k >> pos) & 1u) << bit;
}

// Block keys of more than 64 bits (D * kb <= 128: for instance three dimensions of 22 to
// 31 block-coordinate bits).  The same interleave: key bit (bit * D + d) = bit `bit` of
// coordinate d.
using u128 = unsigned __int128;
__host__ __device__ inline int bitlen128(u128 v) {
    const uint64_t hi = static_cast<uint64_t>(v >> 64);
    return hi ? 64 + bitlen64(hi) : bitlen64(static_cast<uint64_t>(v));
}
__host__ __device__ inline u128 block_key128(const uint32_t* b, int dims, int kb) {
    u128 k = 0;
    for (int bit = kb - 1; bit >= 0; --bit)
        for (int d = dims - 1; d >= 0; --d) k = (k << 1) | ((b[d] >> bit) & 1u);
    return k;
}
__host__ __device__ inline void block_unkey128(u128 k, int dims, int kb, uint32_t* b) {
    for (int d = 0; d < dims; ++d) b[d] = 0;
    int pos = 0;
    for (int bit = 0; bit < kb; ++bit)
        for (int d = 0; d < dims; ++d, ++pos) b[d] |= static_cast<uint32_t>((k >> pos) & 1u) << bit;
}

// Key of block coordinates b and its inverse, for a key type of 32, 64 or 128 bits.
// Three dimensions in a 4- or 8-byte key (kb <= 21) take the plain concatenation of
// the coordinates, b0 | b1 << kb | b2 << 2 kb, instead of the interleave: the encoder
// only needs equal keys <=> equal blocks (no order of blocks), and the fields come back
// with shifts.
template <typename KT>
__host__ __device__ inline KT make_block_key(const uint32_t* b, int dims, int kb) {
    if constexpr (sizeof(KT) == 16) {
        return block_key128(b, dims, kb);
    } else {
        if (dims == 3)
            return static_cast<KT>(b[0]) | (static_cast<KT>(b[1]) << kb) | (static_cast<KT>(b[2]) << (2 * kb));
        return static_cast<KT>(block_key(b, dims, kb));
    }
}
template <typename KT>
__host__ __device__ inline void block_coords(KT k, int dims, int kb, uint32_t* b) {
    if constexpr (sizeof(KT) == 16) {
        block_unkey128(k, dims, kb, b);
    } else {
        if (dims == 3) {
            const KT mask = (static_cast<KT>(1) << kb) - 1;
            b[0] = static_cast<uint32_t>(k & mask);
            b[1] = static_cast<uint32_t>((k >> kb) & mask);
            b[2] = static_cast<uint32_t>(k >> (2 * kb));
            return;
        }
        block_unkey(static_cast<uint64_t>(k), dims, kb, b);
    }
}
template <typename KT>
__host__ __device__ inline int key_bitlen(KT k) {
    if constexpr (sizeof(KT) == 16) return bitlen128(k);
    else return bitlen64(static_cast<uint64_t>(k));
}

// Read-only load of a key (the 128-bit type has no __ldg overload).
template <typename KT>
__device__ __forceinline__ KT ldg_key(const KT* p) {
    if constexpr (sizeof(KT) == 16) {
        const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(p));
        return (static_cast<u128>(v.y) << 64) | v.x;
    } else {
        return __ldg(p);
    }
}

}  // namespace chain
