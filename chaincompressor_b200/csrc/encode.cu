// Chain encoder on sm_100a: FP64 quantization, Z-order block keys + stable radix sort,
// level-1 chaining, level-2 block differencing, candidate selection and the
// interleaved-rANS / bit-packing entropy stage, assembled into an LCG2 v2 container.
//
// Integer semantics follow the reference CPU encoder bit for bit:
//   quantization + exact corrections   cpp/chain/lcps_cpp.cpp:2069-2110 (:1496-1523)
//   next point in the same block       lcps_cpp.cpp:2116-2138
//   level-1 choice                     lcps_cpp.cpp:2155-2200
//   level-2 keep/difference split      lcps_cpp.cpp:1305-1454 (:1221-1262, :1456-1478)
//   candidate codings                  lcps_cpp.cpp:1140-1174 (fixed :856-933,
//                                      tagged :1005-1058, raw value rANS :935-995)
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <type_traits>
#include <vector>

#include "chain_common.cuh"
#include "chain_format.h"
#include "ctx.h"
#include "radix_sort.cuh"
#include "rans.cuh"
#include "scan.cuh"

namespace chain {

// ------------------------------------------------------------------------ state
struct StreamStats {
    uint32_t minv[kMaxDims];
    uint32_t maxv[kMaxDims];
    uint32_t maxall;
    uint32_t maxtag;
    uint64_t tag_bits;        // sum over records of dims * tag
    uint32_t tag_hist[34];    // tag_hist[t], t in 1..32
};

struct StreamChoice {
    uint8_t enc;
    uint8_t max_width;
    uint8_t width[kMaxDims];
    uint32_t dims;
    uint64_t records;
    uint64_t est[4];          // estimated body bytes by encoding (index = Encoding)
    uint32_t sec_prec, sec_alphabet, sec_chunks, table_len, sec_lanes, pad_lanes;
    uint64_t sec_S, sec_count;
    uint64_t payload_bytes;   // sum of the chunk bytes (after coding)
    uint64_t packed_bits;
    uint64_t body_bytes;      // exact, after coding
};

struct EncState {
    uint32_t err;
    uint32_t dims;
    uint64_t n;
    double eb;
    uint64_t p;
    int64_t threshold;
    uint64_t minbits[kMaxDims], maxbits[kMaxDims];
    uint64_t zero_first[kMaxDims][2];   // first index of -0.0 / +0.0
    double mins[kMaxDims];
    uint32_t qmax[kMaxDims];
    uint32_t bmax_all;
    int32_t kb;
    int32_t key_bits;
    int32_t maxb_bits;
    uint64_t ncorr;
    uint32_t B, nkeep, ndiff, pad0;
    uint32_t rec_min, rec_max, rec_maxdiff, pad1;
    int64_t wrap_min, wrap_max, wrap_range, wrap_min_corr, wrap_max_corr;
    StreamStats st[kCodeStreams];
    RansTableDev raw_tab[kCodeStreams];
    RansTableDev tag_tab[kCodeStreams];
    StreamChoice ch[kCodeStreams];
    uint32_t ndistinct;   // distinct exact-correction values
    // level-1 links (idrel != 0), accumulated by k_level1 for IDR0's statistics
    unsigned long long l1_links, l1_link_bits;
    uint32_t l1_link_min, l1_link_max;
    uint32_t done_a;          // CTAs finished (last-CTA hand-offs; zero between them)
    uint64_t total_bytes;
    uint32_t npieces;
    uint32_t done_b;          // second hand-off counter
    uint32_t done_c;          // hand-off counter of the side stream's IDR0 tables
    uint64_t nsegs;
};

// A byte range copied into the container.  Pieces are cut into kCopySeg-byte
// segments so that large payloads spread over many CTAs.  A chunked piece (stream >= 0)
// is the whole payload of one rANS section: its segments never cross a chunk, and a
// segment finds its chunk through the stream's per-chunk segment prefix.
struct Piece {
    const uint8_t* src;
    uint64_t dst;
    uint64_t len;
    uint64_t seg_begin;   // index of this piece's first segment
    int32_t stream;       // -1: plain byte range; else the coded stream whose chunks these are
    int32_t pad;
};
constexpr uint64_t kCopySeg = 4096;

// Per rANS section: where each chunk's bytes sit in its encoder slot and in the
// section payload, and how many copy segments precede it.
struct ChunkMap {
    const uint8_t* slots;
    uint64_t slot_cap;
    const uint32_t* len;   // [chunks]
    uint64_t* off;         // [chunks] byte offset in the payload
    uint32_t* seg;         // [chunks + 1] copy segments before the chunk
    uint32_t chunks;
    uint32_t pad;
};
struct ChunkMaps {
    ChunkMap m[kCodeStreams];
    int sec_stream[kCodeStreams];   // coded streams that have a rANS section
    int nsec;
};

// --------------------------------------------------------------- quantization
template <typename FT, bool SOA>
__device__ __forceinline__ double load_coord(const FT* p, uint64_t n, uint32_t D, uint64_t i, uint32_t d) {
    return static_cast<double>(SOA ? p[static_cast<uint64_t>(d) * n + i] : p[i * D + d]);
}

__device__ void qparams(EncState* st);

// Per-axis extrema (as ordered bits of the double value), the first index of -0.0 and
// of +0.0, and a non-finite flag.  blockIdx.y is the axis.  Values are compared in their
// own type (float -> double is exact and order-preserving; the sign of a zero minimum
// is settled by the first-zero indices).  A contiguous axis (SoA) is read with 16-byte
// loads, two per thread in flight.
template <typename FT, bool SOA>
__global__ void __launch_bounds__(256) k_minmax(const FT* __restrict__ p, uint64_t n, uint32_t D, EncState* st) {
    const uint32_t d = blockIdx.y;
    FT mn = static_cast<FT>(INFINITY), mx = static_cast<FT>(-INFINITY);
    uint64_t zneg = ~0ull, zpos = ~0ull;
    bool bad = false;
    auto visit = [&](FT x, uint64_t i) {
        bad = bad || !chain_isfinite(static_cast<double>(x));
        mn = x < mn ? x : mn;
        mx = x > mx ? x : mx;
        if (x == static_cast<FT>(0)) {
            if (signbit(x)) zneg = i < zneg ? i : zneg;
            else zpos = i < zpos ? i : zpos;
        }
    };
    const uint64_t tid = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    constexpr int V = 16 / sizeof(FT);
    const FT* q = SOA ? p + static_cast<uint64_t>(d) * n : p;
    if (SOA && (reinterpret_cast<uintptr_t>(q) & 15) == 0) {
        using Vec = typename std::conditional<sizeof(FT) == 4, float4, double2>::type;
        const Vec* qv = reinterpret_cast<const Vec*>(q);
        const uint64_t nv = n / V;
        for (uint64_t g = tid; g < nv; g += 2 * nthreads) {
            FT a[V], b[V];
            const bool two = g + nthreads < nv;
            *reinterpret_cast<Vec*>(a) = __ldg(qv + g);
            if (two) *reinterpret_cast<Vec*>(b) = __ldg(qv + g + nthreads);
#pragma unroll
            for (int k = 0; k < V; ++k) visit(a[k], g * V + k);
            if (two) {
#pragma unroll
                for (int k = 0; k < V; ++k) visit(b[k], (g + nthreads) * V + k);
            }
        }
        for (uint64_t i = nv * V + tid; i < n; i += nthreads) visit(q[i], i);
    } else {
        for (uint64_t i = tid; i < n; i += nthreads) visit(SOA ? q[i] : p[i * D + d], i);
    }
    uint64_t omn = ordered_bits(static_cast<double>(mn)), omx = ordered_bits(static_cast<double>(mx));
    omn = warp_min(omn); omx = warp_max(omx); zneg = warp_min(zneg); zpos = warp_min(zpos);
    __shared__ uint64_t s[4][8];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { s[0][w] = omn; s[1][w] = omx; s[2][w] = zneg; s[3][w] = zpos; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < static_cast<int>(blockDim.x >> 5); ++k) {
            omn = s[0][k] < omn ? s[0][k] : omn; omx = s[1][k] > omx ? s[1][k] : omx;
            zneg = s[2][k] < zneg ? s[2][k] : zneg; zpos = s[3][k] < zpos ? s[3][k] : zpos;
        }
        atomicMin(reinterpret_cast<unsigned long long*>(&st->minbits[d]), omn);
        atomicMax(reinterpret_cast<unsigned long long*>(&st->maxbits[d]), omx);
        if (zneg != ~0ull) atomicMin(reinterpret_cast<unsigned long long*>(&st->zero_first[d][0]), zneg);
        if (zpos != ~0ull) atomicMin(reinterpret_cast<unsigned long long*>(&st->zero_first[d][1]), zpos);
    }
    const bool any_bad = __syncthreads_or(bad);
    if (threadIdx.x == 0) {
        if (any_bad) set_error(&st->err, kErrNonFinite);
        // the CTA that finishes last derives the quantization parameters from the
        // completed extrema (no separate launch)
        __threadfence();
        if (atomicAdd(&st->done_a, 1u) == gridDim.x * gridDim.y - 1) {
            __threadfence();
            qparams(st);
            st->done_a = 0;
        }
    }
}

// Per-axis minimum exactly as std::min keeps it (first of equal values, which only
// matters for +0.0 vs -0.0), the largest quantized value and the block-key width.
__device__ void qparams(EncState* st) {
    if (__ldcg(&st->err) & kErrNonFinite) return;
    const double denom = 2.0 * st->eb;
    uint32_t bmax = 0;
    int kb = 0;
    for (uint32_t d = 0; d < st->dims; ++d) {
        // the extrema were combined by other CTAs' atomics: read them from L2
        double mn = from_ordered_bits(__ldcg(&st->minbits[d]));
        if (mn == 0.0) mn = __ldcg(&st->zero_first[d][0]) < __ldcg(&st->zero_first[d][1]) ? -0.0 : 0.0;
        st->mins[d] = mn;
        const double mx = from_ordered_bits(__ldcg(&st->maxbits[d]));
        const double qv = floor((mx - mn) / denom);
        if (!(qv >= 0.0 && qv < 0x1p63)) { set_error(&st->err, kErrQuantOverflow); return; }
        if (qv >= 4294967296.0) { set_error(&st->err, kErrUnsupported); return; }   // 32-bit q
        st->qmax[d] = static_cast<uint32_t>(qv);
        const uint32_t b = static_cast<uint32_t>(static_cast<uint64_t>(st->qmax[d]) / st->p);
        bmax = b > bmax ? b : bmax;
        kb = bitlen32(b) > kb ? bitlen32(b) : kb;
    }
    st->bmax_all = bmax;
    st->kb = kb;
    st->key_bits = kb * static_cast<int>(st->dims);
    st->maxb_bits = bitlen32(bmax);
    if (st->key_bits > 128) set_error(&st->err, kErrUnsupported);
}

// lcps_cpp.cpp:1502-1523
__device__ __forceinline__ bool within_error_bound(double restored, double original, double eb) {
    if (!chain_isfinite(restored)) return false;
    const double difference = __dsub_rn(restored, original);
    const double magnitude = fabs(difference);
    if (magnitude < eb) return true;
    if (!(magnitude == eb)) return false;
    const double virtual_original = __dsub_rn(difference, restored);
    const double remainder = __dadd_rn(__dsub_rn(restored, __dsub_rn(difference, virtual_original)),
                                       __dsub_rn(-original, virtual_original));
    return difference >= 0.0 ? remainder <= 0.0 : remainder >= 0.0;
}

// Block index b = q / p and rel = q - b*p for q < 2^32: a shift and a mask when p is a
// power of two, else a double-precision reciprocal estimate corrected to the exact
// quotient (the estimate is off by at most one).
struct BlockDiv {
    uint64_t p;
    double inv;
    int shift;   // >= 0: p == 2^shift
    __device__ __forceinline__ uint32_t div(uint32_t q) const {
        if (shift >= 0) return shift >= 32 ? 0u : q >> shift;
        if (p > 0xffffffffull) return 0u;
        uint32_t b = static_cast<uint32_t>(static_cast<double>(q) * inv);
        const uint64_t t = static_cast<uint64_t>(b) * p;
        if (t > q) --b;
        else if (t + p <= q) ++b;
        return b;
    }
};

// Quantization of every point (lcps_cpp.cpp:2060-2110): q = floor((x - min) / (2 eb)) in
// IEEE double, the reconstruction fma(q + 0.5, 2 eb, min) checked against eb (values
// outside go to the exact-correction list), the block index and the offset inside the
// block, and the point's Z-order block key.  DIM is the dimension count (0 = run time).
// One CTA per sort tile (SortShape<KT>::kTile consecutive points), so that the CTA can
// also count its tile's first radix digits (key & (2^hist_bits - 1)) into the sort's
// count table (digit-major, `tiles` columns) when hist_counts is set: the first sort
// pass then needs no histogram launch.  The offsets go out as RT (one byte each when
// p <= 256).  Three-dimensional SoA input is processed four points per thread with
// 16-byte loads (the rest of the points, and every other shape, one point per thread).
struct QuantCtx {
    const double* mins;
    double eb, denom, two_eb;
    double inv_denom;   // RN(1 / denom)
    BlockDiv bd;
    EncState* st;
    uint64_t* corr_idx;
    double* corr_val;
    uint64_t corr_cap;
    // Quantizes coordinate x (flat index fi = i*D + d); returns the block index and
    // stores the offset inside the block in rel.
    //
    // floor(RN(a / denom)) without a division for almost every coordinate: t = RN(a *
    // RN(1 / denom)) differs from a / denom by at most 2u|t| and RN(a / denom) by at most
    // 3u|t| (u = 2^-53, to first order), so when t lies farther than m = 2^-49 t from the
    // nearest integer, both have the same floor.  Closer (or not finite) coordinates
    // take the IEEE division.  t - floor(t) is exact (Sterbenz), as is m.
    __device__ __forceinline__ double quotient_floor(double a) const {
        const double t = __dmul_rn(a, inv_denom);
        const double ft = floor(t);
        const double f = __dsub_rn(t, ft), m = __dmul_rn(t, 0x1p-49);
        if (f > m && __dsub_rn(1.0, f) > m) return ft;
        return floor(__ddiv_rn(a, denom));
    }
    __device__ __forceinline__ uint32_t coord(double x, uint32_t d, uint64_t fi, uint32_t& rel) const {
        const double qv = quotient_floor(__dsub_rn(x, mins[d]));
        const uint32_t q = static_cast<uint32_t>(qv);
        const double restored = fma(__dadd_rn(static_cast<double>(q), 0.5), two_eb, mins[d]);
        if (!within_error_bound(restored, x, eb)) {
            const unsigned long long slot = atomicAdd(reinterpret_cast<unsigned long long*>(&st->ncorr), 1ull);
            if (slot < corr_cap) {
                corr_idx[slot] = fi;
                corr_val[slot] = x;
            }
        }
        const uint32_t bb = bd.div(q);
        rel = static_cast<uint32_t>(q - static_cast<uint64_t>(bb) * bd.p);
        return bb;
    }
};

template <typename FT, bool SOA, typename KT, int DIM, typename RT>
__global__ void __launch_bounds__(256)
k_quantize(const FT* __restrict__ p, uint64_t n, uint32_t D_rt, EncState* st, KT* __restrict__ key_out,
           RT* __restrict__ rel_out, uint64_t* __restrict__ corr_idx, double* __restrict__ corr_val,
           uint64_t corr_cap, uint32_t* __restrict__ hist_counts, int hist_bits, uint32_t tiles,
           uint32_t* __restrict__ idrel_zero) {
    static_assert(SortShape<KT>::kTile % 1024 == 0, "tiles hold whole groups of four points per thread");
    constexpr uint64_t TILE = SortShape<KT>::kTile;
    __shared__ double s_min[kMaxDims];
    __shared__ double s_eb;
    __shared__ uint64_t s_p;
    __shared__ int s_kb;
    __shared__ uint32_t s_hist[kSortBins];
    const uint32_t D = DIM ? DIM : D_rt;
    if (threadIdx.x < D) s_min[threadIdx.x] = st->mins[threadIdx.x];
    if (threadIdx.x == 0) { s_eb = st->eb; s_p = st->p; s_kb = st->kb; }
    s_hist[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t hmask = (1u << hist_bits) - 1;
    const bool hist = hist_counts != nullptr;
    QuantCtx Q;
    Q.mins = s_min;
    Q.eb = s_eb;
    Q.denom = 2.0 * s_eb;
    Q.inv_denom = 1.0 / Q.denom;
    Q.two_eb = 2.0 * s_eb;
    Q.bd.p = s_p;
    Q.bd.inv = 1.0 / static_cast<double>(s_p);
    Q.bd.shift = (s_p & (s_p - 1)) == 0 ? bitlen64(s_p) - 1 : -1;
    Q.st = st;
    Q.corr_idx = corr_idx;
    Q.corr_val = corr_val;
    Q.corr_cap = corr_cap;
    const int kb = s_kb;
    const uint64_t tile_begin = static_cast<uint64_t>(blockIdx.x) * TILE;
    const uint64_t tile_end = min(n, tile_begin + TILE);
    uint64_t first_scalar = tile_begin;
    if constexpr (SOA && DIM == 3) {
        const bool vec = ((reinterpret_cast<uintptr_t>(p) | (n * sizeof(FT))) & 15) == 0 &&
                         (reinterpret_cast<uintptr_t>(rel_out) & 15) == 0 &&
                         (reinterpret_cast<uintptr_t>(key_out) & 15) == 0;
        if (vec) {
            const uint64_t ng = tile_end / 4;   // whole groups of four points below tile_end
            for (uint64_t g = tile_begin / 4 + threadIdx.x; g < ng; g += blockDim.x) {
                FT x[3][4];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const FT* src = p + static_cast<uint64_t>(d) * n + 4 * g;
                    if constexpr (sizeof(FT) == 4) {
                        *reinterpret_cast<float4*>(x[d]) = __ldg(reinterpret_cast<const float4*>(src));
                    } else {
                        *reinterpret_cast<double2*>(x[d]) = __ldg(reinterpret_cast<const double2*>(src));
                        *reinterpret_cast<double2*>(x[d] + 2) = __ldg(reinterpret_cast<const double2*>(src) + 1);
                    }
                }
                uint32_t rel[12];
                KT keys[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    uint32_t b[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        b[d] = Q.coord(static_cast<double>(x[d][k]), d, (4 * g + k) * 3 + d, rel[3 * k + d]);
                    keys[k] = make_block_key<KT>(b, 3, kb);
                    if (hist) atomicAdd(&s_hist[static_cast<uint32_t>(keys[k]) & hmask], 1u);
                }
                if constexpr (sizeof(RT) == 4) {
                    uint4* ro = reinterpret_cast<uint4*>(rel_out + 12 * g);
                    ro[0] = make_uint4(rel[0], rel[1], rel[2], rel[3]);
                    ro[1] = make_uint4(rel[4], rel[5], rel[6], rel[7]);
                    ro[2] = make_uint4(rel[8], rel[9], rel[10], rel[11]);
                } else {   // twelve bytes as three little-endian words
                    uint32_t* ro = reinterpret_cast<uint32_t*>(rel_out + 12 * g);
#pragma unroll
                    for (int w = 0; w < 3; ++w)
                        ro[w] = rel[4 * w] | (rel[4 * w + 1] << 8) | (rel[4 * w + 2] << 16) | (rel[4 * w + 3] << 24);
                }
                // idrel starts at zero (level 1 writes only the links)
                reinterpret_cast<uint4*>(idrel_zero)[g] = make_uint4(0, 0, 0, 0);
                if constexpr (sizeof(KT) == 4) {
                    *reinterpret_cast<uint4*>(key_out + 4 * g) = make_uint4(keys[0], keys[1], keys[2], keys[3]);
                } else if constexpr (sizeof(KT) == 16) {
#pragma unroll
                    for (int k = 0; k < 4; ++k) key_out[4 * g + k] = keys[k];
                } else {
                    ulonglong2* ko = reinterpret_cast<ulonglong2*>(key_out + 4 * g);
                    ko[0] = make_ulonglong2(keys[0], keys[1]);
                    ko[1] = make_ulonglong2(keys[2], keys[3]);
                }
            }
            first_scalar = max(ng * 4, tile_begin);
        }
    }
    constexpr int KD = DIM ? DIM : kMaxDims;
    for (uint64_t i = first_scalar + threadIdx.x; i < tile_end; i += blockDim.x) {
        uint32_t b[KD];
#pragma unroll
        for (int d = 0; d < KD; ++d) {
            if (!DIM && d >= static_cast<int>(D)) break;
            uint32_t r;
            b[d] = Q.coord(load_coord<FT, SOA>(p, n, D, i, d), d, i * D + d, r);
            rel_out[i * D + d] = static_cast<RT>(r);
        }
        const KT key = make_block_key<KT>(b, static_cast<int>(D), kb);
        key_out[i] = key;
        idrel_zero[i] = 0;
        if (hist) atomicAdd(&s_hist[static_cast<uint32_t>(key) & hmask], 1u);
    }
    if (hist) {
        __syncthreads();
        if (threadIdx.x <= hmask)
            hist_counts[static_cast<uint64_t>(threadIdx.x) * tiles + blockIdx.x] = s_hist[threadIdx.x];
    }
}

// Eight 16-bit counters packed into two 64-bit registers (bins 0..3 and 4..7), for the
// hot small values of a stream; flushed into shared memory at the end.
struct PackedCount8 {
    uint64_t lo = 0, hi = 0;
    __device__ __forceinline__ void add(uint32_t v) {   // v < 8
        const uint64_t inc = 1ull << ((v & 3u) << 4);
        if (v & 4u) hi += inc;
        else lo += inc;
    }
    // Warp-sums the counters and adds them to bins[0..7] (lane 0).
    __device__ __forceinline__ void flush(uint32_t* bins) {
        uint32_t c[8];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            c[k] = static_cast<uint32_t>(lo >> (16 * k)) & 0xffffu;
            c[4 + k] = static_cast<uint32_t>(hi >> (16 * k)) & 0xffffu;
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t t = warp_sum(c[k]);
            if ((threadIdx.x & 31) == 0 && t) atomicAdd(&bins[k], t);
        }
        lo = hi = 0;
    }
};

// ------------------------------------------------------------------- level 1
// Sorted position k: the sorted neighbour with an equal key is the next point of the
// same block (stable sort keeps indices increasing within a block).  Each thread takes
// groups of four consecutive positions, two groups at a time, and loads them (16-byte
// loads) and each group's fifth neighbour before using any.  `idrel` arrives zeroed
// and only links (idrel != 0, a minority of points) are scattered into it.  DIM: 3, or 0
// for a dimension count read at run time.
template <typename KT, int DIM>
__global__ void __launch_bounds__(256, sizeof(KT) == 4 ? 4 : 3)   // 64-bit keys spill at four CTAs per SM
k_level1(const KT* __restrict__ skey, const uint32_t* __restrict__ sidx, uint64_t n, EncState* st,
         uint32_t* __restrict__ idrel, uint32_t* __restrict__ gh) {
    // IDR0 statistics of the links (idrel_stats adds the zeros)
    constexpr uint32_t kSmallBins = 256;
    __shared__ uint32_t sh[kSmallBins], stag[34];
    __shared__ unsigned long long s_links, s_bits;
    __shared__ uint32_t s_min, s_max;
    for (uint32_t t = threadIdx.x; t < kSmallBins; t += blockDim.x) sh[t] = 0;
    if (threadIdx.x < 34) stag[threadIdx.x] = 0;
    if (threadIdx.x == 0) { s_links = 0; s_bits = 0; s_min = 0xffffffffu; s_max = 0; }
    __syncthreads();
    uint32_t links = 0, lmin = 0xffffffffu, lmax = 0;
    unsigned long long lbits = 0;
    // the common short links (distance < 8, tag < 8) count in registers, not in
    // contended shared-memory bins
    PackedCount8 vc, tc;
    const int D = DIM ? DIM : static_cast<int>(st->dims);
    const int kb3 = st->kb;   // field width of a concatenated 3-D key
    const int64_t maxb_bits = st->maxb_bits;
    const int64_t thr = st->threshold;
    const int64_t c = static_cast<int64_t>(D) * maxb_bits;
    const uint64_t ng = (n + 3) / 4;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    constexpr int kU = 2;   // groups per thread whose loads are in flight together
    for (uint64_t g0 = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g0 < ng; g0 += stride * kU) {
        KT keys[kU][5];
        uint32_t idxs[kU][5];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint64_t g = g0 + u * stride;
            if (4 * g + 4 <= n) {   // four positions by 16-byte loads (the arrays are 256-byte aligned)
                if constexpr (sizeof(KT) == 16) {
#pragma unroll
                    for (int j = 0; j < 4; ++j) keys[u][j] = ldg_key(skey + 4 * g + j);
                } else if constexpr (sizeof(KT) == 4) {
                    const uint4 kv = __ldg(reinterpret_cast<const uint4*>(skey) + g);
                    keys[u][0] = kv.x; keys[u][1] = kv.y; keys[u][2] = kv.z; keys[u][3] = kv.w;
                } else {
                    const ulonglong2 a = __ldg(reinterpret_cast<const ulonglong2*>(skey) + 2 * g);
                    const ulonglong2 b = __ldg(reinterpret_cast<const ulonglong2*>(skey) + 2 * g + 1);
                    keys[u][0] = a.x; keys[u][1] = a.y; keys[u][2] = b.x; keys[u][3] = b.y;
                }
                const uint4 iv = __ldg(reinterpret_cast<const uint4*>(sidx) + g);
                idxs[u][0] = iv.x; idxs[u][1] = iv.y; idxs[u][2] = iv.z; idxs[u][3] = iv.w;
                const uint64_t k = 4 * g + 4;
                keys[u][4] = k < n ? ldg_key(skey + k) : KT(0);
                idxs[u][4] = k < n ? __ldg(sidx + k) : 0u;
            } else {
#pragma unroll
                for (int j = 0; j < 5; ++j) {
                    const uint64_t k = 4 * g + j;
                    keys[u][j] = k < n ? skey[k] : KT(0);
                    idxs[u][j] = k < n ? sidx[k] : 0u;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint64_t g = g0 + u * stride;
            if (g >= ng) break;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint64_t k = 4 * g + j;
                uint32_t out = 0;
                if (k + 1 < n && keys[u][j + 1] == keys[u][j]) {
                    const uint32_t dist = idxs[u][j + 1] - idxs[u][j];
                    // bits of the block's widest coordinate: of the OR of the three fields
                    // of a concatenated 3-D key, else ceil(bitlen(key) / D) of an
                    // interleaved one (bit j of coordinate d sits at key bit j * D + d)
                    int local_bits;
                    if constexpr (DIM == 3 && sizeof(KT) <= 8) {
                        const KT kk = keys[u][j];
                        const KT m = (static_cast<KT>(1) << kb3) - 1;
                        local_bits = bitlen64(static_cast<uint64_t>((kk & m) | ((kk >> kb3) & m) | (kk >> (2 * kb3))));
                    } else {
                        local_bits = (key_bitlen(keys[u][j]) + D - 1) / D;
                    }
                    const int tag_bits = bitlen32(static_cast<uint32_t>(local_bits));
                    const int64_t a = static_cast<int64_t>(local_bits) * D + tag_bits;
                    const int64_t smaller = a < c ? a : c;
                    const int dl = bitlen32(dist);
                    if (static_cast<int64_t>(dl + bitlen32(static_cast<uint32_t>(dl))) < smaller - thr) out = dist;
                }
                if (k < n && out) {   // idrel was zeroed: only links are written
                    idrel[idxs[u][j]] = out;
                    ++links;
                    lmin = out < lmin ? out : lmin;
                    lmax = out > lmax ? out : lmax;
                    const uint32_t tag = bitlen32(out);   // >= 1
                    lbits += tag;
                    if (tag < 8) tc.add(tag);
                    else atomicAdd(&stag[tag], 1u);
                    if (out < 8) vc.add(out);
                    else if (out < kSmallBins) atomicAdd(&sh[out], 1u);
                    else if (out < kRansMaxAlphabet) atomicAdd(&gh[out], 1u);
                }
            }
        }
    }
    // 16-bit counters: a thread handles at most ceil(n / 4 / threads) groups of four
    // positions, far below 65536 links per thread for any launch of this kernel
    vc.flush(sh);
    tc.flush(stag);
    links = warp_sum(links);
    lbits = warp_sum(lbits);
    lmin = warp_min(lmin);
    lmax = warp_max(lmax);
    if ((threadIdx.x & 31) == 0) {
        if (links) {
            atomicAdd(&s_links, static_cast<unsigned long long>(links));
            atomicAdd(&s_bits, lbits);
            atomicMin(&s_min, lmin);
            atomicMax(&s_max, lmax);
        }
    }
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < kSmallBins; t += blockDim.x)
        if (sh[t]) atomicAdd(&gh[t], sh[t]);
    if (threadIdx.x < 34 && stag[threadIdx.x]) {
        atomicAdd(&st->st[0].tag_hist[threadIdx.x], stag[threadIdx.x]);
        atomicMax(&st->st[0].maxtag, threadIdx.x);
    }
    if (threadIdx.x == 0 && s_links) {
        atomicAdd(&st->l1_links, s_links);
        atomicAdd(&st->l1_link_bits, s_bits);
        atomicMin(&st->l1_link_min, s_min);
        atomicMax(&st->l1_link_max, s_max);
    }
}

// IDR0's statistics completed from the level-1 links: the n - links zeros (tag 1) join
// them.  The same values the counting kernel would accumulate from the stream.  part 0
// completes what the value table reads (extrema, value histogram), part 1 what the tag
// table reads (tag histogram, tag bits), so that the two table CTAs each finish their own.
__device__ void idrel_stats(EncState* st, uint32_t* gh, uint64_t n, int part) {
    if (n == 0) return;
    const unsigned long long links = st->l1_links, zeros = n - links;
    StreamStats& g = st->st[0];
    if (part == 0) {
        g.minv[0] = zeros ? 0u : st->l1_link_min;
        g.maxv[0] = links ? st->l1_link_max : 0u;
        g.maxall = g.maxv[0];
        if (zeros) gh[0] += static_cast<uint32_t>(zeros);
    } else {
        if (zeros) {
            g.tag_hist[1] += static_cast<uint32_t>(zeros);
            if (g.maxtag < 1) g.maxtag = 1;
        }
        g.tag_bits = st->l1_link_bits + zeros;
    }
}

// Explicit block records, in index order (lcps_cpp.cpp:2196-2199).
template <typename KT>
struct ExplicitIn {
    const uint32_t* idrel;
    __device__ uint32_t operator()(uint64_t i) const { return idrel[i] == 0 ? 1u : 0u; }
    __host__ __device__ const uint32_t* zero_words() const { return idrel; }
};
// An explicit record is kept as its point's block key (device_flag_gather copies the
// keys), which moves D times fewer bytes than separate coordinates through the level-2
// passes (rec_read takes the coordinates back out: three shifts for three dimensions in
// a 4- or 8-byte key).

// Level-2 work runs with DIM = 3 (three dimensions, kb <= 21) or DIM = 0 (any shape).
__device__ __forceinline__ bool l2_dim3(const EncState* st) { return st->dims == 3 && st->kb <= 21; }

// Block coordinates of an explicit record (a block key, make_block_key).
template <int DIM, typename KT>
__device__ __forceinline__ void rec_read(KT r, int D, int kb, uint32_t* b) {
    block_coords<KT>(r, DIM ? DIM : D, kb, b);
}

// ------------------------------------------------------------------- level 2
// Record minimum, maximum and largest per-dimension difference between consecutive
// records.  Each thread takes groups of four consecutive record keys (16-byte loads for
// 32-bit keys), kU groups in flight at once.
template <typename KT, int DIM>
__global__ void __launch_bounds__(256) k_l2_stats(const KT* __restrict__ rec, EncState* st) {
    const uint32_t B = st->B;
    const int D = DIM ? DIM : static_cast<int>(st->dims);
    const int kb = st->kb;
    if (DIM == 3 && !l2_dim3(st)) return;
    if (DIM == 0 && l2_dim3(st)) return;
    uint32_t mn = 0xffffffffu, mx = 0, md = 0;
    const uint64_t tid = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    constexpr int KD = DIM ? DIM : kMaxDims;
    constexpr int kU = 2;
    const uint64_t ng = (B + 3) / 4;
    for (uint64_t g0 = tid; g0 < ng; g0 += nthreads * kU) {
        KT k[kU][5];   // per group: the previous key, then four keys
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint64_t g = g0 + u * nthreads;
            const uint64_t j0 = 4 * g;
            if (g < ng && j0 + 4 <= B && sizeof(KT) == 4) {
                const uint4 v = __ldg(reinterpret_cast<const uint4*>(rec) + g);
                k[u][1] = static_cast<KT>(v.x); k[u][2] = static_cast<KT>(v.y);
                k[u][3] = static_cast<KT>(v.z); k[u][4] = static_cast<KT>(v.w);
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) k[u][1 + q] = g < ng && j0 + q < B ? ldg_key(rec + j0 + q) : KT(0);
            }
            k[u][0] = g < ng && j0 ? ldg_key(rec + j0 - 1) : KT(0);
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint64_t g = g0 + u * nthreads;
            if (g >= ng) continue;
            uint32_t prev[KD], cur[KD];
            rec_read<DIM>(k[u][0], D, kb, prev);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint64_t j = 4 * g + q;
                if (j >= B) break;
                rec_read<DIM>(k[u][1 + q], D, kb, cur);
#pragma unroll
                for (int d = 0; d < KD; ++d) {
                    if (!DIM && d >= D) break;
                    mn = cur[d] < mn ? cur[d] : mn;
                    mx = cur[d] > mx ? cur[d] : mx;
                    if (j) {
                        const uint32_t df = cur[d] >= prev[d] ? cur[d] - prev[d] : prev[d] - cur[d];
                        md = df > md ? df : md;
                    }
                    prev[d] = cur[d];
                }
            }
        }
    }
    // one update of each global value per CTA (the CTAs all update the same three words)
    __shared__ uint32_t s_mn, s_mx, s_md;
    if (threadIdx.x == 0) { s_mn = 0xffffffffu; s_mx = 0; s_md = 0; }
    __syncthreads();
    mn = warp_min(mn); mx = warp_max(mx); md = warp_max(md);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&s_mn, mn);
        atomicMax(&s_mx, mx);
        atomicMax(&s_md, md);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (s_mn != 0xffffffffu) atomicMin(&st->rec_min, s_mn);
        if (s_mx) atomicMax(&st->rec_max, s_mx);
        if (s_md) atomicMax(&st->rec_maxdiff, s_md);
    }
}

// lcps_cpp.cpp:1221-1253 wrap parameters; also the !l2 keep-all variant (:1456-1478).
__device__ void l2_params(EncState* st) {
    const int64_t mn = st->B ? st->rec_min : 0;
    const int64_t mx = st->rec_max;
    const int64_t range = mx - mn + 1;
    st->wrap_min = mn;
    st->wrap_max = mx;
    st->wrap_range = range;
    st->wrap_max_corr = range / 2 - ((range & 1) == 0 ? 1 : 0);
    st->wrap_min_corr = -(range / 2);
}

// The level-2 rule (lcps_cpp.cpp:1305-1454) for record j given its and its
// predecessor's coordinates: 1 = code it as the difference from the previous record.
__device__ __forceinline__ uint32_t l2_rule(const uint32_t* cur, const uint32_t* prev, int D, uint32_t fvb,
                                           uint32_t fdb) {
    uint32_t mv = 0, md = 0;
    for (int d = 0; d < D; ++d) {
        mv = cur[d] > mv ? cur[d] : mv;
        const uint32_t a = cur[d] >= prev[d] ? cur[d] - prev[d] : prev[d] - cur[d];
        md = a > md ? a : md;
    }
    const int tvw = bitlen32(mv), tdw = bitlen32(md);
    // at most 16 x 32 + 6 bits: 32-bit arithmetic is exact
    const uint32_t tvb = static_cast<uint32_t>(D) * tvw + bitlen32(static_cast<uint32_t>(tvw));
    const uint32_t tdb = static_cast<uint32_t>(D) * tdw + bitlen32(static_cast<uint32_t>(tdw));
    const uint32_t value_bits = tvb < fvb ? tvb : fvb;
    const uint32_t diff_bits = tdb > fdb ? tdb : fdb;
    return value_bits >= diff_bits ? 1u : 0u;
}

__device__ __forceinline__ uint64_t tile0_of_block() { return static_cast<uint64_t>(blockIdx.x) * kFlagTile; }

// choice2[j] for every record (1 = difference from the previous record), one CTA per
// flag-scan tile of kFlagTile records; each CTA also writes its tile's count of
// difference records and the last CTA scans them, so the level-2 flag scan needs no
// launch before its ranked pass.  Each thread
// takes four groups of four consecutive record keys, all loads first.
template <typename KT, int DIM>
__global__ void __launch_bounds__(256) k_l2_choice(const KT* __restrict__ rec, EncState* st, int l2,
                                                   uint8_t* choice2, uint32_t* tile_counts) {
    static_assert(kFlagTile == 4 * 4 * 256, "four groups of four records per thread");
    __shared__ uint32_t wsum[8];
    if (DIM == 3 && !l2_dim3(st)) return;
    if (DIM == 0 && l2_dim3(st)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) l2_params(st);   // read by the level-2 output and the layout
    const uint32_t B = st->B;
    if (tile0_of_block() >= B) {   // the grid covers n >= B entries: an empty tile counts 0
        if (threadIdx.x == 0) tile_counts[blockIdx.x] = 0;
        last_cta_scan_counts(tile_counts, &st->ndiff, &st->done_a);
        return;
    }
    const int D = DIM ? DIM : static_cast<int>(st->dims);
    const int kb = st->kb;
    const uint64_t tile0 = static_cast<uint64_t>(blockIdx.x) * kFlagTile;
    const uint32_t fvb = static_cast<uint32_t>(D) * bitlen32(st->rec_max);
    const uint32_t fdb = static_cast<uint32_t>(D) * bitlen32(st->rec_maxdiff);
    constexpr int KD = DIM ? DIM : kMaxDims;
    constexpr int kG = 4;
    uint32_t cnt = 0;
    KT k[kG][5];   // per group: the previous key, then four keys
#pragma unroll
    for (int u = 0; u < kG; ++u) {
        const uint64_t g = tile0 / 4 + u * 256 + threadIdx.x;
        const uint64_t j0 = 4 * g;
        if (j0 + 4 <= B && sizeof(KT) == 4) {
            const uint4 v = __ldg(reinterpret_cast<const uint4*>(rec) + g);
            k[u][1] = static_cast<KT>(v.x); k[u][2] = static_cast<KT>(v.y);
            k[u][3] = static_cast<KT>(v.z); k[u][4] = static_cast<KT>(v.w);
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) k[u][1 + q] = j0 + q < B ? ldg_key(rec + j0 + q) : KT(0);
        }
        k[u][0] = j0 && j0 - 1 < B ? ldg_key(rec + j0 - 1) : KT(0);
    }
#pragma unroll
    for (int u = 0; u < kG; ++u) {
        const uint64_t g = tile0 / 4 + u * 256 + threadIdx.x;
        const uint64_t j0 = 4 * g;
        if (j0 >= B) continue;
        uint32_t prev[KD], cur[KD];
        rec_read<DIM>(k[u][0], D, kb, prev);
        uint32_t ch[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint64_t j = j0 + q;
            if (j >= B) break;
            rec_read<DIM>(k[u][1 + q], D, kb, cur);
            ch[q] = (l2 && j > 0) ? l2_rule(cur, prev, D, fvb, fdb) : 0u;
            cnt += ch[q];
#pragma unroll
            for (int d = 0; d < KD; ++d) {
                if (!DIM && d >= D) break;
                prev[d] = cur[d];
            }
        }
        if (j0 + 4 <= B && (reinterpret_cast<uintptr_t>(choice2) & 3) == 0) {
            *reinterpret_cast<uint32_t*>(choice2 + j0) = ch[0] | (ch[1] << 8) | (ch[2] << 16) | (ch[3] << 24);
        } else {
            for (int q = 0; q < 4 && j0 + q < B; ++q) choice2[j0 + q] = static_cast<uint8_t>(ch[q]);
        }
    }
    cnt = warp_sum(cnt);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < 8; ++w) t += wsum[w];
        tile_counts[blockIdx.x] = t;
    }
    // the last CTA turns the counts into the flag scan's tile prefixes (total: ndiff)
    last_cta_scan_counts(tile_counts, &st->ndiff, &st->done_a);
}
// Writes record j < B as a kept row or as its ZigZag'd wrapped difference from the
// previous record (lcps_cpp.cpp:1305-1454), ET bytes per value: the ranked pass of the
// flag scan of choice2, with the tiles and ranks of flag_apply_kernel (tile_prefix left
// by k_l2_choice).  Each record's coordinates are decoded once (a difference
// record takes its predecessor's from the neighbouring lane, or from the previous
// round's last lane) and the state's parameters are read once per thread.  DIM as for
// k_l2_choice.
template <typename KT, typename ET, int DIM>
__global__ void __launch_bounds__(kFlagThreads) k_l2_rows(const KT* __restrict__ rec, const EncState* st,
                                                          const uint8_t* __restrict__ choice2, ET* __restrict__ keep,
                                                          ET* __restrict__ diff, const uint32_t* __restrict__ tile_prefix) {
    if (DIM == 3 && !l2_dim3(st)) return;
    if (DIM == 0 && l2_dim3(st)) return;
    __shared__ uint32_t wsum[kFlagThreads / 32];
    const uint32_t B = st->B;
    // the grid covers n >= B entries: tiles wholly past the records have nothing to write
    if (static_cast<uint64_t>(blockIdx.x) * kFlagTile >= B) return;
    const int D = DIM ? DIM : static_cast<int>(st->dims);
    const int kb = st->kb;
    const int64_t wmin = st->wrap_min_corr, wmax = st->wrap_max_corr, wrange = st->wrap_range;
    constexpr int KD = DIM ? DIM : kMaxDims;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kFlagTile + static_cast<uint64_t>(warp) * 32 * kFlagItems;
    // all of the slice's loads first: choice bytes, and the keys when they are at most
    // eight bytes (one round trip to memory per warp instead of one per item)
    constexpr bool kPre = sizeof(KT) <= 8;
    KT kk[kPre ? kFlagItems : 1];
    uint32_t m[kFlagItems];
#pragma unroll
    for (int k = 0; k < kFlagItems; ++k) {
        const uint64_t i = base + 32 * k + lane;
        m[k] = i < B ? choice2[i] : 0u;
        if (kPre) kk[k] = i < B ? ldg_key(rec + i) : KT(0);
    }
    KT kprev = base > 0 && base - 1 < B ? ldg_key(rec + base - 1) : KT(0);
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
    // coordinates of the record before this warp's slice (lane 0 of the first round)
    uint32_t carry[KD];
#pragma unroll
    for (int d = 0; d < KD; ++d) carry[d] = 0;
    if (base > 0 && base - 1 < B) rec_read<DIM>(kprev, D, kb, carry);
#pragma unroll   // constant indices keep m[] and kk[] in registers
    for (int k = 0; k < kFlagItems; ++k) {
        const uint64_t i = base + 32 * k + lane;
        const bool valid = i < B;
        uint32_t cur[KD], prev[KD];
#pragma unroll
        for (int d = 0; d < KD; ++d) cur[d] = 0;
        if (valid) rec_read<DIM>(kPre ? kk[k] : ldg_key(rec + i), D, kb, cur);
#pragma unroll
        for (int d = 0; d < KD; ++d) {
            if (!DIM && d >= D) break;
            const uint32_t up = __shfl_up_sync(0xffffffffu, cur[d], 1);
            prev[d] = lane == 0 ? carry[d] : up;
            carry[d] = __shfl_sync(0xffffffffu, cur[d], 31);
        }
        const uint32_t mk = m[k];
        if (valid) {
            const uint32_t rank = run + __popc(mk & lt);
            if (!((mk >> lane) & 1u)) {
                const uint64_t row = (i - rank) * static_cast<uint64_t>(D);
#pragma unroll
                for (int d = 0; d < KD; ++d)
                    if (DIM || d < D) keep[row + d] = static_cast<ET>(cur[d]);
            } else {
                const uint64_t row = static_cast<uint64_t>(rank) * D;
#pragma unroll
                for (int d = 0; d < KD; ++d) {
                    if (!DIM && d >= D) break;
                    // prediction = previous record (already inside [wrap_min, wrap_max]);
                    // three dimensions of at most 21 bits wrap and ZigZag in 32 bits
                    if (DIM == 3) {
                        int32_t corr = static_cast<int32_t>(prev[d]) - static_cast<int32_t>(cur[d]);
                        if (corr < static_cast<int32_t>(wmin)) corr += static_cast<int32_t>(wrange);
                        else if (corr > static_cast<int32_t>(wmax)) corr -= static_cast<int32_t>(wrange);
                        diff[row + d] = static_cast<ET>((static_cast<uint32_t>(corr) << 1) ^
                                                        static_cast<uint32_t>(corr >> 31));
                    } else {
                        int64_t corr = static_cast<int64_t>(prev[d]) - static_cast<int64_t>(cur[d]);
                        if (corr < wmin) corr += wrange;
                        else if (corr > wmax) corr -= wrange;
                        diff[row + d] = static_cast<ET>((static_cast<uint64_t>(corr) << 1) ^
                                                        static_cast<uint64_t>(corr >> 63));
                    }
                }
            }
        }
        run += __popc(mk);
    }
}

// ------------------------------------------------------------- stream stats
struct StreamRef {
    const void* data;       // record-major, esz bytes per value
    uint32_t dims;
    uint32_t esz;           // 1, 2 or 4
    const uint32_t* count_dev;  // records (device) or null -> count_const
    const uint32_t* count_sub;  // when set, subtracted from *count_dev
    uint64_t count_const;
};
struct StreamRefs {
    StreamRef s[kCodeStreams];
};

// The streams one statistics launch covers (blockIdx.y indexes s[]).
struct StreamSel {
    int s[kCodeStreams];
};

__device__ __forceinline__ uint64_t stream_records(const StreamRef& r) {
    if (!r.count_dev) return r.count_const;
    return static_cast<uint64_t>(*r.count_dev) - (r.count_sub ? *r.count_sub : 0u);
}

// Warp-aggregated histogram increment: lanes holding equal values add once.
__device__ __forceinline__ void warp_hist_add(uint32_t* bins, uint32_t v, bool valid) {
    const uint32_t active = __ballot_sync(0xffffffffu, valid);
    if (!valid) return;
    const uint32_t peers = __match_any_sync(active, v);
    if ((peers & lanemask_lt()) == 0) atomicAdd(&bins[v], static_cast<uint32_t>(__popc(peers)));
}

constexpr int kSmemHistBins = 4096;

__device__ void choice_stats(EncState* st, uint32_t* gh);

// Per-stream statistics in one pass: per-dimension min/max, overall max, the record
// tags (max(1, max_d bitlen v)) histogram and bit total, and the value histogram of
// the raw candidate (values < 2^18; a larger max makes the candidate ineligible).
// Template DIM is the records' dimension count (0 = read it at run time; the encoder
// launches it for streams of more than four dimensions).  Each thread
// takes groups of 4 records with 16-byte loads; values below 8 count in registers,
// below kSmemHistBins in shared memory, the rest in global memory.  Register
// counters flush before they could overflow.  blockIdx.y selects the stream from
// sel[] (the streams of one launch share DIM).
// derive: complete CH20's statistics from the level-2 counts (done once, by block (0, 0)).
template <int DIM>
__global__ void __launch_bounds__(256) k_stream_stats(StreamRefs refs, EncState* st, uint32_t* hist,
                                                       uint64_t hist_stride, StreamSel sel, int derive) {
    if (derive && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) choice_stats(st, hist + hist_stride * 3);
    const int s = sel.s[blockIdx.y];
    const StreamRef r = refs.s[s];
    const uint32_t D = DIM ? DIM : r.dims;
    const uint64_t nrec = stream_records(r);
    __shared__ uint32_t smin[kMaxDims], smax[kMaxDims], stag[34];
    __shared__ uint32_t sh[kSmemHistBins];
    __shared__ unsigned long long sbits;
    if (threadIdx.x < kMaxDims) { smin[threadIdx.x] = 0xffffffffu; smax[threadIdx.x] = 0; }
    if (threadIdx.x < 34) stag[threadIdx.x] = 0;
    constexpr int HB = kSmemHistBins;
    for (int t = threadIdx.x; t < HB; t += blockDim.x) sh[t] = 0;
    if (threadIdx.x == 0) sbits = 0;
    __syncthreads();
    uint32_t* gh = hist + hist_stride * s;
    constexpr int KD = DIM ? DIM : kMaxDims;
    // 4-record groups per thread between flushes of the 16-bit register counters.
    constexpr uint32_t kFlushGroups = 16383 / KD;
    uint32_t mn[KD], mx[KD];
#pragma unroll
    for (int d = 0; d < KD; ++d) { mn[d] = 0xffffffffu; mx[d] = 0; }
    uint64_t bits = 0;
    PackedCount8 vc, tc;
    uint32_t groups_since_flush = 0;
    auto value = [&](uint32_t v, int d, uint32_t& tag) {
        mn[d] = v < mn[d] ? v : mn[d];
        mx[d] = v > mx[d] ? v : mx[d];
        const uint32_t w = bitlen32(v);
        tag = w > tag ? w : tag;
        if (v < 8) vc.add(v);
        else if (v < HB) atomicAdd(&sh[v], 1u);
        else if (v < kRansMaxAlphabet) atomicAdd(&gh[v], 1u);
    };
    auto record_done = [&](uint32_t tag) {
        bits += static_cast<uint64_t>(D) * tag;
        if (tag < 8) tc.add(tag);
        else atomicAdd(&stag[tag], 1u);
    };
    const uint64_t ngroups = (nrec + 3) / 4;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t rounds = (ngroups + stride - 1) / stride;
    const bool vec_ok = (reinterpret_cast<uintptr_t>(r.data) & 15) == 0;
    const uint32_t esz = r.esz;
    for (uint64_t rr = 0; rr < rounds; ++rr) {
        const uint64_t g = rr * stride + static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
        if (g < ngroups) {
            const uint64_t rec0 = 4 * g;
            if (DIM && vec_ok && rec0 + 4 <= nrec) {
                uint32_t v[4 * KD];
                if (esz == 4) {
                    const uint4* p = reinterpret_cast<const uint4*>(static_cast<const uint32_t*>(r.data) + rec0 * D);
#pragma unroll
                    for (int q = 0; q < KD; ++q) {
                        const uint4 t = __ldg(p + q);
                        v[4 * q] = t.x; v[4 * q + 1] = t.y; v[4 * q + 2] = t.z; v[4 * q + 3] = t.w;
                    }
                } else if (esz == 2) {   // 8 KD bytes = 2 KD aligned words
                    const uint32_t* p = reinterpret_cast<const uint32_t*>(static_cast<const uint16_t*>(r.data) + rec0 * D);
#pragma unroll
                    for (int q = 0; q < 2 * KD; ++q) {
                        const uint32_t t = __ldg(p + q);
                        v[2 * q] = t & 0xFFFFu;
                        v[2 * q + 1] = t >> 16;
                    }
                } else {   // 4 KD bytes = KD aligned words
                    const uint32_t* p = reinterpret_cast<const uint32_t*>(static_cast<const uint8_t*>(r.data) + rec0 * D);
#pragma unroll
                    for (int q = 0; q < KD; ++q) {
                        const uint32_t t = __ldg(p + q);
#pragma unroll
                        for (int b = 0; b < 4; ++b) v[4 * q + b] = (t >> (8 * b)) & 0xFFu;
                    }
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    uint32_t tag = 1;
#pragma unroll
                    for (int d = 0; d < KD; ++d) value(v[k * KD + d], d, tag);
                    record_done(tag);
                }
            } else {
                for (uint64_t rec = rec0; rec < rec0 + 4 && rec < nrec; ++rec) {
                    uint32_t tag = 1;
#pragma unroll
                    for (int d = 0; d < KD; ++d)
                        if (DIM || d < static_cast<int>(D)) value(load_elem(r.data, rec * D + d, esz), d, tag);
                    record_done(tag);
                }
            }
        }
        if (++groups_since_flush == kFlushGroups) {
            vc.flush(sh);
            tc.flush(stag);
            groups_since_flush = 0;
        }
    }
    vc.flush(sh);
    tc.flush(stag);
#pragma unroll
    for (int d = 0; d < KD; ++d) {
        if (DIM || d < static_cast<int>(D)) {
            const uint32_t a = warp_min(mn[d]), b = warp_max(mx[d]);
            if ((threadIdx.x & 31) == 0) { atomicMin(&smin[d], a); atomicMax(&smax[d], b); }
        }
    }
    bits = warp_sum(bits);
    if ((threadIdx.x & 31) == 0 && bits) atomicAdd(&sbits, static_cast<unsigned long long>(bits));
    __syncthreads();
    StreamStats& gs = st->st[s];
    if (threadIdx.x < D && smax[threadIdx.x] >= smin[threadIdx.x]) {
        atomicMin(&gs.minv[threadIdx.x], smin[threadIdx.x]);
        atomicMax(&gs.maxv[threadIdx.x], smax[threadIdx.x]);
        atomicMax(&gs.maxall, smax[threadIdx.x]);
    }
    if (threadIdx.x < 34 && stag[threadIdx.x]) {
        atomicAdd(&gs.tag_hist[threadIdx.x], stag[threadIdx.x]);
        atomicMax(&gs.maxtag, threadIdx.x);
    }
    if (threadIdx.x == 0 && sbits) atomicAdd(reinterpret_cast<unsigned long long*>(&gs.tag_bits), sbits);
    for (int t = threadIdx.x; t < HB; t += blockDim.x)
        if (sh[t]) atomicAdd(&gh[t], sh[t]);
}

// ------------------------------------------ stream stats, lane-column counting
// The statistics of k_stream_stats for streams of 1..4 dimensions, counted with one
// conflict-free shared-memory atomic per value: values below kLaneBins and the record
// tags land in a [bin][lane] table (word bin * 32 + lane, so the 32 lanes of a warp
// always hit 32 distinct banks; the warps of a CTA share the table).  A group is DIM
// 16-byte loads (16 / esz records).  The launch's groups, over all selected streams,
// split evenly across the CTAs; a CTA whose range crosses a stream boundary flushes its
// tables at the boundary.  The tag bit total is derived from the tag counts.
constexpr int kLaneBins = 256;
constexpr int kStatsTagBins = 34;
constexpr uint32_t kStatsThreads = 256;
constexpr size_t kStatsLaneBytes = (kLaneBins + kStatsTagBins) * 32 * sizeof(uint32_t);
constexpr size_t kStatsWideBytes = kStatsLaneBytes + kSmemHistBins * sizeof(uint32_t);

__device__ __forceinline__ uint32_t uint4_word(const uint4& a, int i) {
    switch (i & 3) {
        case 0: return a.x;
        case 1: return a.y;
        case 2: return a.z;
        default: return a.w;
    }
}

// Value j of a group held as 16-byte words w[], ESZ bytes per value (j is a constant
// once the callers' loops are unrolled).
template <int ESZ>
__device__ __forceinline__ uint32_t group_value(const uint4* w, int j) {
    if constexpr (ESZ == 1) return (uint4_word(w[j >> 4], j >> 2) >> (8 * (j & 3))) & 0xFFu;
    else if constexpr (ESZ == 2) return (uint4_word(w[j >> 3], j >> 1) >> (16 * (j & 1))) & 0xFFFFu;
    else return uint4_word(w[j >> 2], j);
}

// Groups [u0, u1) of one stream, strided over the CTA's threads.
template <int DIM, int ESZ>
__device__ __forceinline__ void lane_stats_segment(const StreamRef& r, uint64_t nrec, uint64_t u0, uint64_t u1,
                                                   uint32_t* lp, uint32_t* tl, uint32_t* sh, uint32_t* gh,
                                                   uint32_t (&mn)[DIM], uint32_t (&mx)[DIM]) {
    constexpr int GR = 16 / ESZ;   // records per group
    uint32_t* lpl = lp + (threadIdx.x & 31);
    uint32_t* tll = tl + (threadIdx.x & 31);
    const auto record = [&](const uint32_t (&v)[DIM]) {
        uint32_t o = 1;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const uint32_t x = v[d];
            mn[d] = x < mn[d] ? x : mn[d];
            mx[d] = x > mx[d] ? x : mx[d];
            o |= x;
            if (ESZ == 1 || x < static_cast<uint32_t>(kLaneBins)) atomicAdd(lpl + (x << 5), 1u);
            else if (x < static_cast<uint32_t>(kSmemHistBins)) atomicAdd(&sh[x], 1u);
            else if (x < kRansMaxAlphabet) atomicAdd(&gh[x], 1u);
        }
        atomicAdd(tll + (static_cast<uint32_t>(32 - __clz(o)) << 5), 1u);   // tag = max(1, bitlen)
    };
    const bool vec_ok = (reinterpret_cast<uintptr_t>(r.data) & 15) == 0;
    for (uint64_t u = u0 + threadIdx.x; u < u1; u += kStatsThreads) {
        const uint64_t rec0 = u * GR;
        if (vec_ok && rec0 + GR <= nrec) {
            uint4 w[DIM];
            const uint4* p = static_cast<const uint4*>(r.data) + u * DIM;
#pragma unroll
            for (int q = 0; q < DIM; ++q) w[q] = __ldg(p + q);
#pragma unroll
            for (int k = 0; k < GR; ++k) {
                uint32_t v[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) v[d] = group_value<ESZ>(w, k * DIM + d);
                record(v);
            }
        } else {
            for (uint64_t rec = rec0; rec < rec0 + GR && rec < nrec; ++rec) {
                uint32_t v[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) v[d] = load_elem(r.data, rec * DIM + d, ESZ);
                record(v);
            }
        }
    }
}

// streams: bit s selects refs.s[s].  derive: as for k_stream_stats.  wide: some selected
// stream stores 2- or 4-byte values (the table of values kLaneBins..kSmemHistBins-1
// follows the lane tables in dynamic shared memory).
template <int DIM>
__global__ void __launch_bounds__(kStatsThreads, 4) k_stream_stats_lanes(StreamRefs refs, EncState* st,
                                                                         uint32_t* hist, uint64_t hist_stride,
                                                                         uint32_t streams, int derive, int wide) {
    if (derive && blockIdx.x == 0 && threadIdx.x == 0) choice_stats(st, hist + hist_stride * 3);
    extern __shared__ __align__(16) uint32_t sdyn[];
    uint32_t* lp = sdyn;                      // [kLaneBins][32]
    uint32_t* tl = lp + kLaneBins * 32;       // [kStatsTagBins][32]
    uint32_t* sh = tl + kStatsTagBins * 32;   // [kSmemHistBins], wide launches
    __shared__ uint32_t smin[DIM], smax[DIM];
    const uint32_t words = static_cast<uint32_t>((wide ? kStatsWideBytes : kStatsLaneBytes) / 16);
    for (uint32_t t = threadIdx.x; t < words; t += kStatsThreads)
        reinterpret_cast<uint4*>(sdyn)[t] = make_uint4(0, 0, 0, 0);
    uint64_t total = 0;
#pragma unroll 1
    for (int s = 0; s < kCodeStreams; ++s) {
        if (!((streams >> s) & 1u)) continue;
        const StreamRef r = refs.s[s];
        total += (stream_records(r) + 16 / r.esz - 1) / (16 / r.esz);
    }
    const uint64_t lo = total * blockIdx.x / gridDim.x, hi = total * (blockIdx.x + 1) / gridDim.x;
    uint64_t off = 0;
#pragma unroll 1
    for (int s = 0; s < kCodeStreams; ++s) {
        if (!((streams >> s) & 1u)) continue;
        const StreamRef r = refs.s[s];
        const uint64_t nrec = stream_records(r);
        const uint64_t base = off, ng = (nrec + 16 / r.esz - 1) / (16 / r.esz);
        off += ng;
        const uint64_t a = lo > base ? lo : base, b = hi < base + ng ? hi : base + ng;
        if (a >= b) continue;   // uniform over the CTA
        uint32_t* gh = hist + hist_stride * s;
        if (threadIdx.x < DIM) { smin[threadIdx.x] = 0xffffffffu; smax[threadIdx.x] = 0; }
        __syncthreads();
        uint32_t mn[DIM], mx[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) { mn[d] = 0xffffffffu; mx[d] = 0; }
        if (r.esz == 1)
            lane_stats_segment<DIM, 1>(r, nrec, a - base, b - base, lp, tl, sh, gh, mn, mx);
        else if (r.esz == 2)
            lane_stats_segment<DIM, 2>(r, nrec, a - base, b - base, lp, tl, sh, gh, mn, mx);
        else
            lane_stats_segment<DIM, 4>(r, nrec, a - base, b - base, lp, tl, sh, gh, mn, mx);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const uint32_t x = warp_min(mn[d]), y = warp_max(mx[d]);
            if ((threadIdx.x & 31) == 0) { atomicMin(&smin[d], x); atomicMax(&smax[d], y); }
        }
        __syncthreads();
        StreamStats& gs = st->st[s];
        uint32_t vmax = 0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) vmax = smax[d] > vmax ? smax[d] : vmax;
        if (threadIdx.x < DIM) {
            atomicMin(&gs.minv[threadIdx.x], smin[threadIdx.x]);
            atomicMax(&gs.maxv[threadIdx.x], smax[threadIdx.x]);
            atomicMax(&gs.maxall, smax[threadIdx.x]);
        }
        // column sums, read along a diagonal (lane l of a warp reads bank (l + i) & 31),
        // leaving the tables zeroed for the next segment
        const uint32_t nb = vmax < static_cast<uint32_t>(kLaneBins) ? vmax + 1 : static_cast<uint32_t>(kLaneBins);
        for (uint32_t t = threadIdx.x; t < nb; t += kStatsThreads) {
            uint32_t c = 0;
#pragma unroll 8
            for (uint32_t i = 0; i < 32; ++i) {
                uint32_t* q = lp + t * 32 + ((i + t) & 31);
                c += *q;
                *q = 0;
            }
            if (c) atomicAdd(&gh[t], c);
        }
        if (threadIdx.x < static_cast<uint32_t>(kStatsTagBins)) {
            const uint32_t t = threadIdx.x;
            uint32_t c = 0;
#pragma unroll 8
            for (uint32_t i = 0; i < 32; ++i) {
                uint32_t* q = tl + t * 32 + ((i + t) & 31);
                c += *q;
                *q = 0;
            }
            if (c) {
                atomicAdd(&gs.tag_hist[t], c);
                atomicMax(&gs.maxtag, t);
                atomicAdd(reinterpret_cast<unsigned long long*>(&gs.tag_bits),
                          static_cast<unsigned long long>(c) * t * DIM);
            }
        }
        if (r.esz > 1) {
            const uint32_t ne = vmax < static_cast<uint32_t>(kSmemHistBins) ? vmax + 1 : static_cast<uint32_t>(kSmemHistBins);
            for (uint32_t t = kLaneBins + threadIdx.x; t < ne; t += kStatsThreads)
                if (sh[t]) { atomicAdd(&gh[t], sh[t]); sh[t] = 0; }
        }
        __syncthreads();
    }
}

// One CTA per (stream, kind): kind 0 = raw value table, kind 1 = tag table.
__device__ void plan_stream(const StreamRefs& refs, EncState* st, uint32_t bytes_per_lane, uint32_t max_steps, int s);

// The table bytes of stream s's chosen coding into out (and its length into the plan)
// and its encoder symbol entries into et, by one CTA of kTableThreads; stage holds
// 4 * kSerStageSyms bytes.
__device__ void serialize_stream(EncState* st, const uint32_t* prob, const uint32_t* cum, const uint32_t* tag_prob,
                                 const uint32_t* tag_cum, uint64_t hist_stride, int s, uint8_t* out, uint4* et,
                                 uint32_t* stage) {
    StreamChoice& c = st->ch[s];
    const bool raw = c.enc == kEncRaw;
    if (!raw && c.enc != kEncTagged) {
        if (threadIdx.x == 0) c.table_len = 0;
        return;
    }
    const uint32_t* pr = raw ? prob + hist_stride * s : tag_prob + 64 * s;
    const uint32_t* cm = raw ? cum + hist_stride * s : tag_cum + 64 * s;
    const uint32_t len = serialize_table_block(pr, c.sec_alphabet, out, stage);
    if (threadIdx.x == 0) c.table_len = len;
    for (uint32_t a = threadIdx.x; a < c.sec_alphabet; a += blockDim.x) et[a] = make_enc_symbol(pr[a], cm[a], c.sec_prec);
}

// The CTA that finishes last plans the launch's streams (plan_stream), so that the plan
// needs no launch of its own; done is the launch's hand-off counter.  For IDR0 (s0 = 0)
// each CTA first completes the statistics its table reads from the level-1 counts.  With
// ser_out (a launch of one stream), the last CTA also serialises that stream's table to
// ser_out + s0 * ser_stride and writes its encoder entries to etab.
__global__ void __launch_bounds__(kTableThreads) k_tables(StreamRefs refs, EncState* st, uint32_t* hist,
                                                           uint64_t hist_stride, uint32_t* prob, uint32_t* cum,
                                                           uint32_t* tag_prob, uint32_t* tag_cum, int s0,
                                                           uint32_t bytes_per_lane, uint32_t max_steps,
                                                           uint32_t* done, uint8_t* ser_out, uint64_t ser_stride,
                                                           uint4* etab) {
    extern __shared__ __align__(16) uint32_t tstage[];   // kTableStageBytes
    const int s = s0 + blockIdx.x, kind = blockIdx.y;
    const StreamRef r = refs.s[s];
    const uint64_t nrec = stream_records(r);
    if (s == 0) {
        if (threadIdx.x == 0) idrel_stats(st, hist, r.count_const, kind);
        __syncthreads();
    }
    if (kind == 0) {
        const uint32_t maxall = st->st[s].maxall;
        const bool ok = nrec > 0 && maxall < kRansMaxAlphabet;
        build_rans_table(hist + hist_stride * s, ok ? maxall + 1 : 0, ok ? nrec * r.dims : 0,
                         prob + hist_stride * s, cum + hist_stride * s, &st->raw_tab[s], tstage);
    } else {
        const uint32_t A = nrec ? st->st[s].maxtag + 1 : 0;
        build_rans_table(st->st[s].tag_hist, A, nrec, tag_prob + 64 * s, tag_cum + 64 * s, &st->tag_tab[s],
                         tstage);
    }
    __shared__ bool s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(done, 1u) == gridDim.x * gridDim.y - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x < gridDim.x) plan_stream(refs, st, bytes_per_lane, max_steps, s0 + threadIdx.x);
    if (ser_out) {
        __syncthreads();   // the plan of stream s0 is written
        static_assert(4 * kSerStageSyms <= kTableStageBytes, "the serialisation stage fits the table stage");
        serialize_stream(st, prob, cum, tag_prob, tag_cum, hist_stride, s0, ser_out + ser_stride * s0, etab, tstage);
    }
    if (threadIdx.x == 0) *done = 0;
}

__device__ inline uint64_t section_overhead(uint32_t table_bytes, uint32_t chunks, uint32_t lanes, uint32_t prec) {
    return 1 + 4 + 4 + static_cast<uint64_t>(table_bytes) + 8 + 1 + 4 + 8 + 4ull * chunks +
           state_bytes(lanes, chunks, prec);
}

// Chunking of a rANS section: enough lanes that each carries about bytes_per_lane
// coded bytes (the packed final state per lane is the size overhead), and enough that
// no lane codes more than max_steps symbols (the serial depth of the kernel).  Below
// 32 lanes the section is one chunk of W = next power of two lanes.
__device__ inline void plan_chunks(uint64_t count, double est_payload, uint32_t bytes_per_lane, uint32_t max_steps,
                                   uint32_t* chunks, uint64_t* S, uint32_t* lanes) {
    uint64_t need = static_cast<uint64_t>(est_payload / bytes_per_lane) + 1;
    const uint64_t depth = (count + max_steps - 1) / max_steps;
    if (need < depth) need = depth;
    if (need < 32) {
        uint32_t w = 1;
        while (w < need) w <<= 1;
        *lanes = w;
        *S = (count + w - 1) / w * w;
        *chunks = 1;
        return;
    }
    uint64_t ch = (need + 31) / 32;
    const uint64_t max_ch = (count + 31) / 32;
    if (ch > max_ch) ch = max_ch;
    if (ch < 1) ch = 1;
    uint64_t s = (count + ch - 1) / ch;
    s = (s + 31) & ~31ull;
    if (s < 32) s = 32;
    *S = s;
    *lanes = 32;
    *chunks = static_cast<uint32_t>((count + s - 1) / s);
}

// A table descriptor written by another CTA of the same launch, read from L2.
__device__ __forceinline__ RansTableDev load_table_cg(const RansTableDev* t) {
    RansTableDev v;
    v.alphabet = __ldcg(&t->alphabet);
    v.prec = __ldcg(&t->prec);
    v.n = __ldcg(&t->n);
    v.cost_bits = __ldcg(&t->cost_bits);
    v.table_bytes = __ldcg(&t->table_bytes);
    v.pad = 0;
    return v;
}

// Chooses component s's encoding: the smallest estimated size among tagged, fixed and
// raw (ties in that order, as lcps_cpp.cpp:1150-1170), empty when no records.  Runs in
// the table launch's last CTA, once every table of the launch is built.
__device__ void plan_stream(const StreamRefs& refs, EncState* st, uint32_t bytes_per_lane, uint32_t max_steps, int s) {
    const RansTableDev tag_t = load_table_cg(&st->tag_tab[s]);
    const RansTableDev raw_t = load_table_cg(&st->raw_tab[s]);
    const StreamRef r = refs.s[s];
    const uint64_t nrec = stream_records(r);
    StreamChoice& c = st->ch[s];
    const StreamStats& g = st->st[s];
    c.dims = r.dims;
    c.records = nrec;
    c.enc = kEncEmpty;
    c.sec_chunks = 0;
    c.sec_S = 0;
    c.sec_count = 0;
    c.packed_bits = 0;
    c.max_width = 0;
    c.est[0] = c.est[1] = c.est[2] = c.est[3] = ~0ull;
    if (nrec == 0) {
        c.est[kEncEmpty] = 13;
        return;
    }
    if (tag_t.alphabet == 0xFFFFFFFFu || raw_t.alphabet == 0xFFFFFFFFu)
        set_error(&st->err, kErrInternal);
    // fixed (width 0 = constant component)
    uint64_t fixed = 13 + 9ull * r.dims;
    for (uint32_t d = 0; d < r.dims; ++d) {
        const uint32_t span = g.maxv[d] - g.minv[d];
        const int w = bitlen32(span);
        c.width[d] = static_cast<uint8_t>(w);
        fixed += (nrec * w + 7) / 8;
    }
    c.est[kEncFixed] = fixed;
    // tagged
    uint32_t tag_ch = 0, tag_lanes = 0;
    uint64_t tag_S = 0;
    {
        const RansTableDev& t = tag_t;
        const double payload = t.cost_bits / 8.0;
        plan_chunks(nrec, payload, bytes_per_lane, max_steps, &tag_ch, &tag_S, &tag_lanes);
        c.est[kEncTagged] = 13 + 1 + section_overhead(t.table_bytes, tag_ch, tag_lanes, t.prec) +
                            static_cast<uint64_t>(payload) + 1 + 8 + (g.tag_bits + 7) / 8;
    }
    // raw.  Tables too large for the shared-memory fast paths make every coded symbol
    // slower on both sides, so from kLargeTableMinSymbols on their lanes get a shorter
    // serial depth: kLargeTableShortSteps while the frame's chunks still fit one decoder
    // wave, kLargeTableMaxSteps beyond.
    uint32_t raw_ch = 0, raw_lanes = 0;
    uint64_t raw_S = 0;
    if (g.maxall < kRansMaxAlphabet && raw_t.alphabet != 0) {
        const RansTableDev& t = raw_t;
        const double payload = t.cost_bits / 8.0;
        const bool large = (t.alphabet > kSmemEncSyms || (1u << t.prec) > kSmemLookupSlots) &&
                           nrec * r.dims >= kLargeTableMinSymbols;
        const uint32_t deep = nrec * r.dims >= kLargeTableDeepSymbols ? kLargeTableMaxSteps : kLargeTableShortSteps;
        const uint32_t steps = large ? min(max_steps, deep) : max_steps;
        plan_chunks(nrec * r.dims, payload, bytes_per_lane, steps, &raw_ch, &raw_S, &raw_lanes);
        c.est[kEncRaw] = 13 + section_overhead(t.table_bytes, raw_ch, raw_lanes, t.prec) + static_cast<uint64_t>(payload) + 1;
    }
    uint8_t best = kEncTagged;
    if (c.est[kEncFixed] < c.est[best]) best = kEncFixed;
    if (c.est[kEncRaw] < c.est[best]) best = kEncRaw;
    c.enc = best;
    if (best == kEncTagged) {
        const RansTableDev& t = tag_t;
        c.sec_chunks = tag_ch;
        c.sec_S = tag_S;
        c.sec_lanes = tag_lanes;
        c.sec_count = nrec;
        c.sec_prec = t.prec;
        c.sec_alphabet = t.alphabet;
        c.packed_bits = g.tag_bits;
        c.max_width = static_cast<uint8_t>(g.maxtag);
    } else if (best == kEncRaw) {
        const RansTableDev& t = raw_t;
        c.sec_chunks = raw_ch;
        c.sec_S = raw_S;
        c.sec_lanes = raw_lanes;
        c.sec_count = nrec * r.dims;
        c.sec_prec = t.prec;
        c.sec_alphabet = t.alphabet;
    }
}

// ------------------------------------------------------------------ packing
// Tags of a tagged component: max(1, max_d bitlen(v)) per record (lcps_cpp.cpp:1032-1046).
template <typename ET>
__global__ void __launch_bounds__(256) k_tags(const ET* __restrict__ data, uint32_t D, uint64_t nrec,
                                               uint32_t* __restrict__ tags) {
    for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < nrec;
         j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint32_t t = 1;
        for (uint32_t d = 0; d < D; ++d) {
            const uint32_t w = bitlen32(data[j * D + d]);
            t = w > t ? w : t;
        }
        tags[j] = t;
    }
}

// Writes `width` bits of v (MSB first) at bit offset `bit` of a big-endian bitstream
// held as 32-bit words in big-endian byte order (converted when copied out).
__device__ __forceinline__ void put_bits(uint32_t* words, uint64_t bit, uint32_t v, int width) {
    const uint64_t w0 = bit >> 5;
    const int off = static_cast<int>(bit & 31);
    const uint64_t vv = static_cast<uint64_t>(v) << (64 - width);   // left-aligned
    const uint64_t sh = vv >> off;                                  // bits for words w0, w0+1
    const uint32_t hi = static_cast<uint32_t>(sh >> 32), lo = static_cast<uint32_t>(sh);
    if (hi) atomicOr(&words[w0], hi);
    if (lo) atomicOr(&words[w0 + 1], lo);
}

struct TagBitsIn {
    const uint32_t* tags;
    uint32_t D;
    __device__ uint64_t operator()(uint64_t j) const { return static_cast<uint64_t>(tags[j]) * D; }
};
template <typename ET>
struct TagPackOut {
    const ET* data;
    const uint32_t* tags;
    uint32_t D;
    uint32_t* words;
    __device__ void operator()(uint64_t j, uint64_t bit, uint64_t) const {
        const int t = static_cast<int>(tags[j]);
        for (uint32_t d = 0; d < D; ++d, bit += t) put_bits(words, bit, data[j * D + d], t);
    }
};

// Fixed-width packing of every dimension of one stream.  Per dimension d, value k takes
// bits [k*w, (k+1)*w) of an MSB-first bit stream (w = width[d] <= 32), written as
// big-endian 32-bit words so that byte 0 holds the first 8 bits.  Each warp packs a tile
// of 1024 records: it stages the tile's values of dimension d in shared memory
// (coalesced reads), then lane l packs records [32l, 32l+32) into exactly w words.
struct FixedPack {
    uint32_t* words[kMaxDims];   // per-dimension output (nwords[d] words)
    uint64_t nwords[kMaxDims];
    uint32_t minv[kMaxDims];
    uint32_t width[kMaxDims];
};
constexpr int kPackWarps = 8;
template <typename ET>
__device__ __forceinline__ void pack_fixed_tiles(const ET* __restrict__ data, uint32_t D, uint64_t nrec,
                                                 const FixedPack& fp, uint32_t* sw) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t ntiles = (nrec + 1023) / 1024;
    for (uint64_t tile = static_cast<uint64_t>(blockIdx.x) * kPackWarps + warp; tile < ntiles;
         tile += static_cast<uint64_t>(gridDim.x) * kPackWarps) {
        const uint64_t r0 = tile * 1024;
        for (uint32_t d = 0; d < D; ++d) {
            const uint32_t w = fp.width[d];
            if (w == 0) continue;
            const uint32_t mv = fp.minv[d];
            uint32_t x[32];   // all 32 loads in flight together
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const uint64_t k = r0 + 32 * j + lane;
                x[j] = k < nrec ? static_cast<uint32_t>(__ldg(data + k * D + d)) : mv;
            }
#pragma unroll
            for (int j = 0; j < 32; ++j) sw[33 * j + lane] = x[j] - mv;
            __syncwarp();
            uint64_t acc = 0;
            uint32_t nacc = 0, m = 0;
            uint32_t* out = fp.words[d];
            const uint64_t wbase = (r0 / 32 + lane) * w;
            const uint64_t nw = fp.nwords[d];
#pragma unroll 4
            for (int j = 0; j < 32; ++j) {
                acc = (acc << w) | sw[33 * lane + j];
                nacc += w;
                if (nacc >= 32) {
                    nacc -= 32;
                    if (wbase + m < nw) out[wbase + m] = __byte_perm(static_cast<uint32_t>(acc >> nacc), 0, 0x0123);
                    ++m;
                }
            }
            __syncwarp();
        }
    }
}

// The same packing for a one-byte stream whose DIM dimensions all have the width W (1,
// 2, 4 or 8, which divide 32): word t of dimension d holds records [t G, t G + G) (G = 32
// / W) with the first in the top bits, stored byte-swapped as pack_fixed_tiles stores
// it.  Thread t reads the group's G * DIM bytes with 4-byte loads and writes word t of
// every dimension.
template <int W, int DIM>
__device__ __forceinline__ void pack_fixed_u8_equal(const uint8_t* __restrict__ data, uint64_t nrec,
                                                    const FixedPack& fp) {
    constexpr int G = 32 / W, NB = G * DIM, NW = NB / 4;
    static_assert(NB % 4 == 0, "whole words per group");
    const uint64_t nw = (nrec + G - 1) / G;
    const bool aligned = (reinterpret_cast<uintptr_t>(data) & 3) == 0;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < nw; t += stride) {
        const uint64_t r0 = t * G;
        uint32_t acc[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) acc[d] = 0;
        if (aligned && r0 + G <= nrec) {
            const uint32_t* p = reinterpret_cast<const uint32_t*>(data + r0 * DIM);
            uint32_t b[NW];
#pragma unroll
            for (int q = 0; q < NW; ++q) b[q] = __ldg(p + q);
#pragma unroll
            for (int k = 0; k < G; ++k)
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    const int j = k * DIM + d;
                    const uint32_t v = ((b[j >> 2] >> (8 * (j & 3))) & 0xFFu) - fp.minv[d];
                    acc[d] |= v << (32 - W * (k + 1));
                }
        } else {
            for (int k = 0; k < G && r0 + k < nrec; ++k)
#pragma unroll
                for (int d = 0; d < DIM; ++d)
                    acc[d] |= (static_cast<uint32_t>(data[(r0 + k) * DIM + d]) - fp.minv[d]) << (32 - W * (k + 1));
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) fp.words[d][t] = __byte_perm(acc[d], 0, 0x0123);
    }
}

// Every fixed-coded component of a frame in one launch (blockIdx.y = component).
// equal_w: the width all dimensions share when pack_fixed_u8_equal applies (1, 2, 4 or
// 8; one-byte values, at most four dimensions), else 0.
struct FixedJob {
    FixedPack fp;
    const void* data;
    uint64_t nrec;
    uint32_t dims;
    uint32_t esz;
    uint32_t equal_w;
};
struct FixedJobs {
    FixedJob job[kCodeStreams];
};
__global__ void __launch_bounds__(32 * kPackWarps, 3) k_pack_fixed(FixedJobs J) {
    __shared__ uint32_t stage[kPackWarps][33 * 32];
    const FixedJob& j = J.job[blockIdx.y];
    if (j.equal_w) {
        const uint8_t* d8 = static_cast<const uint8_t*>(j.data);
#define CHAIN_PACK_EQ(W)                                                        \
    switch (j.dims) {                                                         \
        case 1: pack_fixed_u8_equal<W, 1>(d8, j.nrec, j.fp); return;          \
        case 2: pack_fixed_u8_equal<W, 2>(d8, j.nrec, j.fp); return;          \
        case 3: pack_fixed_u8_equal<W, 3>(d8, j.nrec, j.fp); return;          \
        default: pack_fixed_u8_equal<W, 4>(d8, j.nrec, j.fp); return;         \
    }
        switch (j.equal_w) {
            case 1: CHAIN_PACK_EQ(1)
            case 2: CHAIN_PACK_EQ(2)
            case 4: CHAIN_PACK_EQ(4)
            default: CHAIN_PACK_EQ(8)
        }
#undef CHAIN_PACK_EQ
    }
    uint32_t* sw = stage[threadIdx.x >> 5];
    if (j.esz == 1) pack_fixed_tiles(static_cast<const uint8_t*>(j.data), j.dims, j.nrec, j.fp, sw);
    else if (j.esz == 2) pack_fixed_tiles(static_cast<const uint16_t*>(j.data), j.dims, j.nrec, j.fp, sw);
    else pack_fixed_tiles(static_cast<const uint32_t*>(j.data), j.dims, j.nrec, j.fp, sw);
}

// rANS section of each coded stream (index into RansJobs, -1 = none).
struct StreamJobs {
    int job[kCodeStreams];
};

// Big-endian words -> bytes in place (so that byte 0 holds the first 8 bits).
__global__ void k_words_to_bytes(uint32_t* words, uint64_t nwords) {
    for (uint64_t w = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; w < nwords;
         w += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        words[w] = __byte_perm(words[w], 0, 0x0123);
}

// Serialises every chosen table of streams s0.. (blockIdx.y == 0, one CTA per stream)
// and writes the streams' encoder symbol entries (make_enc_symbol) for their rANS
// sections (blockIdx.y > 0: kEtabSlices CTAs per stream, each a slice of the alphabet).
__global__ void __launch_bounds__(1024) k_serialize_tables(EncState* st, const uint32_t* prob, const uint32_t* tag_prob,
                                                            uint64_t hist_stride, uint8_t* out, uint64_t out_stride,
                                                            int s0, RansJobs J, StreamJobs sj) {
    extern __shared__ __align__(16) uint32_t ser_stage[];   // kSerStageSyms u32
    const int s = s0 + blockIdx.x;
    if (blockIdx.y > 0) {
        if (sj.job[s] < 0) return;
        const RansJob& jb = J.job[sj.job[s]];
        uint4* et = const_cast<uint4*>(jb.etab);
        for (uint32_t a = (blockIdx.y - 1) * blockDim.x + threadIdx.x; a < jb.alphabet;
             a += (gridDim.y - 1) * blockDim.x)
            et[a] = make_enc_symbol(jb.prob[a], jb.cum[a], jb.prec);
        return;
    }
    StreamChoice& c = st->ch[s];
    uint32_t len = 0;
    if (c.enc == kEncRaw)
        len = serialize_table_block(prob + hist_stride * s, c.sec_alphabet, out + out_stride * s, ser_stage);
    else if (c.enc == kEncTagged)
        len = serialize_table_block(tag_prob + 64 * s, c.sec_alphabet, out + out_stride * s, ser_stage);
    if (threadIdx.x == 0) c.table_len = len;
}
constexpr unsigned kEtabSlices = 8;

// --------------------------------------------------------------- assembly
struct AssemblyIn {
    const uint8_t* table_bytes;   // [kCodeStreams] x table_stride
    uint64_t table_stride;
    const uint32_t* chunk_len[kCodeStreams];
    const uint8_t* states[kCodeStreams];         // packed final lane states
    const uint8_t* slots[kCodeStreams];
    uint64_t slot_cap[kCodeStreams];
    const uint32_t* chunk_segs[kCodeStreams];    // copy-segment prefix (chunks + 1)
    const uint8_t* packed[kCodeStreams];         // fixed/tagged payload (bytes)
    uint64_t packed_dim_stride[kCodeStreams];    // fixed: bytes between dimension payloads
    const uint64_t* corr_dict;                   // distinct corrected values (bits)
    uint8_t input_dtype;
};

struct Writer {
    uint8_t* p;
    uint64_t pos;
    __device__ void u8(uint8_t v) { p[pos++] = v; }
    __device__ void uint(uint64_t v, int bytes) {
        for (int i = 0; i < bytes; ++i) p[pos++] = static_cast<uint8_t>(v >> (8 * i));
    }
    __device__ void f64(double d) {
        uint64_t u;
        memcpy(&u, &d, 8);
        uint(u, 8);
    }
    __device__ void raw(const char* s, int n) {
        for (int i = 0; i < n; ++i) p[pos++] = static_cast<uint8_t>(s[i]);
    }
};

// One CTA per rANS section: payload offsets and copy-segment prefix of its chunks.
__device__ void layout(EncState* st, const AssemblyIn& in, uint8_t* out, Piece* pieces, uint32_t max_pieces);

// The CTA that finishes last lays out the container (layout), so that the layout needs
// no launch of its own; with no rANS section the launch is that one CTA.
__global__ void __launch_bounds__(1024) k_chunk_prefix(ChunkMaps maps, EncState* st, AssemblyIn ain, uint8_t* out,
                                                       Piece* pieces, uint32_t max_pieces) {
    __shared__ uint64_t red[33];
    __shared__ bool s_last;
    if (static_cast<int>(blockIdx.x) < maps.nsec) {
    const int s = maps.sec_stream[blockIdx.x];
    const ChunkMap M = maps.m[s];
    uint64_t carry_b = 0, carry_s = 0;
    for (uint32_t base = 0; base < M.chunks; base += blockDim.x) {
        const uint32_t k = base + threadIdx.x;
        const uint64_t len = k < M.chunks ? M.len[k] : 0;
        const uint64_t nseg = (len + kCopySeg - 1) / kCopySeg;
        uint64_t tb, ts;
        const uint64_t eb = block_exclusive_sum(len, red, &tb);
        const uint64_t es = block_exclusive_sum(nseg, red, &ts);
        if (k < M.chunks) {
            M.off[k] = carry_b + eb;
            M.seg[k] = static_cast<uint32_t>(carry_s + es);
        }
        carry_b += tb;
        carry_s += ts;
    }
    if (threadIdx.x == 0) {
        M.seg[M.chunks] = static_cast<uint32_t>(carry_s);
        st->ch[s].payload_bytes = carry_b;
    }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(&st->done_a, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last || threadIdx.x != 0) return;
    __threadfence();
    layout(st, ain, out, pieces, max_pieces);
    st->done_a = 0;
}

// One thread: writes every header field and emits the list of payload pieces (payload
// sizes and copy-segment counts come from other CTAs of the same launch: read from L2).
__device__ void layout(EncState* st, const AssemblyIn& in, uint8_t* out, Piece* pieces, uint32_t max_pieces) {
    Writer w{out, 0};
    uint32_t np = 0;
    uint64_t segs = 0;
    auto piece = [&](const uint8_t* src, uint64_t len) {
        if (len == 0) return;
        if (np < max_pieces) pieces[np] = Piece{src, w.pos, len, segs, -1, 0};
        ++np;
        segs += (len + kCopySeg - 1) / kCopySeg;
        w.pos += len;
    };
    auto chunked = [&](int s, uint64_t len, uint32_t nseg) {
        if (len == 0) return;
        if (np < max_pieces) pieces[np] = Piece{nullptr, w.pos, len, segs, s, 0};
        ++np;
        segs += nseg;
        w.pos += len;
    };
    const uint32_t D = st->dims;
    w.raw("LCG2", 4);
    w.uint(kFormatVersion, 4);
    w.uint(D, 4);
    w.uint(st->n, 8);
    w.uint(st->p, 8);
    w.f64(st->eb);
    w.uint(static_cast<uint64_t>(st->wrap_min), 8);
    w.uint(static_cast<uint64_t>(st->wrap_max), 8);
    for (uint32_t d = 0; d < D; ++d) w.f64(st->mins[d]);
    w.u8(in.input_dtype);
    w.uint(kStreams, 4);
    // one component body; returns its length
    auto component = [&](int s) -> uint64_t {
        StreamChoice& c = st->ch[s];
        const uint64_t body0 = w.pos;
        w.u8(c.enc);
        w.uint(c.dims, 4);
        w.uint(c.records, 8);
        if (c.enc == kEncFixed) {
            for (uint32_t d = 0; d < c.dims; ++d) {
                w.uint(st->st[s].minv[d], 8);
                w.u8(c.width[d]);
            }
            for (uint32_t d = 0; d < c.dims; ++d)
                piece(in.packed[s] + in.packed_dim_stride[s] * d, (c.records * c.width[d] + 7) / 8);
        } else if (c.enc == kEncTagged || c.enc == kEncRaw) {
            if (c.enc == kEncTagged) w.u8(c.max_width);
            w.u8(static_cast<uint8_t>(c.sec_prec));
            w.uint(c.sec_alphabet, 4);
            w.uint(c.table_len, 4);
            piece(in.table_bytes + in.table_stride * s, c.table_len);
            w.uint(c.sec_S, 8);
            w.u8(static_cast<uint8_t>(c.sec_lanes));
            w.uint(c.sec_chunks, 4);
            const uint64_t payload = __ldcg(&c.payload_bytes);
            w.uint(payload, 8);
            piece(reinterpret_cast<const uint8_t*>(in.chunk_len[s]), 4ull * c.sec_chunks);
            piece(in.states[s], state_bytes(c.sec_lanes, c.sec_chunks, c.sec_prec));
            chunked(s, payload, __ldcg(&in.chunk_segs[s][c.sec_chunks]));
            if (c.enc == kEncTagged) {
                w.uint(c.packed_bits, 8);
                piece(in.packed[s], (c.packed_bits + 7) / 8);
            }
        }
        c.body_bytes = w.pos - body0;
        return c.body_bytes;
    };
    auto sized = [&](int s) {   // u64 length, then the body
        const uint64_t len_pos = w.pos;
        w.pos += 8;
        const uint64_t len = component(s);
        const uint64_t save = w.pos;
        w.pos = len_pos;
        w.uint(len, 8);
        w.pos = save;
    };
    for (int s = 0; s < kStreams; ++s) {
        char name[4];
        stream_name(s, name);
        w.raw(name, 4);
        sized(s);
    }
    w.raw("EXC0", 4);
    const uint64_t exc_len_pos = w.pos;
    w.pos += 8;
    const uint64_t exc0 = w.pos;
    w.uint(st->ncorr, 8);
    if (st->ncorr) {
        w.uint(st->ndistinct, 8);
        piece(reinterpret_cast<const uint8_t*>(in.corr_dict), 8 * st->ndistinct);
        sized(kCorrGaps);
        sized(kCorrIds);
    }
    {
        const uint64_t save = w.pos;
        w.pos = exc_len_pos;
        w.uint(save - exc0, 8);
        w.pos = save;
    }
    st->total_bytes = w.pos;
    st->npieces = np;
    st->nsegs = segs;
    if (np > max_pieces) set_error(&st->err, kErrInternal);
}

// Copies len bytes with the CTA: head bytes up to a 16-byte-aligned destination, then
// 16-byte stores, each assembled from aligned 4-byte source words with funnel shifts
// (any source alignment), then tail bytes.  Source words are read only where they hold
// at least one byte of the range.
__device__ __forceinline__ void block_copy(uint8_t* dst, const uint8_t* src, uint32_t len) {
    const uint32_t head = min(len, static_cast<uint32_t>((16 - (reinterpret_cast<uintptr_t>(dst) & 15)) & 15));
    if (threadIdx.x < head) dst[threadIdx.x] = src[threadIdx.x];
    const uint32_t body = (len - head) & ~15u;
    const uint8_t* s = src + head;
    uint8_t* d = dst + head;
    const uint32_t o = static_cast<uint32_t>(reinterpret_cast<uintptr_t>(s) & 3);
    if (o == 0 && (reinterpret_cast<uintptr_t>(s) & 15) == 0) {
        for (uint32_t i = 16 * threadIdx.x; i < body; i += 16 * blockDim.x)
            *reinterpret_cast<uint4*>(d + i) = *reinterpret_cast<const uint4*>(s + i);
    } else if (o == 0) {
        for (uint32_t i = 16 * threadIdx.x; i < body; i += 16 * blockDim.x) {
            const uint32_t* w = reinterpret_cast<const uint32_t*>(s + i);
            *reinterpret_cast<uint4*>(d + i) = make_uint4(w[0], w[1], w[2], w[3]);
        }
    } else {
        const uint32_t* sa = reinterpret_cast<const uint32_t*>(s - o);   // aligned word holding s[0]
        const uint32_t sh = 8 * o;
        for (uint32_t i = 16 * threadIdx.x; i < body; i += 16 * blockDim.x) {
            const uint32_t* w = sa + i / 4;
            // bytes s[i .. i+16) lie in words w[0..4]; w[4] holds s[i+16-o .. ], needed since o > 0
            const uint32_t w0 = w[0], w1 = w[1], w2 = w[2], w3 = w[3], w4 = w[4];
            *reinterpret_cast<uint4*>(d + i) = make_uint4(__funnelshift_r(w0, w1, sh), __funnelshift_r(w1, w2, sh),
                                                          __funnelshift_r(w2, w3, sh), __funnelshift_r(w3, w4, sh));
        }
    }
    for (uint32_t i = head + body + threadIdx.x; i < len; i += blockDim.x) dst[i] = src[i];
}

// Each CTA copies a contiguous run of 4 KB segments: the pieces (at most max_pieces)
// wait in shared memory, the run's first piece and, for a chunked piece, its first chunk
// are found by binary search, and later segments advance both linearly.
constexpr uint32_t kMaxPieces = 128;
__global__ void __launch_bounds__(256) k_copy_pieces(const Piece* pieces, ChunkMaps maps, const EncState* st,
                                                      uint8_t* out) {
    __shared__ Piece sp[kMaxPieces];
    const uint32_t np = min(st->npieces, kMaxPieces);
    const uint64_t nsegs = st->nsegs;
    for (uint32_t i = threadIdx.x; i < np; i += blockDim.x) sp[i] = pieces[i];
    __syncthreads();
    const uint64_t per = (nsegs + gridDim.x - 1) / gridDim.x;
    const uint64_t g0 = static_cast<uint64_t>(blockIdx.x) * per, g1 = min(nsegs, g0 + per);
    if (g0 >= g1) return;
    uint32_t lo = 0, hi = np - 1;   // last piece with seg_begin <= g0
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (sp[mid].seg_begin <= g0) lo = mid; else hi = mid - 1;
    }
    uint32_t chunk = 0xffffffffu;   // current chunk of a chunked piece (searched on entry)
    for (uint64_t g = g0; g < g1; ++g) {
        while (lo + 1 < np && sp[lo + 1].seg_begin <= g) {
            ++lo;
            chunk = 0xffffffffu;
        }
        const Piece& pc = sp[lo];
        const uint8_t* src;
        uint8_t* dst;
        uint64_t len;
        if (pc.stream < 0) {
            const uint64_t off = (g - pc.seg_begin) * kCopySeg;
            src = pc.src + off;
            dst = out + pc.dst + off;
            len = min(kCopySeg, pc.len - off);
        } else {
            const ChunkMap& M = maps.m[pc.stream];
            const uint32_t ls = static_cast<uint32_t>(g - pc.seg_begin);
            if (chunk == 0xffffffffu) {   // last chunk with seg[k] <= ls
                uint32_t a = 0, b = M.chunks - 1;
                while (a < b) {
                    const uint32_t mid = (a + b + 1) >> 1;
                    if (M.seg[mid] <= ls) a = mid; else b = mid - 1;
                }
                chunk = a;
            } else {
                while (chunk + 1 < M.chunks && M.seg[chunk + 1] <= ls) ++chunk;
            }
            const uint32_t a = chunk;
            const uint64_t clen = M.len[a];
            const uint64_t off = static_cast<uint64_t>(ls - M.seg[a]) * kCopySeg;
            src = M.slots + M.slot_cap * a + (M.slot_cap - clen) + off;
            dst = out + pc.dst + M.off[a] + off;
            len = min(kCopySeg, clen - off);
        }
        block_copy(dst, src, static_cast<uint32_t>(len));
    }
}

// Exact corrections as coded streams: index gaps (index_k - index_{k-1} - 1) and ids
// into the ascending list of distinct values.
__global__ void k_corr_gaps(const uint64_t* idx, uint64_t count, uint32_t* gaps) {
    for (uint64_t k = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; k < count;
         k += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        gaps[k] = static_cast<uint32_t>(idx[k] - (k ? idx[k - 1] + 1 : 0));
}
struct DictIn {
    const uint64_t* sorted_bits;
    __device__ uint32_t operator()(uint64_t k) const {
        return (k == 0 || sorted_bits[k] != sorted_bits[k - 1]) ? 1u : 0u;
    }
};
struct DictOut {
    const uint64_t* sorted_bits;
    const uint32_t* sorted_pos;
    uint64_t* dict;
    uint32_t* ids;
    __device__ void operator()(uint64_t k, uint32_t pre, uint32_t first) const {
        if (first) dict[pre] = sorted_bits[k];
        ids[sorted_pos[k]] = pre + first - 1;
    }
};

__global__ void k_gather_corrections(const uint32_t* perm, const uint64_t* idx_sorted_in, const double* val_in,
                                     uint64_t* idx_out, double* val_out, uint64_t count) {
    for (uint64_t k = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; k < count;
         k += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        idx_out[k] = idx_sorted_in[k];
        val_out[k] = val_in[perm[k]];
    }
}

// Resets the frame state and zeroes the value histograms (hist_words u32, grid-stride).
__global__ void __launch_bounds__(256) k_init_state(EncState* st, uint32_t dims, uint64_t n, double eb, uint64_t p,
                                                    int64_t threshold, uint32_t* hist, uint64_t hist_words) {
    uint4* h4 = reinterpret_cast<uint4*>(hist);   // 256-byte aligned, hist_words a multiple of 4
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < hist_words / 4;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        h4[i] = make_uint4(0, 0, 0, 0);
    if (threadIdx.x || blockIdx.x) return;
    st->err = 0;
    st->done_a = 0;
    st->done_b = 0;
    st->done_c = 0;
    st->dims = dims;
    st->n = n;
    st->eb = eb;
    st->p = p;
    st->threshold = threshold;
    for (int d = 0; d < kMaxDims; ++d) {
        st->minbits[d] = ~0ull;
        st->maxbits[d] = 0;
        st->zero_first[d][0] = st->zero_first[d][1] = ~0ull;
    }
    st->ncorr = 0;
    st->B = st->nkeep = st->ndiff = 0;
    st->rec_min = 0xffffffffu;
    st->rec_max = 0;
    st->rec_maxdiff = 0;
    st->ndistinct = 0;
    st->l1_links = 0;
    st->l1_link_bits = 0;
    st->l1_link_min = 0xffffffffu;
    st->l1_link_max = 0;
    for (int s = 0; s < kCodeStreams; ++s) {
        st->ch[s].enc = kEncEmpty;
        st->ch[s].records = 0;
        StreamStats& g = st->st[s];
        for (int d = 0; d < kMaxDims; ++d) { g.minv[d] = 0xffffffffu; g.maxv[d] = 0; }
        g.maxall = 0;
        g.maxtag = 0;
        g.tag_bits = 0;
        for (int t = 0; t < 34; ++t) g.tag_hist[t] = 0;
    }
    st->total_bytes = 0;
    st->npieces = 0;
}

// ------------------------------------------------------------------- host
static unsigned grid_for(uint64_t n, int threads = 256, unsigned cap = 148u * 16u) {
    uint64_t g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return static_cast<unsigned>(g);
}

static chain_status status_from_err(uint32_t err) {
    if (err & kErrNonFinite) return set_err(CHAIN_ERR_NONFINITE_INPUT, "LCPS coordinates must be finite");
    if (err & kErrQuantOverflow) return set_err(CHAIN_ERR_QUANT_OVERFLOW, "quantized coordinate does not fit int64");
    if (err & kErrUnsupported)
        return set_err(CHAIN_ERR_UNSUPPORTED,
                       "quantized coordinates need more than 31 bits or block keys more than 128 bits "
                       "(eb too small relative to the coordinate range for this build)");
    if (err & kErrCapacity) return set_err(CHAIN_ERR_OUT_OF_MEMORY, "device buffer capacity exceeded");
    return set_err(CHAIN_ERR_DEVICE, "internal encoder error (flags " + std::to_string(err) + ")");
}

// Statistics of CH20 without reading it: its values are 0 and 1 (record 0 is 0), B
// records of which st->ndiff are 1, so every field follows (the same values the
// counting kernel would accumulate from the stream's reset state).
__device__ void choice_stats(EncState* st, uint32_t* gh) {
    const uint64_t B = st->B, ones = st->ndiff;
    if (B == 0) return;
    StreamStats& g = st->st[3];
    g.minv[0] = ones == B ? 1u : 0u;
    g.maxv[0] = ones ? 1u : 0u;
    g.maxall = g.maxv[0];
    g.tag_hist[1] = static_cast<uint32_t>(B);   // tag max(1, bitlen(v)) = 1 for 0 and 1
    g.maxtag = 1;
    g.tag_bits = B;
    gh[0] = static_cast<uint32_t>(B - ones);
    gh[1] = static_cast<uint32_t>(ones);
}

// Statistics of streams s0 .. s0+count-1 (not IDR0, stream 0, whose statistics k_level1
// counts and k_tables completes): one launch for the one-dimensional streams and one for
// the D-dimensional ones (k_stream_stats_lanes for D <= 4, k_stream_stats above); CH20
// (stream 3) is derived from the level-2 counts inside the first of them.
static void launch_stats(const StreamRefs& refs, EncState* st, uint32_t* hist, uint64_t hist_stride, uint32_t dims,
                         uint64_t max_records, int s0, int count, cudaStream_t stream) {
    StreamSel one{}, many{};
    int n1 = 0, nd = 0, derive = 0;
    for (int s = s0; s < s0 + count; ++s) {
        if (s == 3) {
            derive = 1;
        } else if (refs.s[s].dims == 1) {
            one.s[n1++] = s;
        } else {
            many.s[nd++] = s;
        }
    }
    // streams of 1..4 dimensions: the lane-column kernel, its grid sized to the groups
    // the selected streams could hold (each CTA takes an even share of the actual ones)
    const auto lanes = [&](const StreamSel& sel, int ns, uint32_t dm) {
        bool wide = false;
        uint32_t mask = 0;
        for (int i = 0; i < ns; ++i) {
            wide |= refs.s[sel.s[i]].esz > 1;
            mask |= 1u << sel.s[i];
        }
        const uint64_t groups = static_cast<uint64_t>(ns) * ((max_records + 15) / 16);
        const unsigned g = static_cast<unsigned>(
            std::max<uint64_t>(1, std::min<uint64_t>(148ull * 4, (groups + kStatsThreads - 1) / kStatsThreads)));
        const size_t smem = wide ? kStatsWideBytes : kStatsLaneBytes;
        const int w = wide ? 1 : 0;
        // more than the default 48 KB of dynamic shared memory: a failed attribute call
        // fails the launch, which the caller's launch check reports
#define CHAIN_LANES(DM)                                                                                          \
    do {                                                                                                         \
        if (wide)                                                                                                \
            (void)cudaFuncSetAttribute(k_stream_stats_lanes<DM>, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                                       static_cast<int>(kStatsWideBytes));                                      \
        k_stream_stats_lanes<DM><<<g, kStatsThreads, smem, stream>>>(refs, st, hist, hist_stride, mask, derive, w); \
    } while (0)
        switch (dm) {
            case 1: CHAIN_LANES(1); break;
            case 2: CHAIN_LANES(2); break;
            case 3: CHAIN_LANES(3); break;
            default: CHAIN_LANES(4); break;
        }
#undef CHAIN_LANES
        count_launch();
        derive = 0;
    };
    if (n1) lanes(one, n1, 1);
    if (nd && dims <= 4) {
        lanes(many, nd, dims);
    } else if (nd) {   // more than four dimensions
        const unsigned g = grid_for((max_records + 3) / 4, 256, 148u * 4u);
        k_stream_stats<0><<<dim3(g, nd), 256, 0, stream>>>(refs, st, hist, hist_stride, many, derive); count_launch();
    }
}

// hist: the first sort pass's count table (nullptr: no sort follows).
template <typename FT, bool SOA, typename KT, typename RT>
static void launch_quantize(const void* pts, uint64_t n, uint32_t D, EncState* st, void* key, void* rel,
                            uint64_t* cidx, double* cval, uint64_t cap, uint32_t* hist, int hist_bits,
                            uint32_t* idrel, cudaStream_t s) {
    const uint32_t tiles = radix_tiles<KT>(n);
    const unsigned grid = std::max(1u, tiles);
    if (D == 3)
        k_quantize<FT, SOA, KT, 3, RT><<<grid, 256, 0, s>>>(static_cast<const FT*>(pts), n, D, st,
                                                            static_cast<KT*>(key), static_cast<RT*>(rel), cidx, cval,
                                                            cap, hist, hist_bits, tiles, idrel);
    else
        k_quantize<FT, SOA, KT, 0, RT><<<grid, 256, 0, s>>>(static_cast<const FT*>(pts), n, D, st,
                                                            static_cast<KT*>(key), static_cast<RT*>(rel), cidx, cval,
                                                            cap, hist, hist_bits, tiles, idrel);
    count_launch();
}

// The quantizer for a run-time input type, layout, key width and offset width.
template <typename FT, bool SOA>
static void launch_quantize_rt(size_t ksz, uint32_t rel_esz, const void* pts, uint64_t n, uint32_t D, EncState* st,
                               void* key, void* rel, uint64_t* cidx, double* cval, uint64_t cap, uint32_t* hist,
                               int hist_bits, uint32_t* idrel, cudaStream_t s) {
    if (ksz == 16) {
        if (rel_esz == 1) launch_quantize<FT, SOA, u128, uint8_t>(pts, n, D, st, key, rel, cidx, cval, cap, hist, hist_bits, idrel, s);
        else launch_quantize<FT, SOA, u128, uint32_t>(pts, n, D, st, key, rel, cidx, cval, cap, hist, hist_bits, idrel, s);
    } else if (ksz == 8) {
        if (rel_esz == 1) launch_quantize<FT, SOA, uint64_t, uint8_t>(pts, n, D, st, key, rel, cidx, cval, cap, hist, hist_bits, idrel, s);
        else launch_quantize<FT, SOA, uint64_t, uint32_t>(pts, n, D, st, key, rel, cidx, cval, cap, hist, hist_bits, idrel, s);
    } else {
        if (rel_esz == 1) launch_quantize<FT, SOA, uint32_t, uint8_t>(pts, n, D, st, key, rel, cidx, cval, cap, hist, hist_bits, idrel, s);
        else launch_quantize<FT, SOA, uint32_t, uint32_t>(pts, n, D, st, key, rel, cidx, cval, cap, hist, hist_bits, idrel, s);
    }
}

// Stable sort of the block keys (KT each, index order) and the level-1 links from the
// sorted neighbours.
template <typename KT, typename Hook>
static void sort_and_link(void* key_idx, void* key_a, void* key_b, uint32_t* val_a, uint32_t* val_b, uint64_t n,
                          int key_bits, uint32_t dims, uint32_t* counts, EncState* st, uint32_t* idrel, uint32_t* hist,
                          cudaStream_t stream, const Hook& marks) {
    KT* ka = static_cast<KT*>(key_a);
    KT* kb = static_cast<KT*>(key_b);
    const bool in_b = radix_sort_pairs<KT>(static_cast<const KT*>(key_idx), ka, val_a, kb, val_b, n, key_bits, counts,
                                           stream, marks, true);
    if (dims == 3)
        k_level1<KT, 3><<<grid_for(n), 256, 0, stream>>>(in_b ? kb : ka, in_b ? val_b : val_a, n, st, idrel, hist);
    else
        k_level1<KT, 0><<<grid_for(n), 256, 0, stream>>>(in_b ? kb : ka, in_b ? val_b : val_a, n, st, idrel, hist);
    count_launch();
}

// Explicit records (keys of the points with idrel == 0, index order) and level 2: record
// statistics, wrap parameters, choice2 with per-tile difference counts, and the keep /
// diff rows (kd_esz bytes per value).
template <typename KT>
static void run_level2(const KT* key_idx, const uint32_t* idrel, void* rec_v, uint64_t n, EncState* st, int l2, bool d3,
                       uint32_t kd_esz, uint8_t* choice2, void* keep, void* diff, uint32_t* scan32, StageTimer& T,
                       cudaStream_t stream) {
    KT* rec = static_cast<KT*>(rec_v);
    device_flag_gather(ExplicitIn<KT>{idrel}, key_idx, rec, n, scan32, &st->B, &st->done_a, stream);
    T.mark("explicit_records", stream);
    if (d3) {
        k_l2_stats<KT, 3><<<grid_for((n + 3) / 4, 256, 148u * 16u), 256, 0, stream>>>(rec, st); count_launch();
    } else {
        k_l2_stats<KT, 0><<<grid_for((n + 3) / 4, 256, 148u * 16u), 256, 0, stream>>>(rec, st); count_launch();
    }
    T.mark("l2_stats", stream);
    const unsigned tiles = static_cast<unsigned>(flag_tiles(n));
    if (d3) {
        k_l2_choice<KT, 3><<<tiles, 256, 0, stream>>>(rec, st, l2, choice2, scan32); count_launch();
    } else {
        k_l2_choice<KT, 0><<<tiles, 256, 0, stream>>>(rec, st, l2, choice2, scan32); count_launch();
    }
    T.mark("l2_choice", stream);
    // the flag scan of choice2 over tiles of n entries (entries j >= B are not records):
    // k_l2_choice left the tile prefixes
#define CHAIN_L2OUT(ET, DIM)                                                                                   \
    k_l2_rows<KT, ET, DIM><<<tiles, kFlagThreads, 0, stream>>>(rec, st, choice2, static_cast<ET*>(keep),       \
                                                               static_cast<ET*>(diff), scan32)
    if (d3) {
        if (kd_esz == 1) CHAIN_L2OUT(uint8_t, 3);
        else if (kd_esz == 2) CHAIN_L2OUT(uint16_t, 3);
        else CHAIN_L2OUT(uint32_t, 3);
    } else {
        if (kd_esz == 1) CHAIN_L2OUT(uint8_t, 0);
        else if (kd_esz == 2) CHAIN_L2OUT(uint16_t, 0);
        else CHAIN_L2OUT(uint32_t, 0);
    }
#undef CHAIN_L2OUT
    count_launch();
}

template <typename FT, bool SOA>
static void launch_minmax(const void* pts, uint64_t n, uint32_t D, EncState* st, cudaStream_t s) {
    dim3 g(grid_for(n, 256, 148u * 8u), D);
    k_minmax<FT, SOA><<<g, 256, 0, s>>>(static_cast<const FT*>(pts), n, D, st); count_launch();
}

// One attempt at a frame with room for corr_cap exact corrections.  When the frame has
// more, it returns CHAIN_ERR_OUT_OF_MEMORY with *corr_needed set to their count (the
// caller retries with that capacity).
// Creates the context's side stream (highest priority) and its fork/join events on first use.
static chain_status ensure_side_stream(chain_ctx* ctx) {
    if (!ctx->fork_ev) CHAIN_CUDA(cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming));
    if (!ctx->join_ev) CHAIN_CUDA(cudaEventCreateWithFlags(&ctx->join_ev, cudaEventDisableTiming));
    if (!ctx->side) {
        int least = 0, greatest = 0;
        CHAIN_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        CHAIN_CUDA(cudaStreamCreateWithPriority(&ctx->side, cudaStreamNonBlocking, greatest));
    }
    return CHAIN_OK;
}

// Orders the context's stream after the side stream's work when the encoder returns
// between the fork and the join (an error), so that nothing later on the context races
// with it.
struct SideJoin {
    chain_ctx* ctx = nullptr;
    ~SideJoin() {
        if (ctx) cudaStreamWaitEvent(ctx->stream, ctx->join_ev, 0);
    }
};

static chain_status encode_frame_cap(chain_ctx* ctx, const void* points, chain_dtype dtype, chain_layout layout,
                                     uint64_t n, uint32_t dims, double eb, int64_t p, int64_t threshold, int bl, int l1,
                                     int l2, uint32_t bytes_per_lane, uint32_t max_steps, uint64_t corr_cap,
                                     uint64_t* corr_needed, size_t* out_len) {
    cudaStream_t stream = ctx->stream;
    const size_t esz = dtype == CHAIN_F64 ? 8 : 4;
    const uint64_t nd = n * dims;
    const int64_t p_eff = bl ? p : 1;
    // block offsets are < p: one byte each when p <= 256
    const uint32_t rel_esz = p_eff <= 256 ? 1u : 4u;
    if (bytes_per_lane == 0) bytes_per_lane = 4096;
    if (max_steps == 0) max_steps = 1024;

    chain_status st_ = ensure_state(ctx, sizeof(EncState));
    if (st_ != CHAIN_OK) return st_;
    EncState* st = static_cast<EncState*>(ctx->state_dev);
    EncState* hs = static_cast<EncState*>(ctx->state_host);

    // ---- frame arena (sizes known from n, dims and the correction capacity)
    const uint64_t sort_counts = radix_counts_elems(std::max<uint64_t>(n, corr_cap));
    const uint64_t hist_stride = kRansMaxAlphabet;
    size_t need = 0;
    const bool host_input = !is_device_ptr(points);
    if (host_input) need += Arena::need(nd, esz);
    const uint64_t nsort = std::max<uint64_t>(n, corr_cap);
    need += Arena::need(nsort, 4) * 2;                      // sort values ping-pong (keys: ctx->keys)
    need += Arena::need(sort_counts, 4);
    need += Arena::need(scan_scratch_bytes(std::max<uint64_t>(sort_counts, nd)), 1);
    need += Arena::need(nd, 4) * 3;           // rel, keep, diff
    need += Arena::need(n, 4) * 2;            // idrel, choice2
    need += Arena::need(corr_cap, 8) * 4;     // corrections idx/val + sorted copies
    need += Arena::need(hist_stride * kCodeStreams, 4) * 3;  // hist, prob, cum
    need += Arena::need(64 * kCodeStreams, 4) * 2;
    need += Arena::need(corr_cap, 4) * 2 + Arena::need(corr_cap, 8);  // correction gaps, ids, values
    // serialised tables, and IDR0's encoder entries (written on the side stream before
    // the coding buffers are sized)
    const uint64_t table_stride = 4 * kRansMaxAlphabet + 64;
    need += Arena::need(table_stride * kCodeStreams, 1) + Arena::need(kRansMaxAlphabet + 1, 16);
    need += 64 * 256;
    CHAIN_CUDA(ctx->frame.reserve(need));
    Arena& A = ctx->frame;
    const void* pts = points;
    StageTimer& T = ctx->timer;
    T.begin(stream);
    if (host_input) {
        void* d = A.take<uint8_t>(nd * esz);
        CHAIN_CUDA(cudaMemcpyAsync(d, points, nd * esz, cudaMemcpyHostToDevice, stream));
        pts = d;
        T.mark("h2d_points", stream);
    }
    uint32_t* val_a = A.take<uint32_t>(nsort);
    uint32_t* val_b = A.take<uint32_t>(nsort);
    uint32_t* counts = A.take<uint32_t>(sort_counts);
    uint64_t* scanbuf = reinterpret_cast<uint64_t*>(A.take<uint8_t>(scan_scratch_bytes(std::max<uint64_t>(sort_counts, nd))));
    void* rel = A.take<uint8_t>(nd * rel_esz);
    void* keep = A.take<uint32_t>(nd);
    void* diff = A.take<uint32_t>(nd);
    uint32_t* idrel = A.take<uint32_t>(n);
    uint8_t* choice2 = A.take<uint8_t>(n);
    uint64_t* corr_idx = A.take<uint64_t>(corr_cap);
    double* corr_val = A.take<double>(corr_cap);
    uint64_t* corr_idx_s = A.take<uint64_t>(corr_cap);
    double* corr_val_s = A.take<double>(corr_cap);
    uint32_t* hist = A.take<uint32_t>(hist_stride * kCodeStreams);
    uint32_t* prob = A.take<uint32_t>(hist_stride * kCodeStreams);
    uint32_t* cum = A.take<uint32_t>(hist_stride * kCodeStreams);
    uint32_t* tag_prob = A.take<uint32_t>(64 * kCodeStreams);
    uint32_t* tag_cum = A.take<uint32_t>(64 * kCodeStreams);
    uint32_t* corr_gaps = A.take<uint32_t>(corr_cap);
    uint32_t* corr_ids = A.take<uint32_t>(corr_cap);
    uint64_t* corr_dict = A.take<uint64_t>(corr_cap);
    uint8_t* tables = A.take<uint8_t>(table_stride * kCodeStreams);
    uint4* etab0 = A.take<uint4>(kRansMaxAlphabet + 1);
    if (!tag_cum || !etab0) return set_err(CHAIN_ERR_OUT_OF_MEMORY, "encoder frame arena too small");

    static_assert((kRansMaxAlphabet * kCodeStreams) % 4 == 0, "histograms zeroed in 16-byte words");
    k_init_state<<<148, 256, 0, stream>>>(st, dims, n, eb, static_cast<uint64_t>(p_eff), threshold, hist,
                                          hist_stride * kCodeStreams); count_launch();

    // ---- phase 1: extrema and quantization parameters
    const bool soa = layout == CHAIN_SOA;
    if (dtype == CHAIN_F32) soa ? launch_minmax<float, true>(pts, n, dims, st, stream)
                            : launch_minmax<float, false>(pts, n, dims, st, stream);
    else soa ? launch_minmax<double, true>(pts, n, dims, st, stream)
             : launch_minmax<double, false>(pts, n, dims, st, stream);
    CHAIN_LAUNCH_CHECK("encoder phase 1");
    T.mark("extrema", stream);
    CHAIN_CUDA(cudaMemcpyAsync(hs, st, sizeof(EncState), cudaMemcpyDeviceToHost, stream));
    CHAIN_CUDA(cudaStreamSynchronize(stream));
    T.mark("sync1", stream);
    if (hs->err) return status_from_err(hs->err);
    const int key_bits = hs->key_bits;
    const bool wide = key_bits > 32;
    // block keys of 4, 8 or 16 bytes: the index-order keys, the sort's ping-pong keys
    // (which the exact-correction sort reuses with 8-byte keys) and the record keys
    const size_t ksz = key_bits > 64 ? 16 : (key_bits > 32 ? 8 : 4);
    const uint64_t kab = std::max<uint64_t>(n * ksz, corr_cap * 8);
    CHAIN_CUDA(ctx->keys.reserve(Arena::need(n * ksz, 1) * 2 + Arena::need(kab, 1) * 2));
    uint8_t* key_idx = ctx->keys.take<uint8_t>(n * ksz);
    uint8_t* key_a = ctx->keys.take<uint8_t>(kab);
    uint8_t* key_b = ctx->keys.take<uint8_t>(kab);
    uint8_t* rec = ctx->keys.take<uint8_t>(n * ksz);
    if (!rec) return set_err(CHAIN_ERR_OUT_OF_MEMORY, "encoder key arena too small");
    // keep rows hold block coordinates (< 2^kb), diff rows ZigZag'd wrapped differences
    // (<= the record range <= 2^kb): the narrowest width that holds kb + 1 bits
    const uint32_t kd_esz = hs->kb + 1 <= 8 ? 1u : (hs->kb + 1 <= 16 ? 2u : 4u);

    // ---- phase 2: quantize, sort, level 1, level 2, statistics, plan
    // the quantizer counts the first sort pass's digits (when a sort follows)
    const RadixPlan plan = radix_plan(key_bits, static_cast<int>(ksz));
    uint32_t* hist0 = l1 ? counts : nullptr;
#define CHAIN_Q(FT, SOA_) launch_quantize_rt<FT, SOA_>(ksz, rel_esz, pts, n, dims, st, key_idx, rel, corr_idx, corr_val, corr_cap, hist0, plan.bits, idrel, stream)
    if (dtype == CHAIN_F32) {
        if (soa) CHAIN_Q(float, true); else CHAIN_Q(float, false);
    } else {
        if (soa) CHAIN_Q(double, true); else CHAIN_Q(double, false);
    }
#undef CHAIN_Q
    CHAIN_LAUNCH_CHECK("quantize");
    T.mark("quantize", stream);

    if (l1) {   // idrel was zeroed by the quantizer; k_level1 writes the links only
        // stage marks around every scatter pass; the key width is in the name
        const auto sort_marks = [&](bool after) {
            T.mark(after ? (ksz == 16 ? "sort_scatter_k128" : (wide ? "sort_scatter_k64" : "sort_scatter_k32"))
                         : "sort_hist_scan",
                   stream);
        };
        if (ksz == 16)
            sort_and_link<u128>(key_idx, key_a, key_b, val_a, val_b, n, key_bits, dims, counts, st, idrel, hist, stream, sort_marks);
        else if (ksz == 8)
            sort_and_link<uint64_t>(key_idx, key_a, key_b, val_a, val_b, n, key_bits, dims, counts, st, idrel, hist, stream,
                                    sort_marks);
        else
            sort_and_link<uint32_t>(key_idx, key_a, key_b, val_a, val_b, n, key_bits, dims, counts, st, idrel, hist, stream,
                                    sort_marks);
    }
    CHAIN_LAUNCH_CHECK("level 1");
    T.mark("level1", stream);
    // IDR0's statistics are complete after level 1, so its tables and plan are built on
    // the side stream while level 2 and the other streams' statistics run on this one
    st_ = ensure_side_stream(ctx);
    if (st_ != CHAIN_OK) return st_;
    // per device, cheap; set on every call, always to the same value
    CHAIN_CUDA(cudaFuncSetAttribute(k_tables, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(kTableStageBytes)));
    StreamRefs idr{};
    idr.s[0] = StreamRef{idrel, 1, 4, nullptr, nullptr, n};
    CHAIN_CUDA(cudaEventRecord(ctx->fork_ev, stream));
    CHAIN_CUDA(cudaStreamWaitEvent(ctx->side, ctx->fork_ev, 0));
    k_tables<<<dim3(1, 2), kTableThreads, kTableStageBytes, ctx->side>>>(idr, st, hist, hist_stride, prob, cum, tag_prob,
                                                                         tag_cum, 0, bytes_per_lane, max_steps,
                                                                         &st->done_c, tables, table_stride, etab0);
    count_launch();
    CHAIN_CUDA(cudaEventRecord(ctx->join_ev, ctx->side));
    SideJoin join{ctx};
    CHAIN_LAUNCH_CHECK("IDR0 tables");
    uint32_t* scan32 = reinterpret_cast<uint32_t*>(scanbuf);
    const bool d3 = dims == 3 && hs->kb <= 21;
    if (ksz == 16)
        run_level2<u128>(reinterpret_cast<const u128*>(key_idx), idrel, rec, n, st, l2, d3, kd_esz, choice2, keep, diff,
                         scan32, T, stream);
    else if (ksz == 8)
        run_level2<uint64_t>(reinterpret_cast<const uint64_t*>(key_idx), idrel, rec, n, st, l2, d3, kd_esz, choice2, keep,
                             diff, scan32, T, stream);
    else
        run_level2<uint32_t>(reinterpret_cast<const uint32_t*>(key_idx), idrel, rec, n, st, l2, d3, kd_esz, choice2, keep,
                             diff, scan32, T, stream);
    CHAIN_LAUNCH_CHECK("level 2");
    T.mark("l2_rows", stream);
    // The level-2 scan covers n >= B entries; its functors ignore entries j >= B (read
    // from the device), so no host round trip is needed for B.

    StreamRefs refs;
    refs.s[0] = StreamRef{idrel, 1, 4, nullptr, nullptr, n};
    refs.s[1] = StreamRef{diff, dims, kd_esz, &st->ndiff, nullptr, 0};
    refs.s[2] = StreamRef{keep, dims, kd_esz, &st->B, &st->ndiff, 0};   // B - ndiff kept records
    refs.s[3] = StreamRef{choice2, 1, 1, &st->B, nullptr, 0};
    refs.s[4] = StreamRef{rel, dims, rel_esz, nullptr, nullptr, n};
    refs.s[kCorrGaps] = StreamRef{corr_gaps, 1, 4, nullptr, nullptr, 0};
    refs.s[kCorrIds] = StreamRef{corr_ids, 1, 4, nullptr, nullptr, 0};
    launch_stats(refs, st, hist, hist_stride, dims, n, 1, kStreams - 1, stream);
    T.mark("stats", stream);
    CHAIN_CUDA(cudaStreamWaitEvent(stream, ctx->join_ev, 0));   // IDR0's tables and plan
    join.ctx = nullptr;
    k_tables<<<dim3(kStreams - 1, 2), kTableThreads, kTableStageBytes, stream>>>(refs, st, hist, hist_stride, prob, cum,
                                                                                   tag_prob, tag_cum, 1, bytes_per_lane,
                                                                                   max_steps, &st->done_b, nullptr, 0,
                                                                                   nullptr); count_launch();
    CHAIN_LAUNCH_CHECK("plan");
    T.mark("tables+plan", stream);
    CHAIN_CUDA(cudaMemcpyAsync(hs, st, sizeof(EncState), cudaMemcpyDeviceToHost, stream));
    CHAIN_CUDA(cudaStreamSynchronize(stream));
    T.mark("sync2", stream);
    if (hs->err) return status_from_err(hs->err);
    if (hs->ncorr > corr_cap) {
        *corr_needed = hs->ncorr;
        return set_err(CHAIN_ERR_OUT_OF_MEMORY, "more exact corrections than buffered");
    }

    // ---- exact corrections: increasing index order, then gaps + value-id streams
    if (hs->ncorr) {
        if (nd > 0xffffffffull)
            return set_err(CHAIN_ERR_UNSUPPORTED, "exact corrections need n * dims < 2^32 in this build");
        const uint64_t nc = hs->ncorr;
        const int bits = std::max(1, bitlen64(nd - 1));
        uint32_t* scan32b = reinterpret_cast<uint32_t*>(scanbuf);
        uint64_t* ca = reinterpret_cast<uint64_t*>(key_a);   // room for corr_cap 8-byte keys
        uint64_t* cb = reinterpret_cast<uint64_t*>(key_b);
        // flat indices are unique, and equal values need no order for the dictionary,
        // so the small unstable sort serves both sorts here
        bool in_b = sort_pairs<uint64_t>(corr_idx, ca, val_a, cb, val_b, nc, bits, counts, stream);
        k_gather_corrections<<<grid_for(nc), 256, 0, stream>>>(in_b ? val_b : val_a, in_b ? cb : ca, corr_val,
                                                               corr_idx_s, corr_val_s, nc); count_launch();
        k_corr_gaps<<<grid_for(nc), 256, 0, stream>>>(corr_idx_s, nc, corr_gaps); count_launch();
        const uint64_t* vbits = reinterpret_cast<const uint64_t*>(corr_val_s);
        in_b = sort_pairs<uint64_t>(vbits, ca, val_a, cb, val_b, nc, 64, counts, stream);
        device_exclusive_scan<uint32_t>(DictIn{in_b ? cb : ca},
                                        DictOut{in_b ? cb : ca, in_b ? val_b : val_a, corr_dict, corr_ids}, nc,
                                        scan32b, &st->ndistinct, stream);
        refs.s[kCorrGaps].count_const = nc;
        refs.s[kCorrIds].count_const = nc;
        const unsigned g = grid_for(nc, 256, 148u * 4u);
        launch_stats(refs, st, hist, hist_stride, dims, nc, kCorrGaps, 2, stream);
        k_tables<<<dim3(2, 2), kTableThreads, kTableStageBytes, stream>>>(refs, st, hist, hist_stride, prob, cum,
                                                                         tag_prob, tag_cum, kCorrGaps, bytes_per_lane,
                                                                         max_steps, &st->done_b, nullptr, 0, nullptr);
        count_launch();
        CHAIN_LAUNCH_CHECK("corrections");
        CHAIN_CUDA(cudaMemcpyAsync(hs, st, sizeof(EncState), cudaMemcpyDeviceToHost, stream));
        CHAIN_CUDA(cudaStreamSynchronize(stream));
        if (hs->err) return status_from_err(hs->err);
        T.mark("corrections", stream);
    }

    // ---- phase 3: coding buffers
    uint64_t slots_total = 0, packed_total = 0, tags_total = 0, total_chunks = 0;
    uint64_t slot_cap[kCodeStreams] = {0}, slot_off[kCodeStreams] = {0}, packed_off[kCodeStreams] = {0},
             packed_stride[kCodeStreams] = {0}, tags_off[kCodeStreams] = {0};
    for (int s = 0; s < kCodeStreams; ++s) {
        const StreamChoice& c = hs->ch[s];
        if (c.enc == kEncRaw || c.enc == kEncTagged) {
            slot_cap[s] = ((3 * c.sec_S + 64) + 15) & ~15ull;
            slot_off[s] = slots_total;
            slots_total += slot_cap[s] * c.sec_chunks;
            total_chunks += c.sec_chunks;
        }
        if (c.enc == kEncFixed) {
            uint64_t maxw = 0;
            for (uint32_t d = 0; d < c.dims; ++d) maxw = std::max<uint64_t>(maxw, c.width[d]);
            packed_stride[s] = ((c.records * maxw + 31) / 32 + 1) * 4;
            packed_off[s] = packed_total;
            packed_total += packed_stride[s] * c.dims;
        }
        if (c.enc == kEncTagged) {
            packed_off[s] = packed_total;
            packed_total += ((c.packed_bits + 31) / 32 + 2) * 4;
            tags_off[s] = tags_total;
            tags_total += c.records;
        }
    }
    uint64_t etab_total = 0;   // IDR0's entries are in etab0
    for (int s = 1; s < kCodeStreams; ++s)
        if (hs->ch[s].enc == kEncRaw || hs->ch[s].enc == kEncTagged) etab_total += hs->ch[s].sec_alphabet;
    const uint64_t max_pieces = kMaxPieces;
    uint64_t bound = header_bytes(dims) + 40 + 8ull * hs->ndistinct;
    for (int s = 0; s < kCodeStreams; ++s) {
        const StreamChoice& c = hs->ch[s];
        bound += 12 + 13 + 1 + 9ull * c.dims;
        if (c.enc == kEncFixed) bound += packed_stride[s] * c.dims;
        if (c.enc == kEncRaw || c.enc == kEncTagged)
            bound += 64 + 3ull * kRansMaxAlphabet + 132ull * c.sec_chunks + slot_cap[s] * c.sec_chunks;
        if (c.enc == kEncTagged) bound += 8 + (c.packed_bits + 7) / 8;
    }
    size_t need2 = Arena::need(slots_total, 1) + Arena::need(packed_total, 1) + Arena::need(tags_total + 1, 4) +
                   Arena::need(total_chunks + 1, 4) + Arena::need(total_chunks * 32 + 1, 4) * 2 +
                   Arena::need(max_pieces, sizeof(Piece)) +
                   Arena::need(bound, 1) + Arena::need(etab_total + 1, 16) + Arena::need(total_chunks + 1, 8) +
                   Arena::need(total_chunks + kCodeStreams + 1, 4) + 11 * 256;
    CHAIN_CUDA(ctx->coded.reserve(need2));
    Arena& C = ctx->coded;
    uint8_t* slots = C.take<uint8_t>(slots_total + 1);
    // the packed bit streams and the packed final lane states (128 bytes per chunk) are
    // OR-ed into: one zeroing covers both
    uint8_t* packed = C.take<uint8_t>(packed_total + 1);
    uint32_t* packed_states = C.take<uint32_t>(total_chunks * 32 + 1);
    uint32_t* tags = C.take<uint32_t>(tags_total + 1);
    uint32_t* chunk_len = C.take<uint32_t>(total_chunks + 1);
    Piece* pieces = C.take<Piece>(max_pieces);
    uint8_t* container = C.take<uint8_t>(bound);
    uint4* etab = C.take<uint4>(etab_total + 1);
    uint64_t* chunk_off = C.take<uint64_t>(total_chunks + 1);
    uint32_t* chunk_seg = C.take<uint32_t>(total_chunks + kCodeStreams + 1);
    if (!container || !etab || !chunk_seg) return set_err(CHAIN_ERR_OUT_OF_MEMORY, "encoder coding arena too small");
    ChunkMaps maps{};
    uint64_t seg_base = 0;
    uint64_t etab_used = 0;
    if (packed_states) {
        const size_t zero_bytes = reinterpret_cast<uint8_t*>(packed_states + total_chunks * 32 + 1) - packed;
        CHAIN_CUDA(cudaMemsetAsync(packed, 0, zero_bytes, stream));
    }

    FixedJobs fixed;
    StreamJobs stream_jobs;
    for (int s = 0; s < kCodeStreams; ++s) stream_jobs.job[s] = -1;
    unsigned nfixed = 0;
    uint64_t fixed_tiles = 0;
    RansJobs jobs{};
    jobs.njobs = 0;
    uint32_t first = 0;
    AssemblyIn ain{};
    ain.table_bytes = tables;
    ain.table_stride = table_stride;
    ain.corr_dict = corr_dict;
    ain.input_dtype = static_cast<uint8_t>(esz);
    uint64_t chunk_base = 0;
    for (int s = 0; s < kCodeStreams; ++s) {
        const StreamChoice& c = hs->ch[s];
        const StreamRef& r = refs.s[s];
        if (c.enc == kEncFixed) {
            FixedJob& fj = fixed.job[nfixed++];
            fj.fp = FixedPack{};
            for (uint32_t d = 0; d < c.dims; ++d) {
                fj.fp.words[d] = reinterpret_cast<uint32_t*>(packed + packed_off[s] + packed_stride[s] * d);
                fj.fp.nwords[d] = (c.records * c.width[d] + 31) / 32;
                fj.fp.minv[d] = hs->st[s].minv[d];
                fj.fp.width[d] = c.width[d];
            }
            fj.data = r.data;
            fj.nrec = c.records;
            fj.dims = c.dims;
            fj.esz = r.esz;
            fj.equal_w = 0;
            if (r.esz == 1 && c.dims <= 4) {
                const uint32_t w0 = c.width[0];
                bool eq = w0 == 1 || w0 == 2 || w0 == 4 || w0 == 8;
                for (uint32_t d = 1; d < c.dims; ++d) eq = eq && c.width[d] == w0;
                if (eq) fj.equal_w = w0;
            }
            fixed_tiles = std::max<uint64_t>(fixed_tiles, (c.records + 1023) / 1024);
            ain.packed[s] = packed + packed_off[s];
            ain.packed_dim_stride[s] = packed_stride[s];
        }
        const void* symbols = r.data;
        uint32_t sym_esz = r.esz;
        if (c.enc == kEncTagged) {
            uint32_t* tg = tags + tags_off[s];
            uint32_t* words = reinterpret_cast<uint32_t*>(packed + packed_off[s]);
            if (r.esz == 1) {
                const uint8_t* d8 = static_cast<const uint8_t*>(r.data);
                k_tags<uint8_t><<<grid_for(c.records), 256, 0, stream>>>(d8, c.dims, c.records, tg); count_launch();
                device_exclusive_scan<uint64_t>(TagBitsIn{tg, c.dims}, TagPackOut<uint8_t>{d8, tg, c.dims, words},
                                                c.records, scanbuf, static_cast<uint64_t*>(nullptr), stream);
            } else if (r.esz == 2) {
                const uint16_t* d16 = static_cast<const uint16_t*>(r.data);
                k_tags<uint16_t><<<grid_for(c.records), 256, 0, stream>>>(d16, c.dims, c.records, tg); count_launch();
                device_exclusive_scan<uint64_t>(TagBitsIn{tg, c.dims}, TagPackOut<uint16_t>{d16, tg, c.dims, words},
                                                c.records, scanbuf, static_cast<uint64_t*>(nullptr), stream);
            } else {
                const uint32_t* d32 = static_cast<const uint32_t*>(r.data);
                k_tags<uint32_t><<<grid_for(c.records), 256, 0, stream>>>(d32, c.dims, c.records, tg); count_launch();
                device_exclusive_scan<uint64_t>(TagBitsIn{tg, c.dims}, TagPackOut<uint32_t>{d32, tg, c.dims, words},
                                                c.records, scanbuf, static_cast<uint64_t*>(nullptr), stream);
            }
            const uint64_t nwords = (c.packed_bits + 31) / 32;
            k_words_to_bytes<<<grid_for(nwords), 256, 0, stream>>>(words, nwords); count_launch();
            ain.packed[s] = packed + packed_off[s];
            symbols = tg;
            sym_esz = 4;
        }
        if (c.enc == kEncRaw || c.enc == kEncTagged) {
            stream_jobs.job[s] = static_cast<int>(jobs.njobs);
            RansJob& jb = jobs.job[jobs.njobs++];
            jb.sym = symbols;
            jb.sym_esz = sym_esz;
            jb.count = c.sec_count;
            jb.prob = c.enc == kEncRaw ? prob + hist_stride * s : tag_prob + 64 * s;
            jb.cum = c.enc == kEncRaw ? cum + hist_stride * s : tag_cum + 64 * s;
            jb.prec = c.sec_prec;
            jb.alphabet = c.sec_alphabet;
            if (s == 0) {
                jb.etab = etab0;   // written with IDR0's table on the side stream
            } else {
                jb.etab = etab + etab_used;
                etab_used += c.sec_alphabet;
            }
            jb.chunks = c.sec_chunks;
            jb.lanes = c.sec_lanes;
            jb.S = c.sec_S;
            jb.bytes = slots + slot_off[s];
            jb.slot_cap = slot_cap[s];
            jb.chunk_len = chunk_len + chunk_base;
            jb.states = packed_states + chunk_base * 32;
            jb.first_block = first;
            first += (c.sec_chunks + kRansEncWarps - 1) / kRansEncWarps;
            ain.chunk_len[s] = jb.chunk_len;
            ain.states[s] = reinterpret_cast<const uint8_t*>(packed_states + chunk_base * 32);
            ain.slots[s] = jb.bytes;
            ain.slot_cap[s] = slot_cap[s];
            ChunkMap& cm = maps.m[s];
            cm.slots = jb.bytes;
            cm.slot_cap = slot_cap[s];
            cm.len = jb.chunk_len;
            cm.off = chunk_off + chunk_base;
            cm.seg = chunk_seg + seg_base;
            cm.chunks = c.sec_chunks;
            ain.chunk_segs[s] = cm.seg;
            maps.sec_stream[maps.nsec++] = s;
            seg_base += c.sec_chunks + 1;
            chunk_base += c.sec_chunks;
        }
    }
    jobs.total_blocks = first;
    if (nfixed) {
        k_pack_fixed<<<dim3(grid_for(fixed_tiles, kPackWarps, 148u * 16u), nfixed), 32 * kPackWarps, 0, stream>>>(fixed);
        count_launch();
    }
    T.mark("corrections+packing", stream);
    CHAIN_CUDA(cudaFuncSetAttribute(k_serialize_tables, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(4 * kSerStageSyms)));
    // streams 1..: IDR0's table and entries came with its plan on the side stream
    k_serialize_tables<<<dim3(kCodeStreams - 1, 1 + kEtabSlices), 1024, 4 * kSerStageSyms, stream>>>(
        st, prob, tag_prob, hist_stride, tables, table_stride, 1, jobs, stream_jobs); count_launch();
    T.mark("serialize_tables", stream);
    if (jobs.total_blocks) {
        rans_plan_smem(jobs, false);
        if (rans_enc_smem(jobs) > kRansEncSmemMax)
            return set_err(CHAIN_ERR_DEVICE, "internal: rANS encoder shared memory above its fixed maximum");
        {  // per device, cheap; set on every call, always to the same values
            CHAIN_CUDA(cudaFuncSetAttribute(rans_encode_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                            cudaSharedmemCarveoutMaxShared));
            CHAIN_CUDA(cudaFuncSetAttribute(rans_encode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            static_cast<int>(kRansEncSmemMax)));
        }
        rans_encode_kernel<<<jobs.total_blocks, 32 * kRansEncWarps, rans_enc_smem(jobs), stream>>>(jobs, &st->err); count_launch();
    }
    CHAIN_LAUNCH_CHECK("entropy coding");
    T.mark("rans_encode", stream);
    k_chunk_prefix<<<std::max(1, maps.nsec), 1024, 0, stream>>>(maps, st, ain, container, pieces,
                                                             static_cast<uint32_t>(max_pieces)); count_launch();
    k_copy_pieces<<<148u * 16u, 256, 0, stream>>>(pieces, maps, st, container); count_launch();
    CHAIN_LAUNCH_CHECK("assembly");
    T.mark("assemble", stream);
    CHAIN_CUDA(cudaMemcpyAsync(hs, st, sizeof(EncState), cudaMemcpyDeviceToHost, stream));
    CHAIN_CUDA(cudaStreamSynchronize(stream));
    T.mark("sync3", stream);
    CHAIN_CUDA(cudaStreamSynchronize(stream));
    T.finish();
    if (hs->err) return status_from_err(hs->err);
    if (hs->total_bytes > bound) return set_err(CHAIN_ERR_DEVICE, "container exceeds its bound");
    ctx->result = container;
    ctx->result_len = hs->total_bytes;
    ctx->dbg = EncodeDebug{idrel, diff, keep, kd_esz, choice2, rel, rel_esz, n, hs->ndiff, hs->B - hs->ndiff, hs->B, dims};
    *out_len = hs->total_bytes;
    return CHAIN_OK;
}

// Encodes a frame.  Exact corrections are buffered for up to min(n * dims, 2^20) values
// on the first attempt; a frame with more (clipped or tightly bounded data) is encoded
// again with room for exactly as many as the first attempt counted.
chain_status encode_frame(chain_ctx* ctx, const void* points, chain_dtype dtype, chain_layout layout, uint64_t n,
                          uint32_t dims, double eb, int64_t p, int64_t threshold, int bl, int l1, int l2,
                          uint32_t bytes_per_lane, uint32_t max_steps, size_t* out_len) {
    uint64_t cap = std::min<uint64_t>(n * dims, 1ull << 20);
    uint64_t needed = 0;
    chain_status s = encode_frame_cap(ctx, points, dtype, layout, n, dims, eb, p, threshold, bl, l1, l2, bytes_per_lane,
                                      max_steps, cap, &needed, out_len);
    if (s == CHAIN_ERR_OUT_OF_MEMORY && needed > cap) {
        cap = needed;
        needed = 0;
        s = encode_frame_cap(ctx, points, dtype, layout, n, dims, eb, p, threshold, bl, l1, l2, bytes_per_lane,
                             max_steps, cap, &needed, out_len);
        if (s == CHAIN_ERR_OUT_OF_MEMORY && needed > cap)
            return set_err(CHAIN_ERR_DEVICE, "internal: exact-correction count changed between two passes");
    }
    return s;
}

}  // namespace chain
