// Chain decoder on sm_100a: interleaved-rANS decode, bit unpacking, the level-2
// inverse as a modular reset-scan, the level-1 inverse by pointer jumping to each
// chain's explicit block, FP64 reconstruction and exact corrections.
//
// Semantics follow the reference CPU decoder (cpp/chain/lcps_cpp.cpp:1833-1995, also
// cpp/decompress/lcps_cpu_decompress_serial.cpp:1182-1326), including its validation:
// every malformed value sets an error bit instead of being trusted.
//   level-2 inverse      lcps_cpp.cpp:1890-1934
//   level-1 inverse      lcps_cpp.cpp:1936-1961 (backward pass; here: roots by jumping)
//   reconstruction       lcps_cpp.cpp:1963-1993 (fma(q + 0.5, 2 eb, min), corrections)
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <vector>

#include "chain_common.cuh"
#include "chain_format.h"
#include "ctx.h"
#include "rans.cuh"
#include "scan.cuh"

namespace chain {

struct DecState {
    uint32_t err;
    uint32_t done;          // hand-off counter of last-CTA scans (zero between them)
    uint32_t zeros;         // idrel == 0 count
    uint32_t ndiff_seen;
    uint64_t tag_bits[kCodeStreams];
    uint32_t maxtag[kCodeStreams];
    DecodePlan plan;
};

__device__ void dec_init(DecState* st) {
    st->err = 0;
    st->done = 0;
    st->zeros = 0;
    st->ndiff_seen = 0;
    for (int s = 0; s < kCodeStreams; ++s) { st->tag_bits[s] = 0; st->maxtag[s] = 0; }
}

__global__ void k_dec_init(DecState* st) {
    if (threadIdx.x || blockIdx.x) return;
    dec_init(st);
}

// Resets the state and parses a device-resident container (one thread).
__global__ void k_parse(const uint8_t* data, uint64_t len, DecState* st) {
    if (threadIdx.x || blockIdx.x) return;
    dec_init(st);
    parse_container(data, len, &st->plan);
}

// Per rANS section: token table -> prob/cum, and chunk byte offsets.  One CTA each.
struct SectionRef {
    const SectionPlan* sec;   // device pointer into the plan
    uint32_t* scratch;        // table-parse scratch: 8 * (table_len / 64 + 2) u32
    uint32_t* prob;
    uint32_t* cum;
    uint8_t* image;     // the rANS decoder's shared-memory tables (dec_image_bytes), or null
    uint64_t* slots;    // packed slot entries when the section has no image, or null
    uint64_t* chunk_off;
    uint64_t states_first;   // the section's first entry in the decoder's lane-state array
};
struct SectionRefs {
    SectionRef r[kCodeStreams];
    int count;
};

__global__ void __launch_bounds__(1024) k_section_setup(SectionRefs refs, const uint8_t* data, DecState* st) {
    const SectionRef R = refs.r[blockIdx.x];
    const SectionPlan& s = *R.sec;
    __shared__ uint64_t red[33];
    extern __shared__ __align__(16) uint8_t setup_smem[];   // kParseSmem bytes
    uint8_t* stage = setup_smem;
    uint32_t* stage_scratch = reinterpret_cast<uint32_t*>(setup_smem + kParseStage);
    uint32_t* sprob = reinterpret_cast<uint32_t*>(setup_smem + kParseStage + 4 * kParseStageScratch);
    if (!parse_table_block(data + s.table_off, s.table_len, s.alphabet, s.prec, R.prob, R.cum, R.scratch, stage,
                           stage_scratch, sprob) &&
        threadIdx.x == 0)
        set_error(&st->err, kErrCorrupt);
    // chunk offsets: exclusive prefix of the u32 chunk lengths
    uint64_t carry = s.payload_off;
    for (uint32_t base = 0; base < s.chunks; base += blockDim.x) {
        const uint32_t c = base + threadIdx.x;
        uint64_t len = 0;
        if (c < s.chunks) {
            const uint8_t* q = data + s.chunk_tab_off + 4ull * c;
            len = static_cast<uint64_t>(q[0]) | (static_cast<uint64_t>(q[1]) << 8) | (static_cast<uint64_t>(q[2]) << 16) |
                  (static_cast<uint64_t>(q[3]) << 24);
        }
        uint64_t tot;
        const uint64_t ex = block_exclusive_sum(len, red, &tot);
        if (c < s.chunks) R.chunk_off[c] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) {
        R.chunk_off[s.chunks] = carry;
        if (carry != s.payload_off + s.payload_len) set_error(&st->err, kErrCorrupt);
    }
}

// The rANS decoder's tables of section R: its shared-memory image (layout at
// dec_image_bytes), or the packed global slot entries.  A slot's owner is found by
// binary search of the cumulative table.  Blocks bx of nbx cover the section.
__device__ void section_lookup(const SectionRef& R, uint32_t bx, uint32_t nbx) {
    const SectionPlan& s = *R.sec;
    const uint32_t M = 1u << s.prec, A = s.alphabet;
    const bool bucketed = rans_dec_bucketed(s.prec, A);
    const bool smem_look = rans_dec_smem_look(s.prec, A);
    const uint32_t tid = bx * blockDim.x + threadIdx.x, nthreads = nbx * blockDim.x;
    uint16_t* owners = nullptr;
    if (bucketed) {
        uint32_t* cum = reinterpret_cast<uint32_t*>(R.image);
        for (uint32_t i = tid; i <= A; i += nthreads) cum[i] = i < A ? R.cum[i] : M;
        owners = reinterpret_cast<uint16_t*>(R.image + dec_cum_bytes(A));
    } else if (smem_look) {
        if (A <= kSmemTableSyms) {
            uint2* tab = reinterpret_cast<uint2*>(R.image);
            for (uint32_t i = tid; i < A; i += nthreads) tab[i] = make_uint2(R.prob[i], R.cum[i]);
        }
        owners = reinterpret_cast<uint16_t*>(R.image + dec_tab_bytes(A));
    }
    // bucketed: entry b < 2^kBucketBits = owner of slot b << (prec - kBucketBits), the last
    // entry = the last symbol; direct lookup and packed entries: one per slot
    const uint32_t n = bucketed ? kBucketCount + 1 : M;
    for (uint32_t i = tid; i < n; i += nthreads) {
        if (bucketed && i == kBucketCount) {
            owners[i] = static_cast<uint16_t>(A - 1);
            continue;
        }
        const uint32_t slot = bucketed ? i << (s.prec - kBucketBits) : i;
        uint32_t lo = 0, hi = A - 1;   // last symbol with cum <= slot and prob > 0
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (R.cum[mid] <= slot) lo = mid; else hi = mid - 1;
        }
        // zero-probability symbols share their successor's cum; step back to the owner
        while (R.prob[lo] == 0 && lo > 0) --lo;
        if (owners) owners[i] = static_cast<uint16_t>(lo);
        else R.slots[slot] = pack_slot(lo, R.prob[lo], slot - R.cum[lo]);
    }
}

// Unpacks the final lane states of section R's chunks (prec + 10 bits each, MSB-first);
// blocks bx of nbx cover the section.
__device__ void section_states(const SectionRef& R, const uint8_t* data, uint32_t* states_base, uint32_t bx,
                               uint32_t nbx) {
    const SectionPlan& s = *R.sec;
    uint32_t* out = states_base + R.states_first;
    const uint64_t words = static_cast<uint64_t>(s.lanes) * s.chunks;
    const uint32_t B = state_bits(s.prec);   // <= 32
    const uint8_t* q = data + s.states_off;
    for (uint64_t w = static_cast<uint64_t>(bx) * blockDim.x + threadIdx.x; w < words;
         w += static_cast<uint64_t>(nbx) * blockDim.x) {
        // the state's B bits lie in the (at most five) bytes from its first bit's byte
        const uint64_t bit = w * B;
        const uint32_t off = static_cast<uint32_t>(bit & 7), nb = (off + B + 7) >> 3;
        uint64_t acc = 0;
        for (uint32_t i = 0; i < nb; ++i) acc = (acc << 8) | q[(bit >> 3) + i];
        out[w] = static_cast<uint32_t>((acc >> (8 * nb - off - B)) & ((1ull << B) - 1));
    }
}

// Tables (blockIdx.x < kLookupBlocks) and final lane states (the rest) of every section
// (blockIdx.y = section), in one launch.
constexpr uint32_t kLookupBlocks = 256, kStateBlocks = 64;
__global__ void __launch_bounds__(256) k_lookup_states(SectionRefs refs, const DecState* st, const uint8_t* data,
                                                        uint32_t* states_base) {
    const SectionRef R = refs.r[blockIdx.y];
    if (blockIdx.x >= kLookupBlocks) {
        section_states(R, data, states_base, blockIdx.x - kLookupBlocks, kStateBlocks);
        return;
    }
    if (st->err) return;
    section_lookup(R, blockIdx.x, kLookupBlocks);
}

__device__ __forceinline__ uint64_t read_bits_msb(const uint8_t* bytes, uint64_t bit, int width) {
    // width <= 32; reads up to 5 bytes
    const uint64_t b0 = bit >> 3;
    const int off = static_cast<int>(bit & 7);
    const int nbytes = (off + width + 7) >> 3;
    uint64_t acc = 0;
    for (int i = 0; i < nbytes; ++i) acc = (acc << 8) | bytes[b0 + i];
    const int total = nbytes * 8;
    acc >>= (total - off - width);
    return width == 64 ? acc : (acc & ((1ull << width) - 1));
}

// Big-endian 32-bit word at byte offset off of the container (bytes past len read as 0).
__device__ __forceinline__ uint32_t load_be32(const uint8_t* data, uint64_t len, uint64_t off) {
    if (off + 4 <= len && (reinterpret_cast<uintptr_t>(data + off) & 3) == 0)
        return __byte_perm(__ldg(reinterpret_cast<const uint32_t*>(data + off)), 0, 0x0123);
    uint32_t v = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) v = (v << 8) | (off + k < len ? static_cast<uint32_t>(data[off + k]) : 0u);
    return v;
}

// Fixed: one warp per tile of 32*G records.  For dimension d (width w) a group of 32
// records fills exactly w 32-bit words of that dimension's MSB-first bit stream, so the
// tile's words of every dimension (G * sum w <= 512) are loaded at once into shared
// memory; each lane then cuts its records' values out of them.  Values pass through
// shared memory (32*G*D <= 512) so that the tile's outputs are stored contiguously.
constexpr int kUnpackWarps = 8;
constexpr uint32_t kUnpackWords = 512;
__global__ void __launch_bounds__(32 * kUnpackWarps) k_unpack_fixed(const uint8_t* data, uint64_t len,
                                                                     const CompPlan* cp, uint32_t* out,
                                                                     DecState* st, uint32_t G) {
    __shared__ uint64_t s_byte[kMaxDims], s_min[kMaxDims];
    __shared__ uint32_t s_w[kMaxDims], s_pre[kMaxDims + 1], s_fits[kMaxDims];
    __shared__ __align__(16) uint32_t wbuf[kUnpackWarps][kUnpackWords];
    __shared__ __align__(16) uint32_t stage[kUnpackWarps][kUnpackWords];
    const uint32_t D = cp->dims;
    const uint64_t R = cp->records;
    if (threadIdx.x < D) {
        s_byte[threadIdx.x] = cp->packed_off[threadIdx.x];
        s_min[threadIdx.x] = cp->minv[threadIdx.x];
        s_w[threadIdx.x] = cp->width[threadIdx.x];
        // every value of this dimension fits 32 bits: no per-value check needed
        s_fits[threadIdx.x] = cp->minv[threadIdx.x] + ((1ull << cp->width[threadIdx.x]) - 1) <= 0xffffffffull;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (uint32_t d = 0; d < D; ++d) { s_pre[d] = acc; acc += G * s_w[d]; }
        s_pre[D] = acc;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t* wb = wbuf[warp];
    uint32_t* sg = stage[warp];
    const uint32_t TR = 32 * G;
    const uint64_t ntiles = (R + TR - 1) / TR;
    bool bad = false;
    for (uint64_t tile = static_cast<uint64_t>(blockIdx.x) * kUnpackWarps + warp; tile < ntiles;
         tile += static_cast<uint64_t>(gridDim.x) * kUnpackWarps) {
        const uint64_t r0 = tile * TR;
        const uint32_t nr = static_cast<uint32_t>(min(static_cast<uint64_t>(TR), R - r0));
        for (uint32_t d = 0; d < D; ++d) {
            const uint32_t nw = G * s_w[d];
            const uint64_t base = s_byte[d] + 4 * tile * nw;
            for (uint32_t j = lane; j < nw; j += 32) wb[s_pre[d] + j] = load_be32(data, len, base + 4 * j);
        }
        __syncwarp();
        for (uint32_t d = 0; d < D; ++d) {
            const uint32_t w = s_w[d], pre = s_pre[d], nw = G * w;
            const uint32_t mn = static_cast<uint32_t>(s_min[d]);
            const bool fits = s_fits[d];
            for (uint32_t g = 0; g < G; ++g) {
                const uint32_t rec = g * 32 + lane;
                uint32_t val = 0;
                if (w) {
                    const uint32_t bit = rec * w, j = bit >> 5;
                    const uint32_t hi = wb[pre + j];
                    const uint32_t lo = j + 1 < nw ? wb[pre + j + 1] : 0u;
                    val = __funnelshift_l(lo, hi, bit & 31) >> (32 - w);
                }
                if (!fits) bad = bad || (rec < nr && s_min[d] + val > 0xffffffffull);
                sg[rec * D + d] = mn + val;
            }
        }
        __syncwarp();
        uint32_t* o = out + r0 * D;
        const uint32_t nv = nr * D;
        if ((reinterpret_cast<uintptr_t>(o) & 15) == 0) {
            for (uint32_t m = 4 * lane; m + 4 <= nv; m += 128)
                *reinterpret_cast<uint4*>(o + m) = *reinterpret_cast<const uint4*>(sg + m);
            for (uint32_t m = (nv & ~3u) + lane; m < nv; m += 32) o[m] = sg[m];
        } else {
            for (uint32_t m = lane; m < nv; m += 32) o[m] = sg[m];
        }
        __syncwarp();
    }
    if (bad) set_error(&st->err, kErrCorrupt);
}

struct TagIn {
    const uint32_t* tags;
    uint32_t D;
    __device__ uint64_t operator()(uint64_t j) const { return static_cast<uint64_t>(tags[j]) * D; }
};
struct TagUnpackOut {
    const uint8_t* payload;
    const uint32_t* tags;
    const CompPlan* cp;
    uint32_t* out;
    DecState* st;
    int s;
    __device__ void operator()(uint64_t j, uint64_t bit, uint64_t nbits) const {
        const uint32_t D = cp->dims;
        const uint32_t t = tags[j];
        if (t < 1 || t > 32) { set_error(&st->err, kErrCorrupt); return; }
        atomicMax(&st->maxtag[s], t);
        if (j + 1 == cp->records) st->tag_bits[s] = bit + nbits;
        if (bit + nbits > cp->packed_bits) { set_error(&st->err, kErrCorrupt); return; }
        for (uint32_t d = 0; d < D; ++d, bit += t) out[j * D + d] = static_cast<uint32_t>(read_bits_msb(payload, bit, t));
    }
};

__global__ void k_check_tagged(const DecState* st_c, DecState* st) {
    if (threadIdx.x || blockIdx.x) return;
    for (int s = 0; s < kCodeStreams; ++s) {
        const CompPlan& c = st_c->plan.comp[s];
        if (c.enc != kEncTagged) continue;
        if (st->tag_bits[s] != c.packed_bits || st->maxtag[s] != c.max_width) set_error(&st->err, kErrCorrupt);
    }
}

// ------------------------------------------------------------------- level 2
// Reset-scan over the compact block records, three dimensions per pass.  Element j:
//   kept record       -> restart with its offset from wrap_min
//   difference record -> add the modular step -correction (mod range)
// so the inclusive prefix of record j is compact[j] - wrap_min (lcps_cpp.cpp:1890-1934
// computes the same values sequentially).
struct L2Vec {
    uint32_t restart;
    uint32_t v[3];
};
struct ResetAddOp {
    uint32_t range_lo, range_hi;   // range = wrap_max - wrap_min + 1 <= 2^32
    __device__ __forceinline__ uint64_t range() const {
        return static_cast<uint64_t>(range_lo) | (static_cast<uint64_t>(range_hi) << 32);
    }
    __device__ __forceinline__ L2Vec operator()(const L2Vec& a, const L2Vec& b) const {
        if (b.restart) return b;
        const uint64_t r = range();
        L2Vec o;
        o.restart = a.restart;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            uint64_t s = static_cast<uint64_t>(a.v[k]) + b.v[k];
            if (s >= r) s -= r;
            o.v[k] = static_cast<uint32_t>(s);
        }
        return o;
    }
    __device__ __forceinline__ static L2Vec identity() { return L2Vec{0, {0, 0, 0}}; }
    __device__ __forceinline__ static ResetAddOp make(uint64_t range) {
        return ResetAddOp{static_cast<uint32_t>(range), static_cast<uint32_t>(range >> 32)};
    }
};
// The same operator for range <= 2^31: a sum of two reduced values fits 32 bits.
struct ResetAddOp32 {
    uint32_t r;
    __device__ __forceinline__ L2Vec operator()(const L2Vec& a, const L2Vec& b) const {
        if (b.restart) return b;
        L2Vec o;
        o.restart = a.restart;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const uint32_t s = a.v[k] + b.v[k];
            o.v[k] = s >= r ? s - r : s;
        }
        return o;
    }
    __device__ __forceinline__ static ResetAddOp32 make(uint64_t range) {
        return ResetAddOp32{static_cast<uint32_t>(range)};
    }
};

// Difference records per flag-scan tile from CH20's 1-bit packing: one CTA per tile,
// one 32-record word per thread; the last CTA turns the counts into the tiles' exclusive
// prefixes and writes their total (last_cta_scan_counts).
__global__ void __launch_bounds__(kFlagTile / 32) k_choice_counts(const uint8_t* cbits, uint64_t len, uint64_t off,
                                                                  uint64_t B, uint32_t* tile_counts, uint32_t* total,
                                                                  uint32_t* done) {
    __shared__ uint32_t wsum[kFlagTile / 32 / 32];
    const uint64_t j0 = static_cast<uint64_t>(blockIdx.x) * kFlagTile + 32ull * threadIdx.x;
    uint32_t c = 0;
    if (j0 < B) {
        const uint32_t valid = B - j0 >= 32 ? 0xffffffffu : (1u << (B - j0)) - 1u;
        c = __popc(__brev(load_be32(cbits, len, off + j0 / 8)) & valid);
    }
    c = warp_sum(c);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kFlagTile / 32 / 32; ++w) t += wsum[w];
        tile_counts[blockIdx.x] = t;
    }
    last_cta_scan_counts(tile_counts, total, done);
}

// Choice values are clamped to {0, 1} for the ranks (so every derived index stays in
// bounds) and validated separately (lcps_cpp.cpp:1899-1900, 1911-1912).
struct ChoiceIn {
    const uint32_t* choice2;
    __device__ uint32_t operator()(uint64_t j) const { return choice2[j] ? 1u : 0u; }
};

__device__ __forceinline__ int64_t unzigzag(uint64_t sym) {
    return (sym & 1u) ? -static_cast<int64_t>(sym >> 1) - 1 : static_cast<int64_t>(sym >> 1);
}

// Level-2 inverse over tiles of kFlagTile block records (the tiles of the flag scan that
// counted the difference records): 16 warps per tile, each warp kL2Rounds rounds of 32
// consecutive records.  A record's row in `diff` is its rank among difference records
// (tile offset + earlier warps + ballot popcount); a kept record's row in `keep` is its
// index minus that rank.  Three dimensions per pass, starting at d0.
constexpr int kL2Warps = 16;
constexpr int kL2Rounds = kFlagTile / (32 * kL2Warps);
static_assert(kL2Rounds * 32 * kL2Warps == kFlagTile, "level-2 tiles are flag-scan tiles");
struct L2Geo {
    const uint32_t* choice2;     // unpacked choices, when cbits is null
    const uint8_t* cbits;        // else CH20's fixed 1-bit packing (minimum 0): record j = bit j from cbits_off
    uint64_t cbits_off, cbits_len;
    const uint32_t* keep;
    const uint32_t* diff;
    const uint32_t* tile_diff;   // exclusive count of difference records before each tile
    uint64_t B;
    uint32_t D, d0;
    uint64_t range;
    int64_t wrap_min, wrap_max, minc, maxc;
    // Difference-record masks of this warp's rounds and the warp's first diff rank.
    // Contains a __syncthreads: every thread of the CTA calls it.
    // Difference flags of records [j0, j0 + 32) as a lane mask (j0 a multiple of 32).
    __device__ __forceinline__ uint32_t flags32(uint64_t j0) const {
        if (cbits) {
            const uint32_t valid = j0 >= B ? 0u : (B - j0 >= 32 ? 0xffffffffu : (1u << (B - j0)) - 1u);
            return __brev(load_be32(cbits, cbits_len, cbits_off + j0 / 8)) & valid;
        }
        const int lane = threadIdx.x & 31;
        const uint64_t j = j0 + lane;
        return __ballot_sync(0xffffffffu, j < B && choice2[j] != 0);
    }
    __device__ __forceinline__ uint32_t ranks(uint32_t (&m)[kL2Rounds], uint32_t* s_cnt) const {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kFlagTile + static_cast<uint64_t>(warp) * 32 * kL2Rounds;
        uint32_t c = 0;
        uint32_t off = tile_diff[blockIdx.x];   // in flight with the choice words
        // packed choices: lane k loads round k's word, then every lane takes them all
        const uint32_t mine = cbits && lane < kL2Rounds ? flags32(base + 32 * lane) : 0u;
#pragma unroll
        for (int k = 0; k < kL2Rounds; ++k) {
            m[k] = cbits ? __shfl_sync(0xffffffffu, mine, k) : flags32(base + 32 * k);
            c += __popc(m[k]);
        }
        if (lane == 0) s_cnt[warp] = c;
        __syncthreads();
        for (int w = 0; w < warp; ++w) off += s_cnt[w];
        return off;
    }
    // Difference term of dimension d0 + kk: offset_j = offset_{j-1} - corr (mod range).
    __device__ __forceinline__ uint32_t diff_term(uint64_t rank, uint32_t kk, bool& bad) const {
        const int64_t corr = unzigzag(diff[rank * D + d0 + kk]);
        const bool ok = corr >= minc && corr <= maxc;   // lcps_cpp.cpp:1917-1918
        bad = bad || !ok;
        return ok ? static_cast<uint32_t>(corr <= 0 ? -corr : static_cast<int64_t>(range) - corr) : 0u;
    }
    // The same two rules on an already loaded value.
    __device__ __forceinline__ uint32_t diff_value(uint32_t sym, bool& bad) const {
        const int64_t corr = unzigzag(sym);
        const bool ok = corr >= minc && corr <= maxc;   // lcps_cpp.cpp:1917-1918
        bad = bad || !ok;
        return ok ? static_cast<uint32_t>(corr <= 0 ? -corr : static_cast<int64_t>(range) - corr) : 0u;
    }
    __device__ __forceinline__ uint32_t keep_check(uint32_t raw, bool& bad) const {
        const int64_t v = raw;
        const bool ok = v >= wrap_min && v <= wrap_max;   // lcps_cpp.cpp:1905-1907
        bad = bad || !ok;
        return ok ? static_cast<uint32_t>(v - wrap_min) : 0u;
    }
    __device__ __forceinline__ uint32_t keep_value(uint64_t row, uint32_t kk, bool& bad) const {
        const int64_t v = keep[row * D + d0 + kk];
        const bool ok = v >= wrap_min && v <= wrap_max;   // lcps_cpp.cpp:1905-1907
        bad = bad || !ok;
        return ok ? static_cast<uint32_t>(v - wrap_min) : 0u;
    }
};

// Tile aggregate of the reset-scan: the value at the tile's end when the tile holds a
// kept record (restart), else the modular sum of its difference terms.  Only the terms
// after the tile's last kept record are read.
__global__ void __launch_bounds__(32 * kL2Warps, 2) k_l2_tail(L2Geo g, L2Vec* tile_aggr) {
    __shared__ uint32_t s_cnt[kL2Warps];
    __shared__ int s_last[kL2Warps];
    __shared__ unsigned long long s_sum[kL2Warps][3];
    __shared__ uint32_t s_keep[3];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t tile0 = static_cast<uint64_t>(blockIdx.x) * kFlagTile;
    const uint32_t wbase = warp * 32 * kL2Rounds;   // warp's first record within the tile
    uint32_t m[kL2Rounds];
    const uint32_t off = g.ranks(m, s_cnt);
    int last = -1;   // last kept record of this warp (index within the tile)
#pragma unroll
    for (int k = 0; k < kL2Rounds; ++k) {
        const uint64_t j0 = tile0 + wbase + 32 * k;
        const uint32_t valid = j0 >= g.B ? 0u : (g.B - j0 >= 32 ? 0xffffffffu : (1u << (g.B - j0)) - 1u);
        const uint32_t km = valid & ~m[k];
        if (km) last = static_cast<int>(wbase + 32 * k + 31 - __clz(km));
    }
    if (lane == 0) s_last[warp] = last;
    __syncthreads();
    int tl = -1;
    for (int w = 0; w < kL2Warps; ++w) tl = s_last[w] > tl ? s_last[w] : tl;
    bool bad = false;
    unsigned long long acc[3] = {0, 0, 0};
    uint32_t run = off;
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < kL2Rounds; ++k) {
        const uint32_t r = wbase + 32 * k + lane;
        const uint64_t rank = run + __popc(m[k] & lt);
        if (((m[k] >> lane) & 1u) && static_cast<int>(r) > tl) {
#pragma unroll
            for (uint32_t kk = 0; kk < 3; ++kk) {
                if (g.d0 + kk < g.D) {
                    acc[kk] += g.diff_term(rank, kk, bad);   // terms < range: one subtraction keeps acc < range
                    if (acc[kk] >= g.range) acc[kk] -= g.range;
                }
            }
        }
        if (static_cast<int>(r) == tl) {
#pragma unroll
            for (uint32_t kk = 0; kk < 3; ++kk)
                s_keep[kk] = g.d0 + kk < g.D ? g.keep_value(tile0 + r - rank, kk, bad) : 0u;
        }
        run += __popc(m[k]);
    }
    // modular sums (every operand is below range, so one conditional subtraction per
    // addition keeps them reduced; no division)
    const unsigned long long r = g.range;
    auto mod_add = [r](unsigned long long a, unsigned long long b) {
        const unsigned long long s = a + b;
        return s >= r ? s - r : s;
    };
#pragma unroll
    for (int kk = 0; kk < 3; ++kk) {
        unsigned long long a = acc[kk];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a = mod_add(a, __shfl_xor_sync(0xffffffffu, a, o));
        if (lane == 0) s_sum[warp][kk] = a;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        L2Vec o;
        o.restart = tl >= 0 ? 1u : 0u;
#pragma unroll
        for (int kk = 0; kk < 3; ++kk) {
            unsigned long long t = o.restart ? s_keep[kk] : 0ull;
            for (int w = 0; w < kL2Warps; ++w) t = mod_add(t, s_sum[w][kk]);
            o.v[kk] = static_cast<uint32_t>(t);
        }
        tile_aggr[blockIdx.x] = o;
    }
}

// The reset-scan proper: every record's offset from wrap_min, seeded with the tile's
// exclusive prefix; writes compact[j * D + d0 + kk] = wrap_min + offset.  Blocked
// layout: lane l of warp w owns the kL2Rounds consecutive records starting at
// tile + w * 32 * kL2Rounds + l * kL2Rounds, combines them in order, and one warp scan
// of the lane aggregates (then the CTA's warp totals and the tile prefix) seeds them.
// Also checks the choice values (lcps_cpp.cpp:1899-1900, 1911-1912) and the value ranges.
// Shared-memory slot of 16-byte word w when a warp stages 32 lanes x 6 words (lane l's
// words 6 l .. 6 l + 5) and reads them back in order: one word of padding after every 24
// keeps a quarter warp's stores (words 6 l + c, l = 0 .. 7) on eight distinct bank groups.
__device__ __forceinline__ uint32_t pad24(uint32_t w) { return w + w / 24; }
constexpr uint32_t kPad24Words = 192 + 192 / 24;   // slots for 192 words
// per warp: the staged input rows (3 * 32 * kL2Rounds words), reused for the output
constexpr uint32_t kL2WarpWords = 4 * kPad24Words;
static_assert(kL2WarpWords >= 3 * 32 * kL2Rounds, "staged rows fit");
constexpr size_t kL2ApplySmem = static_cast<size_t>(kL2Warps) * kL2WarpWords * 4;
// Op: ResetAddOp, or ResetAddOp32 when range <= 2^31.
template <typename Op>
__global__ void __launch_bounds__(32 * kL2Warps) k_l2_apply(L2Geo g, const L2Vec* tile_prefix, uint32_t* compact,
                                                             DecState* st) {
    constexpr int P = kL2Rounds;   // records per lane
    __shared__ uint32_t s_cnt[kL2Warps];
    __shared__ L2Vec s_tot[kL2Warps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t j0 = static_cast<uint64_t>(blockIdx.x) * kFlagTile + static_cast<uint64_t>(warp) * 32 * P +
                        static_cast<uint64_t>(lane) * P;
    const Op op = Op::make(g.range);
    // the tile's offsets, in flight with the choice loads instead of after the barriers
    const uint32_t tdiff = g.tile_diff[blockIdx.x];
    const L2Vec tpre = tile_prefix[blockIdx.x];
    uint32_t c[P];
    if (g.cbits) {   // records j0 .. j0 + 7: one byte of the packing (j0 is a multiple of 8)
        static_assert(P == 8, "one packed byte per lane");
        const uint64_t at = g.cbits_off + j0 / 8;
        const uint32_t byte = at < g.cbits_len ? __ldg(g.cbits + at) : 0u;
#pragma unroll
        for (int k = 0; k < P; ++k) c[k] = (byte >> (7 - k)) & 1u;
    } else if (j0 + P <= g.B && (reinterpret_cast<uintptr_t>(g.choice2 + j0) & 15) == 0) {
        const uint4* q = reinterpret_cast<const uint4*>(g.choice2 + j0);
#pragma unroll
        for (int v = 0; v < P / 4; ++v) {
            const uint4 w4 = __ldg(q + v);
            c[4 * v] = w4.x; c[4 * v + 1] = w4.y; c[4 * v + 2] = w4.z; c[4 * v + 3] = w4.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < P; ++k) c[k] = j0 + k < g.B ? g.choice2[j0 + k] : 0u;
    }
    bool bad = false;
    uint32_t dmask = 0;
#pragma unroll
    for (int k = 0; k < P; ++k) {
        const uint64_t j = j0 + k;
        if (j < g.B) {
            bad = bad || c[k] > 1 || (j == 0 && c[k] != 0);
            if (c[k]) dmask |= 1u << k;
        }
    }
    const uint32_t cnt = __popc(dmask);
    const uint32_t incl_cnt = warp_inclusive_sum(cnt);
    if (lane == 31) s_cnt[warp] = incl_cnt;
    __syncthreads();
    uint64_t rank = tdiff + incl_cnt - cnt;   // diff records before j0
    for (int w = 0; w < warp; ++w) rank += s_cnt[w];
    // every record's row first (one memory round trip for the lane), then the terms
    uint32_t raw[P][3];
    if (g.D == 3) {
        // The warp's 256 records use one run of diff rows and one of keep rows; both are
        // copied into shared memory with coalesced loads (diff rows first), and every
        // lane takes its records' rows from there.
        extern __shared__ uint32_t l2rows[];   // kL2Warps * kL2WarpWords words
        uint32_t* s = l2rows + warp * kL2WarpWords;
        const uint64_t jw = j0 - static_cast<uint64_t>(lane) * P;   // the warp's first record
        const uint64_t dr0 = __shfl_sync(0xffffffffu, rank, 0);
        const uint32_t nd = __shfl_sync(0xffffffffu, incl_cnt, 31);
        const uint32_t nv = jw >= g.B ? 0u : static_cast<uint32_t>(min(g.B - jw, static_cast<uint64_t>(32 * P)));
        const uint64_t kr0 = jw - dr0;
        const uint32_t* dsrc = g.diff + 3 * dr0;
        const uint32_t* ksrc = g.keep + 3 * kr0 - 3 * static_cast<uint64_t>(nd);   // word w >= 3 nd of the run
        uint32_t v[3 * P];
#pragma unroll
        for (int it = 0; it < 3 * P; ++it) {
            const uint32_t w = lane + 32 * it;
            v[it] = w < 3 * nd ? __ldg(dsrc + w) : (w < 3 * nv ? __ldg(ksrc + w) : 0u);
        }
#pragma unroll
        for (int it = 0; it < 3 * P; ++it) s[lane + 32 * it] = v[it];
        __syncwarp();
        uint32_t rk = static_cast<uint32_t>(rank - dr0);   // diff rows of this warp before the lane's
        const uint32_t rec0 = static_cast<uint32_t>(lane) * P;
#pragma unroll
        for (int k = 0; k < P; ++k) {
            const bool is_diff = (dmask >> k) & 1u;
            const uint32_t row = is_diff ? rk : nd + (rec0 + k - rk);
#pragma unroll
            for (uint32_t kk = 0; kk < 3; ++kk) raw[k][kk] = j0 + k < g.B ? s[3 * row + kk] : 0u;
            rk += is_diff;
        }
    } else {
        uint64_t rk = rank;
#pragma unroll
        for (int k = 0; k < P; ++k) {
            const uint64_t j = j0 + k;
            const bool is_diff = (dmask >> k) & 1u;
            const uint32_t* row = is_diff ? g.diff + rk * g.D + g.d0 : g.keep + (j - rk) * g.D + g.d0;
#pragma unroll
            for (uint32_t kk = 0; kk < 3; ++kk) raw[k][kk] = (j < g.B && g.d0 + kk < g.D) ? __ldg(row + kk) : 0u;
            rk += is_diff;
        }
    }
    L2Vec t[P];
#pragma unroll
    for (int k = 0; k < P; ++k) {
        const uint64_t j = j0 + k;
        t[k] = ResetAddOp::identity();
        if (j >= g.B) continue;
        if ((dmask >> k) & 1u) {
#pragma unroll
            for (uint32_t kk = 0; kk < 3; ++kk)
                if (g.d0 + kk < g.D) t[k].v[kk] = g.diff_value(raw[k][kk], bad);
        } else {
            t[k].restart = 1;
#pragma unroll
            for (uint32_t kk = 0; kk < 3; ++kk)
                if (g.d0 + kk < g.D) t[k].v[kk] = g.keep_check(raw[k][kk], bad);
        }
    }
    L2Vec agg = t[0];
#pragma unroll
    for (int k = 1; k < P; ++k) agg = op(agg, t[k]);
    const L2Vec inc = warp_inclusive_scan_op(agg, op);
    L2Vec exc = shfl_up_any(inc, 1);
    if (lane == 0) exc = ResetAddOp::identity();
    if (lane == 31) s_tot[warp] = inc;
    __syncthreads();
    L2Vec carry = tpre;
    for (int w = 0; w < warp; ++w) carry = op(carry, s_tot[w]);
    carry = op(carry, exc);
    uint32_t o[3 * P];
#pragma unroll
    for (int k = 0; k < P; ++k) {
        carry = op(carry, t[k]);
#pragma unroll
        for (int kk = 0; kk < 3; ++kk) o[3 * k + kk] = static_cast<uint32_t>(g.wrap_min + carry.v[kk]);
    }
    uint32_t* dst = compact + j0 * g.D;
    const uint64_t jw = j0 - static_cast<uint64_t>(lane) * P;   // the warp's first record
    if (g.D == 3 && jw + 32 * P <= g.B && (reinterpret_cast<uintptr_t>(compact + jw * 3) & 15) == 0) {
        // the warp's 256 whole records (3072 bytes) leave through its shared rows as
        // 16-byte words, consecutive lanes on consecutive words
        static_assert(3 * P / 4 == 6, "six 16-byte words per lane");
        extern __shared__ uint32_t l2rows[];
        uint4* s = reinterpret_cast<uint4*>(l2rows + warp * kL2WarpWords);
        __syncwarp();   // every lane has read its input rows
#pragma unroll
        for (int v = 0; v < 6; ++v) s[pad24(6 * lane + v)] = make_uint4(o[4 * v], o[4 * v + 1], o[4 * v + 2], o[4 * v + 3]);
        __syncwarp();
        uint4* q = reinterpret_cast<uint4*>(compact + jw * 3);
#pragma unroll
        for (int w = 0; w < 6; ++w) q[32 * w + lane] = s[pad24(32 * w + lane)];
    } else if (g.D == 3 && j0 + P <= g.B && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
        uint4* q = reinterpret_cast<uint4*>(dst);
#pragma unroll
        for (int v = 0; v < 3 * P / 4; ++v) q[v] = make_uint4(o[4 * v], o[4 * v + 1], o[4 * v + 2], o[4 * v + 3]);
    } else {
#pragma unroll
        for (int k = 0; k < P; ++k) {
            if (j0 + k >= g.B) break;
#pragma unroll
            for (uint32_t kk = 0; kk < 3; ++kk)
                if (g.d0 + kk < g.D) dst[static_cast<uint64_t>(k) * g.D + g.d0 + kk] = o[3 * k + kk];
        }
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) set_error(&st->err, kErrCorrupt);
}

// ------------------------------------------------------------------- level 1
struct ZeroIn {
    const uint32_t* idrel;
    __device__ uint32_t operator()(uint64_t i) const { return idrel[i] == 0 ? 1u : 0u; }
    __host__ __device__ const uint32_t* zero_words() const { return idrel; }
};
// Parent words: bit 31 set = resolved (the low bits are the chain's explicit point).
constexpr uint32_t kResolved = 0x80000000u;
constexpr uint32_t kParentMask = 0x7fffffffu;

// Parents of all points and the list of chained points.  An explicit point is a
// resolved root whose word holds its rank among explicit points (its block's record in
// the compact level-2 output); a chained point i points at i + idrel[i], and its rank
// among chained points is i - (explicit points before i).
struct ZeroRankOut {
    const uint32_t* idrel;
    uint32_t* parent;
    uint32_t* chained;
    DecState* st;
    uint64_t n;
    __device__ void operator()(uint64_t i, uint32_t pre, uint32_t z) const {
        const uint32_t j = idrel[i];
        if (z) { parent[i] = pre | kResolved; return; }
        chained[i - pre] = static_cast<uint32_t>(i);
        if (static_cast<uint64_t>(j) >= n - i) {
            set_error(&st->err, kErrCorrupt);
            parent[i] = kResolved;
            return;
        }
        parent[i] = static_cast<uint32_t>(i + j);
    }
};

// One pass of concurrent pointer jumping over the chained points, highest index first:
// a point repeatedly replaces its parent word by its parent's current word (which that
// parent's own thread keeps advancing the same way), so pointers double while threads
// run side by side, and points reached later (lower indices; parents point forward)
// mostly find resolved parents.  Warps claim 32 * kResolvePer points at a time from
// *next (zero at launch), so the pass follows descending index order however the CTAs
// are scheduled; each lane advances its kResolvePer points together, keeping that many
// independent loads in flight.  Every word written is an ancestor of the point, so any
// interleaving is correct.  A point stops after kResolveHops hops; any point left
// unresolved sets *pending, and the k_jump rounds finish the work.
constexpr int kResolveHops = 64;
constexpr int kResolvePer = 8;
__global__ void __launch_bounds__(256) k_resolve(uint32_t* parent, const uint32_t* chained, const uint32_t* zeros,
                                                  uint64_t n, unsigned long long* next, uint32_t* pending) {
    const uint64_t m = n - *zeros;
    const int lane = threadIdx.x & 31;
    bool left = false;
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(next, 32ull * kResolvePer);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= m) break;
        uint32_t idx[kResolvePer], p[kResolvePer];
#pragma unroll
        for (int k = 0; k < kResolvePer; ++k) {
            const uint64_t t = base + 32 * k + lane;
            idx[k] = t < m ? chained[m - 1 - t] : 0u;
            p[k] = t < m ? parent[idx[k]] : kResolved;
        }
        for (int h = 0; h < kResolveHops; ++h) {
            bool open = false;
#pragma unroll
            for (int k = 0; k < kResolvePer; ++k) {
                if (!(p[k] & kResolved)) {
                    p[k] = parent[p[k]];
                    parent[idx[k]] = p[k];
                    open = true;
                }
            }
            if (!open) break;
        }
#pragma unroll
        for (int k = 0; k < kResolvePer; ++k) left = left || !(p[k] & kResolved);
    }
    if (__syncthreads_or(left) && threadIdx.x == 0) atomicOr(pending, 1u);
}

// One pointer-jumping round over the chained points: an unresolved point takes its
// parent's parent word (and with it the resolved bit).  Round r runs only if
// pending[r] is set and sets pending[r + 1] if any point is still unresolved after it.
// Jumps only point forward, so ceil(log2 N) rounds resolve all.
__global__ void __launch_bounds__(256) k_jump(uint32_t* parent, const uint32_t* chained, const uint32_t* zeros,
                                               uint64_t n, uint32_t* pending, int round) {
    if (pending[round] == 0) return;
    const uint64_t m = n - *zeros;
    bool any = false;
    for (uint64_t k = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; k < m;
         k += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t i = chained[k];
        const uint32_t p = parent[i];
        if (p & kResolved) continue;
        const uint32_t pp = parent[p];
        parent[i] = pp;
        any |= !(pp & kResolved);
    }
    if (__syncthreads_or(any) && threadIdx.x == 0) atomicOr(&pending[round + 1], 1u);
}

// q = block(root) * p + offset, then x = fma(q + 0.5, 2 eb, min) (lcps_cpp.cpp:1496-1500).
// A resolved parent word holds the index of the point's block record in `compact`.
// Points whose parent word is not resolved yet are skipped: the caller runs the
// pointer-jumping rounds and this kernel again (or reports them unresolved).  Each
// thread takes kReconPer consecutive points and issues their block-record gathers
// together.  Four CTAs of 256 threads per SM (64 registers, a few spilled) stream
// faster than three without spills.
constexpr int kReconPer = 4;
constexpr int kReconThreads = 256;
// blk * p + off > INT64_MAX, for 0 <= blk, 0 <= off < p, from the exact 128-bit product
// (the same test as blk > (INT64_MAX - off) / p, without a 64-bit division)
__device__ __forceinline__ bool q_overflows(int64_t blk, int64_t p, int64_t off) {
    const uint64_t b = static_cast<uint64_t>(blk), m = static_cast<uint64_t>(p);
    return __umul64hi(b, m) != 0 || b * m > static_cast<uint64_t>(INT64_MAX) - static_cast<uint64_t>(off);
}
struct ReconCtx {
    const uint32_t* compact;
    uint32_t D, B;
    int64_t p, safe_blk;   // blk * p + off <= INT64_MAX for every off < p whenever blk <= safe_blk
    double two_eb;
    const double* minima;
    __device__ __forceinline__ double coord(uint32_t cr, uint32_t d, int64_t off, bool& bad) const {
        if (off >= p) bad = true;
        const int64_t blk = bad ? 0 : compact[static_cast<uint64_t>(cr) * D + d];
        if (blk > safe_blk && q_overflows(blk, p, off)) bad = true;
        const int64_t q = bad ? 0 : blk * p + off;
        return fma(__dadd_rn(static_cast<double>(q), 0.5), two_eb, minima[d]);
    }
};
// REL0 read straight from its fixed-width packing (three dimensions, widths <= 8) when
// `on`, instead of from an unpacked array: a dimension's value of point i is minv + the
// w bits at bit i * w of that dimension's MSB-first stream.
struct RelBits {
    const uint8_t* data;
    uint64_t len;
    uint64_t off[3];
    uint32_t minv[3], w[3];
    int on;
    // Dimension d of points i0 .. i0 + 3: four w-bit values span at most 39 bits, the
    // five bytes from the first value's byte.
    __device__ __forceinline__ void four(uint64_t i0, uint32_t d, uint32_t (&v)[4]) const {
        const uint32_t wd = w[d];
        const uint64_t bit0 = i0 * wd;
        const uint64_t b = off[d] + (bit0 >> 3);
        uint64_t win = 0;
#pragma unroll
        for (int i = 0; i < 5; ++i) win = (win << 8) | (b + i < len ? __ldg(data + b + i) : 0u);
        const uint32_t top = 40 - static_cast<uint32_t>(bit0 & 7);
#pragma unroll
        for (int k = 0; k < 4; ++k)
            v[k] = minv[d] + (wd ? static_cast<uint32_t>((win >> (top - (k + 1) * wd)) & ((1u << wd) - 1)) : 0u);
    }
};

template <typename OT, bool SOA>
__global__ void __launch_bounds__(kReconThreads, 4)
k_reconstruct(const uint32_t* __restrict__ parent, const uint32_t* __restrict__ compact,
              const uint32_t* __restrict__ rel, const DecState* stc, DecState* st, OT* __restrict__ out,
              RelBits rb) {
    // a warp's 128 three-dimensional points pass through shared memory on the way out,
    // so that each store instruction writes 512 contiguous bytes
    __shared__ __align__(16) OT stage[kReconThreads / 32][kPad24Words * 16 / sizeof(OT)];
    const DecodePlan& P = stc->plan;
    const uint32_t D = P.D;
    const uint64_t n = P.N;
    ReconCtx R;
    R.compact = compact;
    R.D = D;
    R.B = static_cast<uint32_t>(P.comp[3].records);
    R.p = P.p;
    R.safe_blk = (INT64_MAX - (P.p - 1)) / P.p;
    R.two_eb = 2.0 * P.eb;
    R.minima = P.minima;
    bool bad = false;
    const bool vec = ((reinterpret_cast<uintptr_t>(parent) | reinterpret_cast<uintptr_t>(rel) |
                       reinterpret_cast<uintptr_t>(out)) & 15) == 0;
    const uint32_t lane = threadIdx.x & 31;
    OT* sw = stage[threadIdx.x >> 5];
    const uint64_t ng = (n + kReconPer - 1) / kReconPer;
    // the loop runs warp by warp (gw = group of the warp's lane 0), so that every lane of
    // a warp takes the same iterations
    for (uint64_t gw = static_cast<uint64_t>(blockIdx.x) * blockDim.x + (threadIdx.x - lane); gw < ng;
         gw += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t g = gw + lane;
        if (D == 3 && vec && (gw + 32) * kReconPer <= n) {
            // the whole warp holds four whole points per lane: 16-byte loads of parent and
            // rel (or REL0's packed bits), stores staged through shared memory
            uint32_t pw[kReconPer];
            *reinterpret_cast<uint4*>(pw) = __ldg(reinterpret_cast<const uint4*>(parent + g * kReconPer));
            uint32_t rl[12];
            if (rb.on) {
#pragma unroll
                for (uint32_t d = 0; d < 3; ++d) {
                    uint32_t v[4];
                    rb.four(g * kReconPer, d, v);
#pragma unroll
                    for (int k = 0; k < 4; ++k) rl[3 * k + d] = v[k];
                }
            } else {
                const uint4* rp = reinterpret_cast<const uint4*>(rel + g * 12);
                *reinterpret_cast<uint4*>(rl) = __ldg(rp);
                *reinterpret_cast<uint4*>(rl + 4) = __ldg(rp + 1);
                *reinterpret_cast<uint4*>(rl + 8) = __ldg(rp + 2);
            }
            uint32_t blk[kReconPer][3];
#pragma unroll
            for (int k = 0; k < kReconPer; ++k) {
                const uint32_t cr = pw[k] & kParentMask;
                const bool ok = (pw[k] & kResolved) && cr < R.B;
#pragma unroll
                for (int d = 0; d < 3; ++d) blk[k][d] = ok ? compact[static_cast<uint64_t>(cr) * 3 + d] : 0u;
            }
            const uint64_t i0 = g * kReconPer;
            bool all = true;
#pragma unroll
            for (int k = 0; k < kReconPer; ++k) all = all && (pw[k] & kResolved);
            // coordinate d of point k; marks the point bad on a corrupt block or offset
            auto coord = [&](int k, int d, bool& b) -> double {
                const int64_t off = rl[3 * k + d];
                if (off >= R.p) b = true;
                const int64_t bk = b ? 0 : static_cast<int64_t>(blk[k][d]);
                if (bk > R.safe_blk && q_overflows(bk, R.p, off)) b = true;
                const int64_t q = b ? 0 : bk * R.p + off;
                return fma(__dadd_rn(static_cast<double>(q), 0.5), R.two_eb, R.minima[d]);
            };
            if constexpr (!SOA) {
                // two points (six values) at a time into shared memory: lane l's values
                // are the 16-byte words 6 l .. 6 l + 5 of the warp's 3072 bytes (float64)
                // or 3 l .. 3 l + 2 of its 1536 bytes (float32); float64 words are stored
                // at word + word / 24, which keeps a quarter warp's stores on distinct banks
#pragma unroll
                for (int kp = 0; kp < kReconPer / 2; ++kp) {
                    bool b0 = (pw[2 * kp] & kParentMask) >= R.B, b1 = (pw[2 * kp + 1] & kParentMask) >= R.B;
                    double v[6];
#pragma unroll
                    for (int d = 0; d < 3; ++d) v[d] = coord(2 * kp, d, b0);
#pragma unroll
                    for (int d = 0; d < 3; ++d) v[3 + d] = coord(2 * kp + 1, d, b1);
                    bad = bad || (b0 && (pw[2 * kp] & kResolved)) || (b1 && (pw[2 * kp + 1] & kResolved));
                    if constexpr (sizeof(OT) == 8) {
                        double2* s = reinterpret_cast<double2*>(sw);
#pragma unroll
                        for (int c = 0; c < 3; ++c) s[pad24(6 * lane + 3 * kp + c)] = make_double2(v[2 * c], v[2 * c + 1]);
                    } else {
                        float2* s = reinterpret_cast<float2*>(sw + 12 * lane + 6 * kp);
#pragma unroll
                        for (int c = 0; c < 3; ++c)
                            s[c] = make_float2(static_cast<float>(v[2 * c]), static_cast<float>(v[2 * c + 1]));
                    }
                }
                __syncwarp();
                if (__all_sync(0xffffffffu, all)) {
                    // the warp's 128 points (384 values) leave as 16-byte words,
                    // consecutive lanes on consecutive words
                    uint4* o = reinterpret_cast<uint4*>(out + gw * kReconPer * 3);
                    const uint4* s16 = reinterpret_cast<const uint4*>(sw);
                    if constexpr (sizeof(OT) == 8) {
#pragma unroll
                        for (int w = 0; w < 6; ++w) o[32 * w + lane] = s16[pad24(32 * w + lane)];
                    } else {
#pragma unroll
                        for (int w = 0; w < 3; ++w) o[32 * w + lane] = s16[32 * w + lane];
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < kReconPer; ++k) {
                        if (!(pw[k] & kResolved)) continue;
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            const int j = 3 * k + d;
                            OT x;
                            if constexpr (sizeof(OT) == 8)
                                x = sw[2 * pad24(6 * lane + j / 2) + (j & 1)];
                            else
                                x = sw[12 * lane + j];
                            out[(i0 + k) * 3 + d] = x;
                        }
                    }
                }
                __syncwarp();
            } else {
#pragma unroll
                for (int k = 0; k < kReconPer; ++k) {
                    bool b = (pw[k] & kParentMask) >= R.B;
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const double x = coord(k, d, b);
                        if (pw[k] & kResolved) out[static_cast<uint64_t>(d) * n + i0 + k] = static_cast<OT>(x);
                    }
                    bad = bad || (b && (pw[k] & kResolved));
                }
            }
            continue;
        }
        if (g >= ng) continue;
        uint32_t pw[kReconPer];
        const bool full = g * kReconPer + kReconPer <= n;
        if (full && vec) {
            *reinterpret_cast<uint4*>(pw) = __ldg(reinterpret_cast<const uint4*>(parent + g * kReconPer));
        } else {
#pragma unroll
            for (int k = 0; k < kReconPer; ++k) {
                const uint64_t i = g * kReconPer + k;
                pw[k] = i < n ? parent[i] : 0u;
            }
        }
        if (D == 3) {
            uint32_t rl[12];
            if (rb.on) {
#pragma unroll
                for (uint32_t d = 0; d < 3; ++d) {
                    uint32_t v[4];
                    rb.four(g * kReconPer, d, v);
#pragma unroll
                    for (int k = 0; k < 4; ++k) rl[3 * k + d] = v[k];
                }
            }
            uint32_t blk[kReconPer][3];
#pragma unroll
            for (int k = 0; k < kReconPer; ++k) {
                const uint32_t cr = pw[k] & kParentMask;
                const bool ok = (pw[k] & kResolved) && cr < R.B;
#pragma unroll
                for (int d = 0; d < 3; ++d) blk[k][d] = ok ? compact[static_cast<uint64_t>(cr) * 3 + d] : 0u;
            }
#pragma unroll
            for (int k = 0; k < kReconPer; ++k) {
                const uint64_t i = g * kReconPer + k;
                if (i >= n || !(pw[k] & kResolved)) continue;
                bool b = (pw[k] & kParentMask) >= R.B;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const int64_t off = rb.on ? rl[3 * k + d] : rel[i * 3 + d];
                    if (off >= R.p) b = true;
                    const int64_t bk = b ? 0 : static_cast<int64_t>(blk[k][d]);
                    if (bk > R.safe_blk && q_overflows(bk, R.p, off)) b = true;
                    const int64_t q = b ? 0 : bk * R.p + off;
                    const double x = fma(__dadd_rn(static_cast<double>(q), 0.5), R.two_eb, R.minima[d]);
                    out[SOA ? static_cast<uint64_t>(d) * n + i : i * 3 + d] = static_cast<OT>(x);
                }
                bad = bad || b;
            }
        } else {
#pragma unroll
            for (int k = 0; k < kReconPer; ++k) {
                const uint64_t i = g * kReconPer + k;
                if (i >= n || !(pw[k] & kResolved)) continue;
                const uint32_t cr = pw[k] & kParentMask;
                bool b = cr >= R.B;
                for (uint32_t d = 0; d < D; ++d) {
                    const double x = R.coord(cr, d, rel[i * D + d], b);
                    out[SOA ? static_cast<uint64_t>(d) * n + i : i * D + d] = static_cast<OT>(x);
                }
                bad = bad || b;
            }
        }
    }
    if (bad) set_error(&st->err, kErrCorrupt);
}

// Exact corrections: index_k = sum_{m<=k} (gap_m + 1) - 1, value = dictionary[id_k]
// (lcps_cpp.cpp:1979-1992 applies the same records).  Indices are strictly increasing
// by construction; each is checked against n * dims, each id against the dictionary.
struct CorrIn {
    const uint32_t* gaps;
    __device__ uint64_t operator()(uint64_t k) const { return static_cast<uint64_t>(gaps[k]) + 1; }
};
template <typename OT, bool SOA>
struct CorrOut {
    const uint32_t* ids;
    const uint8_t* data;
    const DecState* stc;
    DecState* st;
    OT* out;
    __device__ void operator()(uint64_t k, uint64_t prefix, uint64_t step) const {
        const DecodePlan& P = stc->plan;
        const uint64_t idx = prefix + step - 1;
        const uint32_t id = ids[k];
        const uint64_t nd = P.N * P.D;
        if (idx >= nd || id >= P.exc_ndistinct) { set_error(&st->err, kErrCorrupt); return; }
        uint64_t vb = 0;
        for (int b = 0; b < 8; ++b) vb |= static_cast<uint64_t>(data[P.exc_dict_off + 8ull * id + b]) << (8 * b);
        double v;
        memcpy(&v, &vb, 8);
        if (!chain_isfinite(v)) { set_error(&st->err, kErrCorrupt); return; }
        const uint64_t i = idx / P.D, d = idx - i * P.D;
        out[SOA ? d * P.N + i : idx] = static_cast<OT>(v);
    }
};

// --------------------------------------------------------------------- host
static unsigned dgrid(uint64_t n, int threads = 256, unsigned cap = 148u * 16u) {
    uint64_t g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return static_cast<unsigned>(g);
}

chain_status decode_frame(chain_ctx* ctx, const void* container, size_t len, chain_dtype out_dtype,
                          chain_layout out_layout, void* out, size_t out_capacity, uint64_t* n_out,
                          uint32_t* dims_out) {
    cudaStream_t stream = ctx->stream;
    chain_status s0 = ensure_state(ctx, sizeof(DecState));
    if (s0 != CHAIN_OK) return s0;
    DecState* st = static_cast<DecState*>(ctx->state_dev);
    DecState* hs = static_cast<DecState*>(ctx->state_host);
    const bool host_in = !is_device_ptr(container);
    StageTimer& T = ctx->timer;
    T.begin(stream);
    DecodePlan plan;
    if (host_in) {
        if (!parse_container(static_cast<const uint8_t*>(container), len, &plan))
            return set_err(CHAIN_ERR_CORRUPT_STREAM, "LCG2: container failed validation (check at chain_format.h:" +
                                                         std::to_string(plan.why) + ")");
    }
    // sizes for the arena: parse on the device when the container lives there
    const uint8_t* dcont = static_cast<const uint8_t*>(container);
    size_t base_need = host_in ? Arena::need(len + 16, 1) : 0;
    if (!host_in) {
        k_parse<<<1, 1, 0, stream>>>(dcont, len, st); count_launch();
        CHAIN_LAUNCH_CHECK("parse");
        CHAIN_CUDA(cudaMemcpyAsync(&hs->plan, &st->plan, sizeof(DecodePlan), cudaMemcpyDeviceToHost, stream));
        CHAIN_CUDA(cudaStreamSynchronize(stream));
        T.mark("parse+sync", stream);
        plan = hs->plan;
        if (!plan.ok)
            return set_err(CHAIN_ERR_CORRUPT_STREAM, "LCG2: container failed validation (check at chain_format.h:" +
                                                         std::to_string(plan.why) + ")");
    }
    const uint64_t N = plan.N;
    const uint32_t D = plan.D;
    const uint64_t nd = N * D;
    const size_t osz = out_dtype == CHAIN_F64 ? 8 : 4;
    if (n_out) *n_out = N;
    if (dims_out) *dims_out = D;
    if (out_capacity < nd * osz)
        return set_err(CHAIN_ERR_BUFFER_TOO_SMALL, "output buffer holds " + std::to_string(out_capacity) +
                                                       " bytes, need " + std::to_string(nd * osz));
    const uint64_t B = plan.comp[3].records;
    uint64_t max_prec_slots = 0, total_chunks = 0, max_alpha = 0, tags_total = 0, parse_scratch = 0, images = 0;
    uint64_t tag_off[kCodeStreams] = {0};
    for (int s = 0; s < kCodeStreams; ++s) {
        const CompPlan& c = plan.comp[s];
        if (c.enc == kEncRaw || c.enc == kEncTagged) {
            const uint32_t img = dec_image_bytes(c.sec.prec, c.sec.alphabet);
            images += img;
            if (img == 0) max_prec_slots += 1ull << c.sec.prec;
            total_chunks += c.sec.chunks;
            max_alpha += c.sec.alphabet;
            parse_scratch += 8ull * (c.sec.table_len / kParseSeg + 2);
        }
        if (c.enc == kEncTagged) {
            tag_off[s] = tags_total;
            tags_total += c.records;
        }
    }
    const bool host_out = !is_device_ptr(out);
    size_t need = base_need;
    need += Arena::need(N, 4) * 3;           // idrel, choice2, parent
    need += Arena::need(nd, 4) * 4;          // diff, keep, rel, compact
    need += Arena::need(N, 4);               // drank
    need += Arena::need(tags_total + 1, 4);
    need += Arena::need(images + 16, 1) + Arena::need(max_prec_slots + 1, 8) + Arena::need(max_alpha + 1, 4) * 2;
    need += Arena::need(total_chunks + kCodeStreams + 1, 8) + Arena::need(total_chunks * 32 + 1, 4);
    need += Arena::need(plan.exc_count + 1, 4) * 2;   // correction gaps, ids
    need += Arena::need(scan_scratch_bytes(std::max<uint64_t>(nd, N)), 1);
    need += Arena::need(32, 8);
    need += Arena::need(parse_scratch + 1, 4);
    if (host_out) need += Arena::need(nd, osz);
    need += 24 * 256;
    CHAIN_CUDA(ctx->dec.reserve(need));
    Arena& A = ctx->dec;
    if (host_in) {
        uint8_t* d = A.take<uint8_t>(len + 16);
        CHAIN_CUDA(cudaMemcpyAsync(d, container, len, cudaMemcpyHostToDevice, stream));
        dcont = d;
        hs->plan = plan;
        k_dec_init<<<1, 1, 0, stream>>>(st); count_launch();
        CHAIN_CUDA(cudaMemcpyAsync(&st->plan, &hs->plan, sizeof(DecodePlan), cudaMemcpyHostToDevice, stream));
        T.mark("h2d_container", stream);
    }
    uint32_t* streams[kCodeStreams];
    streams[0] = A.take<uint32_t>(N);
    streams[1] = A.take<uint32_t>(nd);
    streams[2] = A.take<uint32_t>(nd);
    streams[3] = A.take<uint32_t>(N);
    streams[4] = A.take<uint32_t>(nd);
    streams[kCorrGaps] = A.take<uint32_t>(plan.exc_count + 1);
    streams[kCorrIds] = A.take<uint32_t>(plan.exc_count + 1);
    uint32_t* compact = A.take<uint32_t>(nd);
    uint32_t* parent = A.take<uint32_t>(N);
    uint32_t* drank = A.take<uint32_t>(N);
    uint32_t* tags = A.take<uint32_t>(tags_total + 1);
    uint8_t* image_buf = A.take<uint8_t>(images + 16);
    uint64_t* slots64 = A.take<uint64_t>(max_prec_slots + 1);
    uint32_t* prob = A.take<uint32_t>(max_alpha + 1);
    uint32_t* cum = A.take<uint32_t>(max_alpha + 1);
    uint64_t* chunk_off = A.take<uint64_t>(total_chunks + kCodeStreams + 1);
    uint32_t* states = A.take<uint32_t>(total_chunks * 32 + 1);
    uint64_t* scanbuf = reinterpret_cast<uint64_t*>(A.take<uint8_t>(scan_scratch_bytes(std::max<uint64_t>(nd, N))));
    uint64_t* misc = A.take<uint64_t>(32);
    uint32_t* pscratch = A.take<uint32_t>(parse_scratch + 1);
    void* dout = host_out ? A.take<uint8_t>(nd * osz) : out;
    if (!misc || !dout) return set_err(CHAIN_ERR_OUT_OF_MEMORY, "decoder arena too small");
    CHAIN_CUDA(cudaMemsetAsync(misc, 0, 32 * sizeof(uint64_t), stream));

    // ---- entropy sections
    SectionRefs refs{};
    RansJobs jobs{};
    uint64_t slot_base = 0, image_base = 0, alpha_base = 0, chunk_base = 0, off_base = 0, pscr_base = 0;
    uint32_t first = 0;
    int nsec = 0;
    for (int s = 0; s < kCodeStreams; ++s) {
        const CompPlan& c = plan.comp[s];
        if (c.enc != kEncRaw && c.enc != kEncTagged) continue;
        SectionRef& R = refs.r[nsec];
        R.sec = &st->plan.comp[s].sec;
        R.scratch = pscratch + pscr_base;
        pscr_base += 8ull * (c.sec.table_len / kParseSeg + 2);
        R.prob = prob + alpha_base;
        R.cum = cum + alpha_base;
        const uint32_t img = dec_image_bytes(c.sec.prec, c.sec.alphabet);
        R.image = img ? image_buf + image_base : nullptr;
        R.slots = img ? nullptr : slots64 + slot_base;
        R.chunk_off = chunk_off + off_base;
        R.states_first = chunk_base * 32;
        RansJob& jb = jobs.job[jobs.njobs++];
        jb.count = c.sec.count;
        jb.prob = R.prob;
        jb.cum = R.cum;
        jb.image = reinterpret_cast<const uint4*>(R.image);
        jb.slots = R.slots;
        jb.prec = c.sec.prec;
        jb.alphabet = c.sec.alphabet;
        jb.chunks = c.sec.chunks;
        jb.lanes = c.sec.lanes;
        jb.S = c.sec.S;
        jb.bytes = const_cast<uint8_t*>(dcont);
        jb.bytes_len = len;
        jb.chunk_off = R.chunk_off;
        jb.states = states + chunk_base * 32;
        jb.out = c.enc == kEncRaw ? streams[s] : tags + tag_off[s];
        jb.first_block = first;
        first += (c.sec.chunks + kRansDecWarps - 1) / kRansDecWarps;
        if (img) image_base += img;
        else slot_base += 1ull << c.sec.prec;
        alpha_base += c.sec.alphabet;
        chunk_base += c.sec.chunks;
        off_base += c.sec.chunks + 1;
        ++nsec;
    }
    refs.count = nsec;
    jobs.total_blocks = first;
    if (nsec) {
        CHAIN_CUDA(cudaFuncSetAttribute(k_section_setup, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(kParseSmem)));
        k_section_setup<<<nsec, 1024, kParseSmem, stream>>>(refs, dcont, st); count_launch();
        k_lookup_states<<<dim3(kLookupBlocks + kStateBlocks, nsec), 256, 0, stream>>>(refs, st, dcont, states); count_launch();
        T.mark("tables", stream);
        rans_plan_smem(jobs, true);
        if (rans_dec_smem(jobs) > kRansDecSmemMax)
            return set_err(CHAIN_ERR_DEVICE, "internal: rANS decoder shared memory above its fixed maximum");
        {  // per device, cheap; set on every call, always to the same values
            CHAIN_CUDA(cudaFuncSetAttribute(rans_decode_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                            cudaSharedmemCarveoutMaxShared));
            CHAIN_CUDA(cudaFuncSetAttribute(rans_decode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            static_cast<int>(kRansDecSmemMax)));
        }
        rans_decode_kernel<<<jobs.total_blocks, 32 * kRansDecWarps, rans_dec_smem(jobs), stream>>>(jobs, &st->err); count_launch();
    }
    CHAIN_LAUNCH_CHECK("entropy decode");
    T.mark("rans_decode", stream);
    // REL0 fixed-width with three narrow dimensions is read by the reconstruction
    // straight from its packing (no unpacked copy)
    RelBits relbits{};
    {
        const CompPlan& c = plan.comp[4];
        bool on = c.enc == kEncFixed && c.dims == 3 && D == 3;
        for (uint32_t d = 0; on && d < 3; ++d)
            on = c.width[d] <= 8 && c.minv[d] + ((1ull << c.width[d]) - 1) <= 0xffffffffull;
        if (on) {
            relbits.data = dcont;
            relbits.len = len;
            for (uint32_t d = 0; d < 3; ++d) {
                relbits.off[d] = c.packed_off[d];
                relbits.minv[d] = static_cast<uint32_t>(c.minv[d]);
                relbits.w[d] = c.width[d];
            }
            relbits.on = 1;
        }
    }
    // CH20 packed one bit per record with minimum 0 (values 0 and 1) is read bitwise by
    // the level-2 inverse
    const bool choice_packed =
        plan.comp[3].enc == kEncFixed && plan.comp[3].dims == 1 && plan.comp[3].width[0] == 1 && plan.comp[3].minv[0] == 0;
    // ---- tagged and fixed components
    for (int s = 0; s < kCodeStreams; ++s) {
        const CompPlan& c = plan.comp[s];
        const CompPlan* dc = &st->plan.comp[s];
        if ((s == 4 && relbits.on) || (s == 3 && choice_packed)) continue;
        if (c.enc == kEncFixed) {
            uint32_t wsum = 0;
            for (uint32_t d = 0; d < c.dims; ++d) wsum += c.width[d];
            const uint32_t G = std::max<uint32_t>(
                1, std::min<uint32_t>({16u, kUnpackWords / std::max<uint32_t>(wsum, 1), kUnpackWords / (32 * c.dims)}));
            k_unpack_fixed<<<dgrid((c.records + 32 * G - 1) / (32 * G), kUnpackWarps), 32 * kUnpackWarps, 0, stream>>>(
                dcont, len, dc, streams[s], st, G); count_launch();
        } else if (c.enc == kEncTagged) {
            uint32_t* tg = tags + tag_off[s];
            device_exclusive_scan<uint64_t>(TagIn{tg, c.dims},
                                            TagUnpackOut{dcont + c.tagged_off, tg, dc, streams[s], st, s}, c.records,
                                            scanbuf, static_cast<uint64_t*>(nullptr), stream);
        }
    }
    if (tags_total) k_check_tagged<<<1, 1, 0, stream>>>(st, st); count_launch();
    CHAIN_LAUNCH_CHECK("unpack");
    T.mark("unpack", stream);

    // ---- level 2 inverse: difference-record counts per tile, then per three dimensions
    // the tiles' reset-scan aggregates, their exclusive scan, and the records
    const uint64_t range = static_cast<uint64_t>(plan.wrap_max - plan.wrap_min) + 1;
    uint32_t* ndiff_dev = reinterpret_cast<uint32_t*>(misc + 1);
    const uint64_t l2tiles = flag_tiles(B);
    uint32_t* tile_diff = reinterpret_cast<uint32_t*>(scanbuf);
    L2Vec* tile_l2 = reinterpret_cast<L2Vec*>(reinterpret_cast<uint8_t*>(scanbuf) + ((4 * l2tiles + 15) & ~15ull));
    if (l2tiles) {
        // difference records per tile, scanned by the counting launch's last CTA
        if (choice_packed)
            k_choice_counts<<<static_cast<unsigned>(l2tiles), kFlagTile / 32, 0, stream>>>(
                dcont, len, plan.comp[3].packed_off[0], B, tile_diff, ndiff_dev, &st->done);
        else
            flag_count_kernel<ChoiceIn><<<static_cast<unsigned>(l2tiles), kFlagThreads, 0, stream>>>(
                ChoiceIn{streams[3]}, B, tile_diff, ndiff_dev, &st->done);
        count_launch();
        const ResetAddOp l2op{static_cast<uint32_t>(range), static_cast<uint32_t>(range >> 32)};
        L2Geo g;
        g.choice2 = streams[3];
        g.cbits = choice_packed ? dcont : nullptr;
        g.cbits_off = plan.comp[3].packed_off[0];
        g.cbits_len = len;
        g.keep = streams[2];
        g.diff = streams[1];
        g.tile_diff = tile_diff;
        g.B = B;
        g.D = D;
        g.range = range;
        g.wrap_min = plan.wrap_min;
        g.wrap_max = plan.wrap_max;
        const int64_t r = static_cast<int64_t>(range);
        g.maxc = r / 2 - ((r & 1) == 0 ? 1 : 0);
        g.minc = -(r / 2);
        // per device, cheap; set on every call, always to the same value
        const bool narrow = range <= (1ull << 31);
        if (narrow)
            CHAIN_CUDA(cudaFuncSetAttribute(k_l2_apply<ResetAddOp32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            static_cast<int>(kL2ApplySmem)));
        else
            CHAIN_CUDA(cudaFuncSetAttribute(k_l2_apply<ResetAddOp>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            static_cast<int>(kL2ApplySmem)));
        for (uint32_t d0 = 0; d0 < D; d0 += 3) {
            g.d0 = d0;
            k_l2_tail<<<static_cast<unsigned>(l2tiles), 32 * kL2Warps, 0, stream>>>(g, tile_l2); count_launch();
            scan_tilesums_kernel<L2Vec, ResetAddOp><<<1, 1024, 0, stream>>>(tile_l2, l2tiles, static_cast<L2Vec*>(nullptr),
                                                                           l2op); count_launch();
            if (narrow)
                k_l2_apply<ResetAddOp32><<<static_cast<unsigned>(l2tiles), 32 * kL2Warps, kL2ApplySmem, stream>>>(
                    g, tile_l2, compact, st);
            else
                k_l2_apply<ResetAddOp><<<static_cast<unsigned>(l2tiles), 32 * kL2Warps, kL2ApplySmem, stream>>>(
                    g, tile_l2, compact, st);
            count_launch();
        }
    } else {
        CHAIN_CUDA(cudaMemsetAsync(ndiff_dev, 0, sizeof(uint32_t), stream));
    }
    T.mark("level2_inverse", stream);
    // ---- level 1 inverse
    uint32_t* zeros_dev = reinterpret_cast<uint32_t*>(misc + 2);
    uint32_t* chained = drank;  // the choice ranks are no longer needed
    device_flag_scan(ZeroIn{streams[0]}, ZeroRankOut{streams[0], parent, chained, st, N}, N,
                     reinterpret_cast<uint32_t*>(scanbuf), zeros_dev, stream, &st->done);
    T.mark("zero_ranks", stream);
    int rounds = 1;
    while ((1ull << rounds) < N) ++rounds;
    // misc[16..31]: 32 flags; [0] = left unresolved by k_resolve, [r + 1] = after round r
    uint32_t* pending = reinterpret_cast<uint32_t*>(misc + 16);
    unsigned long long* resolve_next = reinterpret_cast<unsigned long long*>(misc + 3);   // zeroed above
    k_resolve<<<dgrid(N), 256, 0, stream>>>(parent, chained, zeros_dev, N, resolve_next, pending); count_launch();
    CHAIN_LAUNCH_CHECK("levels");
    T.mark("pointer_jump", stream);
    // ---- reconstruction (and exact corrections, and the copy to host memory)
    const bool soa = out_layout == CHAIN_SOA;
    const unsigned g = dgrid(N);
    const uint64_t ncx = plan.exc_count;
    const CorrIn cin{streams[kCorrGaps]};
    uint64_t* sb = scanbuf;
    auto reconstruct = [&]() -> chain_status {
        if (out_dtype == CHAIN_F64) {
            double* o = static_cast<double*>(dout);
            if (soa) {
                k_reconstruct<double, true><<<g, 256, 0, stream>>>(parent, compact, streams[4], st, st, o, relbits); count_launch();
                if (ncx) device_exclusive_scan<uint64_t>(cin, CorrOut<double, true>{streams[kCorrIds], dcont, st, st, o},
                                                         ncx, sb, static_cast<uint64_t*>(nullptr), stream);
            } else {
                k_reconstruct<double, false><<<g, 256, 0, stream>>>(parent, compact, streams[4], st, st, o, relbits); count_launch();
                if (ncx) device_exclusive_scan<uint64_t>(cin, CorrOut<double, false>{streams[kCorrIds], dcont, st, st, o},
                                                         ncx, sb, static_cast<uint64_t*>(nullptr), stream);
            }
        } else {
            float* o = static_cast<float*>(dout);
            if (soa) {
                k_reconstruct<float, true><<<g, 256, 0, stream>>>(parent, compact, streams[4], st, st, o, relbits); count_launch();
                if (ncx) device_exclusive_scan<uint64_t>(cin, CorrOut<float, true>{streams[kCorrIds], dcont, st, st, o},
                                                         ncx, sb, static_cast<uint64_t*>(nullptr), stream);
            } else {
                k_reconstruct<float, false><<<g, 256, 0, stream>>>(parent, compact, streams[4], st, st, o, relbits); count_launch();
                if (ncx) device_exclusive_scan<uint64_t>(cin, CorrOut<float, false>{streams[kCorrIds], dcont, st, st, o},
                                                         ncx, sb, static_cast<uint64_t*>(nullptr), stream);
            }
        }
        CHAIN_LAUNCH_CHECK("reconstruct");
        T.mark("reconstruct", stream);
        if (host_out) {
            CHAIN_CUDA(cudaMemcpyAsync(out, dout, nd * osz, cudaMemcpyDeviceToHost, stream));
            T.mark("d2h_points", stream);
        }
        return CHAIN_OK;
    };
    chain_status rs = reconstruct();
    if (rs != CHAIN_OK) return rs;
    uint32_t flags[2] = {0, 0};   // [0]: left unresolved by k_resolve; [1]: after the last round
    CHAIN_CUDA(cudaMemcpyAsync(flags, pending, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    CHAIN_CUDA(cudaStreamSynchronize(stream));
    if (flags[0]) {
        // Chains too long for one pass: pointer-jumping rounds, then reconstruct again.
        for (int r = 0; r < rounds; ++r) {
            k_jump<<<dgrid(N), 256, 0, stream>>>(parent, chained, zeros_dev, N, pending, r); count_launch();
        }
        CHAIN_LAUNCH_CHECK("levels");
        T.mark("pointer_jump_rounds", stream);
        rs = reconstruct();
        if (rs != CHAIN_OK) return rs;
        CHAIN_CUDA(cudaMemcpyAsync(flags + 1, pending + rounds, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    }
    CHAIN_CUDA(cudaMemcpyAsync(hs, st, offsetof(DecState, plan), cudaMemcpyDeviceToHost, stream));
    uint32_t counts[4] = {0, 0, 0, 0};
    CHAIN_CUDA(cudaMemcpyAsync(counts, misc + 1, 2 * sizeof(uint64_t), cudaMemcpyDeviceToHost, stream));
    CHAIN_CUDA(cudaStreamSynchronize(stream));
    T.finish();
    const uint32_t ndiff_seen = counts[0], zeros_seen = counts[2];
    if (hs->err || ndiff_seen != plan.comp[1].records || zeros_seen != B || flags[1])
        return set_err(CHAIN_ERR_CORRUPT_STREAM, "LCG2: invalid integer payload (flags " + std::to_string(hs->err) +
                                                     ")");
    return CHAIN_OK;
}

size_t decode_state_bytes() { return sizeof(DecState); }

}  // namespace chain
