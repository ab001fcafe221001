// Interleaved value-alphabet rANS for the Chain entropy stage.
//
// Replaces the reference's single-state CPU coder (RVN1, lcps_cpp.cpp:560-821 encode,
// :1620-1696 decode) and its nvCOMP ANS calls on the GPU path.  What is kept from the
// reference: the value alphabet (< 2^18 symbols), the precision rule
// prec = clamp(3*min(18, bitlen(#unique)+2)/2, 12, 20) (lcps_cpp.cpp:541-552), the
// state interval [4*2^prec, 1024*2^prec) with byte-wise renormalisation, and the
// compact probability-table tokens (lcps_cpp.cpp:686-729).  What is new: a symbol
// stream is cut into chunks; one warp codes one chunk with W interleaved states
// (W = lanes of the section, 1..32; symbol j of a chunk belongs to lane j % W), and
// the lanes' renormalisation bytes are interleaved in one byte stream per chunk in the
// exact order the decoding warp consumes them (lane order within a step, most
// significant byte first).  Small sections use fewer lanes, since each lane stores its
// final state (prec + 10 bits).
//
// Probability normalisation is this project's own exact-integer scheme (the
// reference's uses x87 long double): symbols with f_s * M / n < 1 get probability 1,
// the others share the remaining mass in proportion (round to nearest), and the
// rounding residue goes to the most probable symbol.  When that symbol cannot absorb
// it, an excess is removed proportionally from the reducible mass and then one unit
// at a time from the largest probabilities.
#pragma once

#include "chain_common.cuh"
#include "chain_format.h"

namespace chain {

struct RansTableDev {
    uint32_t alphabet;   // A; 0 = no table
    uint32_t prec;       // precision bits
    uint64_t n;          // symbols coded with this table
    double cost_bits;    // sum_s f_s * (prec - log2 p_s)
    uint32_t table_bytes;  // serialized token bytes (estimate before serialization)
    uint32_t pad;
};

__device__ inline int rans_precision_bits(uint64_t unique) {
    int u = bitlen64(unique) + 2;
    if (u > 18) u = 18;
    int p = (3 * u) / 2;
    return p < kRansMinPrec ? kRansMinPrec : (p > kRansMaxPrec ? kRansMaxPrec : p);
}

__device__ inline uint32_t rans_token_bytes(uint32_t p) { return 1u + (p >= (1u << 6)) + (p >= (1u << 14)); }

// One CTA of 1024 threads builds the normalised table of one histogram.
//   hist[A] symbol counts (A = alphabet), n = sum(hist)
//   prob[A], cum[A] outputs; *desc receives precision, cost estimate and table size.
constexpr int kTableThreads = 1024;

__device__ inline void table_block_argmax(const uint32_t* prob, uint32_t A, uint32_t* sh_best) {
    // Largest probability; ties go to the largest symbol index.
    uint64_t best = 0;
    for (uint32_t s = threadIdx.x; s < A; s += blockDim.x) {
        const uint64_t key = (static_cast<uint64_t>(prob[s]) << 32) | s;
        if (prob[s] && key > best) best = key;
    }
    best = warp_max(best);
    __shared__ uint64_t wbest[32];
    if ((threadIdx.x & 31) == 0) wbest[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint64_t b = threadIdx.x < (blockDim.x >> 5) ? wbest[threadIdx.x] : 0;
        b = warp_max(b);
        if (threadIdx.x == 0) *sh_best = static_cast<uint32_t>(b & 0xffffffffu);
    }
    __syncthreads();
}

// Tables of up to kTableStageSyms symbols are built in shared memory (the builder makes
// a dozen passes over the histogram and the probabilities).
constexpr uint32_t kTableStageSyms = 16384;
constexpr size_t kTableStageBytes = 2ull * kTableStageSyms * 4;

// Copies n u32 global -> shared with the whole CTA, eight loads in flight per thread.
__device__ __forceinline__ void block_copy32(uint32_t* __restrict__ dst, const uint32_t* __restrict__ src,
                                             uint32_t n) {
    constexpr int kDepth = 8;
    for (uint32_t i0 = threadIdx.x; i0 < n; i0 += blockDim.x * kDepth) {
        uint32_t v[kDepth];
#pragma unroll
        for (int u = 0; u < kDepth; ++u) {
            const uint32_t i = i0 + u * blockDim.x;
            if (i < n) v[u] = __ldg(src + i);
        }
#pragma unroll
        for (int u = 0; u < kDepth; ++u) {
            const uint32_t i = i0 + u * blockDim.x;
            if (i < n) dst[i] = v[u];
        }
    }
}

// Sums of a, b and c over the CTA with one pass of barriers; scratch holds 99 values.
__device__ inline void block_sum3(uint64_t& a, uint64_t& b, uint64_t& c, uint64_t* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    c = warp_sum(c);
    if (lane == 0) { scratch[warp] = a; scratch[33 + warp] = b; scratch[66 + warp] = c; }
    __syncthreads();
    if (warp == 0) {
        uint64_t x = lane < nw ? scratch[lane] : 0, y = lane < nw ? scratch[33 + lane] : 0,
                 z = lane < nw ? scratch[66 + lane] : 0;
        x = warp_sum(x);
        y = warp_sum(y);
        z = warp_sum(z);
        if (lane == 0) { scratch[32] = x; scratch[65] = y; scratch[98] = z; }
    }
    __syncthreads();
    a = scratch[32];
    b = scratch[65];
    c = scratch[98];
    __syncthreads();
}

// stage: kTableStageBytes of shared memory, or null (work in global memory).
__device__ inline void build_rans_table(const uint32_t* __restrict__ hist_in, uint32_t A, uint64_t n,
                                        uint32_t* __restrict__ prob_out, uint32_t* __restrict__ cum,
                                        RansTableDev* desc, uint32_t* stage) {
    __shared__ uint64_t red[99];
    __shared__ double redd[33];
    __shared__ uint32_t sh_best;
    __shared__ uint64_t sh_sum;
    if (A == 0 || n == 0) {
        if (threadIdx.x == 0) {
            desc->alphabet = 0; desc->prec = 0; desc->n = 0; desc->cost_bits = 0; desc->table_bytes = 0;
        }
        return;
    }
    const bool staged = stage && A <= kTableStageSyms;
    const uint32_t* hist = hist_in;
    uint32_t* prob = prob_out;
    if (staged) {
        block_copy32(stage, hist_in, A);
        hist = stage;
        prob = stage + kTableStageSyms;
        __syncthreads();
    }
    uint64_t uniq = 0;
    for (uint32_t s = threadIdx.x; s < A; s += blockDim.x) uniq += hist[s] != 0;
    uniq = block_reduce_sum(uniq, red);
    const int prec = rans_precision_bits(uniq);
    const uint64_t M = 1ull << prec;
    // Symbols with f * M / n < 1 are pinned to probability 1; the remaining mass is
    // shared by the others in proportion (rounded to nearest), re-pinning any that
    // round to 0.  The rounding residue then goes to the most probable symbol.
    constexpr uint32_t kPin = 0x80000000u;
    uint64_t pinned = 0, pinned_f = 0;
    for (uint32_t s = threadIdx.x; s < A; s += blockDim.x) {
        const uint64_t f = hist[s];
        const bool pin = f && f * M < n;
        pinned += pin;
        pinned_f += pin ? f : 0;
        prob[s] = pin ? (kPin | 1u) : 0u;
    }
    uint64_t unused = 0;
    block_sum3(pinned, pinned_f, unused, red);
    uint64_t sum = 0;
    for (int round = 0; round < 16; ++round) {
        const uint64_t budget = M - pinned, rest = n - pinned_f;
        uint64_t newly = 0, newly_f = 0, free_sum = 0;
        for (uint32_t s = threadIdx.x; s < A; s += blockDim.x) {
            const uint64_t f = hist[s];
            if (!f || (prob[s] & kPin) || rest == 0) continue;
            const uint64_t p = (2 * f * budget + rest) / (2 * rest);
            if (p == 0) {
                prob[s] = kPin | 1u;
                ++newly;
                newly_f += f;
            } else {
                prob[s] = static_cast<uint32_t>(p);
                free_sum += p;
            }
        }
        block_sum3(newly, newly_f, free_sum, red);
        pinned += newly;
        pinned_f += newly_f;
        sum = pinned + free_sum;
        if (newly == 0) break;
    }
    for (uint32_t s = threadIdx.x; s < A; s += blockDim.x) prob[s] &= ~kPin;
    __syncthreads();
    if (sum != M) {
        table_block_argmax(prob, A, &sh_best);
        const int64_t fixed = static_cast<int64_t>(prob[sh_best]) + static_cast<int64_t>(M) - static_cast<int64_t>(sum);
        __syncthreads();
        if (fixed >= 1) {
            if (threadIdx.x == 0) prob[sh_best] = static_cast<uint32_t>(fixed);
            sum = M;
        }
        __syncthreads();
    }
    if (sum < M) {
        table_block_argmax(prob, A, &sh_best);
        if (threadIdx.x == 0) prob[sh_best] += static_cast<uint32_t>(M - sum);
        __syncthreads();
    } else if (sum > M) {
        // Excess E <= sum - uniq = reducible mass R because M >= uniq (M >= 4 * uniq by
        // the precision rule), so a valid table always exists.
        for (int round = 0; round < 64; ++round) {
            if (threadIdx.x == 0) sh_sum = sum;
            __syncthreads();
            const uint64_t E = sh_sum - M;
            if (E == 0) break;
            uint64_t R = 0;
            for (uint32_t s = threadIdx.x; s < A; s += blockDim.x) R += prob[s] > 1 ? prob[s] - 1 : 0;
            R = block_reduce_sum(R, red);
            uint64_t cut_total = 0;
            for (uint32_t s = threadIdx.x; s < A; s += blockDim.x) {
                if (prob[s] > 1) {
                    const uint64_t c = (static_cast<uint64_t>(prob[s] - 1) * E) / R;
                    prob[s] -= static_cast<uint32_t>(c);
                    cut_total += c;
                }
            }
            cut_total = block_reduce_sum(cut_total, red);
            sum -= cut_total;
            if (cut_total == 0) {
                // Then E < number of reducible symbols: take one unit from each of the E
                // largest keys (p << 32 | s) among symbols with p > 1.  The E-th largest
                // key is found by binary search on the key value.
                uint64_t lo = 0, hi = (static_cast<uint64_t>(M) << 32) | 0xffffffffull;
                while (lo < hi) {
                    const uint64_t mid = lo + (hi - lo + 1) / 2;
                    uint64_t cnt = 0;
                    for (uint32_t s = threadIdx.x; s < A; s += blockDim.x)
                        cnt += prob[s] > 1 && ((static_cast<uint64_t>(prob[s]) << 32) | s) >= mid;
                    cnt = block_reduce_sum(cnt, red);
                    if (cnt >= E) lo = mid; else hi = mid - 1;
                }
                for (uint32_t s = threadIdx.x; s < A; s += blockDim.x)
                    if (prob[s] > 1 && ((static_cast<uint64_t>(prob[s]) << 32) | s) >= lo) prob[s] -= 1;
                __syncthreads();
                sum -= E;
            }
        }
    }
    __syncthreads();
    // cumulative frequencies (exclusive prefix), the cost estimate and the token bytes
    double cost = 0.0;
    uint64_t tbytes = 0;
    uint64_t carry;
    const auto symbol = [&](uint32_t s, uint64_t p) {
        if (p) {
            // log2(1) = 0 exactly: probability-1 symbols need no logarithm
            const double lg = p == 1 ? 0.0 : log2(static_cast<double>(p));
            cost += static_cast<double>(hist[s]) * (static_cast<double>(prec) - lg);
            tbytes += rans_token_bytes(static_cast<uint32_t>(p));
        } else if (s == 0 || prob[s - 1] != 0) {
            tbytes += 1;  // start of a zero run (runs longer than 64 are counted below)
        }
    };
    if (A <= blockDim.x) {   // one symbol per thread
        const uint32_t s = threadIdx.x;
        const uint64_t p = s < A ? prob[s] : 0;
        const uint64_t c = block_exclusive_sum(p, red, &carry);
        if (s < A) {
            cum[s] = static_cast<uint32_t>(c);
            symbol(s, p);
        }
    } else {
        // warp w owns a contiguous range of the symbols and walks it 32 consecutive
        // symbols at a time (bank-conflict-free in shared memory, coalesced in global);
        // one block scan of the warps' totals gives the ranges' offsets
        const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
        const uint32_t span = ((A + nw - 1) / nw + 31) & ~31u;
        const uint32_t c0 = min(A, warp * span), c1 = min(A, c0 + span);
        uint64_t wsum = 0;
        for (uint32_t b = c0; b < c1; b += 32) wsum += b + lane < c1 ? prob[b + lane] : 0u;
        wsum = warp_sum(wsum);
        uint64_t c = block_exclusive_sum<uint64_t>(lane == 0 ? wsum : 0, red, &carry);
        c = __shfl_sync(0xffffffffu, c, 0);
        for (uint32_t b = c0; b < c1; b += 32) {
            const uint32_t s = b + lane;
            const uint64_t p = s < c1 ? prob[s] : 0u;
            const uint64_t inc = warp_inclusive_sum(p);
            if (s < c1) {
                cum[s] = static_cast<uint32_t>(c + inc - p);
                symbol(s, p);
            }
            c += __shfl_sync(0xffffffffu, inc, 31);
        }
    }
    if (staged)
        for (uint32_t s = threadIdx.x; s < A; s += blockDim.x) prob_out[s] = prob[s];
    uint64_t zeros = 0;
    for (uint32_t s = threadIdx.x; s < A; s += blockDim.x) zeros += prob[s] == 0;
    block_sum3(zeros, tbytes, unused, red);
    // deterministic FP sum: fixed per-thread order, then a fixed tree
    {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cost += __shfl_xor_sync(0xffffffffu, cost, o);
        if (lane == 0) redd[warp] = cost;
        __syncthreads();
        if (warp == 0) {
            double c = lane < static_cast<int>(blockDim.x >> 5) ? redd[lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
            if (lane == 0) redd[32] = c;
        }
        __syncthreads();
        cost = redd[32];
    }
    if (threadIdx.x == 0) {
        desc->alphabet = A;
        desc->prec = static_cast<uint32_t>(prec);
        desc->n = n;
        desc->cost_bits = cost;
        desc->table_bytes = static_cast<uint32_t>(tbytes + zeros / 64);
        if (carry != M) desc->alphabet = 0xFFFFFFFFu;  // internal error marker
    }
    __syncthreads();
}

// Probability-table tokens (the scheme of lcps_cpp.cpp:686-729 without the leading
// alphabet varint, which the section header carries):
//   p in [1, 2^6):   1 byte  p<<2
//   p in [2^6,2^14): 2 bytes (p<<2)|1, p>>6
//   p in [2^14, ..): 3 bytes (p<<2)|2, p>>6, p>>14
//   zero run of k in [1, 64]: 1 byte ((k-1)<<2)|3
// Both directions run with a whole CTA.

// ------------------------------------------------------------ parallel tables

// Block-wide inclusive max-scan for blockDim.x <= 1024 (values >= 0).
__device__ inline uint32_t block_inclusive_max(uint32_t v, uint32_t* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v = t > v ? t : v;
    }
    if (lane == 31) scratch[warp] = v;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < nwarps ? scratch[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w = t > w ? t : w;
        }
        if (lane < nwarps) scratch[lane] = w;
    }
    __syncthreads();
    const uint32_t before = warp ? scratch[warp - 1] : 0u;
    __syncthreads();
    return before > v ? before : v;
}

// Serialises prob[0..A) into tokens with the whole CTA.  Returns the byte count (in
// every thread).  A zero at s starts a token when (s - run_start) % 64 == 0; the
// token covers up to 64 zeros of its run.
constexpr uint32_t kSerStageSyms = 16384;   // alphabets serialized from a shared-memory copy
__device__ inline uint32_t serialize_table_block(const uint32_t* prob_in, uint32_t A, uint8_t* out, uint32_t* stage) {
    __shared__ uint32_t mscratch[33];
    __shared__ uint64_t sscratch[33];
    // the zero-run lookahead below is a chain of dependent reads: serve it from shared
    // memory (`stage`, kSerStageSyms u32) when the alphabet fits
    const uint32_t* prob = prob_in;
    if (A <= kSerStageSyms) {
        for (uint32_t i = threadIdx.x; i < A; i += blockDim.x) stage[i] = prob_in[i];
        __syncthreads();
        prob = stage;
    }
    uint32_t carry_last = 0;   // (index of the last nonzero so far) + 1
    uint64_t carry_off = 0;
    for (uint32_t base = 0; base < A; base += blockDim.x) {
        const uint32_t s = base + threadIdx.x;
        const uint32_t p = s < A ? prob[s] : 1u;
        // run start of a zero = 1 + index of the last nonzero before it
        uint32_t key = (s < A && p != 0) ? s + 1 : 0u;
        uint32_t incl = block_inclusive_max(key, mscratch);
        incl = incl > carry_last ? incl : carry_last;
        uint32_t size = 0, extra = 0;
        if (s < A) {
            if (p) {
                extra = (p >= (1u << 6)) + (p >= (1u << 14));
                size = 1 + extra;
            } else {
                const uint32_t run_start = incl;   // no nonzero at s, so incl excludes s
                if (((s - run_start) & 63u) == 0) {
                    uint32_t k = 0;
                    while (k < 63 && s + k + 1 < A && prob[s + k + 1] == 0) ++k;
                    extra = k;
                    size = 1;
                }
            }
        }
        uint64_t tot;
        const uint64_t off = carry_off + block_exclusive_sum(static_cast<uint64_t>(size), sscratch, &tot);
        if (size) {
            if (p) {
                out[off] = static_cast<uint8_t>((p << 2) | extra);
                for (uint32_t b = 0; b < extra; ++b) out[off + 1 + b] = static_cast<uint8_t>(p >> (8 * (b + 1) - 2));
            } else {
                out[off] = static_cast<uint8_t>((extra << 2) | 3u);
            }
        }
        carry_off += tot;
        // carry for the next chunk: the max over this chunk's keys
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) mscratch[32] = incl;
        __syncthreads();
        carry_last = mscratch[32];
        __syncthreads();
    }
    return static_cast<uint32_t>(carry_off);
}

// Token length and symbol count from a token's first byte.
__device__ __forceinline__ void token_shape(uint8_t first, uint32_t* bytes, uint32_t* syms) {
    const uint32_t t = first & 3u;
    if (t == 3u) { *bytes = 1; *syms = (first >> 2) + 1; }
    else { *bytes = 1 + t; *syms = 1; }
}

constexpr uint32_t kParseSeg = 16;
constexpr uint32_t kParseStage = 49152;   // token bytes staged in shared memory up to this length
constexpr uint32_t kParseStageScratch = 8 * (kParseStage / kParseSeg + 2);   // u32 scratch of a staged parse
constexpr uint32_t kParseProbSyms = 16384;   // alphabets whose probabilities are built in shared memory
constexpr uint32_t kParseSmem = kParseStage + 4 * kParseStageScratch + 4 * kParseProbSyms;   // dynamic shared bytes

// Segment entry maps: where the next segment's first token starts (offset 0, 1 or 2)
// as a function of where this segment's first token starts, 2 bits per entry offset.
// (a after b)(e) = a(b(e)).
constexpr uint32_t kEntryMapId = 0u | (1u << 2) | (2u << 4);
__device__ __forceinline__ uint32_t entry_map_after(uint32_t a, uint32_t b) {
    uint32_t h = 0;
#pragma unroll
    for (uint32_t e = 0; e < 3; ++e) h |= ((a >> (2 * ((b >> (2 * e)) & 3u))) & 3u) << (2 * e);
    return h;
}
// Exclusive block scan of entry maps in thread order: the composition of the maps of
// all lower threads (kEntryMapId for thread 0).  Every thread of the CTA calls it.
__device__ __forceinline__ uint32_t block_entry_map_prefix(uint32_t m, uint32_t* s_warp) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
    uint32_t inc = m;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t prev = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc = entry_map_after(inc, prev);
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {   // the warps' maps scanned by one warp
        uint32_t wi = lane < nwarps ? s_warp[lane] : kEntryMapId;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t prev = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi = entry_map_after(wi, prev);
        }
        const uint32_t we = __shfl_up_sync(0xffffffffu, wi, 1);
        __syncwarp();
        if (lane < nwarps) s_warp[lane] = lane ? we : kEntryMapId;
    }
    __syncthreads();
    const uint32_t pre = s_warp[warp];
    const uint32_t exc_lane = __shfl_up_sync(0xffffffffu, inc, 1);
    return lane ? entry_map_after(exc_lane, pre) : pre;
}

__device__ __forceinline__ uint32_t clamp_u32(uint64_t v) {
    return static_cast<uint32_t>(v > 0xffffffffull ? 0xffffffffull : v);
}

// Parses tokens with the whole CTA.  Every 16-byte segment is parsed speculatively
// from each of its 3 possible entry offsets (a token is at most 3 bytes); a block scan
// of the segments' entry maps gives the true entries, a scan gives each segment's first
// symbol, and the segments are parsed again for real.  Token walks are chains of
// dependent reads, so a table of up to kParseStage bytes is first copied to shared
// memory (`stage`, kParseStage bytes) and its scratch kept there too (`stage_scratch`,
// kParseStageScratch u32); larger ones use `global_scratch`, 8 * (len / 16 + 2) u32.
// A staged table of at most kParseProbSyms symbols builds its probabilities in shared
// memory (`sprob`, kParseProbSyms u32) and scans them there, four per thread, so that
// prob and cum leave with coalesced stores (a single CTA streaming them through global
// memory with per-thread runs was the slowest part of the parse).
// Returns false (in every thread) on malformed input.
__device__ inline bool parse_table_block(const uint8_t* in_global, uint32_t len, uint32_t A, uint32_t prec,
                                         uint32_t* prob, uint32_t* cum, uint32_t* global_scratch, uint8_t* stage,
                                         uint32_t* stage_scratch, uint32_t* sprob) {
    __shared__ int s_ok;
    __shared__ uint64_t sscratch[33];
    __shared__ uint32_t s_wmap[32];
    const uint8_t* in = in_global;
    uint32_t* scratch = global_scratch;
    const bool staged = len <= kParseStage;
    const bool shared_prob = staged && A <= kParseProbSyms;
    constexpr uint32_t kScanRound = 4 * 1024;   // symbols per round of the shared scan (blockDim.x = 1024)
    const uint32_t a_pad = (A + kScanRound - 1) / kScanRound * kScanRound;
    if (staged) {
        constexpr int kDepth = 8;   // loads in flight per thread
        for (uint32_t i0 = threadIdx.x; i0 < len; i0 += blockDim.x * kDepth) {
            uint8_t v[kDepth];
#pragma unroll
            for (int u = 0; u < kDepth; ++u) {
                const uint32_t i = i0 + u * blockDim.x;
                v[u] = i < len ? in_global[i] : 0;
            }
#pragma unroll
            for (int u = 0; u < kDepth; ++u) {
                const uint32_t i = i0 + u * blockDim.x;
                if (i < len) stage[i] = v[u];
            }
        }
        in = stage;   // the __syncthreads below orders the copy before the reads
        scratch = stage_scratch;
    }
    if (shared_prob)   // the scan reads whole rounds: symbols A .. a_pad count zero
        for (uint32_t i = A + threadIdx.x; i < a_pad; i += blockDim.x) sprob[i] = 0;
    const uint32_t nseg = (len + kParseSeg - 1) / kParseSeg;
    uint32_t* ex = scratch;              // [nseg][3] exit offset into the next segment
    uint32_t* cnt = scratch + 3 * nseg;  // [nseg][3] symbols
    uint32_t* entry = scratch + 6 * nseg;
    uint32_t* first_sym = scratch + 7 * nseg;
    if (threadIdx.x == 0) s_ok = (len > 0 && A > 0) ? 1 : 0;
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < nseg; k += blockDim.x) {
        const uint32_t beg = k * kParseSeg, end = min(beg + kParseSeg, len);
        for (uint32_t e = 0; e < 3; ++e) {
            uint32_t pos = beg + e, c = 0;
            while (pos < end) {
                uint32_t b, sy;
                token_shape(in[pos], &b, &sy);
                pos += b;
                c += sy;
            }
            ex[3 * k + e] = pos - end;   // 0..2 (may point past len; checked below)
            cnt[3 * k + e] = c;
        }
    }
    __syncthreads();
    {
        // entry[k] = (F_{k-1} after ... after F_0)(0), F_k(e) = ex[3 k + e]: each thread
        // composes a contiguous run of segments, a block scan of the runs' maps gives each
        // run's entry, and the thread walks its run
        const uint32_t per = (nseg + blockDim.x - 1) / blockDim.x;
        const uint32_t k0 = min(nseg, threadIdx.x * per), k1 = min(nseg, k0 + per);
        uint32_t mine = kEntryMapId;
        for (uint32_t k = k0; k < k1; ++k)
            mine = entry_map_after(ex[3 * k] | (ex[3 * k + 1] << 2) | (ex[3 * k + 2] << 4), mine);
        uint32_t e = block_entry_map_prefix(mine, s_wmap) & 3u;
        for (uint32_t k = k0; k < k1; ++k) {
            entry[k] = e;
            e = ex[3 * k + e];
        }
    }
    __syncthreads();
    // the last segment, entered at its entry, must end exactly at len (an entry past
    // the end of a short last segment leaves a nonzero exit too)
    if (threadIdx.x == 0 && nseg && ex[3 * (nseg - 1) + entry[nseg - 1]] != 0) s_ok = 0;
    __syncthreads();
    if (!s_ok) return false;
    // first symbol of each segment
    uint64_t carry = 0;
    for (uint32_t base = 0; base < nseg; base += blockDim.x) {
        const uint32_t k = base + threadIdx.x;
        const uint64_t c = k < nseg ? cnt[3 * k + entry[k]] : 0;
        uint64_t tot;
        const uint64_t ex_sum = block_exclusive_sum(c, sscratch, &tot);
        if (k < nseg) first_sym[k] = clamp_u32(carry + ex_sum);
        carry += tot;
    }
    if (carry != A) return false;   // uniform: every thread computed the same total
    const uint64_t M = 1ull << prec;
    uint32_t* dst = shared_prob ? sprob : prob;
    for (uint32_t k = threadIdx.x; k < nseg; k += blockDim.x) {
        const uint32_t end = min((k + 1) * kParseSeg, len);
        uint32_t pos = k * kParseSeg + entry[k], s = first_sym[k];
        bool ok = true;
        while (pos < end && ok) {
            const uint8_t first = in[pos];
            uint32_t b, sy;
            token_shape(first, &b, &sy);
            if (pos + b > len || s + sy > A) { ok = false; break; }
            if ((first & 3u) == 3u) {
                for (uint32_t j = 0; j < sy; ++j) dst[s + j] = 0;
            } else {
                uint32_t p = first >> 2;
                for (uint32_t j = 1; j < b; ++j) p |= static_cast<uint32_t>(in[pos + j]) << (6 + 8 * (j - 1));
                if (p == 0 || p > M) ok = false;
                dst[s] = p;
            }
            pos += b;
            s += sy;
        }
        if (!ok) atomicExch(&s_ok, 0);
    }
    __syncthreads();
    if (!s_ok) return false;
    if (shared_prob) {
        // cumulative table in shared memory (the segment scratch is free now): rounds of
        // four consecutive symbols per thread and one block scan, then prob and cum out
        uint32_t* scum = scratch;
        uint64_t run = 0;
        for (uint32_t base = 0; base < a_pad; base += 4 * blockDim.x) {
            const uint32_t i = base + 4 * threadIdx.x;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (i < a_pad) v = *reinterpret_cast<const uint4*>(sprob + i);
            uint64_t tot;
            uint64_t c = run + block_exclusive_sum(static_cast<uint64_t>(v.x) + v.y + v.z + v.w, sscratch, &tot);
            if (i < a_pad) {
                uint4 o;
                o.x = clamp_u32(c); c += v.x;
                o.y = clamp_u32(c); c += v.y;
                o.z = clamp_u32(c); c += v.z;
                o.w = clamp_u32(c);
                *reinterpret_cast<uint4*>(scum + i) = o;
            }
            run += tot;
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < A; i += blockDim.x) {
            prob[i] = sprob[i];
            cum[i] = scum[i];
        }
        return run == M;
    }
    // cumulative table and total: each thread sums a contiguous run of symbols (read
    // eight at a time), one block scan gives the runs' offsets
    const uint32_t per = (A + blockDim.x - 1) / blockDim.x;
    const uint32_t s0 = threadIdx.x * per, s1 = min(A, s0 + per);
    uint64_t run = 0;
    for (uint32_t b = s0; b < s1; b += 8) {
        uint32_t v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = b + u < s1 ? prob[b + u] : 0u;
#pragma unroll
        for (int u = 0; u < 8; ++u) run += v[u];
    }
    uint64_t total;
    uint64_t c = block_exclusive_sum(run, sscratch, &total);
    for (uint32_t b = s0; b < s1; b += 8) {
        uint32_t v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = b + u < s1 ? prob[b + u] : 0u;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            if (b + u < s1) cum[b + u] = clamp_u32(c);
            c += v[u];
        }
    }
    return total == M;
}

// ----------------------------------------------------------------------------- coding
// A rANS section is coded as `chunks` chunks of S symbols (S a multiple of 32; the last
// chunk may be shorter).  Per chunk: W final states and one byte stream.
// Encoder symbol entry (division-free encoding by a precomputed reciprocal, the
// division-by-invariant-integer method as used in F. Giesen's public-domain rans_byte):
//   x' = x + bias + q * cmpl_freq,  q = umulhi(x, rcp_freq) >> rcp_shift = floor(x / freq)
// For freq == 1: rcp_freq = 2^32 - 1, shift 0 (q = x - 1 for x >= 1) and bias = cum + M - 1.
// Exact for x < 2^31 (here x < 1024 * freq <= 2^30).
__device__ __forceinline__ uint4 make_enc_symbol(uint32_t freq, uint32_t cum, uint32_t prec) {
    const uint32_t M = 1u << prec;
    if (freq < 2) return make_uint4(freq, cum + M - 1, 0xffffffffu, (M - freq));
    uint32_t shift = 0;
    while (freq > (1u << shift)) ++shift;
    const uint32_t rcp = static_cast<uint32_t>(((1ull << (shift + 31)) + freq - 1) / freq);
    return make_uint4(freq, cum, rcp, (M - freq) | ((shift - 1) << 24));
}

struct RansJob {
    const uint4* etab;        // encode: symbol entries [A] (make_enc_symbol)
    const void* sym;          // encode: symbols, sym_esz bytes each (1, 2 or 4)
    uint32_t* out;            // decode: symbol output
    uint64_t count;           // symbols
    const uint32_t* prob;     // [A]
    const uint32_t* cum;      // [A]
    const uint4* image;       // decode: the job's shared-memory tables (dec_image_bytes), 16-byte aligned
    const uint64_t* slots;    // decode, tables without an image: slot -> pack_slot(symbol, freq, slot - cum) [M]
    uint32_t prec;
    uint32_t alphabet;
    uint32_t chunks;
    uint32_t lanes;           // interleaved states per chunk (1..32)
    uint32_t first_block;     // first CTA of this job (kRansEncWarps / kRansDecWarps chunks per CTA)
    uint32_t sym_esz;         // encode: bytes per symbol (1, 2 or 4)
    uint64_t S;               // symbols per chunk (multiple of 32)
    uint8_t* bytes;           // encode: chunk slots (slot_cap each); decode: container
    uint64_t bytes_len;       // decode: container length (staged loads stay inside it)
    uint64_t slot_cap;        // encode only
    const uint64_t* chunk_off;  // decode: absolute byte offset of each chunk (chunks + 1)
    uint32_t* chunk_len;      // encode: bytes per chunk
    uint32_t* states;         // encode: the section's final lane states, packed at state_bits(prec)
                              // each (MSB first, big-endian 32-bit words, zeroed beforehand);
                              // decode: unpacked states in
};

constexpr int kMaxRansJobs = 16;
constexpr int kRansEncWarps = 8;              // chunks (warps) per encoder CTA
constexpr int kRansDecWarps = 8;              // chunks (warps) per decoder CTA (shares its table image)
constexpr int kRansTile = 32;                 // steps per staged tile
constexpr uint32_t kSmemTableSyms = 4096;     // decoder prob/cum in shared memory up to this alphabet
constexpr uint32_t kSmemEncSyms = 2048;       // encoder entries (16 B) in shared memory up to this alphabet
constexpr uint32_t kSmemLookupSlots = 16384;  // u16 decode lookup in shared memory up to this M
constexpr uint32_t kBucketBits = 13;          // bucketed decode: 2^13 buckets of slots ...
constexpr uint32_t kBucketMaxSyms = 16384;    // ... for M above kSmemLookupSlots and alphabets up to this
constexpr uint32_t kWindow = 4096;            // decoder byte window per warp
constexpr uint32_t kLargeTableMaxSteps = 512; // serial depth of lanes whose tables are not in shared memory
constexpr uint64_t kLargeTableMinSymbols = 1ull << 18;  // ... on streams at least this long
// Below this many symbols a large-table stream's lanes go to kLargeTableShortSteps: the
// frame's chunks then still fill less than one wave of the decoder (about 16 chunk warps
// per SM), so the shorter chain is the shorter kernel; above it, more chunks would add a
// wave.
constexpr uint64_t kLargeTableDeepSymbols = 1ull << 23;
constexpr uint32_t kLargeTableShortSteps = 256;

// Decoder slot entry for tables kept in global memory: one load per step gives the
// symbol, its frequency and slot - cum[symbol].
__host__ __device__ inline uint64_t pack_slot(uint32_t sym, uint32_t freq, uint32_t bias) {
    return static_cast<uint64_t>(sym) | (static_cast<uint64_t>(freq) << 18) | (static_cast<uint64_t>(bias) << 39);
}

// Bucketed decode (tables too large for a shared-memory slot lookup): the slot range is
// cut into 2^kBucketBits buckets; bucket b's first-slot owner and the cumulative table
// sit in shared memory, and a step binary-searches the symbols between the owners of
// bucket b's and bucket b+1's first slots.  The same rule decides it on every side.
__host__ __device__ inline bool rans_dec_bucketed(uint32_t prec, uint32_t alphabet) {
    return (1u << prec) > kSmemLookupSlots && alphabet <= kBucketMaxSyms;
}
constexpr uint32_t kBucketCount = 1u << kBucketBits;

// A decoder job's shared-memory tables, built once per section in global memory by the
// table stage and copied verbatim by every CTA of the job:
//   bucketed:        u32 cum[A + 1] (cum[A] = M), padded to 16 B; u16 owner[2^kBucketBits + 1]
//   M <= 16384, A <= 65536 (u16 symbols):
//                    A <= kSmemTableSyms: uint2 {prob, cum}[A], padded to 64 B; u16 look[M]
//                    else:                u16 look[M] (prob and cum read from global memory)
//   otherwise:       none (one packed global slot entry per step)
__host__ __device__ inline bool rans_dec_smem_look(uint32_t prec, uint32_t alphabet) {
    return (1u << prec) <= kSmemLookupSlots && alphabet <= 65536;
}
__host__ __device__ inline uint32_t dec_cum_bytes(uint32_t alphabet) { return ((alphabet + 1 + 3) & ~3u) * 4; }
__host__ __device__ inline uint32_t dec_tab_bytes(uint32_t alphabet) {
    return alphabet <= kSmemTableSyms ? ((alphabet + 7) & ~7u) * 8 : 0;
}
__host__ __device__ inline uint32_t dec_image_bytes(uint32_t prec, uint32_t alphabet) {
    if (rans_dec_bucketed(prec, alphabet)) return (dec_cum_bytes(alphabet) + (kBucketCount + 1) * 2 + 15) & ~15u;
    if (rans_dec_smem_look(prec, alphabet)) return (dec_tab_bytes(alphabet) + (2u << prec) + 15) & ~15u;
    return 0;
}

// Copies n16 16-byte words global -> shared with the whole CTA, eight loads in flight
// per thread.
__device__ __forceinline__ void block_copy16(uint4* __restrict__ dst, const uint4* __restrict__ src, uint32_t n16) {
    constexpr int kDepth = 8;
    for (uint32_t i0 = threadIdx.x; i0 < n16; i0 += blockDim.x * kDepth) {
        uint4 v[kDepth];
#pragma unroll
        for (int u = 0; u < kDepth; ++u) {
            const uint32_t i = i0 + u * blockDim.x;
            if (i < n16) v[u] = __ldg(src + i);
        }
#pragma unroll
        for (int u = 0; u < kDepth; ++u) {
            const uint32_t i = i0 + u * blockDim.x;
            if (i < n16) dst[i] = v[u];
        }
    }
}

// Shared memory is sized per launch: the largest table of this launch that fits the
// shared-memory limits, plus staging.
struct RansJobs {
    RansJob job[kMaxRansJobs];
    uint32_t njobs;
    uint32_t total_blocks;
    uint32_t tab_cap;      // encode: tables with alphabet <= tab_cap live in shared memory
    uint32_t table_bytes;  // decode: the largest job image (shared-memory bytes before the windows)
};

inline void rans_plan_smem(RansJobs& J, bool decode) {
    uint32_t tab = 0, image = 0;
    for (uint32_t j = 0; j < J.njobs; ++j) {
        const uint32_t A = J.job[j].alphabet;
        if (!decode && A <= kSmemEncSyms && A > tab) tab = A;
        if (decode) {
            const uint32_t b = dec_image_bytes(J.job[j].prec, A);
            if (b > image) image = b;
        }
    }
    J.tab_cap = (tab + 7) & ~7u;
    J.table_bytes = image;
}
inline size_t rans_enc_smem(const RansJobs& J) {
    return J.tab_cap * 16ull + kRansEncWarps * (kRansTile * 32 * 4 + kWindow);
}
inline size_t rans_dec_smem(const RansJobs& J) {
    return J.table_bytes + kRansDecWarps * kWindow + 16;   // +16: 3-byte renorm reads
}

// Largest dynamic shared memory any launch of the two kernels can request.  The kernels'
// MaxDynamicSharedMemorySize attribute is set to exactly these values: the attribute is
// global to the process, so contexts used from several threads at once must never set
// different values (a smaller one set between another thread's set and launch would make
// that launch fail).
// Two decoder CTAs of the largest size still fit one SM (228 KB less 1 KB per CTA).
constexpr size_t kRansEncSmemMax =
    kSmemEncSyms * 16ull + kRansEncWarps * kRansTile * 32 * 4 + kRansEncWarps * kWindow;
constexpr size_t kDecDirectBytes = kSmemTableSyms * 8ull + kSmemLookupSlots * 2ull;
constexpr size_t kDecBucketBytes = (((kBucketMaxSyms + 1 + 3) & ~3ull) * 4 + (kBucketCount + 1) * 2 + 15) & ~15ull;
constexpr size_t kRansDecSmemMax =
    (kDecDirectBytes > kDecBucketBytes ? kDecDirectBytes : kDecBucketBytes) + kRansDecWarps * kWindow + 16;
static_assert(2 * (kRansDecSmemMax + 1024 + 16) <= 228 * 1024, "two decoder CTAs per SM");

__device__ __forceinline__ int job_of_block(const RansJobs& J) {
    int j = 0;
    while (j + 1 < static_cast<int>(J.njobs) && blockIdx.x >= J.job[j + 1].first_block) ++j;
    return j;
}

// Register layouts of a loaded symbol tile (tile_load -> tile_store).
enum TileLayout : int {
    kTileScalar = 0,   // r[i]      = symbol tb + lane + 32 i
    kTileVec4 = 1,     // r[4i + k] = symbol tb + 4 (lane + 32 i) + k
    kTileVec16 = 2,    // r[16i + k] = symbol tb + 16 (lane + 32 i) + k
    kTileVec8 = 3,     // r[8i + k]  = symbol tb + 8 (lane + 32 i) + k
};

// Loads symbols [tb, te) (a tile of up to 1024) of esz bytes each into regs; full,
// aligned tiles use 16-byte loads.
__device__ __forceinline__ void tile_load(const void* sym_v, uint32_t esz, uint64_t tb, uint64_t te,
                                          uint32_t (&r)[32], int& layout) {
    const int lane = threadIdx.x & 31;
    const bool full = te - tb == 1024;
    if (esz == 1) {
        const uint8_t* sym = static_cast<const uint8_t*>(sym_v);
        if (full && (reinterpret_cast<uintptr_t>(sym + tb) & 15) == 0) {
            layout = kTileVec16;
            const uint4* p = reinterpret_cast<const uint4*>(sym + tb);
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const uint4 v = __ldg(p + lane + 32 * i);
                const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int k = 0; k < 16; ++k) r[16 * i + k] = (w[k >> 2] >> (8 * (k & 3))) & 0xFFu;
            }
        } else {
            layout = kTileScalar;
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                const uint64_t k = tb + lane + 32 * i;
                r[i] = k < te ? static_cast<uint32_t>(__ldg(sym + k)) : 0u;
            }
        }
        return;
    }
    if (esz == 2) {
        const uint16_t* sym = static_cast<const uint16_t*>(sym_v);
        if (full && (reinterpret_cast<uintptr_t>(sym + tb) & 15) == 0) {
            layout = kTileVec8;
            const uint4* p = reinterpret_cast<const uint4*>(sym + tb);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const uint4 v = __ldg(p + lane + 32 * i);
                const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int k = 0; k < 8; ++k) r[8 * i + k] = (w[k >> 1] >> (16 * (k & 1))) & 0xFFFFu;
            }
        } else {
            layout = kTileScalar;
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                const uint64_t k = tb + lane + 32 * i;
                r[i] = k < te ? static_cast<uint32_t>(__ldg(sym + k)) : 0u;
            }
        }
        return;
    }
    const uint32_t* sym = static_cast<const uint32_t*>(sym_v);
    if (full && (reinterpret_cast<uintptr_t>(sym + tb) & 15) == 0) {
        layout = kTileVec4;
        const uint4* p = reinterpret_cast<const uint4*>(sym + tb);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const uint4 v = __ldg(p + lane + 32 * i);
            r[4 * i] = v.x; r[4 * i + 1] = v.y; r[4 * i + 2] = v.z; r[4 * i + 3] = v.w;
        }
    } else {
        layout = kTileScalar;
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            const uint64_t k = tb + lane + 32 * i;
            r[i] = k < te ? __ldg(sym + k) : 0u;
        }
    }
}
// Stores a loaded tile to buf in symbol order (buf[j] = symbol tb + j).
__device__ __forceinline__ void tile_store(uint32_t* buf, const uint32_t (&r)[32], int layout) {
    const int lane = threadIdx.x & 31;
    if (layout == kTileVec4) {
        uint4* p = reinterpret_cast<uint4*>(buf);
#pragma unroll
        for (int i = 0; i < 8; ++i) p[lane + 32 * i] = make_uint4(r[4 * i], r[4 * i + 1], r[4 * i + 2], r[4 * i + 3]);
    } else if (layout == kTileVec8) {
        uint4* p = reinterpret_cast<uint4*>(buf);
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int q = 0; q < 2; ++q)
                p[2 * (lane + 32 * i) + q] =
                    make_uint4(r[8 * i + 4 * q], r[8 * i + 4 * q + 1], r[8 * i + 4 * q + 2], r[8 * i + 4 * q + 3]);
    } else if (layout == kTileVec16) {
        uint4* p = reinterpret_cast<uint4*>(buf);
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int q = 0; q < 4; ++q)
                p[4 * (lane + 32 * i) + q] =
                    make_uint4(r[16 * i + 4 * q], r[16 * i + 4 * q + 1], r[16 * i + 4 * q + 2], r[16 * i + 4 * q + 3]);
    } else {
#pragma unroll
        for (int i = 0; i < 32; ++i) buf[lane + 32 * i] = r[i];
    }
}

// Encoder entry of symbol s (from shared memory when the table is there).
template <bool kSmem>
__device__ __forceinline__ uint4 enc_entry(const uint4* tab, const uint4* etab, uint32_t s) {
    return kSmem ? tab[s] : __ldg(etab + s);
}

// One encoding step of a lane with entry e: renormalise (0..3 bytes, written at the
// warp's descending window position in lane order) and push the symbol.
__device__ __forceinline__ uint32_t rans_encode_step(uint32_t x, const uint4& e, bool act, uint8_t* ow,
                                                     uint32_t& rel, uint32_t lt) {
    const uint32_t xmax = e.x << 10;  // ((L >> prec) << 8) * freq
    const uint32_t nb = act ? (x >= xmax) + ((x >> 8) >= xmax) + ((x >> 16) >= xmax) : 0u;
    const uint32_t b0 = __ballot_sync(0xffffffffu, nb & 1u), b1 = __ballot_sync(0xffffffffu, nb & 2u);
    rel -= __popc(b0) + 2 * __popc(b1);
    uint8_t* o = ow + rel + __popc(b0 & lt) + 2 * __popc(b1 & lt);
    if (nb > 0) o[nb - 1] = static_cast<uint8_t>(x);
    if (b1) {   // some lane emits two or three bytes (rare: skipped warp-uniformly)
        if (nb > 1) o[nb - 2] = static_cast<uint8_t>(x >> 8);
        if (nb > 2) o[0] = static_cast<uint8_t>(x >> 16);
    }
    if (act) {
        x >>= 8 * nb;
        const uint32_t q = __umulhi(x, e.z) >> (e.w >> 24);
        x = x + e.y + q * (e.w & 0xffffffu);
    }
    return x;
}

// A full tile (kRansTile steps, every lane active, W == 32), steps in descending order.
// Symbol entries do not depend on the state, so they are fetched four steps ahead.
template <bool kSmem>
__device__ __forceinline__ uint32_t rans_encode_full_tile(uint32_t x, const uint32_t* cur, const uint4* tab,
                                                          const uint4* etab, uint8_t* ow, uint32_t& rel,
                                                          uint32_t lt) {
    const int lane = threadIdx.x & 31;
    constexpr int kAhead = 4;
    uint4 pf[kAhead];
#pragma unroll
    for (int i = 0; i < kAhead; ++i) pf[i] = enc_entry<kSmem>(tab, etab, cur[(kRansTile - 1 - i) * 32 + lane]);
#pragma unroll
    for (int i = 0; i < kRansTile; ++i) {
        const int j = kRansTile - 1 - i;   // step within the tile
        const uint4 e = pf[i % kAhead];
        if (j >= kAhead) pf[i % kAhead] = enc_entry<kSmem>(tab, etab, cur[(j - kAhead) * 32 + lane]);
        x = rans_encode_step(x, e, true, ow, rel, lt);
    }
    return x;
}

// Encoder: one warp per chunk, kRansEncWarps chunks of one job per CTA.  The job's table
// sits in shared memory when small; the next 32-step tile of symbols is loaded into
// registers while the current one is coded from the warp's shared-memory tile buffer,
// then stored there (one buffer per warp; eight warps per CTA, two CTAs per SM); the
// warp's byte counts are prefix-summed with two ballots
// (0..3 bytes per lane).  Bytes are written backwards into a kWindow-byte shared-memory
// window; before each group of kRansTile steps, if fewer than a group's worst case
// (kRansTile * 96 bytes) are free, the window's 16-byte-aligned written part goes to
// the chunk's slot in global memory with 16-byte stores and the ragged rest (< 16
// bytes) moves to the window's top.  A chunk whose bytes exceed its slot is detected
// after the group that overflowed, before anything reaches global memory.  Offsets are
// 32-bit (a chunk slot is < 4 GB).
static __global__ void __launch_bounds__(32 * kRansEncWarps) rans_encode_kernel(RansJobs J, uint32_t* err) {
    extern __shared__ __align__(16) uint8_t rsm[];
    const RansJob& jb = J.job[job_of_block(J)];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint4* tab = reinterpret_cast<uint4*>(rsm);
    const bool smem_tab = jb.alphabet <= J.tab_cap;
    if (smem_tab) block_copy16(tab, jb.etab, jb.alphabet);
    __syncthreads();
    const uint32_t c = (blockIdx.x - jb.first_block) * kRansEncWarps + warp;
    if (c >= jb.chunks) return;
    uint32_t* buf = reinterpret_cast<uint32_t*>(rsm + J.tab_cap * 16ull) + warp * 1024;
    uint8_t* ow = rsm + J.tab_cap * 16ull + kRansEncWarps * kRansTile * 32 * 4 + warp * kWindow;
    const uint64_t cbeg = static_cast<uint64_t>(c) * jb.S;
    const uint64_t cend = min(cbeg + jb.S, jb.count);
    const uint32_t W = jb.lanes;
    const uint32_t cnt = static_cast<uint32_t>(cend - cbeg);
    const uint32_t steps = (cnt + W - 1) / W;
    const uint32_t full_steps = W == 32 ? cnt / 32 : 0;   // steps in which every lane codes a symbol
    const uint32_t ntiles = (steps + kRansTile - 1) / kRansTile;
    const uint64_t tile_syms = static_cast<uint64_t>(kRansTile) * W;
    const uint32_t prec = jb.prec;
    const uint32_t L = 4u << prec;
    const uint32_t lt = lanemask_lt();
    constexpr uint32_t kGroupBytes = kRansTile * 32 * 3;
    uint32_t x = L;
    uint8_t* out = jb.bytes + static_cast<uint64_t>(c) * jb.slot_cap;
    const bool ovec = (reinterpret_cast<uintptr_t>(out) & 15) == 0 && (jb.slot_cap & 15) == 0;
    uint32_t wtop = static_cast<uint32_t>(jb.slot_cap);   // slot offset of the window's end
    uint32_t rel = kWindow;                               // window index of the lowest byte written
    bool overflow = false;
    uint32_t r[32];
    int layout;
    {
        const uint64_t tb = cbeg + tile_syms * (ntiles - 1);
        tile_load(jb.sym, jb.sym_esz, tb, min(tb + tile_syms, cend), r, layout);
        tile_store(buf, r, layout);
        __syncwarp();
    }
    for (int k = static_cast<int>(ntiles) - 1; k >= 0; --k) {
        if (k > 0) {
            const uint64_t tb = cbeg + tile_syms * (k - 1);
            tile_load(jb.sym, jb.sym_esz, tb, min(tb + tile_syms, cend), r, layout);
        }
        if (rel < kGroupBytes) {   // flush the aligned part of the window
            const uint32_t a = (rel + 15) & ~15u;
            const int64_t gb = static_cast<int64_t>(wtop) - kWindow;   // window index i <-> slot offset gb + i
            if (ovec) {
                for (uint32_t i = a + 16 * lane; i < kWindow; i += 16 * 32)
                    *reinterpret_cast<uint4*>(out + (gb + i)) = *reinterpret_cast<const uint4*>(ow + i);
            } else {
                for (uint32_t i = a + lane; i < kWindow; i += 32) out[gb + i] = ow[i];
            }
            const uint32_t h = a - rel;
            const uint8_t hb = static_cast<uint32_t>(lane) < h ? ow[rel + lane] : 0;
            __syncwarp();
            if (static_cast<uint32_t>(lane) < h) ow[kWindow - h + lane] = hb;
            __syncwarp();
            wtop -= kWindow - a;
            rel = kWindow - h;
        }
        const uint32_t* cur = buf;
        if (static_cast<uint32_t>(32 * k + 32) <= full_steps) {
            x = smem_tab ? rans_encode_full_tile<true>(x, cur, tab, jb.etab, ow, rel, lt)
                         : rans_encode_full_tile<false>(x, cur, tab, jb.etab, ow, rel, lt);
        } else {
            const int t_hi = min(static_cast<int>(steps) - 1, 32 * k + 31);
            uint32_t kl = static_cast<uint32_t>(t_hi) * W + lane;   // symbol index within the chunk
            for (int t = t_hi; t >= 32 * k; --t, kl -= W) {
                const bool act = static_cast<uint32_t>(lane) < W && kl < cnt;
                const uint32_t s = act ? cur[(t - 32 * k) * W + lane] : 0u;
                const uint4 e = smem_tab ? tab[s] : __ldg(jb.etab + s);
                x = rans_encode_step(x, e, act, ow, rel, lt);
            }
        }
        if (kWindow - rel > wtop) {   // the chunk's bytes no longer fit its slot
            overflow = true;
            break;
        }
        if (k > 0) {
            __syncwarp();
            tile_store(buf, r, layout);   // the tile just coded is no longer needed
            __syncwarp();
        }
    }
    if (__any_sync(0xffffffffu, overflow)) {
        if (lane == 0) set_error(err, kErrInternal);
        return;
    }
    __syncwarp();
    const int64_t gb = static_cast<int64_t>(wtop) - kWindow;
    for (uint32_t i = rel + lane; i < kWindow; i += 32) out[gb + i] = ow[i];
    if (static_cast<uint32_t>(lane) < W) {
        // final state of lane (c, lane) at bits [i B, i B + B) of the section's packed states;
        // neighbouring chunks share boundary words, so the bits are OR-ed in (byte order
        // swapped: OR commutes with the swap)
        const uint32_t B = state_bits(prec);
        const uint64_t o = (static_cast<uint64_t>(c) * W + lane) * B;
        uint32_t* words = jb.states + (o >> 5);
        const int shift = 32 - static_cast<int>(o & 31) - static_cast<int>(B);
        if (shift >= 0) {
            atomicOr(words, __byte_perm(x << shift, 0, 0x0123));
        } else {
            atomicOr(words, __byte_perm(x >> -shift, 0, 0x0123));
            atomicOr(words + 1, __byte_perm(x << (32 + shift), 0, 0x0123));
        }
    }
    if (lane == 0) jb.chunk_len[c] = static_cast<uint32_t>(jb.slot_cap - (gb + rel));
}

// Refills a warp's byte window so that it starts at `pos` rounded down to 16 bytes.
__device__ __forceinline__ void window_fill(uint8_t* win, const uint8_t* bytes, uint64_t len, uint64_t wbase) {
    const int lane = threadIdx.x & 31;
    const bool vec = wbase + kWindow <= len && ((reinterpret_cast<uintptr_t>(bytes + wbase) & 15) == 0);
    if (vec) {
        const uint4* p = reinterpret_cast<const uint4*>(bytes + wbase);
        uint4* w = reinterpret_cast<uint4*>(win);
#pragma unroll
        for (int i = 0; i < static_cast<int>(kWindow / 16 / 32); ++i) w[lane + 32 * i] = __ldg(p + lane + 32 * i);
    } else {
        for (uint32_t i = lane; i < kWindow; i += 32) {
            const uint64_t a = wbase + i;
            win[i] = a < len ? bytes[a] : 0;
        }
    }
    __syncwarp();
}

// Where a decoder reads its tables: slot lookup and prob/cum in shared memory; lookup
// in shared memory and prob/cum in global memory; or one packed global slot entry.
enum RansDecMode { kDecSmemAll = 0, kDecSmemLook = 1, kDecBucket = 2, kDecGlobalSlots = 3 };

// Decodes steps [t0, t0 + tn) of a chunk (all lanes active when kFull; then tn ==
// kRansTile).  The state stays in [L, 256 L) for any byte stream: a step leaves
// f * (x >> prec) + (slot - cum) >= 4 and renormalisation shifts in the fewest bytes
// that restore x >= L; so no per-step range check is needed.  Reads stay inside the
// window (plus its 16-byte tail) because a group starts with at least kRansTile * 96
// bytes left in it; running past the chunk's end is detected once per group.
template <int kMode, bool kFull>
__device__ __forceinline__ uint32_t rans_decode_group(uint32_t x, uint32_t& rel, uint32_t& k, uint32_t tn,
                                                      const uint8_t* __restrict__ win,
                                                      const uint16_t* __restrict__ look,
                                                      const uint2* __restrict__ tab, const RansJob& jb,
                                                      uint32_t* __restrict__ outc, uint32_t W, uint32_t cnt,
                                                      uint32_t prec, uint32_t L, uint32_t lt) {
    const uint32_t mask = (1u << prec) - 1;
    const bool lane_in = (threadIdx.x & 31) < W;
#pragma unroll 4
    for (uint32_t t = 0; t < (kFull ? static_cast<uint32_t>(kRansTile) : tn); ++t, k += W) {
        const uint32_t slot = x & mask;
        uint32_t s, xn;
        if (kMode == kDecSmemAll) {
            s = look[slot];
            const uint2 e = tab[s];
            xn = e.x * (x >> prec) + slot - e.y;
        } else if (kMode == kDecSmemLook) {
            s = look[slot];
            xn = __ldg(jb.prob + s) * (x >> prec) + slot - __ldg(jb.cum + s);
        } else if (kMode == kDecBucket) {
            // look = bucket owners [kBucketCount + 1], tab = cumulative table [A + 1]
            const uint32_t* cum = reinterpret_cast<const uint32_t*>(tab);
            const uint32_t b = slot >> (prec - kBucketBits);
            uint32_t lo = look[b], hi = look[b + 1];
            while (lo < hi) {   // last symbol with cum <= slot: the owner
                const uint32_t mid = (lo + hi + 1) >> 1;
                if (cum[mid] <= slot) lo = mid; else hi = mid - 1;
            }
            s = lo;
            const uint32_t c0 = cum[lo];
            xn = (cum[lo + 1] - c0) * (x >> prec) + slot - c0;
        } else {
            const uint64_t e = __ldg(jb.slots + slot);
            s = static_cast<uint32_t>(e & 0x3ffffu);
            xn = static_cast<uint32_t>((e >> 18) & 0x1fffffu) * (x >> prec) + static_cast<uint32_t>(e >> 39);
        }
        if (kFull) {
            outc[k] = s;
        } else {
            const bool act = lane_in && k < cnt;
            if (act) outc[k] = s;
            xn = act ? xn : x;   // an idle lane keeps x >= L and so reads nothing
        }
        const uint32_t nb = (xn < L) + (xn < (L >> 8)) + (xn < (L >> 16));
        const uint32_t b0 = __ballot_sync(0xffffffffu, nb & 1u), b1 = __ballot_sync(0xffffffffu, nb & 2u);
        const uint32_t wo = rel + __popc(b0 & lt) + 2 * __popc(b1 & lt);
        rel += __popc(b0) + 2 * __popc(b1);
        const uint32_t v = (static_cast<uint32_t>(win[wo]) << 16) | (static_cast<uint32_t>(win[wo + 1]) << 8) |
                           static_cast<uint32_t>(win[wo + 2]);
        x = (xn << (8 * nb)) | (v >> (24 - 8 * nb));
    }
    return x;
}

// Decodes one chunk: groups of kRansTile steps, the window refilled before a group
// whenever fewer than kRansTile * 96 bytes (the most a group can consume) remain in it.
// Returns false when the byte stream ran past the chunk's end.
template <int kMode>
__device__ __forceinline__ bool rans_decode_chunk(uint32_t& x, uint64_t& wbase, uint32_t& rel, uint64_t end,
                                                  uint8_t* win, const uint16_t* look, const uint2* tab,
                                                  const RansJob& jb, uint32_t* outc, uint32_t W, uint32_t cnt,
                                                  uint32_t steps, uint32_t prec, uint32_t L) {
    constexpr uint32_t kGroupBytes = kRansTile * 32 * 3;   // most bytes one group of steps consumes
    static_assert(kWindow >= kGroupBytes + 16, "window must hold a group's bytes after a refill");
    const uint32_t lt = lanemask_lt();
    const uint32_t full_steps = W == 32 ? cnt / 32 : 0;   // steps in which every lane codes a symbol
    uint32_t rel_end = static_cast<uint32_t>(min(end - wbase, static_cast<uint64_t>(1u << 30)));
    uint32_t k = threadIdx.x & 31;   // symbol index within the chunk: t * W + lane
    for (uint32_t t0 = 0; t0 < steps; t0 += kRansTile) {
        if (rel > kWindow - kGroupBytes) {
            __syncwarp();
            const uint64_t p = wbase + rel;
            wbase = p & ~15ull;
            rel = static_cast<uint32_t>(p - wbase);
            rel_end = static_cast<uint32_t>(min(end - wbase, static_cast<uint64_t>(1u << 30)));
            window_fill(win, jb.bytes, jb.bytes_len, wbase);
        }
        if (t0 + kRansTile <= full_steps)
            x = rans_decode_group<kMode, true>(x, rel, k, kRansTile, win, look, tab, jb, outc, W, cnt, prec, L, lt);
        else
            x = rans_decode_group<kMode, false>(x, rel, k, min(static_cast<uint32_t>(kRansTile), steps - t0), win,
                                                look, tab, jb, outc, W, cnt, prec, L, lt);
        if (rel > rel_end) return false;
    }
    return true;
}

// Decoder: one warp per chunk, kRansDecWarps chunks of one job per CTA.  The slot->symbol
// lookup and prob/cum live in shared memory when small, the bucket owners and the
// cumulative table when the lookup is too large; the chunk's byte stream is read
// through a kWindow-byte shared-memory window.  Offsets inside a group are 32-bit and
// relative to the window; each lane renormalises by reading 3 bytes unconditionally and
// shifting in the nb it needs.  A malformed stream (initial state out of range, overrun,
// or a final state or position that does not match) sets kErrCorrupt.
static __global__ void __launch_bounds__(32 * kRansDecWarps) rans_decode_kernel(RansJobs J, uint32_t* err) {
    extern __shared__ __align__(16) uint8_t rsm[];
    __shared__ int s_skip;
    if (threadIdx.x == 0) s_skip = *err != 0;  // a failed table parse leaves no valid lookup
    __syncthreads();
    if (s_skip) return;
    const RansJob& jb = J.job[job_of_block(J)];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t prec = jb.prec;
    const uint32_t L = 4u << prec;
    uint8_t* win = rsm + J.table_bytes + warp * kWindow;
    const bool bucketed = rans_dec_bucketed(prec, jb.alphabet);
    const bool smem_look = rans_dec_smem_look(prec, jb.alphabet);
    const bool smem_tab = smem_look && jb.alphabet <= kSmemTableSyms;
    const uint2* tab = reinterpret_cast<const uint2*>(rsm);   // bucketed: the u32 cumulative table
    const uint16_t* look = reinterpret_cast<const uint16_t*>(
        rsm + (bucketed ? dec_cum_bytes(jb.alphabet) : dec_tab_bytes(jb.alphabet)));
    block_copy16(reinterpret_cast<uint4*>(rsm), jb.image, dec_image_bytes(prec, jb.alphabet) / 16);
    __syncthreads();
    const uint32_t c = (blockIdx.x - jb.first_block) * kRansDecWarps + warp;
    if (c >= jb.chunks) return;
    const uint64_t cbeg = static_cast<uint64_t>(c) * jb.S;
    const uint64_t cend = min(cbeg + jb.S, jb.count);
    const uint32_t W = jb.lanes;
    const uint32_t cnt = static_cast<uint32_t>(cend - cbeg);   // symbols of this chunk (S < 2^32)
    const uint32_t steps = (cnt + W - 1) / W;
    uint32_t* outc = jb.out + cbeg;
    const uint64_t pos = jb.chunk_off[c];
    const uint64_t end = jb.chunk_off[c + 1];
    uint32_t x = static_cast<uint32_t>(lane) < W ? jb.states[static_cast<uint64_t>(c) * W + lane] : L;
    bool bad = (x < L) || (static_cast<uint64_t>(x) >= (static_cast<uint64_t>(L) << 8)) || end > jb.bytes_len ||
               pos > end;
    if (__any_sync(0xffffffffu, bad)) {
        if (lane == 0) set_error(err, kErrCorrupt);
        return;
    }
    uint64_t wbase = pos & ~15ull;
    uint32_t rel = static_cast<uint32_t>(pos - wbase);
    window_fill(win, jb.bytes, jb.bytes_len, wbase);
    bool ok;
    if (bucketed)
        ok = rans_decode_chunk<kDecBucket>(x, wbase, rel, end, win, look, tab, jb, outc, W, cnt, steps, prec, L);
    else if (smem_look && smem_tab)
        ok = rans_decode_chunk<kDecSmemAll>(x, wbase, rel, end, win, look, tab, jb, outc, W, cnt, steps, prec, L);
    else if (smem_look)
        ok = rans_decode_chunk<kDecSmemLook>(x, wbase, rel, end, win, look, tab, jb, outc, W, cnt, steps, prec, L);
    else
        ok = rans_decode_chunk<kDecGlobalSlots>(x, wbase, rel, end, win, look, tab, jb, outc, W, cnt, steps, prec, L);
    bad = !ok || (x != L) || (wbase + rel != end);
    if (__any_sync(0xffffffffu, bad) && lane == 0) set_error(err, kErrCorrupt);
}

}  // namespace chain
