// Interleaved value-alphabet rANS for the Chain entropy stage.
//
// Replaces the reference's single-state CPU coder (RVN1, lcps_cpp.cpp:560-821 encode,
// :1620-1696 decode) and its nvCOMP ANS calls on the GPU path.  What is kept from the
// reference: the value alphabet (< 2^18 symbols), the precision rule
// prec = clamp(3*min(18, bitlen(#unique)+2)/2, 12, 20) (lcps_cpp.cpp:541-552), the
// state interval [4*2^prec, 1024*2^prec) with byte-wise renormalisation, and the
// compact probability-table tokens (lcps_cpp.cpp:686-729).  What is new: a symbol
// stream is cut into chunks; one warp codes one chunk with 32 interleaved states
// (symbol j of a chunk belongs to lane j % 32), and the lanes' renormalisation bytes
// are interleaved in one byte stream per chunk in the exact order the decoding warp
// consumes them (lane order within a step, most significant byte first).
//
// Probability normalisation is this project's own exact-integer scheme (the
// reference's uses x87 long double): p_s = max(1, round(f_s * M / n)); a deficit goes
// to the most probable symbol; an excess is removed proportionally from the
// reducible mass and then one unit at a time from the largest probabilities.
#pragma once

#include "chain_common.cuh"

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

__device__ inline void build_rans_table(const uint32_t* __restrict__ hist, uint32_t A, uint64_t n,
                                        uint32_t* __restrict__ prob, uint32_t* __restrict__ cum,
                                        RansTableDev* desc) {
    __shared__ uint64_t red[33];
    __shared__ double redd[33];
    __shared__ uint32_t sh_best;
    __shared__ uint64_t sh_sum;
    if (A == 0 || n == 0) {
        if (threadIdx.x == 0) {
            desc->alphabet = 0; desc->prec = 0; desc->n = 0; desc->cost_bits = 0; desc->table_bytes = 0;
        }
        return;
    }
    uint64_t uniq = 0;
    for (uint32_t s = threadIdx.x; s < A; s += blockDim.x) uniq += hist[s] != 0;
    uniq = block_reduce_sum(uniq, red);
    const int prec = rans_precision_bits(uniq);
    const uint64_t M = 1ull << prec;
    uint64_t sum = 0;
    for (uint32_t s = threadIdx.x; s < A; s += blockDim.x) {
        const uint64_t f = hist[s];
        uint64_t p = f ? (2 * f * M + n) / (2 * n) : 0;
        if (f && p == 0) p = 1;
        prob[s] = static_cast<uint32_t>(p);
        sum += p;
    }
    sum = block_reduce_sum(sum, red);
    __syncthreads();
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
    // cumulative frequencies (exclusive prefix) and the cost estimate
    uint64_t carry = 0;
    double cost = 0.0;
    uint64_t tbytes = 0;
    for (uint32_t base = 0; base < A; base += blockDim.x) {
        const uint32_t s = base + threadIdx.x;
        const uint64_t p = s < A ? prob[s] : 0;
        uint64_t tot;
        const uint64_t ex = block_exclusive_sum(p, red, &tot);
        if (s < A) {
            cum[s] = static_cast<uint32_t>(carry + ex);
            if (p) {
                cost += static_cast<double>(hist[s]) * (static_cast<double>(prec) - log2(static_cast<double>(p)));
                tbytes += rans_token_bytes(static_cast<uint32_t>(p));
            } else if (s == 0 || prob[s - 1] != 0) {
                tbytes += 1;  // start of a zero run (runs longer than 64 are counted below)
            }
        }
        carry += tot;
    }
    uint64_t zeros = 0;
    for (uint32_t s = threadIdx.x; s < A; s += blockDim.x) zeros += prob[s] == 0;
    zeros = block_reduce_sum(zeros, red);
    tbytes = block_reduce_sum(tbytes, red);
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

// Serialises a probability table into tokens (single thread).  Token forms:
//   p in [1, 2^6):  1 byte  p<<2
//   p in [2^6,2^14):2 bytes (p<<2)|1, p>>6
//   p in [2^14,..): 3 bytes (p<<2)|2, p>>6, p>>14
//   zero run of k in [1,64]: 1 byte ((k-1)<<2)|3
// Returns the number of bytes written.
__device__ inline uint32_t serialize_table(const uint32_t* prob, uint32_t A, uint8_t* out) {
    uint32_t o = 0;
    for (uint32_t s = 0; s < A; ++s) {
        const uint32_t p = prob[s];
        if (p == 0) {
            uint32_t extra = 0;
            while (extra < 63 && s + extra + 1 < A && prob[s + extra + 1] == 0) ++extra;
            out[o++] = static_cast<uint8_t>((extra << 2) | 3u);
            s += extra;
            continue;
        }
        const uint32_t eb = (p >= (1u << 6)) + (p >= (1u << 14));
        out[o++] = static_cast<uint8_t>((p << 2) | eb);
        for (uint32_t b = 0; b < eb; ++b) out[o++] = static_cast<uint8_t>(p >> (8 * (b + 1) - 2));
    }
    return o;
}

// Parses tokens back (single thread).  Returns false on malformed input.
__host__ __device__ inline bool parse_table(const uint8_t* in, uint32_t len, uint32_t A, uint32_t prec,
                                            uint32_t* prob, uint32_t* cum) {
    uint32_t o = 0, s = 0;
    uint64_t sum = 0;
    const uint64_t M = 1ull << prec;
    while (s < A) {
        if (o >= len) return false;
        const uint8_t first = in[o++];
        const uint32_t tok = first & 3u;
        if (tok == 3u) {
            const uint32_t k = (first >> 2) + 1;
            if (k > A - s) return false;
            for (uint32_t j = 0; j < k; ++j) { prob[s] = 0; cum[s] = static_cast<uint32_t>(sum); ++s; }
            continue;
        }
        uint32_t p = first >> 2;
        for (uint32_t b = 0; b < tok; ++b) {
            if (o >= len) return false;
            p |= static_cast<uint32_t>(in[o++]) << (6 + 8 * b);
        }
        if (p == 0 || p > M - sum) return false;
        prob[s] = p;
        cum[s] = static_cast<uint32_t>(sum);
        sum += p;
        ++s;
    }
    return o == len && sum == M;
}

// ----------------------------------------------------------------------------- coding
// A rANS section is coded as `chunks` chunks of S symbols (S a multiple of 32; the last
// chunk may be shorter).  Per chunk: 32 final states and one byte stream.
struct RansJob {
    const uint32_t* sym;      // symbols (encode input / decode output)
    uint64_t count;           // symbols
    const uint32_t* prob;     // [A]
    const uint32_t* cum;      // [A]
    const uint32_t* lookup;   // decode: slot -> symbol [M]
    uint32_t prec;
    uint32_t chunks;
    uint64_t S;               // symbols per chunk
    uint8_t* bytes;           // encode: chunk slots (slot_cap each); decode: section payload
    uint64_t slot_cap;        // encode only
    const uint64_t* chunk_off;  // decode: byte offset of each chunk in `bytes` (chunks+1)
    uint32_t* chunk_len;      // encode: bytes per chunk
    uint32_t* states;         // encode: out [chunks*32]; decode: in
    uint32_t* out;            // decode: symbol output
    uint32_t first_chunk;     // global chunk index of this job's chunk 0
    uint32_t pad;
};

constexpr int kMaxRansJobs = 16;
struct RansJobs {
    RansJob job[kMaxRansJobs];
    uint32_t njobs;
    uint32_t total_chunks;
};

__device__ inline int find_job(const RansJobs& J, uint32_t g) {
    int j = 0;
    while (j + 1 < static_cast<int>(J.njobs) && g >= J.job[j + 1].first_chunk) ++j;
    return j;
}

// One warp per chunk; any grid (warps stride over the global chunk list).
static __global__ void __launch_bounds__(128) rans_encode_kernel(RansJobs J, uint32_t* err) {
    const int lane = threadIdx.x & 31;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t g = gw; g < J.total_chunks; g += nw) {
        const RansJob& jb = J.job[find_job(J, g)];
        const uint32_t c = g - jb.first_chunk;
        const uint64_t cbeg = static_cast<uint64_t>(c) * jb.S;
        const uint64_t cend = min(cbeg + jb.S, jb.count);
        const uint32_t steps = static_cast<uint32_t>((cend - cbeg + 31) / 32);
        const uint32_t prec = jb.prec;
        const uint32_t L = 4u << prec;
        uint32_t x = L;
        uint8_t* out = jb.bytes + static_cast<uint64_t>(c) * jb.slot_cap;
        uint64_t pos = jb.slot_cap;
        bool overflow = false;
        for (int t = static_cast<int>(steps) - 1; t >= 0; --t) {
            const uint64_t k = cbeg + static_cast<uint64_t>(t) * 32 + lane;
            const bool act = k < cend;
            uint32_t nb = 0, f = 1, cm = 0;
            if (act) {
                const uint32_t s = __ldg(jb.sym + k);
                f = __ldg(jb.prob + s);
                cm = __ldg(jb.cum + s);
                const uint32_t xmax = f << 10;  // ((L >> prec) << 8) * f
                uint32_t y = x;
                while (y >= xmax) { y >>= 8; ++nb; }
            }
            const uint32_t inc = warp_inclusive_sum(nb);
            const uint32_t total = __shfl_sync(0xffffffffu, inc, 31);
            if (total > pos) { overflow = true; break; }
            const uint64_t base = pos - total + (inc - nb);
            for (uint32_t j = 0; j < nb; ++j) out[base + j] = static_cast<uint8_t>(x >> (8 * (nb - 1 - j)));
            pos -= total;
            if (act) {
                x >>= 8 * nb;
                x = (x / f) * (1u << prec) + (x % f) + cm;
            }
        }
        if (__any_sync(0xffffffffu, overflow)) {
            if (lane == 0) set_error(err, kErrInternal);
            continue;
        }
        jb.states[static_cast<uint64_t>(c) * 32 + lane] = x;
        if (lane == 0) jb.chunk_len[c] = static_cast<uint32_t>(jb.slot_cap - pos);
    }
}

// One warp per chunk.  Every read is bounds-checked against the chunk's byte range;
// a malformed stream sets kErrCorrupt and the warp stops.
static __global__ void __launch_bounds__(128) rans_decode_kernel(RansJobs J, uint32_t* err) {
    if (*err) return;  // a failed table parse leaves no valid lookup table
    const int lane = threadIdx.x & 31;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t g = gw; g < J.total_chunks; g += nw) {
        const RansJob& jb = J.job[find_job(J, g)];
        const uint32_t c = g - jb.first_chunk;
        const uint64_t cbeg = static_cast<uint64_t>(c) * jb.S;
        const uint64_t cend = min(cbeg + jb.S, jb.count);
        const uint32_t steps = static_cast<uint32_t>((cend - cbeg + 31) / 32);
        const uint32_t prec = jb.prec;
        const uint32_t M = 1u << prec, L = 4u << prec;
        const uint8_t* in = jb.bytes;
        uint64_t pos = jb.chunk_off[c];
        const uint64_t end = jb.chunk_off[c + 1];
        uint32_t x = jb.states[static_cast<uint64_t>(c) * 32 + lane];
        bool bad = (x < L) || (static_cast<uint64_t>(x) >= (static_cast<uint64_t>(L) << 8));
        if (__any_sync(0xffffffffu, bad)) {
            if (lane == 0) set_error(err, kErrCorrupt);
            continue;
        }
        for (uint32_t t = 0; t < steps; ++t) {
            const uint64_t k = cbeg + static_cast<uint64_t>(t) * 32 + lane;
            const bool act = k < cend;
            uint32_t nb = 0;
            if (act) {
                const uint32_t slot = x & (M - 1);
                const uint32_t s = __ldg(jb.lookup + slot);
                x = __ldg(jb.prob + s) * (x >> prec) + slot - __ldg(jb.cum + s);
                jb.out[k] = s;
                // a valid step leaves x >= 4, so at most 3 bytes are needed; more means
                // a corrupt stream (and a zero state would never terminate)
                uint32_t y = x;
                while (y < L && nb < 4) { y <<= 8; ++nb; }
                if (nb == 4) { bad = true; nb = 0; }
            }
            const uint32_t inc = warp_inclusive_sum(nb);
            const uint32_t total = __shfl_sync(0xffffffffu, inc, 31);
            if (__any_sync(0xffffffffu, bad) || pos + total > end) { bad = true; break; }
            const uint64_t base = pos + (inc - nb);
            for (uint32_t j = 0; j < nb; ++j) x = (x << 8) | in[base + j];
            pos += total;
        }
        bad = bad || (x != L) || (pos != end);
        if (__any_sync(0xffffffffu, bad) && lane == 0) set_error(err, kErrCorrupt);
    }
}

}  // namespace chain
