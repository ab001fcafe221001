// LCG2 version 2 container: the byte layout this GPU path writes and reads.
//
// It keeps the framing of the reference GPU format, LCG2 version 1
// (cu/chain/lcps_gpu_cpp.cu:1-35): magic "LCG2", a version word, D, N, the block size,
// error bound, wrap range and per-axis minima, then five named components
// IDR0/DIF0/KEP0/CH20/REL0 in that order, each with an encoding byte
// (0 empty, 1 tagged, 2 fixed, 3 raw), its dimension count and record count.
// Version 2 changes what version 1 could not carry bit-exactly or without nvCOMP:
//   * p, wrap_min, wrap_max are int64 and eb, minima are float64 (FP64 semantics of
//     the reference CPU encoder, lcps_cpp.cpp:2306-2329);
//   * one input-dtype byte (4 = float32 input, 8 = float64 input);
//   * entropy sections use codec "interleaved value rANS" (rans.cuh) in place of
//     nvCOMP ANS/Zstd chunks;
//   * an exact-corrections section "EXC0" follows the components (LCP2 stores the
//     same records, lcps_cpp.cpp:2097-2103, 2329).
//
// All integers little-endian, no padding:
//   "LCG2" u32 version=2, u32 D, u64 N, i64 p, f64 eb, i64 wrap_min, i64 wrap_max,
//   f64 minima[D], u8 input_dtype, u32 stream_count=5,
//   5 x { char name[4], u64 body_len, body },
//   "EXC0", u64 body_len, { u64 count; when count > 0: u64 ndistinct,
//                           ndistinct x f64 distinct corrected values (ascending bits),
//                           u64 len, component body of the index gaps,
//                           u64 len, component body of the value ids }.
// Exact corrections (lcps_cpp.cpp:2097-2103) are the points whose FP64 reconstruction
// would miss eb; they are listed by flat index i*D+d in increasing order.  Gap k is
// index_k - index_{k-1} - 1 (index_0 itself for k = 0); id k selects the value.
// Component body:
//   u8 encoding, u32 dims, u64 records, then
//   empty (0):  nothing (records == 0)
//   fixed (2):  dims x { u64 minimum, u8 width }, then per dimension the MSB-first
//               packed offsets v - minimum, each dimension padded to a byte
//               (lcps_cpp.cpp:161-222 bit order)
//   tagged(1):  u8 max_width, rANS section of the per-record widths
//               (max(1, max_d bitlen v)), u64 packed_bits, then the record-major
//               values packed MSB-first at their record's width (lcps_cpp.cpp:1005-1058)
//   raw (3):    rANS section over the record-major values
// rANS section:
//   u8 prec, u32 alphabet, u32 table_bytes, table tokens (rans.cuh), u64 symbols per
//   chunk S, u8 lanes W (1..32, S a multiple of W), u32 chunks, u64 payload bytes (the
//   sum of the chunk bytes), chunks x u32 chunk bytes, the chunks x W final lane states
//   (chunk-major) packed MSB-first at prec + 10 bits each (a final state lies in
//   [4 * 2^prec, 1024 * 2^prec)) and padded to a byte, then the chunk byte streams back
//   to back.
//   Fixed width 0 means a constant component (every value equals its minimum).
#pragma once

#include <stdint.h>
#include <string.h>

#include "chain_common.cuh"

namespace chain {

constexpr uint32_t kFormatVersion = 2;
// Coded streams: the five components, then the two exact-correction streams.
constexpr int kCodeStreams = kStreams + 2;
constexpr int kCorrGaps = kStreams;      // index gaps
constexpr int kCorrIds = kStreams + 1;   // value ids
// Component names, in container order (cu/chain/lcps_gpu_cpp.cu:88).
__host__ __device__ inline void stream_name(int s, char out[4]) {
    const char names[kStreams][4] = {{'I', 'D', 'R', '0'}, {'D', 'I', 'F', '0'}, {'K', 'E', 'P', '0'},
                                     {'C', 'H', '2', '0'}, {'R', 'E', 'L', '0'}};
    for (int i = 0; i < 4; ++i) out[i] = names[s][i];
}

// Bits of one packed final lane state, and the bytes of a section's packed states.
__host__ __device__ inline uint32_t state_bits(uint32_t prec) { return prec + 10; }
__host__ __device__ inline uint64_t state_bytes(uint32_t lanes, uint32_t chunks, uint32_t prec) {
    return (static_cast<uint64_t>(lanes) * chunks * state_bits(prec) + 7) / 8;
}

struct SectionPlan {
    uint32_t prec;
    uint32_t alphabet;
    uint64_t table_off;    // absolute offsets into the container
    uint32_t table_len;
    uint32_t chunks;
    uint32_t lanes;
    uint32_t pad;
    uint64_t S;
    uint64_t count;        // symbols
    uint64_t chunk_tab_off;
    uint64_t states_off;
    uint64_t payload_off;
    uint64_t payload_len;
};

struct CompPlan {
    uint8_t enc;
    uint8_t max_width;
    uint8_t width[kMaxDims];
    uint32_t dims;
    uint64_t records;
    uint64_t minv[kMaxDims];
    uint64_t packed_off[kMaxDims];  // fixed: per-dimension payload offsets
    uint64_t packed_bits;           // tagged
    uint64_t tagged_off;            // tagged payload offset
    SectionPlan sec;
};

struct DecodePlan {
    uint32_t D;
    uint8_t input_dtype;
    uint8_t pad[3];
    uint64_t N;
    int64_t p;
    double eb;
    int64_t wrap_min, wrap_max;
    double minima[kMaxDims];
    CompPlan comp[kCodeStreams];
    uint64_t exc_count;
    uint64_t exc_ndistinct;
    uint64_t exc_dict_off;
    uint32_t ok;      // 1 = parsed and structurally valid
    uint32_t why;     // failure code (line of the failed check) when ok == 0
};

struct ByteReader {
    const uint8_t* p;
    uint64_t len;
    uint64_t pos;
    bool ok;
    __host__ __device__ bool need(uint64_t n) {
        if (!ok || n > len - pos) { ok = false; return false; }
        return true;
    }
    __host__ __device__ uint64_t uint(int bytes) {
        if (!need(bytes)) return 0;
        uint64_t v = 0;
        for (int i = 0; i < bytes; ++i) v |= static_cast<uint64_t>(p[pos + i]) << (8 * i);
        pos += bytes;
        return v;
    }
    __host__ __device__ uint8_t u8() { return static_cast<uint8_t>(uint(1)); }
    __host__ __device__ uint32_t u32() { return static_cast<uint32_t>(uint(4)); }
    __host__ __device__ uint64_t u64() { return uint(8); }
    __host__ __device__ int64_t i64() { return static_cast<int64_t>(uint(8)); }
    __host__ __device__ double f64() {
        uint64_t u = uint(8);
        double d;
        memcpy(&d, &u, 8);
        return d;
    }
    __host__ __device__ bool skip(uint64_t n) {
        if (!need(n)) return false;
        pos += n;
        return true;
    }
    __host__ __device__ bool magic(const char* m) {
        if (!need(4)) return false;
        for (int i = 0; i < 4; ++i)
            if (p[pos + i] != static_cast<uint8_t>(m[i])) { ok = false; return false; }
        pos += 4;
        return true;
    }
};

__host__ __device__ inline bool chain_isfinite(double x) { return x == x && x - x == 0.0; }

#define CHAIN_PARSE_REQUIRE(cond)        \
    do {                                 \
        if (!(cond)) {                   \
            plan->ok = 0;                \
            plan->why = __LINE__;        \
            return false;                \
        }                                \
    } while (0)

__host__ __device__ inline bool parse_section(ByteReader& r, SectionPlan* s, uint64_t count,
                                              DecodePlan* plan) {
    s->count = count;
    s->prec = r.u8();
    s->alphabet = r.u32();
    s->table_len = r.u32();
    CHAIN_PARSE_REQUIRE(r.ok && s->prec >= kRansMinPrec && s->prec <= kRansMaxPrec);
    CHAIN_PARSE_REQUIRE(s->alphabet >= 1 && s->alphabet <= kRansMaxAlphabet);
    s->table_off = r.pos;
    CHAIN_PARSE_REQUIRE(r.skip(s->table_len));
    s->S = r.u64();
    s->lanes = r.u8();
    s->chunks = r.u32();
    CHAIN_PARSE_REQUIRE(r.ok && s->lanes >= 1 && s->lanes <= 32 && s->S >= s->lanes && s->S % s->lanes == 0);
    const uint64_t want = (count + s->S - 1) / s->S;
    CHAIN_PARSE_REQUIRE(want == s->chunks && s->chunks >= 1);
    s->payload_len = r.u64();
    s->chunk_tab_off = r.pos;
    // the chunk lengths must add up to payload_len; the decoder checks that in parallel
    CHAIN_PARSE_REQUIRE(r.skip(4ull * s->chunks));
    s->states_off = r.pos;
    CHAIN_PARSE_REQUIRE(r.skip(state_bytes(s->lanes, s->chunks, s->prec)));
    s->payload_off = r.pos;
    CHAIN_PARSE_REQUIRE(r.skip(s->payload_len));
    return true;
}

// One component body of body_len bytes (the reader sits at its first byte).
__host__ __device__ inline bool parse_component(ByteReader& r, uint64_t body_len, CompPlan* c, uint32_t want_dims,
                                                uint64_t max_records, DecodePlan* plan) {
    CHAIN_PARSE_REQUIRE(r.need(body_len));
    const uint64_t body_end = r.pos + body_len;
    c->enc = r.u8();
    c->dims = r.u32();
    c->records = r.u64();
    CHAIN_PARSE_REQUIRE(r.ok && c->dims == want_dims && c->records <= max_records);
    CHAIN_PARSE_REQUIRE(c->enc <= kEncRaw);
    if (c->enc == kEncEmpty) {
        CHAIN_PARSE_REQUIRE(c->records == 0);
    } else if (c->enc == kEncFixed) {
        CHAIN_PARSE_REQUIRE(c->records > 0);
        for (uint32_t d = 0; d < c->dims; ++d) {
            c->minv[d] = r.u64();
            c->width[d] = r.u8();
            CHAIN_PARSE_REQUIRE(r.ok && c->width[d] <= 32);
        }
        for (uint32_t d = 0; d < c->dims; ++d) {
            c->packed_off[d] = r.pos;
            CHAIN_PARSE_REQUIRE(r.skip((c->records * c->width[d] + 7) / 8));
        }
    } else if (c->enc == kEncTagged) {
        CHAIN_PARSE_REQUIRE(c->records > 0);
        c->max_width = r.u8();
        CHAIN_PARSE_REQUIRE(r.ok && c->max_width >= 1 && c->max_width <= 32);
        if (!parse_section(r, &c->sec, c->records, plan)) return false;
        CHAIN_PARSE_REQUIRE(c->sec.alphabet <= 33u);
        c->packed_bits = r.u64();
        CHAIN_PARSE_REQUIRE(r.ok && c->packed_bits >= c->records * c->dims &&
                            c->packed_bits <= c->records * c->dims * 32ull);
        c->tagged_off = r.pos;
        CHAIN_PARSE_REQUIRE(r.skip((c->packed_bits + 7) / 8));
    } else {
        CHAIN_PARSE_REQUIRE(c->records > 0);
        if (!parse_section(r, &c->sec, c->records * c->dims, plan)) return false;
    }
    CHAIN_PARSE_REQUIRE(r.ok && r.pos == body_end);
    return true;
}

// Parses and structurally validates a container.  Semantic validation of the coded
// integers (ranges, counts, references) happens in the decode kernels.
__host__ __device__ inline bool parse_container(const uint8_t* data, uint64_t len, DecodePlan* plan) {
    ByteReader r{data, len, 0, true};
    plan->ok = 0;
    plan->why = 0;
    CHAIN_PARSE_REQUIRE(r.magic("LCG2"));
    CHAIN_PARSE_REQUIRE(r.u32() == kFormatVersion);
    plan->D = r.u32();
    plan->N = r.u64();
    plan->p = r.i64();
    plan->eb = r.f64();
    plan->wrap_min = r.i64();
    plan->wrap_max = r.i64();
    CHAIN_PARSE_REQUIRE(r.ok && plan->D >= 1 && plan->D <= static_cast<uint32_t>(kMaxDims));
    CHAIN_PARSE_REQUIRE(plan->N >= 1 && plan->N < (1ull << 31) && plan->p > 0);
    CHAIN_PARSE_REQUIRE(plan->eb > 0.0 && chain_isfinite(2.0 * plan->eb));
    CHAIN_PARSE_REQUIRE(plan->wrap_min >= 0 && plan->wrap_max >= plan->wrap_min &&
                        plan->wrap_max <= 0xFFFFFFFFll);
    for (uint32_t d = 0; d < plan->D; ++d) {
        plan->minima[d] = r.f64();
        CHAIN_PARSE_REQUIRE(r.ok && chain_isfinite(plan->minima[d]));
    }
    plan->input_dtype = r.u8();
    CHAIN_PARSE_REQUIRE(r.ok && (plan->input_dtype == 4 || plan->input_dtype == 8));
    CHAIN_PARSE_REQUIRE(r.u32() == kStreams);
    for (int s = 0; s < kStreams; ++s) {
        char name[5] = {0, 0, 0, 0, 0};
        stream_name(s, name);
        CHAIN_PARSE_REQUIRE(r.magic(name));
        const uint64_t body_len = r.u64();
        if (!parse_component(r, body_len, &plan->comp[s], (s == 0 || s == 3) ? 1u : plan->D, plan->N, plan))
            return false;
    }
    CHAIN_PARSE_REQUIRE(plan->comp[0].records == plan->N && plan->comp[4].records == plan->N);
    CHAIN_PARSE_REQUIRE(plan->comp[3].records >= 1 && plan->comp[2].records >= 1);
    CHAIN_PARSE_REQUIRE(plan->comp[1].records + plan->comp[2].records == plan->comp[3].records);
    CHAIN_PARSE_REQUIRE(r.magic("EXC0"));
    const uint64_t exc_len = r.u64();
    CHAIN_PARSE_REQUIRE(r.need(exc_len));
    const uint64_t exc_end = r.pos + exc_len;
    plan->exc_count = r.u64();
    plan->exc_ndistinct = 0;
    plan->comp[kCorrGaps].enc = plan->comp[kCorrIds].enc = kEncEmpty;
    plan->comp[kCorrGaps].records = plan->comp[kCorrIds].records = 0;
    CHAIN_PARSE_REQUIRE(r.ok && plan->exc_count <= plan->N * plan->D);
    if (plan->exc_count) {
        plan->exc_ndistinct = r.u64();
        CHAIN_PARSE_REQUIRE(r.ok && plan->exc_ndistinct >= 1 && plan->exc_ndistinct <= plan->exc_count);
        plan->exc_dict_off = r.pos;
        CHAIN_PARSE_REQUIRE(r.skip(8 * plan->exc_ndistinct));
        for (int s = kCorrGaps; s <= kCorrIds; ++s) {
            const uint64_t body_len = r.u64();
            if (!parse_component(r, body_len, &plan->comp[s], 1u, plan->exc_count, plan)) return false;
            CHAIN_PARSE_REQUIRE(plan->comp[s].records == plan->exc_count);
        }
    }
    CHAIN_PARSE_REQUIRE(r.ok && r.pos == exc_end && r.pos == len);
    plan->ok = 1;
    return true;
}

#undef CHAIN_PARSE_REQUIRE

// Fixed header bytes before the first component.
inline uint64_t header_bytes(uint32_t D) { return 57ull + 8ull * D; }

}  // namespace chain
