// LCG2 version 2 -> the reference CPU Chain's LCP2 container (chain_transcode_lcp2).
//
// Host code only.  The container's integer streams are decoded on the CPU (the same
// sections the GPU decoder reads) and written again as an LCP2 bitstream that the
// reference decoder (cpp/decompress/lcps_cpu_decompress_serial.cpp:1183-1330, and
// lcps_cpp.cpp:1833-1995) reads directly:
//   "LCP2", u32 D, u64 N, i64 p, f64 eb, i64 wrap_min, i64 wrap_max, f64 mins[D],
//   five (u64 length, component) pairs idrel, diff, keep, choice2, rel,
//   u64 correction count, u64 length, Zstd frame of (u64 index, f64 value) records
//   (lcps_cpp.cpp:2306-2329).
// Components are written as
//   RVMX (values below 2^18: value rANS over the point-major values), else
//   RTG4 (per-record widths max(1, max_d bitlen v) by value rANS, then the values packed
//         MSB-first at their record's width, stored without Zstd),
// the two encodings of the reference decoder that need no Zstd compressor
// (decode_component_matrix_cpp, lcps_cpu_decompress_serial.cpp:1076-1178).  Value rANS
// is the RVN1 layout of lcps_cpp.cpp:739-821: u8 precision, u64 count, u32 final state,
// table tokens (VarUint alphabet, then the token scheme of lcps_cpp.cpp:686-729), and the
// renormalisation bytes in decode order; the state lives in [4*2^prec, 1024*2^prec) and
// the decoder ends at 4*2^prec.  The correction records go into a Zstd frame made of raw
// (stored) blocks, a form every Zstd decoder accepts (RFC 8878, sections 3.1.1-3.1.1.2).
// The transcoded container decodes to the same points; it is larger than the
// reference's own output, which Zstd-compresses its packed candidates.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "chain_format.h"
#include "ctx.h"

namespace chain {
namespace {

// ----------------------------------------------------------------- LCG2 reading
struct Fail {
    std::string what;
};

uint32_t le32(const uint8_t* p) { return p[0] | (p[1] << 8) | (p[2] << 16) | (static_cast<uint32_t>(p[3]) << 24); }

uint64_t read_msb(const uint8_t* p, uint64_t bit, uint32_t width) {
    uint64_t v = 0;
    for (uint32_t k = 0; k < width; ++k, ++bit) v = (v << 1) | ((p[bit >> 3] >> (7 - (bit & 7))) & 1u);
    return v;
}

// Probability table of an LCG2 rANS section (token scheme shared with LCP2).
std::vector<uint32_t> section_table(const uint8_t* data, const SectionPlan& s) {
    std::vector<uint32_t> prob(s.alphabet, 0);
    const uint8_t* in = data + s.table_off;
    uint64_t pos = 0, sym = 0, sum = 0;
    while (pos < s.table_len) {
        const uint8_t first = in[pos];
        if ((first & 3u) == 3u) {
            sym += (first >> 2) + 1;
            ++pos;
            continue;
        }
        const uint32_t extra = first & 3u;
        if (pos + 1 + extra > s.table_len || sym >= s.alphabet) throw Fail{"rANS table token outside the table"};
        uint32_t p = first >> 2;
        for (uint32_t j = 0; j < extra; ++j) p |= static_cast<uint32_t>(in[pos + 1 + j]) << (6 + 8 * j);
        prob[sym++] = p;
        sum += p;
        pos += 1 + extra;
    }
    if (sym != s.alphabet || sum != (1ull << s.prec)) throw Fail{"rANS table does not describe the alphabet"};
    return prob;
}

// Decodes an interleaved rANS section: chunk c holds symbols [c*S, min(c*S+S, count));
// symbol k of a chunk belongs to lane k % W at step k / W; per step the lanes decode in
// lane order and take their renormalisation bytes in that order.
std::vector<uint32_t> decode_section(const uint8_t* data, const SectionPlan& s) {
    const std::vector<uint32_t> prob = section_table(data, s);
    const uint32_t M = 1u << s.prec, L = 4u << s.prec;
    std::vector<uint32_t> cum(s.alphabet, 0), lookup(M);
    for (uint32_t a = 0, c = 0; a < s.alphabet; ++a) {
        cum[a] = c;
        for (uint32_t j = 0; j < prob[a]; ++j) lookup[c + j] = a;
        c += prob[a];
    }
    std::vector<uint32_t> out(s.count);
    uint64_t off = s.payload_off;
    const uint64_t payload_end = s.payload_off + s.payload_len;
    for (uint32_t c = 0; c < s.chunks; ++c) {
        const uint64_t beg = static_cast<uint64_t>(c) * s.S, end = std::min(beg + s.S, s.count);
        const uint32_t len = le32(data + s.chunk_tab_off + 4ull * c);
        if (off + len > payload_end) throw Fail{"rANS chunk outside the payload"};
        const uint8_t* bytes = data + off;
        uint64_t pos = 0;
        uint32_t x[32];
        for (uint32_t l = 0; l < s.lanes; ++l) {
            const uint32_t B = state_bits(s.prec);
            x[l] = static_cast<uint32_t>(read_msb(data + s.states_off, (static_cast<uint64_t>(c) * s.lanes + l) * B, B));
            if (x[l] < L || static_cast<uint64_t>(x[l]) >= (static_cast<uint64_t>(L) << 8))
                throw Fail{"rANS lane state out of range"};
        }
        for (uint64_t k = 0; beg + k < end; ++k) {
            uint32_t& v = x[k % s.lanes];
            const uint32_t slot = v & (M - 1), sym = lookup[slot];
            out[beg + k] = sym;
            v = prob[sym] * (v >> s.prec) + slot - cum[sym];
            while (v < L) {
                if (pos >= len) throw Fail{"rANS chunk bytes exhausted"};
                v = (v << 8) | bytes[pos++];
            }
        }
        for (uint32_t l = 0; l < s.lanes; ++l)
            if (x[l] != L) throw Fail{"rANS lane does not end at its initial state"};
        if (pos != len) throw Fail{"rANS chunk has unread bytes"};
        off += len;
    }
    if (off != payload_end) throw Fail{"rANS payload length mismatch"};
    return out;
}


// Record-major values of one component.
std::vector<uint64_t> decode_component(const uint8_t* data, const CompPlan& c) {
    const uint64_t n = c.records, D = c.dims;
    std::vector<uint64_t> v(n * D);
    if (c.enc == kEncEmpty) return v;
    if (c.enc == kEncFixed) {
        for (uint64_t d = 0; d < D; ++d)
            for (uint64_t i = 0; i < n; ++i)
                v[i * D + d] = c.minv[d] + (c.width[d] ? read_msb(data + c.packed_off[d], i * c.width[d], c.width[d]) : 0);
        return v;
    }
    if (c.enc == kEncRaw) {
        const std::vector<uint32_t> s = decode_section(data, c.sec);
        for (uint64_t k = 0; k < n * D; ++k) v[k] = s[k];
        return v;
    }
    const std::vector<uint32_t> tags = decode_section(data, c.sec);
    uint64_t bit = 0;
    for (uint64_t i = 0; i < n; ++i) {
        if (tags[i] < 1 || tags[i] > 32) throw Fail{"invalid tagged width"};
        if (bit + D * tags[i] > c.packed_bits) throw Fail{"tagged values outside their payload"};
        for (uint64_t d = 0; d < D; ++d, bit += tags[i]) v[i * D + d] = read_msb(data + c.tagged_off, bit, tags[i]);
    }
    if (bit != c.packed_bits) throw Fail{"tagged payload length mismatch"};
    return v;
}

// ----------------------------------------------------------------- LCP2 writing
void put_le(std::string& o, uint64_t v, int bytes) {
    for (int i = 0; i < bytes; ++i) o.push_back(static_cast<char>((v >> (8 * i)) & 0xffu));
}
void put_f64(std::string& o, double x) {
    uint64_t u;
    memcpy(&u, &x, 8);
    put_le(o, u, 8);
}
void put_blob(std::string& o, const std::string& b) {
    put_le(o, b.size(), 8);
    o += b;
}
void put_varuint(std::string& o, uint64_t v) {
    do {
        uint8_t b = v & 0x7fu;
        v >>= 7;
        if (v) b |= 0x80u;
        o.push_back(static_cast<char>(b));
    } while (v);
}

int bitlen(uint64_t v) {
    int b = 0;
    while (v) { ++b; v >>= 1; }
    return b;
}

// RVN1 value rANS of `sym` (alphabet max+1 <= 2^18).  The precision follows the
// reference rule (lcps_cpp.cpp:541-552); the table is this file's own normalisation:
// every present symbol gets max(1, round(count * 2^prec / n)), and the total is then
// brought to 2^prec by moving the excess or shortfall across the symbols with the
// largest shares (largest first), never below 1.
std::string rvn1(const std::vector<uint64_t>& sym) {
    std::string o("RVN1", 4);
    const uint64_t n = sym.size();
    if (n == 0) {
        o.push_back(0);
        put_le(o, 0, 8);
        put_le(o, 1, 4);
        put_blob(o, std::string());
        put_blob(o, std::string());
        return o;
    }
    uint64_t mx = 0;
    for (uint64_t s : sym) mx = std::max(mx, s);
    const uint32_t A = static_cast<uint32_t>(mx + 1);
    std::vector<uint64_t> cnt(A, 0);
    for (uint64_t s : sym) ++cnt[s];
    uint64_t unique = 0;
    for (uint64_t c : cnt) unique += c != 0;
    const int ubits = std::min(18, bitlen(unique) + 2);
    const int prec = std::min(20, std::max(12, (3 * ubits) / 2));
    const uint64_t M = 1ull << prec;
    std::vector<uint32_t> prob(A, 0);
    int64_t total = 0;
    for (uint32_t a = 0; a < A; ++a) {
        if (!cnt[a]) continue;
        const uint64_t p = (cnt[a] * M * 2 + n) / (2 * n);
        prob[a] = static_cast<uint32_t>(std::max<uint64_t>(1, p));
        total += prob[a];
    }
    std::vector<uint32_t> order;
    for (uint32_t a = 0; a < A; ++a)
        if (cnt[a]) order.push_back(a);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cnt[a] > cnt[b]; });
    int64_t diff = static_cast<int64_t>(M) - total;
    while (diff != 0) {
        bool moved = false;
        for (uint32_t a : order) {
            if (diff == 0) break;
            if (diff > 0) { ++prob[a]; --diff; moved = true; }
            else if (prob[a] > 1) { --prob[a]; ++diff; moved = true; }
        }
        if (!moved) throw Fail{"rANS table cannot be normalised"};
    }
    std::vector<uint32_t> cum(A, 0);
    for (uint32_t a = 0, c = 0; a < A; ++a) { cum[a] = c; c += prob[a]; }
    // table tokens: runs of up to 64 zeros, else the probability in 1..3 bytes
    std::string table;
    put_varuint(table, A);
    for (uint32_t a = 0; a < A;) {
        if (!prob[a]) {
            uint32_t run = 0;
            while (a + run < A && !prob[a + run] && run < 64) ++run;
            table.push_back(static_cast<char>(((run - 1) << 2) | 3u));
            a += run;
            continue;
        }
        const uint32_t p = prob[a++];
        const uint32_t extra = p < (1u << 6) ? 0 : (p < (1u << 14) ? 1 : 2);
        table.push_back(static_cast<char>(((p & 0x3fu) << 2) | extra));
        for (uint32_t j = 0; j < extra; ++j) table.push_back(static_cast<char>((p >> (6 + 8 * j)) & 0xffu));
    }
    // encode in reverse; the bytes come out in reverse decode order
    const uint64_t L = 4 * M;
    uint64_t x = L;
    std::string rev;
    for (uint64_t k = n; k-- > 0;) {
        const uint32_t f = prob[sym[k]];
        const uint64_t xmax = 1024ull * f;
        while (x >= xmax) {
            rev.push_back(static_cast<char>(x & 0xffu));
            x >>= 8;
        }
        x = (x / f) * M + (x % f) + cum[sym[k]];
    }
    std::string renorm(rev.rbegin(), rev.rend());
    o.push_back(static_cast<char>(prec));
    put_le(o, n, 8);
    put_le(o, x, 4);
    put_blob(o, table);
    put_blob(o, renorm);
    return o;
}

// One component: values record-major (n records x D).
std::string component(const std::vector<uint64_t>& v, uint32_t D, uint64_t n) {
    uint64_t mx = 0;
    for (uint64_t x : v) mx = std::max(mx, x);
    std::string o;
    if (mx < (1ull << 18)) {
        o.assign("RVMX", 4);
        put_le(o, D, 4);
        put_le(o, n, 8);
        put_blob(o, rvn1(v));
        return o;
    }
    o.assign("RTG4", 4);
    put_le(o, D, 4);
    put_le(o, n, 8);
    std::vector<uint64_t> tags(n);
    uint64_t maxw = 0, bits = 0;
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t m = 0;
        for (uint32_t d = 0; d < D; ++d) m = std::max(m, v[i * D + d]);
        tags[i] = std::max(1, bitlen(m));
        maxw = std::max(maxw, tags[i]);
        bits += D * tags[i];
    }
    std::string packed((bits + 7) / 8, '\0');
    uint64_t bit = 0;
    for (uint64_t i = 0; i < n; ++i)
        for (uint32_t d = 0; d < D; ++d)
            for (uint64_t k = tags[i]; k-- > 0; ++bit)
                if ((v[i * D + d] >> k) & 1u) packed[bit >> 3] |= static_cast<char>(0x80u >> (bit & 7));
    o.push_back(static_cast<char>(maxw));
    put_blob(o, rvn1(tags));
    put_blob(o, packed);
    return o;
}

// Zstd frame of stored blocks (RFC 8878 3.1.1): magic, a single-segment frame header
// with an 8-byte content size, then raw blocks of at most 128 KiB.
std::string zstd_stored(const std::string& content) {
    std::string o;
    put_le(o, 0xFD2FB528u, 4);
    o.push_back(static_cast<char>(0xE0));   // content-size field 8 bytes, single segment
    put_le(o, content.size(), 8);
    const uint64_t kBlock = 128 * 1024;
    uint64_t pos = 0;
    do {
        const uint64_t len = std::min<uint64_t>(kBlock, content.size() - pos);
        const bool last = pos + len == content.size();
        put_le(o, (len << 3) | (0u << 1) | (last ? 1u : 0u), 3);
        o.append(content, pos, len);
        pos += len;
    } while (pos < content.size());
    return o;
}

std::string transcode(const uint8_t* data, uint64_t len) {
    DecodePlan plan;
    if (!parse_container(data, len, &plan))
        throw Fail{"LCG2: container failed validation (check at chain_format.h:" + std::to_string(plan.why) + ")"};
    const uint32_t D = plan.D;
    const uint64_t N = plan.N;
    std::string o("LCP2", 4);
    put_le(o, D, 4);
    put_le(o, N, 8);
    put_le(o, static_cast<uint64_t>(plan.p), 8);
    put_f64(o, plan.eb);
    put_le(o, static_cast<uint64_t>(plan.wrap_min), 8);
    put_le(o, static_cast<uint64_t>(plan.wrap_max), 8);
    for (uint32_t d = 0; d < D; ++d) put_f64(o, plan.minima[d]);
    for (int s = 0; s < kStreams; ++s) {
        const CompPlan& c = plan.comp[s];
        put_blob(o, component(decode_component(data, c), c.dims, c.records));
    }
    put_le(o, plan.exc_count, 8);
    if (plan.exc_count == 0) {
        put_blob(o, std::string());
        return o;
    }
    const std::vector<uint64_t> gaps = decode_component(data, plan.comp[kCorrGaps]);
    const std::vector<uint64_t> ids = decode_component(data, plan.comp[kCorrIds]);
    std::string recs;
    uint64_t index = 0;
    for (uint64_t k = 0; k < plan.exc_count; ++k) {
        index = k == 0 ? gaps[0] : index + gaps[k] + 1;
        if (index >= N * D || ids[k] >= plan.exc_ndistinct) throw Fail{"invalid exact correction record"};
        put_le(recs, index, 8);
        recs.append(reinterpret_cast<const char*>(data + plan.exc_dict_off + 8 * ids[k]), 8);
    }
    put_blob(o, zstd_stored(recs));
    return o;
}

}  // namespace
}  // namespace chain

using namespace chain;

extern "C" chain_status chain_transcode_lcp2(const void* container, size_t len, void* out, size_t capacity,
                                             size_t* out_len) {
    if (!container || !out_len) return set_err(CHAIN_ERR_INVALID_ARGUMENT, "null argument");
    if (is_device_ptr(container) || (out && is_device_ptr(out)))
        return set_err(CHAIN_ERR_INVALID_ARGUMENT, "chain_transcode_lcp2 takes host buffers");
    std::string lcp2;
    try {
        lcp2 = transcode(static_cast<const uint8_t*>(container), len);
    } catch (const Fail& f) {
        return set_err(CHAIN_ERR_CORRUPT_STREAM, f.what);
    } catch (const std::bad_alloc&) {
        return set_err(CHAIN_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    *out_len = lcp2.size();
    if (!out || capacity < lcp2.size())
        return set_err(CHAIN_ERR_BUFFER_TOO_SMALL, "LCP2 output needs " + std::to_string(lcp2.size()) + " bytes");
    memcpy(out, lcp2.data(), lcp2.size());
    return set_err(CHAIN_OK, std::string());
}
