/* Chain oracle: CPU restatement of the reference CPU Chain integer pipeline.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  The product GPU path never links, loads or
 * calls this file; only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg do.  Parity pinning: tests/test_oracle.py checks every function here against
 * the reference CPU modules compiled from the reference sources (oracle/_ref) and
 * against the committed golden fixtures in tests/golden/.
 *
 * Built with -ffp-contract=off so that no a*b+c is fused behind our back: the only
 * fused multiply-add is the explicit fma() of the reference's reconstruction.
 */
#include "chain_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static int bitlen_u64(uint64_t v) {
    int b = 0;
    while (v) { ++b; v >>= 1; }
    return b;
}

/* cpp/chain/lcps_cpp.cpp:1496-1500 */
static double reconstruct_coordinate(int64_t q, double minimum, double eb) {
    return fma((double)q + 0.5, 2.0 * eb, minimum);
}

/* cpp/chain/lcps_cpp.cpp:1502-1523: |restored - original| <= eb, with the TwoSum
 * remainder deciding the case where the rounded difference equals eb exactly. */
static int within_error_bound(double restored, double original, double eb) {
    if (!isfinite(restored)) return 0;
    const double difference = restored - original;
    const double magnitude = fabs(difference);
    if (magnitude < eb) return 1;
    if (!(magnitude == eb)) return 0;
    const double virtual_original = difference - restored;
    const double remainder = (restored - (difference - virtual_original))
                           + (-original - virtual_original);
    return difference >= 0.0 ? remainder <= 0.0 : remainder >= 0.0;
}

int co_quantize(const double* pts, uint64_t n, uint32_t dims, double eb, int64_t p_eff,
                double* mins, int64_t* bid, int64_t* rel, uint64_t* corr_idx,
                double* corr_val, uint64_t* ncorr, int64_t* max_bid) {
    if (!(eb > 0.0) || !isfinite(2.0 * eb) || p_eff <= 0 || n == 0 || dims == 0)
        return CO_INVALID_ARGUMENT;
    /* lcps_cpp.cpp:2072-2079: per-dimension minimum, std::min semantics (the first
     * of equal values is kept), every coordinate finite. */
    for (uint32_t d = 0; d < dims; ++d) mins[d] = INFINITY;
    for (uint64_t i = 0; i < n; ++i) {
        for (uint32_t d = 0; d < dims; ++d) {
            const double x = pts[i * dims + d];
            if (!isfinite(x)) return CO_NONFINITE_INPUT;
            if (x < mins[d]) mins[d] = x;
        }
    }
    const double denom = 2.0 * eb;
    uint64_t nc = 0;
    int64_t mb = 0;
    for (uint64_t i = 0; i < n; ++i) {
        for (uint32_t d = 0; d < dims; ++d) {
            const double original = pts[i * dims + d];
            const double qv = floor((original - mins[d]) / denom);
            if (!(qv >= 0.0 && qv < 0x1p63)) return CO_QUANT_OVERFLOW;
            const int64_t q = (int64_t)qv;
            const double restored = reconstruct_coordinate(q, mins[d], eb);
            if (!within_error_bound(restored, original, eb)) {
                corr_idx[nc] = i * dims + d;
                corr_val[nc] = original;
                ++nc;
            }
            const int64_t b = q / p_eff;
            bid[(uint64_t)d * n + i] = b;
            if (b > mb) mb = b;
            rel[(uint64_t)d * n + i] = q - b * p_eff;
        }
    }
    *ncorr = nc;
    *max_bid = mb;
    return CO_OK;
}

/* Open-addressing table keyed by a point's block tuple; value = last index seen. */
static uint64_t tuple_hash(const int64_t* bid, uint64_t n, uint32_t dims, uint64_t i) {
    uint64_t h = 0x9E3779B97F4A7C15ull;
    for (uint32_t d = 0; d < dims; ++d) {
        h ^= (uint64_t)bid[(uint64_t)d * n + i];
        h *= 0xBF58476D1CE4E5B9ull;
        h ^= h >> 31;
    }
    return h;
}

static int same_tuple(const int64_t* bid, uint64_t n, uint32_t dims, uint64_t a, uint64_t b) {
    for (uint32_t d = 0; d < dims; ++d)
        if (bid[(uint64_t)d * n + a] != bid[(uint64_t)d * n + b]) return 0;
    return 1;
}

int co_level1(const int64_t* bid, uint64_t n, uint32_t dims, int64_t threshold, int l1,
              int64_t max_bid, int64_t* idrel, int64_t* blocks, uint64_t* nblocks) {
    uint64_t* next = (uint64_t*)malloc(sizeof(uint64_t) * (n ? n : 1));
    if (!next) return CO_NO_MEMORY;
    for (uint64_t i = 0; i < n; ++i) next[i] = n;
    if (l1) {
        /* lcps_cpp.cpp:2116-2138: next[i] = the smallest j > i in the same block. */
        uint64_t cap = 1;
        while (cap < 2 * n) cap <<= 1;
        uint64_t* slot_first = (uint64_t*)malloc(sizeof(uint64_t) * cap);
        uint64_t* slot_last = (uint64_t*)malloc(sizeof(uint64_t) * cap);
        if (!slot_first || !slot_last) {
            free(next); free(slot_first); free(slot_last);
            return CO_NO_MEMORY;
        }
        for (uint64_t s = 0; s < cap; ++s) slot_first[s] = UINT64_MAX;
        for (uint64_t i = 0; i < n; ++i) {
            uint64_t s = tuple_hash(bid, n, dims, i) & (cap - 1);
            for (;;) {
                if (slot_first[s] == UINT64_MAX) {
                    slot_first[s] = i;
                    slot_last[s] = i;
                    break;
                }
                if (same_tuple(bid, n, dims, slot_first[s], i)) {
                    next[slot_last[s]] = i;
                    slot_last[s] = i;
                    break;
                }
                s = (s + 1) & (cap - 1);
            }
        }
        free(slot_first);
        free(slot_last);
    }
    /* lcps_cpp.cpp:2155-2200: chain to the successor when its distance costs fewer
     * bits than the block record, by more than `threshold`. */
    const int64_t max_bid_bits = bitlen_u64((uint64_t)max_bid);
    uint64_t nb = 0;
    for (uint64_t i = 0; i < n; ++i) {
        if (next[i] != n) {
            const uint64_t dist = next[i] - i;
            int64_t mx = bid[i];
            for (uint32_t d = 1; d < dims; ++d)
                if (bid[(uint64_t)d * n + i] > mx) mx = bid[(uint64_t)d * n + i];
            const int local_bits = bitlen_u64((uint64_t)mx);
            const int tag_bits = bitlen_u64((uint64_t)local_bits);
            int64_t a = (int64_t)local_bits * (int64_t)dims + tag_bits;
            int64_t b = (int64_t)dims * max_bid_bits;
            const int smaller = (int)(a < b ? a : b);
            const int dl = bitlen_u64(dist);
            if ((int64_t)(dl + bitlen_u64((uint64_t)dl)) < (int64_t)smaller - threshold) {
                idrel[i] = (int64_t)dist;
                continue;
            }
        }
        idrel[i] = 0;
        for (uint32_t d = 0; d < dims; ++d) blocks[(uint64_t)d * n + nb] = bid[(uint64_t)d * n + i];
        ++nb;
    }
    *nblocks = nb;
    free(next);
    return CO_OK;
}

int co_make_wrap(int64_t min_value, int64_t max_value, co_wrap* w) {
    if (min_value > max_value) return CO_INVALID_ARGUMENT;
    uint64_t difference;
    if (min_value < 0 && max_value >= 0) {
        const uint64_t negative_magnitude = (uint64_t)(-(min_value + 1)) + 1;
        difference = (uint64_t)max_value + negative_magnitude;
    } else {
        difference = (uint64_t)(max_value - min_value);
    }
    if (difference >= (uint64_t)INT64_MAX) return CO_INVALID_ARGUMENT;
    w->min_value = min_value;
    w->max_value = max_value;
    w->max_difference = (int64_t)(difference + 1);
    w->max_correction = w->max_difference / 2;
    w->min_correction = -w->max_correction;
    if ((w->max_difference & 1) == 0) --w->max_correction;
    return CO_OK;
}

/* lcps_cpp.cpp:1255-1262 */
static uint64_t zigzag(int64_t v) {
    if (v >= 0) return (uint64_t)v << 1;
    return ((uint64_t)(-(v + 1)) << 1) | 1u;
}

static uint64_t absdiff(int64_t a, int64_t b) {
    return a >= b ? (uint64_t)(a - b) : (uint64_t)(b - a);
}

int co_level2(const int64_t* blocks, uint64_t nrec, uint64_t stride, uint32_t dims, int l2,
              int64_t* choice2, int64_t* keep, uint64_t* nkeep, int64_t* diff,
              uint64_t* ndiff, uint64_t stride_out, co_wrap* wrap) {
#define REC(d, i) blocks[(uint64_t)(d) * stride + (i)]
    uint64_t nk = 0, nd = 0;
    if (!l2) {
        /* lcps_cpp.cpp:1456-1478 */
        int64_t mn = INT64_MAX, mx = 0;
        for (uint32_t d = 0; d < dims; ++d)
            for (uint64_t i = 0; i < nrec; ++i) {
                if (REC(d, i) < mn) mn = REC(d, i);
                if (REC(d, i) > mx) mx = REC(d, i);
            }
        for (uint64_t i = 0; i < nrec; ++i) {
            choice2[i] = 0;
            for (uint32_t d = 0; d < dims; ++d) keep[(uint64_t)d * stride_out + i] = REC(d, i);
        }
        *nkeep = nrec;
        *ndiff = 0;
        return co_make_wrap(nrec == 0 ? 0 : mn, mx, wrap);
    }
    if (nrec == 0) {
        *nkeep = *ndiff = 0;
        return co_make_wrap(0, 0, wrap);
    }
    /* lcps_cpp.cpp:1348-1370: global extrema and the largest consecutive difference. */
    int64_t mn = INT64_MAX, mx = INT64_MIN;
    uint64_t maxdiff = 0;
    for (uint64_t i = 0; i < nrec; ++i)
        for (uint32_t d = 0; d < dims; ++d) {
            const int64_t v = REC(d, i);
            if (v < 0) return CO_INVALID_ARGUMENT;
            if (v < mn) mn = v;
            if (v > mx) mx = v;
            if (i) {
                const uint64_t a = absdiff(REC(d, i - 1), v);
                if (a > maxdiff) maxdiff = a;
            }
        }
    int st = co_make_wrap(mn, mx, wrap);
    if (st) return st;
    /* lcps_cpp.cpp:1372-1451: per-record keep/difference decision and wrapped symbols. */
    const uint64_t fixed_value_bits = (uint64_t)dims * bitlen_u64((uint64_t)mx);
    const uint64_t fixed_diff_bits = (uint64_t)dims * bitlen_u64(maxdiff);
    for (uint64_t i = 0; i < nrec; ++i) {
        int use_diff = 0;
        if (i) {
            uint64_t mv = 0, md = 0;
            for (uint32_t d = 0; d < dims; ++d) {
                if ((uint64_t)REC(d, i) > mv) mv = (uint64_t)REC(d, i);
                const uint64_t a = absdiff(REC(d, i - 1), REC(d, i));
                if (a > md) md = a;
            }
            const int tvw = bitlen_u64(mv), tdw = bitlen_u64(md);
            const uint64_t tvb = (uint64_t)dims * tvw + bitlen_u64((uint64_t)tvw);
            const uint64_t tdb = (uint64_t)dims * tdw + bitlen_u64((uint64_t)tdw);
            const uint64_t value_bits = tvb < fixed_value_bits ? tvb : fixed_value_bits;
            const uint64_t diff_bits = tdb > fixed_diff_bits ? tdb : fixed_diff_bits;
            use_diff = value_bits >= diff_bits;
        }
        choice2[i] = use_diff;
        if (!use_diff) {
            for (uint32_t d = 0; d < dims; ++d) keep[(uint64_t)d * stride_out + nk] = REC(d, i);
            ++nk;
            continue;
        }
        for (uint32_t d = 0; d < dims; ++d) {
            int64_t pred = REC(d, i - 1);
            if (pred < wrap->min_value) pred = wrap->min_value;
            if (pred > wrap->max_value) pred = wrap->max_value;
            int64_t corr = pred - REC(d, i);
            if (corr < wrap->min_correction) corr += wrap->max_difference;
            else if (corr > wrap->max_correction) corr -= wrap->max_difference;
            diff[(uint64_t)d * stride_out + nd] = (int64_t)zigzag(corr);
        }
        ++nd;
    }
    *nkeep = nk;
    *ndiff = nd;
    return CO_OK;
#undef REC
}

int co_decode_q(uint64_t n, uint32_t dims, int64_t p, int64_t wrap_min, int64_t wrap_max,
                const int64_t* idrel, const int64_t* diff, uint64_t ndiff,
                const int64_t* keep, uint64_t nkeep, const int64_t* choice2,
                uint64_t nchoice, const int64_t* rel, int64_t* q) {
    co_wrap w;
    if (n == 0 || dims == 0 || p <= 0 || wrap_min < 0) return CO_CORRUPT_STREAM;
    if (co_make_wrap(wrap_min, wrap_max, &w)) return CO_CORRUPT_STREAM;
    int64_t* compact = (int64_t*)malloc(sizeof(int64_t) * (nchoice ? nchoice : 1) * dims);
    if (!compact) return CO_NO_MEMORY;
    int st = CO_OK;
    /* lcps_cpp.cpp:1890-1934: level-2 inverse. */
    uint64_t di = 0, ki = 0;
    const uint64_t range = (uint64_t)w.max_difference;
    for (uint64_t i = 0; i < nchoice && st == CO_OK; ++i) {
        const int64_t c = choice2[i];
        if (c != 0 && c != 1) { st = CO_CORRUPT_STREAM; break; }
        if (c == 0) {
            if (ki >= nkeep) { st = CO_CORRUPT_STREAM; break; }
            for (uint32_t d = 0; d < dims; ++d) {
                const int64_t v = keep[(uint64_t)d * nkeep + ki];
                if (v < wrap_min || v > wrap_max) { st = CO_CORRUPT_STREAM; break; }
                compact[(uint64_t)d * nchoice + i] = v;
            }
            ++ki;
            continue;
        }
        if (i == 0 || di >= ndiff) { st = CO_CORRUPT_STREAM; break; }
        for (uint32_t d = 0; d < dims; ++d) {
            const int64_t s = diff[(uint64_t)d * ndiff + di];
            if (s < 0) { st = CO_CORRUPT_STREAM; break; }
            const uint64_t sym = (uint64_t)s;
            const int64_t corr = (sym & 1u) ? -(int64_t)(sym >> 1) - 1 : (int64_t)(sym >> 1);
            if (corr < w.min_correction || corr > w.max_correction) { st = CO_CORRUPT_STREAM; break; }
            const uint64_t prev = (uint64_t)(compact[(uint64_t)d * nchoice + i - 1] - wrap_min);
            uint64_t off;
            if (corr >= 0) {
                const uint64_t a = (uint64_t)corr;
                off = prev >= a ? prev - a : range - (a - prev);
            } else {
                const uint64_t a = (uint64_t)(-(corr + 1)) + 1;
                off = prev >= range - a ? prev - (range - a) : prev + a;
            }
            compact[(uint64_t)d * nchoice + i] = wrap_min + (int64_t)off;
        }
        ++di;
    }
    if (st == CO_OK && (di != ndiff || ki != nkeep)) st = CO_CORRUPT_STREAM;
    /* lcps_cpp.cpp:1936-1961: backward level-1 pass; q = block * p + offset. */
    if (st == CO_OK) {
        memcpy(q, rel, sizeof(int64_t) * n * dims);
        uint64_t ci = nchoice;
        for (uint64_t i = n; i-- > 0 && st == CO_OK;) {
            const int64_t jump = idrel[i];
            uint64_t succ = i;
            if (jump < 0) { st = CO_CORRUPT_STREAM; break; }
            if (jump == 0) {
                if (ci == 0) { st = CO_CORRUPT_STREAM; break; }
                --ci;
            } else {
                if ((uint64_t)jump >= n - i) { st = CO_CORRUPT_STREAM; break; }
                succ += (uint64_t)jump;
            }
            for (uint32_t d = 0; d < dims; ++d) {
                const int64_t off = q[(uint64_t)d * n + i];
                if (off < 0 || off >= p) { st = CO_CORRUPT_STREAM; break; }
                const int64_t blk = jump == 0 ? compact[(uint64_t)d * nchoice + ci]
                                              : q[(uint64_t)d * n + succ] / p;
                if (blk > (INT64_MAX - off) / p) { st = CO_CORRUPT_STREAM; break; }
                q[(uint64_t)d * n + i] = blk * p + off;
            }
        }
        if (st == CO_OK && ci != 0) st = CO_CORRUPT_STREAM;
    }
    free(compact);
    return st;
}

int co_reconstruct(uint64_t n, uint32_t dims, const int64_t* q, const double* mins, double eb,
                   const uint64_t* corr_idx, const double* corr_val, uint64_t ncorr,
                   double* out) {
    for (uint64_t i = 0; i < n; ++i)
        for (uint32_t d = 0; d < dims; ++d)
            out[i * dims + d] = reconstruct_coordinate(q[(uint64_t)d * n + i], mins[d], eb);
    uint64_t prev = 0;
    for (uint64_t k = 0; k < ncorr; ++k) {
        if (corr_idx[k] >= n * dims || (k && corr_idx[k] <= prev) || !isfinite(corr_val[k]))
            return CO_CORRUPT_STREAM;
        out[corr_idx[k]] = corr_val[k];
        prev = corr_idx[k];
    }
    return CO_OK;
}
