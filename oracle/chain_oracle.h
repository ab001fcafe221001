/* Chain oracle: CPU restatement of the reference CPU Chain integer pipeline.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product path links, loads or calls this
 * code; it is the checker that the GPU path is compared against in tests/, in
 * __graft_entry__.smoke() and in bench.py's cpu_baseline leg.
 *
 * Every function cites the reference file:line it restates (paths relative to the
 * reference checkout).  Streams use the reference's layouts: dimension-major
 * matrices `m[d * count + i]` of int64 values.
 */
#ifndef CHAIN_ORACLE_H
#define CHAIN_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    CO_OK = 0,
    CO_INVALID_ARGUMENT = 1,
    CO_NONFINITE_INPUT = 2,
    CO_QUANT_OVERFLOW = 3,
    CO_CORRUPT_STREAM = 4,
    CO_NO_MEMORY = 5
};

typedef struct {
    int64_t min_value, max_value, max_difference, min_correction, max_correction;
} co_wrap;

/* cpp/chain/lcps_cpp.cpp:2069-2110 (with reconstruct_coordinate_cpp :1496-1500 and
 * within_error_bound_cpp :1502-1523).  pts is point-major (N, D) float64.
 * Outputs: mins[D]; bid[D*N]; rel[D*N]; corrections (index i*D+d, original value)
 * in increasing index order into corr_idx/corr_val (capacity N*D); *ncorr;
 * *max_bid = max over all block ids (0 if none larger). */
int co_quantize(const double* pts, uint64_t n, uint32_t dims, double eb, int64_t p_eff,
                double* mins, int64_t* bid, int64_t* rel, uint64_t* corr_idx,
                double* corr_val, uint64_t* ncorr, int64_t* max_bid);

/* cpp/chain/lcps_cpp.cpp:2112-2200.  next-in-same-block (hash scan in the reference,
 * a stable index sort here) and the level-1 choice.  Outputs idrel[N] and the
 * explicit block records blocks[D*N] (first *nblocks records used, dimension-major
 * with stride N). */
int co_level1(const int64_t* bid, uint64_t n, uint32_t dims, int64_t threshold, int l1,
              int64_t max_bid, int64_t* idrel, int64_t* blocks, uint64_t* nblocks);

/* cpp/chain/lcps_cpp.cpp:1305-1454 (l2), :1456-1478 (!l2), :1221-1253 (wrap).
 * blocks is dimension-major with stride `stride`.  Outputs choice2[B],
 * keep[D*stride_out] (*nkeep records), diff[D*stride_out] (*ndiff records),
 * both dimension-major with stride stride_out, and the wrap parameters. */
int co_level2(const int64_t* blocks, uint64_t nrec, uint64_t stride, uint32_t dims, int l2,
              int64_t* choice2, int64_t* keep, uint64_t* nkeep, int64_t* diff,
              uint64_t* ndiff, uint64_t stride_out, co_wrap* wrap);

/* cpp/chain/lcps_cpp.cpp:1221-1253 */
int co_make_wrap(int64_t min_value, int64_t max_value, co_wrap* wrap);

/* cpp/chain/lcps_cpp.cpp:1890-1961: level-2 inverse and backward level-1 pass.
 * Inputs are the five streams (dimension-major, strides = their own counts).
 * Output q[D*N] dimension-major. */
int co_decode_q(uint64_t n, uint32_t dims, int64_t p, int64_t wrap_min, int64_t wrap_max,
                const int64_t* idrel, const int64_t* diff, uint64_t ndiff,
                const int64_t* keep, uint64_t nkeep, const int64_t* choice2,
                uint64_t nchoice, const int64_t* rel, int64_t* q);

/* cpp/chain/lcps_cpp.cpp:1963-1993: FMA reconstruction plus exact corrections.
 * q is dimension-major; out is point-major (N, D) float64. */
int co_reconstruct(uint64_t n, uint32_t dims, const int64_t* q, const double* mins, double eb,
                   const uint64_t* corr_idx, const double* corr_val, uint64_t ncorr,
                   double* out);

#ifdef __cplusplus
}
#endif
#endif
