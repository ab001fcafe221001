/*
 * chain_b200 -- C ABI of the B200-native Chain compressor (order-preserving,
 * error-bounded lossy compression of particle coordinates).
 *
 * This is the drop-in boundary for the reference's GPU compress/decompress path.
 * Every entry point takes plain pointers and sizes.  Host or device buffers are
 * both accepted wherever a buffer is passed (the library asks the CUDA runtime
 * which one it got).  Errors never abort the process: each call returns a status
 * and leaves a message for chain_last_error_message().
 *
 * Reference interfaces replaced (paths within the reference project):
 *   chain_compress      <- lcps_gpu_cpp.lcps_compress2_gpu
 *                          (cu/chain/lcps_gpu_cpp.cu:718-1091, module :1095-1102),
 *                          wrapped by chain_caller.chain_gpu (chain_caller.py:38-40)
 *   chain_decompress    <- lcps_gpu_decompress_ans.lcps_decompress_gpu
 *                          (cu/decompress/lcps_gpu_decompress_ans.cu:2701-2896,
 *                          module :2898-2921), wrapped by chain_caller.gpu_decompress
 *                          (chain_caller.py:33-35)
 * Integer semantics follow the reference CPU encoder cpp/chain/lcps_cpp.cpp:2017-2338
 * bit for bit (FP64 quantization, level-1 chaining, level-2 block differencing).
 */
#ifndef CHAIN_B200_H
#define CHAIN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CHAIN_B200_ABI_VERSION 1

#if defined(__GNUC__)
#define CHAIN_API __attribute__((visibility("default")))
#else
#define CHAIN_API
#endif

/* Status codes.  They mirror the reference's validation classes: std::invalid_argument
 * (CHAIN_ERR_INVALID_ARGUMENT) and std::runtime_error for everything else. */
typedef enum chain_status {
    CHAIN_OK = 0,
    CHAIN_ERR_INVALID_ARGUMENT = 1, /* eb <= 0, p <= 0, bad shape, bad options        */
    CHAIN_ERR_NONFINITE_INPUT = 2,  /* lcps_cpp.cpp:2075 "coordinates must be finite" */
    CHAIN_ERR_QUANT_OVERFLOW = 3,   /* quantized value outside the supported range    */
    CHAIN_ERR_CORRUPT_STREAM = 4,   /* decoder: container failed validation           */
    CHAIN_ERR_DEVICE = 5,           /* CUDA runtime error                             */
    CHAIN_ERR_OUT_OF_MEMORY = 6,    /* device arena or host allocation failed         */
    CHAIN_ERR_UNSUPPORTED = 7,      /* valid input outside this build's limits        */
    CHAIN_ERR_BUFFER_TOO_SMALL = 8  /* caller buffer smaller than the result          */
} chain_status;

typedef enum chain_dtype { CHAIN_F32 = 4, CHAIN_F64 = 8 } chain_dtype;

/* CHAIN_SOA: coordinates as (D, N), C-contiguous -- the layout lcps_compress2_gpu takes.
 * CHAIN_AOS: coordinates as (N, D), C-contiguous -- the layout lcps_compress2 takes. */
typedef enum chain_layout { CHAIN_SOA = 0, CHAIN_AOS = 1 } chain_layout;

typedef struct chain_ctx chain_ctx;

/* Options.  Zero-initialise, set struct_size = sizeof(chain_opts), then override.
 * bl/l1/l2 are the reference CPU encoder's ablation switches (lcps_cpp.cpp:2340-2355):
 * a negative value means "default" (enabled). */
typedef struct chain_opts {
    uint32_t struct_size;
    int32_t bl;                     /* block partitioning (p used as given; else p = 1)   */
    int32_t l1;                     /* level-1 chaining                                   */
    int32_t l2;                     /* level-2 block differencing                         */
    uint32_t rans_bytes_per_lane;   /* entropy stage: target coded bytes per rANS lane
                                       (each lane adds its final state, prec + 10 bits);
                                       0 = default 4096                                   */
    uint32_t rans_max_steps;        /* entropy stage: most symbols one lane codes
                                       (serial depth); 0 = default 1024                   */
    uint32_t reserved[10];
} chain_opts;

/* Creates a context bound to CUDA device `device`.  `cuda_stream` is a cudaStream_t
 * (NULL = a stream owned by the context).  The context owns a device arena that
 * grows on demand and is reused across calls; calls on one context are serialised
 * by the caller. */
CHAIN_API chain_status chain_ctx_create(int device, void* cuda_stream, chain_ctx** out);
CHAIN_API void chain_ctx_destroy(chain_ctx* ctx);

/* Message of the last failed call on this thread ("" if none). */
CHAIN_API const char* chain_last_error_message(void);

/* Upper bound of the container size for n points of `dims` coordinates. */
CHAIN_API size_t chain_compress_bound(uint64_t n, uint32_t dims);

/* Compresses n points of `dims` coordinates (float32 or float64) with absolute error
 * bound eb, block size p and level-1 threshold `threshold`.  `points` may be host or
 * device memory.  On success the container stays in the context and *out_len is its
 * size; fetch it with chain_result_copy or read it in place at chain_result_device_ptr.
 * Synchronous: returns after the device work is complete. */
CHAIN_API chain_status chain_compress(chain_ctx* ctx, const void* points, chain_dtype dtype,
                            chain_layout layout, uint64_t n, uint32_t dims, double eb,
                            int64_t p, int64_t threshold, const chain_opts* opts,
                            size_t* out_len);

/* Copies the last container of this context to dst (host or device). */
CHAIN_API chain_status chain_result_copy(chain_ctx* ctx, void* dst, size_t capacity);

/* Device address of the last container of this context (valid until the next call). */
CHAIN_API const void* chain_result_device_ptr(const chain_ctx* ctx);

/* Reads N, D and the stored input dtype of a container held in HOST memory. */
CHAIN_API chain_status chain_peek(const void* container, size_t len, uint64_t* n, uint32_t* dims,
                        chain_dtype* input_dtype);

/* Decompresses a container (host or device memory) into `out` (host or device),
 * which must hold n*dims values of out_dtype in out_layout.  CHAIN_F64 output
 * reproduces the reference CPU decoder bit for bit (lcps_cpp.cpp:1963-1993);
 * CHAIN_F32 output is that value rounded to float32. */
CHAIN_API chain_status chain_decompress(chain_ctx* ctx, const void* container, size_t len,
                              chain_dtype out_dtype, chain_layout out_layout, void* out,
                              size_t out_capacity_bytes, uint64_t* n, uint32_t* dims);

/* ---- batches of independent frames ------------------------------------------------
 * A batch object owns `workers` contexts on one device (each with its own stream and
 * arenas, kept between batches).  chain_batch_compress / chain_batch_decompress run
 * the items on those contexts from `workers` host threads, so that many frames'
 * kernels and host round trips overlap; each item's result is identical to the
 * one-frame call's.  Items of one call must not share output buffers.  This is the
 * batched form of the path for collections of frames (for instance 256 frames of
 * 1e4..2e6 particles each); the reference processes such collections one frame per
 * call (chain_caller.py:33-40 in a loop).
 *
 * Item fields, compress:   input = points, dtype/layout/n/dims/eb/p/threshold as for
 *                          chain_compress; output = container buffer (host or device)
 *                          of output_capacity bytes (chain_compress_bound is enough).
 * Item fields, decompress: input = container of input_bytes bytes; dtype/layout = the
 *                          output's; output = points buffer of output_capacity bytes;
 *                          n and dims are returned.
 * Returned in every item:  output_bytes and status.  The call returns CHAIN_OK when
 * every item succeeded, else the first failing item's status, with its index in
 * chain_last_error_message(). */
typedef struct chain_batch chain_batch;
typedef struct chain_batch_item {
    const void* input;
    size_t input_bytes;
    chain_dtype dtype;
    chain_layout layout;
    uint64_t n;
    uint32_t dims;
    double eb;
    int64_t p;
    int64_t threshold;
    void* output;
    size_t output_capacity;
    size_t output_bytes;
    chain_status status;
} chain_batch_item;

CHAIN_API chain_status chain_batch_create(int device, int workers, chain_batch** out);
CHAIN_API void chain_batch_destroy(chain_batch* batch);
CHAIN_API chain_status chain_batch_compress(chain_batch* batch, chain_batch_item* items, size_t count,
                                            const chain_opts* opts);
CHAIN_API chain_status chain_batch_decompress(chain_batch* batch, chain_batch_item* items, size_t count);

/* Autotuner of the batched compress path (no counterpart in the reference, which has
 * no batched path).  Runs `items` (a sample of the frames to come, in the compress item
 * form; their outputs are overwritten) through chain_batch_compress once per candidate:
 * rANS lane depth (chain_opts.rans_max_steps) 1024, 512 or 256, on all, half or a
 * quarter of the batch's contexts; each candidate is timed on the host clock (the best
 * of two runs after one warm-up).  It keeps the fastest candidate whose total container
 * bytes on the sample stay within 0.3% of the default's (1024, all contexts), and from
 * then on chain_batch_compress uses it whenever its opts argument is null.  Kernel block
 * sizes and the 8-bit sort digits are fixed by the kernels' resource budgets and are not
 * tuned. */
typedef struct chain_tune_result {
    uint32_t rans_max_steps;   /* chosen lane depth */
    uint32_t workers;          /* contexts a batch call uses */
    double best_ms;            /* the chosen candidate's sample time */
    double default_ms;         /* the default candidate's sample time */
    uint64_t best_bytes;       /* container bytes of the sample, chosen candidate */
    uint64_t default_bytes;    /* ... default candidate */
} chain_tune_result;
CHAIN_API chain_status chain_batch_tune(chain_batch* batch, chain_batch_item* items, size_t count,
                                        chain_tune_result* result);

/* Rewrites an LCG2 container as the reference CPU Chain's LCP2 bitstream, which the
 * reference decoder (lcps_cpu_decompress.lcps_decompress_serial, chain_caller.py:23-30)
 * reads directly and decodes to the same points.  Host buffers only; no GPU is used.
 * Components become RVMX (values below 2^18) or RTG4 and the exact corrections a Zstd
 * frame of stored blocks, so the result is larger than the reference's own output.
 * With out == NULL or too small a capacity it returns CHAIN_ERR_BUFFER_TOO_SMALL and
 * the needed size in *out_len.  Replaces nothing in the reference (its GPU output,
 * LCG2 v1, has no LCP2 conversion); it is the on-disk bridge between the two formats. */
CHAIN_API chain_status chain_transcode_lcp2(const void* container, size_t len, void* out, size_t capacity,
                                            size_t* out_len);

/* ---- request server ---------------------------------------------------------------
 * A server owns `workers` contexts on one device, each driven by its own host thread.
 * Submitted requests (op 0 = compress, 1 = decompress; the item as for the batch calls,
 * owned by the caller until chain_server_wait returns) wait in one FIFO queue; a free
 * worker admits the head request when its estimated device working set fits in
 * memory_budget_bytes next to the running requests (a request larger than the budget
 * runs alone).  Contexts, arenas and streams stay resident between requests.
 * chain_server_wait blocks until the request has finished and returns its status, its
 * queueing time (submit -> start) and its service time (start -> end), in milliseconds.
 * Every submitted ticket must be waited for once.  chain_server_destroy stops admission,
 * finishes every queued request and returns once no thread is inside chain_server_wait;
 * no call on the server may start after destroy has begun.  No counterpart in the reference,
 * which compresses one frame per synchronous call (chain_caller.py:33-40). */
typedef struct chain_server chain_server;
CHAIN_API chain_status chain_server_create(int device, int workers, size_t memory_budget_bytes,
                                           const chain_opts* opts, chain_server** out);
CHAIN_API void chain_server_destroy(chain_server* server);
CHAIN_API chain_status chain_server_submit(chain_server* server, int op, chain_batch_item* item,
                                           uint64_t* ticket);
CHAIN_API chain_status chain_server_wait(chain_server* server, uint64_t ticket, double* queue_ms,
                                         double* service_ms);

/* Decompression that allocates nothing, for callers that cannot allocate memory when
 * they decode (a plug-in inside an application that owns the device memory pool or
 * runs under a hard memory cap; a loop that must not pay for cudaMalloc/cudaFree, which
 * can synchronise the device).  No counterpart in the reference: it is this library's
 * own addition.  Same arguments, output and errors as chain_decompress, without a
 * context: it runs on the calling thread's current device, on `cuda_stream` (a
 * cudaStream_t; NULL = the default stream), and calls no cudaMalloc, cudaFree or any
 * other allocating routine.  Its working memory is one fixed 64 MiB device array that
 * every GPU on which the library's module is loaded holds until the process exits;
 * frames whose decoder working set does not fit are rejected with
 * CHAIN_ERR_UNSUPPORTED and a message giving the bytes needed.  All calls share that
 * array and keep the last call's contents (each call clears what must start at zero);
 * overlapping calls would race on it, so calls are serialised by a process-wide lock
 * and each returns only after its GPU work has completed.  The first call on a device
 * looks up the array's address (cudaGetSymbolAddress): make it before any stream
 * capture begins on that device. */
CHAIN_API chain_status chain_decompress_noalloc(const void* container, size_t len, chain_dtype out_dtype,
                                                chain_layout out_layout, void* out, size_t out_capacity_bytes,
                                                uint64_t* n, uint32_t* dims, void* cuda_stream);

/* Debug/parity entry: after chain_compress on this context, copies the encoder's
 * integer streams to host buffers (each may be NULL).  Layout is record-major
 * (point-major) int64, matching the order the reference feeds its entropy stage
 * (lcps_cpp.cpp:970-986):  idrel[n], diff[ndiff*dims], keep[nkeep*dims],
 * choice2[nblocks], rel[n*dims]; counts are returned through the pointers. */
CHAIN_API chain_status chain_debug_streams(chain_ctx* ctx, int64_t* idrel, int64_t* diff,
                                 uint64_t* ndiff, int64_t* keep, uint64_t* nkeep,
                                 int64_t* choice2, uint64_t* nblocks, int64_t* rel);

/* Stage timing: when enabled, each call records CUDA events between its stages on the
 * context's stream.  chain_stage_times returns the stages of the last call (name and
 * milliseconds since the previous stage) and their count.  Tracing aid only: timing
 * adds one event record per stage. */
CHAIN_API chain_status chain_set_stage_timing(chain_ctx* ctx, int enabled);

/* Number of CUDA kernels the library has launched in this process so far (all threads,
 * batch workers included). */
CHAIN_API uint64_t chain_launch_count(void);
/* Number of memory allocations (cudaMalloc and cudaMallocHost calls) the library has
 * made in this process so far, all threads included.  Tracing aid: it lets a caller
 * check that a code path allocated nothing (no counterpart in the reference). */
CHAIN_API uint64_t chain_alloc_count(void);
CHAIN_API int chain_stage_times(const chain_ctx* ctx, const char** names, float* ms, int max);

#ifdef __cplusplus
}
#endif
#endif /* CHAIN_B200_H */
