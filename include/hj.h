/* hj.h -- C ABI of the B200 epsilon-join cardinality engine (libhj.so).
 *
 * The engine counts pairs of points in R^d whose Euclidean distance is at most
 * eps: unordered pairs {a, b}, a != b, within one set (self-join), or ordered
 * pairs (a in A, b in B) between two sets. It replaces the count path of the
 * hilbertJoin reference (perdacherMartin/hilbertJoin): the library functions
 * test_ego_loop3_macro / test_ego_loop3_noself behind the executables
 * hilbertSelfJoinCardinality / hilbertJoinCardinality.
 *
 * Pair test (every form returns exactly this count): with acc = 0 and, for
 * k = 0 .. d-1, acc = fma(a_k - b_k, a_k - b_k, acc) evaluated in IEEE FP64,
 * a pair counts iff acc <= eps * eps (FP64). FP32 inputs are widened to FP64
 * exactly first.
 *
 * Conventions: every function returns an hj_status; none exits the process.
 * Inputs are const and never modified (the reference sorts its input in place,
 * hilbertjoin/egojoin.cpp:159-168, and leaves it permuted). No allocation
 * slack is required of the caller (the reference requires +16384 bytes,
 * main.cpp:59). Calls are reentrant: each calling host thread gets its own
 * device context and stream unless it passes its own stream.
 */
#ifndef HJ_H
#define HJ_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define HJ_API __attribute__((visibility("default")))
#else
#define HJ_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The reference has no error reporting: it calls exit(1) on
 * allocation, I/O and argument errors (util/allocation.cpp:14-15,
 * util/dataIo.cpp:125,136, util/arguments.cpp:21). */
typedef enum {
    HJ_OK = 0,
    HJ_ERR_INVALID_ARG = 1,   /* null pointer, n or d out of range, eps <= 0 or not finite,
                                 a non-finite coordinate, or a cell index out of int32 range */
    HJ_ERR_OOM = 2,           /* device allocation failed */
    HJ_ERR_CUDA = 3,          /* a CUDA call failed; hj_last_error() has the text */
    HJ_ERR_TIMEOUT = 4,       /* a bounded device-side wait gave up (kernel returned early) */
    HJ_ERR_BAND_OVERFLOW = 5, /* tensor-core band queue still too small after regrowth */
    HJ_ERR_NO_DEVICE = 6,     /* no usable sm_100 device */
    HJ_ERR_UNSUPPORTED = 7,   /* the requested form cannot run this input (see hj_opts.form) */
    HJ_ERR_BUSY = 8,          /* serving: request rejected by admission (memory budget) */
    HJ_ERR_NOT_FOUND = 9,     /* serving: unknown handle or request id */
    HJ_ERR_CAPACITY = 10      /* pair output: more pairs than the caller's capacity (*n_pairs = the total) */
} hj_status;

/* How pair distances are evaluated. Every form returns the exact count of the
 * pair test above. */
typedef enum {
    /* FP64 direct difference on CUDA cores, early exit every 8 dims once all
     * pairs of a warp exceed eps^2 (the reference's KBLOCK early exit,
     * hilbertjoin/egojoin.h:350-359). The drop-in form; d <= 256. */
    HJ_FORM_PLAIN_FP64 = 0,
    /* dist^2 = |a|^2 + |b|^2 - 2 a.b with a.b on tcgen05 tensor cores in TF32
     * (operands rounded to TF32, FP32 accumulation); every pair within a
     * derived error bound of eps^2 is re-evaluated with the FP64 pair test. */
    HJ_FORM_TC_TF32 = 1,
    /* As TF32, with a.b as the BF16 split three-product
     * a_hi.b_hi + a_hi.b_lo + a_lo.b_hi (a = a_hi + a_lo), FP32 accumulation. */
    HJ_FORM_TC_BF16X3 = 2,
    /* HJ_FORM_TC_FP16 when the input allows it (d <= 256, coordinates within
     * +-1e18) and the join is not small (na * nb * d > 2e10, where the plain
     * form's fewer stages measured faster), else HJ_FORM_PLAIN_FP64. */
    HJ_FORM_AUTO = 3,
    /* As TF32 with FP16 operands at twice the tensor-core rate: the centred
     * coordinates are scaled by a power of two 2^s (exact) so that the largest
     * lands in [2^14, 2^15), then rounded once from FP64 to FP16 (11-bit
     * significand, the precision of TF32); a.b in FP32 accumulation, band
     * pairs re-evaluated with the FP64 pair test. */
    HJ_FORM_TC_FP16 = 4
} hj_form;

/* Operand centring of the tensor-core forms (hj_opts.tc_centring). */
typedef enum {
    /* HJ_CENTRING_BLOCK when, with one global centre, more than an eighth of
     * the block pairs would run on the FP64 kernel (the norm expansion's
     * cancellation limit: eps small against the spread of the data) and
     * d <= 64; HJ_CENTRING_GLOBAL otherwise. */
    HJ_CENTRING_AUTO = 0,
    /* One centre for the whole join (the per-dim midpoint of the data). */
    HJ_CENTRING_GLOBAL = 1,
    /* A centre per 128-point block of the EGO order, exact in the operand
     * type, and each point stored as that centre plus its residual rounded
     * once; the operand rows carry the residual and centre cross terms and
     * the point's norm as extra K columns (about 3d of them), so the error
     * band scales with the residual norms. Every tensor-core form, d <= 64. */
    HJ_CENTRING_BLOCK = 2
} hj_centring;

typedef struct {
    int32_t form;          /* hj_form; default HJ_FORM_PLAIN_FP64 */
    int32_t active_dims;   /* stripes split the first active_dims dims into neighbour cells
                              (the reference's -s; (3^s+1)/2 stripes, main.cpp:54).
                              -1 = default (3 for self-joins, 2 for two-set joins,
                              as egojoin.cpp:847 hard-codes) */
    int32_t ref_compat;    /* nonzero: count only among the first 8*floor(n/8) EGO-sorted
                              points of each set, as the reference's block loops do */
    int32_t device;        /* CUDA device ordinal; -1 = current */
    void *stream;          /* cudaStream_t to run on; NULL = the calling thread's own stream */
    int32_t shard_index;   /* with shard_count > 1: count only shard `shard_index` of the join's */
    int32_t shard_count;   /* work list (contiguous, equal-load ranges of the Hilbert-ordered block
                              pairs, the reference's equal-load split egojoin.h:214-222). The counts
                              of shards 0..shard_count-1 sum to the full count. */
    int32_t reorder_dims;  /* nonzero: order the dims of the cell key (EGO order, stripes)
                              by ascending cost, most selective first, as hj_dim_order
                              computes it from set A (the reference's join driver does this
                              before every join, mainJoin.cpp:97-100). Distances are still
                              summed in the caller's dim order, so the count is unchanged;
                              only the work (candidate pairs) changes. */
    int32_t item_chunk;    /* B tiles per work item of the distance kernel; 0 = default (32 for
                              the tensor-core forms, 16 for the plain form). Smaller chunks
                              balance small joins across the SMs, larger ones keep B tiles in
                              L2; hilbertjoin_b200.autotune picks it per dimension. */
    int32_t tc_centring;   /* hj_centring; 0 = HJ_CENTRING_AUTO */
    int32_t reserved_i;
    uint64_t reserved[1];
} hj_opts;

/* Per-call statistics (all optional). Times are device times of each stage
 * measured with CUDA events. */
typedef struct {
    double h2d_ms;          /* host -> device copy of the input */
    double sort_ms;         /* cell keys + stable LSD radix sort + gather (the reference's SORTTIME) */
    double index_ms;        /* stripe bounds + block-pair work list (the reference's INDEXTIME) */
    double join_ms;         /* distance kernel(s) */
    double kernel_ms;       /* the main distance kernel alone (CUDA events around its launch) */
    double recheck_ms;      /* FP64 re-evaluation of band pairs (tensor-core forms) */
    double total_ms;        /* whole call, host wall clock */
    double loadpercent;     /* candidate pairs / all pairs * 100 (the reference's LOADPERCENT
                               is on 8-point blocks, egojoin.cpp:797) */
    uint64_t candidate_pairs; /* point pairs inside the block-pair work list */
    uint64_t tile_pairs;    /* block pairs in the work list */
    uint64_t work_items;    /* items of the persistent kernel's work list */
    uint64_t band_pairs;    /* pairs sent to the FP64 recheck */
    double band_fraction;   /* band_pairs / candidate_pairs */
    double band_halfwidth_rel; /* tensor-core bound: |dist2 - est| <= c * (|a|^2 + |b|^2) + abs; this is c */
    double max_abs_err_band;   /* largest |est - dist2| over the band pairs (tensor-core forms) */
    uint64_t fp64_items;    /* tensor-core forms: work items routed to the FP64 kernel because
                               their error band would exceed eps^2 / 2 */
    int32_t form_used;      /* hj_form actually run */
    int32_t stripes;        /* stripe count (3^s+1)/2 for self-joins, 3^s for two-set joins */
    int32_t kernel_launches;/* kernels this call launched */
    int32_t tc_centring;    /* hj_centring the tensor-core kernel ran with (0: no tensor-core kernel) */
    double reorder_ms;      /* dimension cost sampling and ordering (opts.reorder_dims) */
    uint64_t reserved[3];
} hj_stats;

HJ_API void hj_opts_init(hj_opts *o);
HJ_API const char *hj_status_str(int status);
/* Text of the last error on this host thread ("" if none). */
HJ_API const char *hj_last_error(void);
/* Library version, e.g. "hj 1.0.0 sm_100a". */
HJ_API const char *hj_version(void);
/* Number of SMs of a device (-1 = current), 0 if there is none. */
HJ_API int hj_device_sm_count(int device);

/* Self-join count over n points of dimension d, row-major (point i at
 * pts[i*d .. i*d+d-1]). Replaces test_ego_loop3_macro
 * (hilbertjoin/egojoin.h:56, egojoin.cpp:777-838). */
HJ_API int hj_self_join_count(const double *pts, uint64_t n, uint32_t d, double eps, const hj_opts *opts,
                       uint64_t *count, hj_stats *stats);
HJ_API int hj_self_join_count_f32(const float *pts, uint64_t n, uint32_t d, double eps, const hj_opts *opts,
                           uint64_t *count, hj_stats *stats);

/* Two-set join count, ordered pairs (a in A, b in B). Replaces
 * test_ego_loop3_noself (hilbertjoin/egojoin.h:64, egojoin.cpp:840-907). */
HJ_API int hj_join_count(const double *A, uint64_t nA, const double *B, uint64_t nB, uint32_t d, double eps,
                  const hj_opts *opts, uint64_t *count, hj_stats *stats);
HJ_API int hj_join_count_f32(const float *A, uint64_t nA, const float *B, uint64_t nB, uint32_t d, double eps,
                      const hj_opts *opts, uint64_t *count, hj_stats *stats);

/* The qualifying pairs themselves. pairs[2k], pairs[2k+1] are the input
 * indices (i, j) of pair k -- the layout of the reference's
 * struct join_pair { size_t p1, p2; } (hilbertjoin/egojoin.h:32-35), whose
 * queue output (hilbertjoin/test_ego_loop3_queue.cpp:19-37) the reference
 * compiles out under COUNT_ONLY. Self joins list each unordered pair once with
 * i < j; two-set joins list (index in A, index in B). Sorted by (i, j).
 * The reference pushes indices into its EGO-sorted array; these are indices
 * into the caller's unsorted input. Always computed by the plain FP64 form
 * (d <= 256; opts->form is ignored), so the pairs are exactly the ones the
 * count functions count. If more than `capacity` pairs qualify nothing is
 * written, *n_pairs is set to the number and HJ_ERR_CAPACITY is returned
 * (capacity 0 with pairs NULL asks for the number alone). At most 2^32 - 1
 * pairs can be listed (the device pair buffer is indexed with 32-bit
 * offsets): a join with more returns HJ_ERR_UNSUPPORTED with *n_pairs set to
 * the count. */
HJ_API int hj_self_join_pairs(const double *pts, uint64_t n, uint32_t d, double eps, const hj_opts *opts,
                              uint64_t *pairs, uint64_t capacity, uint64_t *n_pairs, hj_stats *stats);
HJ_API int hj_self_join_pairs_f32(const float *pts, uint64_t n, uint32_t d, double eps, const hj_opts *opts,
                                  uint64_t *pairs, uint64_t capacity, uint64_t *n_pairs, hj_stats *stats);
HJ_API int hj_join_pairs(const double *A, uint64_t nA, const double *B, uint64_t nB, uint32_t d, double eps,
                         const hj_opts *opts, uint64_t *pairs, uint64_t capacity, uint64_t *n_pairs,
                         hj_stats *stats);
HJ_API int hj_join_pairs_f32(const float *A, uint64_t nA, const float *B, uint64_t nB, uint32_t d, double eps,
                             const hj_opts *opts, uint64_t *pairs, uint64_t capacity, uint64_t *n_pairs,
                             hj_stats *stats);

/* Epsilon-grid order of a point set computed on the device: perm[r] is the
 * input index of the point at rank r, ranks ordered lexicographically by the
 * cell vector floor(x/eps) (dim 0 most significant), ties in input order
 * (stable). If `sorted` is non-null it receives the rows in that order.
 * Replaces epsilonGridOrdering (hilbertjoin/egojoin.cpp:159-168), which sorts
 * the caller's array in place with an unstable quicksort. */
HJ_API int hj_ego_sort(const double *pts, uint64_t n, uint32_t d, double eps, const hj_opts *opts, uint64_t *perm,
                       double *sorted);

/* EGO sort of a device-resident point set that allocates no memory. For
 * callers that cannot call cudaMalloc while they run: an application whose own
 * memory pool owns the device, or a latency-critical stream that must not pay
 * cudaMalloc's implicit synchronisation. All temporaries live in one fixed
 * 32 MiB array inside libhj.so (a file-scope __device__ array that every GPU
 * loading the library holds until the process exits); sizes whose temporaries
 * exceed it (about 4 n (W + 4) bytes, W = 32-bit words of the packed cell key)
 * are rejected with HJ_ERR_INVALID_ARG. pts: device rows [n][d], dtype_bytes 8
 * or 4; perm: device uint32 [n] output, the same stable order as hj_ego_sort.
 * The first call on a device looks up the array's address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * Calls share the array and it keeps the last call's contents: calls that
 * overlap on the GPU race, calls on one stream are ordered. Each call blocks
 * the calling host thread until the cell-statistics kernels on `stream`
 * (NULL = default stream) have finished -- it reads 16 d + 4 bytes back and
 * synchronises `stream` -- then queues the key packing and the sort passes on
 * `stream` and returns without waiting for them. Failures set hj_last_error().
 * This entry point has no counterpart in the reference. */
HJ_API int hj_ego_sort_device_noalloc(const void *pts, int dtype_bytes, uint64_t n, uint32_t d, double eps,
                                      uint32_t *perm, void *stream);

/* Dimension order for the cell key, computed on the device. Per dim j the
 * cost is the number of unordered pairs of sampled points whose cells in dim j
 * are equal or adjacent -- sum h(h-1)/2 + sum h[c-1] h[c] over the sample's
 * cell histogram, the Super-EGO selectivity estimate the reference computes
 * in outputStatistics (hilbertjoin/egojoin.cpp:523-592). Dims are ranked by
 * ascending cost, ties by dim index, and reorder_dim[j] receives the new
 * position of dim j (the reference's convention, egojoin.cpp:587-589). Unlike
 * the reference, the sample is deterministic -- the min(n, 8192) points
 * floor(s n / S), s = 0..S-1 -- and every dim is ranked (the reference leaves
 * dims with cells beyond +-100000 uncosted). costs (optional) receives the d
 * costs. pts: host FP64 rows. */
HJ_API int hj_dim_order(const double *pts, uint64_t n, uint32_t d, double eps, const hj_opts *opts,
                        int32_t *reorder_dim, uint64_t *costs);

/* The same calls on inputs already in device memory (row-major, d per row).
 * `dtype_bytes` is 8 (FP64) or 4 (FP32). The pointers must be device (or
 * managed) memory of the device the call runs on. */
HJ_API int hj_self_join_count_device(const void *pts, int dtype_bytes, uint64_t n, uint32_t d, double eps,
                              const hj_opts *opts, uint64_t *count, hj_stats *stats);
HJ_API int hj_join_count_device(const void *A, uint64_t nA, const void *B, uint64_t nB, int dtype_bytes, uint32_t d,
                         double eps, const hj_opts *opts, uint64_t *count, hj_stats *stats);

/* Drop-in replacements with the reference's exact argument lists. The count
 * uses the reference's convention (first 8*floor(n/8) EGO-sorted points). The
 * input is left untouched (the reference leaves it sorted). Times are in
 * seconds like the reference's. `stripes` is (3^s+1)/2 as main.cpp:54 computes
 * it; `activedims` is ignored exactly as the reference ignores it (it
 * hard-codes 2, egojoin.cpp:847). Errors are reported as *countresult = 0 and
 * hj_last_error(). */
HJ_API void hj_test_ego_loop3_macro(size_t n, size_t d, double epsilon, double *array, size_t *countresult, int stripes,
                             double *sortTime, double *indextime, double *loadpercent);
HJ_API void hj_test_ego_loop3_noself(const size_t nA, const size_t nB, const int d, const double epsilon, double *arrayA,
                              double *arrayB, size_t *countresult, const int activedims, double *sortTime,
                              double *indextime, double *loadpercent);

/* Testing hook: the tensor-core form's dist^2 estimate of every pair (a in
 * A, b in B), written to out[i * nB + j] in input order (nA * nB floats).
 * Runs a two-set join with eps so large that all points share one cell.
 * Not thread-safe; no reference counterpart. */
HJ_API int hj_debug_tc_estimates(const float *A, uint64_t nA, const float *B, uint64_t nB, uint32_t d, int form,
                                 float *out);
/* As hj_debug_tc_estimates with the operand centring (hj_centring) and eps
 * given (eps <= 0: the one that puts all points in one cell); pairs outside
 * the work list are left NaN. Statistics of the join into *stats if non-null.
 * Not thread-safe; no reference counterpart. */
HJ_API int hj_debug_tc_estimates_ex(const float *A, uint64_t nA, const float *B, uint64_t nB, uint32_t d, int form,
                                    int centring, double eps, float *out, hj_stats *stats);

/* Testing hook: with gate_ns > 0, every following tensor-core kernel launch
 * of this process makes its epilogue wait gate_ns on a device barrier that
 * nothing arrives on; the wait runs out, the kernel raises its timeout error,
 * drains the copies and MMAs it issued, frees its tensor memory and returns,
 * and the call returns HJ_ERR_TIMEOUT. 0 restores normal operation. gate_ns
 * must not exceed the engine's wait limit (2 s). Not thread-safe; no
 * reference counterpart (the reference has no device waits). */
HJ_API int hj_debug_set_wait_gate(uint64_t gate_ns);

/* ---------------------------------------------------------------- batching
 * Many joins of uneven n, d and eps in one persistent tensor-core launch. The
 * jobs' inputs are device rows (dtype_bytes 4 or 8, the same for all jobs);
 * b == NULL makes a job a self-join. hj_batch_create plans the batch --
 * every job's EGO sort, layouts and work list, merged into one work list over
 * one operand matrix -- and runs it once (its counts are ready at once);
 * hj_batch_run enqueues another run on `stream` (NULL = the batch's own
 * stream) with no host synchronisation, so a run can be captured into a CUDA
 * graph and replayed; hj_batch_counts waits for the last run and returns one
 * count per job (the same as the job's own hj_*_join_count_device call).
 * opts: form (HJ_FORM_TC_FP16 / _TF32 / _BF16X3; AUTO = FP16), active_dims,
 * ref_compat, device, stream (for planning); d <= 256 per job. The input
 * buffers are read only during hj_batch_create. No counterpart in the
 * reference, which runs one join per process. */
typedef struct {
    const void *a;    /* device rows [na][d] */
    const void *b;    /* device rows [nb][d], or NULL for a self-join of a */
    uint64_t na, nb;
    uint32_t d;
    uint32_t reserved;
    double eps;
} hj_batch_job;
typedef struct hj_batch hj_batch;
HJ_API int hj_batch_create(const hj_batch_job *jobs, uint32_t n_jobs, int dtype_bytes, const hj_opts *opts,
                           hj_batch **out);
HJ_API int hj_batch_run(hj_batch *batch, void *stream);
HJ_API int hj_batch_counts(hj_batch *batch, uint64_t *counts, hj_stats *stats);
/* Frees the batch; its runs must have finished (hj_batch_counts, or a
 * synchronisation of the streams and graphs that ran it). */
HJ_API int hj_batch_destroy(hj_batch *batch);
/* create + counts + destroy. */
HJ_API int hj_batch_count_device(const hj_batch_job *jobs, uint32_t n_jobs, int dtype_bytes, const hj_opts *opts,
                                 uint64_t *counts, hj_stats *stats);

/* ---------------------------------------------------------------- serving
 * A request loop with device-resident point sets: sets are uploaded once and
 * referenced by handle; joins are submitted from any thread, admitted against
 * a device-memory budget, and run as soon as a slot frees, overlapping on the
 * device (continuous batching). No reference counterpart. */
typedef struct hj_server hj_server;

typedef struct {
    uint64_t memory_budget_bytes; /* admission budget for per-request working memory (0 = 40 GiB) */
    int32_t max_inflight;         /* concurrent requests on the device (0 = 8) */
    int32_t device;               /* -1 = current */
    int32_t form;                 /* hj_form for every request */
    int32_t batch_max;            /* tensor-core forms: a free worker takes up to batch_max queued
                                     requests (same dtype, within the budget) and runs them as one
                                     batch (hj_batch_*: one persistent launch); 0 or 1 = one
                                     request per worker */
    int32_t block_centring;       /* 0: the requests' tensor-core joins use one global centre
                                     (HJ_CENTRING_GLOBAL); nonzero: HJ_CENTRING_AUTO, and admission
                                     counts the block-centred operands and band queue of every
                                     request that could use them (d <= 64) */
    int32_t reserved_i;
    uint64_t reserved[3];
} hj_server_opts;

typedef struct {
    uint64_t count;
    int32_t status;      /* hj_status of the request */
    int32_t form_used;
    double queue_ms;     /* submit -> start on device */
    double run_ms;       /* start -> result ready */
    double latency_ms;   /* submit -> result ready */
    uint64_t candidate_pairs;
    uint64_t band_pairs;
} hj_result;

HJ_API void hj_server_opts_init(hj_server_opts *o);
HJ_API int hj_server_create(const hj_server_opts *opts, hj_server **out);
HJ_API int hj_server_destroy(hj_server *s);
/* Uploads a point set (host, row-major; dtype_bytes 4 or 8). The set stays on
 * the device until hj_set_release. */
HJ_API int hj_set_upload(hj_server *s, const void *pts, int dtype_bytes, uint64_t n, uint32_t d, uint64_t *set_id);
HJ_API int hj_set_release(hj_server *s, uint64_t set_id);
/* Queues a self-join (set_b == set_a or set_b == 0) or a two-set join.
 * Returns at once with a request id. */
HJ_API int hj_submit(hj_server *s, uint64_t set_a, uint64_t set_b, double eps, uint64_t *request_id);
/* Non-blocking: HJ_OK with *done = 1 and the result once finished. */
HJ_API int hj_poll(hj_server *s, uint64_t request_id, int *done, hj_result *result);
/* Blocks until the request finishes (timeout_ms < 0: no limit). */
HJ_API int hj_wait(hj_server *s, uint64_t request_id, double timeout_ms, hj_result *result);

#ifdef __cplusplus
}
#endif

#endif /* HJ_H */
