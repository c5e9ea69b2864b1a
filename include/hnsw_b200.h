/*
 * hnsw_b200 -- C ABI of the B200 HNSW query engine (libhnsw_b200.so).
 *
 * Plain pointers and sizes only: every array argument is DEVICE memory owned by the caller (the
 * Python binding passes torch tensors' data pointers); the library owns only its scratch (work
 * queue, visited tables, candidate spill buffers), allocated on demand and freed by
 * hnsw_b200_close. Every entry point returns 0 on success or a negative HNSW_B200_E* code, with a
 * message available from hnsw_b200_last_error() (per calling thread). Nothing is ever trapped on
 * the device: kernels report capacity overflows per query through a status word and the library
 * re-runs those queries with larger scratch.
 *
 * The entry points replace the reference's compiled search calls (anamankev/hnsw-engine):
 *   hnsw_b200_open      <- NumbaEngine.attach_native (src/hnsw_engine/numba_engine.py:827-868):
 *                          borrows the native arrays (already validated by the caller, as
 *                          _validate_native does at numba_engine.py:878-914).
 *   hnsw_b200_search    <- NumbaEngine.batch_search / batch_search_codes / rerank
 *                          (numba_engine.py:652-713) -> _search_batch (:422-503) and
 *                          _rerank_batch (:506-530), fused into one launch; extended with a
 *                          per-query ef array and a filter on code-space searches.
 *   hnsw_b200_exact_knn <- oracle.exact_search (src/hnsw_engine/oracle.py:35-126).
 *   hnsw_b200_validate_graph <- numba_engine._validate_native (numba_engine.py:878-915), on the
 *                          uploaded arrays.
 *   hnsw_b200_quant_*   <- quantization.ScalarQuantizer.fit / encode (quantization.py:37-59).
 *   hnsw_b200_mlp_*     <- no reference counterpart (the learned early-termination network).
 */
#ifndef HNSW_B200_H
#define HNSW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define HNSW_B200_OK 0
#define HNSW_B200_EINVAL (-1)   /* bad argument */
#define HNSW_B200_ECUDA (-2)    /* a CUDA runtime call failed */
#define HNSW_B200_ENOMEM (-3)   /* device allocation failed */
#define HNSW_B200_ERETRY (-4)   /* queries still overflowed scratch after the maximum retries */

/* Metric codes, as numba_engine._METRIC_CODES (numba_engine.py:32). */
#define HNSW_B200_L2 0
#define HNSW_B200_IP 1
#define HNSW_B200_COSINE 2

/* The reference's native arrays (numba_engine.py:36-44), in device memory, unchanged layout. */
typedef struct hnsw_b200_graph {
    const float *vectors;        /* (n, dim) float32, row-major, rows contiguous */
    const uint8_t *codes;        /* (n, dim) uint8 scalar-quantizer codes, or NULL */
    const int32_t *links0;       /* (n, links0_stride) int32; first count0[i] valid */
    const int32_t *count0;       /* (n,) int32 */
    const int64_t *upper_offset; /* (n,) int64; first links_up row of a node, -1 if level 0 */
    const int32_t *links_up;     /* (rows, links_up_stride) int32 */
    const int32_t *count_up;     /* (rows,) int32 */
    int64_t n;                   /* nodes */
    int64_t rows;                /* upper-layer rows */
    int32_t dim;
    int32_t links0_stride;       /* 2M + 1 */
    int32_t links_up_stride;     /* M + 1 */
    int32_t metric;              /* HNSW_B200_L2 / _IP / _COSINE */
    int64_t entry_point;
    int32_t max_level;
    int32_t reserved;
    const uint8_t *vector_bytes; /* (n, dim) uint8 copy of integer-valued vectors in [0, 255] (the
                                    same values, one byte each), or NULL; enables the byte mode */
    const int32_t *node_ids;     /* NULL: the arrays are in the reference's node order. Otherwise
                                    the arrays are stored in an internal node order chosen for
                                    memory locality: row i of every per-node array belongs to the
                                    node whose original id is node_ids[i], link entries and
                                    entry_point are internal ids, and the allowed bitmap is indexed
                                    by internal id. Results are original ids, and equal distances
                                    order by original id, so results equal the reference's. */
} hnsw_b200_graph_t;

/* Distance arithmetic of one search call. */
#define HNSW_B200_DIST_F64 0      /* float64, strictly sequential over dimensions: bit-identical to
                                     the reference's _distance for any data */
#define HNSW_B200_DIST_EXACT_F32 1 /* float32 with warp-parallel sums; the caller asserts that data
                                     and queries are integer-valued with every partial sum below
                                     2^24, so the result is the same exact integer */
#define HNSW_B200_DIST_BYTES 2     /* integer dot products of uint8 rows (graph->codes with use_codes,
                                     else graph->vector_bytes) and uint8 queries (__dp4a): exact; the
                                     caller asserts the queries are integers in [0, 255] and dim is a
                                     multiple of 4 */

typedef struct hnsw_b200_search_args {
    const void *queries;          /* (nq, dim): float32, or float64 if queries_f64 */
    int32_t queries_f64;          /* 1: float64 code-space queries (transform_queries output) */
    int32_t use_codes;            /* 1: distances to graph->codes instead of graph->vectors */
    int64_t nq;
    int32_t k;                    /* results returned per query */
    int32_t k_search;             /* results collected by the beam (>= k; = fetch when reranking) */
    const int32_t *ef;            /* (nq,) efSearch per query; layer 0 uses max(ef[i], k_search) */
    int32_t ef_max;               /* max over ef[] (sizes shared memory) */
    int32_t dist_mode;            /* HNSW_B200_DIST_* */
    const uint32_t *allowed;      /* filter bitmap, bit i of word i/32 = node i allowed; NULL = none */
    float allowed_fraction;       /* share of allowed nodes (sizes scratch); 1 when unfiltered */
    const float *rerank_queries;  /* (nq, dim) float32 prepared queries: when non-NULL the first
                                     k_search beam entries are re-scored exactly against
                                     graph->vectors in float64 and the best k returned */
    int64_t *out_ids;             /* (nq, k) int64, -1 padded */
    double *out_dists;            /* (nq, k) float64, +inf padded */
    int64_t *out_counters;        /* (nq, 2) int64 distance computations, hops; or NULL */
    /* Learned early termination (unfiltered layer 0 only). Every HNSW_B200_STOP_EVERY layer-0
     * expansions the kernel computes HNSW_B200_STOP_FEATURES search-progress features; with a
     * network it stops the query once the prediction falls below stop_threshold. */
    const void *stop_mlp;         /* packed network (hnsw_b200_mlp_pack layout), or NULL */
    float stop_threshold;
    int32_t trace_cap;            /* checkpoints per query in the trace buffers */
    float *trace_feat;            /* (nq, trace_cap, HNSW_B200_STOP_FEATURES) features, or NULL */
    double *trace_dk;             /* (nq, trace_cap, 16) first 16 results' distances at each
                                     checkpoint (+inf beyond the results held) */
    int32_t *trace_count;         /* (nq,) checkpoints recorded */
    int32_t *trace_hops;          /* (nq,) layer-0 expansions of the whole search */
    /* The stop threshold rises by stop_slope per 64 layer-0 expansions beyond stop_slope_from
     * (0 and any: a constant threshold). */
    float stop_slope;
    int32_t stop_slope_from;
    /* Start order: (nq,) int32 device array, or NULL for row order. Queries start in descending
     * priority, equal priorities in row order (a stable sort on the low 16 bits, so values belong
     * in [0, 65535]). Results do not depend on the order -- each query's search is independent --
     * but the batch ends sooner when its longest queries start first. */
    const int32_t *priority;
    /* Per-cell cost learning: with cells ((nq,) device, each query's cell in [0, n_cells), as
     * hnsw_b200_start_priority gives it) every finished query adds its expansions per unit of
     * efSearch, and 1, to cell_cost ((4, n_cells) float64 device: plain sums, stopped sums,
     * plain counts, stopped counts; "stopped" = searched with stop_mlp). NULL: no learning. */
    const int32_t *cells;
    double *cell_cost;
    int32_t n_cells;
    /* Kernel configuration, 0 .. hnsw_b200_kernel_configs(dist_mode) - 1 (0: the default). Every
     * configuration returns the same results; they differ in speed (the autotuner's choices). */
    int32_t kernel_config;
} hnsw_b200_search_args_t;

#define HNSW_B200_STOP_EVERY 16
#define HNSW_B200_STOP_FEATURES 12
#define HNSW_B200_STOP_HIDDEN 64

/* Element types of hnsw_b200_exact_knn inputs. */
#define HNSW_B200_F32 0
#define HNSW_B200_U8 1

typedef struct hnsw_b200_exact_args {
    const void *data;              /* (n, dim) rows, dtype below, device memory */
    const void *queries;           /* (nq, dim) rows, same dtype */
    int32_t dtype;                 /* HNSW_B200_F32 or HNSW_B200_U8 */
    int32_t dim;
    int64_t n;
    int64_t nq;
    int32_t k;                     /* 1 <= k <= n */
    int32_t metric;                /* HNSW_B200_L2 / _IP / _COSINE */
    int32_t integer_valued;        /* 1: every data and query value is an integer with |v| <= 256
                                      (exact in BF16: one tensor-core term instead of three); 0: not
                                      known to be; -1: the library checks on the device. Float rows
                                      are checked on the device for bytes unless this is 0 */
    int32_t reserved;
    int64_t *out_ids;              /* (nq, k) int64, ascending (distance, id) */
    double *out_dists;             /* (nq, k) float64 exact distances */
    double *out_filter_max_error;  /* host: largest |filter value - float64 distance| measured over
                                      every re-scored candidate of the call, or NULL (byte rows:
                                      only candidates whose float value is 2^24 or more are
                                      re-scored, and one result in 16 of each query is checked in
                                      float64) */
    int64_t *out_candidates;       /* host: candidates re-scored in float64, or NULL */
    int64_t *out_launches;         /* host: kernel launches made, or NULL */
    double *out_filter_error_bound; /* host: largest derived bound e_q of the filter's error (the
                                      margin is 2 e_q), or NULL; the measured error never exceeds it */
} hnsw_b200_exact_args_t;

/* Exact k nearest neighbours by brute force on the tensor cores, ties to the lower id. Byte rows
 * (u8, or float rows whose every value is an integer in [0, 255]; L2 or inner product; dim <= 8192)
 * take an integer filter (tcgen05 kind::i8, S32 accumulation) whose values are the exact
 * distances, so no margin is needed and only float copies of 2^24 or more are re-scored; a float64
 * re-score of one result in 16 of each query that differs from it fails the call
 * (HNSW_B200_ECUDA). Other rows
 * take a BF16 filter with FP32 accumulation and a derived error margin, then a float64 re-rank of
 * the survivors. Replaces oracle.exact_search (src/hnsw_engine/oracle.py:35-126). Synchronises
 * `stream`. When more rows fall within a query's margin than its candidate list holds (many exact
 * ties at the k-th distance), the call re-runs with longer lists (fewer queries per chunk) instead
 * of failing. */
int hnsw_b200_exact_knn(const hnsw_b200_exact_args_t *args, void *stream);

/* ---- Early-termination network (no reference counterpart): 12 -> 64 -> 64 -> 1, ReLU.
 * Master parameters are float32 in the order W1[64][12], b1[64], W2[64][64], b2[64], W3[64], b3;
 * forward passes use BF16-rounded weights with FP32 accumulation, as the in-search inference. */
int64_t hnsw_b200_mlp_param_count(void);
int64_t hnsw_b200_mlp_packed_bytes(void);
int64_t hnsw_b200_mlp_scratch_bytes(int32_t batch);
/* One Adam step (step counts from 1) on a batch of (features, target) pairs; loss receives the
 * batch mean squared error (device float). scratch: hnsw_b200_mlp_scratch_bytes(batch) bytes. */
int hnsw_b200_mlp_train_step(float *params, float *adam_m, float *adam_v, int64_t step, float lr,
                             const float *features, const float *targets, int32_t batch,
                             float *scratch, float *loss, void *stream);
/* Gradients of the batch mean squared error with respect to the parameters (no update). */
int hnsw_b200_mlp_gradients(const float *params, const float *features, const float *targets,
                            int32_t batch, float *scratch, float *grads, float *loss, void *stream);
int hnsw_b200_mlp_predict(const float *params, const float *features, int64_t n, float *out,
                          void *stream);
/* Pack master parameters and the feature standardisation (mean, 1/std: 12 floats each, device)
 * into the search kernel's layout (hnsw_b200_mlp_packed_bytes bytes). */
int hnsw_b200_mlp_pack(const float *params, const float *mean, const float *inv_std, void *packed,
                       void *stream);

/* Create a search handle over a graph whose arrays live on the current CUDA device. */
int hnsw_b200_open(const hnsw_b200_graph_t *graph, void **handle);

/* Release the handle and its scratch (never the caller's arrays). */
void hnsw_b200_close(void *handle);

/* Batched search of args->nq queries on `stream` (a cudaStream_t; NULL = legacy default stream).
 * Synchronises the stream once to read the overflow count, re-running overflowed queries with
 * larger scratch; results are complete when it returns 0. */
int hnsw_b200_search(void *handle, const hnsw_b200_search_args_t *args, void *stream);

/* The same search as hnsw_b200_search, issued with no host synchronisation, no allocation and
 * no host read, every launch on `stream`, so that it can be recorded in a CUDA graph and replayed
 * (the reference's search has no counterpart: it runs on the CPU). The handle's scratch must
 * already fit the arguments: a hnsw_b200_search call with arguments of the same size (queries,
 * ef_max, k, filter, rerank, kernel configuration) sizes it, else HNSW_B200_EINVAL. Queries that
 * overflow their scratch are left unwritten and counted on the device: read the count with
 * hnsw_b200_search_failed once the stream has run the search, and search them again with
 * hnsw_b200_search. */
int hnsw_b200_search_async(void *handle, const hnsw_b200_search_args_t *args, void *stream);
/* Queries the last hnsw_b200_search_async on this handle left unwritten; synchronises `stream`. */
int hnsw_b200_search_failed(void *handle, int32_t *failed, void *stream);

/* Batched search without any device allocation, for callers that are not allowed to allocate
 * GPU memory: real-time serving loops where an allocation would stall the loop, plugins whose host
 * owns every device allocation through its own pool, processes under a hard device-memory budget.
 * No counterpart in the reference (its search runs on the CPU). It runs the same unfiltered search
 * kernel as hnsw_b200_search, with all working memory taken from one fixed 32 MiB array inside the
 * library image, which every GPU that loads the library holds until the process exits.
 *   - limits: at most 1,048,576 queries per call; no filter (allowed must be NULL) and no start
 *     order (priority must be NULL; allowed_fraction is not read); the graph's per-warp visited
 *     bitmap (n / 8 bytes) must fit several times in the array, which bounds n at about 60 million
 *     nodes (larger graphs return HNSW_B200_EINVAL before any GPU work);
 *   - fewer queries run at once than in hnsw_b200_search: as many warp slots as fit in the array
 *     (each holds an n / 8-byte bitmap, a list of marked ids, a 4 KB hash and a tie stack), e.g.
 *     about 228 slots (57 blocks) at 1M nodes against 740 blocks for hnsw_b200_search on a B200;
 *   - a query that outgrows its share (the upper-layer visited hash) is left unwritten and the
 *     call returns HNSW_B200_ERETRY; the other queries' outputs are complete (search the failed
 *     ones with hnsw_b200_search);
 *   - each call looks up the array's device address on the current device (no cached pointer);
 *   - every call uses the same array and leaves its contents behind (the counters and bitmaps are
 *     cleared at the start of each call): calls that overlap on the GPU -- on two streams, or two
 *     host threads -- race and must not be issued;
 *   - it waits for `stream` once, to read the overflow count into host memory, before returning. */
int hnsw_b200_search_noalloc(const hnsw_b200_graph_t *graph, const hnsw_b200_search_args_t *args,
                             void *stream);

/* Kernel configurations of the search for a distance mode (no reference counterpart: the
 * autotuner's choices). The byte kernels have four: the layer-0 visited set as a per-slot bitmap or
 * an open-addressing hash, gathered rows held in registers or staged in shared memory by cp.async,
 * and 5 or 4 resident blocks per SM (the register cap); the other modes have one. The name is a
 * static string ("" for an index out of range). */
int32_t hnsw_b200_kernel_configs(int32_t dist_mode);
const char *hnsw_b200_kernel_config_name(int32_t dist_mode, int32_t config);

/* Number of device kernel launches made by the last hnsw_b200_search on this handle. */
int64_t hnsw_b200_last_launches(void *handle);

/* Thread-local text of the last error. */
const char *hnsw_b200_last_error(void);

/* Validation of a graph's uploaded arrays on the GPU: the checks of the reference's
 * _validate_native (numba_engine.py:878-915) -- node levels, entry point on the top layer, link
 * counts within capacity, link targets inside the graph, upper-layer rows tiling [0, rows),
 * upper-layer links landing on nodes present on that layer. levels: (n,) int64 device array.
 * scratch: device memory of hnsw_b200_validate_scratch_bytes(graph->rows) bytes. flags_out (host)
 * receives the failed checks as HNSW_B200_BAD_* bits; 0 means valid. The bits are numbered in the
 * order the host validator checks, so the lowest set bit names the error it would raise.
 * Synchronises the stream. */
#define HNSW_B200_BAD_LEVEL 1u      /* a negative node level */
#define HNSW_B200_BAD_ENTRY 2u      /* the entry point (or max_level) is not the top layer's */
#define HNSW_B200_BAD_COUNT0 4u     /* a layer-0 link count outside [0, 2M] */
#define HNSW_B200_BAD_LINK0 8u      /* a layer-0 link outside the graph */
#define HNSW_B200_BAD_ROWS 16u      /* upper-layer rows overlap or leave gaps */
#define HNSW_B200_BAD_COUNT_UP 32u  /* an upper-layer link count outside [0, M] */
#define HNSW_B200_BAD_LINK_UP 64u   /* an upper-layer link outside the graph */
#define HNSW_B200_BAD_LAYER 128u    /* an upper-layer link to a node absent from that layer */
int64_t hnsw_b200_validate_scratch_bytes(int64_t rows);

/* Scalar quantizer on the GPU (ScalarQuantizer.fit / encode, quantization.py:37-59).
 * hnsw_b200_quant_stats: per-dimension minima lo and maxima hi (float64, device, dim each) of
 * float32 rows, and *integer_valued (host) = 1 if every value is an integer; scratch: device
 * memory of hnsw_b200_quant_scratch_bytes(dim) bytes; synchronises the stream. The caller derives
 * offset = lo and the step exactly as fit does.
 * hnsw_b200_quant_encode: codes[i][j] = clip(rint((double(x[i][j]) - offset[j]) / step), 0, 255),
 * float64 arithmetic as the reference's encode (codes bit for bit equal). */
int64_t hnsw_b200_quant_scratch_bytes(int32_t dim);
int hnsw_b200_quant_stats(const float *vectors, int64_t n, int32_t dim, double *lo, double *hi,
                          int32_t *integer_valued, void *scratch, void *stream);
int hnsw_b200_quant_encode(const float *vectors, int64_t n, int32_t dim, const double *offset,
                           double step, uint8_t *codes, void *stream);
int hnsw_b200_validate_graph(const hnsw_b200_graph_t *graph, const int64_t *levels, int32_t M,
                             void *scratch, uint32_t *flags_out, void *stream);

/* Upload of a float32 query batch to device dst on `stream` (NULL dst: no copy, no GPU work), and
 * in *out whether every value is finite and an integer, with their minimum and maximum, from a
 * read of src on up to `threads` host threads. Replaces, for contiguous float32 batches, the host
 * validator's NaN/inf pass (_validation.py:30-35) and the float32 cast of metrics.py:49-53 (a copy
 * for float32 rows); the statistics select the distance arithmetic without reading the queries
 * back from the GPU. min and max are meaningful only when finite is 1.
 *   - staging NULL: a pageable cudaMemcpyAsync from src, concurrent with the read;
 *   - staging: page-locked host memory of `count` floats, 16-byte aligned, not in use by an
 *     earlier copy; the threads copy src into it as they read (streaming stores) and one
 *     asynchronous DMA follows. The caller keeps it untouched until the copy completes in stream
 *     order.
 * src may be reused on return; dst is complete in stream order. */
typedef struct {
    int32_t finite;   /* 1 if no value is NaN or +-inf */
    int32_t integer;  /* 1 if every value is an integer */
    double min, max;  /* over all values (0 for count == 0) */
} hnsw_b200_value_stats_t;
int hnsw_b200_upload_queries(const float *src, float *dst, int64_t count, int32_t threads,
                             hnsw_b200_value_stats_t *out, float *staging, void *stream);

/* Start priorities for hnsw_b200_search (one launch): each query's cell -- its nearest of the
 * n_cells float32 pivot rows (squared L2 in float32, ties to the lower index) -- into cells, and
 * min(65535, ratio * ef[q] * scale) into priority, where ratio is the cell's expansions per unit
 * of efSearch from cell_cost (the table hnsw_b200_search learns: the plain searches' mean where
 * plain counts are nonzero, else the stopped searches'). queries: (nq, dim) float32 device. */
int hnsw_b200_start_priority(const float *queries, int64_t nq, int32_t dim, const float *pivots,
                             int32_t n_cells, const double *cell_cost, const int32_t *ef,
                             float scale, int32_t *cells, int32_t *priority, void *stream);

/* Library version string. */
const char *hnsw_b200_version(void);

#ifdef __cplusplus
}
#endif

#endif /* HNSW_B200_H */
