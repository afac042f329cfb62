/*
 * hy.h — C-ABI of the B200 IVF engine (libhy.so).
 *
 * This is the drop-in boundary for Harmony's IVF query path.  Every entry
 * point takes plain pointers and sizes (no C++ or framework types), returns an
 * int status (HY_OK on success) and records a message for hy_last_error().
 * The C++ facade in include/harmony/Index.h wraps these calls back into
 * Harmony's `harmony::Index` class.  Reference paths below are relative to the
 * Harmony repository.
 *
 * Threading: one handle is used by one host thread at a time; calls on a
 * handle are serialised (the reference's Index is likewise not reentrant:
 * search mutates its listidqueries member, src/Index.cpp:969).
 *
 * Memory: host-pointer calls copy inputs to the GPU and results back before
 * returning.  *_device calls take device pointers and a cudaStream_t (passed
 * as void*; NULL is the CUDA default stream) and return once the work is
 * enqueued on that stream.
 */
#ifndef HY_H
#define HY_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HY_API __attribute__((visibility("default")))

typedef struct hy_index hy_index;

/* Status codes.  The reference reports errors by C++ exceptions and exit(1)
 * (src/Index.cpp:60,464,1644,1737; src/node.cpp:129-134); the facade maps
 * these codes back to std::runtime_error. */
enum {
    HY_OK = 0,
    HY_ERR_ARG = 1,         /* invalid argument or unsupported size */
    HY_ERR_OOM = 2,         /* device or host allocation failed */
    HY_ERR_CUDA = 3,        /* CUDA runtime error, or no usable GPU */
    HY_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up */
    HY_ERR_STATE = 5,       /* call out of order (e.g. search before add) */
    HY_ERR_IO = 6,          /* file could not be read or written */
    HY_ERR_UNSUPPORTED = 7  /* feature not built for this configuration */
};

/* Metric, same values as harmony::MetricType (src/common.h:20-21). */
enum { HY_METRIC_IP = 0, HY_METRIC_L2 = 1 };

/* Scan forms selectable with hy_index_set_form. */
enum {
    HY_FORM_PLAIN = 0, /* exact FP32 query-major scan with dim-block pruning */
    HY_FORM_BF16 = 1,  /* batched list-major bf16 tensor-core scan + exact FP32 re-rank */
    HY_FORM_FP8 = 2    /* the same on e4m3 codes with per-list / per-query scales, oversampled re-rank */
};

/* How the plain form scans (hy_index_set_plain_scan).  Both return the same
 * answer, bit for bit. */
enum {
    HY_PLAIN_AUTO = 0,        /* list-major when the batch shares lists (>= 4 queries per list on average) */
    HY_PLAIN_QUERY_MAJOR = 1, /* one CTA per (query, probe split) streams that query's probed lists */
    HY_PLAIN_LIST_MAJOR = 2   /* queries probing a list share one pass over it, 32 per group */
};

/* Largest k the scan kernels keep per query. The reference's distributed
 * modes assume k <= 100 (presumeK, src/node.h:89). */
#define HY_MAX_K 256
/* Largest number of dimension blocks. */
#define HY_MAX_DIM_BLOCKS 8

typedef struct {
    size_t d;           /* vector dimension */
    size_t nlist;       /* number of inverted lists */
    size_t nprobe;      /* lists probed per query */
    int metric;         /* HY_METRIC_* */
    int opt_level;      /* harmony::OptLevel accepted at creation */
    size_t dim_blocks;  /* dimension blocks used for partial-distance pruning */
    size_t ntotal;      /* vectors currently held in the lists */
    size_t arena_rows;  /* rows in the device arena, padding included */
    int trained;        /* centroids are set */
    int device;         /* CUDA device ordinal */
    int form;           /* HY_FORM_* */
    int learned;        /* the probe network picks each query's nprobe */
    size_t capq;        /* bf16 form: candidate slots per query */
    size_t row_slice;   /* bf16 form: rows per work item */
} hy_index_info_t;

/* Counters of the last search on a handle (the reference returns a Stats
 * object from Index::search, src/Index.h:82; its pruning counters are
 * src/stats.h). */
typedef struct {
    uint64_t nq;              /* queries searched */
    uint64_t pairs;           /* (query, probed list) pairs scanned */
    uint64_t rows;            /* (query, row) pairs in the probed lists */
    uint64_t tile_blocks;     /* 32-row x one-dim-block tiles loaded */
    uint64_t tile_blocks_max; /* tiles that a scan without pruning would load */
    double coarse_ms;         /* device time of coarse quantisation */
    double scan_ms;           /* device time of the list scan */
    double merge_ms;          /* device time of the top-k merge */
    uint64_t launches;        /* kernels this library launched for the call */
    uint64_t fallback_queries; /* bf16 / e4m3 forms: queries whose candidates overflowed, every one
                                  answered again exactly by the plain scan on the device */
    double mean_nprobe;       /* lists probed per query (learned: the predicted mean) */
    double judge_recall;      /* learned: recall@10 of the judged sample vs fixed nprobe (-1: not judged) */
    uint64_t learned_fallback; /* learned: 1 when the batch was searched again with fixed nprobe */
    double kernel_ms;         /* device time of the scan kernel's launches (plain: scan_plain_kernel;
                                 bf16: batched_scan_kernel, both passes) in the last query chunk */
    uint64_t kernel_launches; /* launches kernel_ms covers */
    uint64_t graph_replayed;  /* device-pointer search in graph mode: 1 when the call replayed a graph */
    uint64_t seg_sums;        /* list-major plain scan: (query, 32-row tile, 16-dimension segment) partial
                                 sums computed: 32 x 16 x 3 FP32 operations each; like kernel_ms, and
                                 with the tile counts, they cover the last query chunk */
    uint64_t seg_sums_max;    /* list-major plain scan: the segment sums a scan without pruning computes */
    uint64_t list_major;      /* plain form: 1 when the search ran the list-major scan */
    uint64_t chunk_queries;   /* device search: queries of its last query chunk, the chunk whose launches
                                 kernel_ms and the scan counters cover */
} hy_search_stats_t;

HY_API const char* hy_last_error(void);
HY_API const char* hy_version(void);

/* Index lifecycle.  Replaces harmony::Index::Index(d, nlist, nprobe, metric,
 * opt_level, ...) (src/Index.h:15-25, src/Index.cpp:24-43).  opt_level is
 * the reference's OptLevel (see hy_index_set_opt_level; callers also pass
 * OPT_ALL through sub_k, src/query.cpp:460, which is accepted).  dim_blocks is
 * the number of dimension blocks the partial-distance prune checks between
 * (the reference hard-codes 4, src/node.cpp:639); 0 selects 4. */
HY_API int hy_index_create(size_t d, size_t nlist, size_t nprobe, int metric, int opt_level, size_t dim_blocks,
                           int device, hy_index** out);
HY_API int hy_index_destroy(hy_index* h);
HY_API int hy_index_info(const hy_index* h, hy_index_info_t* out);

/* k-means training.  Replaces Index::train (src/Index.cpp:381-425): 20 Lloyd
 * iterations (2 with lite), seed 6666, at most 256 sample rows per centroid;
 * centroid sums are accumulated in FP64 on the GPU. */
HY_API int hy_index_train(hy_index* h, size_t n, const float* x, int lite);
HY_API int hy_index_train_device(hy_index* h, size_t n, const float* dx, int lite, void* stream);

/* Centroids, the public centroid_codes field of the reference (src/Index.h:118):
 * nlist x d float32, row-major, host memory. */
HY_API int hy_index_set_centroids(hy_index* h, const float* centroids);
HY_API int hy_index_get_centroids(const hy_index* h, float* centroids);

/* Build the inverted lists.  Replaces Index::add (src/Index.cpp:581-697):
 * lists are rebuilt from scratch on every call; row i of x gets id i; rows
 * are ordered within a list by distance to the centroid. */
HY_API int hy_index_add(hy_index* h, size_t n, const float* x);
HY_API int hy_index_add_device(hy_index* h, size_t n, const float* dx, void* stream);

HY_API int hy_index_set_nprobe(hy_index* h, size_t nprobe);

/* The public opt_level field (src/Index.h:108; callers set it between
 * searches, src/main.cpp:61-70).  OPT_TRIANGLE with the inner-product
 * metric scans, per (query, probed list), only the rows whose inner product
 * with the list's centroid lies in the reference's cos-bound window
 * (src/Index.cpp:1509-1546), built from the query's k-th similarity so far;
 * for unit-norm rows and queries the skipped rows cannot reach the top-k, so
 * the answer is the exact scan's, as in the reference.  The list-major scan
 * applies the window; the query-major scan scans every row.  With L2,
 * OPT_TRIANGLE makes the list-major scan skip the rows whose distance to
 * their centroid differs from the query's by more than the square root of
 * its threshold (|q - x| >= | |q - c| - |x - c| |, an exact prune with margins
 * for FP32 rounding): the answer is unchanged, as in the reference, whose L2
 * triangle code is commented out (src/Index.cpp:1468-1492).  The sub-NN
 * levels change nothing in the reference's search (src/IVFScan.hpp:223-427)
 * and nothing here. */
HY_API int hy_index_set_opt_level(hy_index* h, int opt_level);

/* Scan form (no counterpart in the reference, whose only scan is the exact
 * FP32 one): HY_FORM_PLAIN or HY_FORM_BF16 (d <= 128).  The bf16 form batches
 * queries per list on the tensor cores and re-ranks candidates with exact FP32
 * distances chosen by rigorous error bounds, so its results equal the plain
 * form's.  Queries whose candidates overflow their buffers are answered again
 * by the plain scan on the device, however many overflow. */
HY_API int hy_index_set_form(hy_index* h, int form);

/* Plain form's scan (no counterpart in the reference): HY_PLAIN_AUTO (default),
 * HY_PLAIN_QUERY_MAJOR or HY_PLAIN_LIST_MAJOR.  The list-major scan inverts
 * the (query, probed list) pairs into per-list groups of 32 queries; each
 * group reads a list once, dimension block by dimension block, pruning each
 * (row, query) pair against the query's threshold between blocks, with the
 * query-major scan's arithmetic.  Its two passes (each query's nearest list
 * under the warm-up threshold, then the other probed lists under the k-th
 * distance found so far) keep up to the bf16 form's candidate slots per
 * query; a query with more is answered again by the query-major scan. */
HY_API int hy_index_set_plain_scan(hy_index* h, int mode);

/* bf16 form parameters (0 keeps the current value): candidate slots per
 * query (default 8192, at most 12288; the first pass scans each query's
 * nearest list densely when it has at most this many rows), re-rank
 * oversampling factor (e4m3 form: at most oversample x k candidates are
 * re-ranked) and rows per work item (default 2048, a multiple of 128, at most
 * 2048).  The bf16 form runs the warm-up (at most 3 lists) only for queries
 * whose nearest list is not scanned densely or has fewer than k rows. */
HY_API int hy_index_set_batch_params(hy_index* h, size_t capq, size_t oversample, size_t row_slice);

/* Queries per group of the tensor-core forms' two search passes: 32, 64 or
 * 128 (capped at what d allows), or 0 (default) to pick per pass 64 or 128,
 * the smaller when it holds four times the pass's expected queries per list
 * (fewer accumulator columns and a deeper copy ring for sparse passes; a list
 * probed by more queries than a group holds is read once per group).  The
 * results do not depend on it. */
HY_API int hy_index_set_group_size(hy_index* h, int qg);

/* Coarse quantiser of the bf16 form (no counterpart in the reference, which
 * scores every centroid exactly, src/Index.cpp:985-990).  HY_COARSE_EXACT:
 * exact FP32 scores of every centroid, then the nprobe best.
 * HY_COARSE_TENSOR (default): bf16 tensor-core scores of every centroid with
 * rigorous error bounds, then exact FP32 scores only for the centroids whose
 * bound can reach the nprobe-th best; the probe lists (and the learned
 * predictor's coarse scores) are identical to HY_COARSE_EXACT's.  Used when
 * nprobe <= 256 and d <= 256 (above 2048 lists in two tensor-core launches:
 * a bound from the first 1024 centroids, then a thresholded pass over all);
 * otherwise the exact path runs.
 * The plain and e4m3 forms always use the exact path. */
enum { HY_COARSE_EXACT = 0, HY_COARSE_TENSOR = 1 };
HY_API int hy_index_set_coarse(hy_index* h, int mode);

/* Warm-up threshold parameters.  Mirrors Index::preSearch's warmUpSearchList /
 * warmUpSearchListSize (src/Index.h:90, src/Index.cpp:45-55): when
 * warmup_list > 0, each query's pruning threshold starts at the k-th best
 * distance among the first warmup_list_size rows of its first warmup_list
 * probed lists (src/Index.cpp:999-1051).  warmup_list_size 0 means k. */
HY_API int hy_index_presearch(hy_index* h, size_t warmup_list, size_t warmup_list_size);

/* Search.  Replaces Index::search (src/Index.cpp:1638-1706): D and I are n x k
 * row-major; each row is sorted best first (ascending L2, descending IP);
 * unfilled entries hold FLT_MAX (L2) / -FLT_MAX (IP) and id -1
 * (src/heap.hpp:13-25). */
HY_API int hy_index_search(hy_index* h, size_t n, const float* q, size_t k, float* D, int64_t* I);
HY_API int hy_index_search_device(hy_index* h, size_t n, const float* dq, size_t k, float* dD, int64_t* dI,
                                  void* stream);

/* Autotuner of the bf16 form (no counterpart in the reference): times the
 * search of n sample queries (host pointer) at k for every candidate work
 * shape (rows per work item 512 / 1024 / 2048 x candidate slots per query
 * 8192 / 12288; reps timed searches each, after one untimed) and keeps the
 * fastest whose results equal the first shape's.  report (may be NULL)
 * receives 6 x {row_slice, capq, ms} (ms negated for a shape whose results
 * differed). */
HY_API int hy_index_autotune(hy_index* h, size_t n, const float* q, size_t k, int reps, float* report);

/* List partition across GPUs (the reference's vector partition across
 * teams, src/Index.cpp:288-325, as one index per GPU): after
 * hy_index_set_list_range(h, lo, hi), add() keeps only the rows of lists
 * [lo, hi) (the other lists stay empty, ids stay the row indices of the whole
 * base), so every search scans only this GPU's share of each query's probed
 * lists.  The per-GPU top-k lists, gathered into one [parts][n][k] device
 * array (one all-gather), are merged by hy_merge_topk into the top-k of the
 * whole index; with contiguous ranges in GPU order the merged answer equals
 * the unpartitioned index's, ties included. */
HY_API int hy_index_set_list_range(hy_index* h, size_t lo, size_t hi);
HY_API int hy_merge_topk(const float* dD, const int64_t* dI, size_t parts, size_t n, size_t k, int metric,
                         float* dDout, int64_t* dIout, void* stream);

/* Graph mode for the device-pointer searches (no counterpart in the
 * reference): the first call with given buffers, sizes, stream and index
 * state runs normally and captures its launch sequence (coarse quantisation,
 * probe network, warm-up, the persistent batched scan, re-rank, fallback) in
 * a CUDA graph; identical later calls replay it with one launch.  Any call
 * that changes the index or its parameters retires the graph. */
HY_API int hy_index_set_graph(hy_index* h, int enabled);

/* Search with a per-query nprobe (no counterpart in the reference, whose
 * nprobe is one value per call): query i probes its nprobes[i] nearest lists
 * (clamped to nlist).  The device variant takes the per-query values on the
 * device and their maximum from the caller. */
HY_API int hy_index_search_nprobes(hy_index* h, size_t n, const float* q, size_t k, const int32_t* nprobes, float* D,
                                   int64_t* I);
HY_API int hy_index_search_nprobes_device(hy_index* h, size_t n, const float* dq, size_t k, const int32_t* dnprobes,
                                          size_t max_nprobe, float* dD, int64_t* dI, void* stream);

/* Search with caller-given probe lists (n x nprobe list ids, best first; -1
 * entries are skipped).  This is the list-scan half of the search
 * (src/Index.cpp:1450-1547) fed with the master's listidqueries
 * (src/Index.cpp:969-995). */
HY_API int hy_index_search_preassigned(hy_index* h, size_t n, const float* q, size_t k, size_t nprobe,
                                       const int64_t* probes, float* D, int64_t* I);

/* Coarse quantisation only: the nprobe nearest lists of each query, best
 * first (Index::findNearNprobeOfCentroidIds, src/Index.cpp:899-998).  With
 * the learned predictor on, the lists beyond each query's predicted nprobe
 * are -1, exactly as the search uses them. */
HY_API int hy_index_probes(hy_index* h, size_t n, const float* q, int64_t* probes);

/* Warm-up thresholds only (src/Index.cpp:999-1051 and 1300-1303): for each
 * query the k-th best full-d L2 distance over the first warmup_list_size rows
 * of its first warmup_list probed lists, FLT_MAX when fewer than k rows. */
HY_API int hy_index_warmup_tops(hy_index* h, size_t n, const float* q, size_t k, size_t nprobe,
                                const int64_t* probes, size_t warmup_list, size_t warmup_list_size, float* tops);

HY_API int hy_index_last_stats(const hy_index* h, hy_search_stats_t* out);

/* Inverted-list access (src/IVF.h:51-58): size, then ids / row-major codes /
 * squared norms of one list (any output pointer may be NULL). */
HY_API int hy_index_list_size(const hy_index* h, size_t list, size_t* size);
HY_API int hy_index_get_list(const hy_index* h, size_t list, int64_t* ids, float* codes, float* norms);

/* Persistence in the reference's binary .index format (Index::save_index /
 * load_index, src/Index.cpp:1708-1770; IVF::save_IVF / load_IVF,
 * src/IVF.cpp:76-134). */
HY_API int hy_index_save(const hy_index* h, const char* path);
HY_API int hy_index_load(hy_index* h, const char* path);

/* Reads the header and list table of a .index file without a GPU. */
HY_API int hy_file_inspect(const char* path, size_t* d, size_t* nlist, int* metric, int* opt_level,
                           size_t* nonempty_lists, size_t* ntotal);

/* Search with caller-given probe lists that allocates no device memory (no
 * counterpart in the reference).  For callers that cannot call cudaMalloc
 * while serving — their device memory belongs to another allocator (a
 * framework's caching pool, an arena reserved at start-up), and cudaMalloc can
 * synchronise the device or fail under memory pressure mid-serving.  dq
 * (n x d float32), dprobes (n x nprobe list ids, -1 = skip), dD (n x k) and dI
 * (n x k) are device pointers the caller owns; all temporaries live in a fixed
 * 8 MiB __device__ array inside libhy.so, so a call needs
 * n*nprobe*8 + n*nsplit*K'*8 bytes to fit (K' = k rounded up to 32/64/128/256,
 * nsplit = 1 for n >= 296 queries) and larger batches are rejected with
 * HY_ERR_ARG.  Results equal hy_index_search_preassigned's.  The call enqueues
 * on `stream` and waits for it; its first call on a device looks up the
 * array's device address, so make that call before any stream capture.  The
 * array is shared by every call on a device: calls whose GPU work overlaps
 * race and must be serialised by the caller.  The call holds the index's lock
 * until its work has completed, like the other entry points, so an add, load
 * or reset of the same index from another thread waits for it. */
HY_API int hy_index_search_preassigned_noalloc(hy_index* h, size_t n, const float* dq, size_t k, size_t nprobe,
                                               const int64_t* dprobes, float* dD, int64_t* dI, void* stream);

/* Learned probe predictor (no counterpart in the reference, whose nprobe is
 * fixed per call).  A small MLP (64 -> 256 -> 256 -> 1, GELU, bf16 matrix
 * products with f32 accumulation) reads a query's sorted coarse distances to
 * its 64 nearest lists and predicts how many lists it needs.
 * hy_index_train_probe_model labels n training queries with the exact scan at
 * max_nprobe (stop label = the smallest nprobe whose lists hold the exact
 * top-k_label), trains the network on the GPU with Adam (epochs, lr) and sets
 * a margin so that a `coverage` fraction of held-out queries gets at least
 * its stop label.  report (may be NULL) receives {final training loss,
 * held-out coverage, held-out mean predicted nprobe, held-out mean stop
 * label}.  With hy_index_set_learned(h, 1, judge_fraction, judge_recall) every
 * search predicts a per-query nprobe (at most the index's nprobe); the host
 * search also searches every (1/judge_fraction)-th query again with the fixed
 * nprobe, and if the learned results' recall@10 on that sample is below
 * judge_recall the batch is searched again with the fixed nprobe.  The model
 * is hy_probe_model_size() floats (weights, feature mean and scale, margin,
 * max nprobe). */
HY_API int hy_index_train_probe_model(hy_index* h, size_t n, const float* q, size_t max_nprobe, size_t k_label,
                                      int epochs, float lr, float coverage, float* report);
HY_API int hy_index_set_learned(hy_index* h, int enabled, float judge_fraction, float judge_recall);
HY_API size_t hy_probe_model_size(void);
HY_API int hy_index_get_probe_model(const hy_index* h, float* model);
HY_API int hy_index_set_probe_model(hy_index* h, const float* model);

/* Loss and gradients of the probe network on one batch (host pointers:
 * params hy_probe_model_size()-2*64-2 floats, X B x 64, targets B; grads like
 * params) for checking the training kernels against a reference.  No
 * counterpart in the reference. */
HY_API int hy_mlp_loss_grad(const float* params, int B, const float* X, const float* t, float* loss, float* grads);

/* Diagnostic with no counterpart in the reference: multiplies one 128 x 128
 * bf16 tile pair on the tensor cores exactly as the batched scan does
 * (D = A * B^T, A and B row-major 128 x 128 float32 rounded to bf16, D
 * float32).  Returns HY_OK or an error status. */
HY_API int hy_selftest_tcgen05(const float* A, const float* B, float* D);
/* The same on e4m3 operands: A and B are 128 x 256 (values rounded to e4m3
 * with saturation), D = A B^T is 128 x 128, accumulated by kind::f8f6f4. */
HY_API int hy_selftest_tcgen05_e4m3(const float* A, const float* B, float* D);

#ifdef __cplusplus
}
#endif

#endif /* HY_H */
