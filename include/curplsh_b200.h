/*
 * curplsh_b200.h -- C ABI of the B200-native exact L2 kNN engine.
 *
 * Plain pointers and sizes only (no C++ or framework types), status-code
 * errors.  Every entry point says which cuRPLSH interface it replaces
 * (paths are relative to the cuRPLSH source tree).  The C++ drop-in headers
 * under include/curplsh/ (Index, IndexBF, DeviceResources, tensors) are thin
 * inline wrappers over these functions, and the Python package
 * curplsh_b200 binds them with ctypes.
 *
 * Pointer arguments named "data", "queries", "indices", "distances" may be
 * host or device memory (detected with cudaPointerGetAttributes), as in the
 * reference (include/device_tensor.h:173-185, src/index_bf.cpp:56-73).
 *
 * Errors: every function returns CURPLSH_OK (0) or a CURPLSH_ERR_* code and
 * records a message for curplsh_last_error() (thread-local).  The reference
 * aborts or exits instead (include/internal/assertions.h:7-14,
 * include/internal/cuda_utils.h:991-1001).
 */
#ifndef CURPLSH_B200_H_
#define CURPLSH_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define CURPLSH_OK 0
#define CURPLSH_ERR_INVALID_ARG 1 /* bad argument (null, k out of range, dim mismatch) */
#define CURPLSH_ERR_CUDA 2        /* a CUDA runtime call failed */
#define CURPLSH_ERR_OOM 3         /* device or host allocation failed */
#define CURPLSH_ERR_UNSUPPORTED 4 /* valid request this build does not implement */
#define CURPLSH_ERR_DEVICE 5      /* a kernel reported an internal failure (bounded wait expired, overflow) */
#define CURPLSH_ERR_STATE 6       /* call not valid in the object's current state */

/* ------------------------------------------------------------ enums */
/* MemorySpace (include/memory_space.h:12-17) */
#define CURPLSH_MEMORY_DEVICE 0
#define CURPLSH_MEMORY_UNIFIED 1

/* Precision form of the coarse tensor-core pass; every form ends with an exact
 * FP32 rerank, so returned distances are FP32 squared L2 in all forms. */
#define CURPLSH_PRECISION_FP32_EXACT 0  /* 3 x BF16 split products, k' = k + margin */
#define CURPLSH_PRECISION_BF16_RERANK 1 /* BF16 coarse, k' = rerank_factor * k */
#define CURPLSH_PRECISION_FP8_RERANK 2  /* FP8-E4M3 (per-vector FP32 scale), k' = rerank_factor * k */

/* ------------------------------------------------------------ opaque handles */
typedef struct curplsh_resources curplsh_resources; /* DeviceResources (include/device_resources.h:60-263) */
typedef struct curplsh_index curplsh_index;         /* Index / IndexBF (include/index.h:18-82, include/index_bf.h:21-46) */

/* IndexBFConfig (include/index_bf.h:8-19) including its IndexConfig base
 * (include/index.h:8-16), plus the engine's precision controls. */
typedef struct curplsh_bf_config {
  int32_t device;                  /* IndexConfig::device */
  int32_t memory_space;            /* IndexConfig::memorySpace (CURPLSH_MEMORY_*) */
  int32_t store_transposed;        /* IndexBFConfig::storeTransposed: accepted, layout is always the
                                      engine's K-major tiled copy (the reference leaves it a TODO) */
  int32_t compute_exact_distances; /* IndexBFConfig::computeExactDistances: IndexBF::search always
                                      returns exact squared distances (src/index_bf.cpp:68-69), so is this */
  int32_t precision;               /* CURPLSH_PRECISION_* default for search */
  int32_t rerank_factor;           /* k' = rerank_factor * k for the BF16/FP8 forms; 0 (default): BF16
                                      2k when the coarse-margin check verifies the search, else 4k;
                                      FP8 4k and at least 480 (E4M3's coarse error needs the margin) */
  int32_t borrow_device_data;      /* 1: add() of device memory keeps a reference to the caller's FP32
                                      rows (the reference's aliasing, include/device_tensor.h:97-103);
                                      0 (default): the index copies them */
} curplsh_bf_config;

/* Defaults: device 0, device memory, FP32-exact, rerank_factor 0 (the form's default), copy on add. */
void curplsh_bf_config_init(curplsh_bf_config* cfg);

const char* curplsh_last_error(void);
const char* curplsh_version(void);

/* getNumDevices (include/internal/cuda_utils.h:1230-1258) */
int curplsh_get_num_devices(int* out);

/* ------------------------------------------------------------ DeviceResources */
/* DeviceResources() (include/device_resources.h:62) */
int curplsh_resources_create(curplsh_resources** out);
/* ~DeviceResources (include/device_resources.h:72-108) */
int curplsh_resources_destroy(curplsh_resources* res);
/* initializeForDevice (include/device_resources.h:113-165) */
int curplsh_resources_initialize_for_device(curplsh_resources* res, int device);
/* getDefaultStream (include/device_resources.h:181-184) */
int curplsh_resources_get_default_stream(curplsh_resources* res, int device, void** stream);
/* user default stream (include/device_resources.h:247-248, a map the reference never fills);
 * must be called before the device is initialised */
int curplsh_resources_set_default_stream(curplsh_resources* res, int device, void* stream);
/* getAlternateStreams (include/device_resources.h:187-190); writes up to *count streams */
int curplsh_resources_get_alternate_streams(curplsh_resources* res, int device, void** streams, int* count);
/* getAsyncCopyStream (include/device_resources.h:199-201) */
int curplsh_resources_get_async_copy_stream(curplsh_resources* res, int device, void** stream);
/* syncDefaultStream (include/device_resources.h:220-222) */
int curplsh_resources_sync_default_stream(curplsh_resources* res, int device);

/* ------------------------------------------------------------ Index / IndexBF */
/* IndexBF(DeviceResources*, int dim, IndexBFConfig) (include/index_bf.h:23-24, src/index.cpp:8-27) */
int curplsh_index_bf_create(curplsh_resources* res, int dim, const curplsh_bf_config* cfg,
                            curplsh_index** out);
/* ~IndexBF */
int curplsh_index_destroy(curplsh_index* index);
/* Index::train (include/index.h:29); brute force needs none: a no-op, as src/index_bf.cpp:13-15 */
int curplsh_index_train(curplsh_index* index, int64_t num, const float* data);
/* Index::add (include/index.h:38, src/index_bf.cpp:26-44): rows get sequential labels; squared norms and
 * the quantised operand copies are computed once here.  Unlike the reference (one add only,
 * index_bf.cpp:27) further adds append.  Synchronous; device `data` is read after the work already
 * queued on the legacy default stream (work on other streams that writes it must be complete). */
int curplsh_index_add(curplsh_index* index, int64_t num, const float* data);
/* Index::search (include/index.h:52-53, src/index_bf.cpp:46-74): k nearest rows of every query,
 * ascending squared L2 distance, ties by lower row index; slots beyond the number of rows are
 * (-1, FLT_MAX).  k must be in [1, 1024] (search.cu:121-122).  Uses the index's default precision,
 * runs on the resources' default stream (ordered after the work already queued on the legacy default
 * stream) and returns when the results are in place. */
int curplsh_index_search(curplsh_index* index, int64_t num, const float* queries, int k, int* indices,
                         float* distances);
/* search with an explicit precision form (-1: index default), rerank factor (<= 0: index default)
 * and stream (NULL: the resources' default stream, ordered after the legacy default stream; an
 * explicit stream is ordered only by itself).  When queries, indices and distances are all device memory the
 * call is asynchronous on `stream`; otherwise it synchronises before returning. */
int curplsh_index_search_ex(curplsh_index* index, int64_t num, const float* queries, int k, int precision,
                            int rerank_factor, int* indices, float* distances, void* stream);
/* As curplsh_index_search_ex, synchronous, also returning device-timed milliseconds of the passes
 * (CUDA events on the launching stream): pass_ms[0] query prep (and the sampled bound estimate when
 * one is used), [1] fused tensor-core filter over the whole database, [2] merge + exact rerank,
 * [3] whole search including any host<->device copies and any re-search of queries whose
 * estimate failed. */
int curplsh_index_search_profiled(curplsh_index* index, int64_t num, const float* queries, int k,
                                  int precision, int rerank_factor, int* indices, float* distances,
                                  void* stream, float* pass_ms);
/* Allocation-free search.  No counterpart in the reference: it exists for callers that cannot
 * allocate device memory while serving (a process whose GPU memory is owned by another allocator,
 * or a latency-critical loop where cudaMalloc/cudaFree's device-wide synchronisation is not
 * acceptable).  Same results as curplsh_index_search_ex with the index's default precision, but
 * the per-call working memory is a fixed 64 MiB array inside the library (held by every GPU that
 * loads it, until exit) instead of cudaMalloc'd buffers.  queries [num x dim], indices and
 * distances [num x k] must be device memory of the index's device; calls on one device are
 * serialised and the call returns when the results are written (it synchronises `stream`, NULL =
 * the legacy default stream).  The first call on a device looks up the array's device address, so
 * make it before any stream capture.  Requests whose working set exceeds the array are rejected
 * with CURPLSH_ERR_INVALID_ARG (roughly: num * (2*k'+256+max(k',256)) * 8 bytes must fit, k' the
 * candidate count); an index whose FP8 copy was never built by a regular FP8 search is rejected
 * with CURPLSH_ERR_STATE. */
int curplsh_index_search_noalloc(curplsh_index* index, int64_t num, const float* queries, int k, int* indices,
                                 float* distances, void* stream);
/* Index::reset (include/index.h:56, src/index_bf.cpp:17-24) */
int curplsh_index_reset(curplsh_index* index);
/* getDimension / getNumData / getDevice (include/index.h:58-64) */
int curplsh_index_get_dimension(const curplsh_index* index, int* out);
int curplsh_index_get_num_data(const curplsh_index* index, int64_t* out);
int curplsh_index_get_device(const curplsh_index* index, int* out);

/* ------------------------------------------------------------ free functions */
/* computeL2Norm (include/internal/norm.h:7-8, src/internal/norm.cu:191-202): device pointers,
 * vectors [num x dim] row-major, norms [num]; squared != 0 gives squared norms. */
int curplsh_compute_l2_norm(const float* vectors, int64_t num, int dim, float* norms, int squared,
                            void* stream);
/* searchL2Distance (include/internal/search.h:7-11, src/internal/search.cu:79-216) over device
 * buffers: bases [nb x dim], queries [nq x dim], indices/distances [nq x k].  base_norms is accepted
 * for signature parity and may be NULL (norms are recomputed in the engine's own layout).
 * exact_distances != 0 returns ||q - x||^2; 0 returns the reference's relative form
 * ||x||^2 - 2 q.x (= exact - ||q||^2).  Synchronous. */
int curplsh_search_l2_distance(curplsh_resources* res, const float* bases, int64_t nb, const float* base_norms,
                               const float* queries, int64_t nq, int dim, int k, int* indices,
                               float* distances, int exact_distances);

/* ------------------------------------------------------------ batched search */
/* No counterpart in the reference (its IndexBF::search serves one query matrix against one index
 * per call, src/index_bf.cpp:46-74).  A batch is a fixed list of (index, queries, k, outputs)
 * items, possibly over several indexes of different dimensions, planned once and replayed as ONE
 * CUDA graph launch: per (precision form, dimension) group one segmented query-prep kernel, one
 * persistent fused filter kernel whose balanced schedule spans every item of the group (several
 * small query batches against the same index share query blocks), and one merge + rerank kernel;
 * the groups run as parallel branches of the graph.  Each item's results are the same as curplsh_index_search_ex of that item alone with
 * the same precision and rerank factor. */
typedef struct curplsh_batch curplsh_batch;

typedef struct curplsh_batch_item {
  curplsh_index* index;
  int64_t num;           /* queries in this item (0 allowed) */
  const float* queries;  /* device [num x dim] of the index's device */
  int32_t k;             /* 1..1024 */
  int32_t pad0;
  int32_t* indices;      /* device [num x k] */
  float* distances;      /* device [num x k] */
} curplsh_batch_item;

/* Plans the batch (the pointers are captured: keep them valid and overwrite their contents
 * between runs), allocates its working memory and captures the graph.  precision -1 and
 * rerank_factor <= 0 take each index's default.  All indexes must live on one device.  Must not
 * be called while the calling thread captures a stream. */
int curplsh_batch_create(const curplsh_batch_item* items, int count, int precision, int rerank_factor,
                         curplsh_batch** out);
/* Launches the graph on `stream` (NULL: the first index's default stream, ordered after the work
 * already queued on the legacy default stream).  wait != 0 synchronises
 * and checks the device status word.  An index changed by add()/reset() since the last plan is
 * re-planned (and the graph re-captured) first. */
int curplsh_batch_run(curplsh_batch* batch, void* stream, int wait);
/* Kernel launches in one run of the graph, and bytes of device working memory held. */
int curplsh_batch_get_info(const curplsh_batch* batch, int* kernel_launches, int64_t* workspace_bytes);
int curplsh_batch_destroy(curplsh_batch* batch);

/* ------------------------------------------------------------ serving loop */
/* No counterpart in the reference.  Continuous batching of search requests against one resident
 * index: curplsh_server_submit() queues a request and returns a ticket at once; a scheduler thread
 * forms steps from the waiting requests (first come, first served, at most max_step_queries queries)
 * and issues each step -- prep, fused filter, merge + rerank -- on one of max_inflight streams, so
 * requests that arrive while earlier steps run are admitted and run concurrently with them.
 * Admission is by device memory: all in-flight steps share one arena of memory_budget bytes
 * allocated at creation, and a step waits until its working memory fits.  Every result equals
 * curplsh_index_search_ex of that request alone with the server's precision and rerank factor.
 * queries, indices and distances may be host or device memory (device memory of the index's
 * device); they must stay valid, and unmodified, until curplsh_server_wait() returns for the
 * ticket.  Changing the index (add, reset) while requests are in flight is not supported. */
typedef struct curplsh_server curplsh_server;

typedef struct curplsh_server_config {
  int32_t precision;        /* -1 (default): the index's default precision */
  int32_t rerank_factor;    /* <= 0 (default): the index's */
  int32_t max_inflight;     /* steps on the GPU at once (default 3, at most 16) */
  int32_t max_step_queries; /* queries per step and per request (default 4096) */
  int64_t memory_budget;    /* device bytes for all in-flight steps (default 2 GiB) */
} curplsh_server_config;

typedef struct curplsh_server_stats {
  int64_t requests_done;
  int64_t queries_done;
  int64_t steps;
  int64_t kernel_launches;    /* kernels issued by all steps */
  int64_t max_step_queries;   /* largest step formed */
  int64_t peak_bytes_in_use;  /* largest arena use */
  int32_t max_inflight_seen;  /* most steps on the GPU at once */
  int32_t pad0;
  double busy_seconds;        /* wall time with at least one step on the GPU */
} curplsh_server_stats;

void curplsh_server_config_init(curplsh_server_config* cfg);
int curplsh_server_create(curplsh_index* index, const curplsh_server_config* cfg, curplsh_server** out);
/* Queues num (1..max_step_queries) queries; rejects requests whose working memory alone exceeds the
 * budget. */
int curplsh_server_submit(curplsh_server* server, int64_t num, const float* queries, int k, int32_t* indices,
                          float* distances, int64_t* ticket);
/* Waits for a ticket (timeout_s < 0: no limit; CURPLSH_ERR_STATE on time-out, the ticket stays valid),
 * returns its status and, when latency_s is not NULL, seconds from submit to completion.  A ticket
 * can be waited for once. */
int curplsh_server_wait(curplsh_server* server, int64_t ticket, double timeout_s, double* latency_s);
/* curplsh_server_wait that also splits the latency (host clock) into phases[0..2]: waiting for a
 * step (submit to issue), the step on the device (issue until the scheduler sees its end event
 * complete), and retiring (until the results are visible to wait); phases[3] is the step's device
 * work itself, timed by CUDA events around it on its stream, and phases[4] the time from issue
 * until its begin event was seen complete (both part of phases[1]; the scheduler looks every
 * 200 us while steps are in flight).  phases must hold 5 doubles.  No counterpart in the
 * reference. */
int curplsh_server_wait_phases(curplsh_server* server, int64_t ticket, double timeout_s, double* latency_s,
                               double* phases);
int curplsh_server_get_stats(curplsh_server* server, curplsh_server_stats* out);
/* Finishes every queued request, then frees the server. */
int curplsh_server_destroy(curplsh_server* server);

/* ------------------------------------------------------------ sharded search */
/* No counterpart in the reference (one device per index, include/index.h:18-82).  Merges the top-k
 * lists of a database split by rows over num_shards shards: distances and indices are device arrays
 * [num_shards][num_queries][k] (each shard's search result with shard-local row indices, as an
 * all-gather lays them out), shard_bases a device array [num_shards] of each shard's first global
 * row.  Writes the global top-k, ascending distance, ties by lower global row, padding (-1,
 * FLT_MAX).  Asynchronous on `stream`; num_shards * k <= 16384. */
int curplsh_merge_shard_results(int64_t num_queries, int k, int num_shards, const float* distances,
                                const int32_t* indices, const int64_t* shard_bases, int32_t* out_indices,
                                float* out_distances, void* stream);

/* ------------------------------------------------------------ launch tuning */
/* No counterpart in the reference (its tile sizes are fixed, src/internal/search.cu:12-77).  A
 * process-wide table of fused-pass parameters per (precision, dim, k bucket, query-count bucket),
 * buckets being ceil(log2 k) and floor(log2 num_queries).  Neither parameter changes any result:
 *   split_q4       the longest run of database tiles one candidate pool covers, in quarters of
 *                  the CTA range the search gets alone (4 = the range itself, the default;
 *                  smaller values cut it; values above 4 act as 4);
 *   pool_headroom  candidate-pool slack beyond k' + 128 keys (the k-select width; default 256).
 * Filled by curplsh_b200.autotune, read by search, search_ex, search_profiled and the batch
 * planner (the allocation-free search keeps the defaults). */
int curplsh_tuning_set(int precision, int dim, int k, int64_t num_queries, int split_q4, int pool_headroom);
/* Writes the bucket's parameters (the defaults when it was never set). */
int curplsh_tuning_get(int precision, int dim, int k, int64_t num_queries, int* split_q4, int* pool_headroom);
int curplsh_tuning_clear(void);

/* ------------------------------------------------------------ sampled bound estimate */
/* No counterpart in the reference.  A search of many queries against a large database
 * (curplsh_index_search / _ex / _profiled) may first run the fused pass over a strided sample of
 * the database, keeping per query the smallest distance of every 128-row block of the sample,
 * and start every candidate pool of the full pass at the j-th smallest of those block minima,
 * so far fewer rows survive the filter.  The merge pass verifies the estimate exactly (k'
 * candidates under the final bound prove the result complete); queries it fails are searched
 * again without it, so results are identical with the estimate on or off.  With queries,
 * indices and distances all in device memory and no coarse-margin check (the FP32-exact form,
 * or the check off) the verification runs on the stream (if any query failed, the full pass and
 * merge run again from no bound) and the call stays asynchronous; otherwise the host verifies it
 * and the call returns synchronised.  The switch is process-wide; on (1) by default. */
int curplsh_set_bound_estimate(int enabled);
int curplsh_get_bound_estimate(int* enabled);
/* The estimate a search of num_queries queries with this k / precision / rerank factor would
 * use: *sample_rows = 0 when none, else the sample size, its row step and the rank j among the
 * sample_rows / 128 block minima. */
int curplsh_index_estimate_plan(curplsh_index* index, int64_t num_queries, int k, int precision,
                                int rerank_factor, int* sample_rows, int* step, int* rank);
/* The same plan for a bare shape (N rows, num_queries queries, k' candidates, num_sms SMs),
 * without an index or a device: what any search of that shape would use while the switch is
 * on. */
int curplsh_estimate_plan_shape(int64_t num_rows, int64_t num_queries, int kprime, int num_sms, int* sample_rows,
                                int* step, int* rank);
/* Number of queries this index searched again after their estimate failed (since creation). */
int curplsh_index_get_fallback_count(curplsh_index* index, int64_t* count);

/* ------------------------------------------------------------ coarse-margin check */
/* No counterpart in the reference.  The BF16 and FP8 forms pick k' candidates by coarse
 * distances and rerank them exactly; rows outside the candidates are never looked at again.
 * With the check on, the merge pass compares, per query, the margin between the largest
 * candidate coarse distance and the k-th exact result with the coarse errors (coarse - exact)
 * of the candidates themselves: when the margin is smaller than the largest error plus the
 * errors' spread, the coarse form is too coarse for this query's data and the query is searched
 * again in the FP32-exact form before the call returns (counted by
 * curplsh_index_get_coarse_fallback_count).  Forms whose coarse distances are exact for the data (BF16
 * on integer or BF16-valued rows) always pass.  It is a check of the data against the form's
 * precision, not a proof.  Applies to curplsh_index_search / _ex / _profiled; a search that uses
 * it returns synchronised even with device buffers.  Process-wide; on (1) by default. */
int curplsh_set_coarse_check(int enabled);
int curplsh_get_coarse_check(int* enabled);
/* CTA pairs (engine-specific, no counterpart in cuRPLSH): a fused pass over at least four
 * 128-query blocks runs as clusters of two CTAs, each pair sharing one 256-row tensor-core MMA
 * (tcgen05 cta_group::2) over two query blocks, so every database tile crosses from L2 once per
 * 256 queries instead of once per 128.  0 = off, 1 = on for every such pass, 2 = automatic (the
 * default): on for BF16 passes with d >= 320 and FP32-exact passes with d >= 192, where the
 * tensor work per tile is heavy enough for the halved tile bytes to pay (BF16 at d = 512: 5.98 ->
 * 4.54 ms for 4,096 queries over 10^6 rows; at d = 128 pairs are slower).  Results do not depend
 * on it.  Applies to searches, batches and servers planned after the call.  Process-wide. */
int curplsh_set_cta_pairs(int enabled);
int curplsh_get_cta_pairs(int* enabled);
/* Dual query blocks (engine-specific, no counterpart in cuRPLSH; on by default): an FP8 fused
 * pass over at least four 128-query blocks keeps two blocks resident in each CTA and feeds each
 * 128-row database tile to two 128 x 128 tensor-core MMAs, so a tile crosses from L2 once per 256
 * queries.  Results do not depend on it.  Applies to plans made after the call; process-wide. */
int curplsh_set_dual_blocks(int enabled);
int curplsh_get_dual_blocks(int* enabled);
/* Number of queries this index searched again in the exact form after their coarse margin
 * failed (since creation). */
int curplsh_index_get_coarse_fallback_count(curplsh_index* index, int64_t* count);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* CURPLSH_B200_H_ */
