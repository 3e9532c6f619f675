/*
 * b200knn -- exact brute-force Euclidean neighbour search on NVIDIA B200 (sm_100a).
 *
 * C ABI of libb200knn.so.  Plain pointers and sizes only.  Every entry point
 * returns an int status (B2K_OK on success); b2k_last_error() gives a message
 * for the calling thread's last failure.
 *
 * Results contract (the one mlxlearn.neighbors defines):
 *  - kNN rows are ordered by the exact real squared distance of the float32
 *    coordinates, ties broken by the smaller training index;
 *  - a radius neighbour is a training row with exact squared distance
 *    <= fl64(radius * radius);
 *  - distances are float64 sqrt of the canonical squared distance (a strictly
 *    sequential float64 sum over features of (q_k - x_k)^2, no FMA); radius
 *    distances are sqrt(min(canonical, R2));
 *  - indices are int64.
 *
 * Each declaration cites the reference interface it replaces, by file:line in
 * the mlxlearn source tree.
 */
#ifndef B200KNN_H
#define B200KNN_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define B2K_API __attribute__((visibility("default")))
#else
#define B2K_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define B2K_OK 0
#define B2K_EINVAL 1      /* shape, k, offset, overlap or pointer errors      */
#define B2K_ENONFINITE 2  /* NaN / Inf coordinates                            */
#define B2K_ENOMEM 3      /* device or host allocation failed                 */
#define B2K_ECUDA 4       /* a CUDA runtime call failed                       */
#define B2K_ETIMEOUT 5    /* a bounded device wait gave up (kernel error)     */
#define B2K_EUNSUPPORTED 6 /* e.g. no sm_100 device, or a documented limit    */
#define B2K_EINJECTED 7   /* fault injected through B2K_FAULT (tests only)    */

/* ----------------------------------------------------------- search modes */
#define B2K_MODE_AUTO 0        /* bf16 screen where certified, else fp32      */
#define B2K_MODE_FP32 1        /* plain form: fp32 CUDA-core Gram screen      */
#define B2K_MODE_BF16 2        /* bf16 tcgen05 screen + certified re-rank     */
#define B2K_MODE_EXACT 3       /* float64 exhaustive scan + exact ties (slow) */
#define B2K_MODE_TF32 4        /* plain form on the tensor cores: tf32 tcgen05
                                  screen + the same certified re-rank         */
#define B2K_MODE_U8 5          /* integer pixels: exact u8 tcgen05 (kind::i8)
                                  screen, used by AUTO when the index and the
                                  queries are integers in [0, 255] and k <= 16;
                                  on other data the certified screens run      */
/* Flag ORed into the mode of b2k_knn / b2k_knn_device: distances are returned
 * as the canonical float64 squared distance instead of its square root (the
 * `_squared` option of DeviceNeighborIndex.query,
 * src/mlxlearn_device/_neighbors.py:271-280). */
#define B2K_MODE_SQUARED 16

typedef struct b2k_index b2k_index;

/* Per-call counters (optional: pass NULL). */
typedef struct b2k_stats {
  int32_t mode_used;        /* B2K_MODE_* actually run                         */
  int32_t splits;           /* reference splits of the screen                  */
  int64_t candidates;       /* candidates re-ranked in float64                 */
  int64_t list_entries;     /* screen list appends                             */
  int64_t fallback_rows;    /* queries resolved by the exhaustive exact scan   */
  int64_t second_pass_rows; /* queries the bf16 pass left to the fp32 pass     */
  int64_t exact_compares;   /* near-tie pairs resolved with exact integer keys */
  double screen_ms;         /* device time of the screen kernel (if timed)     */
  double total_ms;          /* device time of the whole call (if timed)        */
  int64_t refined;          /* candidates refined in fp32 by the certify pass  */
  double seed_ms;           /* device time of the screen's seeding pass, which
                               screen_ms includes (0: no seeding pass)        */
} b2k_stats;

/* Library version (major*10000 + minor*100 + patch). */
B2K_API int b2k_version(void);

/* Message for the calling thread's last failed call ("" if none). */
B2K_API const char *b2k_last_error(void);

/* ------------------------------------------------------------------ index */

/* Build a device-resident index from host float32 X[n, d] (C order).  The
 * index owns a copy; later changes to X do not affect it.
 * Replaces build_index / DeviceNeighborIndex construction
 * (src/mlxlearn/_kernels/distance.py:366-392,
 *  src/mlxlearn_device/_neighbors.py:447-466). */
B2K_API int b2k_index_create(const float *X, int64_t n, int32_t d, int32_t device, b2k_index **out);

/* Same from a device pointer (copied on `stream`, a cudaStream_t or NULL). */
B2K_API int b2k_index_create_device(const float *dX, int64_t n, int32_t d, void *stream,
                            b2k_index **out);

/* Release every device buffer of the index. */
B2K_API int b2k_index_destroy(b2k_index *index);

/* n, d of the index. Replaces NeighborIndex.n_samples / n_features
 * (src/mlxlearn/_kernels/distance.py:167-173). */
B2K_API int b2k_index_shape(const b2k_index *index, int64_t *n, int32_t *d);

/* Copy the owned float32 training rows back to host X[n, d]. Replaces
 * NeighborIndex.training_data / .X (src/mlxlearn/_kernels/distance.py:98-103,148-156). */
B2K_API int b2k_index_download(const b2k_index *index, float *X);

/* Device pointer of the owned float32 rows [n, d] (valid until destroy). */
B2K_API const float *b2k_index_device_data(const b2k_index *index);

/* -------------------------------------------------------------------- kNN */

/* k nearest training rows of each of m host queries Q[m, d].
 * Outputs (host): idx int64[m, k]; dist float64[m, k] or NULL.
 * exclude_self: query row i is training row q_offset + i and is skipped.
 * Replaces NeighborIndex.query (src/mlxlearn/_kernels/distance.py:242-270) and
 * the native CPU scan _neighbors_cpu_native.query
 * (src/mlxlearn/_kernels/_neighbors_cpu_native.cpp:362-418). */
B2K_API int b2k_knn(b2k_index *index, const float *Q, int64_t m, int32_t k, int32_t exclude_self,
            int64_t q_offset, int32_t mode, double *dist, int64_t *idx, b2k_stats *stats);

/* Same with device pointers, enqueued on `stream` (cudaStream_t; NULL = legacy
 * default stream).  The call synchronises `stream` before it returns, so
 * device-side errors (bounded-wait timeouts) are reported by its status.
 * dQ may be b2k_index_device_data(index) + q_offset*d for self-queries.
 * Replaces NeighborIndex.query_device / DeviceNeighborIndex.query
 * (src/mlxlearn/_kernels/distance.py:211-240,
 *  src/mlxlearn_device/_neighbors.py:271-443). */
B2K_API int b2k_knn_device(b2k_index *index, const float *dQ, int64_t m, int32_t k,
                   int32_t exclude_self, int64_t q_offset, int32_t mode, double *d_dist,
                   int64_t *d_idx, void *stream, b2k_stats *stats);

/* kNN on device pointers that allocates no memory.  No counterpart in the
 * reference: it exists for callers that must not allocate device memory
 * during a query (a process whose GPU memory is owned by another allocator or
 * arena, or a latency-critical path where cudaMalloc/cudaFree and their
 * implicit synchronisation are not allowed).  Its scratch is a fixed 32 MiB
 * array in the library's device image, reserved on every GPU that loads the
 * library until the process exits; a batch that needs more is rejected with
 * B2K_EINVAL and a message giving the largest allowed query count for that k.
 * The first call on a device looks up the array's device address: make it
 * before any stream capture.  Calls share the array, so calls whose GPU work
 * overlaps race; issue them in order on one stream.  Same results as
 * b2k_knn_device (fp32 screen, certified float64 re-rank, exact ties); the
 * call synchronises `stream` before returning. */
B2K_API int b2k_knn_device_noalloc(b2k_index *index, const float *dQ, int64_t m, int32_t k,
                                   int32_t exclude_self, int64_t q_offset, double *d_dist,
                                   int64_t *d_idx, void *stream);

/* Backward of selected kNN distances, all pointers on the device, enqueued on
 * `stream` (no synchronisation).  idx int64[m, k] fixes the neighbours;
 * grad float32[m, k] is d(loss)/d(distance); squared != 0 differentiates
 * s = ||q - x||^2, else e = sqrt(s) (dist = the forward e, float32[m, k]).
 * Writes grad_q float32[m, d] and/or grad_x float32[n, d] (either may be
 * NULL).  The reference scatter-add is deterministic (no float atomics).
 * No counterpart in the reference (mlxlearn has no differentiable kNN); it
 * backs the torch.autograd.Function in mlxlearn_b200/autograd.py. */
B2K_API int b2k_knn_backward(const float *dQ, int64_t m, const float *dX, int64_t n, int32_t d,
                             int32_t k, const int64_t *d_idx, const float *d_grad,
                             const float *d_dist, int32_t squared, float *d_grad_q,
                             float *d_grad_x, void *stream);

/* Exact kNN for many small problems given as segments of two device
 * arrays, in one call: problem p asks, for every query row in
 * [q_offsets[p], q_offsets[p+1]) of dQ float32[rows, d], for its k nearest
 * reference rows in [x_offsets[p], x_offsets[p+1]) of dX float32[*, d].
 * Offsets are HOST int64[segments + 1] starting at 0.  Writes d_idx
 * int64[rows, k] (indices within the reference segment) and d_dist
 * float64[rows, k] (or NULL), same order and tie rule as b2k_knn_device.
 * exclude_self: every query segment is its reference segment and row i skips
 * itself.  1 <= d <= 64, k <= 29.  Enqueued on `stream`; the call
 * synchronises it.  No counterpart in the reference (one problem per
 * NeighborIndex.query call, src/mlxlearn/_kernels/distance.py:242-270); it
 * backs the batched Chamfer loss of mlxlearn_b200/autograd.py. */
B2K_API int b2k_knn_segments(const float *dQ, const float *dX, int32_t d, const int64_t *q_offsets,
                             const int64_t *x_offsets, int32_t segments, int32_t k,
                             int32_t exclude_self, double *d_dist, int64_t *d_idx, void *stream);

/* Class votes of kNN results on the device (all pointers device, on
 * `stream`; the call synchronises).  codes int32[n_train] are class codes
 * 0..n_classes-1; votes float64[m, n_classes] receives per-class totals (1 or
 * 1/d, zero-distance rows use the 0/1 indicator of their zero entries);
 * pred int64[m] (or NULL) the first maximum (ties -> smallest code).
 * Returns B2K_EINVAL "All neighbors of some sample are getting zero weights."
 * when a row's weights sum to zero.  Replaces the reference's device votes
 * (src/mlxlearn_device/_neighbors_votes.py:12-244) and host np.add.at path
 * (src/mlxlearn/neighbors/_classification.py:150-163). */
B2K_API int b2k_class_votes(const int64_t *d_idx, const double *d_dist, int64_t m, int32_t k,
                            const int32_t *d_codes, int32_t n_classes, int32_t weighted,
                            double *d_votes, int64_t *d_pred, void *stream);

/* ------------------------------------------------------ reference-row shards
 * One rank per GPU holds a contiguous range of the fitted rows (its own
 * index) and answers the same query batch with its exact top-k_in, indices
 * made global (row + offset; -1 where the shard has fewer rows).  After one
 * exchange every rank holds d_dist / d_idx [n_shards, m, k_in] (shard
 * order) and merges them into the answer over all rows; the reference has
 * no multi-device path, so there is no counterpart to cite, and the merged
 * answer follows the neighbour order of one index over all rows
 * (src/mlxlearn/_kernels/_neighbors_cpu_native.cpp:170-190).
 *
 * b2k_shard_merge: out [m, k] from the float64 distances and global rows;
 * self_offset >= 0 drops global row self_offset + r from query r's answer
 * (the shards then search k_in = k + 1 without exclusion).  d_flags[r] = 1
 * marks queries whose shards' candidates lie within each other's float64
 * error interval: for those, every rank calls b2k_shard_keys (exact 640-bit
 * keys of the candidates its own index holds, into a zeroed
 * [n_flagged, n_shards * k_in, 10] buffer), the buffers are summed across
 * ranks (each entry has one owner), and b2k_shard_resolve rewrites those
 * rows in the exact order.  d_flagged lists the flagged queries ascending,
 * the same on every rank.  1 <= n_shards <= 16, 1 <= k <= 256,
 * k <= k_in <= k + 1.  Stream-ordered, no synchronisation. */
B2K_API int b2k_shard_merge(const double *d_dist, const int64_t *d_idx, int32_t n_shards,
                            int64_t m, int32_t k_in, int32_t k, int32_t d, int64_t self_offset,
                            double *d_out_dist, int64_t *d_out_idx, int32_t *d_flags,
                            void *stream);
B2K_API int b2k_shard_keys(b2k_index *index, int64_t row_offset, const float *dQ,
                           const int64_t *d_idx, int32_t n_shards, int64_t m, int32_t k_in,
                           const int64_t *d_flagged, int64_t n_flagged, uint64_t *d_keys,
                           void *stream);
B2K_API int b2k_shard_resolve(const double *d_dist, const int64_t *d_idx, int32_t n_shards,
                              int64_t m, int32_t k_in, int32_t k, int64_t self_offset,
                              const int64_t *d_flagged, int64_t n_flagged,
                              const uint64_t *d_keys, double *d_out_dist, int64_t *d_out_idx,
                              void *stream);

/* ---------------------------------------------------------------- batches */

/* One independent kNN problem of a batch: a fitted index and a device query
 * block answered into device outputs (same meaning as b2k_knn_device). */
typedef struct b2k_problem {
  b2k_index *index;
  const float *queries; /* device float32[m, d] of the index's d          */
  int64_t m;
  int32_t k;
  int32_t exclude_self;
  int64_t q_offset;
  double *dist;         /* device float64[m, k] or NULL                   */
  int64_t *idx;         /* device int64[m, k]                             */
} b2k_problem;

typedef struct b2k_batch b2k_batch;

typedef struct b2k_batch_stats {
  int32_t problems;        /* problems in the batch                           */
  int32_t graph_problems;  /* problems inside the captured graph              */
  int32_t screen_launches; /* persistent screen launches per run              */
  int32_t work_items;      /* (problem, query tile, reference range) units    */
  int64_t candidates;      /* re-ranked candidates (last finished run)        */
  int64_t fallback_rows;   /* rows answered by the exhaustive scan            */
  int64_t exact_compares;  /* exact comparator calls                          */
  float tune_ms;           /* time spent autotuning at create                 */
  float run_ms;            /* device time of the last finished run's graph    */
} b2k_batch_stats;

#define B2K_BATCH_AUTOTUNE 1 /* time the tuning candidates at create (cached per process) */

/* Plan a batch of independent problems (uneven n, d, k, m) and capture it as
 * one CUDA graph: a batched query preparation, one persistent tcgen05 screen
 * launch per (heap width, epilogue width) over a device work queue of
 * (problem, query tile, reference range) items balanced across the SMs, one
 * batched certify launch and one batched exhaustive-scan launch for the rows
 * that need it.  Problems the bf16 screen cannot certify (d < 16, k > 64,
 * coordinates outside its range) are answered by b2k_knn_device inside
 * b2k_batch_finish.  All indices must live on one device; queries and
 * outputs are read and written in place on every run, so refilling the
 * query buffers and running again answers the new queries.  No counterpart
 * in the reference (mlxlearn answers one problem per call); results are
 * identical to calling b2k_knn_device per problem. */
B2K_API int b2k_batch_create(const b2k_problem *problems, int32_t count, int32_t flags,
                             void *stream, b2k_batch **out);
/* Launch one run of the batch's graph on `stream` (asynchronous). */
B2K_API int b2k_batch_run(b2k_batch *batch, void *stream);
/* Wait for the last run on `stream`, check the device status, answer the
 * problems outside the graph (and any whose queries left the screen's range)
 * and fill `stats` (may be NULL). */
B2K_API int b2k_batch_finish(b2k_batch *batch, void *stream, b2k_batch_stats *stats);
B2K_API int b2k_batch_destroy(b2k_batch *batch);
/* create + run + finish + destroy. */
B2K_API int b2k_batch_submit(const b2k_problem *problems, int32_t count, void *stream);

/* ----------------------------------------------------------------- radius */

typedef struct b2k_radius_result b2k_radius_result;

/* Every training row within `radius` (inclusive, exact) of each host query.
 * The result is held by the library; read its size with
 * b2k_radius_result_nnz, copy it out with b2k_radius_result_fetch, then
 * release it.  Rows ascend by training index, or by (distance, index) when
 * sort_results is set.
 * Replaces NeighborIndex.query_radius_csr / RadiusSearch.query_with_plan and
 * the Metal screen (src/mlxlearn/_kernels/distance.py:285-342,
 * src/mlxlearn/_kernels/radius.py:380-453,
 * src/mlxlearn/_kernels/radius_metal_v1.py:552-611). */
B2K_API int b2k_radius(b2k_index *index, const float *Q, int64_t m, double radius,
               int32_t exclude_self, int64_t q_offset, int32_t need_distance,
               int32_t sort_results, b2k_radius_result **out);

/* Number of (query, neighbour) pairs of a radius result. */
B2K_API int b2k_radius_result_nnz(const b2k_radius_result *res, int64_t *nnz);

/* Copy a radius result into host CSR buffers: indptr int64[m+1],
 * indices int64[nnz], dist float64[nnz] or NULL (RadiusCSR,
 * src/mlxlearn/_kernels/radius_result.py:33-55). */
B2K_API int b2k_radius_result_fetch(const b2k_radius_result *res, int64_t *indptr, int64_t *indices,
                            double *dist);

/* Class votes of a radius result on the device, without downloading it:
 * codes int32[n_train] (device) are class codes 0..n_classes-1; votes
 * float64[m, n_classes] and counts int64[m] (device) receive per-row totals of
 * weight 1, or 1/d with a row's zero distances taking its 0/1 indicator
 * (weighted != 0 needs a result with distances), summed in ascending
 * training-index order.  Synchronises `stream`.  Replaces the host
 * reductions of RadiusNeighborsClassifier
 * (src/mlxlearn/_kernels/radius_reduce.py:19-60). */
B2K_API int b2k_radius_result_class_votes(const b2k_radius_result *res, const int32_t *d_codes,
                                          int32_t n_classes, int32_t weighted, double *d_votes,
                                          int64_t *d_counts, void *stream);

/* Predicted class codes of a radius result with uniform weights, on the
 * device: pred int64[m] receives each row's first maximum of its class counts
 * (ties -> smallest code; 0 for an empty row) and counts int64[m] its
 * neighbour count; the votes themselves are not written.  Equal to the argmax
 * of the normalised votes: the counts are integers, and dividing them by the
 * row's total keeps distinct counts distinct.  Synchronises `stream`.
 * Replaces the host argmax of RadiusNeighborsClassifier.predict
 * (src/mlxlearn/neighbors/_radius.py:110-136,180-205).  No separate reference entry
 * point: the reference computes the probabilities and takes their argmax. */
B2K_API int b2k_radius_result_class_predict(const b2k_radius_result *res,
                                            const int32_t *d_codes, int32_t n_classes,
                                            int64_t *d_pred, int64_t *d_counts, void *stream);

/* Means of float64 targets[n_train] (device) over each radius row, weight 1 or
 * 1/d as above; NaN for empty rows.  means float64[m], counts int64[m]
 * (device).  Replaces src/mlxlearn/_kernels/radius_reduce.py:62-94
 * (RadiusNeighborsRegressor). */
B2K_API int b2k_radius_result_means(const b2k_radius_result *res, const double *d_targets,
                                    int32_t weighted, double *d_means, int64_t *d_counts,
                                    void *stream);

B2K_API int b2k_radius_result_release(b2k_radius_result *res);

#ifdef __cplusplus
}
#endif
#endif /* B200KNN_H */
