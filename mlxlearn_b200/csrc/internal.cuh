// Internal declarations shared by the library's translation units.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/b200knn.h"

namespace b2k {

constexpr int kTcBM = 128;   // query rows per tcgen05 tile (TMEM lanes)
constexpr int kTcBN = 256;   // reference rows per tcgen05 tile (TMEM columns)
constexpr int kTcBK = 64;    // 16-bit elements per 128-byte swizzle row
constexpr int kTcAug = 16;   // norm columns appended to every operand row (one K=16 step)
constexpr int kTcBKf = 32;   // fp32 (tf32) elements per 128-byte swizzle row
constexpr int kTcAugF = 8;   // tf32 norm columns (one K=8 step, 32 bytes like kTcAug)
constexpr int kTcBKu = 128;  // u8 elements per 128-byte swizzle row
constexpr int kU8MaxK = 16;  // largest k of the exact u8 screen
constexpr int kU8MaxD = 16384;  // ||x||^2 and -2<q, x> of u8 rows fit int32
constexpr int kSimtBM = 128; // query rows per CUDA-core tile
constexpr int kSimtBN = 64;  // reference rows per CUDA-core tile
constexpr int kListCap = 512;      // screen list entries per (split, query)
constexpr int kCertifyCap = 1024;  // re-rank candidates per query held in shared memory
constexpr int kExactCap = 4096;    // exhaustive-scan candidates per query
constexpr int kMaxK = 64;          // largest k the screens track in registers
constexpr int kMaxShards = 16;     // reference-row shards one merge takes
constexpr int kMaxShardK = 256;    // largest k of a shard merge

// Outputs of a screen kernel: per (split, query) a list of (v, column)
// candidates, the list length (may exceed cap = overflow), and the k smallest
// v values the split saw.
struct ScreenOut {
  int2* lists;     // [S][m_pad][cap]
  int* counts;     // [S][m_pad]
  float* kth;      // [S][m_pad][k], or null: the lists alone give V_k (lazy screens)
  int cap;
  int m_pad;
};

// Device-resident index (one per fitted estimator).
struct Index {
  int device = 0;
  int64_t n = 0;
  int32_t d = 0;
  float* X = nullptr;        // [n, d] owned float32 copy
  float* center = nullptr;   // [d] fl32 of the column means (screens work on x - center)
  double* colsum = nullptr;  // [d] column sums (float64)
  float* nx32 = nullptr;     // [n] fl32(||x - center||^2)
  double* nx64 = nullptr;    // [n] ||x - center||^2 in float64
  // screen statistics (device scalars, then cached on host)
  float* stats_dev = nullptr;  // [8]: see prep kernels
  float xn_max = 0, nx_max = 0;  // max ||fp32 operand||, max ||x - center||^2
  float ex32_max = 0;            // max ||(x - center) - fp32 operand||
  bool range_ok = false;         // all |x| in {0} U [2^-60, 2^50]
  // bf16 copy for the tcgen05 screen (lazy)
  bool bf16_ready = false;
  int64_t n_pad_tc = 0;          // multiple of kTcBN
  int32_t dp = 0;                // d padded to a multiple of kTcBK
  uint16_t* Xh = nullptr;        // [n_pad_tc, dp]
  float xh_max = 0, ex_max = 0;  // max ||bf16 operand||, max ||(x - center) - bf16 operand||
  CUtensorMap tmap_b;            // TMA map over Xh, box 64 x 256
  uint16_t* Xaug = nullptr;      // [n_pad_tc, 16] bf16 [n_hi, n_mid, n_lo, 0...] of ||x - c||^2
  uint16_t* aug_ones = nullptr;  // [128, 16] bf16 [1, 1, 1, 0...] (query side)
  CUtensorMap tmap_baug;         // over Xaug, box 16 x 256, 32-byte swizzle
  CUtensorMap tmap_aaug;         // over aug_ones, box 16 x 128, 32-byte swizzle
  // tf32 copy for the tcgen05 kind::tf32 screen (lazy, same row order as Xh)
  bool tf32_ready = false;
  int32_t dpt = 0;               // d padded to a multiple of kTcBKf
  float* Xt = nullptr;           // [n_pad_tc, dpt] tf32-rounded centred rows
  float* Xtaug = nullptr;        // [n_pad_tc, 8] tf32 [n_hi, n_mid, n_lo, 0...] of ||x - c||^2
  float* taug_ones = nullptr;    // [128, 8] [1, 1, 1, 0...] (query side)
  float xt_max = 0, ext_max = 0; // max ||tf32 operand||, max ||(x - c) - tf32 operand||
  CUtensorMap tmap_bt, tmap_btaug, tmap_ataug;
  // u8 copy for the exact integer screen (lazy; training row order), when
  // every coordinate is an integer in [0, 255]
  int u8_state = 0;              // 0 not checked, 1 integer pixels, -1 not
  bool u8_ready = false;
  int32_t dpu = 0;               // d padded to a multiple of kTcBKu
  uint8_t* Xu = nullptr;         // [n_pad_tc, dpu]
  int* nxu = nullptr;            // [n_pad_tc] ||x||^2 exactly; INT_MAX on padding rows
  CUtensorMap tmap_bu;           // over Xu, box 128 x 256, 128-byte swizzle
  // Row grouping of the bf16 operand (reorder.cu): operand row i holds
  // training row xperm[i]; rows sharing a nearest pivot are consecutive, so a
  // query tile's candidates fall in few reference tiles.  Null: identity.
  int* xperm = nullptr;          // [n] operand row -> training row
  int* xinv = nullptr;           // [n] training row -> operand row
  int* group_start = nullptr;    // [n_pivots + 1] first operand row of each pivot's group
  // pivots for query ordering (reorder.cu)
  int n_pivots = 0;
  float* pivots = nullptr;       // [n_pivots, d] centred rows
  float* pivot_norms = nullptr;  // [n_pivots]
  uint16_t* pivots_h = nullptr;  // bf16 pivots for the assignment, zero padded:
  int pivot_dpa = 0;             // [pivot_rows_padded(n_pivots), pivot_dpa]
  cudaStream_t stream = nullptr;
  std::mutex mu;
};

// ------------------------------------------------------------ prep kernels
void launch_prep_index(Index* ix, cudaStream_t st);
// flag |= 1 when some value is NaN or infinite
void launch_nonfinite_check(const float* v, int64_t count, int* flag, cudaStream_t st);
// bf16 operand rows [n_pad, dp] (n_pad = n rounded up to 256) into Xh, row i
// from training row rows[i] (rows null: row i); the operand statistics go to
// the index's stats_dev [3], [4].
void launch_prep_index_bf16(const Index* ix, uint16_t* Xh, cudaStream_t st,
                            const int* rows = nullptr);
// norm columns [n_pad, 16] into Xaug (row i from training row rows[i]); when
// `ones` is set, also the query-side columns [128, 16].
void launch_prep_aug(const Index* ix, uint16_t* Xaug, uint16_t* ones, cudaStream_t st,
                     const int* rows = nullptr);
// The same for the tf32 screen: operand rows [n_pad, dpt] (statistics into
// stats_dev [6], [7]) and norm columns [n_pad, 8] with the ones [128, 8].
void launch_prep_index_tf32(const Index* ix, float* Xt, cudaStream_t st, const int* rows);
void launch_prep_aug_tf32(const Index* ix, float* Xtaug, float* ones, cudaStream_t st,
                          const int* rows);
// ------------------------------------------------- exact u8 screen (exact_u8.cu)
// flag |= 1 when some value is not an integer in [0, 255]
void launch_u8_check(const float* v, int64_t count, int* flag, cudaStream_t st);
// rows [rows_pad, dpu] u8 of v [rows, d] (zero padding) and their squared norms
// (exact; `pad_norm` on padding rows)
void launch_prep_u8(const float* v, int64_t rows, int d, int64_t rows_pad, int dpu, uint8_t* out,
                    int* norms, int64_t* norms64, int pad_norm, cudaStream_t st);
// Per query: the k smallest (v, column) over the S lists of k entries each
// (v = ||x||^2 - 2<q, x>, INT_MAX = empty), then squared distance ||q||^2 + v
// (exact) or its square root, and the column as index.  rows: the query's
// output row (null: its own).
void launch_u8_merge(const int2* lists, int S, int64_t m, int64_t m_pad, int k,
                     const int64_t* nq, int squared, double* dist, int64_t* idx,
                     const int* status, cudaStream_t st);

// Query preparation: per-row fp32/bf16 error bounds and the bf16 operand.
struct QueryPrep {
  float* E;        // [m_pad] screen error bound (fp32, rounded up)
  uint16_t* Ah;    // [m_pad, dp] -2*bf16(q - center) (bf16 mode only)
  float* At;       // [m_pad, dpt] -2*tf32(q - center) (tf32 mode only)
  int* flags;      // [1]: bit 0 = some coordinate outside the screen range
  double* nq;      // [m_pad] ||q - center||^2 (float64), optional
};
void launch_prep_queries(const Index* ix, const float* Q, int64_t m, int64_t m_pad, int mode,
                         QueryPrep qp, cudaStream_t st);
// One problem of a query preparation (the batched form takes a table of them).
struct PrepProblem {
  const float* Q;
  int64_t m, m_pad;
  int d, dp, mode;
  const float* center;
  float xh_max, nx_max, ex_max;  // operand statistics of the index for `mode`
  float* E;
  uint16_t* Ah;                  // [m_pad, dp] (bf16 mode)
  float* At;                     // [m_pad, dp] (tf32 mode; dp is then the tf32 width)
  double* nq;
  int* flags;
};
PrepProblem prep_problem(const Index* ix, const float* Q, int64_t m, int64_t m_pad, int mode,
                         const QueryPrep& qp);
void launch_prep_queries_batch(const PrepProblem* tab, const int64_t* row_start, int P,
                               int64_t total_rows, cudaStream_t st);

// ---------------------------------------------------------- screen kernels
constexpr int kSinkKnn = 0, kSinkRadiusCount = 1, kSinkRadiusFill = 2, kSinkRadiusList = 3;
struct SinkArgs;
// tf32: the kind::tf32 form over the index's tf32 operand (kNN sinks only).
// home (with S = 1): query tile t scans only reference tiles
// [home[t], home[t] + home_tiles) -- the seeding pass of grouped rows.
int launch_screen_tc(Index* ix, const CUtensorMap* tmap_a, int64_t m, int64_t m_pad,
                     int exclude_self, int64_t q_offset, int S, const float* E, int sink_kind,
                     const SinkArgs& sa, int* status, cudaStream_t st,
                     const int* perm = nullptr, int* unit_counter = nullptr, bool tf32 = false,
                     const int* home = nullptr, int home_tiles = 0);
// The exact u8 screen (kind::i8; index and queries integers in [0, 255]):
// per (split, column group, query) the k smallest (||x||^2 - 2<q, x>, column)
// into sa.out.lists (cap = k), columns in training order; E unused.
int launch_screen_tc_u8(Index* ix, const CUtensorMap* tmap_a, int64_t m, int64_t m_pad,
                        int exclude_self, int64_t q_offset, int S, const SinkArgs& sa,
                        int* status, cudaStream_t st, int* unit_counter);
int tc_column_groups(int k);
int tc_u8_column_groups(int k);  // lists per (split, row) of the u8 screen
int tc_radius_groups();  // candidate lists per (split, row) of the tcgen05 radius screens
bool tc_lazy_sink(int k);  // the tcgen05 kNN screen's lazy tracker (no k-th output)
// noalloc: one scanner per row (half the list memory of the default two)
void launch_screen_simt(const Index* ix, const float* Q, int64_t m, int64_t m_pad,
                        int exclude_self, int64_t q_offset, int S, const float* E, int sink_kind,
                        const SinkArgs& sa, cudaStream_t st, const int* perm = nullptr,
                        bool noalloc = false);
// candidate lists per (split, query) of the CUDA-core screen
int simt_column_groups(int sink_kind, bool noalloc = false);

// ----------------------------------------------------------- query order
int pivot_count(int64_t n);
int pivot_rows_padded(int P);  // pivots padded to the assignment's tile
int pivot_dims_padded(int d);  // features padded to its chunk
void launch_pivots(Index* ix, cudaStream_t st);
// perm[i] = original row of sorted position i; Qp = Q[perm]
void launch_query_order(const Index* ix, const float* Q, int64_t m, int* key, int* hist,
                        int* perm, float* Qp, cudaStream_t st);
// key[r] = nearest pivot of row r of X [n, d] (the index's centre applied);
// hist[p] = rows per pivot
void launch_assign_rows(const Index* ix, const float* X, int64_t n, int* key, int* hist,
                        cudaStream_t st);
// home[t] = first reference tile of query tile t's window of `window` tiles:
// the tiles holding the grouped rows of the pivot nearest to the tile's
// middle query (perm, key: the query order and pivot keys of
// launch_query_order)
void launch_home_tiles(const int* perm, const int* key, int64_t m, const int* group_start,
                       int n_tiles, int window, int* home, int m_tiles, cudaStream_t st);

// second pass over uncertified rows: Qout[i] = Qs[rows[i]], pout[i] = perm[rows[i]]
void launch_gather_fallback(const float* Qs, int d, const int* rows, const int* perm, int count,
                            float* Qout, int* pout, cudaStream_t st);

// -------------------------------------------------- certify + re-rank + exact
struct CertifyArgs {
  const float* X;
  const float* Q;
  int64_t n, m;
  int d, k, S;
  ScreenOut scr;
  const float* E;
  double* dist;        // [m, k] or null
  int64_t* idx;        // [m, k]
  int* fallback_list;  // [m] query ids needing the exhaustive scan
  int* fallback_count; // [1]
  unsigned long long* counters;  // [4]: candidates, entries, exact compares, -
  const int* perm;     // row -> output row (or null)
  int64_t row_base;    // added to the row in fallback_list entries (batched runs)
  int squared;         // write squared distances (else their square roots)
  const int* cols;     // list column -> training row (grouped operand rows), or null
  const int* status;   // error word of the call: nonzero (a screen gave up) = do nothing
  const double* nq;    // [m] ||q - center||^2 (float64): enables the two-stage refine, or null
  unsigned long long* refined;  // candidates refined in fp32 (counter), or null
};
void launch_certify(const CertifyArgs& a, cudaStream_t st);
// problem p owns global rows [row_start[p], row_start[p + 1]) of the batch
void launch_certify_batch(const CertifyArgs* tab, const int64_t* row_start, int P,
                          int64_t total_rows, cudaStream_t st);

struct ExactArgs {
  const float* X;
  const float* Q;
  int64_t n, m;
  int d, k;
  int exclude_self;
  int64_t q_offset;
  const int* rows;      // query ids to process, or null = all rows
  const int* row_count; // device count for `rows`
  double* scratch;      // [grid][n]
  int grid;
  double* dist;
  int64_t* idx;
  unsigned long long* counters;
  int* status;
  const int* perm;      // row -> original query row for output and self (or null)
  int squared;          // write squared distances (else their square roots)
};
void launch_exact(const ExactArgs& a, cudaStream_t st);
// rows: global row ids of the batch; scratch: [grid][n_max] or null
void launch_exact_batch(const ExactArgs* tab, const int64_t* row_start, int P, const int* rows,
                        const int* row_count, double* scratch, int64_t n_max, int grid,
                        cudaStream_t st);

// ------------------------------------------------------------------ radius
// Average candidates per row from which classify and compact take one CTA
// per row instead of one warp.
constexpr int kWideRowCandidates = 512;
struct RadiusPlanArgs {
  const float* X;
  const float* Q;
  int d;
  int64_t m, m_pad;
  int S;
  const int64_t* roff;   // [S][m_pad] candidate offsets
  const int* rcount;     // [S][m_pad] candidate counts
  const int* cols;       // candidates (training rows) at roff
  bool wide;             // one CTA per row (long rows), else one warp per row
  double* cdist;         // [ncand] member distance or -1
  int64_t* mcount;       // [m] members per query
  double R2;
  unsigned long long* exact_tests;
  const int* status;     // error word of the call: nonzero = leave the outputs alone
};
void launch_radius_threshold(const double* nq, const float* E, int64_t m, int64_t m_pad,
                             double R2, float* thr, cudaStream_t st);
// Multi-block scans; `scratch` holds scan_scratch_len(m) int64 values.
int64_t scan_scratch_len(int64_t m);
void launch_scan_split_counts(const int* counts, int S, int64_t m, int64_t m_pad, int64_t* off,
                              int64_t* total, int64_t* scratch, cudaStream_t st);
void launch_scan_rows(const int64_t* counts, int64_t m, int64_t* indptr, int64_t* scratch,
                      cudaStream_t st);
void launch_classify(const RadiusPlanArgs& r, cudaStream_t st);
// Single-pass screen: rows whose count passed `cap` in any of their S lists
// are appended to rows[] (rows[m] = how many) and their counts zeroed, so
// classify and compact skip them.
void launch_radius_overflow(int* rcount, int S, int64_t m, int64_t m_pad, int cap, int* rows,
                            cudaStream_t st);
// Candidates to one array at their scanned offsets roff, as training rows
// (xperm: grouped operand rows, else null).  src: lists of `cap` entries at
// slot * cap (single pass), or cap = 0 and src == dst (counted form: the
// fill's `count` candidates translated in place).  Nothing when *status is an
// error.
void launch_radius_pack(const int* src, int cap, const int* rcount, int S, int64_t m,
                        int64_t m_pad, const int64_t* roff, const int* xperm, int* dst,
                        int64_t count, const int* status, cudaStream_t st);
// mcount[rows[i]] = sub_indptr[i + 1] - sub_indptr[i]: members of the rows a
// counted sub-call answered
void launch_radius_sub_counts(const int* rows, int count, const int64_t* sub_indptr,
                              int64_t* mcount, cudaStream_t st);
// the sub-call's rows into the CSR at indptr[rows[i]] (dist, sub_dist may be null)
void launch_radius_sub_scatter(const int* rows, int count, const int64_t* sub_indptr,
                               const int64_t* sub_indices, const double* sub_dist,
                               const int64_t* indptr, int64_t* indices, double* dist,
                               cudaStream_t st);
void launch_compact(const RadiusPlanArgs& r, const int64_t* indptr, int64_t* indices,
                    double* dist, cudaStream_t st);
// Per-row sort by (distance, index), or by index alone when !by_dist (dist,
// if not null, then moves with its index).
// mid_rows/big_rows: scratch lists of m rows each, their counts zeroed.
void launch_sort_rows(const int64_t* indptr, int64_t m, int64_t* indices, double* dist,
                      int* mid_rows, int* mid_count, int* big_rows, int* big_count, int grid,
                      cudaStream_t st, bool by_dist = true);
void launch_sort_big_rows(const int64_t* indptr, const int* rows, int count, int64_t* indices,
                          double* dist, double* tmp_d, int64_t* tmp_i, int64_t tmp_stride,
                          int grid, cudaStream_t st, bool by_dist = true);
int radius_sort_cap();

// ------------------------------------------------------------------- votes
void launch_votes(const int64_t* idx, const double* dist, int64_t m, int k, const int* codes,
                  int n_classes, int weighted, double* votes, int64_t* pred, int* status,
                  cudaStream_t st);

// votes may be null when pred is given: pred[i] = the row's first maximum.
void launch_radius_votes(const int64_t* indptr, const int64_t* indices, const double* dist,
                         int64_t m, const int* codes, int n_classes, int weighted, double* votes,
                         int64_t* counts, cudaStream_t st, int64_t* pred = nullptr);
void launch_radius_means(const int64_t* indptr, const int64_t* indices, const double* dist,
                         int64_t m, const double* targets, int weighted, double* means,
                         int64_t* counts, cudaStream_t st);

// ---------------------------------------------------------------- backward
int knn_backward(const float* Q, int64_t m, const float* X, int64_t n, int d, int k,
                 const int64_t* idx, const float* G, const float* E, int squared, float* dQ,
                 float* dX, int* workspace, cudaStream_t st);
size_t knn_backward_workspace_ints(int64_t m, int64_t n, int k);

// helpers
int report_error(int code, const char* msg);  // sets b2k_last_error(), returns code
int check_knn_args(const Index& ix, int64_t m, int32_t k, int32_t exclude_self,
                   int64_t q_offset);
Index* index_of(b2k_index* h);
// kNN outputs (m x k, 8-byte entries) overlapping the queries (m x d floats)
// or each other; null outputs overlap nothing
bool buffers_overlap(const float* dQ, int64_t m, int d, int k, const double* dist,
                     const int64_t* idx);

// ------------------------------------------------------------ row shards
void launch_shard_merge(const double* D, const int64_t* I, int S, int64_t m, int kin, int kout,
                        int64_t self_offset, double eps, double* out_d, int64_t* out_i,
                        int32_t* flags, cudaStream_t st);
void launch_shard_keys(const double* D, const int64_t* I, int S, int64_t m, int kin,
                       const float* Q, const float* X, int64_t n_local, int d, int64_t row_lo,
                       const int64_t* flagged, int64_t F, uint64_t* keys, cudaStream_t st);
void launch_shard_resolve(const double* D, const int64_t* I, int S, int64_t m, int kin, int kout,
                          int64_t self_offset, const int64_t* flagged, int64_t F,
                          const uint64_t* keys, double* out_d, int64_t* out_i, cudaStream_t st);
// knn on device pointers (b2k_knn_device without the stats), synchronises st
int knn_device_run(Index& ix, const float* dQ, int64_t m, int k, int exclude_self,
                   int64_t q_offset, int mode, double* d_dist, int64_t* d_idx, cudaStream_t st);
int injected_fault();  // B2K_FAULT: 0 none, 1 alloc, 2 launch, 3 timeout
// bf16 operand rows and norm columns of an index into caller buffers, and the
// operand statistics the query bound needs (synchronises st)
int index_prepare_bf16_stats(Index& ix, uint16_t* Xh, uint16_t* Xaug, uint16_t* ones,
                             cudaStream_t st, float* xh_max, float* ex_max);
bool tensor_map_2d_bf16(CUtensorMap* map, const void* base, uint64_t inner, uint64_t outer,
                        uint32_t box_inner, uint32_t box_outer, int swizzle_bytes = 128);
bool tensor_map_2d_f32(CUtensorMap* map, const void* base, uint64_t inner, uint64_t outer,
                       uint32_t box_inner, uint32_t box_outer, int swizzle_bytes = 128);
int num_sms(int device);
// Polls a screen's bounded waits make before giving up: 2^26 unless
// B2K_SPIN_LIMIT sets it (tests force the timeout path with it).
uint32_t device_spin_limit();

}  // namespace b2k
