// Radius search: exact membership S(q,x) <= R2 = fl64(r*r) as CSR.
//
// Pipeline (host side in b200knn.cu, b2k_radius):
//   1. threshold : T = R2 - ||y_q||^2 + E per query (rounded up): a column with
//                  v > T has S > R2 and is certainly not a neighbour.
//   2. screen    : the tcgen05 screen with RadiusListSink in one pass: each
//                  (split, column group, query) list keeps up to `cap`
//                  columns in ascending order and counts them all; rows whose
//                  count passed `cap` are answered again by a counted
//                  sub-call (RadiusCountSink, then RadiusFillSink at scanned
//                  offsets) -- the form the CUDA-core screen always uses.
//   2b. pack     : the lists (or, in the counted form, the fill) to one
//                  contiguous candidate array at the scanned offsets, operand
//                  rows mapped to training rows when the rows are grouped.
//   3. classify  : canonical float64 value s of every candidate; member iff
//                  s <= f64_in, non-member iff s > f64_out, otherwise the exact
//                  integer test key(S) <= floor(R2 * 2^298) (exact.cuh) --
//                  the reference's contract, src/mlxlearn/_kernels/radius_contract.py:129-217.
//   4. compact   : warp ballots + per-query offsets -> indptr / indices /
//                  distances sqrt(min(s, R2)), rows in ascending index order.
//   5. sort      : optional per-row (distance, index) order
//                  (src/mlxlearn/_kernels/radius_result.py:160-187).
// With grouped operand rows (reorder.cu) the screen yields operand rows:
// step 2b maps them to training rows, and rows are sorted by training index
// after step 4 when no distance order is asked for.
// Replaces the reference's Metal screen + host finisher
// (src/mlxlearn/_kernels/radius_metal_v1.py:257-611, src/mlxlearn_device/_radius.py:54-330).
#include <algorithm>
#include <cfloat>

#include "common.cuh"
#include "exact.cuh"
#include "internal.cuh"

namespace b2k {

namespace {

__global__ void radius_threshold_kernel(const double* __restrict__ nq, const float* __restrict__ E,
                                        int64_t m, int64_t m_pad, double R2,
                                        float* __restrict__ thr) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m_pad) return;
  if (r >= m) {
    thr[r] = -INFINITY;
    return;
  }
  if (isinf(R2)) {
    thr[r] = INFINITY;
    return;
  }
  // v <= R2 - nq + E  (float64 with upward rounding, then rounded up to fp32)
  const double t = __dadd_ru(__dadd_ru(R2, -nq[r]), (double)E[r]);
  thr[r] = __double2float_ru(t);
}

// Multi-block exclusive scan of int64 values (the radius path's offsets):
// each block scans a tile of kScanTile values (four per thread, warp
// shuffles, then the warp totals), writes the tile-local scan and the tile's
// total; one block scans the tile totals; a last pass adds each tile's base.
constexpr int kScanThreads = 1024;
constexpr int kScanTile = 4 * kScanThreads;

__device__ __forceinline__ int64_t warp_incl_scan(int64_t v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Exclusive scan of the block's kScanThreads values `v` (returned), the
// block total in *total_out (all threads).
__device__ __forceinline__ int64_t block_excl_scan(int64_t v, int64_t* warp_sums,
                                                   int64_t* total_out) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t incl = warp_incl_scan(v, lane);
  if (lane == 31) warp_sums[w] = incl;
  __syncthreads();
  if (w == 0) {
    const int64_t ws = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
    const int64_t wi = warp_incl_scan(ws, lane);
    warp_sums[lane] = wi - ws;  // exclusive
    if (lane == 31) warp_sums[32] = wi;
  }
  __syncthreads();
  const int64_t r = warp_sums[w] + incl - v;
  *total_out = warp_sums[32];
  __syncthreads();
  return r;
}

// Tile-local exclusive scan of in[0..n) into out, tile totals into part.
__global__ void __launch_bounds__(kScanThreads)
    scan_tiles_kernel(const int64_t* __restrict__ in, int64_t n, int64_t* __restrict__ out,
                      int64_t* __restrict__ part) {
  __shared__ int64_t warp_sums[33];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + 4 * (int64_t)threadIdx.x;
  int64_t x[4], sum = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    x[j] = base + j < n ? in[base + j] : 0;
    sum += x[j];
  }
  int64_t tile_total;
  int64_t acc = block_excl_scan(sum, warp_sums, &tile_total);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (base + j < n) out[base + j] = acc;
    acc += x[j];
  }
  if (threadIdx.x == 0) part[blockIdx.x] = tile_total;
}

// Exclusive scan of the nt tile totals in place (one block, any nt); the
// grand total into *total.
__global__ void __launch_bounds__(kScanThreads)
    scan_parts_kernel(int64_t* __restrict__ part, int64_t nt, int64_t* __restrict__ total) {
  __shared__ int64_t warp_sums[33];
  int64_t carry = 0;
  for (int64_t b0 = 0; b0 < nt; b0 += kScanThreads) {
    const int64_t i = b0 + threadIdx.x;
    const int64_t v = i < nt ? part[i] : 0;
    int64_t chunk;
    const int64_t e = block_excl_scan(v, warp_sums, &chunk);
    if (i < nt) part[i] = carry + e;
    carry += chunk;
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(kScanThreads)
    scan_add_kernel(int64_t* __restrict__ out, int64_t n, const int64_t* __restrict__ part) {
  const int64_t i = (int64_t)blockIdx.x * kScanThreads + threadIdx.x;
  if (i < n) out[i] += part[i / kScanTile];
}

// Per row: the total over its lists (a coalesced pass over rows).
__global__ void row_totals_kernel(const int* __restrict__ counts, int S, int64_t m,
                                  int64_t m_pad, int64_t* __restrict__ tot) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m) return;
  int64_t sum = 0;
  for (int s = 0; s < S; ++s) sum += counts[(size_t)s * m_pad + r];
  tot[r] = sum;
}

// Per (list, row) offsets in row-major (row, list) order from the row offsets.
__global__ void split_offsets_kernel(const int* __restrict__ counts, int S, int64_t m,
                                     int64_t m_pad, const int64_t* __restrict__ row_off,
                                     int64_t* __restrict__ off) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m) return;
  int64_t acc = row_off[r];
  for (int s = 0; s < S; ++s) {
    off[(size_t)s * m_pad + r] = acc;
    acc += counts[(size_t)s * m_pad + r];
  }
}

struct ClassifyArgs {
  const float* X;
  const float* Q;
  int d;
  int64_t m;
  int S;
  int64_t m_pad;
  const int64_t* roff;   // [S][m_pad] candidate offsets
  const int* rcount;     // [S][m_pad]
  const int* cols;       // candidates (training rows)
  double* cdist;         // [ncand]: distance of members, -1 for non-members
  int64_t* mcount;       // [m]
  double R2, f_in, f_out;
  int all;               // R2 = inf
  int r2_huge;           // R2 * 2^298 exceeds every key
  ExactKey r2key;        // floor(R2 * 2^298)
  unsigned long long* exact_tests;
  const int* status;     // nonzero: the fill pass gave up, its candidates are unfinished
};

// Warp-uniform: lane 0's read of the call's error word decides for the warp.
__device__ __forceinline__ bool call_failed(const int* status, int lane) {
  const int st = lane == 0 ? *reinterpret_cast<volatile const int*>(status) : 0;
  return __shfl_sync(0xffffffffu, st, 0) != DEV_OK;
}

__device__ __forceinline__ bool key_le(const ExactKey& a, const ExactKey& b) {
  return key_cmp(a, b) <= 0;
}

// One warp per query row.
// A row's candidates are contiguous across its lists (offsets in (row, list)
// order): [roff[row], roff[row] + its total).
__device__ __forceinline__ int64_t row_candidates(const ClassifyArgs& a, int64_t row,
                                                  int64_t* base) {
  *base = a.roff[row];
  int64_t total = 0;
  for (int s = 0; s < a.S; ++s) total += a.rcount[(size_t)s * a.m_pad + row];
  return total;
}

// Member distance sqrt(min(s, R2)) of candidate row x with canonical value
// sv, or -1 for a non-member; band cases take the exact key (counted).
__device__ __forceinline__ double classify_one(const ClassifyArgs& a, const float* q,
                                               const float* x, double sv, unsigned& exact) {
  if (a.all) return sqrt(sv);  // min(s, inf) = s
  bool in;
  if (sv <= a.f_in) in = true;
  else if (!(sv <= a.f_out)) in = false;
  else if (a.r2_huge) in = true;
  else {
    ExactKey k;
    exact_key(q, x, a.d, k);
    in = key_le(k, a.r2key);
    ++exact;
  }
  return in ? sqrt(sv < a.R2 ? sv : a.R2) : -1.0;
}

// Candidates [i0, total) of a row with step `stride`, two per thread at a
// time (i and i + stride, interleaved canonical chains); returns the members.
__device__ __forceinline__ int64_t classify_range(const ClassifyArgs& a, const float* q,
                                                  int64_t base, int64_t i0, int64_t total,
                                                  int stride, unsigned& exact) {
  int64_t members = 0;
  for (int64_t i = i0; i < total; i += 2 * (int64_t)stride) {
    const bool two = i + stride < total;
    const float* x0 = a.X + (size_t)a.cols[base + i] * a.d;
    const float* x1 = two ? a.X + (size_t)a.cols[base + i + stride] * a.d : x0;
    double s0, s1;
    canonical_d2_pair(q, x0, x1, a.d, s0, s1);
    const double d0 = classify_one(a, q, x0, s0, exact);
    a.cdist[base + i] = d0;
    members += d0 >= 0.0;
    if (two) {
      const double d1 = classify_one(a, q, x1, s1, exact);
      a.cdist[base + i + stride] = d1;
      members += d1 >= 0.0;
    }
  }
  return members;
}

// One warp per query row; each lane takes candidates i and i + 32 of every 64
// together (two interleaved canonical chains).
__global__ void classify_kernel(const ClassifyArgs a) {
  const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= a.m) return;
  if (call_failed(a.status, lane)) {  // no members: the host reports the error
    if (lane == 0) a.mcount[row] = 0;
    return;
  }
  const float* q = a.Q + (size_t)row * a.d;
  int64_t base;
  const int64_t total = row_candidates(a, row, &base);
  unsigned exact = 0;
  int64_t members = classify_range(a, q, base, lane, total, 32, exact);
  for (int o = 16; o; o >>= 1) {
    members += __shfl_xor_sync(0xffffffffu, members, o);
    exact += __shfl_xor_sync(0xffffffffu, exact, o);
  }
  if (lane == 0) {
    a.mcount[row] = members;
    if (exact) atomicAdd(a.exact_tests, (unsigned long long)exact);
  }
}

// One warp per query row: order-preserving compaction of the members.
__global__ void compact_kernel(const ClassifyArgs a, const int64_t* __restrict__ indptr,
                               int64_t* __restrict__ indices, double* __restrict__ dist) {
  const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= a.m || call_failed(a.status, lane)) return;
  int64_t base;
  const int64_t total = row_candidates(a, row, &base);
  int64_t out = indptr[row];
  for (int64_t i0 = 0; i0 < total; i0 += 32) {
    const int64_t i = i0 + lane;
    double dv = -1.0;
    int col = 0;
    if (i < total) {
      dv = a.cdist[base + i];
      col = a.cols[base + i];
    }
    const bool keep = dv >= 0.0;
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    if (keep) {
      const int64_t pos = out + __popc(bal & ((1u << lane) - 1));
      indices[pos] = col;
      if (dist) dist[pos] = dv;
    }
    out += __popc(bal);
  }
}

// Long rows (the overflow sub-call's rows hold thousands of candidates):
// one CTA per row, so a few rows still spread over the whole GPU.
constexpr int kWideThreads = 256;

// The call's error word, read once by thread 0 and shared with the block.
__device__ __forceinline__ bool block_failed(const int* status, int* s_flag) {
  if (threadIdx.x == 0) *s_flag = *reinterpret_cast<volatile const int*>(status);
  __syncthreads();
  return *s_flag != DEV_OK;
}

__global__ void __launch_bounds__(kWideThreads) classify_wide_kernel(const ClassifyArgs a) {
  __shared__ int s_flag;
  __shared__ long long s_members[kWideThreads / 32];
  __shared__ unsigned s_exact[kWideThreads / 32];
  const int64_t row = blockIdx.x;  // grid = m: every thread of the block has a row
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (block_failed(a.status, &s_flag)) {
    if (threadIdx.x == 0) a.mcount[row] = 0;
    return;
  }
  const float* q = a.Q + (size_t)row * a.d;
  int64_t base;
  const int64_t total = row_candidates(a, row, &base);
  unsigned exact = 0;
  int64_t members = classify_range(a, q, base, threadIdx.x, total, kWideThreads, exact);
  for (int o = 16; o; o >>= 1) {
    members += __shfl_xor_sync(0xffffffffu, members, o);
    exact += __shfl_xor_sync(0xffffffffu, exact, o);
  }
  if (lane == 0) {
    s_members[w] = members;
    s_exact[w] = exact;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    long long mm = 0;
    unsigned ee = 0;
    for (int i = 0; i < kWideThreads / 32; ++i) {
      mm += s_members[i];
      ee += s_exact[i];
    }
    a.mcount[row] = mm;
    if (ee) atomicAdd(a.exact_tests, (unsigned long long)ee);
  }
}

// One CTA per row, order preserved: warp w compacts the w-th contiguous chunk
// of the row's candidates at the members counted before it.
__global__ void __launch_bounds__(kWideThreads)
    compact_wide_kernel(const ClassifyArgs a, const int64_t* __restrict__ indptr,
                        int64_t* __restrict__ indices, double* __restrict__ dist) {
  constexpr int kWarps = kWideThreads / 32;
  __shared__ int s_flag;
  __shared__ long long s_cnt[kWarps];
  const int64_t row = blockIdx.x;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (block_failed(a.status, &s_flag)) return;
  int64_t base;
  const int64_t total = row_candidates(a, row, &base);
  const int64_t chunk = ((total + kWarps - 1) / kWarps + 31) / 32 * 32;
  const int64_t lo = min(total, w * chunk), hi = min(total, lo + chunk);
  long long cnt = 0;
  for (int64_t i0 = lo; i0 < hi; i0 += 32) {
    const int64_t i = i0 + lane;
    cnt += __popc(__ballot_sync(0xffffffffu, i < hi && a.cdist[base + i] >= 0.0));
  }
  if (lane == 0) s_cnt[w] = cnt;
  __syncthreads();
  int64_t out = indptr[row];
  for (int i = 0; i < w; ++i) out += s_cnt[i];
  for (int64_t i0 = lo; i0 < hi; i0 += 32) {
    const int64_t i = i0 + lane;
    double dv = -1.0;
    int col = 0;
    if (i < hi) {
      dv = a.cdist[base + i];
      col = a.cols[base + i];
    }
    const bool keep = dv >= 0.0;
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    if (keep) {
      const int64_t pos = out + __popc(bal & ((1u << lane) - 1));
      indices[pos] = col;
      if (dist) dist[pos] = dv;
    }
    out += __popc(bal);
  }
}

// Candidates already at their offsets to training rows, in place, one thread
// per entry (the counted form's fill pass on grouped operand rows).
__global__ void translate_kernel(int* cand, int64_t count, const int* __restrict__ xperm,
                                 const int* __restrict__ status) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (*reinterpret_cast<volatile const int*>(status) != DEV_OK) return;
  if (i < count) cand[i] = __ldg(xperm + cand[i]);
}

// One thread per row: a row whose count passed the list capacity in any of
// its lists lost candidates; list it for the counted sub-call and zero its
// counts (classify then gives it no members and compact writes nothing).
__global__ void radius_overflow_kernel(int* __restrict__ rcount, int S, int64_t m, int64_t m_pad,
                                       int cap, int* __restrict__ rows) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m) return;
  bool over = false;
  for (int s = 0; s < S; ++s) over |= rcount[(size_t)s * m_pad + r] > cap;
  if (!over) return;
  for (int s = 0; s < S; ++s) rcount[(size_t)s * m_pad + r] = 0;
  rows[atomicAdd(rows + m, 1)] = (int)r;
}

// One warp per row: the candidates of the row's S lists to their scanned
// offsets, as training rows.  src holds lists of `cap` entries at slot * cap,
// or (cap = 0) the candidates already at their offsets, translated in place
// (each entry is read and written by the same lane).
__global__ void radius_pack_kernel(const int* src, int cap, const int* __restrict__ rcount,
                                   int S, int64_t m, int64_t m_pad,
                                   const int64_t* __restrict__ roff,
                                   const int* __restrict__ xperm, int* dst,
                                   const int* __restrict__ status) {
  const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= m || call_failed(status, lane)) return;
  for (int s = 0; s < S; ++s) {
    const size_t slot = (size_t)s * m_pad + row;
    const int cnt = rcount[slot];
    const int64_t o = roff[slot];
    const int* in = cap ? src + slot * (size_t)cap : src + o;
    for (int i = lane; i < cnt; i += 32) {
      const int c = in[i];
      dst[o + i] = xperm ? __ldg(xperm + c) : c;
    }
  }
}

__global__ void radius_sub_counts_kernel(const int* __restrict__ rows, int count,
                                         const int64_t* __restrict__ sub_indptr,
                                         int64_t* __restrict__ mcount) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) mcount[rows[i]] = sub_indptr[i + 1] - sub_indptr[i];
}

// One warp per sub-call row.
__global__ void radius_sub_scatter_kernel(const int* __restrict__ rows, int count,
                                          const int64_t* __restrict__ sub_indptr,
                                          const int64_t* __restrict__ sub_indices,
                                          const double* __restrict__ sub_dist,
                                          const int64_t* __restrict__ indptr,
                                          int64_t* __restrict__ indices,
                                          double* __restrict__ dist) {
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= count) return;
  const int64_t b = sub_indptr[w], e = sub_indptr[w + 1], o = indptr[rows[w]] - b;
  for (int64_t i = b + lane; i < e; i += 32) {
    indices[o + i] = sub_indices[i];
    if (dist) dist[o + i] = sub_dist[i];
  }
}

// Sort order of the per-row sorts: (distance, index), or index alone.
template <bool BY_DIST>
__device__ __forceinline__ bool sort_after(double x, int64_t xi, double y, int64_t yi) {
  if constexpr (BY_DIST) return (x > y) || (x == y && xi > yi);
  return xi > yi;
}

// Per-row sorts; `dist` may be null for an index sort.  Rows of at most
// kWarpSortCap entries: one warp each, bitonic in the warp's shared memory;
// longer rows go to a list for one CTA each (at most kRadiusSortCap entries),
// and longer still to the global-memory sort.
constexpr int kWarpSortCap = 256;
constexpr int kWarpSortWarps = 8;
constexpr int kRadiusSortCap = 4096;
constexpr int kSortThreads = 512;

// Index-order sorts move one 64-bit key per entry, (training index << 16) |
// position in the row: training indices are distinct within a row and below
// 2^31, positions below kRadiusSortCap <= 2^16, so the keys are distinct and
// ascend with the index; the distances follow by position afterwards.
constexpr int kKeyPosBits = 16;
static_assert(kRadiusSortCap <= (1 << kKeyPosBits), "row positions fit the key");
__device__ __forceinline__ int64_t index_key(int64_t idx, int pos) {
  return (idx << kKeyPosBits) | pos;
}

template <bool BY_DIST>
__global__ void __launch_bounds__(kWarpSortWarps * 32)
    sort_rows_warp_kernel(const int64_t* __restrict__ indptr, int64_t m,
                          int64_t* __restrict__ indices, double* __restrict__ dist,
                          int* __restrict__ mid_rows, int* __restrict__ mid_count) {
  __shared__ double sd_all[kWarpSortWarps][kWarpSortCap];
  __shared__ int64_t si_all[kWarpSortWarps][kWarpSortCap];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* sd = sd_all[w];
  int64_t* si = si_all[w];
  const int64_t warps = (int64_t)gridDim.x * kWarpSortWarps;
  for (int64_t row = (int64_t)blockIdx.x * kWarpSortWarps + w; row < m; row += warps) {
    const int64_t a0 = indptr[row], len = indptr[row + 1] - a0;
    if (len <= 1) continue;
    if (len > kWarpSortCap) {
      if (lane == 0) mid_rows[atomicAdd(mid_count, 1)] = (int)row;
      continue;
    }
    int P = 2;
    while (P < len) P <<= 1;
    if constexpr (BY_DIST) {
      for (int i = lane; i < P; i += 32) {
        sd[i] = (i < len && dist) ? dist[a0 + i] : DBL_MAX;
        si[i] = i < len ? indices[a0 + i] : INT64_MAX;
      }
      __syncwarp();
      for (int size = 2; size <= P; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
          for (int t = lane; t < P / 2; t += 32) {
            const int i = 2 * t - (t & (stride - 1)), j = i + stride;
            const bool up = (i & size) == 0;
            const double x = sd[i], y = sd[j];
            const int64_t xi = si[i], yi = si[j];
            if (sort_after<BY_DIST>(x, xi, y, yi) == up) {
              sd[i] = y;
              sd[j] = x;
              si[i] = yi;
              si[j] = xi;
            }
          }
          __syncwarp();
        }
      for (int i = lane; i < len; i += 32) {
        if (dist) dist[a0 + i] = sd[i];
        indices[a0 + i] = si[i];
      }
    } else {
      // index order: one key per entry, the distance gathered by position
      for (int i = lane; i < P; i += 32) {
        if (i < len && dist) sd[i] = dist[a0 + i];
        si[i] = i < len ? index_key(indices[a0 + i], i) : INT64_MAX;
      }
      __syncwarp();
      for (int size = 2; size <= P; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
          for (int t = lane; t < P / 2; t += 32) {
            const int i = 2 * t - (t & (stride - 1)), j = i + stride;
            const int64_t x = si[i], y = si[j];
            if ((x > y) == ((i & size) == 0)) {
              si[i] = y;
              si[j] = x;
            }
          }
          __syncwarp();
        }
      for (int i = lane; i < len; i += 32) {
        const int64_t key = si[i];
        indices[a0 + i] = key >> kKeyPosBits;
        if (dist) dist[a0 + i] = sd[key & ((1 << kKeyPosBits) - 1)];
      }
    }
    __syncwarp();
  }
}

// Rows listed by the warp sort: one CTA per row.
template <bool BY_DIST>
__global__ void sort_rows_kernel(const int64_t* __restrict__ indptr,
                                 const int* __restrict__ rows, const int* __restrict__ row_count,
                                 int64_t* __restrict__ indices, double* __restrict__ dist,
                                 int* __restrict__ big_rows, int* __restrict__ big_count) {
  extern __shared__ uint8_t smem[];
  double* sd = reinterpret_cast<double*>(smem);
  int64_t* si = reinterpret_cast<int64_t*>(sd + kRadiusSortCap);
  const int count = *row_count;
  for (int it = blockIdx.x; it < count; it += gridDim.x) {
    const int64_t row = rows[it];
    const int64_t a0 = indptr[row], len = indptr[row + 1] - a0;
    if (len > kRadiusSortCap) {
      if (threadIdx.x == 0) big_rows[atomicAdd(big_count, 1)] = (int)row;
      continue;
    }
    int P = 2;
    while (P < len) P <<= 1;
    if constexpr (BY_DIST) {
      for (int i = threadIdx.x; i < P; i += blockDim.x) {
        sd[i] = (i < len && dist) ? dist[a0 + i] : DBL_MAX;
        si[i] = i < len ? indices[a0 + i] : INT64_MAX;
      }
      __syncthreads();
      for (int size = 2; size <= P; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
          for (int t = threadIdx.x; t < P / 2; t += blockDim.x) {
            const int i = 2 * t - (t & (stride - 1)), j = i + stride;
            const bool up = (i & size) == 0;
            const double x = sd[i], y = sd[j];
            const int64_t xi = si[i], yi = si[j];
            const bool gt = sort_after<BY_DIST>(x, xi, y, yi);
            if (gt == up) {
              sd[i] = y;
              sd[j] = x;
              si[i] = yi;
              si[j] = xi;
            }
          }
          __syncthreads();
        }
      for (int i = threadIdx.x; i < len; i += blockDim.x) {
        if (dist) dist[a0 + i] = sd[i];
        indices[a0 + i] = si[i];
      }
    } else {
      // index order: one key per entry, the distance gathered by position
      for (int i = threadIdx.x; i < P; i += blockDim.x) {
        if (i < len && dist) sd[i] = dist[a0 + i];
        si[i] = i < len ? index_key(indices[a0 + i], i) : INT64_MAX;
      }
      __syncthreads();
      for (int size = 2; size <= P; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
          for (int t = threadIdx.x; t < P / 2; t += blockDim.x) {
            const int i = 2 * t - (t & (stride - 1)), j = i + stride;
            const int64_t x = si[i], y = si[j];
            if ((x > y) == ((i & size) == 0)) {
              si[i] = y;
              si[j] = x;
            }
          }
          __syncthreads();
        }
      for (int i = threadIdx.x; i < len; i += blockDim.x) {
        const int64_t key = si[i];
        indices[a0 + i] = key >> kKeyPosBits;
        if (dist) dist[a0 + i] = sd[key & ((1 << kKeyPosBits) - 1)];
      }
    }
    __syncthreads();
  }
}

// Rows longer than the shared-memory sort: bitonic sort in global scratch
// (padded to a power of two), one CTA per row.
template <bool BY_DIST>
__global__ void sort_big_rows_kernel(const int64_t* __restrict__ indptr,
                                     const int* __restrict__ rows, int count,
                                     int64_t* __restrict__ indices, double* __restrict__ dist,
                                     double* __restrict__ tmp_d, int64_t* __restrict__ tmp_i,
                                     int64_t tmp_stride) {
  for (int it = blockIdx.x; it < count; it += gridDim.x) {
    const int64_t row = rows[it];
    const int64_t a0 = indptr[row], len = indptr[row + 1] - a0;
    int64_t P = 2;
    while (P < len) P <<= 1;
    double* sd = tmp_d + (size_t)blockIdx.x * tmp_stride;
    int64_t* si = tmp_i + (size_t)blockIdx.x * tmp_stride;
    for (int64_t i = threadIdx.x; i < P; i += blockDim.x) {
      sd[i] = (i < len && dist) ? dist[a0 + i] : DBL_MAX;
      si[i] = i < len ? indices[a0 + i] : INT64_MAX;
    }
    __syncthreads();
    for (int64_t size = 2; size <= P; size <<= 1)
      for (int64_t stride = size >> 1; stride > 0; stride >>= 1) {
        for (int64_t t = threadIdx.x; t < P / 2; t += blockDim.x) {
          const int64_t i = 2 * t - (t & (stride - 1)), j = i + stride;
          const bool up = (i & size) == 0;
          const double x = sd[i], y = sd[j];
          const int64_t xi = si[i], yi = si[j];
          const bool gt = sort_after<BY_DIST>(x, xi, y, yi);
          if (gt == up) {
            sd[i] = y;
            sd[j] = x;
            si[i] = yi;
            si[j] = xi;
          }
        }
        __syncthreads();
      }
    for (int64_t i = threadIdx.x; i < len; i += blockDim.x) {
      if (dist) dist[a0 + i] = sd[i];
      indices[a0 + i] = si[i];
    }
    __syncthreads();
  }
}

}  // namespace

// ------------------------------------------------------------ host launchers

void launch_radius_threshold(const double* nq, const float* E, int64_t m, int64_t m_pad,
                             double R2, float* thr, cudaStream_t st) {
  if (m_pad <= 0) return;
  radius_threshold_kernel<<<(unsigned)((m_pad + 255) / 256), 256, 0, st>>>(nq, E, m, m_pad, R2,
                                                                            thr);
}

int64_t scan_scratch_len(int64_t n) { return 2 * n + (n + kScanTile - 1) / kScanTile + 2; }

void launch_exclusive_scan(const int64_t* in, int64_t n, int64_t* out, int64_t* total,
                           int64_t* part, cudaStream_t st) {
  if (n <= 0) {
    cudaMemsetAsync(total, 0, sizeof(int64_t), st);
    return;
  }
  const int64_t nt = (n + kScanTile - 1) / kScanTile;
  scan_tiles_kernel<<<(unsigned)nt, kScanThreads, 0, st>>>(in, n, out, part);
  scan_parts_kernel<<<1, kScanThreads, 0, st>>>(part, nt, total);
  if (nt > 1)
    scan_add_kernel<<<(unsigned)((n + kScanThreads - 1) / kScanThreads), kScanThreads, 0, st>>>(
        out, n, part);
}

void launch_scan_split_counts(const int* counts, int S, int64_t m, int64_t m_pad, int64_t* off,
                              int64_t* total, int64_t* scratch, cudaStream_t st) {
  if (m <= 0) {
    cudaMemsetAsync(total, 0, sizeof(int64_t), st);
    return;
  }
  int64_t* tot = scratch;           // [m] row totals
  int64_t* row_off = scratch + m;   // [m] row offsets
  int64_t* part = scratch + 2 * m;  // tile totals
  const unsigned blocks = (unsigned)((m + 255) / 256);
  row_totals_kernel<<<blocks, 256, 0, st>>>(counts, S, m, m_pad, tot);
  launch_exclusive_scan(tot, m, row_off, total, part, st);
  split_offsets_kernel<<<blocks, 256, 0, st>>>(counts, S, m, m_pad, row_off, off);
}

void launch_scan_rows(const int64_t* counts, int64_t m, int64_t* indptr, int64_t* scratch,
                      cudaStream_t st) {
  launch_exclusive_scan(counts, m, indptr, indptr + m, scratch, st);
}

// Thresholds of the float64 band (radius_contract.py:129-153) and the exact
// key of R2.
static double down(double v) { return nextafter(v, -INFINITY); }
static double up(double v) { return nextafter(v, INFINITY); }

void radius_band(int d, double R2, double* f_in, double* f_out, int* all, int* r2_huge,
                 uint64_t* key10) {
  *all = std::isinf(R2) ? 1 : 0;
  *r2_huge = 0;
  for (int i = 0; i < 10; ++i) key10[i] = 0;
  if (*all) {
    *f_in = *f_out = INFINITY;
    return;
  }
  const double u = ldexp(1.0, -53);
  const double g = (double)(d + 2) * u / (1.0 - (double)(d + 2) * u);
  if (R2 == 0.0) {
    *f_in = *f_out = 0.0;
  } else {
    const double fin = down(down(R2 * down(1.0 - 2.0 * g)));
    *f_in = fin > 0.0 ? fin : 0.0;
    *f_out = up(up(R2 * up(1.0 + 2.0 * g)));
  }
  // floor(R2 * 2^298), R2 = M * 2^E
  int e2;
  const double fr = frexp(R2, &e2);
  const uint64_t M = (uint64_t)ldexp(fr, 53);
  const int shift = e2 - 53 + 298;
  if (shift >= 0) {
    if (shift + 53 > 639) {
      *r2_huge = 1;
      return;
    }
    const int limb = shift >> 6, bit = shift & 63;
    key10[limb] = M << bit;
    if (bit && limb + 1 < 10) key10[limb + 1] = M >> (64 - bit);
  } else if (-shift < 64) {
    key10[0] = M >> (-shift);
  }
}

void launch_classify(const RadiusPlanArgs& r, cudaStream_t st) {
  ClassifyArgs a{};
  a.X = r.X;
  a.Q = r.Q;
  a.d = r.d;
  a.m = r.m;
  a.S = r.S;
  a.m_pad = r.m_pad;
  a.roff = r.roff;
  a.rcount = r.rcount;
  a.cols = r.cols;
  a.cdist = r.cdist;
  a.mcount = r.mcount;
  a.R2 = r.R2;
  a.exact_tests = r.exact_tests;
  a.status = r.status;
  radius_band(r.d, r.R2, &a.f_in, &a.f_out, &a.all, &a.r2_huge, a.r2key.w);
  if (r.m <= 0) return;
  if (r.wide) {
    classify_wide_kernel<<<(unsigned)r.m, kWideThreads, 0, st>>>(a);
    return;
  }
  const int warps = 8;
  classify_kernel<<<(unsigned)((r.m + warps - 1) / warps), warps * 32, 0, st>>>(a);
}

void launch_compact(const RadiusPlanArgs& r, const int64_t* indptr, int64_t* indices,
                    double* dist, cudaStream_t st) {
  ClassifyArgs a{};
  a.m = r.m;
  a.S = r.S;
  a.m_pad = r.m_pad;
  a.roff = r.roff;
  a.rcount = r.rcount;
  a.cols = r.cols;
  a.cdist = r.cdist;
  a.status = r.status;
  if (r.m <= 0) return;
  if (r.wide) {
    compact_wide_kernel<<<(unsigned)r.m, kWideThreads, 0, st>>>(a, indptr, indices, dist);
    return;
  }
  const int warps = 8;
  compact_kernel<<<(unsigned)((r.m + warps - 1) / warps), warps * 32, 0, st>>>(a, indptr,
                                                                                 indices, dist);
}

void launch_radius_overflow(int* rcount, int S, int64_t m, int64_t m_pad, int cap, int* rows,
                            cudaStream_t st) {
  if (m <= 0) return;
  radius_overflow_kernel<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(rcount, S, m, m_pad, cap,
                                                                      rows);
}

void launch_radius_pack(const int* src, int cap, const int* rcount, int S, int64_t m,
                        int64_t m_pad, const int64_t* roff, const int* xperm, int* dst,
                        int64_t count, const int* status, cudaStream_t st) {
  if (m <= 0) return;
  if (cap == 0) {  // in place: one thread per entry
    if (src != dst || !xperm) return;
    if (count > 0)
      translate_kernel<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(dst, count, xperm,
                                                                         status);
    return;
  }
  radius_pack_kernel<<<(unsigned)((m + 7) / 8), 256, 0, st>>>(src, cap, rcount, S, m, m_pad,
                                                             roff, xperm, dst, status);
}

void launch_radius_sub_counts(const int* rows, int count, const int64_t* sub_indptr,
                              int64_t* mcount, cudaStream_t st) {
  if (count <= 0) return;
  radius_sub_counts_kernel<<<(count + 255) / 256, 256, 0, st>>>(rows, count, sub_indptr, mcount);
}

void launch_radius_sub_scatter(const int* rows, int count, const int64_t* sub_indptr,
                               const int64_t* sub_indices, const double* sub_dist,
                               const int64_t* indptr, int64_t* indices, double* dist,
                               cudaStream_t st) {
  if (count <= 0) return;
  radius_sub_scatter_kernel<<<(unsigned)((count + 7) / 8), 256, 0, st>>>(
      rows, count, sub_indptr, sub_indices, sub_dist, indptr, indices, dist);
}

void launch_sort_rows(const int64_t* indptr, int64_t m, int64_t* indices, double* dist,
                      int* mid_rows, int* mid_count, int* big_rows, int* big_count, int grid,
                      cudaStream_t st, bool by_dist) {
  if (m <= 0) return;
  const unsigned wgrid = (unsigned)std::min<int64_t>((m + kWarpSortWarps - 1) / kWarpSortWarps,
                                                     (int64_t)grid * 4);
  if (by_dist)
    sort_rows_warp_kernel<true><<<wgrid, kWarpSortWarps * 32, 0, st>>>(indptr, m, indices, dist,
                                                                        mid_rows, mid_count);
  else
    sort_rows_warp_kernel<false><<<wgrid, kWarpSortWarps * 32, 0, st>>>(indptr, m, indices,
                                                                         dist, mid_rows,
                                                                         mid_count);
  const size_t smem = (size_t)kRadiusSortCap * (sizeof(double) + sizeof(int64_t));
  auto kern = by_dist ? sort_rows_kernel<true> : sort_rows_kernel<false>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<grid, kSortThreads, smem, st>>>(indptr, mid_rows, mid_count, indices, dist, big_rows,
                                         big_count);
}

void launch_sort_big_rows(const int64_t* indptr, const int* rows, int count, int64_t* indices,
                          double* dist, double* tmp_d, int64_t* tmp_i, int64_t tmp_stride,
                          int grid, cudaStream_t st, bool by_dist) {
  if (count <= 0) return;
  auto kern = by_dist ? sort_big_rows_kernel<true> : sort_big_rows_kernel<false>;
  kern<<<grid, 1024, 0, st>>>(indptr, rows, count, indices, dist, tmp_d, tmp_i, tmp_stride);
}

int radius_sort_cap() { return kRadiusSortCap; }

}  // namespace b2k
