// Query ordering (and index row grouping) for the screens.
//
// A screen tile holds 128 query rows and each epilogue warp 32 of them; the
// warp leaves its fast path whenever ANY of its rows admits a column.  With
// queries in arbitrary order the rows of a warp come from unrelated parts of
// the space and the admissions of the different rows hit different column
// chunks, so nearly every chunk takes the slow path.  Grouping queries that
// are close to each other makes their admissions coincide.
//
// Method: P pivots (every (n/P)-th training row), each query goes to its
// nearest pivot (fp32 Gram form, the assignment only affects speed), then a
// counting sort by pivot gives the permutation `perm` (sorted position ->
// original query row) and the permuted query matrix.  Results are written
// back to the original rows by the certify / exact kernels, so the answer
// does not depend on the order.
//
// The same assignment groups the rows of the index's bf16 operand by pivot
// (b200knn.cu): a tile of grouped queries then finds its candidates in a few
// consecutive reference tiles, and the other tiles' chunks skip admission.
#include "common.cuh"
#include "internal.cuh"

namespace b2k {

namespace {

constexpr int kPivTile = 32;     // pivots per shared-memory tile
constexpr int kDChunk = 64;      // features per shared-memory chunk
constexpr int kAssignThreads = 128;

__global__ void pivot_rows_kernel(const float* __restrict__ X, int64_t n, int d, int P,
                                  const float* __restrict__ center, float* __restrict__ piv,
                                  float* __restrict__ pnorm) {
  const int p = blockIdx.x;
  if (p >= P) return;
  const int64_t row = (int64_t)p * (n / P);
  double s = 0.0;
  for (int i = threadIdx.x; i < d; i += 32) {
    const float y = X[row * d + i] - center[i];
    piv[(size_t)p * d + i] = y;
    s += (double)y * (double)y;
  }
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) pnorm[p] = (float)s;
}

// 128 queries per block: argmin_p ||p||^2 - 2 <y_q, p>.  Per 32-pivot tile
// warp w takes pivots [8w, 8w + 8) and lane l the queries l, l + 32, l + 64,
// l + 96, so each feature step is 6 shared-memory loads (4 query values, two
// 16-byte pivot loads) for 32 FMAs.  Each (query, pivot) sum runs over the
// features in order, and ties go to the smaller pivot, so the keys do not
// depend on this layout.
__global__ void __launch_bounds__(kAssignThreads)
    assign_kernel(const float* __restrict__ Q, int64_t m, int d, const float* __restrict__ center,
                  const float* __restrict__ piv, const float* __restrict__ pnorm, int P,
                  int* __restrict__ key, int* __restrict__ hist) {
  __shared__ __align__(16) float sp[kDChunk][kPivTile];  // pivot tile, transposed
  __shared__ float sq[kDChunk][kAssignThreads + 1];       // query tile, transposed
  __shared__ float red_v[4][kAssignThreads];
  __shared__ int red_p[4][kAssignThreads];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t q0 = (int64_t)blockIdx.x * kAssignThreads;
  float best[4];
  int best_p[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    best[i] = INFINITY;
    best_p[i] = 0;
  }
  for (int p0 = 0; p0 < P; p0 += kPivTile) {
    float acc[4][8];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;
    for (int k0 = 0; k0 < d; k0 += kDChunk) {
      __syncthreads();
      for (int i = threadIdx.x; i < kPivTile * kDChunk; i += kAssignThreads) {
        const int j = i % kPivTile, k = i / kPivTile;
        sp[k][j] = (p0 + j < P && k0 + k < d) ? piv[(size_t)(p0 + j) * d + k0 + k] : 0.0f;
      }
      // coalesced: consecutive threads read consecutive features of one query
      for (int i = threadIdx.x; i < kAssignThreads * kDChunk; i += kAssignThreads) {
        const int r = i / kDChunk, k = i % kDChunk;
        const int64_t qr = q0 + r;
        sq[k][r] = (qr < m && k0 + k < d) ? Q[qr * d + k0 + k] - center[k0 + k] : 0.0f;
      }
      __syncthreads();
      const int kend = min(kDChunk, d - k0);
      for (int k = 0; k < kend; ++k) {
        const float4 pa = *reinterpret_cast<const float4*>(&sp[k][8 * w]);
        const float4 pb = *reinterpret_cast<const float4*>(&sp[k][8 * w + 4]);
        const float pv[8] = {pa.x, pa.y, pa.z, pa.w, pb.x, pb.y, pb.z, pb.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const float y = sq[k][lane + 32 * i];
#pragma unroll
          for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(y, pv[j], acc[i][j]);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int pj = p0 + 8 * w + j;
      if (pj < P) {
        const float pn = pnorm[pj];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const float v = fmaf(-2.0f, acc[i][j], pn);
          if (v < best[i]) {
            best[i] = v;
            best_p[i] = pj;
          }
        }
      }
    }
  }
  // each warp's best per query, then the smallest (value, pivot) over warps
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    red_v[w][lane + 32 * i] = best[i];
    red_p[w][lane + 32 * i] = best_p[i];
  }
  __syncthreads();
  const int64_t q = q0 + threadIdx.x;
  if (q < m) {
    float bv = red_v[0][threadIdx.x];
    int bp = red_p[0][threadIdx.x];
    for (int ww = 1; ww < 4; ++ww) {
      const float v = red_v[ww][threadIdx.x];
      const int pp = red_p[ww][threadIdx.x];
      if (v < bv || (v == bv && pp < bp)) {
        bv = v;
        bp = pp;
      }
    }
    key[q] = bp;
    atomicAdd(hist + bp, 1);
  }
}

__global__ void bin_scan_kernel(int* __restrict__ hist, int P) {
  // exclusive scan in place (P small), single thread
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int acc = 0;
    for (int p = 0; p < P; ++p) {
      const int v = hist[p];
      hist[p] = acc;
      acc += v;
    }
  }
}

__global__ void scatter_kernel(const int* __restrict__ key, int64_t m, int* __restrict__ cursor,
                               int* __restrict__ perm) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= m) return;
  perm[atomicAdd(cursor + key[q], 1)] = (int)q;
}

__global__ void gather_rows_kernel(const float* __restrict__ Q, const int* __restrict__ perm,
                                   int64_t m, int d, float* __restrict__ Qp) {
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (row >= m) return;
  const float* src = Q + (size_t)perm[row] * d;
  float* dst = Qp + (size_t)row * d;
  for (int i = threadIdx.x & 31; i < d; i += 32) dst[i] = src[i];
}

// Rows the certify pass could not finish, for a second pass: their query
// rows (in the pass's row order) and their output rows.
__global__ void gather_fallback_kernel(const float* __restrict__ Qs, int d,
                                       const int* __restrict__ rows,
                                       const int* __restrict__ perm, int count,
                                       float* __restrict__ Qout, int* __restrict__ pout) {
  const int64_t i = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (i >= count) return;
  const int r = rows[i];
  const float* src = Qs + (size_t)r * d;
  float* dst = Qout + (size_t)i * d;
  for (int c = threadIdx.x & 31; c < d; c += 32) dst[c] = src[c];
  if ((threadIdx.x & 31) == 0) pout[i] = perm ? perm[r] : r;
}

__global__ void home_tiles_kernel(const int* __restrict__ perm, const int* __restrict__ key,
                                  int64_t m, const int* __restrict__ group_start, int n_tiles,
                                  int window, int* __restrict__ home, int m_tiles) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m_tiles) return;
  const int64_t mid = min((int64_t)t * kTcBM + kTcBM / 2, m - 1);
  const int row = group_start[key[perm[mid]]];
  // one tile of margin before the group; the window stays inside the index
  int j0 = row / kTcBN - 1;
  j0 = min(j0, n_tiles - window);
  home[t] = max(j0, 0);
}

}  // namespace

void launch_home_tiles(const int* perm, const int* key, int64_t m, const int* group_start,
                       int n_tiles, int window, int* home, int m_tiles, cudaStream_t st) {
  if (m_tiles <= 0 || m <= 0) return;
  home_tiles_kernel<<<(unsigned)((m_tiles + 127) / 128), 128, 0, st>>>(
      perm, key, m, group_start, n_tiles, window, home, m_tiles);
}

void launch_gather_fallback(const float* Qs, int d, const int* rows, const int* perm, int count,
                            float* Qout, int* pout, cudaStream_t st) {
  if (count <= 0) return;
  gather_fallback_kernel<<<(unsigned)((count + 7) / 8), 256, 0, st>>>(Qs, d, rows, perm, count,
                                                                      Qout, pout);
}

int pivot_count(int64_t n) {
  int P = 512;
  while (P > 1 && (int64_t)P * 64 > n) P >>= 1;
  return P;
}

void launch_pivots(Index* ix, cudaStream_t st) {
  pivot_rows_kernel<<<ix->n_pivots, 32, 0, st>>>(ix->X, ix->n, ix->d, ix->n_pivots, ix->center,
                                                 ix->pivots, ix->pivot_norms);
}

void launch_assign_rows(const Index* ix, const float* X, int64_t n, int* key, int* hist,
                        cudaStream_t st) {
  cudaMemsetAsync(hist, 0, (size_t)ix->n_pivots * sizeof(int), st);
  assign_kernel<<<(unsigned)((n + kAssignThreads - 1) / kAssignThreads), kAssignThreads, 0, st>>>(
      X, n, ix->d, ix->center, ix->pivots, ix->pivot_norms, ix->n_pivots, key, hist);
}

void launch_query_order(const Index* ix, const float* Q, int64_t m, int* key, int* hist,
                        int* perm, float* Qp, cudaStream_t st) {
  const int P = ix->n_pivots;
  cudaMemsetAsync(hist, 0, (size_t)P * sizeof(int), st);
  assign_kernel<<<(unsigned)((m + kAssignThreads - 1) / kAssignThreads), kAssignThreads, 0, st>>>(
      Q, m, ix->d, ix->center, ix->pivots, ix->pivot_norms, P, key, hist);
  bin_scan_kernel<<<1, 32, 0, st>>>(hist, P);
  scatter_kernel<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(key, m, hist, perm);
  gather_rows_kernel<<<(unsigned)((m + 7) / 8), 256, 0, st>>>(Q, perm, m, ix->d, Qp);
}

}  // namespace b2k
