// Backward of selected kNN distances (b2k_knn_backward).
//
// Forward (elsewhere): indices idx[m, k] are fixed by the exact search; the
// differentiable outputs are the selected distances
//   squared:    s_ij = ||q_i - x_idx(i,j)||^2
//   euclidean:  e_ij = sqrt(s_ij)
// Given upstream gradients G[m, k]:
//   dQ_i   = sum_j c_ij (q_i - x_idx(i,j)),      c = 2 G (squared) or G / e (euclidean, 0 at e = 0)
//   dX_r   = sum_{(i,j): idx(i,j) = r} c_ij (x_r - q_i)
// dQ is a per-row reduction.  dX is a scatter-add made deterministic without
// float atomics: the (i, j) pairs are bucketed by reference row with a
// counting sort, each bucket is put in ascending flat order i*k + j, and every
// bucket is summed by one warp in that order.  Results are bitwise identical
// from run to run.
//
// The reference has no differentiable kNN; this is the building block for
// point-set losses such as a Chamfer term.
#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.cuh"

namespace b2k {

namespace {

__device__ __forceinline__ float coef_of(float g, float e, int squared) {
  if (squared) return 2.0f * g;
  return e > 0.0f ? g / e : 0.0f;
}

// One warp per query row; lanes over features.
__global__ void grad_q_kernel(const float* __restrict__ Q, const float* __restrict__ X,
                              const int64_t* __restrict__ idx, const float* __restrict__ G,
                              const float* __restrict__ E, int64_t m, int d, int k, int squared,
                              float* __restrict__ dQ) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= m) return;
  for (int f = lane; f < d; f += 32) {
    const float q = Q[i * d + f];
    float acc = 0.0f;
    for (int j = 0; j < k; ++j) {
      const int64_t r = idx[i * k + j];
      const float c = coef_of(G[i * k + j], E ? E[i * k + j] : 0.0f, squared);
      acc = fmaf(c, q - X[r * d + f], acc);
    }
    dQ[i * d + f] = acc;
  }
}

__global__ void bucket_count_kernel(const int64_t* __restrict__ idx, int64_t mk,
                                    int* __restrict__ counts) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < mk) atomicAdd(counts + idx[t], 1);
}

// Exclusive scan of n counts in three passes: per-block sums (2048 counts
// per block), a scan of those sums by one block, then each block's own scan.
constexpr int kScanThreads = 256, kScanPer = 8, kScanBlock = kScanThreads * kScanPer;

__device__ __forceinline__ int block_exclusive(int v, int* sh) {
  // exclusive prefix of v over the block; sh holds kScanThreads / 32 ints
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) sh[w] = incl;
  __syncthreads();
  if (w == 0) {
    int s = lane < kScanThreads / 32 ? sh[lane] : 0;
    int si = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, si, o);
      if (lane >= o) si += t;
    }
    if (lane < kScanThreads / 32) sh[lane] = si - s;
  }
  __syncthreads();
  const int r = sh[w] + incl - v;
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kScanThreads)
    scan_sums_kernel(const int* __restrict__ counts, int64_t n, int* __restrict__ sums) {
  __shared__ int sh[kScanThreads / 32];
  const int64_t base = (int64_t)blockIdx.x * kScanBlock + threadIdx.x * kScanPer;
  int s = 0;
#pragma unroll
  for (int e = 0; e < kScanPer; ++e)
    if (base + e < n) s += counts[base + e];
  const int before = block_exclusive(s, sh);
  if (threadIdx.x == kScanThreads - 1) sums[blockIdx.x] = before + s;
}

// Exclusive scan of the nb block sums in place (one block, chunks of 256);
// sums[nb] receives the total.
__global__ void __launch_bounds__(kScanThreads) scan_top_kernel(int* sums, int nb) {
  __shared__ int sh[kScanThreads / 32];
  int carry = 0;
  for (int c0 = 0; c0 < nb; c0 += kScanThreads) {
    const int i = c0 + threadIdx.x;
    const int v = i < nb ? sums[i] : 0;
    const int ex = block_exclusive(v, sh);
    if (i < nb) sums[i] = carry + ex;
    // block total: the last thread's exclusive prefix plus its value
    __shared__ int total;
    if (threadIdx.x == kScanThreads - 1) total = ex + v;
    __syncthreads();
    carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[nb] = carry;
}

__global__ void __launch_bounds__(kScanThreads)
    scan_apply_kernel(const int* __restrict__ counts, int64_t n, const int* __restrict__ sums,
                      int nb, int* __restrict__ offsets) {
  __shared__ int sh[kScanThreads / 32];
  const int64_t base = (int64_t)blockIdx.x * kScanBlock + threadIdx.x * kScanPer;
  int v[kScanPer], s = 0;
#pragma unroll
  for (int e = 0; e < kScanPer; ++e) {
    v[e] = base + e < n ? counts[base + e] : 0;
    s += v[e];
  }
  int acc = sums[blockIdx.x] + block_exclusive(s, sh);
#pragma unroll
  for (int e = 0; e < kScanPer; ++e) {
    if (base + e < n) offsets[base + e] = acc;
    acc += v[e];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) offsets[n] = sums[nb];
}

__global__ void bucket_fill_kernel(const int64_t* __restrict__ idx, int64_t mk,
                                   const int* __restrict__ offsets, int* __restrict__ cursor,
                                   int* __restrict__ order) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= mk) return;
  const int64_t r = idx[t];
  order[offsets[r] + atomicAdd(cursor + r, 1)] = (int)t;
}

// Narrow rows (d <= 8): one thread per query row, same summation order.
__global__ void grad_q_narrow_kernel(const float* __restrict__ Q, const float* __restrict__ X,
                                     const int64_t* __restrict__ idx, const float* __restrict__ G,
                                     const float* __restrict__ E, int64_t m, int d, int k,
                                     int squared, float* __restrict__ dQ) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  float q[8];
#pragma unroll
  for (int f = 0; f < 8; ++f) q[f] = f < d ? Q[i * d + f] : 0.0f;
  for (int j = 0; j < k; ++j) {
    const int64_t r = idx[i * k + j];
    const float c = coef_of(G[i * k + j], E ? E[i * k + j] : 0.0f, squared);
#pragma unroll
    for (int f = 0; f < 8; ++f)
      if (f < d) acc[f] = fmaf(c, q[f] - X[r * d + f], acc[f]);
  }
#pragma unroll
  for (int f = 0; f < 8; ++f)
    if (f < d) dQ[i * d + f] = acc[f];
}

// Narrow rows (d <= 8): one thread per reference row.
__global__ void grad_x_narrow_kernel(const float* __restrict__ Q, const float* __restrict__ X,
                                     const float* __restrict__ G, const float* __restrict__ E,
                                     const int* __restrict__ offsets, int* __restrict__ order,
                                     int64_t n, int d, int k, int squared,
                                     float* __restrict__ dX) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int a = offsets[r], b = offsets[r + 1];
  for (int p = a + 1; p < b; ++p) {
    const int v = order[p];
    int q = p;
    while (q > a && order[q - 1] > v) {
      order[q] = order[q - 1];
      --q;
    }
    order[q] = v;
  }
  float x[8], acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int f = 0; f < 8; ++f) x[f] = f < d ? X[r * d + f] : 0.0f;
  for (int p = a; p < b; ++p) {
    const int t = order[p];
    const int64_t i = t / k;
    const float c = coef_of(G[t], E ? E[t] : 0.0f, squared);
#pragma unroll
    for (int f = 0; f < 8; ++f)
      if (f < d) acc[f] = fmaf(c, x[f] - Q[i * d + f], acc[f]);
  }
#pragma unroll
  for (int f = 0; f < 8; ++f)
    if (f < d) dX[r * d + f] = acc[f];
}

// One warp per reference row: put its bucket in ascending flat position
// (each lane ranks some entries against the whole bucket and writes them to
// `sorted`: linear per entry, so rows that many queries picked stay cheap),
// then accumulate in that order.
__global__ void grad_x_kernel(const float* __restrict__ Q, const float* __restrict__ X,
                              const float* __restrict__ G, const float* __restrict__ E,
                              const int* __restrict__ offsets, const int* __restrict__ order,
                              int* __restrict__ sorted, int64_t n, int d, int k, int squared,
                              float* __restrict__ dX) {
  const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  const int a = offsets[r], b = offsets[r + 1], cnt = b - a;
  for (int e = lane; e < cnt; e += 32) {
    const int v = order[a + e];
    int rank = 0;
    for (int f = 0; f < cnt; ++f) rank += order[a + f] < v;  // flat positions are distinct
    sorted[a + rank] = v;
  }
  __syncwarp();
  for (int f = lane; f < d; f += 32) {
    const float x = X[r * d + f];
    float acc = 0.0f;
    for (int p = a; p < b; ++p) {
      const int t = sorted[p];
      const int64_t i = t / k;
      const float c = coef_of(G[t], E ? E[t] : 0.0f, squared);
      acc = fmaf(c, x - Q[i * d + f], acc);
    }
    dX[r * d + f] = acc;
  }
}

}  // namespace

int knn_backward(const float* Q, int64_t m, const float* X, int64_t n, int d, int k,
                 const int64_t* idx, const float* G, const float* E, int squared, float* dQ,
                 float* dX, int* workspace, cudaStream_t st) {
  const int warps = 8;
  const bool narrow = d <= 8;
  if (dQ && m > 0) {
    if (narrow)
      grad_q_narrow_kernel<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(Q, X, idx, G, E, m, d, k,
                                                                        squared, dQ);
    else
      grad_q_kernel<<<(unsigned)((m + warps - 1) / warps), warps * 32, 0, st>>>(
          Q, X, idx, G, E, m, d, k, squared, dQ);
  }
  if (dX && n > 0) {
    const int64_t mk = m * (int64_t)k;
    int* counts = workspace;           // [n]
    int* offsets = counts + n;         // [n + 1]
    int* cursor = offsets + n + 1;     // [n]
    int* order = cursor + n;           // [mk]
    int* sums = order + mk;            // [nb + 1] block sums of the scan
    const int nb = (int)((n + kScanBlock - 1) / kScanBlock);
    int* sorted = sums + nb + 1;       // [mk] buckets in ascending flat order
    cudaMemsetAsync(counts, 0, (size_t)n * sizeof(int), st);
    cudaMemsetAsync(cursor, 0, (size_t)n * sizeof(int), st);
    if (mk > 0)
      bucket_count_kernel<<<(unsigned)((mk + 255) / 256), 256, 0, st>>>(idx, mk, counts);
    scan_sums_kernel<<<nb, kScanThreads, 0, st>>>(counts, n, sums);
    scan_top_kernel<<<1, kScanThreads, 0, st>>>(sums, nb);
    scan_apply_kernel<<<nb, kScanThreads, 0, st>>>(counts, n, sums, nb, offsets);
    if (mk > 0)
      bucket_fill_kernel<<<(unsigned)((mk + 255) / 256), 256, 0, st>>>(idx, mk, offsets, cursor,
                                                                       order);
    if (narrow)
      grad_x_narrow_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
          Q, X, G, E, offsets, order, n, d, k, squared, dX);
    else
      grad_x_kernel<<<(unsigned)((n + warps - 1) / warps), warps * 32, 0, st>>>(
          Q, X, G, E, offsets, order, sorted, n, d, k, squared, dX);
  }
  return (int)cudaGetLastError();
}

size_t knn_backward_workspace_ints(int64_t m, int64_t n, int k) {
  return (size_t)(3 * n + 1) + 2 * (size_t)m * k + (size_t)((n + kScanBlock - 1) / kScanBlock) +
         1;
}

}  // namespace b2k
