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

// Exclusive scan of n counts (single CTA, chunked).
__global__ void bucket_scan_kernel(const int* __restrict__ counts, int64_t n,
                                   int* __restrict__ offsets) {
  __shared__ long long part[1024];
  const int t = threadIdx.x;
  const int64_t per = (n + blockDim.x - 1) / blockDim.x;
  const int64_t a = min(n, (int64_t)t * per), b = min(n, a + per);
  long long s = 0;
  for (int64_t r = a; r < b; ++r) s += counts[r];
  part[t] = s;
  __syncthreads();
  if (t == 0) {
    long long acc = 0;
    for (int i = 0; i < (int)blockDim.x; ++i) {
      const long long v = part[i];
      part[i] = acc;
      acc += v;
    }
    offsets[n] = (int)acc;
  }
  __syncthreads();
  long long acc = part[t];
  for (int64_t r = a; r < b; ++r) {
    offsets[r] = (int)acc;
    acc += counts[r];
  }
}

__global__ void bucket_fill_kernel(const int64_t* __restrict__ idx, int64_t mk,
                                   const int* __restrict__ offsets, int* __restrict__ cursor,
                                   int* __restrict__ order) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= mk) return;
  const int64_t r = idx[t];
  order[offsets[r] + atomicAdd(cursor + r, 1)] = (int)t;
}

// One warp per reference row: order its bucket (insertion sort by flat
// position, buckets are short), then accumulate in that order.
__global__ void grad_x_kernel(const float* __restrict__ Q, const float* __restrict__ X,
                              const float* __restrict__ G, const float* __restrict__ E,
                              const int* __restrict__ offsets, int* __restrict__ order,
                              int64_t n, int d, int k, int squared, float* __restrict__ dX) {
  const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  const int a = offsets[r], b = offsets[r + 1];
  if (lane == 0) {
    for (int p = a + 1; p < b; ++p) {
      const int v = order[p];
      int q = p;
      while (q > a && order[q - 1] > v) {
        order[q] = order[q - 1];
        --q;
      }
      order[q] = v;
    }
  }
  __syncwarp();
  for (int f = lane; f < d; f += 32) {
    const float x = X[r * d + f];
    float acc = 0.0f;
    for (int p = a; p < b; ++p) {
      const int t = order[p];
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
  if (dQ && m > 0)
    grad_q_kernel<<<(unsigned)((m + warps - 1) / warps), warps * 32, 0, st>>>(
        Q, X, idx, G, E, m, d, k, squared, dQ);
  if (dX && n > 0) {
    const int64_t mk = m * (int64_t)k;
    int* counts = workspace;           // [n]
    int* offsets = counts + n;         // [n + 1]
    int* cursor = offsets + n + 1;     // [n]
    int* order = cursor + n;           // [mk]
    cudaMemsetAsync(counts, 0, (size_t)n * sizeof(int), st);
    cudaMemsetAsync(cursor, 0, (size_t)n * sizeof(int), st);
    if (mk > 0)
      bucket_count_kernel<<<(unsigned)((mk + 255) / 256), 256, 0, st>>>(idx, mk, counts);
    bucket_scan_kernel<<<1, 1024, 0, st>>>(counts, n, offsets);
    if (mk > 0)
      bucket_fill_kernel<<<(unsigned)((mk + 255) / 256), 256, 0, st>>>(idx, mk, offsets, cursor,
                                                                       order);
    grad_x_kernel<<<(unsigned)((n + warps - 1) / warps), warps * 32, 0, st>>>(
        Q, X, G, E, offsets, order, n, d, k, squared, dX);
  }
  return (int)cudaGetLastError();
}

size_t knn_backward_workspace_ints(int64_t m, int64_t n, int k) {
  return (size_t)(3 * n + 1) + (size_t)m * k;
}

}  // namespace b2k
