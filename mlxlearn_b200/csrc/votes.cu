// Device-side class votes for KNeighborsClassifier.predict / predict_proba.
//
// One thread per query: the k neighbours' class codes are accumulated in
// neighbour order (deterministic) in float64, with weight 1 or 1/d; a row
// containing a zero distance uses the 0/1 indicator of its zero entries
// (the reference's rule, src/mlxlearn/neighbors/_base.py:752-785).  The
// prediction is the first maximum, i.e. ties go to the smallest class code
// (src/mlxlearn_device/_neighbors_votes.py:12-244 for the reference's device
// form, src/mlxlearn/neighbors/_classification.py:150-163 for its host form).
#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.cuh"

namespace b2k {

namespace {

__global__ void votes_kernel(const int64_t* __restrict__ idx, const double* __restrict__ dist,
                             int64_t m, int k, const int* __restrict__ codes, int n_classes,
                             int weighted, double* __restrict__ votes,
                             int64_t* __restrict__ pred, int* __restrict__ status) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  double* v = votes + i * n_classes;
  for (int c = 0; c < n_classes; ++c) v[c] = 0.0;
  bool zero_row = false;
  if (weighted)
    for (int j = 0; j < k; ++j) zero_row |= dist[i * k + j] == 0.0;
  for (int j = 0; j < k; ++j) {
    const int c = codes[idx[i * k + j]];
    double w = 1.0;
    if (weighted) {
      const double dd = dist[i * k + j];
      w = zero_row ? (dd == 0.0 ? 1.0 : 0.0) : 1.0 / dd;
    }
    v[c] += w;
  }
  int best = 0;
  double bv = v[0], total = 0.0;
  for (int c = 0; c < n_classes; ++c) {
    total += v[c];
    if (v[c] > bv) {
      bv = v[c];
      best = c;
    }
  }
  if (total == 0.0) atomicOr(status, 1);  // all weights zero: the caller raises
  if (pred) pred[i] = best;
}

// Radius neighbourhoods (CSR rows, ascending training index): one thread per
// query sums its row in entry order -- the order numpy's bincount uses in the
// reference's reductions (src/mlxlearn/_kernels/radius_reduce.py:19-94), so
// the float64 sums are identical.  Weights: 1, or 1/d with the zero-distance
// rule of a row.
__device__ __forceinline__ bool radius_zero_row(const double* dist, int64_t a, int64_t b) {
  for (int64_t e = a; e < b; ++e)
    if (dist[e] == 0.0) return true;
  return false;
}

__global__ void radius_votes_kernel(const int64_t* __restrict__ indptr,
                                    const int64_t* __restrict__ indices,
                                    const double* __restrict__ dist, int64_t m,
                                    const int* __restrict__ codes, int n_classes, int weighted,
                                    double* __restrict__ votes, int64_t* __restrict__ counts) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int64_t a = indptr[i], b = indptr[i + 1];
  double* v = votes + i * n_classes;
  for (int c = 0; c < n_classes; ++c) v[c] = 0.0;
  const bool zero_row = weighted && radius_zero_row(dist, a, b);
  for (int64_t e = a; e < b; ++e) {
    double w = 1.0;
    if (weighted) w = zero_row ? (dist[e] == 0.0 ? 1.0 : 0.0) : 1.0 / dist[e];
    v[codes[indices[e]]] += w;
  }
  counts[i] = b - a;
}

__global__ void radius_means_kernel(const int64_t* __restrict__ indptr,
                                    const int64_t* __restrict__ indices,
                                    const double* __restrict__ dist, int64_t m,
                                    const double* __restrict__ targets, int weighted,
                                    double* __restrict__ means, int64_t* __restrict__ counts) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int64_t a = indptr[i], b = indptr[i + 1];
  const bool zero_row = weighted && radius_zero_row(dist, a, b);
  double num = 0.0, den = 0.0;
  for (int64_t e = a; e < b; ++e) {
    const double y = targets[indices[e]];
    if (weighted) {
      const double w = zero_row ? (dist[e] == 0.0 ? 1.0 : 0.0) : 1.0 / dist[e];
      num = __dadd_rn(num, __dmul_rn(y, w));  // product first, then the sum (no FMA)
      den = __dadd_rn(den, w);
    } else {
      num = __dadd_rn(num, y);
    }
  }
  if (!weighted) den = (double)(b - a);
  means[i] = b > a ? num / den : __longlong_as_double(0x7ff8000000000000ll);
  counts[i] = b - a;
}

}  // namespace

void launch_radius_votes(const int64_t* indptr, const int64_t* indices, const double* dist,
                         int64_t m, const int* codes, int n_classes, int weighted, double* votes,
                         int64_t* counts, cudaStream_t st) {
  if (m <= 0) return;
  radius_votes_kernel<<<(unsigned)((m + 127) / 128), 128, 0, st>>>(
      indptr, indices, dist, m, codes, n_classes, weighted, votes, counts);
}

void launch_radius_means(const int64_t* indptr, const int64_t* indices, const double* dist,
                         int64_t m, const double* targets, int weighted, double* means,
                         int64_t* counts, cudaStream_t st) {
  if (m <= 0) return;
  radius_means_kernel<<<(unsigned)((m + 127) / 128), 128, 0, st>>>(
      indptr, indices, dist, m, targets, weighted, means, counts);
}

void launch_votes(const int64_t* idx, const double* dist, int64_t m, int k, const int* codes,
                  int n_classes, int weighted, double* votes, int64_t* pred, int* status,
                  cudaStream_t st) {
  if (m <= 0) return;
  votes_kernel<<<(unsigned)((m + 127) / 128), 128, 0, st>>>(idx, dist, m, k, codes, n_classes,
                                                            weighted, votes, pred, status);
}

}  // namespace b2k
