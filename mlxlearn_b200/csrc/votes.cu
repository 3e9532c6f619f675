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

// Radius neighbourhoods (CSR rows, ascending training index): every class's
// float64 sum runs over the row in entry order -- the order numpy's bincount
// uses in the reference's reductions (src/mlxlearn/_kernels/radius_reduce.py:19-94),
// so the sums are identical.  Weights: 1, or 1/d with the zero-distance rule
// of a row.
// One warp per row: the lanes load 32 entries at a time (class code and
// weight), then each lane walks them in entry order through shuffles and
// adds the weights of its own class, 32 classes per pass over the row.  A
// long row is no longer one thread's chain of dependent global updates.
constexpr int kVoteWarps = 8;

// votes may be null when pred is not: pred[i] is then the row's first
// maximum over the classes (ties -> smallest code, 0 for an empty row), as
// numpy's argmax.
__global__ void __launch_bounds__(kVoteWarps * 32)
    radius_votes_kernel(const int64_t* __restrict__ indptr, const int64_t* __restrict__ indices,
                        const double* __restrict__ dist, int64_t m,
                        const int* __restrict__ codes, int n_classes, int weighted,
                        double* __restrict__ votes, int64_t* __restrict__ counts,
                        int64_t* __restrict__ pred) {
  const int lane = threadIdx.x & 31;
  const int64_t i = (int64_t)blockIdx.x * kVoteWarps + (threadIdx.x >> 5);
  if (i >= m) return;  // warp-uniform
  const int64_t a = indptr[i], b = indptr[i + 1];
  bool zero_row = false;
  if (weighted)
    for (int64_t e0 = a; e0 < b && !zero_row; e0 += 32) {
      const int64_t e = e0 + lane;
      zero_row = __any_sync(0xffffffffu, e < b && dist[e] == 0.0);
    }
  double best = -INFINITY;  // pred: the first maximum so far and its class
  int best_class = 0;
  for (int c0 = 0; c0 < n_classes; c0 += 32) {
    const int mine = c0 + lane;
    double acc = 0.0;
    for (int64_t e0 = a; e0 < b; e0 += 32) {
      const int64_t e = e0 + lane;
      int cls = -1;
      double w = 1.0;
      if (e < b) {
        cls = codes[indices[e]];
        if (weighted) w = zero_row ? (dist[e] == 0.0 ? 1.0 : 0.0) : 1.0 / dist[e];
      }
      const int n = b - e0 < 32 ? (int)(b - e0) : 32;
      for (int t = 0; t < n; ++t) {
        const int ct = __shfl_sync(0xffffffffu, cls, t);
        const double wt = __shfl_sync(0xffffffffu, w, t);
        if (ct == mine) acc += wt;
      }
    }
    if (votes && mine < n_classes) votes[i * n_classes + mine] = acc;
    if (pred) {
      // this pass's maximum, the smallest class among equal values; a later
      // pass replaces the running one only when strictly larger
      double v = mine < n_classes ? acc : -INFINITY;
      int c = mine;
      for (int o = 16; o; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oc = __shfl_xor_sync(0xffffffffu, c, o);
        if (ov > v || (ov == v && oc < c)) {
          v = ov;
          c = oc;
        }
      }
      if (v > best) {
        best = v;
        best_class = c;
      }
    }
  }
  if (lane == 0) {
    counts[i] = b - a;
    if (pred) pred[i] = best_class;
  }
}

// Weighted or plain mean of the row's targets, one warp per row: entries are
// loaded 32 at a time and every lane forms the same sums in entry order
// (product first, then the sum, no FMA), as the reference's host reduction.
__global__ void __launch_bounds__(kVoteWarps * 32)
    radius_means_kernel(const int64_t* __restrict__ indptr, const int64_t* __restrict__ indices,
                        const double* __restrict__ dist, int64_t m,
                        const double* __restrict__ targets, int weighted,
                        double* __restrict__ means, int64_t* __restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const int64_t i = (int64_t)blockIdx.x * kVoteWarps + (threadIdx.x >> 5);
  if (i >= m) return;  // warp-uniform
  const int64_t a = indptr[i], b = indptr[i + 1];
  bool zero_row = false;
  if (weighted)
    for (int64_t e0 = a; e0 < b && !zero_row; e0 += 32) {
      const int64_t e = e0 + lane;
      zero_row = __any_sync(0xffffffffu, e < b && dist[e] == 0.0);
    }
  double num = 0.0, den = 0.0;
  for (int64_t e0 = a; e0 < b; e0 += 32) {
    const int64_t e = e0 + lane;
    double y = 0.0, w = 1.0;
    if (e < b) {
      y = targets[indices[e]];
      if (weighted) w = zero_row ? (dist[e] == 0.0 ? 1.0 : 0.0) : 1.0 / dist[e];
    }
    const int n = b - e0 < 32 ? (int)(b - e0) : 32;
    for (int t = 0; t < n; ++t) {
      const double yt = __shfl_sync(0xffffffffu, y, t);
      if (weighted) {
        const double wt = __shfl_sync(0xffffffffu, w, t);
        num = __dadd_rn(num, __dmul_rn(yt, wt));
        den = __dadd_rn(den, wt);
      } else {
        num = __dadd_rn(num, yt);
      }
    }
  }
  if (lane == 0) {
    if (!weighted) den = (double)(b - a);
    means[i] = b > a ? num / den : __longlong_as_double(0x7ff8000000000000ll);
    counts[i] = b - a;
  }
}

}  // namespace

void launch_radius_votes(const int64_t* indptr, const int64_t* indices, const double* dist,
                         int64_t m, const int* codes, int n_classes, int weighted, double* votes,
                         int64_t* counts, cudaStream_t st, int64_t* pred) {
  if (m <= 0) return;
  radius_votes_kernel<<<(unsigned)((m + kVoteWarps - 1) / kVoteWarps), kVoteWarps * 32, 0, st>>>(
      indptr, indices, dist, m, codes, n_classes, weighted, votes, counts, pred);
}

void launch_radius_means(const int64_t* indptr, const int64_t* indices, const double* dist,
                         int64_t m, const double* targets, int weighted, double* means,
                         int64_t* counts, cudaStream_t st) {
  if (m <= 0) return;
  radius_means_kernel<<<(unsigned)((m + kVoteWarps - 1) / kVoteWarps), kVoteWarps * 32, 0, st>>>(
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
