// Exact kNN for integer data in [0, 255] (image pixels and the like).
//
// When every coordinate of the index and of the queries is an integer in
// [0, 255], the tcgen05 kind::i8 screen computes <q, x> exactly (u8 x u8
// products summed in s32), so v = ||x||^2 - 2<q, x> and the squared distance
// S = ||q||^2 + v are exact integers: the screen's per-list top-k (sinks.cuh,
// ExactU8Sink) is already the answer for its list, and a merge of the lists
// by (S, index) gives the result with no certified band, no re-rank and no
// exact-key resolution.  The float64 distance sqrt(S) equals the reference's
// canonical value: each term (q_i - x_i)^2 and every partial sum is an
// integer below 2^53, so the sequential float64 sum is exact.
//
// The reference's integer screen (src/mlxlearn_device/_neighbors_integer.py:
// 40-201) quantises arbitrary rows to int8 with per-row scales and certifies
// a band with the measured quantisation error; data that are already 8-bit
// integers need no quantisation and no band, which is the case handled here.
#include <climits>

#include "common.cuh"
#include "internal.cuh"

namespace b2k {

namespace {

__global__ void u8_check_kernel(const float* __restrict__ v, int64_t count, int* flag) {
  bool bad = false;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float x = v[i];
    // NaN fails the first test
    bad |= !(x >= 0.0f && x <= 255.0f) || x != rintf(x);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

// One warp per row: u8 row padded with zeros, and its squared norm.
__global__ void prep_u8_kernel(const float* __restrict__ v, int64_t rows, int d, int64_t rows_pad,
                               int dpu, uint8_t* __restrict__ out, int* __restrict__ norms,
                               int64_t* __restrict__ norms64, int pad_norm) {
  const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= rows_pad) return;
  uint8_t* o = out + (size_t)r * dpu;
  int64_t acc = 0;
  for (int c = lane; c < dpu; c += 32) {
    int x = 0;
    if (r < rows && c < d) x = (int)v[(size_t)r * d + c];
    o[c] = (uint8_t)x;
    acc += x * x;
  }
  for (int s = 16; s; s >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, s);
  if (lane == 0) {
    if (norms) norms[r] = r < rows ? (int)acc : pad_norm;
    if (norms64) norms64[r] = r < rows ? acc : 0;
  }
}

// One warp per query: the k smallest (v, column) of its S lists, then
// distances.  Keys (v, column) are unique (a column is in one list), so a
// 64-bit key v * 2^32 + column orders by value and then by index.
__global__ void u8_merge_kernel(const int2* __restrict__ lists, int S, int64_t m, int64_t m_pad,
                                int k, const int64_t* __restrict__ nq, int squared,
                                double* __restrict__ dist, int64_t* __restrict__ idx,
                                const int* __restrict__ status) {
  const int64_t q = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (q >= m) return;
  const int st = lane == 0 ? *reinterpret_cast<volatile const int*>(status) : 0;
  if (__shfl_sync(0xffffffffu, st, 0) != DEV_OK) return;
  const int total = S * k;
  // k rounds; each takes the smallest key above the previous winner
  auto key_at = [&](int e) -> long long {
    const int s = e / k, t = e % k;
    const int2 x = lists[((size_t)s * m_pad + q) * k + t];
    return x.x == INT_MAX ? LLONG_MAX : (long long)x.x * 4294967296LL + (unsigned)x.y;
  };
  long long last = LLONG_MIN;  // below every key: v >= -2^31
  for (int t = 0; t < k; ++t) {
    long long best = LLONG_MAX;
    for (int e = lane; e < total; e += 32) {
      const long long key = key_at(e);
      if (key > last && key < best) best = key;
    }
    for (int o = 16; o; o >>= 1) {
      const long long other = __shfl_xor_sync(0xffffffffu, best, o);
      best = other < best ? other : best;
    }
    last = best;
    if (lane == 0) {
      const size_t out = (size_t)q * k + t;
      if (best == LLONG_MAX) {  // fewer than k rows (cannot happen for a valid k)
        idx[out] = -1;
        if (dist) dist[out] = NAN;
      } else {
        const int v = (int)(best >> 32);
        const int col = (int)(best & 0xffffffffLL);
        const int64_t s2 = nq[q] + v;
        idx[out] = col;
        if (dist) dist[out] = squared ? (double)s2 : sqrt((double)s2);
      }
    }
  }
}

}  // namespace

void launch_u8_check(const float* v, int64_t count, int* flag, cudaStream_t st) {
  if (count <= 0) return;
  int64_t blocks = (count + 255) / 256;
  if (blocks > 4096) blocks = 4096;
  u8_check_kernel<<<(unsigned)blocks, 256, 0, st>>>(v, count, flag);
}

void launch_prep_u8(const float* v, int64_t rows, int d, int64_t rows_pad, int dpu, uint8_t* out,
                    int* norms, int64_t* norms64, int pad_norm, cudaStream_t st) {
  if (rows_pad <= 0) return;
  prep_u8_kernel<<<(unsigned)((rows_pad + 7) / 8), 256, 0, st>>>(v, rows, d, rows_pad, dpu, out,
                                                                 norms, norms64, pad_norm);
}

void launch_u8_merge(const int2* lists, int S, int64_t m, int64_t m_pad, int k,
                     const int64_t* nq, int squared, double* dist, int64_t* idx,
                     const int* status, cudaStream_t st) {
  if (m <= 0) return;
  u8_merge_kernel<<<(unsigned)((m + 7) / 8), 256, 0, st>>>(lists, S, m, m_pad, k, nq, squared,
                                                           dist, idx, status);
}

}  // namespace b2k
