// Reference-row shards: merging per-shard kNN answers into the answer over
// all rows.
//
// Each shard (one per GPU) holds a contiguous range of the fitted rows and
// answers the whole query batch with its own exact top-k, indices made
// global.  After one exchange of those lists, every rank merges them here:
//
//   shard_merge_kernel   one thread per query: k-way merge of the S lists,
//                        taking the smallest (float64 distance, global index)
//                        head each time.  Within a list the order is already
//                        the exact one; between lists the float64 order is
//                        exact unless two heads' error intervals overlap (the
//                        canonical distance is within eps of the exact one),
//                        in which case the query is flagged.
//   shard_keys_kernel    for flagged queries only: the 640-bit exact key of
//                        every candidate this shard owns (exact.cuh).
//   shard_resolve_kernel for flagged queries, once every shard's keys are
//                        summed in: the first k by (exact key, global index).
//
// The order is the neighbour path's exact order with ties to the smaller row
// (reference src/mlxlearn/_kernels/_neighbors_cpu_native.cpp:170-190); the
// reference itself has no multi-device path.
#include <cfloat>

#include "common.cuh"
#include "exact.cuh"
#include "internal.cuh"

namespace b2k {

namespace {


struct ShardLists {
  const double* D;     // [S, m, kin] ascending within each (shard, query)
  const int64_t* I;    // [S, m, kin] global rows, -1 past the shard's rows
  int S;
  int64_t m;
  int kin;
  __device__ __forceinline__ size_t at(int s, int64_t q, int j) const {
    return ((size_t)s * m + q) * kin + j;
  }
};

__global__ void shard_merge_kernel(ShardLists L, int kout, int64_t self_offset, double eps,
                                   double* __restrict__ out_d, int64_t* __restrict__ out_i,
                                   int32_t* __restrict__ flags) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= L.m) return;
  const int64_t self = self_offset >= 0 ? self_offset + q : -2;
  int head[kMaxShards];
  for (int s = 0; s < L.S; ++s) head[s] = 0;
  int flag = 0;
  for (int p = 0; p < kout; ++p) {
    int best = -1;
    double bd = 0.0;
    int64_t bi = 0;
    for (int s = 0; s < L.S; ++s) {
      while (head[s] < L.kin && L.I[L.at(s, q, head[s])] == self) ++head[s];
      if (head[s] >= L.kin) continue;
      const size_t o = L.at(s, q, head[s]);
      const int64_t g = L.I[o];
      if (g < 0) continue;  // the shard has no more rows
      const double dd = L.D[o];
      if (best < 0 || dd < bd || (dd == bd && g < bi)) {
        best = s;
        bd = dd;
        bi = g;
      }
    }
    if (best < 0) {  // fewer candidates than k (rejected by the host before launch)
      out_d[q * kout + p] = DBL_MAX;
      out_i[q * kout + p] = -1;
      flag = 1;
      continue;
    }
    // another shard's head whose distance interval reaches this one's
    for (int s = 0; s < L.S; ++s) {
      if (s == best || head[s] >= L.kin) continue;
      const size_t o = L.at(s, q, head[s]);
      if (L.I[o] < 0) continue;
      if (bd * (1.0 + eps) >= L.D[o] * (1.0 - eps)) flag = 1;
    }
    out_d[q * kout + p] = bd;
    out_i[q * kout + p] = bi;
    ++head[best];
  }
  flags[q] = flag;
}

__global__ void shard_keys_kernel(ShardLists L, const float* __restrict__ Q,
                                  const float* __restrict__ X, int64_t n_local, int d,
                                  int64_t row_lo, const int64_t* __restrict__ flagged, int64_t F,
                                  uint64_t* __restrict__ keys) {
  const int64_t per = (int64_t)L.S * L.kin;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= F * per) return;
  const int64_t f = t / per;
  const int c = (int)(t % per);
  const int s = c / L.kin, j = c % L.kin;
  const int64_t q = flagged[f];
  const int64_t g = L.I[L.at(s, q, j)];
  if (g < row_lo || g >= row_lo + n_local) return;  // another shard's row (or none)
  ExactKey key;
  exact_key(Q + (size_t)q * d, X + (size_t)(g - row_lo) * d, d, key);
  uint64_t* out = keys + (size_t)t * kKeyLimbs;
#pragma unroll
  for (int w = 0; w < kKeyLimbs; ++w) out[w] = key.w[w];
}

// (key_a, row a) < (key_b, row b)
__device__ __forceinline__ bool key_row_less(const uint64_t* a, int64_t ra, const uint64_t* b,
                                             int64_t rb) {
  for (int w = kKeyLimbs - 1; w >= 0; --w)
    if (a[w] != b[w]) return a[w] < b[w];
  return ra < rb;
}

__global__ void shard_resolve_kernel(ShardLists L, int kout, int64_t self_offset,
                                     const int64_t* __restrict__ flagged, int64_t F,
                                     const uint64_t* __restrict__ keys, double* __restrict__ out_d,
                                     int64_t* __restrict__ out_i) {
  const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  const int64_t q = flagged[f];
  const int64_t self = self_offset >= 0 ? self_offset + q : -2;
  const int per = L.S * L.kin;
  uint32_t taken[(kMaxShards * (kMaxShardK + 1) + 31) / 32];
  for (int w = 0; w < (per + 31) / 32; ++w) taken[w] = 0;
  const uint64_t* kq = keys + (size_t)f * per * kKeyLimbs;
  for (int p = 0; p < kout; ++p) {
    int best = -1;
    int64_t bg = 0;
    for (int c = 0; c < per; ++c) {
      if (taken[c >> 5] >> (c & 31) & 1u) continue;
      const int64_t g = L.I[L.at(c / L.kin, q, c % L.kin)];
      if (g < 0 || g == self) continue;
      if (best < 0 ||
          key_row_less(kq + (size_t)c * kKeyLimbs, g, kq + (size_t)best * kKeyLimbs, bg)) {
        best = c;
        bg = g;
      }
    }
    if (best < 0) break;
    taken[best >> 5] |= 1u << (best & 31);
    out_d[q * kout + p] = L.D[L.at(best / L.kin, q, best % L.kin)];
    out_i[q * kout + p] = bg;
  }
}

}  // namespace

void launch_shard_merge(const double* D, const int64_t* I, int S, int64_t m, int kin, int kout,
                        int64_t self_offset, double eps, double* out_d, int64_t* out_i,
                        int32_t* flags, cudaStream_t st) {
  if (m <= 0) return;
  const ShardLists L{D, I, S, m, kin};
  const int tb = 128;
  shard_merge_kernel<<<(unsigned)((m + tb - 1) / tb), tb, 0, st>>>(L, kout, self_offset, eps,
                                                                   out_d, out_i, flags);
}

void launch_shard_keys(const double* D, const int64_t* I, int S, int64_t m, int kin,
                       const float* Q, const float* X, int64_t n_local, int d, int64_t row_lo,
                       const int64_t* flagged, int64_t F, uint64_t* keys, cudaStream_t st) {
  const int64_t total = F * S * kin;
  if (total <= 0) return;
  const ShardLists L{D, I, S, m, kin};
  const int tb = 128;
  shard_keys_kernel<<<(unsigned)((total + tb - 1) / tb), tb, 0, st>>>(L, Q, X, n_local, d, row_lo,
                                                                      flagged, F, keys);
}

void launch_shard_resolve(const double* D, const int64_t* I, int S, int64_t m, int kin, int kout,
                          int64_t self_offset, const int64_t* flagged, int64_t F,
                          const uint64_t* keys, double* out_d, int64_t* out_i, cudaStream_t st) {
  if (F <= 0) return;
  const ShardLists L{D, I, S, m, kin};
  const int tb = 64;
  shard_resolve_kernel<<<(unsigned)((F + tb - 1) / tb), tb, 0, st>>>(L, kout, self_offset,
                                                                     flagged, F, keys, out_d,
                                                                     out_i);
}

}  // namespace b2k
