// Exact kNN over many (query segment, reference segment) pairs of small width
// in one launch — the forward of point-set losses such as a Chamfer term,
// where every pair of clouds is its own small problem.
//
// The tensor-core screen needs an index per problem and one call per
// problem; for d <= 64 and a few thousand rows a direct scan is cheaper.
// One block takes 128 queries of one segment; the segment's reference rows
// pass through shared memory in 32 KB tiles, and every thread keeps the KS
// smallest fp32 squared distances of its query (KS >= k + 3) in registers.
// The fp32 value s of a pair is within g S + d 2^-126 of the exact S,
// g = (d + 5) 2^-24 (1.01) (a sum of rounded squares of rounded differences,
// whatever the order).  The query is certified when the KS-th value's lower
// bound exceeds the k-th value's upper bound (or the segment has at most KS
// rows): every row that can be in the answer is then among the KS kept,
// and those whose intervals reach the k-th upper bound are ordered by their
// canonical float64 values, with the exact integer comparator for float64
// near-ties (the order mlxlearn defines,
// src/mlxlearn/_kernels/_neighbors_cpu_native.cpp:170-190).  Other queries,
// and every query when some coordinate lies outside [2^-60, 2^50] in
// magnitude, go to the exhaustive exact kernel (certify.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstdio>
#include <vector>

#include "common.cuh"
#include "exact.cuh"
#include "internal.cuh"

namespace b2k {
namespace {

constexpr int kSegThreads = 128;  // queries per block
// reference rows per shared-memory tile: 32 KB of padded rows, at most 512
__host__ __device__ constexpr int seg_tile_rows(int D) { return D <= 16 ? 512 : 8192 / D; }

struct SegArgs {
  const float* Q;
  const float* X;
  int d;
  const int64_t* qseg;  // [P + 1] query row offsets
  const int64_t* xseg;  // [P + 1] reference row offsets
  const int2* blocks;   // per block: (segment, first query row within it)
  int k, exclude_self;
  double* dist;         // [rows, k] or null
  int64_t* idx;         // [rows, k] indices within the reference segment
  int* fallback_list;   // global query rows for the exhaustive kernel
  int* flags;           // [0] fallback count, [1] coordinate out of range
};

__device__ __forceinline__ bool seg_coord_ok(float v) {
  const uint32_t a = __float_as_uint(v) & 0x7fffffffu;
  return a == 0 || (a >= (67u << 23) && a <= (177u << 23));  // 0 or [2^-60, 2^50]
}

__global__ void seg_range_kernel(const float* __restrict__ v, int64_t count, int* flags) {
  bool ok = true;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x)
    ok &= seg_coord_ok(v[i]);
  if (!__all_sync(0xffffffffu, ok) && (threadIdx.x & 31) == 0) atomicOr(flags + 1, 1);
}

// D: padded width (4, 8 or 16) of the shared-memory rows; DC: coordinates
// actually computed (D, or 3 for three-dimensional points).
// Packed pairs of fp32 values (one 64-bit register), for the paired
// sub / fma instructions: each half is rounded exactly as the scalar op.
__device__ __forceinline__ uint64_t pk(float lo, float hi) {
  uint64_t x;
  asm("mov.b64 %0, {%1,%2};" : "=l"(x) : "f"(lo), "f"(hi));
  return x;
}
__device__ __forceinline__ void upk(uint64_t x, float& lo, float& hi) {
  asm("mov.b64 {%0,%1}, %2;" : "=f"(lo), "=f"(hi) : "l"(x));
}
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

template <int KS>
__device__ __forceinline__ void seg_offer(float s, int j, int self, float (&kv)[KS],
                                          int (&ki)[KS]) {
  if (s < kv[KS - 1] && j != self) {
    // insertion after any equal value: equal values keep scan (index) order
    float cv = s;
    int cj = j;
#pragma unroll
    for (int i = 0; i < KS; ++i) {
      if (cv < kv[i]) {
        const float tv = kv[i];
        const int tj = ki[i];
        kv[i] = cv;
        ki[i] = cj;
        cv = tv;
        cj = tj;
      }
    }
  }
}

template <int D, int KS, int DC = D>
__global__ void __launch_bounds__(kSegThreads) seg_scan_kernel(const __grid_constant__ SegArgs a) {
  constexpr int D4 = D / 4;
  constexpr int kSegTile = seg_tile_rows(D);
  __shared__ float4 tile[kSegTile * D4];
  const int2 blk = a.blocks[blockIdx.x];
  const int64_t q_lo = a.qseg[blk.x], q_hi = a.qseg[blk.x + 1];
  const int64_t x_lo = a.xseg[blk.x], x_hi = a.xseg[blk.x + 1];
  const int n = (int)(x_hi - x_lo);
  const int64_t qi = q_lo + blk.y + threadIdx.x;
  const bool active = qi < q_hi;
  const int d = a.d;
  const int self = (a.exclude_self && active) ? (int)(qi - q_lo) : -1;
  const bool range_bad = *reinterpret_cast<volatile const int*>(a.flags + 1) != 0;

  float q[D];
#pragma unroll
  for (int c = 0; c < D; ++c) q[c] = (active && c < d) ? a.Q[qi * d + c] : 0.0f;
  float kv[KS];
  int ki[KS];
#pragma unroll
  for (int i = 0; i < KS; ++i) {
    kv[i] = INFINITY;
    ki[i] = -1;
  }
  for (int t0 = 0; t0 < n && !range_bad; t0 += kSegTile) {
    const int cnt = min(kSegTile, n - t0);
    __syncthreads();
    for (int i = threadIdx.x; i < cnt * D4; i += kSegThreads) {
      const int r = i / D4, c = (i % D4) * 4;
      const float* x = a.X + (x_lo + t0 + r) * d;
      tile[i] = make_float4(c < d ? x[c] : 0.0f, c + 1 < d ? x[c + 1] : 0.0f,
                            c + 2 < d ? x[c + 2] : 0.0f, c + 3 < d ? x[c + 3] : 0.0f);
    }
    __syncthreads();
    if (active && DC == 3) {
      // three coordinates, two reference rows per paired instruction; the
      // sums are formed in the scalar order e0^2, e1^2, e2^2
      const uint64_t q0 = pk(q[0], q[0]), q1 = pk(q[1], q[1]), q2 = pk(q[2], q[2]);
      int r = 0;
#pragma unroll 2
      for (; r + 1 < cnt; r += 2) {
        const float4 v0 = tile[r], v1 = tile[r + 1];
        const uint64_t e0 = sub2(q0, pk(v0.x, v1.x));
        const uint64_t e1 = sub2(q1, pk(v0.y, v1.y));
        const uint64_t e2 = sub2(q2, pk(v0.z, v1.z));
        uint64_t s2 = fma2(e0, e0, pk(0.0f, 0.0f));
        s2 = fma2(e1, e1, s2);
        s2 = fma2(e2, e2, s2);
        float s0, s1;
        upk(s2, s0, s1);
        seg_offer<KS>(s0, t0 + r, self, kv, ki);
        seg_offer<KS>(s1, t0 + r + 1, self, kv, ki);
      }
      if (r < cnt) {
        const float4 v = tile[r];
        const float e0 = q[0] - v.x, e1 = q[1] - v.y, e2 = q[2] - v.z;
        float s0 = fmaf(e0, e0, 0.0f);
        s0 = fmaf(e1, e1, s0);
        s0 = fmaf(e2, e2, s0);
        seg_offer<KS>(s0, t0 + r, self, kv, ki);
      }
    } else if (active) {
#pragma unroll 4
      for (int r = 0; r < cnt; ++r) {
        float s = 0.0f;
#pragma unroll
        for (int c4 = 0; c4 < D4; ++c4) {
          const float4 v = tile[r * D4 + c4];
          const float e0 = q[4 * c4] - v.x, e1 = q[4 * c4 + 1] - v.y;
          const float e2 = q[4 * c4 + 2] - v.z;
          s = fmaf(e0, e0, s);
          s = fmaf(e1, e1, s);
          s = fmaf(e2, e2, s);
          if (4 * c4 + 3 < DC) {
            const float e3 = q[4 * c4 + 3] - v.w;
            s = fmaf(e3, e3, s);
          }
        }
        seg_offer<KS>(s, t0 + r, self, kv, ki);
      }
    }
  }
  if (!active) return;
  const int k = a.k;
  const int n_eff = n - (self >= 0 && self < n ? 1 : 0);
  const float g32 = (float)((double)(d + 5) * 0x1p-24 * 1.01);
  const float abs32 = (float)d * 0x1p-126f;
  const float U = __fadd_ru(__fmul_ru(kv[k - 1], 1.0f + g32), abs32);
  bool certified = !range_bad;
  if (certified && n_eff > KS)
    certified = __fsub_rd(__fmul_rd(kv[KS - 1], 1.0f - g32), abs32) > U;
  if (!certified) {
    a.fallback_list[atomicAdd(a.flags, 1)] = (int)qi;
    return;
  }
  // survivors: a prefix of the kept values (ascending)
  int Cs = 0;
#pragma unroll
  for (int i = 0; i < KS; ++i)
    if (ki[i] >= 0 && __fsub_rd(__fmul_rd(kv[i], 1.0f - g32), abs32) <= U) Cs = i + 1;
  const float* qp = a.Q + qi * d;
  const float* xs = a.X + x_lo * d;
  double cs[KS];
  int id[KS];
#pragma unroll
  for (int i = 0; i < KS; ++i) {
    id[i] = ki[i];
    cs[i] = i < Cs ? canonical_d2(qp, xs + (size_t)ki[i] * d, d) : DBL_MAX;
  }
  // sort the survivors by (canonical value, index)
  for (int i = 1; i < Cs; ++i) {
    const double sv = cs[i];
    const int sj = id[i];
    int b = i;
    while (b > 0 && (cs[b - 1] > sv || (cs[b - 1] == sv && id[b - 1] > sj))) {
      cs[b] = cs[b - 1];
      id[b] = id[b - 1];
      --b;
    }
    cs[b] = sv;
    id[b] = sj;
  }
  // runs of overlapping float64 error intervals that reach into the top k:
  // exact order by the integer comparator, ties by the smaller index
  const double g2 = 2.0 * (double)(d + 2) * 0x1p-53 / (1.0 - (double)(d + 2) * 0x1p-53);
  int i = 0;
  while (i < k && i < Cs) {
    int j = i + 1;
    while (j < Cs && __dmul_rd(cs[j], 1.0 - g2) <= __dmul_ru(cs[j - 1], 1.0 + g2)) ++j;
    if (j - i > 1 && cs[j - 1] != 0.0) {
      for (int t = i + 1; t < j; ++t) {
        const double st = cs[t];
        const int it = id[t];
        int b = t;
        while (b > i) {
          const int c = exact_compare(qp, xs + (size_t)it * d, xs + (size_t)id[b - 1] * d, d);
          if (c > 0 || (c == 0 && it > id[b - 1])) break;
          cs[b] = cs[b - 1];
          id[b] = id[b - 1];
          --b;
        }
        cs[b] = st;
        id[b] = it;
      }
    }
    i = j;
  }
  for (int t = 0; t < k; ++t) {
    a.idx[qi * k + t] = id[t];
    if (a.dist) a.dist[qi * k + t] = sqrt(cs[t]);
  }
}

template <int D, int DC = D>
void launch_seg_scan(const SegArgs& a, int ks, int blocks, cudaStream_t st) {
  if (ks <= 4) seg_scan_kernel<D, 4, DC><<<blocks, kSegThreads, 0, st>>>(a);
  else if (ks <= 8) seg_scan_kernel<D, 8, DC><<<blocks, kSegThreads, 0, st>>>(a);
  else if (ks <= 16) seg_scan_kernel<D, 16, DC><<<blocks, kSegThreads, 0, st>>>(a);
  else seg_scan_kernel<D, 32, DC><<<blocks, kSegThreads, 0, st>>>(a);
}

int seg_fail(int code, const char* msg) { return report_error(code, msg); }

}  // namespace
}  // namespace b2k

using namespace b2k;

extern "C" B2K_API int b2k_knn_segments(const float* dQ, const float* dX, int32_t d,
                                        const int64_t* q_offsets, const int64_t* x_offsets,
                                        int32_t segments, int32_t k, int32_t exclude_self,
                                        double* d_dist, int64_t* d_idx, void* stream) {
  if (segments < 0 || !q_offsets || !x_offsets)
    return seg_fail(B2K_EINVAL, "segment offsets must not be NULL");
  if (d <= 0 || d > 64)
    return seg_fail(B2K_EUNSUPPORTED, "b2k_knn_segments handles 1 <= d <= 64; use the index API");
  if (k <= 0) return seg_fail(B2K_EINVAL, "Expected n_neighbors > 0.");
  if (k > 29) return seg_fail(B2K_EUNSUPPORTED, "b2k_knn_segments handles k <= 29");
  if (q_offsets[0] != 0 || x_offsets[0] != 0)
    return seg_fail(B2K_EINVAL, "segment offsets must start at 0");
  std::vector<int2> blocks;
  int64_t n_max = 0;
  for (int p = 0; p < segments; ++p) {
    const int64_t m = q_offsets[p + 1] - q_offsets[p], n = x_offsets[p + 1] - x_offsets[p];
    if (m < 0 || n < 0) return seg_fail(B2K_EINVAL, "segment offsets must not decrease");
    if (n >= ((int64_t)1 << 31) || q_offsets[p + 1] >= ((int64_t)1 << 31))
      return seg_fail(B2K_EINVAL, "segments must fit int32 row counts");
    if (m == 0) continue;
    if (exclude_self && m != n)
      return seg_fail(B2K_EINVAL,
                      "exclude_self requires every query segment to be its reference segment");
    const int64_t limit = n - (exclude_self ? 1 : 0);
    if (k > limit) {
      char msg[128];
      snprintf(msg, sizeof(msg), "n_neighbors must be <= %lld, got %d.", (long long)limit, k);
      return seg_fail(B2K_EINVAL, msg);
    }
    n_max = std::max(n_max, n);
    for (int64_t q0 = 0; q0 < m; q0 += kSegThreads) blocks.push_back(make_int2(p, (int)q0));
  }
  const int64_t rows = segments ? q_offsets[segments] : 0;
  if (blocks.empty()) return B2K_OK;
  if (!dQ || !dX || !d_idx) return seg_fail(B2K_EINVAL, "device pointers must not be NULL");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int P = segments;
  // one stream-ordered scratch block: offsets, block list, exact-scan table,
  // fallback list, flags, counters
  const size_t off_b = (size_t)(P + 1) * sizeof(int64_t);
  const size_t blk_b = blocks.size() * sizeof(int2);
  const size_t tab_b = (size_t)P * sizeof(ExactArgs);
  auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
  const size_t bytes = 2 * al(off_b) + al(blk_b) + al(tab_b) + al((size_t)rows * sizeof(int)) +
                       al(16 * sizeof(int)) + al(4 * sizeof(unsigned long long));
  unsigned char* base = nullptr;
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&base), bytes, st);
  if (e != cudaSuccess)
    return seg_fail(e == cudaErrorMemoryAllocation ? B2K_ENOMEM : B2K_ECUDA,
                    "scratch allocation for b2k_knn_segments failed");
  unsigned char* c = base;
  int64_t* qseg = reinterpret_cast<int64_t*>(c);
  c += al(off_b);
  int64_t* xseg = reinterpret_cast<int64_t*>(c);
  c += al(off_b);
  int2* dblocks = reinterpret_cast<int2*>(c);
  c += al(blk_b);
  ExactArgs* tab = reinterpret_cast<ExactArgs*>(c);
  c += al(tab_b);
  int* fb = reinterpret_cast<int*>(c);
  c += al((size_t)rows * sizeof(int));
  int* flags = reinterpret_cast<int*>(c);  // [0] fallback count, [1] range, [2] exact status
  c += al(16 * sizeof(int));
  unsigned long long* counters = reinterpret_cast<unsigned long long*>(c);

  std::vector<ExactArgs> ex(P);
  for (int p = 0; p < P; ++p) {
    ExactArgs& t = ex[p];
    t = ExactArgs{};
    t.X = dX + x_offsets[p] * d;
    t.Q = dQ + q_offsets[p] * d;
    t.n = x_offsets[p + 1] - x_offsets[p];
    t.m = q_offsets[p + 1] - q_offsets[p];
    t.d = d;
    t.k = k;
    t.exclude_self = exclude_self;
    t.q_offset = 0;
    t.dist = d_dist ? d_dist + q_offsets[p] * k : nullptr;
    t.idx = d_idx + q_offsets[p] * k;
    t.counters = counters;
    t.status = flags + 2;
  }
  int rc = B2K_OK;
  int hflags[16];
  do {
    if ((e = cudaMemcpyAsync(qseg, q_offsets, off_b, cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync(xseg, x_offsets, off_b, cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync(dblocks, blocks.data(), blk_b, cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync(tab, ex.data(), tab_b, cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemsetAsync(flags, 0, 16 * sizeof(int), st)) ||
        (e = cudaMemsetAsync(counters, 0, 4 * sizeof(unsigned long long), st))) {
      rc = seg_fail(B2K_ECUDA, "b2k_knn_segments: copy to the device failed");
      break;
    }
    const int64_t nq = rows * d, nx = x_offsets[P] * d;
    seg_range_kernel<<<(unsigned)std::min<int64_t>((nq + 255) / 256 + 1, 1024), 256, 0, st>>>(
        dQ, nq, flags);
    seg_range_kernel<<<(unsigned)std::min<int64_t>((nx + 255) / 256 + 1, 1024), 256, 0, st>>>(
        dX, nx, flags);
    SegArgs a{};
    a.Q = dQ;
    a.X = dX;
    a.d = d;
    a.qseg = qseg;
    a.xseg = xseg;
    a.blocks = dblocks;
    a.k = k;
    a.exclude_self = exclude_self;
    a.dist = d_dist;
    a.idx = d_idx;
    a.fallback_list = fb;
    a.flags = flags;
    const int ks = k + 3;
    const int nb = (int)blocks.size();
    if (d <= 3) launch_seg_scan<4, 3>(a, ks, nb, st);
    else if (d <= 4) launch_seg_scan<4>(a, ks, nb, st);
    else if (d <= 8) launch_seg_scan<8>(a, ks, nb, st);
    else if (d <= 16) launch_seg_scan<16>(a, ks, nb, st);
    else if (d <= 32) launch_seg_scan<32>(a, ks, nb, st);
    else launch_seg_scan<64>(a, ks, nb, st);
    if ((e = cudaGetLastError())) {
      rc = seg_fail(B2K_ECUDA, "b2k_knn_segments: scan launch failed");
      break;
    }
    // uncertified queries: exhaustive exact scan of their segment
    int dev = 0;
    cudaGetDevice(&dev);
    launch_exact_batch(tab, qseg, P, fb, flags, nullptr, n_max, 2 * num_sms(dev), st);
    if ((e = cudaGetLastError())) {
      rc = seg_fail(B2K_ECUDA, "b2k_knn_segments: exact launch failed");
      break;
    }
    if ((e = cudaMemcpyAsync(hflags, flags, sizeof(hflags), cudaMemcpyDeviceToHost, st)) ||
        (e = cudaStreamSynchronize(st))) {
      rc = seg_fail(B2K_ECUDA, "b2k_knn_segments: device error");
      break;
    }
    if (hflags[2] == DEV_TOO_MANY_TIES)
      rc = seg_fail(B2K_EUNSUPPORTED,
                    "more than 4096 reference rows tie (within float64 error) with a query's "
                    "k-th neighbour");
  } while (false);
  cudaFreeAsync(base, st);
  return rc;
}
