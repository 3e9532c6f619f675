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
// nearest pivot (bf16 Gram form on the tensor cores: the assignment only
// affects speed, a near tie may go either way), then a
// counting sort by pivot gives the permutation `perm` (sorted position ->
// original query row) and the permuted query matrix.  Results are written
// back to the original rows by the certify / exact kernels, so the answer
// does not depend on the order.
//
// The same assignment groups the rows of the index's bf16 operand by pivot
// (b200knn.cu): a tile of grouped queries then finds its candidates in a few
// consecutive reference tiles, and the other tiles' chunks skip admission.
#include <cuda_bf16.h>

#include "common.cuh"
#include "internal.cuh"

namespace b2k {

namespace {

constexpr int kAssignThreads = 128;  // 4 warps x 32 queries
constexpr int kMmaP = 64;            // pivots per shared-memory tile
constexpr int kMmaK = 64;            // features per shared-memory chunk
constexpr int kMmaLd = kMmaK + 8;    // padded row: conflict-free fragment loads

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

// The bf16 copy of the pivots, [P_pad, dpa] (multiples of 64), zero padded.
__global__ void pivots_bf16_kernel(const float* __restrict__ piv, int P, int d, int P_pad, int dpa,
                                   uint16_t* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)P_pad * dpa) return;
  const int p = (int)(i / dpa), f = (int)(i % dpa);
  const float v = (p < P && f < d) ? piv[(size_t)p * d + f] : 0.0f;
  out[i] = __bfloat16_as_ushort(__float2bfloat16_rn(v));
}

// D (16 x 8, fp32) += A (16 x 16, bf16, row major) * B (16 x 8, bf16, column major)
__device__ __forceinline__ void mma_16816(float (&c)[4], const uint32_t (&a)[4], uint32_t b0,
                                          uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, "
      "{%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// 128 queries per block: argmin_p ||p||^2 - 2 <y_q, p> with bf16 operands and
// fp32 accumulation.  Warp w takes queries [32w, 32w + 32) (two 16-row
// fragments) against each 64-pivot tile (eight 8-column fragments), the
// features streamed through shared memory 64 at a time.  In a fragment of D,
// lane (g = lane / 4, t = lane % 4) holds rows g and g + 8, columns 2t and
// 2t + 1; it sees its pivots in ascending order and the quad's reduction
// prefers the smaller pivot on equal values, so keys are deterministic.
__global__ void __launch_bounds__(kAssignThreads)
    assign_kernel(const float* __restrict__ Q, int64_t m, int d, const float* __restrict__ center,
                  const uint16_t* __restrict__ piv_h, int dpa, const float* __restrict__ pnorm,
                  int P, int* __restrict__ key, int* __restrict__ hist) {
  __shared__ __align__(16) uint16_t sq[kAssignThreads][kMmaLd];
  __shared__ __align__(16) uint16_t sp[kMmaP][kMmaLd];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int64_t q0 = (int64_t)blockIdx.x * kAssignThreads;
  const int P_pad = (P + kMmaP - 1) / kMmaP * kMmaP;
  float best[4];  // rows 32w + 16 (i / 2) + g + 8 (i % 2)
  int best_p[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    best[i] = INFINITY;
    best_p[i] = 0;
  }
  for (int p0 = 0; p0 < P_pad; p0 += kMmaP) {
    float acc[2][8][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 8; ++b)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0f;
    for (int k0 = 0; k0 < dpa; k0 += kMmaK) {
      __syncthreads();
      // coalesced: consecutive threads read consecutive features of one query
      for (int i = threadIdx.x; i < kAssignThreads * kMmaK; i += kAssignThreads) {
        const int r = i / kMmaK, k = i % kMmaK;
        const int64_t qr = q0 + r;
        const int f = k0 + k;
        const float y = (qr < m && f < d) ? Q[qr * d + f] - center[f] : 0.0f;
        sq[r][k] = __bfloat16_as_ushort(__float2bfloat16_rn(y));
      }
      for (int i = threadIdx.x; i < kMmaP * (kMmaK / 8); i += kAssignThreads) {
        const int r = i / (kMmaK / 8), c8 = i % (kMmaK / 8);
        *reinterpret_cast<uint4*>(&sp[r][c8 * 8]) =
            *reinterpret_cast<const uint4*>(piv_h + (size_t)(p0 + r) * dpa + k0 + c8 * 8);
      }
      __syncthreads();
#pragma unroll
      for (int kk = 0; kk < kMmaK; kk += 16) {
        uint32_t a[2][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
          const int r = 32 * w + 16 * mt + g;
          a[mt][0] = *reinterpret_cast<const uint32_t*>(&sq[r][kk + 2 * t]);
          a[mt][1] = *reinterpret_cast<const uint32_t*>(&sq[r + 8][kk + 2 * t]);
          a[mt][2] = *reinterpret_cast<const uint32_t*>(&sq[r][kk + 2 * t + 8]);
          a[mt][3] = *reinterpret_cast<const uint32_t*>(&sq[r + 8][kk + 2 * t + 8]);
        }
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
          const uint32_t b0 = *reinterpret_cast<const uint32_t*>(&sp[8 * nt + g][kk + 2 * t]);
          const uint32_t b1 = *reinterpret_cast<const uint32_t*>(&sp[8 * nt + g][kk + 2 * t + 8]);
          mma_16816(acc[0][nt], a[0], b0, b1);
          mma_16816(acc[1][nt], a[1], b0, b1);
        }
      }
    }
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int pj = p0 + 8 * nt + 2 * t + (e & 1);
        if (pj < P) {
          const float pn = pnorm[pj];
#pragma unroll
          for (int mt = 0; mt < 2; ++mt) {
            const int i = 2 * mt + (e >> 1);
            const float v = fmaf(-2.0f, acc[mt][nt][e], pn);
            if (v < best[i]) {
              best[i] = v;
              best_p[i] = pj;
            }
          }
        }
      }
  }
  // the quad's four lanes hold different pivots of the same rows
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int o = 1; o < 4; o <<= 1) {
      const float ov = __shfl_xor_sync(0xffffffffu, best[i], o);
      const int op = __shfl_xor_sync(0xffffffffu, best_p[i], o);
      if (ov < best[i] || (ov == best[i] && op < best_p[i])) {
        best[i] = ov;
        best_p[i] = op;
      }
    }
  if (t == 0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int64_t q = q0 + 32 * w + 16 * (i >> 1) + g + 8 * (i & 1);
      if (q < m) {
        key[q] = best_p[i];
        atomicAdd(hist + best_p[i], 1);
      }
    }
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

int pivot_rows_padded(int P) { return (P + kMmaP - 1) / kMmaP * kMmaP; }
int pivot_dims_padded(int d) { return (d + kMmaK - 1) / kMmaK * kMmaK; }

void launch_pivots(Index* ix, cudaStream_t st) {
  pivot_rows_kernel<<<ix->n_pivots, 32, 0, st>>>(ix->X, ix->n, ix->d, ix->n_pivots, ix->center,
                                                 ix->pivots, ix->pivot_norms);
  const int64_t total = (int64_t)pivot_rows_padded(ix->n_pivots) * ix->pivot_dpa;
  pivots_bf16_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(
      ix->pivots, ix->n_pivots, ix->d, pivot_rows_padded(ix->n_pivots), ix->pivot_dpa,
      ix->pivots_h);
}

void launch_assign_rows(const Index* ix, const float* X, int64_t n, int* key, int* hist,
                        cudaStream_t st) {
  cudaMemsetAsync(hist, 0, (size_t)ix->n_pivots * sizeof(int), st);
  assign_kernel<<<(unsigned)((n + kAssignThreads - 1) / kAssignThreads), kAssignThreads, 0, st>>>(
      X, n, ix->d, ix->center, ix->pivots_h, ix->pivot_dpa, ix->pivot_norms, ix->n_pivots, key,
      hist);
}

void launch_query_order(const Index* ix, const float* Q, int64_t m, int* key, int* hist,
                        int* perm, float* Qp, cudaStream_t st) {
  const int P = ix->n_pivots;
  cudaMemsetAsync(hist, 0, (size_t)P * sizeof(int), st);
  assign_kernel<<<(unsigned)((m + kAssignThreads - 1) / kAssignThreads), kAssignThreads, 0, st>>>(
      Q, m, ix->d, ix->center, ix->pivots_h, ix->pivot_dpa, ix->pivot_norms, P, key, hist);
  bin_scan_kernel<<<1, 32, 0, st>>>(hist, P);
  scatter_kernel<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(key, m, hist, perm);
  gather_rows_kernel<<<(unsigned)((m + 7) / 8), 256, 0, st>>>(Q, perm, m, ix->d, Qp);
}

}  // namespace b2k
