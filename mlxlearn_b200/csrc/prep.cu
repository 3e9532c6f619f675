// Index and query preparation kernels.
//
// Both screens work on centred coordinates y = x - c (c = fl32 of the mean of
// the training rows, as the reference centres its Gram screen,
// src/mlxlearn_device/_neighbors.py:232-239): distances are translation
// invariant, and centring keeps the Gram cancellation error proportional to
// the spread of the data instead of its offset.
//
// A screen compares v = fl32(||y_x||^2) - 2 <q^, x^> (q^, x^ = the fp32 or
// bf16 operands of y_q, y_x) against a per-query threshold.  Each query gets
// a certified bound E with |S(q,x) - (||y_q||^2 + v)| <= E, where S is the
// exact squared distance, built from norms measured here (the pattern of the
// reference's compact screen, src/mlxlearn_device/_neighbors_compact.py:83-88,
// and its Gram lower bound, src/mlxlearn_device/_neighbors_general.py:188-242):
//
//   e = y - y^ (operand rounding, measured in float64), u = 2^-24,
//   E = 2(|q^||e_x| + |e_q||x^| + |e_q||e_x|)      operand rounding
//     + 2 g |q^||x^|                               dot-product accumulation
//     + 2u ||y_x||^2 + 2u |q^||x^| (1.01)          stored norm + final add
//     + 2^-50 ||y_q||^2,  times (1 + 2^-16), plus dp 2^-120 for underflow,
// with the x-side norms replaced by their maxima over the index and
//   g = (d + 4) u (1.01)          fp32 FMA chains (CUDA-core screen),
//   g = (dp + 16) 2^-20           tcgen05 fp32 accumulation (16 ulp per add).
// The tf32 screen (kind::tf32) works the same way on operands rounded to
// tf32 here (10 explicit mantissa bits, so the tensor core reads them
// exactly) with the norm split into three tf32 parts in 8 columns; its
// measured operand errors are about 8x smaller than bf16's.
#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"
#include "internal.cuh"

namespace b2k {

namespace {

// Screen inputs must avoid fp32 overflow of products/norms: every coordinate
// is 0 or has magnitude in [2^-60, 2^50] (the reference's FP32 Gram screen
// has the same kind of guard, src/mlxlearn/_kernels/radius_contract.py:46-50).
__device__ __forceinline__ bool coord_in_range(float v) {
  uint32_t a = __float_as_uint(v) & 0x7fffffffu;
  return a == 0 || (a >= (67u << 23) && a <= (177u << 23));
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// positive float max via integer atomics (bit patterns of non-negative floats are ordered)
__device__ __forceinline__ void atomic_max_pos(float* addr, float v) {
  atomicMax(reinterpret_cast<int*>(addr), __float_as_int(v));
}

// Column sums of X (float64), accumulated per block then atomically.
__global__ void column_sum_kernel(const float* __restrict__ X, int64_t n, int d,
                                  int64_t rows_per_block, double* __restrict__ sums) {
  const int64_t r0 = (int64_t)blockIdx.x * rows_per_block;
  const int64_t r1 = min(n, r0 + rows_per_block);
  for (int c = threadIdx.x; c < d; c += blockDim.x) {
    double s = 0.0;
    for (int64_t r = r0; r < r1; ++r) s += (double)X[r * d + c];
    atomicAdd(sums + c, s);
  }
}

__global__ void center_kernel(const double* __restrict__ sums, int64_t n, int d,
                              float* __restrict__ center) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < d) center[c] = (float)(sums[c] / (double)n);
}

// stats: [0] max |x^| fp32 operand, [1] max ||y||^2, [2] range violations (int),
//        [3] max |x~| bf16 operand, [4] max |e| bf16, [5] max |e| fp32,
//        [6] max |x~| tf32 operand, [7] max |e| tf32
__global__ void prep_index_kernel(const float* __restrict__ X, int64_t n, int d,
                                  const float* __restrict__ center, float* __restrict__ nx32,
                                  double* __restrict__ nx64, float* __restrict__ stats) {
  int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  int lane = threadIdx.x & 31;
  if (row >= n) return;
  const float* x = X + row * d;
  double yy = 0.0, hh = 0.0, ee = 0.0;
  bool ok = true;
  for (int i = lane; i < d; i += 32) {
    const float v = x[i];
    ok &= coord_in_range(v);
    const double y = (double)v - (double)center[i];
    const float h = v - center[i];  // fp32 operand of the CUDA-core screen
    const double e = y - (double)h;
    yy += y * y;
    hh += (double)h * (double)h;
    ee += e * e;
  }
  yy = warp_sum(yy);
  hh = warp_sum(hh);
  ee = warp_sum(ee);
  ok = __all_sync(0xffffffffu, ok);
  if (lane == 0) {
    nx64[row] = yy;
    nx32[row] = (float)yy;
    atomic_max_pos(stats + 0, __double2float_ru(sqrt(hh) * (1.0 + 1e-15)));
    atomic_max_pos(stats + 1, __double2float_ru(yy * (1.0 + 1e-15)));
    atomic_max_pos(stats + 5, __double2float_ru(sqrt(ee) * (1.0 + 1e-15) + 0x1p-50 * sqrt(yy)));
    if (!ok) atomicAdd(reinterpret_cast<int*>(stats + 2), 1);
  }
}

__global__ void prep_index_bf16_kernel(const float* __restrict__ X, int64_t n, int d,
                                       int64_t n_pad, int dp, const float* __restrict__ center,
                                       const int* __restrict__ rows,
                                       __nv_bfloat16* __restrict__ Xh,
                                       float* __restrict__ stats) {
  int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  int lane = threadIdx.x & 31;
  if (row >= n_pad) return;
  __nv_bfloat16* xh = Xh + row * dp;
  if (row >= n) {
    // padding rows: zero operands (their NaN norm column keeps them out)
    for (int i = lane; i < dp; i += 32) xh[i] = __float2bfloat16_rn(0.0f);
    return;
  }
  const float* x = X + (rows ? (int64_t)rows[row] : row) * d;
  double hn = 0.0, en = 0.0, yy = 0.0;
  for (int i = lane; i < dp; i += 32) {
    const float v = i < d ? x[i] : 0.0f;
    const float c = i < d ? center[i] : 0.0f;
    const double y = (double)v - (double)c;
    const __nv_bfloat16 h = __float2bfloat16_rn(v - c);
    xh[i] = h;
    const double hv = (double)__bfloat162float(h);
    const double e = y - hv;
    hn += hv * hv;
    en += e * e;
    yy += y * y;
  }
  hn = warp_sum(hn);
  en = warp_sum(en);
  yy = warp_sum(yy);
  if (lane == 0) {
    atomic_max_pos(stats + 3, __double2float_ru(sqrt(hn) * (1.0 + 1e-15)));
    atomic_max_pos(stats + 4, __double2float_ru(sqrt(en) * (1.0 + 1e-15) + 0x1p-50 * sqrt(yy)));
  }
}

// tf32 operand rows of the index (row i from training row rows[i]).
__global__ void prep_index_tf32_kernel(const float* __restrict__ X, int64_t n, int d,
                                       int64_t n_pad, int dpt, const float* __restrict__ center,
                                       const int* __restrict__ rows, float* __restrict__ Xt,
                                       float* __restrict__ stats) {
  int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  int lane = threadIdx.x & 31;
  if (row >= n_pad) return;
  float* xt = Xt + row * dpt;
  if (row >= n) {
    for (int i = lane; i < dpt; i += 32) xt[i] = 0.0f;
    return;
  }
  const float* x = X + (rows ? (int64_t)rows[row] : row) * d;
  double hn = 0.0, en = 0.0, yy = 0.0;
  for (int i = lane; i < dpt; i += 32) {
    const float v = i < d ? x[i] : 0.0f;
    const float c = i < d ? center[i] : 0.0f;
    const double y = (double)v - (double)c;
    const float h = tf32_rne(v - c);
    xt[i] = h;
    const double e = y - (double)h;
    hn += (double)h * (double)h;
    en += e * e;
    yy += y * y;
  }
  hn = warp_sum(hn);
  en = warp_sum(en);
  yy = warp_sum(yy);
  if (lane == 0) {
    atomic_max_pos(stats + 6, __double2float_ru(sqrt(hn) * (1.0 + 1e-15)));
    atomic_max_pos(stats + 7, __double2float_ru(sqrt(en) * (1.0 + 1e-15) + 0x1p-50 * sqrt(yy)));
  }
}

// Norm columns of the tf32 screen: ||y_x||^2 as three tf32 parts (residual
// below 2^-33 of the value), NaN on padding rows; query side [1, 1, 1, 0...].
__global__ void prep_aug_tf32_kernel(const double* __restrict__ nx64, int64_t n, int64_t n_pad,
                                     const int* __restrict__ rows, float* __restrict__ Xtaug,
                                     float* __restrict__ ones) {
  const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ones && row < kTcBM) {
    for (int c = 0; c < kTcAugF; ++c) ones[row * kTcAugF + c] = c < 3 ? 1.0f : 0.0f;
  }
  if (row >= n_pad) return;
  float* a = Xtaug + row * kTcAugF;
  for (int c = 3; c < kTcAugF; ++c) a[c] = 0.0f;
  if (row >= n) {
    a[0] = __uint_as_float(0x7fc00000u);
    a[1] = 0.0f;
    a[2] = 0.0f;
    return;
  }
  const double v = nx64[rows ? (int64_t)rows[row] : row];
  const float hi = tf32_rne((float)v);
  const double r1 = v - (double)hi;
  const float mid = tf32_rne((float)r1);
  const double r2 = r1 - (double)mid;
  a[0] = hi;
  a[1] = mid;
  a[2] = tf32_rne((float)r2);
}

// Norm columns for the tensor-core screen: ||y_x||^2 (float64) as three bf16
// parts hi + mid + lo (residual below 2^-26 of the value), NaN on padding
// rows; the query side is [1, 1, 1, 0, ...].
__global__ void prep_aug_kernel(const double* __restrict__ nx64, int64_t n, int64_t n_pad,
                                const int* __restrict__ rows,
                                __nv_bfloat16* __restrict__ Xaug,
                                __nv_bfloat16* __restrict__ ones) {
  const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ones && row < kTcBM) {
    for (int c = 0; c < kTcAug; ++c)
      ones[row * kTcAug + c] = __float2bfloat16_rn(c < 3 ? 1.0f : 0.0f);
  }
  if (row >= n_pad) return;
  __nv_bfloat16* a = Xaug + row * kTcAug;
  for (int c = 3; c < kTcAug; ++c) a[c] = __float2bfloat16_rn(0.0f);
  if (row >= n) {
    const __nv_bfloat16 nan = __ushort_as_bfloat16((unsigned short)0x7fc0);
    a[0] = nan;
    a[1] = __float2bfloat16_rn(0.0f);
    a[2] = __float2bfloat16_rn(0.0f);
    return;
  }
  const double v = nx64[rows ? (int64_t)rows[row] : row];
  const __nv_bfloat16 hi = __float2bfloat16_rn((float)v);
  const double r1 = v - (double)__bfloat162float(hi);
  const __nv_bfloat16 mid = __float2bfloat16_rn((float)r1);
  const double r2 = r1 - (double)__bfloat162float(mid);
  a[0] = hi;
  a[1] = mid;
  a[2] = __float2bfloat16_rn((float)r2);
}

// One query row: error bound E, the bf16 operand row (bf16 mode), ||y||^2.
__device__ __forceinline__ void prep_query_row(const PrepProblem& P, int64_t row, int lane) {
  const double u = 0x1p-24;
  const bool bf16 = P.mode == B2K_MODE_BF16;
  const bool tf32 = P.mode == B2K_MODE_TF32;
  const bool tc = bf16 || tf32;  // tensor-core screens: padded width, norm columns
  const int d = P.d, dp = P.dp;
  __nv_bfloat16* Ah = reinterpret_cast<__nv_bfloat16*>(P.Ah);
  if (row >= P.m) {
    if (bf16)
      for (int i = lane; i < dp; i += 32) Ah[row * dp + i] = __float2bfloat16_rn(0.0f);
    if (tf32)
      for (int i = lane; i < dp; i += 32) P.At[row * dp + i] = 0.0f;
    if (lane == 0) P.E[row] = 0.0f;
    return;
  }
  const float* q = P.Q + row * d;
  double yy = 0.0, hn = 0.0, en = 0.0;
  bool ok = true;
  const int width = tc ? dp : d;
  for (int i = lane; i < width; i += 32) {
    const float v = i < d ? q[i] : 0.0f;
    const float c = i < d ? P.center[i] : 0.0f;
    ok &= coord_in_range(v);
    const double y = (double)v - (double)c;
    const float h32 = v - c;
    double hv;
    if (bf16) {
      const __nv_bfloat16 h = __float2bfloat16_rn(h32);
      hv = (double)__bfloat162float(h);
      Ah[row * dp + i] = __float2bfloat16_rn(-2.0f * __bfloat162float(h));  // exact
    } else if (tf32) {
      const float h = tf32_rne(h32);
      hv = (double)h;
      P.At[row * dp + i] = -2.0f * h;  // exact
    } else {
      hv = (double)h32;
    }
    const double e = y - hv;
    yy += y * y;
    hn += hv * hv;
    en += e * e;
  }
  yy = warp_sum(yy);
  hn = warp_sum(hn);
  en = warp_sum(en);
  ok = __all_sync(0xffffffffu, ok);
  if (lane == 0) {
    const double qh = sqrt(hn) * (1.0 + 1e-15);
    const double eq = sqrt(en) * (1.0 + 1e-15) + 0x1p-50 * sqrt(yy);
    const double XH = P.xh_max, EX = P.ex_max, NX = P.nx_max;
    // tensor cores: dp feature columns + 16 norm columns accumulated in fp32;
    // the accumulation also carries ||y_x||^2 itself (the g * NX term)
    const double g = bf16   ? (double)(dp + kTcAug + 16) * 0x1p-20
                     : tf32 ? (double)(dp + kTcAugF + 16) * 0x1p-20
                            : (double)(d + 4) * u * 1.01;
    double bound = 2.0 * (qh * EX + eq * XH + eq * EX) + 2.0 * g * qh * XH + 2.0 * u * NX +
                   2.0 * u * qh * XH * 1.01 + 0x1p-50 * yy + (tc ? g * NX * 1.01 : 0.0);
    bound = bound * (1.0 + 0x1p-16) + (double)width * 0x1p-120;
    P.E[row] = __double2float_ru(bound);
    if (P.nq) P.nq[row] = yy;
    if (!ok) atomicOr(P.flags, 1);
  }
}

__global__ void prep_queries_kernel(const __grid_constant__ PrepProblem P) {
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (row >= P.m_pad) return;
  prep_query_row(P, row, threadIdx.x & 31);
}

// Batched form: rows of all problems back to back, problem p owning padded
// rows [row_start[p], row_start[p + 1]).
__global__ void prep_queries_batch_kernel(const PrepProblem* __restrict__ tab,
                                          const int64_t* __restrict__ row_start, int P,
                                          int64_t total) {
  const int64_t r = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (r >= total) return;
  const int p = problem_of(row_start, P, r);
  prep_query_row(tab[p], r - row_start[p], threadIdx.x & 31);
}

__global__ void nonfinite_kernel(const float* __restrict__ v, int64_t count, int* flag) {
  bool bad = false;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if ((reinterpret_cast<uintptr_t>(v) & 15) == 0) {
    const int64_t n4 = count / 4;
    const float4* v4 = reinterpret_cast<const float4*>(v);
    for (int64_t i = i0; i < n4; i += stride) {
      const float4 x = __ldg(v4 + i);
      bad |= ((__float_as_uint(x.x) & 0x7f800000u) == 0x7f800000u) |
             ((__float_as_uint(x.y) & 0x7f800000u) == 0x7f800000u) |
             ((__float_as_uint(x.z) & 0x7f800000u) == 0x7f800000u) |
             ((__float_as_uint(x.w) & 0x7f800000u) == 0x7f800000u);
    }
    for (int64_t i = 4 * n4 + i0; i < count; i += stride)
      bad |= (__float_as_uint(v[i]) & 0x7f800000u) == 0x7f800000u;
  } else {
    for (int64_t i = i0; i < count; i += stride)
      bad |= (__float_as_uint(v[i]) & 0x7f800000u) == 0x7f800000u;
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

}  // namespace

void launch_nonfinite_check(const float* v, int64_t count, int* flag, cudaStream_t st) {
  if (count <= 0) return;
  const int64_t blocks = std::min<int64_t>((count / 4 + 255) / 256 + 1, 4096);
  nonfinite_kernel<<<(unsigned)blocks, 256, 0, st>>>(v, count, flag);
}

void launch_prep_index(Index* ix, cudaStream_t st) {
  // about eight blocks per SM, at least 16 rows each
  const int64_t rows_per_block = std::max<int64_t>(16, (ix->n + 1183) / 1184);
  const int64_t blocks = (ix->n + rows_per_block - 1) / rows_per_block;
  cudaMemsetAsync(ix->colsum, 0, (size_t)ix->d * sizeof(double), st);
  column_sum_kernel<<<(unsigned)blocks, 128, 0, st>>>(ix->X, ix->n, ix->d, rows_per_block,
                                                      ix->colsum);
  center_kernel<<<(ix->d + 127) / 128, 128, 0, st>>>(ix->colsum, ix->n, ix->d, ix->center);
  const int warps = 8;
  prep_index_kernel<<<(unsigned)((ix->n + warps - 1) / warps), warps * 32, 0, st>>>(
      ix->X, ix->n, ix->d, ix->center, ix->nx32, ix->nx64, ix->stats_dev);
}

void launch_prep_index_bf16(const Index* ix, uint16_t* Xh, cudaStream_t st, const int* rows) {
  const int warps = 8;
  const int64_t n_pad = (ix->n + kTcBN - 1) / kTcBN * kTcBN;
  const int dp = (ix->d + kTcBK - 1) / kTcBK * kTcBK;
  const int64_t blocks = (n_pad + warps - 1) / warps;
  prep_index_bf16_kernel<<<(unsigned)blocks, warps * 32, 0, st>>>(
      ix->X, ix->n, ix->d, n_pad, dp, ix->center, rows, reinterpret_cast<__nv_bfloat16*>(Xh),
      ix->stats_dev);
}

void launch_prep_aug(const Index* ix, uint16_t* Xaug, uint16_t* ones, cudaStream_t st,
                     const int* rows) {
  const int64_t n_pad = (ix->n + kTcBN - 1) / kTcBN * kTcBN;
  const int64_t threads = n_pad > kTcBM ? n_pad : kTcBM;
  prep_aug_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
      ix->nx64, ix->n, n_pad, rows, reinterpret_cast<__nv_bfloat16*>(Xaug),
      reinterpret_cast<__nv_bfloat16*>(ones));
}

void launch_prep_index_tf32(const Index* ix, float* Xt, cudaStream_t st, const int* rows) {
  const int warps = 8;
  const int64_t n_pad = (ix->n + kTcBN - 1) / kTcBN * kTcBN;
  const int dpt = (ix->d + kTcBKf - 1) / kTcBKf * kTcBKf;
  const int64_t blocks = (n_pad + warps - 1) / warps;
  prep_index_tf32_kernel<<<(unsigned)blocks, warps * 32, 0, st>>>(ix->X, ix->n, ix->d, n_pad, dpt,
                                                                  ix->center, rows, Xt,
                                                                  ix->stats_dev);
}

void launch_prep_aug_tf32(const Index* ix, float* Xtaug, float* ones, cudaStream_t st,
                          const int* rows) {
  const int64_t n_pad = (ix->n + kTcBN - 1) / kTcBN * kTcBN;
  const int64_t threads = n_pad > kTcBM ? n_pad : kTcBM;
  prep_aug_tf32_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
      ix->nx64, ix->n, n_pad, rows, Xtaug, ones);
}

PrepProblem prep_problem(const Index* ix, const float* Q, int64_t m, int64_t m_pad, int mode,
                         const QueryPrep& qp) {
  const bool bf16 = mode == B2K_MODE_BF16;
  const bool tf32 = mode == B2K_MODE_TF32;
  PrepProblem P{};
  P.Q = Q;
  P.m = m;
  P.m_pad = m_pad;
  P.d = ix->d;
  P.dp = tf32 ? (ix->d + kTcBKf - 1) / kTcBKf * kTcBKf : (ix->d + kTcBK - 1) / kTcBK * kTcBK;
  P.mode = mode;
  P.center = ix->center;
  P.xh_max = bf16 ? ix->xh_max : tf32 ? ix->xt_max : ix->xn_max;
  P.nx_max = ix->nx_max;
  P.ex_max = bf16 ? ix->ex_max : tf32 ? ix->ext_max : ix->ex32_max;
  P.E = qp.E;
  P.Ah = qp.Ah;
  P.At = qp.At;
  P.nq = qp.nq;
  P.flags = qp.flags;
  return P;
}

void launch_prep_queries(const Index* ix, const float* Q, int64_t m, int64_t m_pad, int mode,
                         QueryPrep qp, cudaStream_t st) {
  const int warps = 8;
  const int64_t blocks = (m_pad + warps - 1) / warps;
  if (blocks == 0) return;
  prep_queries_kernel<<<(unsigned)blocks, warps * 32, 0, st>>>(
      prep_problem(ix, Q, m, m_pad, mode, qp));
}

void launch_prep_queries_batch(const PrepProblem* tab, const int64_t* row_start, int P,
                               int64_t total_rows, cudaStream_t st) {
  const int warps = 8;
  const int64_t blocks = (total_rows + warps - 1) / warps;
  if (blocks == 0) return;
  prep_queries_batch_kernel<<<(unsigned)blocks, warps * 32, 0, st>>>(tab, row_start, P,
                                                                       total_rows);
}

}  // namespace b2k
