// Exact squared-distance keys for float32 coordinates (device side).
//
// Every float32 is an integer multiple of 2^-149, so for a query q and a
// training row x the value S(q,x) * 2^298 = sum_i D_i^2, with D_i the exact
// integer difference (q_i - x_i) * 2^149, is an exact non-negative integer of
// at most 587 bits.  The key holds it in ten 64-bit limbs.  Comparing keys
// orders training rows by their exact real squared distance, which is the
// order mlxlearn's neighbour path defines (reference
// src/mlxlearn/_kernels/_neighbors_cpu_native.cpp:170-190 and
// src/mlxlearn/_kernels/radius_contract.py:155-198).  Only near-tie
// candidates whose float64 intervals overlap ever reach this code.
#pragma once
#include <cstdint>

namespace b2k {

constexpr int kKeyLimbs = 10;

struct ExactKey {
  uint64_t w[kKeyLimbs];
};

__device__ __forceinline__ void f32_decode(float v, uint64_t& m, int& e, int& neg) {
  uint32_t b = __float_as_uint(v);
  uint32_t ex = (b >> 23) & 255u;
  m = (uint64_t)((b & 0x7fffffu) | (ex ? 0x800000u : 0u));
  e = ex ? (int)ex - 1 : 0;
  neg = (int)(b >> 31);
}

// acc += v << shift, v has nv limbs (nv <= 10).
__device__ __forceinline__ void key_add_shifted(ExactKey& acc, const uint64_t* v, int nv,
                                                int shift) {
  int base = shift >> 6, bit = shift & 63;
  uint64_t carry = 0;
  for (int i = 0; i + base < kKeyLimbs; ++i) {
    uint64_t part = 0;
    if (i < nv) part = v[i] << bit;
    if (bit && i > 0 && i - 1 < nv) part |= v[i - 1] >> (64 - bit);
    uint64_t a = acc.w[i + base];
    uint64_t s = a + part;
    uint64_t c1 = s < a;
    uint64_t s2 = s + carry;
    uint64_t c2 = s2 < s;
    acc.w[i + base] = s2;
    carry = c1 + c2;
    if (i >= nv && !carry) break;
  }
}

// dst (5 limbs) = m << shift, m < 2^24, shift <= 253.
__device__ __forceinline__ void big5_shifted(uint64_t* dst, uint64_t m, int shift) {
#pragma unroll
  for (int i = 0; i < 5; ++i) dst[i] = 0;
  int limb = shift >> 6, bit = shift & 63;
  dst[limb] = m << bit;
  if (bit && limb + 1 < 5) dst[limb + 1] = m >> (64 - bit);
}

__device__ __forceinline__ int big5_cmp(const uint64_t* a, const uint64_t* b) {
  for (int i = 4; i >= 0; --i)
    if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
  return 0;
}

__device__ __forceinline__ void big5_sub(uint64_t* r, const uint64_t* a, const uint64_t* b) {
  uint64_t borrow = 0;
  for (int i = 0; i < 5; ++i) {
    uint64_t bi = b[i] + borrow;
    uint64_t nb = (bi < borrow) || (a[i] < bi);
    r[i] = a[i] - bi;
    borrow = nb;
  }
}

__device__ __forceinline__ void big5_add(uint64_t* r, const uint64_t* a, const uint64_t* b) {
  uint64_t carry = 0;
  for (int i = 0; i < 5; ++i) {
    uint64_t s = a[i] + b[i];
    uint64_t c1 = s < a[i];
    uint64_t s2 = s + carry;
    uint64_t c2 = s2 < s;
    r[i] = s2;
    carry = c1 + c2;
  }
}

// Exact key of S(q, x) for d features.
static __device__ __noinline__ void exact_key(const float* __restrict__ q, const float* __restrict__ x,
                                       int d, ExactKey& out) {
  for (int i = 0; i < kKeyLimbs; ++i) out.w[i] = 0;
  for (int i = 0; i < d; ++i) {
    uint64_t ma, mb;
    int ea, eb, na, nb;
    f32_decode(q[i], ma, ea, na);
    f32_decode(x[i], mb, eb, nb);
    if (!ma && !mb) continue;
    int e0 = ea < eb ? ea : eb;
    uint64_t D[5];
    if (ea - e0 <= 39 && eb - e0 <= 39) {
      // Fast path: both aligned significands fit in 63 bits.
      int64_t A = (int64_t)(ma << (ea - e0));
      int64_t B = (int64_t)(mb << (eb - e0));
      if (na) A = -A;
      if (nb) B = -B;
      // |A - B| < 2^64
      uint64_t diff = (A >= B) ? (uint64_t)A - (uint64_t)B : (uint64_t)B - (uint64_t)A;
      if (!diff) continue;
      uint64_t sq[2] = {diff * diff, __umul64hi(diff, diff)};
      key_add_shifted(out, sq, sq[1] ? 2 : 1, 2 * e0);
      continue;
    }
    uint64_t A[5], B[5];
    big5_shifted(A, ma, ea - e0);
    big5_shifted(B, mb, eb - e0);
    if (na == nb) {
      if (big5_cmp(A, B) >= 0) big5_sub(D, A, B);
      else big5_sub(D, B, A);
    } else {
      big5_add(D, A, B);
    }
    int nd = 5;
    while (nd > 0 && D[nd - 1] == 0) --nd;
    if (!nd) continue;
    uint64_t sq[10];
    for (int t = 0; t < 10; ++t) sq[t] = 0;
    for (int a = 0; a < nd; ++a) {
      uint64_t carry = 0;
      for (int b = 0; b < nd; ++b) {
        // t = D[a]*D[b] + sq[a+b] + carry (< 2^128)
        uint64_t lo = D[a] * D[b];
        uint64_t hi = __umul64hi(D[a], D[b]);
        uint64_t s = lo + sq[a + b];
        hi += s < lo;
        uint64_t s2 = s + carry;
        hi += s2 < s;
        sq[a + b] = s2;
        carry = hi;
      }
      int pos = a + nd;
      while (carry && pos < 10) {
        uint64_t s = sq[pos] + carry;
        carry = s < carry;
        sq[pos] = s;
        ++pos;
      }
    }
    int ns = 2 * nd;
    while (ns > 0 && sq[ns - 1] == 0) --ns;
    key_add_shifted(out, sq, ns, 2 * e0);
  }
}

__device__ __forceinline__ int key_cmp(const ExactKey& a, const ExactKey& b) {
  for (int i = kKeyLimbs - 1; i >= 0; --i)
    if (a.w[i] != b.w[i]) return a.w[i] < b.w[i] ? -1 : 1;
  return 0;
}

// Exact sign of S(q,a) - S(q,b).  Bitwise-identical rows are equal without
// forming keys (duplicated training rows are the common source of ties).
static __device__ __noinline__ int exact_compare(const float* q, const float* a, const float* b, int d) {
  bool same = true;
  for (int i = 0; i < d && same; ++i) same = __float_as_uint(a[i]) == __float_as_uint(b[i]);
  if (same) return 0;
  ExactKey ka, kb;
  exact_key(q, a, d, ka);
  exact_key(q, b, d, kb);
  return key_cmp(ka, kb);
}

}  // namespace b2k
