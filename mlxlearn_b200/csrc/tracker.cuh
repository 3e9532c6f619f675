// Per-query candidate admission shared by the screen kernels.
//
// A screen computes, for query q and training row x, v = fl(-2<q,x> + ||x||^2)
// with a certified bound |S(q,x) - (||q||^2 + v)| <= E(q).  Each query row
// keeps, in registers, the KMAX smallest v seen so far (kv, ascending; the
// first KMAX-k slots hold -inf so kv[KMAX-1] is the k-th smallest), and the
// admission threshold T = kv[KMAX-1] + 2E rounded up.  Every v <= T is
// appended to the row's candidate list.
//
// Why the final lists certify the answer: let V_k be the k-th smallest v over
// all splits.  The k rows with the smallest v have S <= V_k + ||q||^2 + E, so
// the exact k-th distance D_k obeys D_k <= V_k + ||q||^2 + E.  A row that was
// not appended had v > T >= V_k + 2E at the time (T only decreases, and a
// split's k-th smallest is >= the global one), hence
// S >= v + ||q||^2 - E > V_k + ||q||^2 + E >= D_k: it is strictly farther than
// the k-th neighbour and cannot enter the answer, not even by the index
// tie rule.  The re-rank therefore only needs the entries with v <= V_k + 2E.
// This replaces the reference's per-tile "omitted barrier" certificate
// (src/mlxlearn_device/_neighbors_screen.py:78-217,
//  src/mlxlearn/_kernels/neighbors_cpu.py:314-364) with a streaming form.
#pragma once
#include <cstdint>

#include "common.cuh"

namespace b2k {

template <int KMAX>
struct RowTracker {
  float kv[KMAX];
  float T;
  float E2;
  int cnt;
  int self;
  int cap;
  int2* list;

  B2K_DEV void init(int k, float E, int self_col, int2* lst, int cap_) {
#pragma unroll
    for (int i = 0; i < KMAX; ++i) kv[i] = (i < KMAX - k) ? -INFINITY : INFINITY;
    T = INFINITY;
    E2 = __fmul_ru(2.0f, E);
    cnt = 0;
    self = self_col;
    list = lst;
    cap = cap_;
  }

  // Caller guarantees v <= T and col is not the excluded self column.
  B2K_DEV void admit(float v, int col) {
    if (cnt < cap) list[cnt] = make_int2(__float_as_int(v), col);
    ++cnt;
    if (v < kv[KMAX - 1]) {
#pragma unroll
      for (int i = KMAX - 1; i > 0; --i) kv[i] = fminf(kv[i], fmaxf(kv[i - 1], v));
      kv[0] = fminf(kv[0], v);
      T = __fadd_ru(kv[KMAX - 1], E2);
    }
  }

  // Offer 32 consecutive columns col0.. whose values are in v[]; `spill` is
  // this thread's 33-float scratch in shared memory (slow path only).
  B2K_DEV void offer32(const float (&v)[32], int col0, float* spill) {
    float a[11];
#pragma unroll
    for (int i = 0; i < 10; ++i) a[i] = min3f(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
    a[10] = fminf(v[30], v[31]);
    float b0 = min3f(a[0], a[1], a[2]), b1 = min3f(a[3], a[4], a[5]);
    float b2 = min3f(a[6], a[7], a[8]), b3 = fminf(a[9], a[10]);
    float mn = fminf(min3f(b0, b1, b2), b3);
    if (mn <= T) {
      // T only decreases while admitting, so `mask` is a superset of the
      // columns that will be admitted.
      uint32_t mask = 0;
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        mask |= (v[i] <= T ? 1u : 0u) << i;
        spill[i] = v[i];
      }
      while (mask) {
        const int i = __ffs(mask) - 1;
        mask &= mask - 1;
        const float x = spill[i];
        if (x <= T && col0 + i != self) admit(x, col0 + i);
      }
    }
  }

  // k smallest values seen (ascending) to out[0..k).
  B2K_DEV void write_kth(float* out, int k) const {
#pragma unroll
    for (int i = 0; i < KMAX; ++i)
      if (i >= KMAX - k) out[i - (KMAX - k)] = kv[i];
  }
};

}  // namespace b2k
