// Certification, float64 re-rank and exact tie resolution.
//
// certify_kernel (one warp per query) turns the screen's candidate lists into
// the final answer:
//   1. V_k = k-th smallest screen value over all splits (bisection over the
//      splits' k smallest values); threshold Tf = V_k + 2E (rounded up).
//   2. Candidates = list entries with v <= Tf (tracker.cuh proves that no other
//      row can be in the answer).
//   3. fp32 refinement with a certified relative bound, in two stages when
//      the query's squared norm is known: first the k candidates with the
//      smallest screen values, whose k-th smallest upper bound U0 then drops
//      every other candidate whose screen lower bound (||y_q||^2 + v - E)
//      exceeds it -- such a row cannot reach the top k -- and only the rest
//      are refined.  The survivors are those whose fp32 lower bound reaches
//      the k-th smallest fp32 upper bound.
//   3b. Canonical float64 squared distance of each survivor (strictly
//      sequential, no FMA: bit-identical to the host canonical value).
//   4. Sort by (value, index); within every run of neighbours whose float64
//      error intervals overlap (and which reaches into the first k), order by
//      the exact integer key (exact.cuh), ties by index.
// Queries whose lists overflowed go to exact_kernel.
//
// Replaces the reference's refine / certify / exact-order passes
// (src/mlxlearn_device/_neighbors_fused.py:545-834,
//  _neighbors_shortlist.py:16-170, _neighbors_precision.py:9-259) and its
// partitioned exact fallback (_neighbors_fallback.py:62-298).
#include <cfloat>

#include "common.cuh"
#include "exact.cuh"
#include "internal.cuh"

namespace b2k {

namespace {

constexpr int kCertWarps = 8;
constexpr int kSurvivorCap = 256;  // candidates that can still reach the top k
constexpr size_t kCertWarpBytes =
    (size_t)kCertifyCap * (sizeof(int) + sizeof(float)) +
    (size_t)kSurvivorCap * (sizeof(double) + sizeof(int)) + 256 * sizeof(unsigned);

// |canonical - S| <= g S with g = (d+2)u/(1-(d+2)u), u = 2^-53, for a
// sequential sum of d non-negative rounded terms (reference
// src/mlxlearn/_kernels/radius_contract.py:16-25); intervals use 2g.
__device__ __forceinline__ double interval_g2(int d) {
  const double u = 0x1p-53;
  return 2.0 * (double)(d + 2) * u / (1.0 - (double)(d + 2) * u);
}

__device__ __forceinline__ uint32_t float_key(float f) {
  uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// Ascending (s, id) bitonic sort of P (power of two) entries by one warp.
__device__ void warp_bitonic(double* s, int* id, int P, int lane) {
  for (int size = 2; size <= P; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = lane; t < P / 2; t += 32) {
        const int i = 2 * t - (t & (stride - 1));
        const int j = i + stride;
        const bool up = (i & size) == 0;
        const double a = s[i], b = s[j];
        const int ia = id[i], ib = id[j];
        const bool gt = (a > b) || (a == b && ia > ib);
        if (gt == up) {
          s[i] = b;
          s[j] = a;
          id[i] = ib;
          id[j] = ia;
        }
      }
      __syncwarp();
    }
  }
}

// Sort C candidates (padded to a power of two P) and fix the order of every
// near-tie run that starts inside the first k.  Runs only lane 0 for the
// exact part.  Returns the number of exact comparisons made.
__device__ unsigned warp_sort_resolve(double* s, int* id, int C, int k, const float* q,
                                      const float* X, int d, int lane) {
  int P = 2;
  while (P < C) P <<= 1;
  for (int i = C + lane; i < P; i += 32) {
    s[i] = DBL_MAX;
    id[i] = INT_MAX;
  }
  __syncwarp();
  warp_bitonic(s, id, P, lane);
  unsigned compares = 0;
  if (lane == 0) {
    const double g2 = interval_g2(d);
    const double lo_f = 1.0 - g2, hi_f = 1.0 + g2;
    int i = 0;
    while (i < k && i < C) {
      int j = i + 1;
      while (j < C && __dmul_rd(s[j], lo_f) <= __dmul_ru(s[j - 1], hi_f)) ++j;
      if (j - i > 1 && s[j - 1] != 0.0) {
        // exact insertion sort of the run [i, j)
        for (int a = i + 1; a < j; ++a) {
          const double sa = s[a];
          const int ia = id[a];
          int b = a;
          while (b > i) {
            const int ib = id[b - 1];
            int c = exact_compare(q, X + (size_t)ia * d, X + (size_t)ib * d, d);
            ++compares;
            if (c > 0 || (c == 0 && ia > ib)) break;
            s[b] = s[b - 1];
            id[b] = ib;
            --b;
          }
          s[b] = sa;
          id[b] = ia;
        }
      }
      i = j;
    }
  }
  __syncwarp();
  return compares;
}

// k-th smallest (1-based) of `count` unsigned keys, by one warp: four 8-bit
// radix passes with a 256-bin shared-memory histogram (`hist`).
// `visit(f)` calls f(key) for every key this lane owns.
template <class Visit>
__device__ uint32_t warp_radix_select(Visit visit, int k, unsigned* hist, int lane) {
  uint32_t prefix = 0, mask = 0;
  unsigned rank = (unsigned)k;
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int b = lane; b < 256; b += 32) hist[b] = 0;
    __syncwarp();
    visit([&](uint32_t key) {
      if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 255u], 1u);
    });
    __syncwarp();
    unsigned local[8], s = 0;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      local[b] = hist[lane * 8 + b];
      s += local[b];
    }
    unsigned incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    const unsigned excl = incl - s;
    const unsigned owners = __ballot_sync(0xffffffffu, excl < rank && rank <= incl);
    const int owner = __ffs(owners) - 1;
    int digit = 0;
    unsigned before = 0;
    if (lane == owner) {
      unsigned acc = excl;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        if (acc + local[b] >= rank) {
          digit = lane * 8 + b;
          break;
        }
        acc += local[b];
      }
      before = acc;
    }
    digit = __shfl_sync(0xffffffffu, digit, owner);
    before = __shfl_sync(0xffffffffu, before, owner);
    rank -= before;
    prefix |= (uint32_t)digit << shift;
    mask |= 255u << shift;
    __syncwarp();
  }
  return prefix;
}

// k-th smallest (1-based, k <= n) of n <= 32 keys, lane l holding key l
// (lanes >= n hold anything): every lane counts the keys below its own (ties
// by lane), and the lane of rank k - 1 holds the answer.
__device__ __forceinline__ uint32_t warp_kth_32(uint32_t key, int n, int k, int lane) {
  int rank = 0;
#pragma unroll 8
  for (int j = 0; j < 32; ++j) {
    const uint32_t o = __shfl_sync(0xffffffffu, key, j);
    rank += (j < n && (o < key || (o == key && j < lane))) ? 1 : 0;
  }
  const unsigned hit = __ballot_sync(0xffffffffu, lane < n && rank == k - 1);
  return __shfl_sync(0xffffffffu, key, __ffs(hit) - 1);
}

template <class KeyFn>
__device__ uint32_t warp_radix_kth(KeyFn key_of, int count, int k, unsigned* hist, int lane) {
  return warp_radix_select(
      [&](auto f) {
        for (int i = lane; i < count; i += 32) f(key_of(i));
      },
      k, hist, lane);
}

// fp32 direct squared distance of candidate rows, 8 lanes per row (coalesced
// 16-byte loads), so each warp handles 4 candidates per step.  Sum of d
// non-negative terms, each (fl(q_i - x_i))^2 accumulated with FMA: the result
// is within (d + 5) u (1.01) S + d 2^-126 of the exact S, u = 2^-24, whatever
// the order of the additions.
// Vectorised form for d <= 32 NI (16-byte aligned rows): the query's pieces
// stay in registers, and each 8-lane group loads UNR candidate rows before
// using any of them, so a warp keeps 4 UNR rows of loads in flight.
template <int NI, int UNR>
__device__ __forceinline__ void refine_vec(const float* __restrict__ q,
                                           const float* __restrict__ X, int d, const int* ci,
                                           float* cv, int C, int lane) {
  const int grp = lane >> 3, l8 = lane & 7;
  const int d4 = d / 4;
  const float4* q4 = reinterpret_cast<const float4*>(q);
  float4 qr[NI];
#pragma unroll
  for (int i = 0; i < NI; ++i) {
    const int f = l8 + 8 * i;
    qr[i] = f < d4 ? __ldg(q4 + f) : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  for (int c0 = 0; c0 < C; c0 += 4 * UNR) {
    float4 b[UNR][NI];
#pragma unroll
    for (int u = 0; u < UNR; ++u) {
      const int c = c0 + 4 * u + grp;
      const float4* x4 =
          reinterpret_cast<const float4*>(X + (size_t)(c < C ? ci[c] : ci[0]) * d);
#pragma unroll
      for (int i = 0; i < NI; ++i) {
        const int f = l8 + 8 * i;
        b[u][i] = (c < C && f < d4) ? __ldg(x4 + f) : qr[i];
      }
    }
#pragma unroll
    for (int u = 0; u < UNR; ++u) {
      float acc0 = 0.f, acc1 = 0.f;
#pragma unroll
      for (int i = 0; i < NI; ++i) {
        const float e0 = qr[i].x - b[u][i].x, e1 = qr[i].y - b[u][i].y;
        const float e2 = qr[i].z - b[u][i].z, e3 = qr[i].w - b[u][i].w;
        acc0 = fmaf(e0, e0, acc0);
        acc1 = fmaf(e1, e1, acc1);
        acc0 = fmaf(e2, e2, acc0);
        acc1 = fmaf(e3, e3, acc1);
      }
      float acc = acc0 + acc1;
      acc += __shfl_xor_sync(0xffffffffu, acc, 4);
      acc += __shfl_xor_sync(0xffffffffu, acc, 2);
      acc += __shfl_xor_sync(0xffffffffu, acc, 1);
      const int c = c0 + 4 * u + grp;
      if (l8 == 0 && c < C) cv[c] = acc;
    }
  }
}

__device__ __forceinline__ void refine_fp32(const float* __restrict__ q,
                                            const float* __restrict__ X, int d, const int* ci,
                                            float* cv, int C, int lane) {
  const int grp = lane >> 3, l8 = lane & 7;
  const bool vec = (d & 3) == 0 && (reinterpret_cast<uintptr_t>(q) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(X) & 15) == 0;
  if (vec && C > 0) {
    if (d <= 64) return refine_vec<2, 8>(q, X, d, ci, cv, C, lane);
    if (d <= 128) return refine_vec<4, 4>(q, X, d, ci, cv, C, lane);
    if (d <= 256) return refine_vec<8, 2>(q, X, d, ci, cv, C, lane);
  }
  for (int c0 = 0; c0 < C; c0 += 4) {
    const int c = c0 + grp;
    float acc0 = 0.f, acc1 = 0.f;
    if (c < C) {
      const float* x = X + (size_t)ci[c] * d;
      if (vec) {
        const float4* q4 = reinterpret_cast<const float4*>(q);
        const float4* x4 = reinterpret_cast<const float4*>(x);
        for (int f = l8; f < d / 4; f += 8) {
          const float4 a = __ldg(q4 + f), b = __ldg(x4 + f);
          const float e0 = a.x - b.x, e1 = a.y - b.y, e2 = a.z - b.z, e3 = a.w - b.w;
          acc0 = fmaf(e0, e0, acc0);
          acc1 = fmaf(e1, e1, acc1);
          acc0 = fmaf(e2, e2, acc0);
          acc1 = fmaf(e3, e3, acc1);
        }
      } else {
        for (int f = l8; f < d; f += 8) {
          const float e = __ldg(q + f) - __ldg(x + f);
          acc0 = fmaf(e, e, acc0);
        }
      }
    }
    float acc = acc0 + acc1;
    acc += __shfl_xor_sync(0xffffffffu, acc, 4);
    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    if (l8 == 0 && c < C) cv[c] = acc;
  }
}

// fp32 refinement of the C gathered candidates (ci columns, cv screen values
// on entry).  Returns C' and leaves ci[0..C') / cv[0..C') = the refined
// candidates and their fp32 squared distances; every dropped candidate has a
// certified lower bound above the k-th smallest upper bound of the refined
// ones, so it could not have survived.  `sa` / `av` are scratch for at most
// kSurvivorCap stage-one candidates.
// U0 (out): the k-th smallest fp32 upper bound of the stage-one candidates,
// INFINITY when the refinement ran in one stage.
__device__ __forceinline__ int refine_candidates(const CertifyArgs& a, int64_t row,
                                                 const float* q, int* ci, float* cv, int* sa,
                                                 float* av, unsigned* hist, int C, float up_f,
                                                 float abs32, float Vk, float* U0out, int lane) {
  const int k = a.k;
  *U0out = INFINITY;
  if (a.nq && C >= 4 * k) {
    // stage one: the candidates whose screen value is at most the k-th
    // smallest, which is V_k itself: the k smallest screen values of the query
    // are in its lists' k smallest (and all of them are <= Tf, so listed here)
    const float Vsel = Vk;
    int nA = 0;
    for (int base = 0; base < C; base += 32) {
      const int c = base + lane;
      const bool in = c < C && cv[c] <= Vsel;
      const unsigned bal = __ballot_sync(0xffffffffu, in);
      const int pos = nA + __popc(bal & ((1u << lane) - 1));
      if (in && pos < kSurvivorCap) sa[pos] = ci[c];
      nA += __popc(bal);
    }
    if (nA <= kSurvivorCap) {
      __syncwarp();
      refine_fp32(q, a.X, a.d, sa, av, nA, lane);
      __syncwarp();
      auto upper_key = [&](int j) { return float_key(__fadd_ru(__fmul_ru(av[j], up_f), abs32)); };
      const float U0 = key_float(
          nA <= 32 ? warp_kth_32(lane < nA ? upper_key(lane) : 0u, nA, k, lane)
                   : warp_radix_kth(upper_key, nA, k, hist, lane));
      *U0out = U0;
      // stage two: the other candidates whose screen lower bound
      // ||y_q||^2 + v - E (rounded down) reaches U0, compacted in place
      const double nq = a.nq[row], E = (double)a.E[row];
      int w = 0;
      for (int base = 0; base < C; base += 32) {
        const int c = base + lane;
        int col = 0;
        float v = 0.0f;
        bool keep = false;
        if (c < C) {
          col = ci[c];
          v = cv[c];
          keep = v > Vsel && __dadd_rd(__dadd_rd(nq, (double)v), -E) <= (double)U0;
        }
        // every lane has read its entry before any write (a write lands at or
        // below its writer's own position)
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (keep) {
          const int p = w + __popc(bal & ((1u << lane) - 1));
          ci[p] = col;
        }
        w += __popc(bal);
      }
      __syncwarp();
      refine_fp32(q, a.X, a.d, ci, cv, w, lane);
      __syncwarp();
      for (int j = lane; j < nA; j += 32) {
        ci[w + j] = sa[j];
        cv[w + j] = av[j];
      }
      __syncwarp();
      return w + nA;
    }
    __syncwarp();
  }
  refine_fp32(q, a.X, a.d, ci, cv, C, lane);
  __syncwarp();
  return C;
}

// One query row of one problem, by one warp; `wbase` is the warp's shared
// memory (kCertWarpBytes).
__device__ __forceinline__ void certify_row(const CertifyArgs& a, int64_t row, uint8_t* wbase, int lane) {
  int* ci = reinterpret_cast<int*>(wbase);                          // [kCertifyCap]
  float* cv = reinterpret_cast<float*>(ci + kCertifyCap);           // [kCertifyCap]
  double* cs = reinterpret_cast<double*>(cv + kCertifyCap);         // [kSurvivorCap]
  int* si = reinterpret_cast<int*>(cs + kSurvivorCap);              // [kSurvivorCap]
  unsigned* hist = reinterpret_cast<unsigned*>(si + kSurvivorCap);  // [256] radix histogram
  const ScreenOut& so = a.scr;
  const int k = a.k, S = a.S;
  // a screen that gave up left the lists unfinished: touch nothing (the call
  // reports the error); lane 0's read decides for the whole warp
  if (a.status) {
    const int st = lane == 0 ? *reinterpret_cast<volatile const int*>(a.status) : 0;
    if (__shfl_sync(0xffffffffu, st, 0) != DEV_OK) return;
  }

  // 1. overflow check
  bool overflow = false;
  unsigned entries = 0;
  for (int s = lane; s < S; s += 32) {
    int c = so.counts[(size_t)s * so.m_pad + row];
    overflow |= c > so.cap;
    entries += c;
  }
  overflow = __any_sync(0xffffffffu, overflow);
  if (overflow) {
    if (lane == 0) a.fallback_list[atomicAdd(a.fallback_count, 1)] = (int)(a.row_base + row);
    return;
  }
  entries = __reduce_add_sync(0xffffffffu, entries);

  // 2. V_k = k-th smallest of the lists' k smallest values (radix select);
  // screens without per-slot k-th values list every value up to their own
  // threshold, which covers the k smallest overall: select over the lists.
  const int total = S * k;
  float Vk;
  if (!so.kth) {
    Vk = key_float(warp_radix_select(
        [&](auto f) {
          for (int s = 0; s < S; ++s) {
            const size_t slot = (size_t)s * so.m_pad + row;
            const int cnt = so.counts[slot];
            const int2* lst = so.lists + slot * so.cap;
            for (int i = lane; i < cnt; i += 32) f(float_key(__int_as_float(lst[i].x)));
          }
        },
        k, hist, lane));
  } else if (total <= kCertifyCap) {
    uint32_t* keys = reinterpret_cast<uint32_t*>(ci);  // ci is free until step 3
    for (int i = lane; i < total; i += 32) {
      const int s = i / k, t = i % k;
      keys[i] = float_key(so.kth[((size_t)s * so.m_pad + row) * k + t]);
    }
    __syncwarp();
    if (S <= 32) {
      // each list's k values ascend: k rounds of a warp minimum over the
      // lists' heads (lane s walks list s), the k-th winner is V_k
      int p = 0;
      uint32_t head = lane < S ? keys[lane * k] : 0xffffffffu, kth_key = 0;
      for (int t = 0; t < k; ++t) {
        uint32_t mv = head;
        int ml = lane;
#pragma unroll
        for (int o = 16; o; o >>= 1) {
          const uint32_t ov = __shfl_xor_sync(0xffffffffu, mv, o);
          const int ol = __shfl_xor_sync(0xffffffffu, ml, o);
          if (ov < mv || (ov == mv && ol < ml)) {
            mv = ov;
            ml = ol;
          }
        }
        kth_key = mv;
        if (lane == ml) head = ++p < k ? keys[lane * k + p] : 0xffffffffu;
      }
      Vk = key_float(kth_key);
    } else {
      Vk = key_float(warp_radix_kth([&](int i) { return keys[i]; }, total, k, hist, lane));
    }
    __syncwarp();
  } else {
    Vk = key_float(warp_radix_kth(
        [&](int i) {
          const int s = i / k, t = i % k;
          return float_key(so.kth[((size_t)s * so.m_pad + row) * k + t]);
        },
        total, k, hist, lane));
  }
  const float Tf = __fadd_ru(Vk, __fmul_ru(2.0f, a.E[row]));

  // 3. gather candidates v <= Tf.  Each lane keeps four list entries in
  // flight (the loop is bound by their latency), and the columns of grouped
  // operand rows are mapped to training rows afterwards, all at once.
  int C = 0;
  bool too_many = false;
  constexpr int kAhead = 4;
  for (int s = 0; s < S && !too_many; ++s) {
    const size_t slot = (size_t)s * so.m_pad + row;
    const int cnt = so.counts[slot];
    const int2* lst = so.lists + slot * so.cap;
    for (int base = 0; base < cnt && !too_many; base += 32 * kAhead) {
      int2 e[kAhead];
#pragma unroll
      for (int u = 0; u < kAhead; ++u) {
        const int i = base + 32 * u + lane;
        e[u] = i < cnt ? lst[i] : make_int2(0, 0);
      }
#pragma unroll
      for (int u = 0; u < kAhead; ++u) {
        const int i = base + 32 * u + lane;
        const float v = __int_as_float(e[u].x);
        const bool pass = i < cnt && v <= Tf;
        const unsigned bal = __ballot_sync(0xffffffffu, pass);
        const int pos = C + __popc(bal & ((1u << lane) - 1));
        if (pass && pos < kCertifyCap) {
          ci[pos] = e[u].y;
          cv[pos] = v;  // the screen value until the refinement overwrites it
        }
        C += __popc(bal);
      }
      too_many = C > kCertifyCap;
    }
  }
  // grouped operand rows: the lists hold operand rows, the answer training rows
  if (!too_many && a.cols) {
    __syncwarp();
#pragma unroll 4
    for (int c = lane; c < C; c += 32) ci[c] = __ldg(a.cols + ci[c]);
  }
  if (too_many || C < k) {
    if (lane == 0) a.fallback_list[atomicAdd(a.fallback_count, 1)] = (int)(a.row_base + row);
    return;
  }
  __syncwarp();
  // 4. fp32 refine with a certified relative bound
  const float* q = a.Q + (size_t)row * a.d;
  const float g32 = (float)((double)(a.d + 5) * 0x1p-24 * 1.01);
  const float abs32 = (float)a.d * 0x1p-126f;
  const float up_f = 1.0f + g32, lo_f = 1.0f - g32;
  float U0;
  const int Cr = refine_candidates(a, row, q, ci, cv, si, reinterpret_cast<float*>(cs), hist, C,
                                   up_f, abs32, Vk, &U0, lane);
  // 5. U = k-th smallest upper bound.  After a two-stage refinement the
  // stage-one candidates (among the refined) put k upper bounds at or below
  // U0, so only those bounds can be the k-th smallest: when at most 32, a
  // rank select among them; otherwise a radix select over all.
  auto upper_key = [&](int c) { return float_key(__fadd_ru(__fmul_ru(cv[c], up_f), abs32)); };
  uint32_t Ukey = 0;
  bool small = false;
  if (U0 < INFINITY) {
    // the keys <= U0, gathered through the survivor scratch (free until step 6)
    uint32_t* tmp = reinterpret_cast<uint32_t*>(si);
    const uint32_t u0 = float_key(U0);
    int n = 0;
    for (int base = 0; base < Cr && n <= 32; base += 32) {
      const int c = base + lane;
      const uint32_t key = c < Cr ? upper_key(c) : 0xffffffffu;
      const bool le = c < Cr && key <= u0;
      const unsigned bal = __ballot_sync(0xffffffffu, le);
      const int pos = n + __popc(bal & ((1u << lane) - 1));
      if (le && pos < 32) tmp[pos] = key;
      n += __popc(bal);
    }
    __syncwarp();
    if (n <= 32 && n >= k) {
      Ukey = warp_kth_32(lane < n ? tmp[lane] : 0u, n, k, lane);
      small = true;
    }
    __syncwarp();
  }
  if (!small) Ukey = warp_radix_kth(upper_key, Cr, k, hist, lane);
  const float U = key_float(Ukey);
  // 6. survivors: lower bound <= U (everything that can still be in the top k)
  int Cs = 0;
  for (int base = 0; base < Cr; base += 32) {
    const int c = base + lane;
    const bool keep = c < Cr && __fsub_rd(__fmul_rd(cv[c], lo_f), abs32) <= U;
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    const int pos = Cs + __popc(bal & ((1u << lane) - 1));
    if (keep && pos < kSurvivorCap) si[pos] = ci[c];
    Cs += __popc(bal);
  }
  if (Cs > kSurvivorCap) {
    if (lane == 0) a.fallback_list[atomicAdd(a.fallback_count, 1)] = (int)(a.row_base + row);
    return;
  }
  __syncwarp();
  // 7. canonical float64 values of the survivors, sort, exact near-tie runs
  for (int c = lane; c < Cs; c += 32) cs[c] = canonical_d2(q, a.X + (size_t)si[c] * a.d, a.d);
  __syncwarp();
  const unsigned cmp = warp_sort_resolve(cs, si, Cs, k, q, a.X, a.d, lane);
  const int64_t orow = a.perm ? a.perm[row] : row;
  for (int t = lane; t < k; t += 32) {
    a.idx[orow * k + t] = si[t];
    if (a.dist) a.dist[orow * k + t] = a.squared ? cs[t] : sqrt(cs[t]);
  }
  if (lane == 0) {
    atomicAdd(&a.counters[0], (unsigned long long)C);
    atomicAdd(&a.counters[1], (unsigned long long)entries);
    if (a.refined) atomicAdd(a.refined, (unsigned long long)Cr);
    if (cmp) atomicAdd(&a.counters[2], (unsigned long long)cmp);
  }
}

__global__ void __launch_bounds__(kCertWarps * 32, 2)
    certify_kernel(const __grid_constant__ CertifyArgs a) {
  extern __shared__ uint8_t smem[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * kCertWarps + w;
  if (row >= a.m) return;
  certify_row(a, row, smem + (size_t)w * kCertWarpBytes, lane);
}

// Batched form: problem p owns global rows [row_start[p], row_start[p + 1]).
__global__ void __launch_bounds__(kCertWarps * 32, 2)
    certify_batch_kernel(const CertifyArgs* __restrict__ tab, const int64_t* __restrict__ row_start,
                         int P, int64_t total) {
  extern __shared__ uint8_t smem[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t r = (int64_t)blockIdx.x * kCertWarps + w;
  if (r >= total) return;
  const int p = problem_of(row_start, P, r);
  certify_row(tab[p], r - row_start[p], smem + (size_t)w * kCertWarpBytes, lane);
}

// ---------------------------------------------------------------------------
// Exhaustive exact scan: one CTA per query.  Canonical float64 values of all
// rows, an exact radix select of the k-th smallest value, every row whose
// error interval reaches it, then the same sort + exact resolution.
// ---------------------------------------------------------------------------
constexpr int kExactThreads = 256;

// `orow` is the query's original row (the one exclude_self refers to).
__device__ __forceinline__ double exact_value(const ExactArgs& a, const float* q, int64_t orow,
                                              int64_t j, const double* sc) {
  if (sc) return sc[j];
  if (a.exclude_self && j == a.q_offset + orow) return INFINITY;
  return canonical_d2(q, a.X + (size_t)j * a.d, a.d);
}

struct ExactShared {
  double* cs;  // [kExactCap]
  int* ci;     // [kExactCap]
  unsigned* hist;
  unsigned long long* prefix;
  int* rank;
  int* count;
  int* flag;   // the call's error word as thread 0 read it for this row
};

// One query row of one problem, by the whole CTA.  `sc` is the CTA's scratch
// of a.n canonical values (or null: recompute per pass).
__device__ __forceinline__ void exact_row(const ExactArgs& a, int64_t row, double* sc, const ExactShared& sh) {
  const int tid = threadIdx.x;
  // an earlier kernel of the call gave up (its fallback rows may be
  // unfinished), or another row of this launch failed: leave the outputs
  // alone.  Thread 0's read decides for the CTA (the word can change while
  // this kernel runs).
  if (tid == 0) *sh.flag = *reinterpret_cast<volatile const int*>(a.status);
  __syncthreads();
  if (*sh.flag != DEV_OK) return;
  double* cs = sh.cs;
  int* ci = sh.ci;
  unsigned* hist = sh.hist;
  const int64_t orow = a.perm ? a.perm[row] : row;
  const float* q = a.Q + (size_t)row * a.d;
  if (sc) {
    for (int64_t j = tid; j < a.n; j += kExactThreads) {
      sc[j] = (a.exclude_self && j == a.q_offset + orow)
                  ? INFINITY
                  : canonical_d2(q, a.X + (size_t)j * a.d, a.d);
    }
    __syncthreads();
  }
  // radix select over the bit patterns of non-negative doubles (monotone)
  unsigned long long prefix = 0, mask = 0;
  if (tid == 0) *sh.rank = a.k;
  __syncthreads();
  for (int shift = 56; shift >= 0; shift -= 8) {
    hist[tid] = 0;
    __syncthreads();
    for (int64_t j = tid; j < a.n; j += kExactThreads) {
      const unsigned long long b = __double_as_longlong(exact_value(a, q, orow, j, sc));
      if ((b & mask) == prefix) atomicAdd(&hist[(b >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (tid == 0) {
      int r = *sh.rank;
      unsigned acc = 0;
      int dgt = 0;
      for (; dgt < 256; ++dgt) {
        if (acc + hist[dgt] >= (unsigned)r) break;
        acc += hist[dgt];
      }
      *sh.rank = r - (int)acc;
      *sh.prefix = prefix | ((unsigned long long)dgt << shift);
    }
    __syncthreads();
    prefix = *sh.prefix;
    mask |= 255ull << shift;
  }
  const double Vk = __longlong_as_double((long long)prefix);
  const double g2 = interval_g2(a.d);
  const double reach = __dmul_ru(Vk, 1.0 + g2);
  if (tid == 0) *sh.count = 0;
  __syncthreads();
  for (int64_t j = tid; j < a.n; j += kExactThreads) {
    const double v = exact_value(a, q, orow, j, sc);
    if (v != INFINITY && __dmul_rd(v, 1.0 - g2) <= reach) {
      const int pos = atomicAdd(sh.count, 1);
      if (pos < kExactCap) {
        cs[pos] = v;
        ci[pos] = (int)j;
      }
    }
  }
  __syncthreads();
  const int C = *sh.count;
  if (C > kExactCap) {
    if (tid == 0) atomicCAS(a.status, DEV_OK, DEV_TOO_MANY_TIES);
  } else if (C < a.k) {
    // fewer than k comparable values: only a NaN query coordinate does this
    // (the call reports it as non-finite input); leave a defined answer
    for (int t = tid; t < a.k; t += kExactThreads) {
      a.idx[orow * a.k + t] = -1;
      if (a.dist) a.dist[orow * a.k + t] = __longlong_as_double(0x7ff8000000000000ll);
    }
  } else if (tid < 32) {
    const unsigned cmp = warp_sort_resolve(cs, ci, C, a.k, q, a.X, a.d, tid);
    for (int t = tid; t < a.k; t += 32) {
      a.idx[orow * a.k + t] = ci[t];
      if (a.dist) a.dist[orow * a.k + t] = a.squared ? cs[t] : sqrt(cs[t]);
    }
    if (tid == 0) {
      atomicAdd(&a.counters[3], 1ull);
      if (cmp) atomicAdd(&a.counters[2], (unsigned long long)cmp);
    }
  }
  __syncthreads();
}

#define B2K_EXACT_SHARED                                                   \
  extern __shared__ uint8_t smem[];                                        \
  __shared__ unsigned hist[256];                                           \
  __shared__ unsigned long long s_prefix;                                  \
  __shared__ int s_rank, s_count, s_flag;                                  \
  ExactShared sh;                                                          \
  sh.cs = reinterpret_cast<double*>(smem);                                 \
  sh.ci = reinterpret_cast<int*>(sh.cs + kExactCap);                       \
  sh.hist = hist;                                                          \
  sh.prefix = &s_prefix;                                                   \
  sh.rank = &s_rank;                                                       \
  sh.count = &s_count;                                                     \
  sh.flag = &s_flag;

__global__ void __launch_bounds__(kExactThreads)
    exact_kernel(const __grid_constant__ ExactArgs a) {
  B2K_EXACT_SHARED
  const int count = a.rows ? *a.row_count : (int)a.m;
  double* sc = a.scratch ? a.scratch + (size_t)blockIdx.x * a.n : nullptr;
  for (int it = blockIdx.x; it < count; it += gridDim.x)
    exact_row(a, a.rows ? a.rows[it] : it, sc, sh);
}

// Batched form over a list of global rows (problem p owns rows
// [row_start[p], row_start[p + 1])); scratch holds n_max values per CTA.
__global__ void __launch_bounds__(kExactThreads)
    exact_batch_kernel(const ExactArgs* __restrict__ tab, const int64_t* __restrict__ row_start,
                       int P, const int* __restrict__ rows, const int* __restrict__ row_count,
                       double* scratch, int64_t n_max) {
  B2K_EXACT_SHARED
  const int count = *row_count;
  double* sc = scratch ? scratch + (size_t)blockIdx.x * n_max : nullptr;
  for (int it = blockIdx.x; it < count; it += gridDim.x) {
    const int64_t r = rows[it];
    const int p = problem_of(row_start, P, r);
    exact_row(tab[p], r - row_start[p], sc, sh);
  }
}
#undef B2K_EXACT_SHARED

}  // namespace

void launch_certify(const CertifyArgs& a, cudaStream_t st) {
  if (a.m <= 0) return;
  const size_t smem = (size_t)kCertWarps * kCertWarpBytes;
  cudaFuncSetAttribute(certify_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const unsigned grid = (unsigned)((a.m + kCertWarps - 1) / kCertWarps);
  certify_kernel<<<grid, kCertWarps * 32, smem, st>>>(a);
}

void launch_certify_batch(const CertifyArgs* tab, const int64_t* row_start, int P,
                          int64_t total_rows, cudaStream_t st) {
  if (total_rows <= 0) return;
  const size_t smem = (size_t)kCertWarps * kCertWarpBytes;
  cudaFuncSetAttribute(certify_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)smem);
  const unsigned grid = (unsigned)((total_rows + kCertWarps - 1) / kCertWarps);
  certify_batch_kernel<<<grid, kCertWarps * 32, smem, st>>>(tab, row_start, P, total_rows);
}

void launch_exact_batch(const ExactArgs* tab, const int64_t* row_start, int P, const int* rows,
                        const int* row_count, double* scratch, int64_t n_max, int grid,
                        cudaStream_t st) {
  if (grid <= 0) return;
  const size_t smem = (size_t)kExactCap * (sizeof(double) + sizeof(int));
  cudaFuncSetAttribute(exact_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)smem);
  exact_batch_kernel<<<grid, kExactThreads, smem, st>>>(tab, row_start, P, rows, row_count,
                                                        scratch, n_max);
}

void launch_exact(const ExactArgs& a, cudaStream_t st) {
  if (a.grid <= 0) return;
  const size_t smem = (size_t)kExactCap * (sizeof(double) + sizeof(int));
  cudaFuncSetAttribute(exact_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  exact_kernel<<<a.grid, kExactThreads, smem, st>>>(a);
}

}  // namespace b2k
