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

// Order-preserving map of floats to unsigned keys (for atomicMin / bisection).
__device__ __forceinline__ uint32_t float_key(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}
constexpr uint32_t kNoKey = 0xffffffffu;  // "nothing published yet"

// The screens of one query run in several places at once (reference splits
// on different CTAs, column halves on different warps).  Each publishes its
// own k-th smallest value to a per-query word in global memory (atomicMin on
// the ordered key) and reads the others' back once per tile.  Any published
// value is the k-th smallest of a subset of the query's values, hence >= the
// final V_k, so min(own, shared) + 2E is still a valid admission threshold.
template <int KMAX>
struct RowTracker {
  float kv[KMAX];
  float T;
  float E2;
  float shared_kth;   // last value read from the shared word
  int cnt;
  int self;
  int cap;
  int2* list;
  uint32_t* shared;   // per-query shared k-th key (may be null)
  bool dirty;         // own k-th improved since the last publish

  B2K_DEV void init(int k, float E, int self_col, int2* lst, int cap_, uint32_t* shared_word) {
#pragma unroll
    for (int i = 0; i < KMAX; ++i) kv[i] = (i < KMAX - k) ? -INFINITY : INFINITY;
    T = INFINITY;
    E2 = __fmul_ru(2.0f, E);
    shared_kth = INFINITY;
    cnt = 0;
    self = self_col;
    list = lst;
    cap = cap_;
    shared = shared_word;
    dirty = false;
    // start from the k-th value other lists of this query already published
    // (earlier reference splits run first): this list then skips most of its
    // own fill phase, k (1 + ln(n / k)) admissions above the final band
    sync_shared();
  }

  B2K_DEV void update_threshold() { T = __fadd_ru(fminf(kv[KMAX - 1], shared_kth), E2); }

  // Once per tile, in two halves so the L2 round trip overlaps the tile's
  // work: fetch_shared() issues the load (start of tile), apply_shared()
  // publishes our k-th if it improved and folds the fetched value in (end).
  B2K_DEV uint32_t fetch_shared() const {
    uint32_t key = kNoKey;
    if (shared) asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(key) : "l"(shared));
    return key;
  }
  B2K_DEV void apply_shared(uint32_t key) {
    if (!shared) return;
    if (dirty) {
      atomicMin(shared, float_key(kv[KMAX - 1]));
      dirty = false;
    }
    if (key != kNoKey) {
      const float g = key_float(key);
      if (g < shared_kth) {
        shared_kth = g;
        update_threshold();
      }
    }
  }
  B2K_DEV void sync_shared() { apply_shared(fetch_shared()); }

  // The list is full: drop the entries above the current threshold.  T only
  // decreases, and (see above) every value above it is more than 2E above the
  // final V_k, so the certify pass would discard those entries anyway.
  B2K_DEV void compact() {
    int w = 0;
    for (int i = 0; i < cap; ++i) {
      const int2 e = list[i];
      if (__int_as_float(e.x) <= T) list[w++] = e;
    }
    cnt = w;
  }

  // Caller guarantees v <= T and col is not the excluded self column.
  B2K_DEV void admit(float v, int col) {
    if (cnt == cap) compact();
    if (cnt < cap) list[cnt] = make_int2(__float_as_int(v), col);
    ++cnt;
    if (v < kv[KMAX - 1]) {
#pragma unroll
      for (int i = KMAX - 1; i > 0; --i) kv[i] = fminf(kv[i], fmaxf(kv[i - 1], v));
      kv[0] = fminf(kv[0], v);
      update_threshold();
      dirty = true;
    }
  }

  // Offer 32 consecutive columns col0.. whose values are in v[]; `spill` is
  // this thread's 33-float scratch in shared memory (slow path only).
  // Minima of the four 8-column groups, then of the chunk; only groups whose
  // minimum passes are spilled and scanned (a warp pays for a group if any of
  // its 32 rows admits there).
  B2K_DEV void offer32(const float (&v)[32], int col0, float* spill) {
    float g[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float a = min3f(v[8 * q], v[8 * q + 1], v[8 * q + 2]);
      const float b = min3f(v[8 * q + 3], v[8 * q + 4], v[8 * q + 5]);
      g[q] = min3f(a, b, fminf(v[8 * q + 6], v[8 * q + 7]));
    }
    if (fminf(min3f(g[0], g[1], g[2]), g[3]) <= T) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (g[q] <= T) {
          // T only decreases while admitting, so `mask` is a superset of the
          // columns that will be admitted.
          uint32_t mask = 0;
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            mask |= (v[8 * q + e] <= T ? 1u : 0u) << e;
            spill[e] = v[8 * q + e];
          }
          while (mask) {
            const int e = __ffs(mask) - 1;
            mask &= mask - 1;
            const float x = spill[e];
            const int col = col0 + 8 * q + e;
            if (x <= T && col != self) admit(x, col);
          }
        }
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

// Lazy form for large k (the insertion network above costs O(KMAX) per
// admission, and while the k-th value settles a row admits about
// k (1 + ln(n / k)) values).  No per-row heap: every v <= T is appended, and
// T is refreshed from the list itself when the list nears capacity: the
// whole warp selects the row's k-th smallest listed value V (radix select in
// shared memory), sets T = min(V, shared) + 2E and drops the entries above
// T.  The list always holds every value seen that is <= the current T, in
// particular the k smallest seen so far, so V is the k-th smallest value seen
// and the certificate argument above applies unchanged.
//
// Every method is warp-collective: all 32 lanes call it, rows past the end
// of the query block included (inactive: they admit nothing).
struct LazyTracker {
  float T, E2, shared_kth, own_kth;
  int cnt, self, cap, k;
  int trig;  // compact once cnt exceeds this (cap - 32)
  int2* list;
  uint32_t* shared;
  bool active, dirty;

  B2K_DEV void init(int k_, float E, int self_col, int2* lst, int cap_, uint32_t* shared_word,
                    bool active_) {
    active = active_;
    T = active_ ? INFINITY : -INFINITY;
    E2 = __fmul_ru(2.0f, E);
    shared_kth = INFINITY;
    own_kth = INFINITY;
    cnt = 0;
    self = self_col;
    k = k_;
    list = lst;
    cap = cap_;
    trig = cap_ - 32;
    shared = active_ ? shared_word : nullptr;
    dirty = false;
    sync_shared();  // start from the k-th value other lists already published
  }

  B2K_DEV uint32_t fetch_shared() const {
    uint32_t key = kNoKey;
    if (shared) asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(key) : "l"(shared));
    return key;
  }
  B2K_DEV void apply_shared(uint32_t key) {
    if (!shared) return;
    if (dirty) {
      atomicMin(shared, float_key(own_kth));
      dirty = false;
    }
    if (key != kNoKey) {
      const float g = key_float(key);
      if (g < shared_kth) {
        shared_kth = g;
        T = fminf(T, __fadd_ru(g, E2));
      }
    }
  }
  B2K_DEV void sync_shared() { apply_shared(fetch_shared()); }

  // k-th smallest value of lane `src`'s list (c entries, c >= kk), by the
  // whole warp: keys in registers, 4 radix passes over a 256-bin histogram in
  // `hist` (this warp's shared memory).  Also returns how many are smaller.
  B2K_DEV static uint32_t warp_kth(const int2* lst, int c, int kk, unsigned* hist, int lane,
                                   int* n_less) {
    constexpr int kPer = 16;  // up to 512 entries
    uint32_t key[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const int i = lane + 32 * j;
      key[j] = i < c ? float_key(__int_as_float(lst[i].x)) : 0xffffffffu;
    }
    uint32_t prefix = 0, mask = 0;
    int rank = kk, less = 0;
#pragma unroll 1
    for (int shift = 24; shift >= 0; shift -= 8) {
#pragma unroll
      for (int b = 0; b < 8; ++b) hist[lane * 8 + b] = 0;
      __syncwarp();
#pragma unroll
      for (int j = 0; j < kPer; ++j)
        if (lane + 32 * j < c && (key[j] & mask) == prefix)
          atomicAdd(&hist[(key[j] >> shift) & 255u], 1u);
      __syncwarp();
      unsigned local[8], sum = 0;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        local[b] = hist[lane * 8 + b];
        sum += local[b];
      }
      unsigned incl = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      const unsigned excl = incl - sum;
      // the lane whose bins cross `rank` finds the digit
      int digit = -1;
      unsigned below = 0;
      if (excl < (unsigned)rank && incl >= (unsigned)rank) {
        unsigned acc = excl;
#pragma unroll
        for (int b = 0; b < 8; ++b) {
          if (digit < 0 && acc + local[b] >= (unsigned)rank) {
            digit = lane * 8 + b;
            below = acc;
          }
          acc += local[b];
        }
      }
      const unsigned owner = __ballot_sync(0xffffffffu, digit >= 0);
      const int src_lane = __ffs(owner) - 1;
      digit = __shfl_sync(0xffffffffu, digit, src_lane);
      below = __shfl_sync(0xffffffffu, below, src_lane);
      rank -= (int)below;
      less += (int)below;
      prefix |= (uint32_t)digit << shift;
      mask |= 255u << shift;
      __syncwarp();
    }
    *n_less = less;
    return prefix;
  }

  // Compact the lists that are within 32 entries of capacity (a chunk admits
  // at most 32 values per row).  Each compaction costs the warp ~200
  // instructions; a row scanning n columns needs about
  // k (1 + ln(n / k)) / (cap - k) of them.
  B2K_DEV void maintain(unsigned* hist, int lane) {
    unsigned todo = __ballot_sync(0xffffffffu, active && cnt > trig && cnt >= k && cnt <= cap);
    if (todo) __syncwarp();  // the lanes' appends are visible to the whole warp
    while (todo) {
      const int src = __ffs(todo) - 1;
      todo &= todo - 1;
      int2* lst = reinterpret_cast<int2*>(__shfl_sync(0xffffffffu, (unsigned long long)list, src));
      const int c = __shfl_sync(0xffffffffu, cnt, src);
      const int kk = __shfl_sync(0xffffffffu, k, src);
      const float e2 = __shfl_sync(0xffffffffu, E2, src);
      const float sh = __shfl_sync(0xffffffffu, shared_kth, src);
      int n_less;
      const float V = key_float(warp_kth(lst, c, kk, hist, lane, &n_less));
      const float Tn = __fadd_ru(fminf(V, sh), e2);
      // in-place stream compaction: writes never pass the reads of the same
      // or a later round
      int w = 0;
      for (int base = 0; base < c; base += 32) {
        const int i = base + lane;
        int2 e = make_int2(0, 0);
        bool keep = false;
        if (i < c) {
          e = lst[i];
          keep = __int_as_float(e.x) <= Tn;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (keep) lst[w + __popc(bal & ((1u << lane) - 1))] = e;
        w += __popc(bal);
      }
      __syncwarp();
      if (lane == src) {
        cnt = w;
        own_kth = V;
        T = fminf(T, Tn);
        dirty = true;
      }
    }
  }

  B2K_DEV void offer32(const float (&v)[32], int col0, unsigned* hist, int lane) {
    float g[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float a = min3f(v[8 * q], v[8 * q + 1], v[8 * q + 2]);
      const float b = min3f(v[8 * q + 3], v[8 * q + 4], v[8 * q + 5]);
      g[q] = min3f(a, b, fminf(v[8 * q + 6], v[8 * q + 7]));
    }
    if (fminf(min3f(g[0], g[1], g[2]), g[3]) <= T) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (g[q] <= T) {
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            const float x = v[8 * q + e];
            const int col = col0 + 8 * q + e;
            if (x <= T && col != self) {
              if (cnt < cap) list[cnt] = make_int2(__float_as_int(x), col);
              ++cnt;
            }
          }
        }
      }
    }
    maintain(hist, lane);
  }

};

}  // namespace b2k
