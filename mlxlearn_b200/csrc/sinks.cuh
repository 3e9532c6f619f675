// Per-row consumers of the screen values ("sinks").
//
// A screen kernel hands each row's values v (see prep.cu) to a sink, 32
// columns at a time (offer32) or one at a time (offer1).  Columns flagged NaN
// (padding) are never admitted, nor is the row's excluded self column.
//   KnnSink        : the running k-smallest tracker + candidate list (tracker.cuh)
//   RadiusCountSink: counts columns with v <= T (T fixed per row: R2 - ||y_q||^2 + E)
//   RadiusFillSink : writes those columns, in ascending order, at a precomputed offset
//   RadiusListSink : writes them into a fixed-capacity list per (split, row), counting all
#pragma once
#include "internal.cuh"
#include "tracker.cuh"

namespace b2k {

struct SinkArgs {
  // kNN
  ScreenOut out;
  int k;
  uint32_t* shared_kth;  // [m_pad] per-query shared k-th key, or null
  // radius
  const float* thr;      // [m_pad] admission threshold per row
  int* rcount;           // [S][m_pad]
  const int64_t* roff;   // [S][m_pad]
  int* rcols;            // candidate columns (RadiusListSink: [S][m_pad][rcap] lists)
  int m_pad;
  int rcap;              // RadiusListSink: entries kept per list
};

// Admitted columns of a 32-column chunk as a bit mask (bit i: v[i] <= T),
// the excluded column (self, when it lies in the chunk) cleared.  The four
// 8-column group minima come first (3-input minima); only groups
// whose minimum passes build their bits, so a warp pays for a group only
// where one of its rows admits.  NaN values (padding rows) never pass.
__device__ __forceinline__ uint32_t admit_mask32(const float (&v)[32], float T, int col0,
                                                 int self) {
  float g[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float a = min3f(v[8 * q], v[8 * q + 1], v[8 * q + 2]);
    const float b = min3f(v[8 * q + 3], v[8 * q + 4], v[8 * q + 5]);
    g[q] = min3f(a, b, fminf(v[8 * q + 6], v[8 * q + 7]));
  }
  if (!(fminf(min3f(g[0], g[1], g[2]), g[3]) <= T)) return 0u;
  uint32_t m = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q)
    if (g[q] <= T) {
      uint32_t bits = 0;
#pragma unroll
      for (int e = 0; e < 8; ++e) bits |= (v[8 * q + e] <= T) ? (1u << e) : 0u;
      m |= bits << (8 * q);
    }
  const unsigned s = (unsigned)(self - col0);
  if (s < 32u) m &= ~(1u << s);
  return m;
}

template <int KMAX>
struct KnnSink {
  static constexpr bool kWarpWide = false;
  RowTracker<KMAX> tr;
  size_t slot;
  B2K_DEV void init(const SinkArgs& a, int row, int split, float E, int self) {
    slot = (size_t)split * a.out.m_pad + row;
    tr.init(a.k, E, self, a.out.lists + slot * a.out.cap, a.out.cap,
            a.shared_kth ? a.shared_kth + row : nullptr);
  }
  B2K_DEV void tile_sync() { tr.sync_shared(); }
  B2K_DEV uint32_t tile_fetch() const { return tr.fetch_shared(); }
  B2K_DEV void tile_apply(uint32_t key) { tr.apply_shared(key); }
  B2K_DEV void offer32(const float (&v)[32], int col0, float* spill) { tr.offer32(v, col0, spill); }
  B2K_DEV void offer1(float x, int col) {
    if (x <= tr.T && col != tr.self) tr.admit(x, col);
  }
  B2K_DEV void finish(const SinkArgs& a) {
    a.out.counts[slot] = tr.cnt;
    tr.write_kth(a.out.kth + slot * a.k, a.k);
  }
};

struct RadiusCountSink {
  static constexpr bool kWarpWide = false;
  float T;
  int self, cnt;
  size_t slot;
  B2K_DEV void init(const SinkArgs& a, int row, int split, float /*E*/, int self_col) {
    slot = (size_t)split * a.m_pad + row;
    T = a.thr[row];
    self = self_col;
    cnt = 0;
  }
  B2K_DEV void offer32(const float (&v)[32], int col0, float*) {
    cnt += __popc(admit_mask32(v, T, col0, self));
  }
  B2K_DEV void offer1(float x, int col) { cnt += (x <= T && col != self) ? 1 : 0; }
  B2K_DEV void tile_sync() {}
  B2K_DEV uint32_t tile_fetch() const { return 0; }
  B2K_DEV void tile_apply(uint32_t) {}
  B2K_DEV void finish(const SinkArgs& a) { a.rcount[slot] = cnt; }
};

struct RadiusFillSink {
  static constexpr bool kWarpWide = false;
  float T;
  int self;
  int* out;
  B2K_DEV void init(const SinkArgs& a, int row, int split, float /*E*/, int self_col) {
    const size_t slot = (size_t)split * a.m_pad + row;
    T = a.thr[row];
    self = self_col;
    out = a.rcols + a.roff[slot];
  }
  B2K_DEV void offer32(const float (&v)[32], int col0, float*) {
    // ascending columns: lowest set bit first
    for (uint32_t m = admit_mask32(v, T, col0, self); m; m &= m - 1) *out++ = col0 + __ffs(m) - 1;
  }
  B2K_DEV void offer1(float x, int col) {
    if (x <= T && col != self) *out++ = col;
  }
  B2K_DEV void tile_sync() {}
  B2K_DEV uint32_t tile_fetch() const { return 0; }
  B2K_DEV void tile_apply(uint32_t) {}
  B2K_DEV void finish(const SinkArgs&) {}
};

// Single-pass radius: the admitted columns of (split, row), ascending, into a
// list of rcap entries at slot * rcap; the count goes on past rcap, so a
// count above it marks a row whose list lost columns (the caller answers that
// row again with the counted two-pass form).
struct RadiusListSink {
  static constexpr bool kWarpWide = false;
  float T;
  int self, cnt, cap;
  int* out;
  size_t slot;
  B2K_DEV void init(const SinkArgs& a, int row, int split, float /*E*/, int self_col) {
    slot = (size_t)split * a.m_pad + row;
    T = a.thr[row];
    self = self_col;
    cnt = 0;
    cap = a.rcap;
    out = a.rcols + slot * (size_t)a.rcap;
  }
  B2K_DEV void put(int col) {
    if (cnt < cap) out[cnt] = col;
    ++cnt;
  }
  B2K_DEV void offer32(const float (&v)[32], int col0, float*) {
    const uint32_t m = admit_mask32(v, T, col0, self);
    if (m) {
      // the entries that still fit, ascending (lowest set bit first); the
      // count goes on past the capacity
      int c = cnt;
      for (uint32_t f = m; f && c < cap; f &= f - 1) out[c++] = col0 + __ffs(f) - 1;
      cnt += __popc(m);
    }
  }
  B2K_DEV void offer1(float x, int col) {
    if (x <= T && col != self) put(col);
  }
  B2K_DEV void tile_sync() {}
  B2K_DEV uint32_t tile_fetch() const { return 0; }
  B2K_DEV void tile_apply(uint32_t) {}
  B2K_DEV void finish(const SinkArgs& a) { a.rcount[slot] = cnt; }
};

// Exact kNN sink of the u8 screen: values are exact integers
// v = ||x||^2 - 2<q, x>, so the list keeps just the k smallest (v, column)
// in registers, ascending, equal values in column order.  Columns reach a
// list in ascending order, so a value equal to the current k-th is never
// better (a larger index); one equal to a k-th published by another list may
// be (ties across lists are resolved by the merge), so the shared bound is
// inclusive.  The padding rows' v is INT_MAX and never admitted.
template <int KMAX>
struct ExactU8Sink {
  static constexpr bool kWarpWide = false;
  int kv[KMAX], kc[KMAX];
  int bound;          // admit v <= bound: min(k-th - 1, shared k-th)
  int shared_v;       // smallest k-th published for this query (INT_MAX: none)
  int self;
  bool dirty;
  uint32_t* shared;
  size_t slot;
  B2K_DEV static uint32_t key_of(int v) { return (uint32_t)v ^ 0x80000000u; }
  B2K_DEV static int value_of(uint32_t key) { return (int)(key ^ 0x80000000u); }
  B2K_DEV void init(const SinkArgs& a, int row, int split, float /*E*/, int self_col) {
    slot = (size_t)split * a.out.m_pad + row;
#pragma unroll
    for (int i = 0; i < KMAX; ++i) {
      // KMAX - k sentinels below every value, then k empty places
      kv[i] = i < KMAX - a.k ? INT_MIN : INT_MAX;
      kc[i] = -1;
    }
    shared_v = INT_MAX;
    self = self_col;
    dirty = false;
    shared = a.shared_kth ? a.shared_kth + row : nullptr;
    set_bound();
    sync_shared();
  }
  B2K_DEV void set_bound() {
    const int own = kv[KMAX - 1] == INT_MAX ? INT_MAX - 1 : kv[KMAX - 1] - 1;
    bound = min(own, shared_v);
  }
  // x < kv[KMAX - 1]: insert after the values <= x
  B2K_DEV void insert(int x, int c) {
#pragma unroll
    for (int i = KMAX - 1; i > 0; --i) {
      const bool shift = kv[i - 1] > x, here = kv[i] > x;
      const int nv = shift ? kv[i - 1] : (here ? x : kv[i]);
      const int nc = shift ? kc[i - 1] : (here ? c : kc[i]);
      kv[i] = nv;
      kc[i] = nc;
    }
    if (kv[0] > x) {
      kv[0] = x;
      kc[0] = c;
    }
    dirty = true;
    set_bound();
  }
  B2K_DEV void offer32i(const int (&v)[32], int col0) {
    int a[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) a[i] = min(v[2 * i], v[2 * i + 1]);
#pragma unroll
    for (int w = 8; w > 0; w >>= 1)
#pragma unroll
      for (int i = 0; i < w; ++i) a[i] = min(a[i], a[i + w]);
    if (a[0] <= bound) {
#pragma unroll
      for (int i = 0; i < 32; ++i)
        if (v[i] <= bound && col0 + i != self) insert(v[i], col0 + i);
    }
  }
  B2K_DEV uint32_t fetch_shared() const {
    uint32_t key = kNoKey;
    if (shared) asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(key) : "l"(shared));
    return key;
  }
  B2K_DEV void apply_shared(uint32_t key) {
    if (!shared) return;
    if (dirty && kv[KMAX - 1] != INT_MAX) {
      atomicMin(shared, key_of(kv[KMAX - 1]));
      dirty = false;
    }
    if (key != kNoKey && value_of(key) < shared_v) {
      shared_v = value_of(key);
      set_bound();
    }
  }
  B2K_DEV void sync_shared() { apply_shared(fetch_shared()); }
  B2K_DEV void tile_sync() { sync_shared(); }
  B2K_DEV uint32_t tile_fetch() const { return fetch_shared(); }
  B2K_DEV void tile_apply(uint32_t key) { apply_shared(key); }
  B2K_DEV void finish(const SinkArgs& a) {
    int2* out = a.out.lists + slot * a.out.cap;
#pragma unroll
    for (int i = 0; i < KMAX; ++i)
      if (i >= KMAX - a.k) out[i - (KMAX - a.k)] = make_int2(kv[i], kc[i]);
  }
};

// kNN sink for large k on the lazy tracker (tracker.cuh).  Warp-collective:
// every lane of the warp calls every method, `active` false for rows past the
// end of the query block; `hist` is the warp's 256-word shared scratch.
static_assert(kListCap <= 512, "the lazy tracker's warp select holds 16 entries per lane");
struct LazyKnnSink {
  static constexpr bool kWarpWide = true;
  LazyTracker tr;
  size_t slot;
  unsigned* hist;
  int lane;
  B2K_DEV void init_warp(const SinkArgs& a, int row, int split, float E, int self, bool active,
                         unsigned* warp_hist) {
    slot = (size_t)split * a.out.m_pad + row;
    hist = warp_hist;
    lane = threadIdx.x & 31;
    tr.init(a.k, E, self, a.out.lists + slot * a.out.cap, a.out.cap,
            a.shared_kth ? a.shared_kth + row : nullptr, active);
  }
  B2K_DEV void tile_sync() { tr.sync_shared(); }
  B2K_DEV uint32_t tile_fetch() const { return tr.fetch_shared(); }
  B2K_DEV void tile_apply(uint32_t key) { tr.apply_shared(key); }
  B2K_DEV void offer32(const float (&v)[32], int col0, float*) { tr.offer32(v, col0, hist, lane); }
  // Only the list length: the certify pass selects V_k from the lists.
  B2K_DEV void finish_warp(const SinkArgs& a) {
    if (tr.active) a.out.counts[slot] = tr.cnt;
  }
};

}  // namespace b2k
