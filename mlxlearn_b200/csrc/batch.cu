// Batches of independent kNN problems: one planned device work queue, one
// CUDA graph per batch.
//
// The reference answers one problem per call (NeighborIndex.query,
// src/mlxlearn/_kernels/distance.py:242-270); a caller with many small
// problems pays a launch sequence and a host synchronisation for each.  Here
// a batch of problems of uneven n, d, k and m becomes:
//
//   memset         status block, per-query shared k-th words
//   prep (1)       every problem's query rows: bound E, -2 bf16(q - c) operand
//   screen (L)     one persistent tcgen05 launch per (heap width, epilogue
//                  width): CTAs walk host-balanced lists of work items
//                  (problem, 128-query tile, range of 256-row reference tiles)
//   certify (1)    every problem's query rows, one warp each
//   exact (1)      the rows certify could not finish (a device-side count)
//
// captured once as a CUDA graph and replayed per run.  Problems with the same
// padded width dp share one concatenated bf16 operand buffer per side, so a
// launch addresses all of its problems through at most kBatchGroups sets of
// three tensor maps passed as kernel parameters.
//
// Balance: items are costed (reference tiles x (64-column blocks + 1)) and
// sorted longest first; each CTA claims the next item of that list when it
// finishes one (an online longest-processing-time-first schedule that also
// absorbs per-tile costs the model misses); items of one problem stay
// adjacent, so CTAs running at the same time read the same reference tiles
// from L2.
//
// Autotuner: per (dp, heap width) bucket the epilogue width (4, 8 or 16 warps),
// and for the whole batch the split granularity (items per CTA), chosen by
// timing graph runs of the batch itself; choices are cached per process.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <queue>
#include <tuple>
#include <vector>

#include "internal.cuh"
#include "tc_batch.cuh"

namespace b2k {
namespace {

int bfail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int bfail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return report_error(code, buf);
}

#define BCUDA(call)                                                                          \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return bfail(e_ == cudaErrorMemoryAllocation ? B2K_ENOMEM : B2K_ECUDA, "%s: %s (%s:%d)", \
                   #call, cudaGetErrorString(e_), __FILE__, __LINE__);                       \
  } while (0)

int64_t rup(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

// heap width of the screen's tracker; 64 = the lazy tracker (k > 16)
int kmax_class(int k) { return k <= 8 ? 8 : k <= 12 ? 12 : k <= 16 ? 16 : 64; }

// ---------------------------------------------------------------- tuning
// Epilogue warps per (dp, heap width) bucket; 0 = the default (16 for the
// register-heap trackers, 8 for the lazy tracker).
struct Tuning {
  int ew = 0;
};
int default_ew(int kmax) { return kmax <= 16 ? 16 : 8; }
struct TuneKey {
  int dp, kmax;
  bool operator<(const TuneKey& o) const { return dp != o.dp ? dp < o.dp : kmax < o.kmax; }
};
std::mutex g_tune_mu;
std::map<TuneKey, Tuning> g_tune;
int g_gran = 0;  // tuned split granularity (0: not tuned yet)
constexpr int kDefaultGran = 4;

struct Owned {
  std::vector<void*> ptrs;
  template <typename T>
  int alloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    if (injected_fault() == 1)
      return bfail(B2K_ENOMEM, "injected allocation failure (B2K_FAULT=alloc)");
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T));
    if (e != cudaSuccess)
      return bfail(e == cudaErrorMemoryAllocation ? B2K_ENOMEM : B2K_ECUDA,
                   "batch allocation of %zu bytes failed: %s", count * sizeof(T),
                   cudaGetErrorString(e));
    ptrs.push_back(*p);
    return B2K_OK;
  }
  void release() {
    for (void* p : ptrs) cudaFree(p);
    ptrs.clear();
  }
};

struct BProb {
  Index* ix;
  const float* Q;
  int64_t m;
  int k, exclude_self;
  int64_t q_offset;
  double* dist;
  int64_t* idx;
  bool in_graph = false;
  int gi = -1;          // index among graph problems
  // static layout
  int dp = 0, KB = 0, n_tiles = 0, m_pad = 0, m_tiles = 0, kmax = 0;
  int dpg = -1;         // dp group
  int64_t a_row0 = 0, b_row0 = 0, pad0 = 0, row0 = 0;
  float xh_max = 0, ex_max = 0;
  // tuned layout
  int ew = 8, halves = 2, S = 1, tps = 0, S_lists = 2, cap = kListCap;
  int launch = -1, group = -1;
  size_t lists_off = 0, counts_off = 0, kth_off = 0;
};

struct DpGroup {
  int dp;
  int64_t a_rows = 0, b_rows = 0;
  uint16_t *A = nullptr, *B = nullptr, *Baug = nullptr;
  CUtensorMap ma, mb, mbaug;
};

struct LaunchSpec {
  int kmax, ew;
  bool a_stream;
  std::vector<int> dpgs;   // dp groups of this launch (map slots)
  std::vector<int> probs;  // graph problem indices
};

}  // namespace
}  // namespace b2k

struct b2k_batch {
  int device = 0;
  std::vector<b2k::BProb> probs;
  std::vector<b2k::DpGroup> dpg;
  int n_graph = 0;
  int64_t total_pad = 0, total_rows = 0, n_max = 0;
  b2k::Owned fixed;    // buffers independent of the tuning
  b2k::Owned tuned;    // buffers of the current tuning
  // fixed device buffers
  int* zero_block = nullptr;  // [8 + n_graph] status words, then per-problem range flags
  unsigned long long* counters = nullptr;  // [4]
  uint32_t* skth = nullptr;   // [total_pad]
  float* E = nullptr;         // [total_pad]
  double* nq = nullptr;       // [total_pad] ||q - c||^2 (certify's two-stage refinement)
  uint16_t* ones = nullptr;   // [128, 16]
  CUtensorMap m_ones;
  int64_t* pad_start = nullptr;  // [n_graph + 1]
  int64_t* row_start = nullptr;  // [n_graph + 1]
  b2k::PrepProblem* prep_tab = nullptr;
  b2k::ExactArgs* exact_tab = nullptr;
  int* fb_list = nullptr;     // [total_rows]
  double* scratch = nullptr;  // [exact_grid, n_max]
  int exact_grid = 0;
  // tuned state
  std::vector<b2k::LaunchSpec> specs;
  std::vector<b2k::TcBatchLaunch> launches;
  b2k::CertifyArgs* cert_tab = nullptr;
  int* item_counters = nullptr;  // [launches]
  int work_items = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t own = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float tune_ms = 0;
  bool ran = false;
};

namespace b2k {
namespace {

void drop_graph(b2k_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

// ------------------------------------------------------------ static layout
int build_fixed(b2k_batch* b, cudaStream_t st) {
  std::map<int, int> dp_index;
  std::map<const Index*, std::pair<int64_t, int>> placed;  // index -> (b_row0, dp group)
  int gi = 0;
  for (auto& p : b->probs) {
    if (!p.in_graph) continue;
    p.gi = gi++;
    p.dp = (int)rup(p.ix->d, kTcBK);
    p.KB = p.dp / kTcBK;
    p.n_tiles = (int)(rup(p.ix->n, kTcBN) / kTcBN);
    p.m_pad = (int)rup(p.m, kTcBM);
    p.m_tiles = p.m_pad / kTcBM;
    p.kmax = kmax_class(p.k);
    auto it = dp_index.find(p.dp);
    if (it == dp_index.end()) {
      it = dp_index.emplace(p.dp, (int)b->dpg.size()).first;
      DpGroup g;
      g.dp = p.dp;
      b->dpg.push_back(g);
    }
    p.dpg = it->second;
    DpGroup& g = b->dpg[p.dpg];
    p.a_row0 = g.a_rows;
    g.a_rows += p.m_pad;
    auto pl = placed.find(p.ix);
    if (pl == placed.end()) {
      pl = placed.emplace(p.ix, std::make_pair(g.b_rows, p.dpg)).first;
      g.b_rows += rup(p.ix->n, kTcBN);
    }
    p.b_row0 = pl->second.first;
    p.pad0 = b->total_pad;
    b->total_pad += p.m_pad;
    p.row0 = b->total_rows;
    b->total_rows += p.m;
    b->n_max = std::max<int64_t>(b->n_max, p.ix->n);
  }
  b->n_graph = gi;
  if (gi == 0) return B2K_OK;
  if (b->total_pad >= ((int64_t)1 << 31) || b->total_rows >= ((int64_t)1 << 31))
    return bfail(B2K_EINVAL, "a batch may hold at most 2^31 query rows");
  Owned& o = b->fixed;
  int rc;
  for (auto& g : b->dpg) {
    if (g.a_rows >= ((int64_t)1 << 31) || g.b_rows >= ((int64_t)1 << 31))
      return bfail(B2K_EINVAL, "a batch may hold at most 2^31 rows of one width");
    if ((rc = o.alloc(&g.A, (size_t)g.a_rows * g.dp))) return rc;
    if ((rc = o.alloc(&g.B, (size_t)g.b_rows * g.dp))) return rc;
    if ((rc = o.alloc(&g.Baug, (size_t)g.b_rows * kTcAug))) return rc;
    if (!tensor_map_2d_bf16(&g.ma, g.A, (uint64_t)g.dp, (uint64_t)g.a_rows, kTcBK, kTcBM) ||
        !tensor_map_2d_bf16(&g.mb, g.B, (uint64_t)g.dp, (uint64_t)g.b_rows, kTcBK, kTcBN) ||
        !tensor_map_2d_bf16(&g.mbaug, g.Baug, kTcAug, (uint64_t)g.b_rows, kTcAug, kTcBN, 32))
      return bfail(B2K_ECUDA, "cuTensorMapEncodeTiled failed for a batch operand buffer");
  }
  if ((rc = o.alloc(&b->ones, (size_t)kTcBM * kTcAug))) return rc;
  if (!tensor_map_2d_bf16(&b->m_ones, b->ones, kTcAug, kTcBM, kTcAug, kTcBM, 32))
    return bfail(B2K_ECUDA, "cuTensorMapEncodeTiled failed for the norm columns");
  // reference operands, once per distinct index
  bool ones_done = false;
  std::map<const Index*, std::pair<float, float>> stats;
  for (auto& p : b->probs) {
    if (!p.in_graph) continue;
    auto s = stats.find(p.ix);
    if (s == stats.end()) {
      DpGroup& g = b->dpg[p.dpg];
      float xh = 0, ex = 0;
      rc = index_prepare_bf16_stats(*p.ix, g.B + (size_t)p.b_row0 * g.dp,
                                    g.Baug + (size_t)p.b_row0 * kTcAug,
                                    ones_done ? nullptr : b->ones, st, &xh, &ex);
      if (rc) return rc;
      ones_done = true;
      s = stats.emplace(p.ix, std::make_pair(xh, ex)).first;
    }
    p.xh_max = s->second.first;
    p.ex_max = s->second.second;
  }
  const int P = b->n_graph;
  if ((rc = o.alloc(&b->zero_block, 8 + (size_t)P))) return rc;
  if ((rc = o.alloc(&b->counters, 4))) return rc;
  if ((rc = o.alloc(&b->skth, (size_t)b->total_pad))) return rc;
  if ((rc = o.alloc(&b->E, (size_t)b->total_pad))) return rc;
  if ((rc = o.alloc(&b->nq, (size_t)b->total_pad))) return rc;
  if ((rc = o.alloc(&b->pad_start, (size_t)P + 1))) return rc;
  if ((rc = o.alloc(&b->row_start, (size_t)P + 1))) return rc;
  if ((rc = o.alloc(&b->prep_tab, (size_t)P))) return rc;
  if ((rc = o.alloc(&b->exact_tab, (size_t)P))) return rc;
  if ((rc = o.alloc(&b->fb_list, (size_t)b->total_rows))) return rc;
  b->exact_grid = num_sms(b->device);
  if ((rc = o.alloc(&b->scratch, (size_t)b->exact_grid * b->n_max))) return rc;

  std::vector<int64_t> pad_start(P + 1), row_start(P + 1);
  std::vector<PrepProblem> prep(P);
  std::vector<ExactArgs> ex(P);
  for (auto& p : b->probs) {
    if (!p.in_graph) continue;
    const DpGroup& g = b->dpg[p.dpg];
    pad_start[p.gi] = p.pad0;
    row_start[p.gi] = p.row0;
    PrepProblem& q = prep[p.gi];
    q = PrepProblem{};
    q.Q = p.Q;
    q.m = p.m;
    q.m_pad = p.m_pad;
    q.d = p.ix->d;
    q.dp = p.dp;
    q.mode = B2K_MODE_BF16;
    q.center = p.ix->center;
    q.xh_max = p.xh_max;
    q.nx_max = p.ix->nx_max;
    q.ex_max = p.ex_max;
    q.E = b->E + p.pad0;
    q.Ah = g.A + (size_t)p.a_row0 * g.dp;
    q.nq = b->nq + p.pad0;
    q.flags = b->zero_block + 8 + p.gi;
    ExactArgs& e = ex[p.gi];
    e = ExactArgs{};
    e.X = p.ix->X;
    e.Q = p.Q;
    e.n = p.ix->n;
    e.m = p.m;
    e.d = p.ix->d;
    e.k = p.k;
    e.exclude_self = p.exclude_self;
    e.q_offset = p.q_offset;
    e.dist = p.dist;
    e.idx = p.idx;
    e.counters = b->counters;
    e.status = b->zero_block;
  }
  pad_start[P] = b->total_pad;
  row_start[P] = b->total_rows;
  BCUDA(cudaMemcpyAsync(b->pad_start, pad_start.data(), (P + 1) * sizeof(int64_t),
                        cudaMemcpyHostToDevice, st));
  BCUDA(cudaMemcpyAsync(b->row_start, row_start.data(), (P + 1) * sizeof(int64_t),
                        cudaMemcpyHostToDevice, st));
  BCUDA(cudaMemcpyAsync(b->prep_tab, prep.data(), P * sizeof(PrepProblem),
                        cudaMemcpyHostToDevice, st));
  BCUDA(cudaMemcpyAsync(b->exact_tab, ex.data(), P * sizeof(ExactArgs), cudaMemcpyHostToDevice,
                        st));
  BCUDA(cudaStreamSynchronize(st));
  return B2K_OK;
}

// ------------------------------------------------------------- tuned layout
Tuning tuning_for(const BProb& p, const std::map<TuneKey, Tuning>& tune) {
  auto it = tune.find(TuneKey{p.dp, p.kmax});
  return it == tune.end() ? Tuning{} : it->second;
}

int build_tuned(b2k_batch* b, const std::map<TuneKey, Tuning>& tune, int gran,
                cudaStream_t st) {
  drop_graph(b);
  b->tuned.release();
  b->specs.clear();
  b->launches.clear();
  const int P = b->n_graph;
  if (P == 0) return B2K_OK;
  const int sms = num_sms(b->device);
  // 1. epilogue width and launch class per problem
  std::map<std::tuple<int, int, bool>, std::vector<int>> classes;
  double total_cost = 0;
  for (auto& p : b->probs) {
    if (!p.in_graph) continue;
    const Tuning t = tuning_for(p, tune);
    p.ew = t.ew ? t.ew : default_ew(p.kmax);
    p.halves = p.ew / 4;
    total_cost += (double)p.m_tiles * p.n_tiles * (p.KB + 1);
    classes[std::make_tuple(p.kmax, p.ew, p.KB > 4)].push_back((int)(&p - b->probs.data()));
  }
  // 2. splits: items no larger than the per-CTA share / gran
  const double target = std::max(1.0, total_cost / ((double)sms * gran));
  size_t lists = 0, counts = 0, kth = 0;
  for (auto& p : b->probs) {
    if (!p.in_graph) continue;
    const double item = (double)p.n_tiles * (p.KB + 1);
    int S = (int)std::ceil(item / target);
    S = std::max(1, std::min({S, 16, p.n_tiles}));
    p.tps = (p.n_tiles + S - 1) / S;
    p.S = (p.n_tiles + p.tps - 1) / p.tps;
    p.S_lists = p.S * p.halves;
    // a list never holds more than the columns its slot scans
    p.cap = (int)std::min<int64_t>(kListCap, (int64_t)p.tps * kTcBN / p.halves);
    p.lists_off = lists;
    p.counts_off = counts;
    p.kth_off = kth;
    lists += (size_t)p.S_lists * p.m_pad * p.cap;
    counts += (size_t)p.S_lists * p.m_pad;
    if (p.kmax != 64) kth += (size_t)p.S_lists * p.m_pad * p.k;  // lazy: none
  }
  Owned& o = b->tuned;
  int rc;
  int2* d_lists = nullptr;
  int* d_counts = nullptr;
  float* d_kth = nullptr;
  if ((rc = o.alloc(&d_lists, lists))) return rc;
  if ((rc = o.alloc(&d_counts, counts))) return rc;
  if ((rc = o.alloc(&d_kth, kth))) return rc;
  if ((rc = o.alloc(&b->cert_tab, (size_t)P))) return rc;
  // 3. launches (at most kBatchGroups dp groups each), problem tables
  std::vector<TcProblem> tc(P);
  std::vector<CertifyArgs> cert(P);
  for (auto& cl : classes) {
    LaunchSpec* cur = nullptr;
    for (int pi : cl.second) {
      BProb& p = b->probs[pi];
      if (!cur || (std::find(cur->dpgs.begin(), cur->dpgs.end(), p.dpg) == cur->dpgs.end() &&
                   (int)cur->dpgs.size() == kBatchGroups)) {
        b->specs.push_back(LaunchSpec{std::get<0>(cl.first), std::get<1>(cl.first),
                                      std::get<2>(cl.first), {}, {}});
        cur = &b->specs.back();
      }
      auto g = std::find(cur->dpgs.begin(), cur->dpgs.end(), p.dpg);
      if (g == cur->dpgs.end()) {
        cur->dpgs.push_back(p.dpg);
        g = cur->dpgs.end() - 1;
      }
      p.group = (int)(g - cur->dpgs.begin());
      p.launch = (int)(b->specs.size() - 1);
      cur->probs.push_back(p.gi);
      ScreenOut so{};
      so.lists = d_lists + p.lists_off;
      so.counts = d_counts + p.counts_off;
      so.kth = p.kmax == 64 ? nullptr : d_kth + p.kth_off;
      so.cap = p.cap;
      so.m_pad = p.m_pad;
      TcProblem& t = tc[p.gi];
      t = TcProblem{};
      t.m = (int)p.m;
      t.KB = p.KB;
      t.n_tiles = p.n_tiles;
      t.tiles_per_split = p.tps;
      t.exclude_self = p.exclude_self;
      t.group = p.group;
      t.a_row0 = (int)p.a_row0;
      t.b_row0 = (int)p.b_row0;
      t.q_offset = p.q_offset;
      t.E = b->E + p.pad0;
      t.perm = nullptr;
      t.sink = SinkArgs{};
      t.sink.out = so;
      t.sink.k = p.k;
      t.sink.shared_kth = b->skth + p.pad0;
      t.sink.m_pad = p.m_pad;
      CertifyArgs& c = cert[p.gi];
      c = CertifyArgs{};
      c.X = p.ix->X;
      c.Q = p.Q;
      c.n = p.ix->n;
      c.m = p.m;
      c.d = p.ix->d;
      c.k = p.k;
      c.S = p.S_lists;
      c.scr = so;
      c.E = b->E + p.pad0;
      c.nq = b->nq + p.pad0;  // two-stage refinement (certify.cu)
      c.dist = p.dist;
      c.idx = p.idx;
      c.fallback_list = b->fb_list;
      c.fallback_count = b->zero_block + 2;
      c.counters = b->counters;
      c.perm = nullptr;
      c.row_base = p.row0;
      c.status = b->zero_block;  // a screen that gave up leaves its lists unfinished
    }
  }
  TcProblem* d_tc = nullptr;
  if ((rc = o.alloc(&d_tc, (size_t)P))) return rc;
  BCUDA(cudaMemcpyAsync(d_tc, tc.data(), P * sizeof(TcProblem), cudaMemcpyHostToDevice, st));
  BCUDA(cudaMemcpyAsync(b->cert_tab, cert.data(), P * sizeof(CertifyArgs),
                        cudaMemcpyHostToDevice, st));
  // 4. work items per launch, longest first; the CTAs claim them in that
  //    order as they finish their previous item (greedy LPT online)
  std::vector<const BProb*> by_gi(P);
  for (auto& q : b->probs)
    if (q.in_graph) by_gi[q.gi] = &q;
  b->work_items = 0;
  for (auto& spec : b->specs) {
    struct Item {
      int4 v;
      double cost;
    };
    std::vector<Item> items;
    for (int gi : spec.probs) {
      const TcProblem& t = tc[gi];
      const BProb* p = by_gi[gi];
      for (int s = 0; s < p->S; ++s) {
        const int j0 = s * p->tps, j1 = std::min(j0 + p->tps, t.n_tiles);
        for (int tt = 0; tt < p->m_tiles; ++tt)
          items.push_back(Item{make_int4(gi, tt, j0, j1), (double)(j1 - j0) * (t.KB + 1)});
      }
    }
    std::stable_sort(items.begin(), items.end(),
                     [](const Item& a, const Item& c) { return a.cost > c.cost; });
    const int grid = (int)std::min<size_t>((size_t)sms, items.size());
    std::vector<int4> flat;
    flat.reserve(items.size());
    for (const Item& it : items) flat.push_back(it.v);
    int4* d_items = nullptr;
    if ((rc = o.alloc(&d_items, flat.size()))) return rc;
    BCUDA(cudaMemcpyAsync(d_items, flat.data(), flat.size() * sizeof(int4),
                          cudaMemcpyHostToDevice, st));
    TcBatchLaunch L{};
    L.groups = (int)spec.dpgs.size();
    L.KB_max = 0;
    for (int g = 0; g < L.groups; ++g) {
      const DpGroup& dg = b->dpg[spec.dpgs[g]];
      L.a[g] = dg.ma;
      L.b[g] = dg.mb;
      L.baug[g] = dg.mbaug;
      L.KB_max = std::max(L.KB_max, dg.dp / kTcBK);
    }
    L.aaug = b->m_ones;
    L.probs = d_tc;
    L.items = d_items;
    L.cta_begin = nullptr;
    L.n_items = (int)flat.size();
    L.grid = grid;
    L.kmax = spec.kmax;
    L.ew = spec.ew;
    L.a_stream = spec.a_stream;
    L.status = b->zero_block;
    const int pr = prepare_screen_tc_batch(L.kmax, L.ew, L.a_stream, L.KB_max);
    if (pr) return bfail(B2K_ECUDA, "batched screen setup failed: %s",
                         cudaGetErrorString((cudaError_t)pr));
    b->launches.push_back(L);
    b->work_items += (int)flat.size();
  }
  // one item counter per launch, zeroed at the start of every run
  if ((rc = o.alloc(&b->item_counters, b->launches.size()))) return rc;
  for (size_t i = 0; i < b->launches.size(); ++i)
    b->launches[i].item_counter = b->item_counters + i;
  BCUDA(cudaStreamSynchronize(st));
  return B2K_OK;
}

// The device work of one run, in stream order.
int record(b2k_batch* b, cudaStream_t st) {
  const int P = b->n_graph;
  if (P == 0) return B2K_OK;
  BCUDA(cudaMemsetAsync(b->zero_block, 0, (8 + (size_t)P) * sizeof(int), st));
  BCUDA(cudaMemsetAsync(b->counters, 0, 4 * sizeof(unsigned long long), st));
  BCUDA(cudaMemsetAsync(b->item_counters, 0, b->launches.size() * sizeof(int), st));
  BCUDA(cudaMemsetAsync(b->skth, 0xff, (size_t)b->total_pad * sizeof(uint32_t), st));
  launch_prep_queries_batch(b->prep_tab, b->pad_start, P, b->total_pad, st);
  BCUDA(cudaGetLastError());
  for (const auto& L : b->launches) {
    const int lr = launch_screen_tc_batch(L, st);
    if (lr) return bfail(B2K_ECUDA, "batched tcgen05 screen launch failed: %s",
                         cudaGetErrorString((cudaError_t)lr));
  }
  launch_certify_batch(b->cert_tab, b->row_start, P, b->total_rows, st);
  BCUDA(cudaGetLastError());
  launch_exact_batch(b->exact_tab, b->row_start, P, b->fb_list, b->zero_block + 2, b->scratch,
                     b->n_max, b->exact_grid, st);
  BCUDA(cudaGetLastError());
  return B2K_OK;
}

int capture(b2k_batch* b) {
  drop_graph(b);
  if (b->n_graph == 0) return B2K_OK;
  BCUDA(cudaStreamBeginCapture(b->own, cudaStreamCaptureModeRelaxed));
  int rc = record(b, b->own);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(b->own, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess)
    return bfail(B2K_ECUDA, "graph capture of the batch failed: %s", cudaGetErrorString(e));
  b->graph = g;
  BCUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
  return B2K_OK;
}

// Device status of the last run: error code, per-problem range flags, counters.
int read_status(b2k_batch* b, cudaStream_t st, std::vector<int>& flags,
                unsigned long long* cnt) {
  const int P = b->n_graph;
  flags.assign(8 + P, 0);
  memset(cnt, 0, 4 * sizeof(unsigned long long));
  if (P == 0) return B2K_OK;
  BCUDA(cudaMemcpyAsync(flags.data(), b->zero_block, (8 + P) * sizeof(int),
                        cudaMemcpyDeviceToHost, st));
  BCUDA(cudaMemcpyAsync(cnt, b->counters, 4 * sizeof(unsigned long long),
                        cudaMemcpyDeviceToHost, st));
  BCUDA(cudaStreamSynchronize(st));
  if (injected_fault() == 3) flags[0] = DEV_TIMEOUT_FULL;
  if (flags[0] == DEV_TOO_MANY_TIES)
    return bfail(B2K_EUNSUPPORTED,
                 "more than %d training rows tie (within float64 error) with a query's k-th "
                 "neighbour",
                 kExactCap);
  if (flags[0] != DEV_OK)
    return bfail(B2K_ETIMEOUT, "a bounded device wait gave up (code %d)", flags[0]);
  return B2K_OK;
}

// Time `reps` graph runs (after one warm-up); returns the best in ms, or < 0.
float time_graph(b2k_batch* b, int reps) {
  if (!b->exec) return 0.0f;
  float best = -1.0f;
  for (int r = 0; r <= reps; ++r) {
    cudaEventRecord(b->ev0, b->own);
    if (cudaGraphLaunch(b->exec, b->own) != cudaSuccess) return -1.0f;
    cudaEventRecord(b->ev1, b->own);
    if (cudaEventSynchronize(b->ev1) != cudaSuccess) return -1.0f;
    float ms = 0;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    if (r > 0 && (best < 0 || ms < best)) best = ms;
  }
  std::vector<int> flags;
  unsigned long long cnt[4];
  if (read_status(b, b->own, flags, cnt)) return -1.0f;
  return best;
}

// Coordinate search over the tuning knobs, timing the batch's own graph.
int autotune(b2k_batch* b, std::map<TuneKey, Tuning>& tune, int& gran) {
  std::vector<TuneKey> keys;
  std::map<TuneKey, double> weight;
  for (auto& p : b->probs) {
    if (!p.in_graph) continue;
    TuneKey k{p.dp, p.kmax};
    if (!weight.count(k)) keys.push_back(k);
    weight[k] += (double)p.m_tiles * p.n_tiles * (p.KB + 1);
  }
  std::sort(keys.begin(), keys.end(),
            [&](const TuneKey& a, const TuneKey& c) { return weight[a] > weight[c]; });
  auto trial = [&](float* ms) -> int {
    int rc = build_tuned(b, tune, gran, b->own);
    if (rc) return rc;
    if ((rc = capture(b))) return rc;
    *ms = time_graph(b, 2);
    if (*ms < 0) return bfail(B2K_ECUDA, "autotuning run failed");
    return B2K_OK;
  };
  float best = 0;
  int rc = trial(&best);
  if (rc) return rc;
  // split granularity (whole batch)
  int best_gran = gran;
  for (int g : {2, 8}) {
    gran = g;
    float ms;
    if ((rc = trial(&ms))) return rc;
    if (ms < best * 0.98f) {
      best = ms;
      best_gran = g;
    }
  }
  gran = best_gran;
  // epilogue width per (dp, heap width) bucket
  for (const TuneKey& k : keys) {
    const Tuning cur = tune.count(k) ? tune[k] : Tuning{};
    const int ew0 = cur.ew ? cur.ew : default_ew(k.kmax);
    Tuning keep = cur;
    for (int ew : {16, 8, 4}) {
      if (ew == ew0 || (ew == 16 && k.kmax > 16)) continue;
      Tuning alt;
      alt.ew = ew;
      tune[k] = alt;
      float ms;
      if ((rc = trial(&ms))) return rc;
      if (ms < best * 0.98f) {
        best = ms;
        keep = alt;
      }
    }
    tune[k] = keep;
  }
  return B2K_OK;
}

}  // namespace
}  // namespace b2k

using namespace b2k;

extern "C" {

int b2k_batch_destroy(b2k_batch* b) {
  if (!b) return B2K_OK;
  cudaSetDevice(b->device);
  if (b->own) cudaStreamSynchronize(b->own);
  drop_graph(b);
  b->tuned.release();
  b->fixed.release();
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->own) cudaStreamDestroy(b->own);
  delete b;
  return B2K_OK;
}

int b2k_batch_create(const b2k_problem* problems, int32_t count, int32_t flags, void* stream,
                     b2k_batch** out) {
  if (!out) return bfail(B2K_EINVAL, "out must not be NULL");
  *out = nullptr;
  if (count < 0 || (count > 0 && !problems)) return bfail(B2K_EINVAL, "invalid problem list");
  auto* b = new b2k_batch();
  int device = -1;
  for (int i = 0; i < count; ++i) {
    const b2k_problem& q = problems[i];
    Index* ix = index_of(q.index);
    if (!ix) {
      delete b;
      return bfail(B2K_EINVAL, "problem %d: index must not be NULL", i);
    }
    if (device < 0) device = ix->device;
    if (ix->device != device) {
      delete b;
      return bfail(B2K_EINVAL, "problem %d: all indices of a batch must be on one device", i);
    }
    int rc = check_knn_args(*ix, q.m, q.k, q.exclude_self, q.q_offset);
    if (rc) {
      delete b;
      return rc;
    }
    if (q.m > 0 && (!q.queries || !q.idx)) {
      delete b;
      return bfail(B2K_EINVAL, "problem %d: queries and idx must not be NULL", i);
    }
    BProb p;
    p.ix = ix;
    p.Q = q.queries;
    p.m = q.m;
    p.k = q.k;
    p.exclude_self = q.exclude_self;
    p.q_offset = q.q_offset;
    p.dist = q.dist;
    p.idx = q.idx;
    // the bf16 screen certifies these; the rest go through b2k_knn_device
    p.in_graph = q.m > 0 && ix->range_ok && q.k <= kMaxK && ix->d >= 16;
    b->probs.push_back(p);
  }
  b->device = device < 0 ? 0 : device;
  int rc;
  auto bail = [&](int code) {
    b2k_batch_destroy(b);
    return code;
  };
  if (cudaSetDevice(b->device) != cudaSuccess) return bail(bfail(B2K_ECUDA, "cudaSetDevice failed"));
  if (cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess)
    return bail(bfail(B2K_ECUDA, "stream or event creation failed"));
  // queries may have been written on the caller's stream (NULL: legacy default)
  if (cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) != cudaSuccess)
    return bail(bfail(B2K_ECUDA, "cudaStreamSynchronize failed"));
  if ((rc = build_fixed(b, b->own))) return bail(rc);
  std::map<TuneKey, Tuning> tune;
  int gran;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    tune = g_tune;
    gran = g_gran ? g_gran : kDefaultGran;
  }
  if ((flags & B2K_BATCH_AUTOTUNE) && b->n_graph > 0) {
    bool cached = g_gran != 0;
    for (auto& p : b->probs)
      if (p.in_graph && !tune.count(TuneKey{p.dp, p.kmax})) cached = false;
    if (!cached) {
      cudaEvent_t t0, t1;
      cudaEventCreate(&t0);
      cudaEventCreate(&t1);
      cudaEventRecord(t0, b->own);
      if ((rc = autotune(b, tune, gran))) return bail(rc);
      cudaEventRecord(t1, b->own);
      cudaEventSynchronize(t1);
      cudaEventElapsedTime(&b->tune_ms, t0, t1);
      cudaEventDestroy(t0);
      cudaEventDestroy(t1);
      std::lock_guard<std::mutex> lock(g_tune_mu);
      for (auto& kv : tune) g_tune[kv.first] = kv.second;
      g_gran = gran;
    }
  }
  if ((rc = build_tuned(b, tune, gran, b->own))) return bail(rc);
  // one plain run (sets kernel attributes, checks the plan), then the graph
  if ((rc = record(b, b->own))) return bail(rc);
  {
    std::vector<int> fl;
    unsigned long long cnt[4];
    if ((rc = read_status(b, b->own, fl, cnt))) return bail(rc);
  }
  if ((rc = capture(b))) return bail(rc);
  *out = b;
  return B2K_OK;
}

int b2k_batch_run(b2k_batch* b, void* stream) {
  if (!b) return bfail(B2K_EINVAL, "batch must not be NULL");
  if (injected_fault() == 2) return bfail(B2K_ECUDA, "injected kernel launch failure (B2K_FAULT=launch)");
  BCUDA(cudaSetDevice(b->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (b->exec) {
    BCUDA(cudaEventRecord(b->ev0, st));
    BCUDA(cudaGraphLaunch(b->exec, st));
    BCUDA(cudaEventRecord(b->ev1, st));
  }
  b->ran = true;
  return B2K_OK;
}

int b2k_batch_finish(b2k_batch* b, void* stream, b2k_batch_stats* stats) {
  if (!b) return bfail(B2K_EINVAL, "batch must not be NULL");
  BCUDA(cudaSetDevice(b->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::vector<int> flags;
  unsigned long long cnt[4] = {0, 0, 0, 0};
  int rc = read_status(b, st, flags, cnt);
  if (rc) return rc;
  float run_ms = 0;
  if (b->exec && b->ran) cudaEventElapsedTime(&run_ms, b->ev0, b->ev1);
  // problems outside the graph, and graph problems whose queries left the
  // screen's safe coordinate range (answered exactly)
  int64_t redone = 0;
  for (auto& p : b->probs) {
    if (p.m == 0) continue;
    int mode = -1;
    if (!p.in_graph)
      mode = B2K_MODE_AUTO;
    else if (flags[8 + p.gi] & 1)
      mode = B2K_MODE_EXACT;
    if (mode < 0) continue;
    rc = knn_device_run(*p.ix, p.Q, p.m, p.k, p.exclude_self, p.q_offset, mode, p.dist, p.idx,
                        st);
    if (rc) return rc;
    ++redone;
  }
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->problems = (int32_t)b->probs.size();
    stats->graph_problems = b->n_graph;
    stats->screen_launches = (int32_t)b->launches.size();
    stats->work_items = b->work_items;
    stats->candidates = (int64_t)cnt[0];
    stats->exact_compares = (int64_t)cnt[2];
    stats->fallback_rows = (int64_t)cnt[3];
    stats->tune_ms = b->tune_ms;
    stats->run_ms = run_ms;
  }
  (void)redone;
  return B2K_OK;
}

int b2k_batch_submit(const b2k_problem* problems, int32_t count, void* stream) {
  b2k_batch* b = nullptr;
  int rc = b2k_batch_create(problems, count, 0, stream, &b);
  if (rc) return rc;
  rc = b2k_batch_run(b, stream);
  if (!rc) rc = b2k_batch_finish(b, stream, nullptr);
  b2k_batch_destroy(b);
  return rc;
}

}  // extern "C"
