// C ABI of libb200knn.so: index lifetime and the kNN entry points.
//
// Call flow of one kNN batch (all on one stream):
//   prep_queries  -> per-query screen bound E (and the -2*bf16(q) operand)
//   screen        -> tcgen05 bf16 (screen_tc.cu) or fp32 CUDA-core (screen_simt.cu)
//   certify       -> float64 re-rank + exact near-tie resolution (certify.cu)
//   exact         -> exhaustive exact scan of the rare rows certify could not
//                    finish (list overflow), no-op otherwise
// Scratch buffers come from the stream-ordered allocator (cudaMallocAsync).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdarg>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "internal.cuh"
#include "sinks.cuh"

struct b2k_index {
  b2k::Index ix;
};

namespace b2k {

// ------------------------------------------------------------------ errors
static thread_local std::string g_last_error;

static int fail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
static int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define B2K_CUDA(call)                                                                      \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return fail(e_ == cudaErrorMemoryAllocation ? B2K_ENOMEM : B2K_ECUDA, "%s: %s (%s:%d)", \
                  #call, cudaGetErrorString(e_), __FILE__, __LINE__);                       \
  } while (0)

// Host-side fault injection for failure-path tests (B2K_FAULT=alloc|launch|timeout).
static int fault_mode() {
  const char* f = getenv("B2K_FAULT");
  if (!f || !*f) return 0;
  if (!strcmp(f, "alloc")) return 1;
  if (!strcmp(f, "launch")) return 2;
  if (!strcmp(f, "timeout")) return 3;
  return 0;
}

uint32_t device_spin_limit() {
  const char* e = getenv("B2K_SPIN_LIMIT");
  if (e && *e) {
    const unsigned long v = strtoul(e, nullptr, 10);
    if (v > 0 && v <= kSpinLimit) return (uint32_t)v;
  }
  return kSpinLimit;
}

int num_sms(int device) {
  static int cached[64] = {0};
  if (device < 0 || device >= 64) return 148;
  if (!cached[device]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || v <= 0)
      v = 148;
    cached[device] = v;
  }
  return cached[device];
}

// --------------------------------------------------------------- TMA maps
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

static bool tensor_map_2d(CUtensorMap* map, CUtensorMapDataType type, uint64_t elem_bytes,
                          const void* base, uint64_t inner, uint64_t outer, uint32_t box_inner,
                          uint32_t box_outer, int swizzle_bytes) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {inner, outer};
  cuuint64_t strides[1] = {inner * elem_bytes};
  cuuint32_t box[2] = {box_inner, box_outer};
  cuuint32_t estr[2] = {1, 1};
  const CUtensorMapSwizzle sw = swizzle_bytes == 32   ? CU_TENSOR_MAP_SWIZZLE_32B
                                : swizzle_bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B
                                                      : CU_TENSOR_MAP_SWIZZLE_128B;
  CUresult r = fn(map, type, 2, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

bool tensor_map_2d_bf16(CUtensorMap* map, const void* base, uint64_t inner, uint64_t outer,
                        uint32_t box_inner, uint32_t box_outer, int swizzle_bytes) {
  return tensor_map_2d(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, inner, outer, box_inner,
                       box_outer, swizzle_bytes);
}

bool tensor_map_2d_f32(CUtensorMap* map, const void* base, uint64_t inner, uint64_t outer,
                       uint32_t box_inner, uint32_t box_outer, int swizzle_bytes) {
  return tensor_map_2d(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, inner, outer, box_inner,
                       box_outer, swizzle_bytes);
}

// ------------------------------------------------------------------ helpers
static int check_device(int device) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0)
    return fail(B2K_EUNSUPPORTED, "no CUDA device is available");
  if (device < 0 || device >= count) return fail(B2K_EINVAL, "invalid device %d", device);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess)
    return fail(B2K_ECUDA, "cudaGetDeviceProperties failed");
  if (prop.major != 10)
    return fail(B2K_EUNSUPPORTED, "libb200knn needs an sm_100 (B200) device, found sm_%d%d",
                prop.major, prop.minor);
  return B2K_OK;
}

template <typename T>
static int dalloc(T** p, size_t count, cudaStream_t st) {
  if (fault_mode() == 1) return fail(B2K_ENOMEM, "injected allocation failure (B2K_FAULT=alloc)");
  *p = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(p), count * sizeof(T), st);
  if (e != cudaSuccess)
    return fail(e == cudaErrorMemoryAllocation ? B2K_ENOMEM : B2K_ECUDA,
                "device allocation of %zu bytes failed: %s", count * sizeof(T),
                cudaGetErrorString(e));
  return B2K_OK;
}

static int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

static bool overlaps(const void* a, size_t an, const void* b, size_t bn);

// Whether kNN outputs overlap the queries or each other (internal.cuh).
bool buffers_overlap(const float* dQ, int64_t m, int d, int k, const double* dist,
                     const int64_t* idx) {
  const size_t q = (size_t)m * d * sizeof(float), o = (size_t)m * k * 8;
  return overlaps(idx, o, dQ, q) || overlaps(dist, o, dQ, q) || overlaps(idx, o, dist, o);
}

static bool overlaps(const void* a, size_t an, const void* b, size_t bn) {
  if (!a || !b || !an || !bn) return false;
  auto x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
  return x < y + bn && y < x + an;
}

// Free a list of stream-ordered allocations (ignores nulls).
struct StreamFree {
  cudaStream_t st;
  std::vector<void*> ptrs;
  ~StreamFree() {
    for (void* p : ptrs)
      if (p) cudaFreeAsync(p, st);
  }
  template <typename T>
  T* keep(T* p) {
    ptrs.push_back(p);
    return p;
  }
};

static int finish_index(Index& ix, cudaStream_t st) {
  float init[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  B2K_CUDA(cudaMemcpyAsync(ix.stats_dev, init, sizeof(init), cudaMemcpyHostToDevice, st));
  launch_prep_index(&ix, st);
  B2K_CUDA(cudaGetLastError());
  float stats[8];
  B2K_CUDA(cudaMemcpyAsync(stats, ix.stats_dev, sizeof(stats), cudaMemcpyDeviceToHost, st));
  B2K_CUDA(cudaStreamSynchronize(st));
  ix.xn_max = stats[0];
  ix.nx_max = stats[1];
  ix.ex32_max = stats[5];
  int bad;
  memcpy(&bad, &stats[2], 4);
  ix.range_ok = bad == 0;
  return B2K_OK;
}

// Pivots for query grouping and row grouping (the caller holds ix.mu).
static int make_pivots(Index& ix) {
  if (ix.pivots) return B2K_OK;
  ix.n_pivots = pivot_count(ix.n);
  B2K_CUDA(cudaMalloc(&ix.pivots, (size_t)ix.n_pivots * ix.d * sizeof(float)));
  B2K_CUDA(cudaMalloc(&ix.pivot_norms, (size_t)ix.n_pivots * sizeof(float)));
  ix.pivot_dpa = pivot_dims_padded(ix.d);
  B2K_CUDA(cudaMalloc(&ix.pivots_h,
                      (size_t)pivot_rows_padded(ix.n_pivots) * ix.pivot_dpa * sizeof(uint16_t)));
  launch_pivots(&ix, ix.stream);
  B2K_CUDA(cudaGetLastError());
  B2K_CUDA(cudaStreamSynchronize(ix.stream));
  return B2K_OK;
}

// Indexes of at least this many rows get grouped operand rows (unless
// B2K_GROUP_ROWS=0; tests run both ways).
constexpr int64_t kGroupMinRows = 8192;
static bool group_rows_enabled(const Index& ix) {
  const char* e = getenv("B2K_GROUP_ROWS");
  return ix.n >= kGroupMinRows && !(e && e[0] == '0');
}

// Operand row order grouped by nearest pivot (the caller holds ix.mu): a
// counting sort on the host, stable, so rows keep their training order
// within a group and the layout is the same on every build.
static int make_row_groups(Index& ix) {
  cudaStream_t st = ix.stream;
  int rc = make_pivots(ix);
  if (rc) return rc;
  const int P = ix.n_pivots;
  int *key = nullptr, *hist = nullptr;
  B2K_CUDA(cudaMalloc(&key, (size_t)ix.n * sizeof(int)));
  if (cudaMalloc(&hist, (size_t)P * sizeof(int)) != cudaSuccess) {
    cudaFree(key);
    return fail(B2K_ENOMEM, "device allocation failed");
  }
  launch_assign_rows(&ix, ix.X, ix.n, key, hist, st);
  std::vector<int> hkey((size_t)ix.n);
  cudaError_t e = cudaMemcpyAsync(hkey.data(), key, (size_t)ix.n * sizeof(int),
                                  cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(key);
  cudaFree(hist);
  if (e != cudaSuccess) return fail(B2K_ECUDA, "row grouping: %s", cudaGetErrorString(e));
  std::vector<int64_t> start((size_t)P + 1, 0);
  for (int64_t r = 0; r < ix.n; ++r) ++start[(size_t)hkey[(size_t)r] + 1];
  for (int p = 0; p < P; ++p) start[(size_t)p + 1] += start[(size_t)p];
  std::vector<int> gstart(start.begin(), start.end());  // before the scatter advances them
  std::vector<int> perm((size_t)ix.n), inv((size_t)ix.n);
  for (int64_t r = 0; r < ix.n; ++r) {
    const int64_t pos = start[(size_t)hkey[(size_t)r]]++;
    perm[(size_t)pos] = (int)r;
    inv[(size_t)r] = (int)pos;
  }
  B2K_CUDA(cudaMalloc(&ix.xperm, (size_t)ix.n * sizeof(int)));
  B2K_CUDA(cudaMalloc(&ix.xinv, (size_t)ix.n * sizeof(int)));
  B2K_CUDA(cudaMemcpyAsync(ix.xperm, perm.data(), (size_t)ix.n * sizeof(int),
                           cudaMemcpyHostToDevice, st));
  B2K_CUDA(cudaMemcpyAsync(ix.xinv, inv.data(), (size_t)ix.n * sizeof(int),
                           cudaMemcpyHostToDevice, st));
  B2K_CUDA(cudaMalloc(&ix.group_start, gstart.size() * sizeof(int)));
  B2K_CUDA(cudaMemcpyAsync(ix.group_start, gstart.data(), gstart.size() * sizeof(int),
                           cudaMemcpyHostToDevice, st));
  B2K_CUDA(cudaStreamSynchronize(st));
  return B2K_OK;
}

// Row grouping shared by the tensor-core operands (the caller holds ix.mu):
// decided once, with the first operand built.
static int ensure_row_groups(Index& ix) {
  if (ix.xperm || ix.bf16_ready || ix.tf32_ready || !group_rows_enabled(ix)) return B2K_OK;
  return make_row_groups(ix);
}

static int ensure_bf16(Index& ix) {
  std::lock_guard<std::mutex> lock(ix.mu);
  if (ix.bf16_ready) return B2K_OK;
  cudaStream_t st = ix.stream;
  ix.dp = (int32_t)round_up(ix.d, kTcBK);
  ix.n_pad_tc = round_up(ix.n, kTcBN);
  int rc;
  if ((rc = ensure_row_groups(ix))) return rc;
  B2K_CUDA(cudaMalloc(&ix.Xh, (size_t)ix.n_pad_tc * ix.dp * sizeof(uint16_t)));
  launch_prep_index_bf16(&ix, ix.Xh, st, ix.xperm);
  B2K_CUDA(cudaGetLastError());
  float stats[8];
  B2K_CUDA(cudaMemcpyAsync(stats, ix.stats_dev, sizeof(stats), cudaMemcpyDeviceToHost, st));
  B2K_CUDA(cudaStreamSynchronize(st));
  ix.xh_max = stats[3];
  ix.ex_max = stats[4];
  if (!tensor_map_2d_bf16(&ix.tmap_b, ix.Xh, (uint64_t)ix.dp, (uint64_t)ix.n_pad_tc, kTcBK, kTcBN))
    return fail(B2K_ECUDA, "cuTensorMapEncodeTiled failed for the reference rows");
  // norm columns of the reference rows and the matching query-side ones
  B2K_CUDA(cudaMalloc(&ix.Xaug, (size_t)ix.n_pad_tc * kTcAug * sizeof(uint16_t)));
  B2K_CUDA(cudaMalloc(&ix.aug_ones, (size_t)kTcBM * kTcAug * sizeof(uint16_t)));
  launch_prep_aug(&ix, ix.Xaug, ix.aug_ones, st, ix.xperm);
  B2K_CUDA(cudaGetLastError());
  B2K_CUDA(cudaStreamSynchronize(st));
  if (!tensor_map_2d_bf16(&ix.tmap_baug, ix.Xaug, kTcAug, (uint64_t)ix.n_pad_tc, kTcAug, kTcBN,
                          32) ||
      !tensor_map_2d_bf16(&ix.tmap_aaug, ix.aug_ones, kTcAug, kTcBM, kTcAug, kTcBM, 32))
    return fail(B2K_ECUDA, "cuTensorMapEncodeTiled failed for the norm columns");
  ix.bf16_ready = true;
  return B2K_OK;
}

// tf32 operand of the kind::tf32 screen, in the same row order as the bf16 one.
static int ensure_tf32(Index& ix) {
  std::lock_guard<std::mutex> lock(ix.mu);
  if (ix.tf32_ready) return B2K_OK;
  cudaStream_t st = ix.stream;
  ix.dpt = (int32_t)round_up(ix.d, kTcBKf);
  ix.n_pad_tc = round_up(ix.n, kTcBN);
  int rc;
  if ((rc = ensure_row_groups(ix))) return rc;
  B2K_CUDA(cudaMalloc(&ix.Xt, (size_t)ix.n_pad_tc * ix.dpt * sizeof(float)));
  launch_prep_index_tf32(&ix, ix.Xt, st, ix.xperm);
  B2K_CUDA(cudaGetLastError());
  B2K_CUDA(cudaMalloc(&ix.Xtaug, (size_t)ix.n_pad_tc * kTcAugF * sizeof(float)));
  B2K_CUDA(cudaMalloc(&ix.taug_ones, (size_t)kTcBM * kTcAugF * sizeof(float)));
  launch_prep_aug_tf32(&ix, ix.Xtaug, ix.taug_ones, st, ix.xperm);
  B2K_CUDA(cudaGetLastError());
  float stats[8];
  B2K_CUDA(cudaMemcpyAsync(stats, ix.stats_dev, sizeof(stats), cudaMemcpyDeviceToHost, st));
  B2K_CUDA(cudaStreamSynchronize(st));
  ix.xt_max = stats[6];
  ix.ext_max = stats[7];
  if (!tensor_map_2d_f32(&ix.tmap_bt, ix.Xt, (uint64_t)ix.dpt, (uint64_t)ix.n_pad_tc, kTcBKf,
                         kTcBN) ||
      !tensor_map_2d_f32(&ix.tmap_btaug, ix.Xtaug, kTcAugF, (uint64_t)ix.n_pad_tc, kTcAugF, kTcBN,
                         32) ||
      !tensor_map_2d_f32(&ix.tmap_ataug, ix.taug_ones, kTcAugF, kTcBM, kTcAugF, kTcBM, 32))
    return fail(B2K_ECUDA, "cuTensorMapEncodeTiled failed for the tf32 operand");
  ix.tf32_ready = true;
  return B2K_OK;
}

// Whether every one of `count` values is an integer in [0, 255]: one check
// kernel and a 4-byte read (the flag is freed on every path).
static int all_u8(const float* v, int64_t count, cudaStream_t st, bool* yes) {
  *yes = false;
  int* flag = nullptr;
  int rc = dalloc(&flag, 1, st);
  if (rc) return rc;
  int h = 1;
  cudaError_t e = cudaMemsetAsync(flag, 0, sizeof(int), st);
  if (e == cudaSuccess) {
    launch_u8_check(v, count, flag, st);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFreeAsync(flag, st);
  if (e != cudaSuccess) return fail(B2K_ECUDA, "u8 check: %s", cudaGetErrorString(e));
  *yes = h == 0;
  return B2K_OK;
}

// The exact u8 screen's operand, when every training coordinate is an
// integer in [0, 255] (checked once); *ok tells whether the index qualifies.
static int ensure_u8(Index& ix, bool* ok) {
  std::lock_guard<std::mutex> lock(ix.mu);
  *ok = false;
  if (ix.d > kU8MaxD) return B2K_OK;
  cudaStream_t st = ix.stream;
  int rc;
  if (ix.u8_state == 0) {
    bool yes = false;
    if ((rc = all_u8(ix.X, ix.n * (int64_t)ix.d, st, &yes))) return rc;
    ix.u8_state = yes ? 1 : -1;
  }
  if (ix.u8_state < 0) return B2K_OK;
  if (!ix.u8_ready) {
    // a failed build leaves nothing allocated, so a later call starts over
    struct Partial {
      Index& ix;
      bool done = false;
      ~Partial() {
        if (done) return;
        cudaFree(ix.Xu);
        cudaFree(ix.nxu);
        ix.Xu = nullptr;
        ix.nxu = nullptr;
      }
    } partial{ix};
    ix.dpu = (int32_t)round_up(ix.d, kTcBKu);
    ix.n_pad_tc = round_up(ix.n, kTcBN);
    B2K_CUDA(cudaMalloc(&ix.Xu, (size_t)ix.n_pad_tc * ix.dpu));
    B2K_CUDA(cudaMalloc(&ix.nxu, (size_t)ix.n_pad_tc * sizeof(int)));
    // padding rows: v = INT_MAX, never admitted
    launch_prep_u8(ix.X, ix.n, ix.d, ix.n_pad_tc, ix.dpu, ix.Xu, ix.nxu, nullptr, INT_MAX, st);
    B2K_CUDA(cudaGetLastError());
    B2K_CUDA(cudaStreamSynchronize(st));
    if (!tensor_map_2d(&ix.tmap_bu, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, ix.Xu, (uint64_t)ix.dpu,
                       (uint64_t)ix.n_pad_tc, kTcBKu, kTcBN, 128))
      return fail(B2K_ECUDA, "cuTensorMapEncodeTiled failed for the u8 operand");
    partial.done = true;
    ix.u8_ready = true;
  }
  *ok = true;
  return B2K_OK;
}

static int choose_splits(int64_t m_tiles, int64_t n_tiles, int64_t slots);

// Exact kNN of integer queries on a u8 index (exact_u8.cu): prep, the
// kind::i8 screen, the merge of the lists.  dQ's rows are integers in [0, 255].
static int run_u8(Index& ix, const float* dQ, int64_t m, int k, int exclude_self,
                  int64_t q_offset, double* d_dist, int64_t* d_idx, int squared, int* status,
                  cudaStream_t st, StreamFree& fr, int* splits_out) {
  int rc;
  const int64_t m_pad = round_up(m, kTcBM);
  const int64_t n_tiles = ix.n_pad_tc / kTcBN;
  const int S = choose_splits(m_pad / kTcBM, n_tiles, num_sms(ix.device));
  const int S_lists = S * tc_u8_column_groups(k);
  *splits_out = S;
  uint8_t* Qu = nullptr;
  int64_t* nq = nullptr;
  uint32_t* shared_kth = nullptr;
  if ((rc = dalloc(&Qu, (size_t)m_pad * ix.dpu, st))) return rc;
  fr.keep(Qu);
  if ((rc = dalloc(&nq, (size_t)m_pad, st))) return rc;
  fr.keep(nq);
  if ((rc = dalloc(&shared_kth, (size_t)m_pad, st))) return rc;
  fr.keep(shared_kth);
  B2K_CUDA(cudaMemsetAsync(shared_kth, 0xff, (size_t)m_pad * sizeof(uint32_t), st));
  launch_prep_u8(dQ, m, ix.d, m_pad, ix.dpu, Qu, nullptr, nq, 0, st);
  ScreenOut so{};
  so.cap = k;
  so.m_pad = (int)m_pad;
  if ((rc = dalloc(&so.lists, (size_t)S_lists * m_pad * k, st))) return rc;
  fr.keep(so.lists);
  SinkArgs sa{};
  sa.out = so;
  sa.k = k;
  sa.shared_kth = shared_kth;
  CUtensorMap tmap_a;
  if (!tensor_map_2d(&tmap_a, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, Qu, (uint64_t)ix.dpu,
                     (uint64_t)m_pad, kTcBKu, kTcBM, 128))
    return fail(B2K_ECUDA, "cuTensorMapEncodeTiled failed for the u8 query rows");
  // status[6] (zeroed by the caller) counts the claimed work units
  const int lr = launch_screen_tc_u8(&ix, &tmap_a, m, m_pad, exclude_self, q_offset, S, sa,
                                     status, st, status + 6);
  if (lr) return fail(B2K_ECUDA, "u8 tcgen05 screen launch failed: %s",
                      cudaGetErrorString((cudaError_t)lr));
  launch_u8_merge(so.lists, S_lists, m, m_pad, k, nq, squared, d_dist, d_idx, status, st);
  B2K_CUDA(cudaGetLastError());
  return B2K_OK;
}

static int ensure_pivots(Index& ix) {
  std::lock_guard<std::mutex> lock(ix.mu);
  return make_pivots(ix);
}

// Query grouping is on unless B2K_REORDER=0 (tests run both ways).
static bool reorder_enabled() {
  const char* e = getenv("B2K_REORDER");
  return !(e && e[0] == '0');
}

// Seeding pass over each query tile's home window (grouped rows): on unless
// B2K_SEED=0 (tests run both ways).
// Reference tiles per query tile of the seeding pass's home window
// (B2K_SEED_TILES overrides).  16 was the fastest of 8, 16 and 32 on 100k
// queries of the 1M x 128 mixture, k = 10: 8 tiles admit 4% more list
// entries in the main pass, 32 spend 0.22 ms more seeding than they save.
static int seed_tiles() {
  const char* e = getenv("B2K_SEED_TILES");
  const int t = e ? atoi(e) : 16;
  return t < 1 ? 1 : (t > 256 ? 256 : t);
}
static bool seed_enabled() {
  const char* e = getenv("B2K_SEED");
  return !(e && e[0] == '0');
}

// Reference splits: fill the GPU with (query tile, split) work units while
// keeping the number of candidate lists per query small.  Up to 64 splits, so
// a batch of one or two query tiles (a small call, or the second pass over a
// few uncertified rows) still spreads over most of the SMs.
constexpr int kMaxSplits = 64;
static int choose_splits(int64_t m_tiles, int64_t n_tiles, int64_t slots) {
  if (m_tiles <= 0 || n_tiles <= 0) return 1;
  int best = 1;
  double best_cost = 1e300;
  for (int S = 1; S <= kMaxSplits && S <= n_tiles; ++S) {
    const double units = (double)m_tiles * S;
    const double waves = std::ceil(units / (double)slots);
    // time ~ waves * (n_tiles / S); small penalty per extra split (more list traffic)
    const double cost = waves * std::ceil((double)n_tiles / S) * (1.0 + 0.01 * (S - 1));
    if (cost < best_cost - 1e-9) {
      best_cost = cost;
      best = S;
    }
  }
  return best;
}

static int run_exact(Index& ix, const float* dQ, int64_t m, int k, int exclude_self,
                     int64_t q_offset, double* d_dist, int64_t* d_idx, const int* rows,
                     const int* row_count, unsigned long long* counters, int* status,
                     cudaStream_t st, StreamFree& fr, bool use_scratch,
                     const int* perm = nullptr, int squared = 0) {
  ExactArgs ea{};
  ea.perm = perm;
  ea.squared = squared;
  ea.X = ix.X;
  ea.Q = dQ;
  ea.n = ix.n;
  ea.m = m;
  ea.d = ix.d;
  ea.k = k;
  ea.exclude_self = exclude_self;
  ea.q_offset = q_offset;
  ea.rows = rows;
  ea.row_count = row_count;
  ea.dist = d_dist;
  ea.idx = d_idx;
  ea.counters = counters;
  ea.status = status;
  const int sms = num_sms(ix.device);
  ea.grid = (int)std::min<int64_t>(rows ? sms : m, (int64_t)2 * sms);
  if (ea.grid <= 0) return B2K_OK;
  ea.scratch = nullptr;
  if (use_scratch) {
    int rc = dalloc(&ea.scratch, (size_t)ea.grid * ix.n, st);
    if (rc) return rc;
    fr.keep(ea.scratch);
  }
  launch_exact(ea, st);
  B2K_CUDA(cudaGetLastError());
  return B2K_OK;
}

// ext_perm (optional): the rows of dQ are already in screen order, and row i
// answers query ext_perm[i] (its output row and self index); used for the
// second pass over rows a bf16 pass could not certify.
static int knn_device_impl(Index& ix, const float* dQ, int64_t m, int k, int exclude_self,
                           int64_t q_offset, int mode, double* d_dist, int64_t* d_idx,
                           cudaStream_t st, b2k_stats* stats, const int* ext_perm = nullptr) {
  const int fm = fault_mode();
  if (fm == 2) return fail(B2K_ECUDA, "injected kernel launch failure (B2K_FAULT=launch)");
  const int squared = (mode & B2K_MODE_SQUARED) ? 1 : 0;
  const int sq_flag = squared ? B2K_MODE_SQUARED : 0;
  mode &= ~B2K_MODE_SQUARED;
  int rc;
  bool u8 = false;
  // Integer pixels: the exact u8 screen, when the index and every query
  // coordinate are integers in [0, 255] (AUTO in the bf16 screen's size range,
  // or asked for); otherwise the certified screens.
  if (m > 0 && k <= kU8MaxK && ix.range_ok &&
      (mode == B2K_MODE_U8 || (mode == B2K_MODE_AUTO && ix.d >= 16 && ix.n >= 2048))) {
    bool ok = false;
    if ((rc = ensure_u8(ix, &ok))) return rc;
    if (ok) {
      cudaSetDevice(ix.device);
      if ((rc = all_u8(dQ, m * (int64_t)ix.d, st, &ok))) return rc;
    }
    u8 = ok;
  }
  if (mode == B2K_MODE_U8) mode = B2K_MODE_AUTO;  // not integer pixels: the certified screens
  if (u8) mode = B2K_MODE_U8;
  if (mode == B2K_MODE_AUTO)
    mode = (!ix.range_ok || k > kMaxK) ? B2K_MODE_EXACT
           : (ix.d >= 16 && ix.n >= 2048) ? B2K_MODE_BF16
                                         : B2K_MODE_FP32;
  if (mode != B2K_MODE_EXACT && !u8 && (!ix.range_ok || k > kMaxK)) mode = B2K_MODE_EXACT;
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->mode_used = mode;
  }
  if (m == 0) return B2K_OK;
  cudaSetDevice(ix.device);
  StreamFree fr{st, {}};
  // call start, screen start, screen end, call end, seeding pass end
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  bool seeded = false;
  if (stats)
    for (auto& e : ev) cudaEventCreate(&e);
  if (stats) cudaEventRecord(ev[0], st);

  int* status = nullptr;
  unsigned long long* counters = nullptr;
  if ((rc = dalloc(&status, 8, st))) return rc;
  fr.keep(status);
  if ((rc = dalloc(&counters, 8, st))) return rc;
  fr.keep(counters);
  B2K_CUDA(cudaMemsetAsync(status, 0, 8 * sizeof(int), st));
  B2K_CUDA(cudaMemsetAsync(counters, 0, 8 * sizeof(unsigned long long), st));
  // NaN / inf queries: flagged on the device, reported with the final status
  // read (the search itself stays bounded on such inputs)
  launch_nonfinite_check(dQ, m * (int64_t)ix.d, status + 5, st);

  int S = 1;
  int64_t second_pass_rows = 0, second_exact_rows = 0;
  if (mode == B2K_MODE_EXACT) {
    rc = run_exact(ix, dQ, m, k, exclude_self, q_offset, d_dist, d_idx, nullptr, nullptr,
                   counters, status, st, fr, true, ext_perm, squared);
    if (rc) return rc;
  } else if (mode == B2K_MODE_U8) {
    if (stats) cudaEventRecord(ev[1], st);
    rc = run_u8(ix, dQ, m, k, exclude_self, q_offset, d_dist, d_idx, squared, status, st, fr, &S);
    if (rc) return rc;
    if (stats) cudaEventRecord(ev[2], st);
  } else {
    if (mode == B2K_MODE_BF16 && (rc = ensure_bf16(ix))) return rc;
    if (mode == B2K_MODE_TF32 && (rc = ensure_tf32(ix))) return rc;
    const bool tf32 = mode == B2K_MODE_TF32;
    const bool tc = mode == B2K_MODE_BF16 || tf32;
    const int64_t bm = tc ? kTcBM : kSimtBM;
    const int64_t m_pad = round_up(m, bm);
    const int64_t n_tiles = tc ? ix.n_pad_tc / kTcBN : (ix.n + kSimtBN - 1) / kSimtBN;
    const int sms = num_sms(ix.device);
    S = choose_splits(m_pad / bm, n_tiles, tc ? sms : 2 * sms);
    // lists per query: one per (split, column group of the screen)
    const int S_lists = S * (tc ? tc_column_groups(k) : simt_column_groups(kSinkKnn));
    // Group nearby queries (reorder.cu); results go back to the original rows.
    const int* perm = ext_perm;
    const float* Qs = dQ;
    int* key = nullptr;  // nearest pivot of each query (query grouping)
    if (!ext_perm && m >= 2048 && reorder_enabled()) {
      if ((rc = ensure_pivots(ix))) return rc;
      int *hist = nullptr, *pm = nullptr;
      float* Qp = nullptr;
      if ((rc = dalloc(&key, (size_t)m, st))) return rc;
      fr.keep(key);
      if ((rc = dalloc(&hist, (size_t)ix.n_pivots, st))) return rc;
      fr.keep(hist);
      if ((rc = dalloc(&pm, (size_t)m, st))) return rc;
      fr.keep(pm);
      if ((rc = dalloc(&Qp, (size_t)m * ix.d, st))) return rc;
      fr.keep(Qp);
      launch_query_order(&ix, dQ, m, key, hist, pm, Qp, st);
      B2K_CUDA(cudaGetLastError());
      perm = pm;
      Qs = Qp;
    }
    uint32_t* shared_kth = nullptr;
    if ((rc = dalloc(&shared_kth, (size_t)m_pad, st))) return rc;
    fr.keep(shared_kth);
    B2K_CUDA(cudaMemsetAsync(shared_kth, 0xff, (size_t)m_pad * sizeof(uint32_t), st));
    QueryPrep qp{};
    if ((rc = dalloc(&qp.E, (size_t)m_pad, st))) return rc;
    fr.keep(qp.E);
    qp.flags = status + 4;  // shares the zeroed status block
    // ||y_q||^2 for the certify pass's two-stage refinement
    if ((rc = dalloc(&qp.nq, (size_t)m_pad, st))) return rc;
    fr.keep(qp.nq);
    if (tc && !tf32) {
      if ((rc = dalloc(&qp.Ah, (size_t)m_pad * ix.dp, st))) return rc;
      fr.keep(qp.Ah);
    }
    if (tf32) {
      if ((rc = dalloc(&qp.At, (size_t)m_pad * ix.dpt, st))) return rc;
      fr.keep(qp.At);
    }
    launch_prep_queries(&ix, Qs, m, m_pad, mode, qp, st);
    B2K_CUDA(cudaGetLastError());
    ScreenOut so{};
    // the register trackers' lists hold 4 x kListCap entries per (split, query)
    // whatever the column groups (the lazy tracker's select is sized for kListCap)
    so.cap = (tc && !tc_lazy_sink(k)) ? kListCap * 4 / tc_column_groups(k) : kListCap;
    so.m_pad = (int)m_pad;
    if ((rc = dalloc(&so.lists, (size_t)S_lists * m_pad * so.cap, st))) return rc;
    fr.keep(so.lists);
    if ((rc = dalloc(&so.counts, (size_t)S_lists * m_pad, st))) return rc;
    fr.keep(so.counts);
    if (!(tc && tc_lazy_sink(k))) {  // lazy screens leave V_k to the lists
      if ((rc = dalloc(&so.kth, (size_t)S_lists * m_pad * k, st))) return rc;
      fr.keep(so.kth);
    }
    SinkArgs sa{};
    sa.out = so;
    sa.k = k;
    sa.shared_kth = shared_kth;
    if (stats) cudaEventRecord(ev[1], st);
    if (tc) {
      CUtensorMap tmap_a;
      const bool map_ok =
          tf32 ? tensor_map_2d_f32(&tmap_a, qp.At, (uint64_t)ix.dpt, (uint64_t)m_pad, kTcBKf,
                                   kTcBM)
               : tensor_map_2d_bf16(&tmap_a, qp.Ah, (uint64_t)ix.dp, (uint64_t)m_pad, kTcBK,
                                    kTcBM);
      if (!map_ok) return fail(B2K_ECUDA, "cuTensorMapEncodeTiled failed for the query rows");
      // Seeding: with grouped rows, a query's neighbours sit in the few
      // reference tiles of its pivot's group, which the main screen may
      // reach late; until then its lists would admit the band around the
      // nearest other clusters.  A first pass over each query tile's home
      // window publishes k-th screen values (its sink keeps no list:
      // capacity 0) to the per-query words the main screen's lists start
      // from.  A published value is the k-th smallest of real screen values
      // of the query, so it is >= the final V_k and the certificate holds.
      const int64_t m_tiles = m_pad / kTcBM;
      const int kSeedTiles = seed_tiles();
      if (key && ix.group_start && !tc_lazy_sink(k) && n_tiles >= 2 * kSeedTiles &&
          seed_enabled()) {
        const int G = tc_column_groups(k);
        int* home = nullptr;
        int* seed_counts = nullptr;
        float* seed_kth = nullptr;
        if ((rc = dalloc(&home, (size_t)m_tiles, st))) return rc;
        fr.keep(home);
        if ((rc = dalloc(&seed_counts, (size_t)G * m_pad, st))) return rc;
        fr.keep(seed_counts);
        if ((rc = dalloc(&seed_kth, (size_t)G * m_pad * k, st))) return rc;
        fr.keep(seed_kth);
        launch_home_tiles(perm, key, m, ix.group_start, (int)n_tiles, kSeedTiles, home,
                          (int)m_tiles, st);
        SinkArgs sb = sa;
        sb.out.cap = 0;  // the trackers only: no list entry is written
        sb.out.counts = seed_counts;
        sb.out.kth = seed_kth;
        // status[7] (zeroed above) counts this pass's claimed units
        int lr = launch_screen_tc(&ix, &tmap_a, m, m_pad, exclude_self, q_offset, 1, qp.E,
                                  kSinkKnn, sb, status, st, perm, status + 7, tf32, home,
                                  kSeedTiles);
        if (lr) return fail(B2K_ECUDA, "tcgen05 seeding screen launch failed: %s",
                            cudaGetErrorString((cudaError_t)lr));
        if (stats) cudaEventRecord(ev[4], st);
        seeded = true;
      }
      // status[6] (zeroed above) counts the claimed work units
      int lr = launch_screen_tc(&ix, &tmap_a, m, m_pad, exclude_self, q_offset, S, qp.E,
                                kSinkKnn, sa, status, st, perm, status + 6, tf32);
      if (lr) return fail(B2K_ECUDA, "tcgen05 screen launch failed: %s",
                          cudaGetErrorString((cudaError_t)lr));
    } else {
      launch_screen_simt(&ix, Qs, m, m_pad, exclude_self, q_offset, S, qp.E, kSinkKnn, sa, st,
                         perm);
      B2K_CUDA(cudaGetLastError());
    }
    if (stats) cudaEventRecord(ev[2], st);
    int* fb_list = nullptr;
    if ((rc = dalloc(&fb_list, (size_t)m, st))) return rc;
    fr.keep(fb_list);
    CertifyArgs ca{};
    ca.X = ix.X;
    ca.Q = Qs;
    ca.n = ix.n;
    ca.m = m;
    ca.d = ix.d;
    ca.k = k;
    ca.S = S_lists;
    ca.scr = so;
    ca.E = qp.E;
    ca.dist = d_dist;
    ca.idx = d_idx;
    ca.fallback_list = fb_list;
    ca.fallback_count = status + 2;
    ca.counters = counters;
    ca.perm = perm;
    ca.squared = squared;
    ca.cols = tc ? ix.xperm : nullptr;  // lists of the grouped bf16 operand
    ca.status = status;
    ca.nq = qp.nq;
    ca.refined = counters + 4;
    launch_certify(ca, st);
    B2K_CUDA(cudaGetLastError());
    // Rows the screen could not certify (a list past capacity, too many
    // candidates or survivors).  After a bf16 pass they get a second pass with
    // the fp32 screen, whose bound is ~50x tighter; otherwise (and for rows the
    // fp32 pass cannot certify) the exhaustive exact scan.
    bool second_pass = false;
    if (tc) {
      int nfb = 0;
      B2K_CUDA(cudaMemcpyAsync(&nfb, status + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
      B2K_CUDA(cudaStreamSynchronize(st));
      if (nfb > 0) {
        float* Qfb = nullptr;
        int* pfb = nullptr;
        if ((rc = dalloc(&Qfb, (size_t)nfb * ix.d, st))) return rc;
        fr.keep(Qfb);
        if ((rc = dalloc(&pfb, (size_t)nfb, st))) return rc;
        fr.keep(pfb);
        launch_gather_fallback(Qs, ix.d, fb_list, perm, nfb, Qfb, pfb, st);
        B2K_CUDA(cudaGetLastError());
        b2k_stats sub{};
        rc = knn_device_impl(ix, Qfb, nfb, k, exclude_self, q_offset, B2K_MODE_FP32 | sq_flag,
                             d_dist, d_idx, st, &sub, pfb);
        if (rc) return rc;
        second_pass_rows = nfb;
        second_exact_rows = sub.fallback_rows;
      }
      second_pass = true;
    }
    if (!second_pass) {
      rc = run_exact(ix, Qs, m, k, exclude_self, q_offset, d_dist, d_idx, fb_list, status + 2,
                     counters, status, st, fr, false, perm, squared);
      if (rc) return rc;
    }
  }
  if (stats) cudaEventRecord(ev[3], st);
  int hstatus[8];
  unsigned long long hcnt[5];
  B2K_CUDA(cudaMemcpyAsync(hstatus, status, sizeof(hstatus), cudaMemcpyDeviceToHost, st));
  B2K_CUDA(cudaMemcpyAsync(hcnt, counters, sizeof(hcnt), cudaMemcpyDeviceToHost, st));
  B2K_CUDA(cudaStreamSynchronize(st));
  if (fm == 3) hstatus[0] = DEV_TIMEOUT_FULL;
  if (hstatus[5]) return fail(B2K_ENONFINITE, "training and query coordinates must be finite");
  if (hstatus[0] == DEV_TOO_MANY_TIES)
    return fail(B2K_EUNSUPPORTED,
                "more than %d training rows tie (within float64 error) with a query's k-th "
                "neighbour",
                kExactCap);
  if (hstatus[0] != DEV_OK)
    return fail(B2K_ETIMEOUT, "a bounded device wait gave up (code %d)", hstatus[0]);
  if (hstatus[4] & 1) {
    // Some query coordinate is outside the screens' safe range: redo exactly.
    return knn_device_impl(ix, dQ, m, k, exclude_self, q_offset, B2K_MODE_EXACT | sq_flag,
                           d_dist, d_idx, st, stats, ext_perm);
  }
  if (stats) {
    stats->splits = S;
    stats->candidates = (int64_t)hcnt[0];
    stats->list_entries = (int64_t)hcnt[1];
    stats->exact_compares = (int64_t)hcnt[2];
    stats->fallback_rows = (int64_t)hcnt[3] + second_exact_rows;
    stats->second_pass_rows = second_pass_rows;
    stats->refined = (int64_t)hcnt[4];
    float ms = 0;
    if (mode != B2K_MODE_EXACT && cudaEventElapsedTime(&ms, ev[1], ev[2]) == cudaSuccess)
      stats->screen_ms = ms;
    if (cudaEventElapsedTime(&ms, ev[0], ev[3]) == cudaSuccess) stats->total_ms = ms;
    if (seeded && cudaEventElapsedTime(&ms, ev[1], ev[4]) == cudaSuccess) stats->seed_ms = ms;
    for (auto& e : ev) cudaEventDestroy(e);
  }
  return B2K_OK;
}

static int validate_knn(const Index& ix, int64_t m, int32_t k, int32_t exclude_self,
                        int64_t q_offset, int32_t mode) {
  if (m < 0) return fail(B2K_EINVAL, "negative query count");
  if (k <= 0) return fail(B2K_EINVAL, "Expected n_neighbors > 0. Got %d", k);
  const int64_t limit = ix.n - (exclude_self ? 1 : 0);
  if (k > limit) return fail(B2K_EINVAL, "n_neighbors must be <= %lld, got %d.", (long long)limit, k);
  if (m >= (int64_t)1 << 31) return fail(B2K_EINVAL, "query count must fit int32");
  if (exclude_self && (q_offset < 0 || q_offset + m > ix.n))
    return fail(B2K_EINVAL,
                "exclude_self requires the query matrix to be the training matrix: got %lld "
                "query rows at offset %lld and %lld training rows.",
                (long long)m, (long long)q_offset, (long long)ix.n);
  const int32_t base = mode & ~B2K_MODE_SQUARED;
  if (base < B2K_MODE_AUTO || base > B2K_MODE_U8) return fail(B2K_EINVAL, "unknown mode %d", mode);
  return B2K_OK;
}

// Shared with the other host translation units (internal.cuh).
int report_error(int code, const char* msg) { return fail(code, "%s", msg); }
int check_knn_args(const Index& ix, int64_t m, int32_t k, int32_t exclude_self,
                   int64_t q_offset) {
  return validate_knn(ix, m, k, exclude_self, q_offset, B2K_MODE_AUTO);
}
Index* index_of(b2k_index* h) { return h ? &h->ix : nullptr; }
int knn_device_run(Index& ix, const float* dQ, int64_t m, int k, int exclude_self,
                   int64_t q_offset, int mode, double* d_dist, int64_t* d_idx, cudaStream_t st) {
  return knn_device_impl(ix, dQ, m, k, exclude_self, q_offset, mode, d_dist, d_idx, st, nullptr);
}
int injected_fault() { return fault_mode(); }
int index_prepare_bf16_stats(Index& ix, uint16_t* Xh, uint16_t* Xaug, uint16_t* ones,
                             cudaStream_t st, float* xh_max, float* ex_max) {
  std::lock_guard<std::mutex> lock(ix.mu);
  launch_prep_index_bf16(&ix, Xh, st);
  B2K_CUDA(cudaGetLastError());
  launch_prep_aug(&ix, Xaug, ones, st);
  B2K_CUDA(cudaGetLastError());
  float stats[8];
  B2K_CUDA(cudaMemcpyAsync(stats, ix.stats_dev, sizeof(stats), cudaMemcpyDeviceToHost, st));
  B2K_CUDA(cudaStreamSynchronize(st));
  *xh_max = stats[3];
  *ex_max = stats[4];
  return B2K_OK;
}

// Whether count device floats are all finite (one pass on the device).
static int device_finite(const float* dv, size_t count, cudaStream_t st, bool* ok) {
  int* flag = nullptr;
  int rc = dalloc(&flag, 1, st);
  if (rc) return rc;
  int h = 0;
  cudaMemsetAsync(flag, 0, sizeof(int), st);
  launch_nonfinite_check(dv, (int64_t)count, flag, st);
  cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(flag, st);
  B2K_CUDA(cudaStreamSynchronize(st));
  *ok = h == 0;
  return B2K_OK;
}


}  // namespace b2k

using namespace b2k;

// ===================================================================== C ABI
extern "C" {

int b2k_version(void) { return 100; }

const char* b2k_last_error(void) { return g_last_error.c_str(); }

static int create_common(int device, int64_t n, int32_t d, b2k_index** out) {
  if (!out) return fail(B2K_EINVAL, "out must not be NULL");
  *out = nullptr;
  if (n <= 0 || d <= 0) return fail(B2K_EINVAL, "X must be a nonempty two-dimensional matrix");
  if (n >= ((int64_t)1 << 31)) return fail(B2K_EINVAL, "training row count must fit int32 indices");
  if (fault_mode() == 1) return fail(B2K_ENOMEM, "injected allocation failure (B2K_FAULT=alloc)");
  return check_device(device);
}

// Keep the stream-ordered pool's memory mapped between calls (the default
// release threshold of 0 unmaps it at every synchronisation, so each query
// batch would re-map its scratch).
static void keep_pool(int device) {
  static bool done[64] = {false};
  if (device < 0 || device >= 64 || done[device]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t threshold = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
  }
  done[device] = true;
}

static int build_from_device(b2k_index* h, const float* src, cudaMemcpyKind kind,
                             cudaStream_t user_st) {
  Index& ix = h->ix;
  B2K_CUDA(cudaSetDevice(ix.device));
  keep_pool(ix.device);
  B2K_CUDA(cudaStreamCreateWithFlags(&ix.stream, cudaStreamNonBlocking));
  const size_t bytes = (size_t)ix.n * ix.d * sizeof(float);
  B2K_CUDA(cudaMalloc(&ix.X, bytes));
  B2K_CUDA(cudaMalloc(&ix.nx32, (size_t)ix.n * sizeof(float)));
  B2K_CUDA(cudaMalloc(&ix.center, (size_t)ix.d * sizeof(float)));
  B2K_CUDA(cudaMalloc(&ix.colsum, (size_t)ix.d * sizeof(double)));
  B2K_CUDA(cudaMalloc(&ix.nx64, (size_t)ix.n * sizeof(double)));
  B2K_CUDA(cudaMalloc(&ix.stats_dev, 8 * sizeof(float)));
  if (kind == cudaMemcpyDeviceToDevice && user_st) {
    B2K_CUDA(cudaMemcpyAsync(ix.X, src, bytes, kind, user_st));
    B2K_CUDA(cudaStreamSynchronize(user_st));
  } else {
    B2K_CUDA(cudaMemcpyAsync(ix.X, src, bytes, kind, ix.stream));
  }
  return finish_index(ix, ix.stream);
}

int b2k_index_create(const float* X, int64_t n, int32_t d, int32_t device, b2k_index** out) {
  int rc = create_common(device, n, d, out);
  if (rc) return rc;
  if (!X) return fail(B2K_EINVAL, "X must not be NULL");
  auto* h = new b2k_index();
  h->ix.device = device;
  h->ix.n = n;
  h->ix.d = d;
  rc = build_from_device(h, X, cudaMemcpyHostToDevice, nullptr);
  bool ok = true;
  if (!rc) rc = device_finite(h->ix.X, (size_t)n * d, h->ix.stream, &ok);
  if (!rc && !ok) rc = fail(B2K_ENONFINITE, "training coordinates must be finite");
  if (rc) {
    b2k_index_destroy(h);
    return rc;
  }
  *out = h;
  return B2K_OK;
}

int b2k_index_create_device(const float* dX, int64_t n, int32_t d, void* stream,
                            b2k_index** out) {
  int device = 0;
  cudaPointerAttributes attr;
  if (dX && cudaPointerGetAttributes(&attr, dX) == cudaSuccess && attr.type == cudaMemoryTypeDevice)
    device = attr.device;
  int rc = create_common(device, n, d, out);
  if (rc) return rc;
  if (!dX) return fail(B2K_EINVAL, "X must not be NULL");
  auto* h = new b2k_index();
  h->ix.device = device;
  h->ix.n = n;
  h->ix.d = d;
  rc = build_from_device(h, dX, cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
  bool ok = true;
  if (!rc) rc = device_finite(h->ix.X, (size_t)n * d, h->ix.stream, &ok);
  if (!rc && !ok) rc = fail(B2K_ENONFINITE, "training coordinates must be finite");
  if (rc) {
    b2k_index_destroy(h);
    return rc;
  }
  *out = h;
  return B2K_OK;
}

int b2k_index_destroy(b2k_index* h) {
  if (!h) return B2K_OK;
  Index& ix = h->ix;
  cudaSetDevice(ix.device);
  if (ix.stream) cudaStreamSynchronize(ix.stream);
  cudaFree(ix.X);
  cudaFree(ix.nx32);
  cudaFree(ix.center);
  cudaFree(ix.colsum);
  cudaFree(ix.nx64);
  cudaFree(ix.stats_dev);
  cudaFree(ix.Xh);
  cudaFree(ix.pivots);
  cudaFree(ix.pivot_norms);
  cudaFree(ix.pivots_h);
  cudaFree(ix.Xaug);
  cudaFree(ix.aug_ones);
  cudaFree(ix.xperm);
  cudaFree(ix.xinv);
  cudaFree(ix.group_start);
  cudaFree(ix.Xt);
  cudaFree(ix.Xtaug);
  cudaFree(ix.taug_ones);
  cudaFree(ix.Xu);
  cudaFree(ix.nxu);
  if (ix.stream) cudaStreamDestroy(ix.stream);
  delete h;
  return B2K_OK;
}

int b2k_index_shape(const b2k_index* h, int64_t* n, int32_t* d) {
  if (!h) return fail(B2K_EINVAL, "index must not be NULL");
  if (n) *n = h->ix.n;
  if (d) *d = h->ix.d;
  return B2K_OK;
}

int b2k_index_download(const b2k_index* h, float* X) {
  if (!h || !X) return fail(B2K_EINVAL, "index and X must not be NULL");
  cudaSetDevice(h->ix.device);
  B2K_CUDA(cudaMemcpy(X, h->ix.X, (size_t)h->ix.n * h->ix.d * sizeof(float),
                      cudaMemcpyDeviceToHost));
  return B2K_OK;
}

const float* b2k_index_device_data(const b2k_index* h) { return h ? h->ix.X : nullptr; }

int b2k_knn_device(b2k_index* h, const float* dQ, int64_t m, int32_t k, int32_t exclude_self,
                   int64_t q_offset, int32_t mode, double* d_dist, int64_t* d_idx, void* stream,
                   b2k_stats* stats) {
  if (!h) return fail(B2K_EINVAL, "index must not be NULL");
  Index& ix = h->ix;
  int rc = validate_knn(ix, m, k, exclude_self, q_offset, mode);
  if (rc) return rc;
  if (m > 0 && (!dQ || !d_idx)) return fail(B2K_EINVAL, "queries and indices must not be NULL");
  if (overlaps(d_idx, (size_t)m * k * 8, dQ, (size_t)m * ix.d * 4) ||
      overlaps(d_dist, (size_t)m * k * 8, dQ, (size_t)m * ix.d * 4) ||
      overlaps(d_idx, (size_t)m * k * 8, d_dist, (size_t)m * k * 8))
    return fail(B2K_EINVAL, "output buffers must not overlap inputs or each other");
  return knn_device_impl(ix, dQ, m, k, exclude_self, q_offset, mode, d_dist, d_idx,
                         (cudaStream_t)stream, stats);
}

int b2k_knn(b2k_index* h, const float* Q, int64_t m, int32_t k, int32_t exclude_self,
            int64_t q_offset, int32_t mode, double* dist, int64_t* idx, b2k_stats* stats) {
  if (!h) return fail(B2K_EINVAL, "index must not be NULL");
  Index& ix = h->ix;
  int rc = validate_knn(ix, m, k, exclude_self, q_offset, mode);
  if (rc) return rc;
  if (m == 0) {
    if (stats) memset(stats, 0, sizeof(*stats));
    return B2K_OK;
  }
  if (!Q || !idx) return fail(B2K_EINVAL, "queries and indices must not be NULL");
  cudaSetDevice(ix.device);
  cudaStream_t st = ix.stream;
  float* dQ = nullptr;
  double* dd = nullptr;
  int64_t* di = nullptr;
  StreamFree fr{st, {}};
  if ((rc = dalloc(&dQ, (size_t)m * ix.d, st))) return rc;
  fr.keep(dQ);
  if ((rc = dalloc(&di, (size_t)m * k, st))) return rc;
  fr.keep(di);
  if (dist) {
    if ((rc = dalloc(&dd, (size_t)m * k, st))) return rc;
    fr.keep(dd);
  }
  B2K_CUDA(cudaMemcpyAsync(dQ, Q, (size_t)m * ix.d * sizeof(float), cudaMemcpyHostToDevice, st));
  // finiteness is checked on the device inside the search (one pass over HBM)
  rc = knn_device_impl(ix, dQ, m, k, exclude_self, q_offset, mode, dd, di, st, stats);
  if (rc) return rc;
  B2K_CUDA(cudaMemcpyAsync(idx, di, (size_t)m * k * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  if (dist)
    B2K_CUDA(cudaMemcpyAsync(dist, dd, (size_t)m * k * sizeof(double), cudaMemcpyDeviceToHost, st));
  B2K_CUDA(cudaStreamSynchronize(st));
  return B2K_OK;
}

}  // extern "C"

// =================================================================== radius
struct b2k_radius_result {
  int device = 0;
  int64_t m = 0, nnz = 0;
  int64_t* indptr = nullptr;   // device [m+1]
  int64_t* indices = nullptr;  // device [nnz]
  double* dist = nullptr;      // device [nnz] or null
  int64_t exact_tests = 0;
  int64_t candidates = 0;
};

namespace b2k {

// Entries per list of the single-pass radius screen: B2K_RADIUS_CAP when set
// (0 = the counted two-pass form), else what a 512 MB budget for the block's
// lists allows (B2K_RADIUS_LIST_MB), a multiple of 32 in [64, 1024], or 0 when
// that budget holds fewer than 64 per list.
static int radius_list_cap(int S_lists, int64_t m_pad) {
  if (const char* e = getenv("B2K_RADIUS_CAP")) {
    const long c = atol(e);
    return c <= 0 ? 0 : (int)std::min<long>(c, 1 << 20);
  }
  const char* mb = getenv("B2K_RADIUS_LIST_MB");
  const int64_t budget = (int64_t)(mb ? atoll(mb) : 512) << 20;
  int64_t c = budget / ((int64_t)S_lists * m_pad * (int64_t)sizeof(int)) / 32 * 32;
  return c < 64 ? 0 : (int)std::min<int64_t>(c, 1024);
}

// One block of queries: screen, classify, compact, sort.  The tcgen05 screen
// runs once into fixed-capacity lists; rows that overflow a list are answered
// by a counted sub-call (count pass, then fill at scanned offsets) on those
// rows alone, the form the CUDA-core screen always uses (`counted`).
// qrows: the block row of each query for self-exclusion (sub-calls), or null.
// Stores device CSR pieces in `res` (which then owns them).
static int radius_block(Index& ix, const float* dQ, int64_t m, double R2, int exclude_self,
                        int64_t q_offset, bool need_distance, bool sort_results, bool admit_all,
                        cudaStream_t st, b2k_radius_result* res, const int* qrows = nullptr,
                        bool counted = false, bool sort_rows = true) {
  StreamFree fr{st, {}};
  int rc;
  int mode = (!admit_all && ix.d >= 16 && ix.n >= 2048) ? B2K_MODE_BF16 : B2K_MODE_FP32;
  if (mode == B2K_MODE_BF16 && (rc = ensure_bf16(ix))) return rc;
  const bool tc = mode == B2K_MODE_BF16;
  const int64_t bm = tc ? kTcBM : kSimtBM;
  const int64_t m_pad = round_up(m, bm);
  const int64_t n_tiles = tc ? ix.n_pad_tc / kTcBN : (ix.n + kSimtBN - 1) / kSimtBN;
  const int sms = num_sms(ix.device);
  const int S = choose_splits(m_pad / bm, n_tiles, tc ? sms : 2 * sms);
  // candidate lists per row: one per (split, column group of the screen)
  const int S_lists = S * (tc ? tc_radius_groups() : simt_column_groups(kSinkRadiusCount));
  const int cap = (tc && !counted) ? radius_list_cap(S_lists, m_pad) : 0;

  int* status = nullptr;
  if ((rc = dalloc(&status, 8, st))) return rc;
  fr.keep(status);
  unsigned long long* counters = nullptr;
  if ((rc = dalloc(&counters, 2, st))) return rc;
  fr.keep(counters);
  B2K_CUDA(cudaMemsetAsync(status, 0, 8 * sizeof(int), st));
  B2K_CUDA(cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned long long), st));
  QueryPrep qp{};
  if ((rc = dalloc(&qp.E, (size_t)m_pad, st))) return rc;
  fr.keep(qp.E);
  if ((rc = dalloc(&qp.nq, (size_t)m_pad, st))) return rc;
  fr.keep(qp.nq);
  qp.flags = status + 4;
  if (tc) {
    if ((rc = dalloc(&qp.Ah, (size_t)m_pad * ix.dp, st))) return rc;
    fr.keep(qp.Ah);
  }
  launch_prep_queries(&ix, dQ, m, m_pad, mode, qp, st);
  float* thr = nullptr;
  if ((rc = dalloc(&thr, (size_t)m_pad, st))) return rc;
  fr.keep(thr);
  launch_radius_threshold(qp.nq, qp.E, m, m_pad, admit_all ? INFINITY : R2, thr, st);
  B2K_CUDA(cudaGetLastError());

  SinkArgs sa{};
  sa.thr = thr;
  sa.m_pad = (int)m_pad;
  sa.rcap = cap;
  if ((rc = dalloc(&sa.rcount, (size_t)S_lists * m_pad, st))) return rc;
  fr.keep(sa.rcount);
  int64_t* roff = nullptr;
  if ((rc = dalloc(&roff, (size_t)S_lists * m_pad + 1, st))) return rc;
  fr.keep(roff);
  sa.roff = roff;
  int* ovf = nullptr;  // single pass: overflowed rows [m] + their count
  if (cap) {
    if ((rc = dalloc(&sa.rcols, (size_t)S_lists * m_pad * cap, st))) return rc;
    fr.keep(sa.rcols);
    if ((rc = dalloc(&ovf, (size_t)m + 1, st))) return rc;
    fr.keep(ovf);
    B2K_CUDA(cudaMemsetAsync(ovf + m, 0, sizeof(int), st));
  }
  CUtensorMap tmap_a;
  if (tc && !tensor_map_2d_bf16(&tmap_a, qp.Ah, (uint64_t)ix.dp, (uint64_t)m_pad, kTcBK, kTcBM))
    return fail(B2K_ECUDA, "cuTensorMapEncodeTiled failed for the query rows");
  auto screen = [&](int kind) -> int {
    if (tc) {
      int lr = launch_screen_tc(&ix, &tmap_a, m, m_pad, exclude_self, q_offset, S, qp.E, kind,
                                sa, status, st, qrows);
      if (lr) return fail(B2K_ECUDA, "tcgen05 screen launch failed: %s",
                          cudaGetErrorString((cudaError_t)lr));
      return B2K_OK;
    }
    launch_screen_simt(&ix, dQ, m, m_pad, exclude_self, q_offset, S, qp.E, kind, sa, st, qrows);
    B2K_CUDA(cudaGetLastError());
    return B2K_OK;
  };
  if ((rc = screen(cap ? kSinkRadiusList : kSinkRadiusCount))) return rc;
  if (cap) launch_radius_overflow(sa.rcount, S_lists, m, m_pad, cap, ovf, st);
  int64_t* scan_scratch = nullptr;  // multi-block scans (count offsets, then indptr)
  if ((rc = dalloc(&scan_scratch, (size_t)scan_scratch_len(m), st))) return rc;
  fr.keep(scan_scratch);
  launch_scan_split_counts(sa.rcount, S_lists, m, m_pad, roff, roff + (size_t)S_lists * m_pad,
                           scan_scratch, st);
  int64_t ncand = 0;
  int hstatus[8];
  int n_ovf = 0;
  B2K_CUDA(cudaMemcpyAsync(&ncand, roff + (size_t)S_lists * m_pad, sizeof(int64_t),
                           cudaMemcpyDeviceToHost, st));
  B2K_CUDA(cudaMemcpyAsync(hstatus, status, sizeof(hstatus), cudaMemcpyDeviceToHost, st));
  if (cap) B2K_CUDA(cudaMemcpyAsync(&n_ovf, ovf + m, sizeof(int), cudaMemcpyDeviceToHost, st));
  B2K_CUDA(cudaStreamSynchronize(st));
  if (hstatus[0] != DEV_OK)
    return fail(B2K_ETIMEOUT, "a bounded device wait gave up (code %d)", hstatus[0]);
  if ((hstatus[4] & 1) && !admit_all)
    return radius_block(ix, dQ, m, R2, exclude_self, q_offset, need_distance, sort_results, true,
                        st, res, qrows, counted, sort_rows);
  // the candidates in one array at their scanned offsets, as training rows
  // (grouped operand rows are mapped); rows are re-sorted by index after the
  // compaction when their lists are out of index order (grouped rows, or
  // several lists per row, whose columns interleave)
  const bool grouped = tc && ix.xperm;
  int* cand = nullptr;
  if ((rc = dalloc(&cand, (size_t)ncand, st))) return rc;
  fr.keep(cand);
  if (cap) {
    launch_radius_pack(sa.rcols, cap, sa.rcount, S_lists, m, m_pad, roff,
                       grouped ? ix.xperm : nullptr, cand, ncand, status, st);
  } else {
    sa.rcols = cand;
    if ((rc = screen(kSinkRadiusFill))) return rc;
    if (grouped)
      launch_radius_pack(cand, 0, sa.rcount, S_lists, m, m_pad, roff, ix.xperm, cand, ncand,
                         status, st);
  }
  const bool unordered = grouped || S_lists > S;
  const bool keep_dist = need_distance || sort_results;

  RadiusPlanArgs ra{};
  ra.X = ix.X;
  ra.Q = dQ;
  ra.d = ix.d;
  ra.m = m;
  ra.m_pad = m_pad;
  ra.S = S_lists;
  ra.roff = roff;
  ra.rcount = sa.rcount;
  ra.cols = cand;
  // long rows (an overflow sub-call's) take a CTA each in classify and compact
  ra.wide = ncand >= (int64_t)kWideRowCandidates * m;
  ra.R2 = R2;
  ra.exact_tests = counters;
  ra.status = status;
  if ((rc = dalloc(&ra.cdist, (size_t)ncand, st))) return rc;
  fr.keep(ra.cdist);
  if ((rc = dalloc(&ra.mcount, (size_t)m, st))) return rc;
  fr.keep(ra.mcount);
  launch_classify(ra, st);

  // rows that overflowed their lists: the counted form over those rows alone
  // (their own block; self-exclusion through their block rows)
  b2k_radius_result* sub = nullptr;
  struct SubFree {
    b2k_radius_result*& r;
    ~SubFree() {
      if (r) b2k_radius_result_release(r);
    }
  } sub_free{sub};
  if (n_ovf > 0) {
    float* Qo = nullptr;
    int* orow = nullptr;
    if ((rc = dalloc(&Qo, (size_t)n_ovf * ix.d, st))) return rc;
    fr.keep(Qo);
    if ((rc = dalloc(&orow, (size_t)n_ovf, st))) return rc;
    fr.keep(orow);
    // sub-call row i answers block row ovf[i] (any order: the scatter places it)
    launch_gather_fallback(dQ, ix.d, ovf, qrows, n_ovf, Qo, orow, st);
    B2K_CUDA(cudaGetLastError());
    sub = new b2k_radius_result();
    sub->device = ix.device;
    if ((rc = radius_block(ix, Qo, n_ovf, R2, exclude_self, q_offset, keep_dist, false, admit_all,
                           st, sub, orow, true, false)))
      return rc;
    launch_radius_sub_counts(ovf, n_ovf, sub->indptr, ra.mcount, st);
  }

  int64_t* indptr = nullptr;
  if ((rc = dalloc(&indptr, (size_t)m + 1, st))) return rc;
  launch_scan_rows(ra.mcount, m, indptr, scan_scratch, st);
  B2K_CUDA(cudaGetLastError());
  int64_t nnz = 0;
  unsigned long long hc[2];
  B2K_CUDA(cudaMemcpyAsync(&nnz, indptr + m, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  B2K_CUDA(cudaMemcpyAsync(hc, counters, sizeof(hc), cudaMemcpyDeviceToHost, st));
  B2K_CUDA(cudaMemcpyAsync(hstatus, status, sizeof(hstatus), cudaMemcpyDeviceToHost, st));
  B2K_CUDA(cudaStreamSynchronize(st));
  if (hstatus[0] != DEV_OK) {  // the fill pass gave up (classify skipped its rows)
    cudaFreeAsync(indptr, st);
    return fail(B2K_ETIMEOUT, "a bounded device wait gave up (code %d)", hstatus[0]);
  }
  int64_t* indices = nullptr;
  double* dist = nullptr;
  if ((rc = dalloc(&indices, (size_t)nnz, st))) {
    cudaFreeAsync(indptr, st);
    return rc;
  }
  if (keep_dist && (rc = dalloc(&dist, (size_t)nnz, st))) {
    cudaFreeAsync(indptr, st);
    cudaFreeAsync(indices, st);
    return rc;
  }
  launch_compact(ra, indptr, indices, dist, st);
  if (sub)
    launch_radius_sub_scatter(ovf, n_ovf, sub->indptr, sub->indices, sub->dist, indptr, indices,
                              dist, st);
  B2K_CUDA(cudaGetLastError());
  if (sort_rows && (sort_results || unordered) && nnz > 1) {
    // (distance, index) order when asked for, else ascending training index
    // (grouped operand rows list candidates out of index order)
    const bool by_dist = sort_results;
    // row lists for the longer rows: [m] rows + count, twice
    int* lists = nullptr;
    if ((rc = dalloc(&lists, 2 * (size_t)m + 2, st))) return rc;
    fr.keep(lists);
    int* mid = lists;
    int* big = lists + m + 1;
    B2K_CUDA(cudaMemsetAsync(mid + m, 0, sizeof(int), st));
    B2K_CUDA(cudaMemsetAsync(big + m, 0, sizeof(int), st));
    launch_sort_rows(indptr, m, indices, dist, mid, mid + m, big, big + m,
                     (int)std::min<int64_t>(m, 4 * sms), st, by_dist);
    int nbig = 0;
    B2K_CUDA(cudaMemcpyAsync(&nbig, big + m, sizeof(int), cudaMemcpyDeviceToHost, st));
    B2K_CUDA(cudaStreamSynchronize(st));
    if (nbig > 0) {
      // scratch sized for the longest row (<= n), one slot per CTA
      int64_t P = 2;
      while (P < ix.n) P <<= 1;
      const int grid = std::min(nbig, 16);
      double* td = nullptr;
      int64_t* ti = nullptr;
      if ((rc = dalloc(&td, (size_t)grid * P, st))) return rc;
      fr.keep(td);
      if ((rc = dalloc(&ti, (size_t)grid * P, st))) return rc;
      fr.keep(ti);
      launch_sort_big_rows(indptr, big, nbig, indices, dist, td, ti, P, grid, st, by_dist);
      B2K_CUDA(cudaGetLastError());
    }
  }
  B2K_CUDA(cudaStreamSynchronize(st));
  if (!need_distance && dist) {
    cudaFree(dist);
    dist = nullptr;
  }
  res->m = m;
  res->nnz = nnz;
  res->indptr = indptr;
  res->indices = indices;
  res->dist = dist;
  res->exact_tests = (int64_t)hc[0] + (sub ? sub->exact_tests : 0);
  res->candidates = ncand + (sub ? sub->candidates : 0);
  return B2K_OK;
}

}  // namespace b2k

extern "C" {

int b2k_radius(b2k_index* h, const float* Q, int64_t m, double radius, int32_t exclude_self,
               int64_t q_offset, int32_t need_distance, int32_t sort_results,
               b2k_radius_result** out) {
  if (!h || !out) return fail(B2K_EINVAL, "index and out must not be NULL");
  *out = nullptr;
  Index& ix = h->ix;
  if (std::isnan(radius)) return fail(B2K_EINVAL, "radius must not be NaN");
  if (radius < 0) return fail(B2K_EINVAL, "radius must be non-negative, got %g", radius);
  if (m < 0 || m >= ((int64_t)1 << 31)) return fail(B2K_EINVAL, "invalid query count");
  if (exclude_self && (q_offset < 0 || q_offset + m > ix.n))
    return fail(B2K_EINVAL,
                "exclude_self requires the query matrix to be the training matrix: got %lld "
                "query rows at offset %lld and %lld training rows.",
                (long long)m, (long long)q_offset, (long long)ix.n);
  if (m > 0 && !Q) return fail(B2K_EINVAL, "queries must not be NULL");
  if (fault_mode() == 2) return fail(B2K_ECUDA, "injected kernel launch failure (B2K_FAULT=launch)");
  const double R2 = radius * radius;
  cudaSetDevice(ix.device);
  cudaStream_t st = ix.stream;
  auto* res = new b2k_radius_result();
  res->device = ix.device;
  if (m == 0) {
    res->m = 0;
    if (cudaMalloc(&res->indptr, sizeof(int64_t)) != cudaSuccess ||
        cudaMemset(res->indptr, 0, sizeof(int64_t)) != cudaSuccess) {
      b2k_radius_result_release(res);
      return fail(B2K_ENOMEM, "allocation failed");
    }
    *out = res;
    return B2K_OK;
  }
  float* dQ = nullptr;
  int rc = dalloc(&dQ, (size_t)m * ix.d, st);
  if (rc) {
    delete res;
    return rc;
  }
  cudaMemcpyAsync(dQ, Q, (size_t)m * ix.d * sizeof(float), cudaMemcpyHostToDevice, st);
  bool finite = true;
  rc = device_finite(dQ, (size_t)m * ix.d, st, &finite);
  if (!rc && !finite) rc = fail(B2K_ENONFINITE, "training and query coordinates must be finite");
  if (rc) {
    cudaFreeAsync(dQ, st);
    delete res;
    return rc;
  }
  rc = radius_block(ix, dQ, m, R2, exclude_self, q_offset, need_distance != 0,
                    sort_results != 0, !ix.range_ok, st, res);
  cudaFreeAsync(dQ, st);
  cudaStreamSynchronize(st);
  if (rc) {
    b2k_radius_result_release(res);
    return rc;
  }
  *out = res;
  return B2K_OK;
}

int b2k_radius_result_nnz(const b2k_radius_result* res, int64_t* nnz) {
  if (!res || !nnz) return fail(B2K_EINVAL, "result and nnz must not be NULL");
  *nnz = res->nnz;
  return B2K_OK;
}

int b2k_radius_result_fetch(const b2k_radius_result* res, int64_t* indptr, int64_t* indices,
                            double* dist) {
  if (!res || !indptr) return fail(B2K_EINVAL, "result and indptr must not be NULL");
  if (res->nnz && !indices) return fail(B2K_EINVAL, "indices must not be NULL");
  if (dist && res->nnz && !res->dist)
    return fail(B2K_EINVAL, "distances were not requested for this result");
  cudaSetDevice(res->device);
  B2K_CUDA(cudaMemcpy(indptr, res->indptr, (size_t)(res->m + 1) * sizeof(int64_t),
                      cudaMemcpyDeviceToHost));
  if (res->nnz) {
    B2K_CUDA(cudaMemcpy(indices, res->indices, (size_t)res->nnz * sizeof(int64_t),
                        cudaMemcpyDeviceToHost));
    if (dist)
      B2K_CUDA(cudaMemcpy(dist, res->dist, (size_t)res->nnz * sizeof(double),
                          cudaMemcpyDeviceToHost));
  }
  return B2K_OK;
}

int b2k_knn_backward(const float* dQ, int64_t m, const float* dX, int64_t n, int32_t d,
                     int32_t k, const int64_t* d_idx, const float* d_grad, const float* d_dist,
                     int32_t squared, float* d_grad_q, float* d_grad_x, void* stream) {
  if (m < 0 || n <= 0 || d <= 0 || k <= 0) return fail(B2K_EINVAL, "invalid backward shapes");
  if (m > 0 && (!dQ || !dX || !d_idx || !d_grad))
    return fail(B2K_EINVAL, "backward inputs must not be NULL");
  if (!squared && !d_dist)
    return fail(B2K_EINVAL, "the euclidean backward needs the forward distances");
  if (fault_mode() == 2) return fail(B2K_ECUDA, "injected kernel launch failure (B2K_FAULT=launch)");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int* ws = nullptr;
  int rc = 0;
  if (d_grad_x) {
    if ((rc = dalloc(&ws, knn_backward_workspace_ints(m, n, k), st))) return rc;
  }
  const int e = knn_backward(dQ, m, dX, n, d, k, d_idx, d_grad, squared ? nullptr : d_dist,
                             squared, d_grad_q, d_grad_x, ws, st);
  if (ws) cudaFreeAsync(ws, st);
  if (e) return fail(B2K_ECUDA, "backward launch failed: %s", cudaGetErrorString((cudaError_t)e));
  return B2K_OK;
}

int b2k_class_votes(const int64_t* d_idx, const double* d_dist, int64_t m, int32_t k,
                    const int32_t* d_codes, int32_t n_classes, int32_t weighted,
                    double* d_votes, int64_t* d_pred, void* stream) {
  if (m < 0 || k <= 0 || n_classes <= 0) return fail(B2K_EINVAL, "invalid vote shapes");
  if (m > 0 && (!d_idx || !d_codes || !d_votes)) return fail(B2K_EINVAL, "NULL vote buffer");
  if (weighted && !d_dist) return fail(B2K_EINVAL, "distance weights need distances");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int* status = nullptr;
  int rc = dalloc(&status, 1, st);
  if (rc) return rc;
  B2K_CUDA(cudaMemsetAsync(status, 0, sizeof(int), st));
  launch_votes(d_idx, d_dist, m, k, d_codes, n_classes, weighted, d_votes, d_pred, status, st);
  int h = 0;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(status, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(B2K_ECUDA, "votes failed: %s", cudaGetErrorString(e));
  if (h) return fail(B2K_EINVAL, "All neighbors of some sample are getting zero weights.");
  return B2K_OK;
}

// -------------------------------------------------------------- row shards
// Relative bound on |canonical distance - exact distance|: the canonical
// squared value is within g = (d+2)u/(1-(d+2)u) of the exact one (u = 2^-53),
// its square root adds half of that plus one rounding; 2g + 4u is generous.
static double shard_eps(int d) {
  const double u = 0x1p-53;
  const double g = (d + 2) * u / (1.0 - (d + 2) * u);
  return 2 * g + 4 * u;
}

static int check_shard_shapes(int32_t n_shards, int64_t m, int32_t k_in, int32_t k) {
  if (n_shards < 1 || n_shards > kMaxShards)
    return fail(B2K_EINVAL, "shard count must be in [1, %d], got %d", kMaxShards, n_shards);
  if (m < 0) return fail(B2K_EINVAL, "query count must be non-negative");
  if (k < 1 || k > kMaxShardK || k_in < k || k_in > kMaxShardK + 1)
    return fail(B2K_EINVAL,
                "shard merge needs 1 <= k <= %d and k <= k_in <= k + 1, got k=%d k_in=%d",
                kMaxShardK, k, k_in);
  return B2K_OK;
}

int b2k_shard_merge(const double* d_dist, const int64_t* d_idx, int32_t n_shards, int64_t m,
                    int32_t k_in, int32_t k, int32_t d, int64_t self_offset, double* d_out_dist,
                    int64_t* d_out_idx, int32_t* d_flags, void* stream) {
  int rc = check_shard_shapes(n_shards, m, k_in, k);
  if (rc) return rc;
  if (d < 1) return fail(B2K_EINVAL, "feature count must be positive");
  if (m == 0) return B2K_OK;
  if (!d_dist || !d_idx || !d_out_dist || !d_out_idx || !d_flags)
    return fail(B2K_EINVAL, "device pointers must not be NULL");
  launch_shard_merge(d_dist, d_idx, n_shards, m, k_in, k, self_offset, shard_eps(d), d_out_dist,
                     d_out_idx, d_flags, static_cast<cudaStream_t>(stream));
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return fail(B2K_ECUDA, "shard merge launch failed: %s", cudaGetErrorString(e));
  return B2K_OK;
}

int b2k_shard_keys(b2k_index* h, int64_t row_lo, const float* dQ, const int64_t* d_idx,
                   int32_t n_shards, int64_t m, int32_t k_in, const int64_t* d_flagged,
                   int64_t n_flagged, uint64_t* d_keys, void* stream) {
  if (!h) return fail(B2K_EINVAL, "index must not be NULL");
  int rc = check_shard_shapes(n_shards, m, k_in, k_in > 1 ? k_in - 1 : 1);
  if (rc) return rc;
  if (row_lo < 0) return fail(B2K_EINVAL, "row offset must be non-negative");
  if (n_flagged < 0 || n_flagged > m) return fail(B2K_EINVAL, "invalid flagged query count");
  if (n_flagged == 0) return B2K_OK;
  if (!dQ || !d_idx || !d_flagged || !d_keys)
    return fail(B2K_EINVAL, "device pointers must not be NULL");
  Index& ix = h->ix;
  B2K_CUDA(cudaSetDevice(ix.device));
  launch_shard_keys(nullptr, d_idx, n_shards, m, k_in, dQ, ix.X, ix.n, ix.d, row_lo, d_flagged,
                    n_flagged, d_keys, static_cast<cudaStream_t>(stream));
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return fail(B2K_ECUDA, "shard keys launch failed: %s", cudaGetErrorString(e));
  return B2K_OK;
}

int b2k_shard_resolve(const double* d_dist, const int64_t* d_idx, int32_t n_shards, int64_t m,
                      int32_t k_in, int32_t k, int64_t self_offset, const int64_t* d_flagged,
                      int64_t n_flagged, const uint64_t* d_keys, double* d_out_dist,
                      int64_t* d_out_idx, void* stream) {
  int rc = check_shard_shapes(n_shards, m, k_in, k);
  if (rc) return rc;
  if (n_flagged < 0 || n_flagged > m) return fail(B2K_EINVAL, "invalid flagged query count");
  if (n_flagged == 0) return B2K_OK;
  if (!d_dist || !d_idx || !d_flagged || !d_keys || !d_out_dist || !d_out_idx)
    return fail(B2K_EINVAL, "device pointers must not be NULL");
  launch_shard_resolve(d_dist, d_idx, n_shards, m, k_in, k, self_offset, d_flagged, n_flagged,
                       d_keys, d_out_dist, d_out_idx, static_cast<cudaStream_t>(stream));
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return fail(B2K_ECUDA, "shard resolve launch failed: %s", cudaGetErrorString(e));
  return B2K_OK;
}

int b2k_radius_result_class_votes(const b2k_radius_result* res, const int32_t* d_codes,
                                  int32_t n_classes, int32_t weighted, double* d_votes,
                                  int64_t* d_counts, void* stream) {
  if (!res) return fail(B2K_EINVAL, "result must not be NULL");
  if (n_classes <= 0) return fail(B2K_EINVAL, "n_classes must be positive");
  if (res->m > 0 && (!d_codes || !d_votes || !d_counts))
    return fail(B2K_EINVAL, "device pointers must not be NULL");
  if (weighted && res->m > 0 && res->nnz > 0 && !res->dist)
    return fail(B2K_EINVAL, "distance weights need a result with distances");
  if (res->m == 0) return B2K_OK;
  B2K_CUDA(cudaSetDevice(res->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  launch_radius_votes(res->indptr, res->indices, res->dist, res->m, d_codes, n_classes,
                      weighted, d_votes, d_counts, st);
  B2K_CUDA(cudaGetLastError());
  B2K_CUDA(cudaStreamSynchronize(st));
  return B2K_OK;
}

int b2k_radius_result_class_predict(const b2k_radius_result* res, const int32_t* d_codes,
                                    int32_t n_classes, int64_t* d_pred, int64_t* d_counts,
                                    void* stream) {
  if (!res) return fail(B2K_EINVAL, "result must not be NULL");
  if (n_classes <= 0) return fail(B2K_EINVAL, "n_classes must be positive");
  if (res->m > 0 && (!d_codes || !d_pred || !d_counts))
    return fail(B2K_EINVAL, "device pointers must not be NULL");
  if (res->m == 0) return B2K_OK;
  B2K_CUDA(cudaSetDevice(res->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  launch_radius_votes(res->indptr, res->indices, res->dist, res->m, d_codes, n_classes,
                      /*weighted=*/0, /*votes=*/nullptr, d_counts, st, d_pred);
  B2K_CUDA(cudaGetLastError());
  B2K_CUDA(cudaStreamSynchronize(st));
  return B2K_OK;
}

int b2k_radius_result_means(const b2k_radius_result* res, const double* d_targets,
                            int32_t weighted, double* d_means, int64_t* d_counts,
                            void* stream) {
  if (!res) return fail(B2K_EINVAL, "result must not be NULL");
  if (res->m > 0 && (!d_targets || !d_means || !d_counts))
    return fail(B2K_EINVAL, "device pointers must not be NULL");
  if (weighted && res->m > 0 && res->nnz > 0 && !res->dist)
    return fail(B2K_EINVAL, "distance weights need a result with distances");
  if (res->m == 0) return B2K_OK;
  B2K_CUDA(cudaSetDevice(res->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  launch_radius_means(res->indptr, res->indices, res->dist, res->m, d_targets, weighted,
                      d_means, d_counts, st);
  B2K_CUDA(cudaGetLastError());
  B2K_CUDA(cudaStreamSynchronize(st));
  return B2K_OK;
}

int b2k_radius_result_release(b2k_radius_result* res) {
  if (!res) return B2K_OK;
  cudaSetDevice(res->device);
  cudaFree(res->indptr);
  cudaFree(res->indices);
  cudaFree(res->dist);
  delete res;
  return B2K_OK;
}

}  // extern "C"
