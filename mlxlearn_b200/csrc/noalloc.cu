// kNN entry point that allocates no memory: b2k_knn_device_noalloc.
//
// Who needs it: callers that must not allocate device memory during a query.
// Examples are serving processes whose whole GPU memory budget is owned by
// another allocator (a framework's caching allocator, a pre-reserved arena),
// and latency-critical paths where cudaMalloc/cudaFree, which can synchronise
// the device, are not allowed.  The regular entry points take their scratch
// from the stream-ordered pool; this one takes it from a fixed array that
// lives in the library's device image.
//
// The scratch is a file-scope __device__ array of kNoAllocScratchBytes
// (32 MiB).  Every GPU that loads the library keeps that much device memory
// reserved until the process exits.  In host code the array's name is only a
// host-side stand-in, never a device address: the device address is obtained
// once per device with cudaGetSymbolAddress, with that device current, on the
// first call made on that device.  Make that first call before any stream
// capture begins.
//
// All calls share the one array and it keeps the previous call's contents;
// everything that must start at zero is cleared on the caller's stream at the
// start of each call.  Calls whose GPU work overlaps (different streams, or
// several host threads without ordering) race on the array and must not be
// issued.
//
// The search is the plain fp32 screen (one reference split) followed by the
// certified float64 re-rank and exact tie resolution, so the answer is the
// same as b2k_knn_device's.  Rows the screen cannot certify, inputs outside
// the screen's safe coordinate range, and k > 64 use the exhaustive exact scan
// in its scratch-free form.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "internal.cuh"
#include "sinks.cuh"

namespace b2k {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

std::mutex g_scratch_mu;
void* g_scratch_dev[64] = {nullptr};

// Device address of the scratch array on `device` (the current device).
int scratch_address(int device, unsigned char** out) {
  if (device < 0 || device >= 64) return report_error(B2K_EINVAL, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_dev[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return report_error(B2K_ECUDA, "cudaGetSymbolAddress of the no-alloc scratch failed");
    g_scratch_dev[device] = p;
  }
  *out = static_cast<unsigned char*>(g_scratch_dev[device]);
  return B2K_OK;
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Bytes of scratch one call needs for m queries and k neighbours.  The
// exhaustive scan alone (unscreened calls) needs only the status and counter
// blocks.
size_t scratch_bytes(int64_t m, int k, bool screened) {
  const size_t m_pad = (size_t)((m + kSimtBM - 1) / kSimtBM) * kSimtBM;
  size_t b = 256 /*status*/ + 256 /*counters*/;
  if (!screened) return b;
  b += align256(m_pad * sizeof(float));                       // E
  b += align256(m_pad * sizeof(int));                         // counts
  b += align256(m_pad * (size_t)k * sizeof(float));           // kth
  b += align256((size_t)m * sizeof(int));                     // fallback rows
  b += align256(m_pad * (size_t)kListCap * sizeof(int2));     // candidate lists
  return b;
}

}  // namespace

}  // namespace b2k

using namespace b2k;

extern "C" B2K_API int b2k_knn_device_noalloc(b2k_index* h, const float* dQ, int64_t m,
                                              int32_t k, int32_t exclude_self, int64_t q_offset,
                                              double* d_dist, int64_t* d_idx, void* stream) {
  Index* ixp = index_of(h);
  if (!ixp) return report_error(B2K_EINVAL, "index must not be NULL");
  Index& ix = *ixp;
  int rc = check_knn_args(ix, m, k, exclude_self, q_offset);
  if (rc) return rc;
  if (m == 0) return B2K_OK;
  if (!dQ || !d_idx) return report_error(B2K_EINVAL, "queries and indices must not be NULL");
  if (buffers_overlap(dQ, m, ix.d, k, d_dist, d_idx))
    return report_error(B2K_EINVAL, "output buffers must not overlap inputs or each other");
  // the screen runs for in-range indexes and k <= 64; otherwise the
  // exhaustive scan alone, which needs only the status block
  const bool screened = ix.range_ok && k <= kMaxK;
  const size_t need = scratch_bytes(m, k, screened);
  if (need > kNoAllocScratchBytes) {
    // largest batch that fits, for the message
    int64_t lo = 0, hi = m;
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) / 2;
      if (scratch_bytes(mid, k, screened) <= kNoAllocScratchBytes) lo = mid;
      else hi = mid - 1;
    }
    char msg[256];
    snprintf(msg, sizeof(msg),
             "b2k_knn_device_noalloc: %lld queries need %zu bytes of scratch, more than the "
             "fixed %zu bytes; at most %lld queries per call for k=%d",
             (long long)m, need, kNoAllocScratchBytes, (long long)lo, (int)k);
    return report_error(B2K_EINVAL, msg);
  }
  cudaError_t e = cudaSetDevice(ix.device);
  if (e != cudaSuccess) return report_error(B2K_ECUDA, "cudaSetDevice failed");
  unsigned char* base = nullptr;
  if ((rc = scratch_address(ix.device, &base))) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  // carve the scratch
  const int64_t m_pad = (m + kSimtBM - 1) / kSimtBM * kSimtBM;
  unsigned char* p = base;
  int* status = reinterpret_cast<int*>(p);
  p += 256;
  unsigned long long* counters = reinterpret_cast<unsigned long long*>(p);
  p += 256;
  float* E = reinterpret_cast<float*>(p);
  p += align256((size_t)m_pad * sizeof(float));
  int* counts = reinterpret_cast<int*>(p);
  p += align256((size_t)m_pad * sizeof(int));
  float* kth = reinterpret_cast<float*>(p);
  p += align256((size_t)m_pad * k * sizeof(float));
  int* fb_list = reinterpret_cast<int*>(p);
  p += align256((size_t)m * sizeof(int));
  int2* lists = reinterpret_cast<int2*>(p);

  // zero what must start at zero (the array keeps the previous call's data)
  if (cudaMemsetAsync(status, 0, 256, st) != cudaSuccess ||
      cudaMemsetAsync(counters, 0, 256, st) != cudaSuccess)
    return report_error(B2K_ECUDA, "cudaMemsetAsync on the no-alloc scratch failed");
  // NaN / inf queries: flagged on the device (status[5]) and reported after
  // the search, which stays bounded on such inputs, as in b2k_knn_device
  launch_nonfinite_check(dQ, m * (int64_t)ix.d, status + 5, st);

  if (screened) {
    QueryPrep qp{};
    qp.E = E;
    qp.flags = status + 4;
    launch_prep_queries(&ix, dQ, m, m_pad, B2K_MODE_FP32, qp, st);
    ScreenOut so{};
    so.lists = lists;
    so.counts = counts;
    so.kth = kth;
    so.cap = kListCap;
    so.m_pad = (int)m_pad;
    SinkArgs sa{};
    sa.out = so;
    sa.k = k;
    launch_screen_simt(&ix, dQ, m, m_pad, exclude_self, q_offset, 1, E, kSinkKnn, sa, st,
                       nullptr, /*noalloc=*/true);
    CertifyArgs ca{};
    ca.X = ix.X;
    ca.Q = dQ;
    ca.n = ix.n;
    ca.m = m;
    ca.d = ix.d;
    ca.k = k;
    ca.S = 1;
    ca.scr = so;
    ca.E = E;
    ca.dist = d_dist;
    ca.idx = d_idx;
    ca.fallback_list = fb_list;
    ca.fallback_count = status + 2;
    ca.counters = counters;
    ca.status = status;
    launch_certify(ca, st);
  }
  ExactArgs ea{};
  ea.X = ix.X;
  ea.Q = dQ;
  ea.n = ix.n;
  ea.m = m;
  ea.d = ix.d;
  ea.k = k;
  ea.exclude_self = exclude_self;
  ea.q_offset = q_offset;
  ea.rows = screened ? fb_list : nullptr;
  ea.row_count = screened ? status + 2 : nullptr;
  ea.scratch = nullptr;  // recompute form: no scratch
  ea.dist = d_dist;
  ea.idx = d_idx;
  ea.counters = counters;
  ea.status = status;
  const int sms = num_sms(ix.device);
  ea.grid = (int)(screened ? 2 * sms : (m < 2 * sms ? m : 2 * sms));
  launch_exact(ea, st);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return report_error(B2K_ECUDA, cudaGetErrorString(e));
  int hstatus[8];
  if (cudaMemcpyAsync(hstatus, status, sizeof(hstatus), cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return report_error(B2K_ECUDA, "reading the device status failed");
  if (hstatus[5]) return report_error(B2K_ENONFINITE, "training and query coordinates must be finite");
  if (hstatus[0] == DEV_TOO_MANY_TIES)
    return report_error(B2K_EUNSUPPORTED,
                        "too many training rows tie with a query's k-th neighbour");
  if (hstatus[0] != DEV_OK) return report_error(B2K_ETIMEOUT, "a bounded device wait gave up");
  if (screened && (hstatus[4] & 1)) {
    // a query coordinate is outside the screen's safe range: exhaustive exact scan
    if (cudaMemsetAsync(status, 0, 256, st) != cudaSuccess)
      return report_error(B2K_ECUDA, "cudaMemsetAsync on the no-alloc scratch failed");
    ea.rows = nullptr;
    ea.row_count = nullptr;
    ea.grid = (int)(m < 2 * sms ? m : 2 * sms);
    launch_exact(ea, st);
    if (cudaMemcpyAsync(hstatus, status, sizeof(hstatus), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return report_error(B2K_ECUDA, "reading the device status failed");
    if (hstatus[0] != DEV_OK) return report_error(B2K_ETIMEOUT, "a bounded device wait gave up");
  }
  return B2K_OK;
}
