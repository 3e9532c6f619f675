// Shared device/host helpers for the B200 neighbour-search library.
//
// PTX wrappers for mbarriers, TMA bulk-tensor loads and the tcgen05 (5th
// generation tensor core) instructions used by the screen kernels, plus
// bounded spin-waits: every wait gives up after a fixed number of polls,
// records an error code in device memory and lets the kernel return, so a
// logic error can never hang the GPU.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define B2K_DEV __device__ __forceinline__

namespace b2k {

// Error codes written by kernels into the per-call status word.
enum DevError : int {
  DEV_OK = 0,
  DEV_TIMEOUT_FULL = 1,    // consumer waited too long for a TMA stage
  DEV_TIMEOUT_EMPTY = 2,   // producer waited too long for a free stage
  DEV_TIMEOUT_ACC = 3,     // MMA / epilogue accumulator hand-off timed out
  DEV_TIMEOUT_A = 4,       // query tile hand-off timed out
  DEV_TOO_MANY_TIES = 5,   // exact fallback candidate buffer overflowed
  DEV_TIMEOUT_DRAIN = 6,   // the exit path's wait for the CTA's own async work gave up
};

// ~2^26 polls of try_wait (each poll may itself suspend for a short time):
// several seconds, far beyond any legitimate wait in these kernels.  Kernels
// take their limit as a parameter (default this); drain waits on the exit
// path always use it.
constexpr uint32_t kSpinLimit = 1u << 26;

B2K_DEV uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ------------------------------------------------------------------ mbarrier
B2K_DEV void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
B2K_DEV void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
B2K_DEV void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
B2K_DEV void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(
                   smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
B2K_DEV bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase with the given parity to complete.  Returns false
// (after recording `code` in *status) after `limit` polls, or when another
// role of this kernel already reported an error.
B2K_DEV bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* status, int code,
                       uint32_t limit = kSpinLimit) {
  for (uint32_t i = 0; i < limit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 1023u) == 1023u && *status != DEV_OK) return false;
  }
  atomicCAS(const_cast<int*>(status), DEV_OK, code);
  return false;
}
// Exit-path wait for this CTA's own asynchronous work (a bulk copy or the
// tensor-core operations it issued): those complete by themselves, so it
// ignores other roles' errors and uses the full limit.
B2K_DEV bool mbar_wait_drain(uint64_t* bar, uint32_t parity, volatile int* status) {
  for (uint32_t i = 0; i < kSpinLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  atomicCAS(const_cast<int*>(status), DEV_OK, DEV_TIMEOUT_DRAIN);
  return false;
}

// ----------------------------------------------------------------------- TMA
B2K_DEV void tma_load_2d(void* smem_dst, const void* tmap, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}
B2K_DEV void prefetch_tmap(const void* tmap) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tmap)) : "memory");
}

// ------------------------------------------------------------------- tcgen05
B2K_DEV void tmem_alloc(uint32_t* smem_slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(smem_slot)),
               "r"(ncols)
               : "memory");
}
B2K_DEV void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
B2K_DEV void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
B2K_DEV void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
B2K_DEV void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// D[tmem] (+)= A[smem] * B[smem]^T, kind::f16 (bf16 or f16 operands, f32 accum).
B2K_DEV void mma_f16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                     uint32_t accumulate) {
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "setp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n"
      "}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// D[tmem] (+)= A[smem] * B[smem]^T, kind::tf32 (fp32 operands read as tf32,
// f32 accumulation; the operands here are already rounded to tf32).
B2K_DEV void mma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                      uint32_t accumulate) {
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "setp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n"
      "}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// D[tmem] (+)= A[smem] * B[smem]^T, kind::i8 (8-bit integer operands, s32
// accumulation: every product and sum is exact while it fits 32 bits).
B2K_DEV void mma_i8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                    uint32_t accumulate) {
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "setp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n"
      "}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// Arrive on `bar` when all previously issued tcgen05.mma of this thread complete.
B2K_DEV void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}
// 32 lanes x 32 consecutive 32-bit columns: thread t of the warp gets lane
// (base_lane + t), columns [col, col+32).
B2K_DEV void tmem_ld_32x32b_x32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(taddr));
}
B2K_DEV void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
// Wait for outstanding TMEM loads; the registers are in/out operands so no use
// of them can be scheduled before the wait.
B2K_DEV void tmem_ld_wait_regs(uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.wait::ld.sync.aligned;"
      : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]),
        "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]),
        "+r"(r[13]), "+r"(r[14]), "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]),
        "+r"(r[19]), "+r"(r[20]), "+r"(r[21]), "+r"(r[22]), "+r"(r[23]), "+r"(r[24]),
        "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]), "+r"(r[29]), "+r"(r[30]),
        "+r"(r[31])
      :
      : "memory");
}
// Named barrier over `count` threads (id 0 is __syncthreads).
B2K_DEV void named_bar_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Shared-memory matrix descriptor for a K-major operand stored in the 128-byte
// swizzled layout written by TMA (rows of 128 B, 8-row / 1024 B swizzle atoms).
B2K_DEV uint64_t smem_desc_sw128(const void* smem_tile) {
  uint64_t addr = smem_u32(smem_tile);
  uint64_t desc = 0;
  desc |= (addr & 0x3FFFFull) >> 4;          // start address
  desc |= (uint64_t)1 << 16;                 // leading byte offset (unused for SW128 K-major)
  desc |= (uint64_t)(1024 >> 4) << 32;       // stride byte offset: 8 rows x 128 B
  desc |= (uint64_t)1 << 46;                 // descriptor version (tcgen05)
  desc |= (uint64_t)2 << 61;                 // layout: 128-byte swizzle
  return desc;
}

// Instruction descriptor, kind::f16: D f32, A/B bf16 (ab_bf16=1) or f16 (0),
// both K-major, shape M x N.
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N, int ab_bf16) {
  return (1u << 4) | (uint32_t(ab_bf16) << 7) | (uint32_t(ab_bf16) << 10) |
         (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

// Instruction descriptor, kind::tf32: D f32, A/B tf32 (format 2), both
// K-major, shape M x N.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(N >> 3) << 17) |
         (uint32_t(M >> 4) << 24);
}

// Instruction descriptor, kind::i8: D s32 (format 2), A and B unsigned 8-bit
// (format 0), both K-major, shape M x N.
__host__ __device__ constexpr uint32_t idesc_u8(int M, int N) {
  return (2u << 4) | (0u << 7) | (0u << 10) | (uint32_t(N >> 3) << 17) |
         (uint32_t(M >> 4) << 24);
}

// Round a finite float to the nearest tf32 value (10 explicit mantissa bits,
// ties to even): the low 13 bits become zero, so the tensor core reads the
// value exactly.
B2K_DEV float tf32_rne(float v) {
  uint32_t u = __float_as_uint(v);
  u += 0x0FFFu + ((u >> 13) & 1u);
  return __uint_as_float(u & 0xFFFFE000u);
}

// --------------------------------------------------------------- arithmetic
// Batched kernels: the problem owning global row r, i.e. the largest p with
// row_start[p] <= r (row_start ascending; problems with no rows are skipped).
B2K_DEV int problem_of(const int64_t* __restrict__ row_start, int P, int64_t r) {
  int lo = 0, hi = P - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (row_start[mid] <= r)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

B2K_DEV float min3f(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
// Two independent f32 additions in one instruction.
B2K_DEV void add_f32x2(float& a0, float& a1, float b0, float b1) {
  uint64_t x, y, s;
  asm("mov.b64 %0, {%1,%2};" : "=l"(x) : "f"(a0), "f"(a1));
  asm("mov.b64 %0, {%1,%2};" : "=l"(y) : "f"(b0), "f"(b1));
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(s) : "l"(x), "l"(y));
  asm("mov.b64 {%0,%1}, %2;" : "=f"(a0), "=f"(a1) : "l"(s));
}

// Canonical float64 squared distance: strictly sequential over features with
// no fused multiply-add, so the value is bit-reproducible on host and device.
B2K_DEV double canonical_d2(const float* __restrict__ q, const float* __restrict__ x, int d) {
  double s = 0.0;
  if ((d & 3) == 0 && ((reinterpret_cast<uintptr_t>(q) | reinterpret_cast<uintptr_t>(x)) & 15) == 0) {
    // same sequential order, 16-byte loads
    const float4* q4 = reinterpret_cast<const float4*>(q);
    const float4* x4 = reinterpret_cast<const float4*>(x);
    for (int i = 0; i < d / 4; ++i) {
      const float4 a = q4[i], b = __ldg(x4 + i);
      double t = __dsub_rn((double)a.x, (double)b.x);
      s = __dadd_rn(s, __dmul_rn(t, t));
      t = __dsub_rn((double)a.y, (double)b.y);
      s = __dadd_rn(s, __dmul_rn(t, t));
      t = __dsub_rn((double)a.z, (double)b.z);
      s = __dadd_rn(s, __dmul_rn(t, t));
      t = __dsub_rn((double)a.w, (double)b.w);
      s = __dadd_rn(s, __dmul_rn(t, t));
    }
    return s;
  }
  for (int i = 0; i < d; ++i) {
    double t = __dsub_rn((double)q[i], (double)x[i]);
    s = __dadd_rn(s, __dmul_rn(t, t));
  }
  return s;
}

// canonical_d2 of two rows against one query, the two sequential chains
// interleaved so each covers the other's latency; each result is bit-identical
// to canonical_d2(q, x, d).
B2K_DEV void canonical_d2_pair(const float* __restrict__ q, const float* __restrict__ x0,
                               const float* __restrict__ x1, int d, double& s0, double& s1) {
  s0 = 0.0;
  s1 = 0.0;
  if ((d & 3) == 0 &&
      ((reinterpret_cast<uintptr_t>(q) | reinterpret_cast<uintptr_t>(x0) |
        reinterpret_cast<uintptr_t>(x1)) & 15) == 0) {
    const float4* q4 = reinterpret_cast<const float4*>(q);
    const float4* a4 = reinterpret_cast<const float4*>(x0);
    const float4* b4 = reinterpret_cast<const float4*>(x1);
    for (int i = 0; i < d / 4; ++i) {
      const float4 c = q4[i], a = __ldg(a4 + i), b = __ldg(b4 + i);
      const float cq[4] = {c.x, c.y, c.z, c.w}, xa[4] = {a.x, a.y, a.z, a.w},
                  xb[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const double ta = __dsub_rn((double)cq[e], (double)xa[e]);
        const double tb = __dsub_rn((double)cq[e], (double)xb[e]);
        s0 = __dadd_rn(s0, __dmul_rn(ta, ta));
        s1 = __dadd_rn(s1, __dmul_rn(tb, tb));
      }
    }
    return;
  }
  for (int i = 0; i < d; ++i) {
    const double ta = __dsub_rn((double)q[i], (double)x0[i]);
    const double tb = __dsub_rn((double)q[i], (double)x1[i]);
    s0 = __dadd_rn(s0, __dmul_rn(ta, ta));
    s1 = __dadd_rn(s1, __dmul_rn(tb, tb));
  }
}

}  // namespace b2k
