// bf16 distance screen on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// Replaces the reference's Gram screens (src/mlxlearn_device/_neighbors_general.py:188-329,
// the fp16 compact screen _neighbors_compact.py:20-371 and the int8 MPP
// screen _neighbors_integer.py:40-201), which materialise the distance tile in
// memory.  Here the tile lives only in TMEM.
//
// The accumulator holds the screen value itself, v = ||y_x||^2 - 2 <q^, x^>:
// besides the dp feature columns, every reference row carries 16 extra bf16
// columns [n_hi, n_mid, n_lo, 0...] (||y_x||^2 split into three bf16 parts)
// and every query [1, 1, 1, 0...], so one more K=16 MMA per tile adds the norm.
//
// One persistent CTA per SM, warp-specialised:
//   warp 0      TMA producer: query tile A (128 rows x dp, bf16) once per
//               work unit; reference tiles B (256 rows x 64 columns, 128-byte
//               swizzle) into an NST-deep shared-memory ring, the norm
//               columns (256 rows x 16, 32-byte swizzle) with the last block.
//   warp 1      MMA issuer: tcgen05.mma kind::f16, M=128 N=256 K=16, fp32
//               accumulators in TMEM, double-buffered (2 x 256 columns).
//               It polls one mbarrier (go) per chunk of C = min(KB, stages/2)
//               64-column blocks, i.e. once per tile for d <= 128: the thread
//               issuing MMAs runs only about one MMA ahead of the tensor pipe,
//               so every poll it makes idles the pipe; a poll per block plus
//               one for the accumulator cost up to 2x in measured MMA
//               throughput.
//   last warp   gate: per chunk, waits for its TMA stages (at a tile's first
//               chunk also for the epilogue's release of the accumulator
//               buffer; at a unit's start for the query tile), then arrives
//               on go.  A chunk never needs more stages than the ring holds.
//   warps 2..   EW epilogue warps.  Warp w reads TMEM lane group w % 4 (the
//               hardware's rule); the EW / 4 warps of a lane group take
//               equal column ranges of each tile (16 warps for k <= 16, 8 for
//               the lazy tracker).  Per 32-column
//               chunk: tcgen05.ld (two loads in flight), 3-input min over
//               8-column groups, and only when a group passes the row's
//               threshold, admit its columns (sinks.cuh).  The accumulator is
//               handed back to the MMA warp as soon as its last chunk is in
//               registers.  The distance tile never reaches HBM.
// A work unit is (query tile of 128 rows, split s of the reference tiles);
// units are numbered split-major and claimed in order by the persistent CTAs
// (an atomic counter, broadcast to the CTA's warps through a shared-memory
// ring), so the CTAs of a wave stream the same reference range (it stays in
// L2), later splits start from the k-th values the earlier ones published,
// and CTAs whose tiles run slow take fewer units.  Candidate lists are kept
// per (split, column group, row).
//
// Operands are the centred coordinates rounded to bf16 (A = -2 bf16(q - c),
// B = bf16(x - c)); the certified error bound of v is derived in prep.cu with
// g = (dp + 32) 2^-20 for the tensor-core fp32 accumulation.
//
// The TF32 instantiation is the plain (full-width) form on the tensor cores:
// kind::tf32 MMAs (M=128, N=256, K=8) over operands rounded to tf32.  In bytes
// nothing changes: a 128-byte swizzle row holds 32 fp32 instead of 64 bf16,
// each MMA still advances 32 bytes of K, and the norm columns are 8 fp32
// (three tf32 parts) instead of 16 bf16 -- the same 32 bytes per row.
#include <cuda_bf16.h>

#include <cstdlib>

#include "common.cuh"
#include "internal.cuh"
#include "sinks.cuh"
#include "tc_batch.cuh"

namespace b2k {

namespace {

struct TcParams {
  uint32_t spin_limit;       // polls of a main-loop wait before it gives up
  int stages;
  int a_blocks;              // 64-column query blocks the resident A region holds
  int m_tiles, S;            // single problem: m_tiles * S units, dealt round-robin
  const TcProblem* probs;    // batched: problem table
  const int4* items;         // batched: (problem, query tile, first tile, end tile)
  const int* cta_begin;      // batched: CTA b runs items [cta_begin[b], cta_begin[b + 1])
  int* status;
  int* unit_counter;         // units claimed dynamically (or null: round-robin / per-CTA lists)
  const int* home;           // single problem, seeding pass: tile t's window starts at home[t]
  int n_items;               // batched, claimed: items in the list
  TcProblem one;             // single problem
};

// Tensor maps of a launch: per operand group, the query tiles (A), reference
// tiles (B) and reference norm columns; the query-side ones columns are common.
template <int G>
struct TcMapSet {
  CUtensorMap a[G], b[G], baug[G];
  CUtensorMap aaug;
};

struct TcUnit {
  const TcProblem* pr;
  int t, j0, j1, slot;
};

// Dynamically claimed units are broadcast by the producer thread through a
// small ring in shared memory (index -1: no units left).
constexpr int kUnitRing = 4;
struct UnitRing {
  int* idx;          // [kUnitRing]
  uint64_t* full;    // [kUnitRing] producer -> consumers
  uint64_t* empty;   // [kUnitRing] consumers (MMA thread + epilogue threads) -> producer
};

// The sequence of work units of this CTA; every warp role walks it in step.
// Batched launches read host-balanced per-CTA lists; a single problem either
// deals units round-robin or, with a unit counter, lets the producer claim
// the next unit when it starts one, so CTAs whose tiles run slow take fewer.
template <bool BATCH>
struct UnitCursor {
  int u, end, step;
  bool dyn, producer;
  UnitRing ring;
  uint32_t rs, rph;
  B2K_DEV UnitCursor(const TcParams& p, const UnitRing& r, bool is_producer) {
    dyn = p.unit_counter != nullptr;
    producer = is_producer;
    ring = r;
    rs = 0;
    rph = 0;
    if (BATCH && dyn) {
      u = 0;
      end = p.n_items;
      step = 1;
    } else if (BATCH) {
      u = p.cta_begin[blockIdx.x];
      end = p.cta_begin[blockIdx.x + 1];
      step = 1;
    } else {
      u = blockIdx.x;
      end = p.m_tiles * p.S;
      step = gridDim.x;
    }
  }
  // Next unit index, -1 when done; false also when a bounded wait gave up.
  B2K_DEV bool claim(const TcParams& p, int* v) {
    if (!dyn) {
      if (u >= end) return false;
      *v = u;
      u += step;
      return true;
    }
    bool ok;
    if (producer) {
      int w = atomicAdd(p.unit_counter, 1);
      if (w >= end) w = -1;
      ok = mbar_wait(&ring.empty[rs], rph ^ 1, p.status, DEV_TIMEOUT_A, p.spin_limit);
      if (ok) {
        ring.idx[rs] = w;
        mbar_arrive(&ring.full[rs]);
      }
      *v = w;
    } else {
      ok = mbar_wait(&ring.full[rs], rph, p.status, DEV_TIMEOUT_A, p.spin_limit);
      if (ok) {
        *v = *reinterpret_cast<volatile int*>(&ring.idx[rs]);
        mbar_arrive(&ring.empty[rs]);
      }
    }
    if (++rs == (uint32_t)kUnitRing) {
      rs = 0;
      rph ^= 1;
    }
    return ok && *v >= 0;
  }
  B2K_DEV bool next(const TcParams& p, TcUnit& x) {
    int w;
    if (!claim(p, &w)) return false;
    if (BATCH) {
      const int4 it = p.items[w];
      x.pr = p.probs + it.x;
      x.t = it.y;
      x.j0 = it.z;
      x.j1 = it.w;
      x.slot = it.z / x.pr->tiles_per_split;
    } else {
      const int s = w / p.m_tiles;
      x.pr = &p.one;
      x.t = w % p.m_tiles;
      x.j0 = p.home ? p.home[x.t] : s * p.one.tiles_per_split;
      x.j1 = min(x.j0 + p.one.tiles_per_split, p.one.n_tiles);
      x.slot = s;
    }
    return true;
  }
  // Whether another unit follows (always assumed when units are claimed).
  B2K_DEV bool more() const { return dyn || u < end; }
};

constexpr uint32_t kATileBytes = kTcBM * kTcBK * 2;     // 16 KB per 64-column block
constexpr uint32_t kBTileBytes = kTcBN * kTcBK * 2;     // 32 KB per 64-column block
constexpr uint32_t kAAugBytes = kTcBM * kTcAug * 2;     // 4 KB (query ones)
constexpr uint32_t kBAugBytes = kTcBN * kTcAug * 2;     // 8 KB (reference norms)
constexpr int kSpillStride = 9;
// go barriers (gate -> MMA issuer), used in turn by successive chunks: the gate
// runs at most `stages` chunks (each at least one stage) ahead of the MMA
// issuer, so with more barriers than the deepest ring a barrier's next phase
// never starts before the issuer has consumed the previous one.
constexpr int kGoRing = 16;  // 8 spilled values per thread, conflict-free stride
// A CTA allocates all 512 TMEM columns, so no two may share an SM: ask for at
// least this much shared memory (more than half of the SM's 228 KB).
constexpr size_t kMinCtaSmem = 116 * 1024;

__host__ __device__ inline uint32_t tc_stage_bytes(bool a_stream) {
  return (a_stream ? kATileBytes : 0) + kBTileBytes + kBAugBytes;
}

__host__ __device__ inline size_t tc_smem_bytes(int KB, int stages, bool a_stream, int ew) {
  size_t a = a_stream ? 0 : (size_t)KB * kATileBytes;
  size_t spill = (size_t)ew * 32 * kSpillStride * sizeof(float);
  size_t bars = (2 * (size_t)stages + 8 + kGoRing + 2 * kUnitRing) * sizeof(uint64_t) + 16 +
                kUnitRing * sizeof(int);
  return 1024 /*alignment slack*/ + kAAugBytes + a + (size_t)tc_stage_bytes(a_stream) * stages +
         spill + bars;
}

// Shared-memory descriptor of a K-major operand in the 32-byte swizzled layout
// (rows of 32 B = 16 bf16, 8-row / 256 B atoms), as TMA writes it.
B2K_DEV uint64_t smem_desc_sw32(const void* smem_tile) {
  uint64_t addr = smem_u32(smem_tile);
  uint64_t desc = 0;
  desc |= (addr & 0x3FFFFull) >> 4;     // start address
  desc |= (uint64_t)1 << 16;            // leading byte offset (unused, K fits the atom)
  desc |= (uint64_t)(256 >> 4) << 32;   // stride byte offset: 8 rows x 32 B
  desc |= (uint64_t)1 << 46;            // descriptor version (tcgen05)
  desc |= (uint64_t)6 << 61;            // layout: 32-byte swizzle
  return desc;
}

// Threads per CTA: producer warp, MMA warp, EW epilogue warps, gate warp.
__host__ __device__ constexpr int tc_block_threads(int ew) { return 96 + 32 * ew; }

// Operand kinds of the screen kernel.
constexpr int kKindBf16 = 0, kKindTf32 = 1, kKindU8 = 2;

template <class Sink, bool A_STREAM, int EW, bool BATCH, int KIND>
__global__ void __launch_bounds__(tc_block_threads(EW), 1)
    screen_tc_kernel(const __grid_constant__ TcMapSet<BATCH ? kBatchGroups : 1> maps,
                     const __grid_constant__ TcParams p) {
  constexpr int G = BATCH ? kBatchGroups : 1;
  constexpr bool TF32 = KIND == kKindTf32;
  constexpr bool U8 = KIND == kKindU8;  // exact integer products, no norm columns
  constexpr int kEpiThreads = 32 * EW;
  constexpr int kHalves = EW / 4;                 // column groups per tile
  constexpr int kChunks = kTcBN / 32 / kHalves;   // 32-column chunks per epilogue warp
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int nst = p.stages;
  uint8_t* aaug_smem = smem;                                   // 4 KB, 1024-aligned
  uint8_t* a_smem = smem + kAAugBytes;                         // KB x 16 KB (1024-aligned)
  uint8_t* b_smem = a_smem + (A_STREAM ? 0 : p.a_blocks * kATileBytes);
  const uint32_t stage_bytes = tc_stage_bytes(A_STREAM);
  const uint32_t b_off = A_STREAM ? kATileBytes : 0;           // B tile inside a stage
  const uint32_t baug_off = b_off + kBTileBytes;               // norm columns inside a stage
  float* spill_all = reinterpret_cast<float*>(b_smem + (size_t)nst * stage_bytes);
  uint64_t* bars = reinterpret_cast<uint64_t*>(spill_all + kEpiThreads * kSpillStride);
  uint64_t* full = bars;
  uint64_t* empty = bars + nst;
  uint64_t* a_full = bars + 2 * nst;
  uint64_t* a_empty = a_full + 1;
  uint64_t* acc_full = a_empty + 1;   // [2]
  uint64_t* acc_empty = acc_full + 2; // [2]
  uint64_t* aaug_full = acc_empty + 2;
  uint64_t* mma_drain = aaug_full + 1;  // the MMA issuer's exit: all its MMAs complete
  uint64_t* go = mma_drain + 1;       // [kGoRing] gate -> MMA issuer, one per chunk in turn
  UnitRing ring;
  ring.full = go + kGoRing;            // [kUnitRing]
  ring.empty = ring.full + kUnitRing;  // [kUnitRing]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(ring.empty + kUnitRing);
  ring.idx = reinterpret_cast<int*>(tmem_slot + 4);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  volatile int* status = p.status;
  const uint32_t lim = p.spin_limit;

  if (threadIdx.x == 0) {
    for (int s = 0; s < nst; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(a_full, 1);
    // the query tile is free once its unit's MMAs are done (MMA commit) and
    // its load has landed (gate; a unit may have no tiles at all)
    mbar_init(a_empty, 2);
    mbar_init(&acc_full[0], 1);
    mbar_init(&acc_full[1], 1);
    // one arrival per epilogue warp: 512 per-thread arrivals on one barrier
    // serialise in shared memory and delayed every release by ~700 cycles
    mbar_init(&acc_empty[0], EW);
    mbar_init(&acc_empty[1], EW);
    mbar_init(aaug_full, 1);
    mbar_init(mma_drain, 1);
    for (int g = 0; g < kGoRing; ++g) mbar_init(&go[g], 1);
    for (int r = 0; r < kUnitRing; ++r) {
      mbar_init(&ring.full[r], 1);
      mbar_init(&ring.empty[r], 2 + kEpiThreads);  // MMA issuer, gate, epilogue threads
    }
    fence_mbar_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
#pragma unroll
      for (int g = 0; g < G; ++g) {
        prefetch_tmap(&maps.a[g]);
        prefetch_tmap(&maps.b[g]);
        if (!U8) prefetch_tmap(&maps.baug[g]);
      }
      if (U8) {
        mbar_arrive(aaug_full);  // no norm columns: the epilogue adds ||x||^2
      } else {
        prefetch_tmap(&maps.aaug);
        // the query-side norm columns are the same for every tile: load once
        mbar_arrive_expect_tx(aaug_full, kAAugBytes);
        tma_load_2d(aaug_smem, &maps.aaug, aaug_full, 0, 0);
      }
      uint32_t stage = 0, phase = 0, a_phase = 0;
      // copies issued, for the exit path: per stage the parity of the full
      // phase its latest load completes, and the same for the query tile
      uint32_t pend = 0, pend_par = 0, a_loads = 0;
      UnitCursor<BATCH> cur(p, ring, true);
      TcUnit x;
      while (cur.next(p, x)) {
        const int KB = x.pr->KB;
        // TMA coordinates count elements of the map's type: a 128-byte block
        // is 64 bf16, 32 fp32 or 128 u8 columns
        constexpr int kx = TF32 ? kTcBKf : (U8 ? kTcBKu : kTcBK);
        const int g = G == 1 ? 0 : x.pr->group;
        const int a_row = x.pr->a_row0 + x.t * kTcBM;
        const int b_row0 = x.pr->b_row0;
        const CUtensorMap* tmA = &maps.a[g];
        const CUtensorMap* tmB = &maps.b[g];
        const CUtensorMap* tmBaug = &maps.baug[g];
        if (!A_STREAM) {
          if (!mbar_wait(a_empty, a_phase ^ 1, status, DEV_TIMEOUT_A, lim)) goto prod_done;
          a_phase ^= 1;
          ++a_loads;
          mbar_arrive_expect_tx(a_full, KB * kATileBytes);
          for (int kb = 0; kb < KB; ++kb)
            tma_load_2d(a_smem + kb * kATileBytes, tmA, a_full, kb * kx, a_row);
        }
        for (int j = x.j0; j < x.j1; ++j) {
          const int b_row = b_row0 + j * kTcBN;
          for (int kb = 0; kb < KB; ++kb) {
            if (!mbar_wait(&empty[stage], phase ^ 1, status, DEV_TIMEOUT_EMPTY, lim))
              goto prod_done;
            pend |= 1u << stage;
            pend_par = (pend_par & ~(1u << stage)) | (phase << stage);
            uint8_t* st = b_smem + (size_t)stage * stage_bytes;
            const bool last = !U8 && kb == KB - 1;  // with the norm columns
            mbar_arrive_expect_tx(&full[stage], (A_STREAM ? kATileBytes : 0) + kBTileBytes +
                                                    (last ? kBAugBytes : 0));
            if (A_STREAM) tma_load_2d(st, tmA, &full[stage], kb * kx, a_row);
            tma_load_2d(st + b_off, tmB, &full[stage], kb * kx, b_row);
            if (last) tma_load_2d(st + baug_off, tmBaug, &full[stage], 0, b_row);
            if (++stage == (uint32_t)nst) {
              stage = 0;
              phase ^= 1;
            }
          }
        }
      }
      // Drain: wait until the consumer released every stage we filled.
      for (int s = 0; s < nst; ++s) {
        if (!mbar_wait(&empty[stage], phase ^ 1, status, DEV_TIMEOUT_EMPTY, lim)) break;
        if (++stage == (uint32_t)nst) {
          stage = 0;
          phase ^= 1;
        }
      }
      // with claimed units the MMA warp releases the query tile after every
      // unit: take the last release so no arrival lands after the CTA exits
      if (!A_STREAM && cur.dyn) mbar_wait(a_empty, a_phase ^ 1, status, DEV_TIMEOUT_A, lim);
    prod_done:
      // Whichever way the loop ended (a wait that gave up included), no bulk
      // copy of this CTA may still be in flight when it exits: wait for the
      // latest load of every stage, of the query tile and of the ones columns.
      for (int s = 0; s < nst; ++s)
        if (pend & (1u << s)) mbar_wait_drain(&full[s], (pend_par >> s) & 1u, status);
      if (a_loads) mbar_wait_drain(a_full, (a_loads - 1) & 1u, status);
      mbar_wait_drain(aaug_full, 0, status);
    }
  } else if (warp == 1) {
    // --------------------------------------------------------- MMA issuer
    if (lane == 0) {
      constexpr uint32_t idesc = TF32 ? idesc_tf32(kTcBM, kTcBN)
                                 : U8 ? idesc_u8(kTcBM, kTcBN)
                                      : idesc_f16(kTcBM, kTcBN, 1);
      // one MMA of the screen's kind: 32 bytes of K (16 bf16, 8 tf32 or 32 u8)
      auto mma = [&](uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t acc) {
        if constexpr (TF32)
          mma_tf32(d_tmem, a, b, idesc, acc);
        else if constexpr (U8)
          mma_i8(d_tmem, a, b, idesc, acc);
        else
          mma_f16(d_tmem, a, b, idesc, acc);
      };
      uint32_t stage = 0, acc_it = 0, chunk = 0;
      bool issued = false;  // any MMA (for the exit path's drain)
      {
        const uint64_t aaug_desc = smem_desc_sw32(aaug_smem);
        UnitCursor<BATCH> cur(p, ring, false);
        TcUnit x;
        while (cur.next(p, x)) {
          const int KB = x.pr->KB;
          const int C = max(1, min(KB, nst / 2));  // blocks per gated chunk
          for (int j = x.j0; j < x.j1; ++j) {
            const uint32_t buf = acc_it & 1;
            const uint32_t d_tmem = tmem_base + buf * kTcBN;
            for (int kb = 0; kb < KB; ++kb) {
              if (kb % C == 0) {
                // the chunk's operands are in shared memory (and, at kb 0, the
                // accumulator is free)
                if (!mbar_wait(&go[chunk % kGoRing], (chunk / kGoRing) & 1, status,
                               DEV_TIMEOUT_ACC, lim))
                  goto mma_done;
                ++chunk;
                tc_fence_after();
              }
              issued = true;
              uint8_t* st = b_smem + (size_t)stage * stage_bytes;
              const uint8_t* a_tile = A_STREAM ? st : a_smem + kb * kATileBytes;
              const uint64_t adesc = smem_desc_sw128(a_tile);
              const uint64_t bdesc = smem_desc_sw128(st + b_off);
#pragma unroll
              for (int kk = 0; kk < 4; ++kk) {
                // advance 32 bytes inside the 128-byte swizzle atom: +2 in 16-byte units
                mma(d_tmem, adesc + 2 * kk, bdesc + 2 * kk, (kb | kk) != 0);
              }
              if (!U8 && kb == KB - 1)  // + ||y_x||^2 through the norm columns
                mma(d_tmem, aaug_desc, smem_desc_sw32(st + baug_off), 1);
              mma_commit(&empty[stage]);
              if (++stage == (uint32_t)nst) stage = 0;
            }
            mma_commit(&acc_full[buf]);
            ++acc_it;
          }
          // Release the query tile for the next unit (not after the last one, so
          // no arrival can land after the CTA has exited).
          if (!A_STREAM && cur.more()) mma_commit(a_empty);
        }
      }
    mma_done:
      // every MMA this thread issued has completed before the CTA moves on to
      // free its TMEM (on the normal path the epilogue has seen them all)
      if (issued) {
        mma_commit(mma_drain);
        mbar_wait_drain(mma_drain, 0, status);
      }
    }
  } else if (warp == 2 + EW) {
    // --------------------------------------------------------------- gate
    if (lane == 0) {
      uint32_t stage = 0, phase = 0, a_phase = 0, acc_it = 0, chunk = 0;
      if (!mbar_wait(aaug_full, 0, status, DEV_TIMEOUT_A, lim)) goto gate_done;
      {
        UnitCursor<BATCH> cur(p, ring, false);
        TcUnit x;
        while (cur.next(p, x)) {
          const int KB = x.pr->KB;
          const int C = max(1, min(KB, nst / 2));  // as the MMA issuer
          if (!A_STREAM) {
            if (!mbar_wait(a_full, a_phase, status, DEV_TIMEOUT_A, lim)) goto gate_done;
            a_phase ^= 1;
          }
          for (int j = x.j0; j < x.j1; ++j) {
            const uint32_t buf = acc_it & 1, apar = (acc_it >> 1) & 1;
            // the epilogue has read this buffer's previous tile
            if (!mbar_wait(&acc_empty[buf], apar ^ 1, status, DEV_TIMEOUT_ACC, lim))
              goto gate_done;
            for (int kb = 0; kb < KB; ++kb) {
              if (!mbar_wait(&full[stage], phase, status, DEV_TIMEOUT_FULL, lim)) goto gate_done;
              if (++stage == (uint32_t)nst) {
                stage = 0;
                phase ^= 1;
              }
              if ((kb + 1) % C == 0 || kb + 1 == KB) {
                mbar_arrive(&go[chunk % kGoRing]);
                ++chunk;
              }
            }
            ++acc_it;
          }
          // (not after the last unit, as with the MMA issuer's release)
          if (!A_STREAM && cur.more()) mbar_arrive(a_empty);
        }
      }
    gate_done:;
    }
  } else {
    // ----------------------------------------------------------- epilogue
    const int ew = warp - 2;                // 0 .. EW-1
    const int g = warp & 3;                 // TMEM lane group this warp may access
    const int half = ew / 4;                // column group of this warp
    const int row_in_tile = g * 32 + lane;
    const int et = threadIdx.x - 64;        // 0 .. kEpiThreads-1
    float* spill = spill_all + et * kSpillStride;
    // u8: the warp's ||x||^2 values of the current tile (its spill rows are unused)
    int* nx_warp = reinterpret_cast<int*>(spill_all + (size_t)ew * 32 * kSpillStride);
    uint32_t acc_it = 0;
    UnitCursor<BATCH> cur(p, ring, false);
    TcUnit x;
    for (;;) {
      // warp-uniform: a bounded wait that gave up in one lane ends the warp
      if (!__all_sync(0xffffffffu, cur.next(p, x))) break;
      const TcProblem& pr = *x.pr;
      const int row = x.t * kTcBM + row_in_tile;
      const bool valid = row < pr.m;
      const int c0 = half * kChunks;  // first 32-column chunk of this warp
      // warp-collective sinks run on every lane (inactive past the block's end)
      const bool live = Sink::kWarpWide || valid;
      Sink sink;
      // the excluded column of a self-query: its training row, or that row's
      // place among grouped reference rows
      auto self_column = [&](int orig) -> int {
        const long long r = pr.q_offset + orig;
        return pr.self_col ? pr.self_col[r] : (int)r;
      };
      if constexpr (Sink::kWarpWide) {
        const int orig = valid ? (pr.perm ? pr.perm[row] : row) : 0;
        sink.init_warp(pr.sink, row, x.slot * kHalves + half, (valid && pr.E) ? pr.E[row] : 0.0f,
                       (valid && pr.exclude_self) ? self_column(orig) : -1, valid,
                       reinterpret_cast<unsigned*>(spill_all + (size_t)ew * 32 * kSpillStride));
      } else if (valid) {
        const int orig = pr.perm ? pr.perm[row] : row;
        sink.init(pr.sink, row, x.slot * kHalves + half, pr.E ? pr.E[row] : 0.0f,
                  pr.exclude_self ? self_column(orig) : -1);
      }
      uint32_t pending_key = kNoKey;
      for (int j = x.j0; j < x.j1; ++j) {
        // the other warps' k-th values for this query: consumed after the tile
        // the load issued one tile earlier is consumed at the end of this one
        const uint32_t shared_key = pending_key;
        pending_key = live ? sink.tile_fetch() : 0u;
        const uint32_t buf = acc_it & 1, apar = (acc_it >> 1) & 1;
        // u8: ||x||^2 of this warp's columns, fetched before the wait
        int nxr[kChunks];
        if constexpr (U8) {
          const int* g_nx = pr.nxu + (size_t)j * kTcBN + c0 * 32 + lane;
#pragma unroll
          for (int c = 0; c < kChunks; ++c) nxr[c] = __ldg(g_nx + c * 32);
        }
        // warp-uniform outcome, so collective sinks never run on a partial warp
        if (!__all_sync(0xffffffffu,
                        mbar_wait(&acc_full[buf], apar, status, DEV_TIMEOUT_ACC, lim)))
          goto epi_done;
        tc_fence_after();
        if constexpr (U8) {
          // into the warp's scratch, read back as broadcasts (the previous
          // tile's reads are done first)
          __syncwarp();
#pragma unroll
          for (int c = 0; c < kChunks; ++c) nx_warp[c * 32 + lane] = nxr[c];
          __syncwarp();
        }
        const uint32_t tbase = tmem_base + ((uint32_t)(g * 32) << 16) + buf * kTcBN + c0 * 32;
        auto process = [&](const uint32_t(&r)[32], int c) {
          if constexpr (U8) {
            // v = ||x||^2 - 2<q, x>, exact in int32
            const int4* nx4 = reinterpret_cast<const int4*>(nx_warp + c * 32);
            int v[32];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              const int4 t = nx4[i];
              v[4 * i] = t.x - 2 * (int)r[4 * i];
              v[4 * i + 1] = t.y - 2 * (int)r[4 * i + 1];
              v[4 * i + 2] = t.z - 2 * (int)r[4 * i + 2];
              v[4 * i + 3] = t.w - 2 * (int)r[4 * i + 3];
            }
            if (live) sink.offer32i(v, j * kTcBN + (c0 + c) * 32);
          } else {
            float v[32];
#pragma unroll
            for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
            if (live) sink.offer32(v, j * kTcBN + (c0 + c) * 32, spill);
          }
        };
        if constexpr (EW == 16) {
          // four warps per lane group: one 32-column buffer each (register budget);
          // the other warps of the SM cover the load latency
#pragma unroll 1
          for (int c = 0; c < kChunks; ++c) {
            uint32_t ra[32];
            tmem_ld_32x32b_x32(tbase + c * 32, ra);
            tmem_ld_wait_regs(ra);
            if (c == kChunks - 1) {
              // every lane's loads are complete (wait::ld) before the warp's arrival
              tc_fence_before();
              __syncwarp();
              if (lane == 0) mbar_arrive(&acc_empty[buf]);
            }
            process(ra, c);
          }
        } else {
        // Two 32-column TMEM loads in flight: load chunk c+1 while chunk c is scanned.
        uint32_t ra[32], rb[32];
        tmem_ld_32x32b_x32(tbase, ra);
        tmem_ld_wait_regs(ra);
#pragma unroll 1
        for (int c = 0; c < kChunks; c += 2) {
          tmem_ld_32x32b_x32(tbase + (c + 1) * 32, rb);
          process(ra, c);
          tmem_ld_wait_regs(rb);
          if (c + 2 < kChunks) {
            tmem_ld_32x32b_x32(tbase + (c + 2) * 32, ra);
            process(rb, c + 1);
            tmem_ld_wait_regs(ra);
          } else {
            // all of this warp's columns are in registers: hand the buffer back
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[buf]);
            process(rb, c + 1);
          }
        }
        }
        ++acc_it;
        if (live) sink.tile_apply(shared_key);
      }
      if constexpr (Sink::kWarpWide) {
        sink.tile_sync();
        sink.finish_warp(pr.sink);
      } else if (valid) {
        sink.tile_sync();
        sink.finish(pr.sink);
      }
    }
  epi_done:;
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, 512);
  }
}

template <class Sink, bool A_STREAM, int EW, bool BATCH, int KIND = kKindBf16>
size_t tc_variant_smem(int KB_max, int* stages_out) {
  const size_t budget = 227 * 1024;
  int stages = 8;
  while (stages > 2 && tc_smem_bytes(KB_max, stages, A_STREAM, EW) > budget) --stages;
  if (stages_out) *stages_out = stages;
  size_t smem = tc_smem_bytes(KB_max, stages, A_STREAM, EW);
  return smem < kMinCtaSmem ? kMinCtaSmem : smem;
}

template <class Sink, bool A_STREAM, int EW, bool BATCH, int KIND = kKindBf16>
int prepare_tc_variant(int KB_max) {
  const size_t smem = tc_variant_smem<Sink, A_STREAM, EW, BATCH>(KB_max, nullptr);
  auto kern = screen_tc_kernel<Sink, A_STREAM, EW, BATCH, KIND>;
  return (int)cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <class Sink, bool A_STREAM, int EW, bool BATCH, int KIND = kKindBf16>
int launch_tc_variant(const TcMapSet<BATCH ? kBatchGroups : 1>& maps, const TcParams& p, int KB_max,
                      int grid, cudaStream_t st) {
  int stages = 0;
  const size_t smem = tc_variant_smem<Sink, A_STREAM, EW, BATCH>(KB_max, &stages);
  TcParams q = p;
  q.stages = stages;
  q.a_blocks = KB_max;
  q.spin_limit = device_spin_limit();
  auto kern = screen_tc_kernel<Sink, A_STREAM, EW, BATCH, KIND>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return (int)e;
  kern<<<grid, tc_block_threads(EW), smem, st>>>(maps, q);
  return (int)cudaGetLastError();
}

}  // namespace

// Column groups (epilogue warps per TMEM lane group) of the kNN screen for k:
// each group keeps its own candidate lists.
// Epilogue warps of the single-problem kNN screen: four per TMEM lane group
// for the register-heap trackers (k <= 16), which shortens each warp's
// per-tile chain and cuts the MMA warp's waits for a free accumulator
// (B2K_TC_EW=8 selects two); two for the lazy tracker.
static int tc_knn_ew(int k) {
  if (k > 16) return 8;
  static const int ew = [] {
    const char* e = getenv("B2K_TC_EW");
    return (e && atoi(e) == 8) ? 8 : 16;
  }();
  return ew;
}
int tc_column_groups(int k) { return tc_knn_ew(k) / 4; }
// Radius screens: four epilogue warps per TMEM lane group, one list per
// (split, column group, row).
constexpr int kRadiusEW = 16;
int tc_radius_groups() { return kRadiusEW / 4; }
bool tc_lazy_sink(int k) { return k > 16; }

int launch_screen_tc(Index* ix, const CUtensorMap* tmap_a, int64_t m, int64_t m_pad,
                     int exclude_self, int64_t q_offset, int S, const float* E, int sink_kind,
                     const SinkArgs& sa, int* status, cudaStream_t st, const int* perm,
                     int* unit_counter, bool tf32, const int* home, int home_tiles) {
  if (tf32 && sink_kind != kSinkKnn) return (int)cudaErrorInvalidValue;
  if (home && (S != 1 || home_tiles <= 0)) return (int)cudaErrorInvalidValue;
  TcParams p{};
  p.unit_counter = unit_counter;
  p.home = home;
  TcProblem& one = p.one;
  one.m = (int)m;
  one.KB = tf32 ? ix->dpt / kTcBKf : ix->dp / kTcBK;
  one.n_tiles = (int)(ix->n_pad_tc / kTcBN);
  one.tiles_per_split = home ? home_tiles : (one.n_tiles + S - 1) / S;
  one.exclude_self = exclude_self;
  one.q_offset = q_offset;
  one.E = E;
  one.perm = perm;
  one.self_col = ix->xinv;
  one.sink = sa;
  p.S = S;
  p.m_tiles = (int)(m_pad / kTcBM);
  p.status = status;
  const int KB = one.KB;
  const bool a_stream = KB > 4;
  const int units = p.m_tiles * S;
  const int grid = units < num_sms(ix->device) ? units : num_sms(ix->device);
  if (grid <= 0) return 0;
  TcMapSet<1> maps;
  maps.a[0] = *tmap_a;
  maps.b[0] = tf32 ? ix->tmap_bt : ix->tmap_b;
  maps.baug[0] = tf32 ? ix->tmap_btaug : ix->tmap_baug;
  maps.aaug = tf32 ? ix->tmap_ataug : ix->tmap_aaug;
  if (tf32) {
#define B2K_TC_LAUNCH_TF32(SINK, EW)                                                 \
  (a_stream ? launch_tc_variant<SINK, true, EW, false, kKindTf32>(maps, p, KB, grid, st) \
            : launch_tc_variant<SINK, false, EW, false, kKindTf32>(maps, p, KB, grid, st))
    if (tc_knn_ew(sa.k) == 16) {
      if (sa.k <= 8) return B2K_TC_LAUNCH_TF32(KnnSink<8>, 16);
      if (sa.k <= 12) return B2K_TC_LAUNCH_TF32(KnnSink<12>, 16);
      return B2K_TC_LAUNCH_TF32(KnnSink<16>, 16);
    }
    if (sa.k <= 8) return B2K_TC_LAUNCH_TF32(KnnSink<8>, 8);
    if (sa.k <= 12) return B2K_TC_LAUNCH_TF32(KnnSink<12>, 8);
    if (!tc_lazy_sink(sa.k)) return B2K_TC_LAUNCH_TF32(KnnSink<16>, 8);
    return B2K_TC_LAUNCH_TF32(LazyKnnSink, 8);
#undef B2K_TC_LAUNCH_TF32
  }
#define B2K_TC_LAUNCH(SINK, EW)                                                \
  (a_stream ? launch_tc_variant<SINK, true, EW, false>(maps, p, KB, grid, st) \
            : launch_tc_variant<SINK, false, EW, false>(maps, p, KB, grid, st))
  if (sink_kind == kSinkRadiusCount) return B2K_TC_LAUNCH(RadiusCountSink, kRadiusEW);
  if (sink_kind == kSinkRadiusFill) return B2K_TC_LAUNCH(RadiusFillSink, kRadiusEW);
  if (sink_kind == kSinkRadiusList) return B2K_TC_LAUNCH(RadiusListSink, kRadiusEW);
  if (tc_knn_ew(sa.k) == 16) {
    if (sa.k <= 8) return B2K_TC_LAUNCH(KnnSink<8>, 16);
    if (sa.k <= 12) return B2K_TC_LAUNCH(KnnSink<12>, 16);
    return B2K_TC_LAUNCH(KnnSink<16>, 16);
  }
  if (sa.k <= 8) return B2K_TC_LAUNCH(KnnSink<8>, 8);
  if (sa.k <= 12) return B2K_TC_LAUNCH(KnnSink<12>, 8);
  if (!tc_lazy_sink(sa.k)) return B2K_TC_LAUNCH(KnnSink<16>, 8);
  return B2K_TC_LAUNCH(LazyKnnSink, 8);
#undef B2K_TC_LAUNCH
}

int launch_screen_tc_u8(Index* ix, const CUtensorMap* tmap_a, int64_t m, int64_t m_pad,
                        int exclude_self, int64_t q_offset, int S, const SinkArgs& sa,
                        int* status, cudaStream_t st, int* unit_counter) {
  if (sa.k < 1 || sa.k > kU8MaxK || !ix->u8_ready) return (int)cudaErrorInvalidValue;
  TcParams p{};
  p.unit_counter = unit_counter;
  TcProblem& one = p.one;
  one.m = (int)m;
  one.KB = ix->dpu / kTcBKu;
  one.n_tiles = (int)(ix->n_pad_tc / kTcBN);
  one.tiles_per_split = (one.n_tiles + S - 1) / S;
  one.exclude_self = exclude_self;
  one.q_offset = q_offset;
  one.nxu = ix->nxu;  // training order: the self column is the training row
  one.sink = sa;
  p.S = S;
  p.m_tiles = (int)(m_pad / kTcBM);
  p.status = status;
  const int KB = one.KB;
  const bool a_stream = KB > 4;
  const int units = p.m_tiles * S;
  const int grid = units < num_sms(ix->device) ? units : num_sms(ix->device);
  if (grid <= 0) return 0;
  TcMapSet<1> maps{};  // no norm-column maps: the epilogue adds ||x||^2
  maps.a[0] = *tmap_a;
  maps.b[0] = ix->tmap_bu;
#define B2K_TC_LAUNCH_U8(SINK, EW)                                                 \
  (a_stream ? launch_tc_variant<SINK, true, EW, false, kKindU8>(maps, p, KB, grid, st) \
            : launch_tc_variant<SINK, false, EW, false, kKindU8>(maps, p, KB, grid, st))
  return sa.k <= 8 ? B2K_TC_LAUNCH_U8(ExactU8Sink<8>, 16) : B2K_TC_LAUNCH_U8(ExactU8Sink<16>, 8);
#undef B2K_TC_LAUNCH_U8
}
// u8 screen: 16 epilogue warps while the 8-wide heap fits their registers,
// 8 warps (two TMEM loads in flight each) for k = 9..16
int tc_u8_column_groups(int k) { return k <= 8 ? 4 : 2; }

// Batched launches: kNN sinks only, with 4 or 8 epilogue warps.  Heap width
// class 64 stands for the lazy tracker (every k > 16).
#define B2K_TC_BATCH_DISPATCH(CALL)                                         \
  switch (kmax * 32 + ew) {                                                 \
    case 8 * 32 + 16: return CALL(KnnSink<8>, 16);                          \
    case 12 * 32 + 16: return CALL(KnnSink<12>, 16);                        \
    case 16 * 32 + 16: return CALL(KnnSink<16>, 16);                        \
    case 8 * 32 + 8: return CALL(KnnSink<8>, 8);                            \
    case 8 * 32 + 4: return CALL(KnnSink<8>, 4);                            \
    case 12 * 32 + 8: return CALL(KnnSink<12>, 8);                          \
    case 12 * 32 + 4: return CALL(KnnSink<12>, 4);                          \
    case 16 * 32 + 8: return CALL(KnnSink<16>, 8);                          \
    case 16 * 32 + 4: return CALL(KnnSink<16>, 4);                          \
    case 64 * 32 + 8: return CALL(LazyKnnSink, 8);                          \
    case 64 * 32 + 4: return CALL(LazyKnnSink, 4);                          \
    default: return (int)cudaErrorInvalidValue;                             \
  }

int prepare_screen_tc_batch(int kmax, int ew, bool a_stream, int KB_max) {
  if (!a_stream && KB_max > 4) return (int)cudaErrorInvalidValue;
#define B2K_PREP(SINK, EW)                                         \
  (a_stream ? prepare_tc_variant<SINK, true, EW, true>(KB_max) \
            : prepare_tc_variant<SINK, false, EW, true>(KB_max))
  B2K_TC_BATCH_DISPATCH(B2K_PREP)
#undef B2K_PREP
}

int launch_screen_tc_batch(const TcBatchLaunch& L, cudaStream_t st) {
  if (L.grid <= 0) return 0;
  if (L.groups < 1 || L.groups > kBatchGroups) return (int)cudaErrorInvalidValue;
  if (!L.a_stream && L.KB_max > 4) return (int)cudaErrorInvalidValue;
  TcMapSet<kBatchGroups> maps;
  for (int g = 0; g < kBatchGroups; ++g) {
    // unused slots repeat group 0 (never addressed: every problem names a live group)
    const int s = g < L.groups ? g : 0;
    maps.a[g] = L.a[s];
    maps.b[g] = L.b[s];
    maps.baug[g] = L.baug[s];
  }
  maps.aaug = L.aaug;
  TcParams p{};
  p.probs = L.probs;
  p.items = L.items;
  p.cta_begin = L.cta_begin;
  p.unit_counter = L.item_counter;
  p.n_items = L.n_items;
  p.status = L.status;
  const int kmax = L.kmax, ew = L.ew, KB = L.KB_max, grid = L.grid;
  const bool a_stream = L.a_stream;
#define B2K_LAUNCH(SINK, EW)                                                       \
  (a_stream ? launch_tc_variant<SINK, true, EW, true>(maps, p, KB, grid, st) \
            : launch_tc_variant<SINK, false, EW, true>(maps, p, KB, grid, st))
  B2K_TC_BATCH_DISPATCH(B2K_LAUNCH)
#undef B2K_LAUNCH
}
#undef B2K_TC_BATCH_DISPATCH

}  // namespace b2k
