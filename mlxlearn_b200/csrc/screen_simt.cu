// Plain fp32 distance screen on the CUDA cores (the "plain FP32" form).
//
// Same contract and outputs as the tensor-core screen (tracker.cuh): per
// (split, query) candidate lists of v = fl(||y_x||^2 - 2 fl(<q^,x^>)), where
// q^ = fl32(q - c), x^ = fl32(x - c) are the centred operands (prep.cu) and the
// dot products are accumulated in fp32 FMA chains.  Replaces the reference's exact
// binary32 GEMM + Gram lower bound (src/mlxlearn_device/_binary32.py:71-296,
// _neighbors_general.py:188-242) and its direct scans for small d
// (_neighbors_fused.py:34-100).
//
// Error bound: prep.cu, with g = (d+4) u (1.01) for the fp32 FMA chains.
//
// Tile: 128 queries x 64 reference rows per CTA step, 16-wide k chunks staged
// through shared memory, an 8x4 register micro-tile per thread (256 threads).
// The finished v tile is transposed through shared memory and scanned by all
// 256 threads: for the kNN sink two threads per query row, each with its own
// tracker over one 32-column half of every tile (its own candidate list);
// radius sinks keep one scanner per row so each row's columns arrive in
// ascending order.  Trackers live in shared memory between tiles, so the
// GEMM phase holds only the accumulators and two CTAs fit on an SM.
#include "common.cuh"
#include "internal.cuh"
#include "sinks.cuh"

namespace b2k {

namespace {

constexpr int BM = kSimtBM, BN = kSimtBN, BK = 16;
constexpr int LDA = BM + 4, LDB = BN + 4, LDV = BN + 1;
constexpr int kThreads = 256;
static_assert(BM == 128 && BN == 64, "thread mapping below assumes a 128 x 64 tile");

struct SimtParams {
  const float* Q;
  const float* X;
  const float* nx;
  const float* E;
  const float* center;
  int m, n, d, S, tiles_per_split, n_tiles, exclude_self;
  long long q_offset;
  const int* perm;  // row -> original query row (or null)
  SinkArgs sink;
};

template <class Sink, int HALVES>
__host__ __device__ constexpr size_t simt_smem_bytes() {
  return (size_t)(2 * BK * LDA + 2 * BK * LDB + BM * LDV) * sizeof(float) +
         (size_t)BM * HALVES * sizeof(Sink);
}

// HALVES = scanners per row (2: kNN, each scans 32 columns of a tile; 1: radius).
template <class Sink, int HALVES>
__global__ void __launch_bounds__(kThreads, (sizeof(Sink) <= 160 ? 2 : 1))
    screen_simt_kernel(const __grid_constant__ SimtParams p) {
  extern __shared__ float sm[];
  float* As = sm;                        // [2][BK][LDA]
  float* Bs = As + 2 * BK * LDA;         // [2][BK][LDB]
  float* Vs = Bs + 2 * BK * LDB;         // [BM][LDV]
  Sink* sinks = reinterpret_cast<Sink*>(Vs + BM * LDV);  // [BM * HALVES]

  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;  // micro-tile: rows ty*8.., columns tx*4..
  const int t = blockIdx.x / p.S, s = blockIdx.x % p.S;
  const int row0 = t * BM;
  const int j0 = s * p.tiles_per_split;
  const int j1 = min(j0 + p.tiles_per_split, p.n_tiles);

  // scanner role: row r, half h
  const int r = tid & (BM - 1), h = tid >> 7;
  const int my_row = row0 + r;
  const bool scanner = h < HALVES && my_row < p.m;
  constexpr int kScanCols = BN / HALVES;
  if (scanner) {
    Sink sink;
    sink.init(p.sink, my_row, s * HALVES + h, p.E[my_row],
              p.exclude_self ? (int)(p.q_offset + (p.perm ? p.perm[my_row] : my_row)) : -1);
    sinks[tid] = sink;
  }

  // global -> register staging: column c = tid % 16 of the k chunk;
  // A rows tid / 16 + 16 i (8 of them), B rows tid / 16 + 16 i (4 of them)
  const int lc = tid & 15, lr = tid >> 4;
  float ra[8], rb[4];
  auto load_regs = [&](int k0, int col_base) {
    const int kq = k0 + lc;
    const bool kin = kq < p.d;
    const float c = kin ? __ldg(p.center + kq) : 0.0f;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int qi = row0 + lr + 16 * i;
      ra[i] = (qi < p.m && kin) ? __ldg(p.Q + (size_t)qi * p.d + kq) - c : 0.0f;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int xi = col_base + lr + 16 * i;
      rb[i] = (xi < p.n && kin) ? __ldg(p.X + (size_t)xi * p.d + kq) - c : 0.0f;
    }
  };
  auto store_regs = [&](int buf) {
#pragma unroll
    for (int i = 0; i < 8; ++i) As[(buf * BK + lc) * LDA + lr + 16 * i] = ra[i];
#pragma unroll
    for (int i = 0; i < 4; ++i) Bs[(buf * BK + lc) * LDB + lr + 16 * i] = rb[i];
  };

  const int nk = (p.d + BK - 1) / BK;
  for (int j = j0; j < j1; ++j) {
    const int col_base = j * BN;
    float acc[8][4];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = 0.0f;

    load_regs(0, col_base);
    store_regs(0);
    __syncthreads();
    for (int kc = 0; kc < nk; ++kc) {
      const int buf = kc & 1;
      if (kc + 1 < nk) load_regs((kc + 1) * BK, col_base);
#pragma unroll
      for (int kk = 0; kk < BK; ++kk) {
        const float4* ap = reinterpret_cast<const float4*>(As + (buf * BK + kk) * LDA + ty * 8);
        const float4 b0 = *reinterpret_cast<const float4*>(Bs + (buf * BK + kk) * LDB + tx * 4);
        const float4 a0 = ap[0], a1 = ap[1];
        const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
        // packed fp32 pairs: one fma.rn.f32x2 per two accumulators (each lane
        // result is the same rounded FMA as fmaf), half the FMA instructions
        uint64_t b01, b23;
        asm("mov.b64 %0, {%1, %2};" : "=l"(b01) : "f"(b0.x), "f"(b0.y));
        asm("mov.b64 %0, {%1, %2};" : "=l"(b23) : "f"(b0.z), "f"(b0.w));
#pragma unroll
        for (int a = 0; a < 8; ++a) {
          uint64_t aa, c01, c23;
          asm("mov.b64 %0, {%1, %1};" : "=l"(aa) : "f"(av[a]));
          asm("mov.b64 %0, {%1, %2};" : "=l"(c01) : "f"(acc[a][0]), "f"(acc[a][1]));
          asm("mov.b64 %0, {%1, %2};" : "=l"(c23) : "f"(acc[a][2]), "f"(acc[a][3]));
          asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(c01) : "l"(aa), "l"(b01));
          asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(c23) : "l"(aa), "l"(b23));
          asm("mov.b64 {%0, %1}, %2;" : "=f"(acc[a][0]), "=f"(acc[a][1]) : "l"(c01));
          asm("mov.b64 {%0, %1}, %2;" : "=f"(acc[a][2]), "=f"(acc[a][3]) : "l"(c23));
        }
      }
      if (kc + 1 < nk) store_regs(buf ^ 1);
      __syncthreads();
    }
    // v tile to shared memory (NaN marks columns past n: never admitted)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int col = col_base + tx * 4 + b;
      const float nxv = col < p.n ? __ldg(p.nx + col) : __int_as_float(0x7fc00000);
#pragma unroll
      for (int a = 0; a < 8; ++a) Vs[(ty * 8 + a) * LDV + tx * 4 + b] = fmaf(-2.0f, acc[a][b], nxv);
    }
    __syncthreads();
    if (scanner) {
      Sink sink = sinks[tid];
      sink.tile_sync();
      float* vr = Vs + r * LDV + h * kScanCols;
#pragma unroll
      for (int c0 = 0; c0 < kScanCols; c0 += 32) {
        float v[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] = vr[c0 + i];
        // the slow path may overwrite vr[c0 .. c0+8): those values are in v[]
        sink.offer32(v, col_base + h * kScanCols + c0, vr + c0);
      }
      sinks[tid] = sink;
    }
    __syncthreads();
  }
  if (scanner) {
    Sink sink = sinks[tid];
    sink.tile_sync();
    sink.finish(p.sink);
  }
}

template <class Sink, int HALVES>
void launch_simt_variant(const SimtParams& p, int grid, cudaStream_t st) {
  constexpr size_t smem = simt_smem_bytes<Sink, HALVES>();
  cudaFuncSetAttribute(screen_simt_kernel<Sink, HALVES>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  screen_simt_kernel<Sink, HALVES><<<grid, kThreads, smem, st>>>(p);
}

}  // namespace

int simt_column_groups(int sink_kind, bool noalloc) {
  return (sink_kind == kSinkKnn && !noalloc) ? 2 : 1;
}

void launch_screen_simt(const Index* ix, const float* Q, int64_t m, int64_t m_pad,
                        int exclude_self, int64_t q_offset, int S, const float* E, int sink_kind,
                        const SinkArgs& sa, cudaStream_t st, const int* perm, bool noalloc) {
  SimtParams p{};
  p.Q = Q;
  p.X = ix->X;
  p.nx = ix->nx32;
  p.center = ix->center;
  p.E = E;
  p.m = (int)m;
  p.n = (int)ix->n;
  p.d = ix->d;
  p.S = S;
  p.n_tiles = (int)((ix->n + BN - 1) / BN);
  p.tiles_per_split = (p.n_tiles + S - 1) / S;
  p.exclude_self = exclude_self;
  p.q_offset = q_offset;
  p.perm = perm;
  p.sink = sa;
  const int m_tiles = (int)(m_pad / BM);
  const int grid = m_tiles * S;
  if (grid <= 0) return;
  if (sink_kind == kSinkRadiusCount) return launch_simt_variant<RadiusCountSink, 1>(p, grid, st);
  if (sink_kind == kSinkRadiusFill) return launch_simt_variant<RadiusFillSink, 1>(p, grid, st);
  if (simt_column_groups(sink_kind, noalloc) == 1) {
    if (sa.k <= 16) return launch_simt_variant<KnnSink<16>, 1>(p, grid, st);
    if (sa.k <= 32) return launch_simt_variant<KnnSink<32>, 1>(p, grid, st);
    return launch_simt_variant<KnnSink<64>, 1>(p, grid, st);
  }
  if (sa.k <= 16) return launch_simt_variant<KnnSink<16>, 2>(p, grid, st);
  if (sa.k <= 32) return launch_simt_variant<KnnSink<32>, 2>(p, grid, st);
  launch_simt_variant<KnnSink<64>, 2>(p, grid, st);
}

}  // namespace b2k
