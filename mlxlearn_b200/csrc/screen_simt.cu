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
// Tile: 128 queries x 128 reference rows per CTA step, 16-wide k chunks staged
// through shared memory, an 8x8 register micro-tile per thread; the finished
// v tile is transposed through shared memory so that each of 128 threads scans
// one query row with its own tracker.
#include "common.cuh"
#include "internal.cuh"
#include "sinks.cuh"

namespace b2k {

namespace {

constexpr int BM = kSimtBM, BN = kSimtBN, BK = 16, LDA = BM + 4, LDV = BN + 1;
constexpr int kThreads = 256;

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

template <class Sink>
__global__ void __launch_bounds__(kThreads) screen_simt_kernel(const SimtParams p) {
  extern __shared__ float sm[];
  float* As = sm;                    // [2][BK][LDA]
  float* Bs = As + 2 * BK * LDA;     // [2][BK][LDA]
  float* Vs = Bs + 2 * BK * LDA;     // [BM][LDV]

  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int t = blockIdx.x / p.S, s = blockIdx.x % p.S;
  const int row0 = t * BM;
  const int j0 = s * p.tiles_per_split;
  const int j1 = min(j0 + p.tiles_per_split, p.n_tiles);

  Sink sink;
  const int my_row = row0 + tid;
  const bool scanner = tid < BM && my_row < p.m;
  if (scanner)
    sink.init(p.sink, my_row, s, p.E[my_row],
              p.exclude_self ? (int)(p.q_offset + (p.perm ? p.perm[my_row] : my_row)) : -1);

  // global -> register staging: thread loads 8 elements of each tile,
  // column c = tid % 16, rows r = tid / 16 + 16 i.
  const int lc = tid & 15, lr = tid >> 4;
  float ra[8], rb[8];

  auto load_regs = [&](int k0, int col_base) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      int r = lr + 16 * i;
      int kq = k0 + lc;
      int qi = row0 + r, xi = col_base + r;
      const float c = kq < p.d ? __ldg(p.center + kq) : 0.0f;
      ra[i] = (qi < p.m && kq < p.d) ? __ldg(p.Q + (size_t)qi * p.d + kq) - c : 0.0f;
      rb[i] = (xi < p.n && kq < p.d) ? __ldg(p.X + (size_t)xi * p.d + kq) - c : 0.0f;
    }
  };
  auto store_regs = [&](int buf) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      As[(buf * BK + lc) * LDA + lr + 16 * i] = ra[i];
      Bs[(buf * BK + lc) * LDA + lr + 16 * i] = rb[i];
    }
  };

  const int nk = (p.d + BK - 1) / BK;
  for (int j = j0; j < j1; ++j) {
    const int col_base = j * BN;
    float acc[8][8];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
      for (int b = 0; b < 8; ++b) acc[a][b] = 0.0f;

    load_regs(0, col_base);
    store_regs(0);
    __syncthreads();
    for (int kc = 0; kc < nk; ++kc) {
      const int buf = kc & 1;
      if (kc + 1 < nk) load_regs((kc + 1) * BK, col_base);
#pragma unroll
      for (int kk = 0; kk < BK; ++kk) {
        const float4* ap = reinterpret_cast<const float4*>(As + (buf * BK + kk) * LDA + ty * 8);
        const float4* bp = reinterpret_cast<const float4*>(Bs + (buf * BK + kk) * LDA + tx * 8);
        float4 a0 = ap[0], a1 = ap[1], b0 = bp[0], b1 = bp[1];
        float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
        float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
          for (int b = 0; b < 8; ++b) acc[a][b] = fmaf(av[a], bv[b], acc[a][b]);
      }
      if (kc + 1 < nk) store_regs(buf ^ 1);
      __syncthreads();
    }
    // v tile to shared memory (NaN marks columns past n: never admitted)
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const int col = col_base + tx * 8 + b;
      const float nxv = col < p.n ? __ldg(p.nx + col) : __int_as_float(0x7fc00000);
#pragma unroll
      for (int a = 0; a < 8; ++a) Vs[(ty * 8 + a) * LDV + tx * 8 + b] = fmaf(-2.0f, acc[a][b], nxv);
    }
    __syncthreads();
    if (scanner) {
      sink.tile_sync();
      const float* vr = Vs + tid * LDV;
#pragma unroll 4
      for (int c = 0; c < BN; ++c) {
        sink.offer1(vr[c], col_base + c);
      }
    }
    __syncthreads();
  }
  if (scanner) sink.finish(p.sink);
}

template <class Sink>
void launch_simt_variant(const SimtParams& p, int grid, size_t smem, cudaStream_t st) {
  cudaFuncSetAttribute(screen_simt_kernel<Sink>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)smem);
  screen_simt_kernel<Sink><<<grid, kThreads, smem, st>>>(p);
}

}  // namespace

void launch_screen_simt(const Index* ix, const float* Q, int64_t m, int64_t m_pad,
                        int exclude_self, int64_t q_offset, int S, const float* E, int sink_kind,
                        const SinkArgs& sa, cudaStream_t st, const int* perm) {
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
  const size_t smem = (size_t)(4 * BK * LDA + BM * LDV) * sizeof(float);
  const int grid = m_tiles * S;
  if (grid <= 0) return;
  if (sink_kind == kSinkRadiusCount) return launch_simt_variant<RadiusCountSink>(p, grid, smem, st);
  if (sink_kind == kSinkRadiusFill) return launch_simt_variant<RadiusFillSink>(p, grid, smem, st);
  if (sa.k <= 16) return launch_simt_variant<KnnSink<16>>(p, grid, smem, st);
  if (sa.k <= 32) return launch_simt_variant<KnnSink<32>>(p, grid, smem, st);
  launch_simt_variant<KnnSink<64>>(p, grid, smem, st);
}

}  // namespace b2k
