// Band-limited DFT passes of the SOCS imaging and its adjoint (FP32 SIMT path).
//
// Every SOCS kernel H_k is supported on a band S of Nr x Nc integer
// frequencies. Then (exactly, in exact arithmetic)
//   E_k(x)   = sum_{v in S} H_k(v) m(v) e^{2 pi i v.x/N},  m = DFT_N(M)|_S / N^2
//   I(x)     = sum_k w'_k |E_k(x)|^2 = sum_{d in D} c(d) e^{2 pi i d.x/N},  D = S - S
// and c(d) is obtained exactly from a Pr x Pc grid (Pr >= 2Nr-1, Pc >= 2Nc-1):
//   e_k(j) = sum_v H_k(v) m(v) e^{2 pi i v.j/P},  c(d) = DFT_P(sum_k w'_k |e_k|^2)(d)/(Pr Pc).
// The adjoint of source/utils/gradient.cpp:34-109 becomes
//   g'(d)    = DFT_N(dL/dI)|_D / N^2,   gamma(j) = sum_{d in D} g'(d) e^{2 pi i d.j/P}
//   Z_k(u)   = DFT_P(e_k gamma)(u)/(Pr Pc) = sum_v H_k(v) m(v) g'(u - v)
//   X(u)     = scale sum_k w'_k conj(H_k(u)) Z_k(u),  grad(y) = Re sum_{u in S} X(u) e^{2 pi i u.y/N}.
// So the full-resolution work is two K-independent separable passes per
// direction: a tile analysis (row DFT of a 128 x 128 tile, then its column
// contraction, giving one band partial per tile) and a row synthesis GEMM with
// a fused elementwise epilogue. The K-dependent work lives on the small grid.
#include <cuda_runtime.h>

#include <type_traits>

#include <algorithm>

#include <cuda_bf16.h>

#include "device_common.cuh"
#include "tc_ptx.cuh"

namespace litho_b200 {

// ---------------------------------------------------------------- GEMM main loop
// acc[i][j] += sum_{k in [kbeg, kend)} A(m0 + ty*TM + i, k) * B[(n0 + tx + j*BNT) * ldb + k]
// with 256 threads (BMT x BNT), A produced by a functor (load4 of 4 consecutive k),
// shared tiles As[BK][BM + 4] (transposed, float4 reads) and Bs[BK][BN + 1].
template <int BMT, int BNT, int TM, int TN, int BK, class ALoad>
__device__ __forceinline__ void gemm_mainloop(ALoad& aload, const float* __restrict__ B, int ldb,
                                              int Nn, int m0, int n0, int kbeg, int kend,
                                              float* As, float* Bs, float (&acc)[TM][TN]) {
  constexpr int BM = BMT * TM, BN = BNT * TN, NT = BMT * BNT;
  constexpr int AS = BM + 4, BS = BN + 1;
  const int tid = threadIdx.x, tx = tid % BNT, ty = tid / BNT;
  for (int kt = kbeg; kt < kend; kt += BK) {
    for (int e = tid; e < BM * (BK / 4); e += NT) {
      const int mm = e / (BK / 4);
      const int kq = (e % (BK / 4)) * 4;
      float v[4];
      aload.load4(m0 + mm, kt + kq, kend, v);
#pragma unroll
      for (int q = 0; q < 4; ++q) As[(kq + q) * AS + mm] = v[q];
    }
    for (int e = tid; e < BN * BK; e += NT) {
      const int nn = e / BK, kk = e % BK;
      const int gn = n0 + nn, gk = kt + kk;
      Bs[kk * BS + nn] = (gn < Nn && gk < kend) ? __ldg(B + (size_t)gn * ldb + gk) : 0.f;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < BK; ++kk) {
      float a[TM];
#pragma unroll
      for (int i = 0; i < TM; i += 4) {
        const float4 t = *reinterpret_cast<const float4*>(&As[kk * AS + ty * TM + i]);
        a[i] = t.x; a[i + 1] = t.y; a[i + 2] = t.z; a[i + 3] = t.w;
      }
      float b[TN];
#pragma unroll
      for (int j = 0; j < TN; ++j) b[j] = Bs[kk * BS + tx + j * BNT];
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- tile analysis
// mode 0: A = in;  mode 1: A = (1 + cos(in))/2 (theta -> mask), optional mask_out.
// Non-finite inputs raise flag[0].
struct ImageLoad {
  const float* in;
  float* mask_out;
  int* flag;
  int N;
  int mode;
  int vec4;  // rows are 16-byte aligned (N % 4 == 0 and an aligned base pointer)
  __device__ __forceinline__ void load4(int m, int k, int kend, float* v) {
    if (vec4 && m < N && k + 3 < kend) {
      const float4 t = __ldg(reinterpret_cast<const float4*>(in + (size_t)m * N + k));
      v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else {
#pragma unroll
      for (int q = 0; q < 4; ++q)
        v[q] = (m < N && k + q < kend) ? __ldg(in + (size_t)m * N + k + q) : 0.f;
    }
    bool bad = false;
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (m < N && k + q < kend) bad |= !isfinite(v[q]);
    if (bad) atomicOr(flag, 1);
    if (mode == 1) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const bool in_range = m < N && k + q < kend;
        v[q] = in_range ? 0.5f * (1.f + cosf(v[q])) : 0.f;
        if (mask_out && in_range) mask_out[(size_t)m * N + k + q] = v[q];
      }
    }
  }
};

constexpr int AT_BMT = 16, AT_BNT = 16, AT_TM = 8, AT_BK = 32, AT_NT = 256;
constexpr int AT_TILE = AT_BMT * AT_TM;  // 128 rows, and 128 columns of x per tile
constexpr int AT_RC = 16;                // band rows staged per chunk in phase 2

struct AnalysisArgs {
  ImageLoad ld;
  const float* tw;     // [2 * ncols][N] real rows (Re, Im of the column twiddles)
  int N, ncols;
  const float2* TY;    // [nr][N] row twiddles
  int nrows_out, nr, sym;
  float2* part;        // [tiles][nrows_out][ncols]
};

template <int BN>
__device__ void analysis_phase2(float* smem, const AnalysisArgs& a, int y0, int f0, int tile);

template <int TN>
__global__ void __launch_bounds__(AT_NT)
analysis_tile_kernel(AnalysisArgs a) {
  extern __shared__ __align__(16) float smem[];
  constexpr int BN = AT_BNT * TN;   // real columns (2 per complex frequency)
  float* As = smem;
  float* Bs = smem + AT_BK * (AT_TILE + 4);
  const int tid = threadIdx.x, tx = tid % AT_BNT, ty = tid / AT_BNT;
  const int x0 = blockIdx.x * AT_TILE, y0 = blockIdx.y * AT_TILE;
  const int f0 = blockIdx.z * BN;
  const int Nn = 2 * a.ncols;
  ImageLoad ld = a.ld;
  pdl_trigger();
  pdl_wait();

  // Phase 1: R[y][f] = sum_{x in tile} A[y][x] tw[f][x]  (128 rows x BN real columns).
  float acc[AT_TM][TN];
#pragma unroll
  for (int i = 0; i < AT_TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = 0.f;
  gemm_mainloop<AT_BMT, AT_BNT, AT_TM, TN, AT_BK>(ld, a.tw, a.N, Nn, y0, f0, x0,
                                                  min(a.N, x0 + AT_TILE), As, Bs, acc);
  // Phase 2 input: R staged as [128][BN + 4] floats.
  constexpr int RS = BN + 4;
#pragma unroll
  for (int i = 0; i < AT_TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) smem[(ty * AT_TM + i) * RS + tx + j * AT_BNT] = acc[i][j];
  analysis_phase2<BN>(smem, a, y0, f0, blockIdx.y * gridDim.x + blockIdx.x);
}

// Phase 2 of a tile analysis: P[r][c] = sum_{y in tile} T(r, y) R[y][c] for the
// tile's rows, R given in smem as [128][BN + 4] floats (complex column c at
// floats 2c, 2c + 1), as a register-tiled complex product: each thread owns 2
// band rows x 2 columns. Every thread of the CTA (AT_NT) must call it; it
// begins with a barrier, so the caller's writes of R need no extra one.
template <int BN>
__device__ void analysis_phase2(float* smem, const AnalysisArgs& a, int y0, int f0, int tile) {
  constexpr int BNC = BN / 2;
  constexpr int RS = BN + 4;                         // keeps float4 alignment of R rows
  const float* Rs = smem;                            // [128][RS]
  float2* TYs = reinterpret_cast<float2*>(smem + AT_TILE * RS);  // [RC][128]
  const int tid = threadIdx.x;
  constexpr int CP = BNC / 2;                        // column pairs
  const int cp = tid % CP, rp = tid / CP;            // rows 2rp, 2rp+1 of each chunk
  const bool active = rp < AT_RC / 2;
  const int c0g = f0 / 2 + 2 * cp;                   // first of the two global columns
  for (int r0 = 0; r0 < a.nrows_out; r0 += AT_RC) {
    __syncthreads();
    for (int e = tid; e < AT_RC * AT_TILE; e += AT_NT) {
      const int r = e / AT_TILE, yy = e % AT_TILE;
      const int row = r0 + r, y = y0 + yy;
      float2 t = make_float2(0.f, 0.f);
      if (row < a.nrows_out && y < a.N) {
        if (!a.sym) {
          t = a.TY[(size_t)row * a.N + y];
        } else {
          const int d = row - (a.nr - 1);
          t = d >= 0 ? a.TY[(size_t)d * a.N + y] : conjf2(a.TY[(size_t)(-d) * a.N + y]);
        }
      }
      TYs[r * AT_TILE + yy] = t;
    }
    __syncthreads();
    if (active && r0 + 2 * rp < a.nrows_out) {
      float2 p00 = make_float2(0.f, 0.f), p01 = p00, p10 = p00, p11 = p00;
      const float2* t0 = TYs + (2 * rp) * AT_TILE;
      const float2* t1 = t0 + AT_TILE;
#pragma unroll 4
      for (int yy = 0; yy < AT_TILE; ++yy) {
        const float4 rv = *reinterpret_cast<const float4*>(&Rs[yy * RS + 4 * cp]);
        const float2 ra = make_float2(rv.x, rv.y), rb = make_float2(rv.z, rv.w);
        const float2 ta = t0[yy], tb = t1[yy];
        cfma(p00, ta, ra);
        cfma(p01, ta, rb);
        cfma(p10, tb, ra);
        cfma(p11, tb, rb);
      }
      const int row0 = r0 + 2 * rp;
      float2* out0 = a.part + ((size_t)tile * a.nrows_out + row0) * a.ncols;  // [tile][row][c]
      if (c0g < a.ncols) out0[c0g] = p00;
      if (c0g + 1 < a.ncols) out0[c0g + 1] = p01;
      if (row0 + 1 < a.nrows_out) {
        float2* out1 = out0 + a.ncols;
        if (c0g < a.ncols) out1[c0g] = p10;
        if (c0g + 1 < a.ncols) out1[c0g + 1] = p11;
      }
    }
  }
}

template <int TN>
static cudaError_t analysis_tile_t(cudaStream_t s, const AnalysisArgs& a) {
  constexpr int BN = AT_BNT * TN;
  const size_t p1 = (size_t)(AT_BK * (AT_TILE + 4) + AT_BK * (BN + 1)) * sizeof(float);
  const size_t p2 = (size_t)AT_TILE * (BN + 4) * sizeof(float) +
                    (size_t)AT_RC * AT_TILE * sizeof(float2);
  const size_t smem = p1 > p2 ? p1 : p2;
  cudaError_t e = cudaFuncSetAttribute(analysis_tile_kernel<TN>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int t = (a.N + AT_TILE - 1) / AT_TILE;
  dim3 grid(t, t, (2 * a.ncols + BN - 1) / BN);
  return launch_pdl(analysis_tile_kernel<TN>, grid, dim3(AT_NT), smem, s, a);
}

int analysis_tiles(int N) {
  const int t = (N + AT_TILE - 1) / AT_TILE;
  return t * t;
}

// Tile partials of sum_{y, x} T(a, y) A[y][x] tw(c, x) for every 128 x 128 tile:
// part[tile][a][c], tiles in row-major order of the tile grid (each tile's partials
// contiguous, so that the tensor-core epilogue writes them as one coalesced block).
cudaError_t launch_analysis(cudaStream_t s, int mode, const float* in, float* mask_out,
                            int* flag, const float* tw, int N, int ncols, const float2* TY,
                            int nrows_out, int nr, int sym, float2* part) {
  const int vec4 = (N % 4 == 0) && (reinterpret_cast<uintptr_t>(in) % 16 == 0);
  AnalysisArgs a{ImageLoad{in, mask_out, flag, N, mode, vec4}, tw, N, ncols, TY, nrows_out,
                 nr, sym, part};
  const int n2 = 2 * ncols;
  if (n2 <= 32) return analysis_tile_t<2>(s, a);
  if (n2 <= 48) return analysis_tile_t<3>(s, a);
  if (n2 <= 64) return analysis_tile_t<4>(s, a);
  if (n2 <= 80) return analysis_tile_t<5>(s, a);
  if (n2 <= 96) return analysis_tile_t<6>(s, a);
  return analysis_tile_t<8>(s, a);
}

// out[o] = scale * sum_t part[t][o] in a fixed order: RT_G tile groups (group g sums
// tiles g, g + RT_G, ... in turn), then a fixed tree over the groups. A CTA covers
// RT_E consecutive entries, so each group's loads are coalesced.
constexpr int RT_E = 16, RT_G = 32;
__global__ void __launch_bounds__(RT_E * RT_G)
reduce_tiles_kernel(const float2* __restrict__ part, int tiles, int count, int trows,
                    float scale, float2* __restrict__ out) {
  pdl_trigger();
  pdl_wait();
  part += (size_t)blockIdx.y * tiles * count;   // image b of a batch: [b][tile][entry]
  out += (size_t)blockIdx.y * count;
  __shared__ float2 sh[RT_G][RT_E];
  const int e = threadIdx.x % RT_E, g = threadIdx.x / RT_E;
  const int o = blockIdx.x * RT_E + e;
  float2 v = make_float2(0.f, 0.f);
  if (o < count) {
#pragma unroll 8
    for (int t = g; t < tiles; t += RT_G) {
      const float2 p = __ldg(part + (size_t)t * count + o);
      v.x += p.x;
      v.y += p.y;
    }
  }
  sh[g][e] = v;
  __syncthreads();
#pragma unroll
  for (int h = RT_G / 2; h > 0; h >>= 1) {
    if (g < h) {
      sh[g][e].x += sh[g + h][e].x;
      sh[g][e].y += sh[g + h][e].y;
    }
    __syncthreads();
  }
  // Entry o of a tile block is (row, c) = (o / ncols, o % ncols), or with trows > 0
  // (column-major blocks of trows rows) (o % trows, o / trows); out is row-major.
  const int oo = trows > 0 ? (o % trows) * (count / trows) + o / trows : o;
  if (g == 0 && o < count) out[oo] = make_float2(sh[0][e].x * scale, sh[0][e].y * scale);
}

cudaError_t launch_reduce_tiles(cudaStream_t s, const float2* part, int tiles, int count,
                                float scale, float2* out, int batch, int trows) {
  return launch_pdl(reduce_tiles_kernel, dim3((count + RT_E - 1) / RT_E, batch),
                    dim3(RT_E * RT_G), 0, s, part, tiles, count, trows, scale, out);
}

// ---------------------------------------------------------------- row synthesis
// out[y][x] = sum_f AY[y][f] * Bt[x][f] (K = kp) with the epilogue applied to the
// tile through shared memory in two halves, so that every global access of the
// epilogue is a coalesced float4 (or scalar at ragged edges).
struct AYLoad {
  const float* AY;
  int N, kp;
  __device__ __forceinline__ void load4(int m, int k, int kend, float* v) {
    if (m < N && k + 3 < kend) {
      const float4 t = __ldg(reinterpret_cast<const float4*>(AY + (size_t)m * kp + k));
      v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else {
#pragma unroll
      for (int q = 0; q < 4; ++q) v[q] = (m < N && k + q < kend) ? AY[(size_t)m * kp + k + q] : 0.f;
    }
  }
};

constexpr int SY_BMT = 16, SY_BNT = 16, SY_TM = 8, SY_TN = 8, SY_BK = 16;
constexpr int SY_NT = SY_BMT * SY_BNT;
constexpr int SY_TILE = 128;
constexpr int SY_SS = SY_TILE + 4;  // staging row stride

template <class Epi>
__global__ void __launch_bounds__(SY_NT)
synth_kernel(const float* __restrict__ AY, const float* __restrict__ Bt, int N, int kp, Epi epi) {
  __shared__ __align__(16) float As[SY_BK * (SY_TILE + 4)];
  __shared__ float Bs[SY_BK * (SY_TILE + 1)];
  extern __shared__ __align__(16) float stage[];  // [64][SY_SS]
  const int tid = threadIdx.x, tx = tid % SY_BNT, ty = tid / SY_BNT;
  const int m0 = blockIdx.y * SY_TILE, n0 = blockIdx.x * SY_TILE;
  pdl_trigger();
  pdl_wait();
  float acc[SY_TM][SY_TN];
#pragma unroll
  for (int i = 0; i < SY_TM; ++i)
#pragma unroll
    for (int j = 0; j < SY_TN; ++j) acc[i][j] = 0.f;
  AYLoad ld{AY, N, kp};
  gemm_mainloop<SY_BMT, SY_BNT, SY_TM, SY_TN, SY_BK>(ld, Bt, kp, N, m0, n0, 0, kp, As, Bs, acc);
  for (int h = 0; h < 2; ++h) {
    __syncthreads();
    if (ty / 8 == h) {
#pragma unroll
      for (int i = 0; i < SY_TM; ++i)
#pragma unroll
        for (int j = 0; j < SY_TN; ++j)
          stage[(ty * SY_TM + i - 64 * h) * SY_SS + tx + j * SY_BNT] = acc[i][j];
    }
    __syncthreads();
    for (int e = tid; e < 64 * (SY_TILE / 4); e += SY_NT) {
      const int r = e / (SY_TILE / 4), c4 = (e % (SY_TILE / 4)) * 4;
      const int m = m0 + 64 * h + r, n = n0 + c4;
      if (m >= N || n >= N) continue;
      const float4 v = *reinterpret_cast<const float4*>(&stage[r * SY_SS + c4]);
      epi.store4(m, n, v, min(4, N - n));
    }
  }
  epi.finish();
}

static dim3 synth_grid(int N) {
  const int t = (N + SY_TILE - 1) / SY_TILE;
  return dim3(t, t, 1);
}

template <class Epi>
static cudaError_t launch_synth(cudaStream_t s, const float* AY, const float* Bt, int N, int kp,
                                const Epi& e) {
  const int smem = 64 * SY_SS * sizeof(float);
  cudaError_t err = cudaFuncSetAttribute(synth_kernel<Epi>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (err != cudaSuccess) return err;
  return launch_pdl(synth_kernel<Epi>, synth_grid(N), dim3(SY_NT), smem, s, AY, Bt, N, kp, e);
}


cudaError_t launch_synth_resist(cudaStream_t s, const float* AY, const float* Bt, int N, int kp,
                                const ResistEpilogue& ep, int* nblocks) {
  const dim3 grid = synth_grid(N);
  *nblocks = grid.x * grid.y;
  const int vec = N % 4 == 0 && aligned16(ep.aerial) && aligned16(ep.wafer) &&
                  aligned16(ep.target) && aligned16(ep.pe_window) && aligned16(ep.pen_window) &&
                  aligned16(ep.dldi);
  return launch_synth(s, AY, Bt, N, kp, ResistEpi{ep, N, vec, 0.0, 0.0});
}

cudaError_t launch_synth_grad(cudaStream_t s, const float* AY, const float* Bt, int N, int kp,
                              const GradEpilogue& ep, int* nblocks) {
  const dim3 grid = synth_grid(N);
  *nblocks = grid.x * grid.y;
  const int vec = N % 4 == 0 && aligned16(ep.grad_mask) && aligned16(ep.theta) &&
                  aligned16(ep.grad_theta);
  return launch_synth(s, AY, Bt, N, kp, GradEpi{ep, N, vec, 0.0});
}

// ---------------------------------------------------------------- small-grid band stage
// Small tables (a few tens of KB for a 35 x 35 band) are staged in shared
// memory when they fit in SMEM_STAGE bytes; otherwise the kernels read them
// from global memory (L2-resident), with the same arithmetic.
constexpr size_t SMEM_STAGE = 200 * 1024;

// dst[i] = load(i) for i < n, the NT threads of the CTA striding through i: every
// thread issues B loads before its B shared-memory stores, so the global (L2)
// latencies of a staging pass overlap instead of adding up.
template <int NT, int B = 8, class T, class Load>
__device__ __forceinline__ void fill_batched(T* dst, int n, Load load) {
  for (int base = threadIdx.x; base < n; base += NT * B) {
    T v[B];
#pragma unroll
    for (int q = 0; q < B; ++q) {
      const int i = base + q * NT;
      if (i < n) v[q] = load(i);
    }
#pragma unroll
    for (int q = 0; q < B; ++q) {
      const int i = base + q * NT;
      if (i < n) dst[i] = v[q];
    }
  }
}

// Forward 1: grid (K, column chunks of W, batch). CTA (k, q) owns small-grid
// columns jc in [q W, q W + W): A = H_k m on the band, T = A ESc^T restricted to
// those columns (Nr x W) and e_k = ESr T (Pr x W); ik = w_k |e_k|^2. Columns are
// independent, so the split costs no recomputation. Every thread accumulates four
// adjacent columns, so one row operand from shared memory feeds four complex FMAs.
constexpr int BF_NT = 512;   // threads of the fields and Z kernels (more loads in flight while staging)
constexpr int BW_ONE = 8, BW_BATCH = 16;   // chunk widths (multiples of 4): one image, a batch
__host__ __device__ constexpr int even_up(int n) { return (n + 1) & ~1; }
__device__ __forceinline__ void cfma4(float2 (&acc)[4], float2 a, const float2* b4) {
  const float4 b01 = *reinterpret_cast<const float4*>(b4);
  const float4 b23 = *reinterpret_cast<const float4*>(b4 + 2);
  cfma(acc[0], a, make_float2(b01.x, b01.y));
  cfma(acc[1], a, make_float2(b01.z, b01.w));
  cfma(acc[2], a, make_float2(b23.x, b23.y));
  cfma(acc[3], a, make_float2(b23.z, b23.w));
}

// The small-grid tables are zero-padded DFTs of even length P = 2 n: for band frequency
// f, ES[f][j + n] = (-1)^f ES[f][j]. A transform over the P outputs folds into n:
// out[j] = Ev[j] + Od[j] and out[j + n] = Ev[j] - Od[j], Ev and Od the sums over the
// frequencies of even and odd f (each in increasing order), and a transform over the
// P inputs into n: out = sum_{j < n} ES[f][j] (in[j] + (-1)^f in[j + n]). Every kernel
// of a stage folds the same way with the same operation order, so chunked, whole-grid,
// batched and single-image launches stay bit-identical.
__device__ __forceinline__ float2 fold_sum(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 fold_diff(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

template <int W>
__global__ void __launch_bounds__(BF_NT)
band_fields_kernel(const float2* __restrict__ H, const float2* __restrict__ mband,
                   const float* __restrict__ w, int Nr, int Nc, int Pr, int Pc, int row0,
                   const float2* __restrict__ ESc_t, const float2* __restrict__ ESr_t,
                   int stage_tables, float2* __restrict__ e, float* __restrict__ ik) {
  static_assert(W % 4 == 0, "four columns per thread");
  constexpr int JB = W / 4;
  extern __shared__ __align__(16) float2 sm2[];
  const int k = blockIdx.x;
  const int j0 = blockIdx.y * W;
  const int cw = min(W, Pc - j0);
  {  // image b of a batch
    const size_t b = blockIdx.z;
    mband += b * Nr * Nc;
    e += b * gridDim.x * Pr * Pc;
    ik += b * gridDim.x * Pr * Pc;
  }
  float2* A = sm2;                      // [Nr][Nc]
  float2* T = A + even_up(Nr * Nc);     // [Nr][W]
  float2* esc = T + Nr * W;             // [Nc][W] (columns past cw are zero)
  float2* esr = esc + Nc * W;           // [Nr][Pr] (staged when stage_tables)
  pdl_trigger();
  fill_batched<BF_NT>(esc, Nc * W, [&](int i) {
    const int c = i / W, jj = i % W;
    return jj < cw ? ESc_t[(size_t)c * Pc + j0 + jj] : make_float2(0.f, 0.f);
  });
  const float2* ESR = ESr_t;
  if (stage_tables) {
    fill_batched<BF_NT>(esr, Nr * Pr, [&](int i) { return ESr_t[i]; });
    ESR = esr;
  }
  pdl_wait();
  fill_batched<BF_NT>(A, Nr * Nc, [&](int i) { return cmul(H[(size_t)k * Nr * Nc + i], mband[i]); });
  __syncthreads();
  for (int it = threadIdx.x; it < Nr * JB; it += BF_NT) {
    const int r = it / JB, jb = 4 * (it % JB);
    float2 acc[4] = {};
    for (int c = 0; c < Nc; ++c) cfma4(acc, A[r * Nc + c], esc + c * W + jb);
    *reinterpret_cast<float4*>(T + r * W + jb) = make_float4(acc[0].x, acc[0].y, acc[1].x, acc[1].y);
    *reinterpret_cast<float4*>(T + r * W + jb + 2) =
        make_float4(acc[2].x, acc[2].y, acc[3].x, acc[3].y);
  }
  __syncthreads();
  const float wk = w[k];
  // e_k rows jr and jr + Nr from the two parity classes of the band rows (fold_rows).
  const int r_even = row0 & 1;   // first r with row0 + r even
  for (int it = threadIdx.x; it < Nr * JB; it += BF_NT) {
    const int jr = it / JB, jb = 4 * (it % JB);
    float2 ev[4] = {}, od[4] = {};
    for (int r = r_even; r < Nr; r += 2) cfma4(ev, ESR[r * Pr + jr], T + r * W + jb);
    for (int r = 1 - r_even; r < Nr; r += 2) cfma4(od, ESR[r * Pr + jr], T + r * W + jb);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (jb + q >= cw) break;
      const float2 v[2] = {fold_sum(ev[q], od[q]), fold_diff(ev[q], od[q])};
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const size_t o = ((size_t)k * Pr + jr + h * Nr) * Pc + j0 + jb + q;
        e[o] = v[h];
        ik[o] = wk * (v[h].x * v[h].x + v[h].y * v[h].y);
      }
    }
  }
}

// C = A B over operands in shared memory: each thread owns an RT x 2 block of C (rows
// m0 .. m0 + RT - 1, columns 2p and 2p + 1) and adds the terms in k order with cfma,
// the operand order and summation order of the chunked kernels, so every element is
// bit-identical to theirs. Work items run pair-fastest: a warp's B loads are adjacent
// 16-byte words and its A loads mostly one broadcast address. a(m, k) returns A[m][k];
// B[k][n] is at B + k ldb + n (ldb even, B 16-byte aligned).
template <int RT, int NT, class ALoad, class Store>
__device__ __forceinline__ void cgemm_rt2(int M, int npairs, int Kd, ALoad a,
                                          const float2* __restrict__ B, int ldb, Store store) {
  const int rblocks = (M + RT - 1) / RT;
  for (int it = threadIdx.x; it < rblocks * npairs; it += NT) {
    const int m0 = (it / npairs) * RT, p = it % npairs;
    float2 acc[RT][2];
#pragma unroll
    for (int i = 0; i < RT; ++i) acc[i][0] = acc[i][1] = make_float2(0.f, 0.f);
    for (int k = 0; k < Kd; ++k) {
      const float4 b = *reinterpret_cast<const float4*>(B + (size_t)k * ldb + 2 * p);
      const float2 b0 = make_float2(b.x, b.y), b1 = make_float2(b.z, b.w);
#pragma unroll
      for (int i = 0; i < RT; ++i) {
        const float2 av = a(min(m0 + i, M - 1), k);
        cfma(acc[i][0], av, b0);
        cfma(acc[i][1], av, b1);
      }
    }
#pragma unroll
    for (int i = 0; i < RT; ++i) {
      if (m0 + i < M) {
        store(m0 + i, 2 * p, acc[i][0]);
        store(m0 + i, 2 * p + 1, acc[i][1]);
      }
    }
  }
}

// C = A B folded over the output rows (the transform over P = 2 M outputs): output rows
// m and m + M of each column pair from Ev = sum over k of the parity class k0, k0 + 2,
// ... and Od = sum over the other class, each in increasing k with cfma, stored as
// Ev + Od (row m) and Ev - Od (row m + M). Each thread owns RT rows x 2 columns.
template <int RT, int NT, class ALoad, class Store>
__device__ __forceinline__ void fold_rows(int M, int npairs, int Kd, int k0, ALoad a,
                                          const float2* __restrict__ B, int ldb, Store store) {
  const int rblocks = (M + RT - 1) / RT;
  for (int it = threadIdx.x; it < rblocks * npairs; it += NT) {
    const int m0 = (it / npairs) * RT, p = it % npairs;
    float2 ev[RT][2], od[RT][2];
#pragma unroll
    for (int i = 0; i < RT; ++i) ev[i][0] = ev[i][1] = od[i][0] = od[i][1] = make_float2(0.f, 0.f);
    for (int k = k0; k < Kd; k += 2) {
      const float4 b = *reinterpret_cast<const float4*>(B + (size_t)k * ldb + 2 * p);
      const float2 b0 = make_float2(b.x, b.y), b1 = make_float2(b.z, b.w);
#pragma unroll
      for (int i = 0; i < RT; ++i) {
        const float2 av = a(min(m0 + i, M - 1), k);
        cfma(ev[i][0], av, b0);
        cfma(ev[i][1], av, b1);
      }
    }
    for (int k = 1 - k0; k < Kd; k += 2) {
      const float4 b = *reinterpret_cast<const float4*>(B + (size_t)k * ldb + 2 * p);
      const float2 b0 = make_float2(b.x, b.y), b1 = make_float2(b.z, b.w);
#pragma unroll
      for (int i = 0; i < RT; ++i) {
        const float2 av = a(min(m0 + i, M - 1), k);
        cfma(od[i][0], av, b0);
        cfma(od[i][1], av, b1);
      }
    }
#pragma unroll
    for (int i = 0; i < RT; ++i) {
      if (m0 + i < M) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          store(m0 + i, 2 * p + h, fold_sum(ev[i][h], od[i][h]));
          store(m0 + i + M, 2 * p + h, fold_diff(ev[i][h], od[i][h]));
        }
      }
    }
  }
}

// Forward 1, whole small grid per CTA: grid (K, 1, batch), CTA (k, b) computes all of
// e_k = ESr (A ESc^T) (Pr x Pc) and ik = w_k |e_k|^2 for image b, every table staged
// once per CTA instead of once per column chunk. Same arithmetic as
// band_fields_kernel (bit-identical results), register-blocked: 5 rows x 2 columns of
// T and, folded over the row parity classes, 5 row pairs (jr, jr + Nr) x 2 columns of
// e_k per thread.
constexpr int BG_NT = 256;
__global__ void __launch_bounds__(BG_NT)
band_fields_whole_kernel(const float2* __restrict__ H, const float2* __restrict__ mband,
                         const float* __restrict__ w, int Nr, int Nc, int Pr, int Pc, int row0,
                         const float2* __restrict__ ESc_t, const float2* __restrict__ ESr_t,
                         float2* __restrict__ e, float* __restrict__ ik) {
  extern __shared__ __align__(16) float2 sm2[];
  const int k = blockIdx.x;
  {  // image b of a batch
    const size_t b = blockIdx.z;
    mband += b * Nr * Nc;
    e += b * gridDim.x * Pr * Pc;
    ik += b * gridDim.x * Pr * Pc;
  }
  float2* esc = sm2;                    // [Nc][Pc]
  float2* esr = esc + Nc * Pc;          // [Nr][Pr]
  float2* T = esr + Nr * Pr;            // [Nr][Pc]
  float2* A = T + Nr * Pc;              // [Nr][Nc]
  pdl_trigger();
  fill_batched<BG_NT>(esc, Nc * Pc, [&](int i) { return ESc_t[i]; });
  fill_batched<BG_NT>(esr, Nr * Pr, [&](int i) { return ESr_t[i]; });
  pdl_wait();
  fill_batched<BG_NT>(A, Nr * Nc, [&](int i) { return cmul(H[(size_t)k * Nr * Nc + i], mband[i]); });
  __syncthreads();
  cgemm_rt2<5, BG_NT>(Nr, Pc / 2, Nc, [&](int r, int c) { return A[r * Nc + c]; }, esc, Pc,
                      [&](int r, int j, float2 v) { T[r * Pc + j] = v; });
  __syncthreads();
  const float wk = w[k];
  float2* ek = e + (size_t)k * Pr * Pc;
  float* ikk = ik + (size_t)k * Pr * Pc;
  fold_rows<5, BG_NT>(Nr, Pc / 2, Nr, row0 & 1, [&](int jr, int r) { return esr[r * Pr + jr]; }, T,
                      Pc, [&](int jr, int j, float2 v) {
                        const size_t o = (size_t)jr * Pc + j;
                        ek[o] = v;
                        ikk[o] = wk * (v.x * v.x + v.y * v.y);
                      });
}

static size_t fields_whole_smem(const BandGeom& g) {
  return (size_t)(g.Nc * g.Pc + g.Nr * g.Pr + g.Nr * g.Pc + g.Nr * g.Nc) * sizeof(float2);
}

template <int W>
static size_t fields_smem(const BandGeom& g, bool staged) {
  return (size_t)(even_up(g.Nr * g.Nc) + g.Nr * W + g.Nc * W + (staged ? g.Nr * g.Pr : 0)) *
         sizeof(float2);
}
size_t band_fields_smem(const BandGeom& g) {
  return fields_smem<(BW_ONE > BW_BATCH ? BW_ONE : BW_BATCH)>(g, false);
}

// Forward 2: i[j] = sum_k ik[k][j] in k order.
__global__ void sum_k_kernel(const float* __restrict__ ik, int K, int n, float* __restrict__ iP) {
  pdl_trigger();
  pdl_wait();
  ik += (size_t)blockIdx.y * K * n;   // image b of a batch
  iP += (size_t)blockIdx.y * n;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  float s = 0.f;
  for (int k = 0; k < K; ++k) s += ik[(size_t)k * n + j];
  iP[j] = s;
}

// Sum of a value over SPLIT adjacent lanes (a power of two dividing 32), added in a
// fixed order ((0 + 1) + (2 + 3) for 4); every lane of the warp must call it.
template <int SPLIT>
__device__ __forceinline__ float2 split_sum(float2 a) {
#pragma unroll
  for (int o = 1; o < SPLIT; o <<= 1) {
    a.x += __shfl_xor_sync(0xffffffffu, a.x, o);
    a.y += __shfl_xor_sync(0xffffffffu, a.y, o);
  }
  return a;
}

// Forward 3 (one CTA per band row dr >= 0): chat[dr][dc] = DFT_P(i)(dr, dc) / (Pr Pc)
// for dc in [-(Nc-1), Nc-1].
constexpr int BI_NT = 256;
__global__ void __launch_bounds__(BI_NT)
band_chat_kernel(const float* __restrict__ iP, int Nr, int Nc, int Pr, int Pc,
                 const float2* __restrict__ EDr_t, const float2* __restrict__ EDc, float inv,
                 float2* __restrict__ chat) {
  // Operands are staged with one parallel round trip; the products then run
  // from shared memory (the L2 latency chains of a per-thread loop dominated).
  extern __shared__ float2 sb[];
  const int nd = 2 * Nc - 1;
  float2* v = sb;                                    // [Pc]
  float2* ed = v + Pc;                               // [Pr]
  float2* edc = ed + Pr;                             // [Pc][nd]
  float* ip = reinterpret_cast<float*>(edc + Pc * nd);  // [Pr][Pc]
  const int dr = blockIdx.x;
  iP += (size_t)blockIdx.y * Pr * Pc;   // image b of a batch
  chat += (size_t)blockIdx.y * Nr * nd;
  pdl_trigger();
  fill_batched<BI_NT>(ed, Pr, [&](int jr) { return EDr_t[(size_t)(dr + Nr - 1) * Pr + jr]; });
  fill_batched<BI_NT>(edc, Pc * nd, [&](int i) { return EDc[i]; });
  pdl_wait();
  fill_batched<BI_NT>(ip, Pr * Pc, [&](int i) { return iP[i]; });
  __syncthreads();
  // Each output is summed by SPLIT adjacent lanes (terms sub, sub + SPLIT, ...), their
  // partial sums then added in a fixed order; whole warps iterate together.
  constexpr int SPLIT = 4, GROUPS = BI_NT / SPLIT;
  const int sub = threadIdx.x % SPLIT, grp = threadIdx.x / SPLIT;
  for (int base = 0; base < Pc; base += GROUPS) {
    const int jc = base + grp;
    float2 a = make_float2(0.f, 0.f);
    if (jc < Pc)
      for (int jr = sub; jr < Pr; jr += SPLIT) {
        const float i0 = ip[jr * Pc + jc];
        a.x = fmaf(ed[jr].x, i0, a.x); a.y = fmaf(-ed[jr].y, i0, a.y);
      }
    a = split_sum<SPLIT>(a);
    if (jc < Pc && sub == 0) v[jc] = a;
  }
  __syncthreads();
  for (int base = 0; base < nd; base += GROUPS) {
    const int dc = base + grp;
    float2 a = make_float2(0.f, 0.f);
    if (dc < nd)
      for (int jc = sub; jc < Pc; jc += SPLIT) cfma(a, v[jc], conjf2(edc[jc * nd + dc]));
    a = split_sum<SPLIT>(a);
    if (dc < nd && sub == 0) chat[(size_t)dr * nd + dc] = make_float2(a.x * inv, a.y * inv);
  }
}

// Four interleaved partial sums added as (0 + 1) + (2 + 3): the order split_sum<4>
// gives the lane sums of the per-row kernels.
__device__ __forceinline__ float2 sum4(const float2 (&a)[4]) {
  return make_float2((a[0].x + a[1].x) + (a[2].x + a[3].x), (a[0].y + a[1].y) + (a[2].y + a[3].y));
}

// Forward 3 with BC_DR band rows per CTA: grid (ceil(Nr / BC_DR), batch). The tables and
// the image's small-grid intensity are staged once per BC_DR rows instead of once per
// row; one thread per pair of outputs keeps the four interleaved partial sums of
// band_chat_kernel and adds them in its order, so the results are bit-identical.
constexpr int BC_DR = 5;
__global__ void __launch_bounds__(256)
band_chat_rows_kernel(const float* __restrict__ iP, int Nr, int Nc, int Pr, int Pc,
                      const float2* __restrict__ EDr_t, const float2* __restrict__ EDc, float inv,
                      float2* __restrict__ chat) {
  extern __shared__ __align__(16) float2 sb[];
  const int nd = 2 * Nc - 1, ndE = even_up(nd);
  const int dr0 = blockIdx.x * BC_DR, nr = min(BC_DR, Nr - dr0);
  iP += (size_t)blockIdx.y * Pr * Pc;   // image b of a batch
  chat += (size_t)blockIdx.y * Nr * nd;
  float2* edc = sb;                                    // [Pc][ndE] (column nd zero)
  float2* ed = edc + Pc * ndE;                         // [BC_DR][Pr]
  float2* V = ed + BC_DR * Pr;                         // [BC_DR][Pc]
  float* ip = reinterpret_cast<float*>(V + BC_DR * Pc);  // [Pr][Pc]
  pdl_trigger();
  fill_batched<256>(ed, nr * Pr, [&](int i) {
    return EDr_t[(size_t)(dr0 + i / Pr + Nr - 1) * Pr + i % Pr];
  });
  fill_batched<256>(edc, Pc * ndE, [&](int i) {
    const int jc = i / ndE, dc = i % ndE;
    return dc < nd ? EDc[(size_t)jc * nd + dc] : make_float2(0.f, 0.f);
  });
  pdl_wait();
  fill_batched<256>(ip, Pr * Pc, [&](int i) { return iP[i]; });
  __syncthreads();
  // V[r][jc] = sum_jr conj(ed[r][jr]) ip[jr][jc], two columns per thread.
  const int pc2 = Pc / 2;
  for (int it = threadIdx.x; it < nr * pc2; it += 256) {
    const int r = it / pc2, jc = 2 * (it % pc2);
    float2 a0[4], a1[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) a0[s] = a1[s] = make_float2(0.f, 0.f);
    for (int jr0 = 0; jr0 < Pr; jr0 += 4) {
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int jr = jr0 + s;
        if (jr < Pr) {
          const float2 e = ed[r * Pr + jr];
          const float2 i2 = *reinterpret_cast<const float2*>(ip + jr * Pc + jc);
          a0[s].x = fmaf(e.x, i2.x, a0[s].x); a0[s].y = fmaf(-e.y, i2.x, a0[s].y);
          a1[s].x = fmaf(e.x, i2.y, a1[s].x); a1[s].y = fmaf(-e.y, i2.y, a1[s].y);
        }
      }
    }
    V[r * Pc + jc] = sum4(a0);
    V[r * Pc + jc + 1] = sum4(a1);
  }
  __syncthreads();
  // chat[dr][dc] = inv sum_jc V[r][jc] conj(EDc[jc][dc]), two outputs per thread.
  const int nd2 = ndE / 2;
  for (int it = threadIdx.x; it < nr * nd2; it += 256) {
    const int r = it / nd2, dc = 2 * (it % nd2);
    float2 a0[4], a1[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) a0[s] = a1[s] = make_float2(0.f, 0.f);
    for (int jc0 = 0; jc0 < Pc; jc0 += 4) {
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int jc = jc0 + s;
        if (jc < Pc) {
          const float2 v = V[r * Pc + jc];
          const float4 t = *reinterpret_cast<const float4*>(edc + jc * ndE + dc);
          cfma(a0[s], v, make_float2(t.x, -t.y));
          cfma(a1[s], v, make_float2(t.z, -t.w));
        }
      }
    }
    const float2 c0 = sum4(a0), c1 = sum4(a1);
    float2* out = chat + (size_t)(dr0 + r) * nd;
    out[dc] = make_float2(c0.x * inv, c0.y * inv);
    if (dc + 1 < nd) out[dc + 1] = make_float2(c1.x * inv, c1.y * inv);
  }
}

static size_t chat_rows_smem(const BandGeom& g) {
  const int ndE = even_up(2 * g.Nc - 1);
  return (size_t)(g.Pc * ndE + BC_DR * g.Pr + BC_DR * g.Pc) * sizeof(float2) +
         (size_t)g.Pr * g.Pc * sizeof(float);
}

static size_t chat_smem(const BandGeom& g) {
  const int nd = 2 * g.Nc - 1;
  return (size_t)(g.Pc + g.Pr + g.Pc * nd) * sizeof(float2) + (size_t)g.Pr * g.Pc * sizeof(float);
}

// Band -> image columns: Ut[x][2a + {0,1}] = kappa(a) sum_c coef[a][c] phase(c, x) for
// a 64-column x strip and 8 band rows per CTA (coefficients and phases staged).
// mode 0 (band S): phase = conj(TX[c][x]) (TX = e^{-2 pi i s_c x/N}), kappa = 1.
// mode 1 (difference set D, c in [0, 2nc-1), d = c - (nc-1)):
//   phase = d >= 0 ? conj(TX[d][x]) : TX[-d][x], kappa(a) = a > 0 ? 2 : 1 (Hermitian half).
// Columns 2*nrows .. kp-1 of Ut are zero.
// With img set (tensor-core path) the result goes
// straight into the split-BF16 operand image of the row synthesis instead of Ut:
// x tile x / 128 at img + (x / 128) * img_tile_bytes, hi of column f at
// sw128_offset(128, x % 128, f) and lo at sw128_offset(128, x % 128, kp + f).
//
// Both modes are summed over the nph = nc phase rows T_j = TX[j][x] = (t, u) as
// sum_j S_j t + D_j u. For a coefficient A of phase conj(T_j) and B of phase T_j,
// A conj(T_j) + B T_j = (A + B) t + (A.y - B.y, B.x - A.x) u, so
//   S_j = A + B, D_j = (A.y - B.y, B.x - A.x),
// with A = coef[a][j], B = 0 in mode 0 and A = coef[a][nc-1+j], B = coef[a][nc-1-j]
// (B = 0 for j = 0) in mode 1: each conjugate pair of the difference set costs one
// complex-by-real product pair instead of two complex products. Every output adds
// its terms in j order as fma(D, u, fma(S, t, acc)) per component, in every kernel
// below, so the batched and per-image expansions give bit-identical results.
constexpr int EX_X = 64, EX_NT = 256;

// S_j and D_j of band row coef_row for phase row j, as (S.x, S.y, D.x, D.y).
__device__ __forceinline__ float4 expand_sd(const float2* __restrict__ coef_row, int mode, int nc,
                                            int j) {
  const float2 A = coef_row[mode ? nc - 1 + j : j];
  const float2 B = (mode && j > 0) ? coef_row[nc - 1 - j] : make_float2(0.f, 0.f);
  return make_float4(A.x + B.x, A.y + B.y, A.y - B.y, B.x - A.x);
}
// acc + S t + D u, lane by lane fma(D, u, fma(S, t, acc)) (packed FP32x2, the
// rounding of two scalar fmaf per lane).
__device__ __forceinline__ float2 sd_fma(float2 acc, float4 sd, float t, float u) {
  return __ffma2_rn(make_float2(sd.z, sd.w), make_float2(u, u),
                    __ffma2_rn(make_float2(sd.x, sd.y), make_float2(t, t), acc));
}
// Phase rows of an expansion: nc for the difference set, ncoef for the band S.
__host__ __device__ __forceinline__ int expand_nph(int mode, int ncoef, int nc) {
  return mode ? nc : ncoef;
}

// The accumulation and store of the expansion for one CTA of 8 PAIRS band rows, from
// its staged coefficient pairs sd [8 PAIRS][nph] and phases ph [nph][EX_X]. Each
// output is summed over j in order whatever PAIRS is.
template <int PAIRS>
__device__ __forceinline__ void expand_store(const float4* sd, const float2* ph, int nrows,
                                             int nph, int N, int mode, int kp, int a0, int x0,
                                             float* __restrict__ Ut, uint8_t* __restrict__ img,
                                             uint32_t img_tile_bytes) {
  // Thread (xx, rq): row pairs p of rows a0 + 2 (PAIRS rq + p) + {0, 1}, each pair the
  // four consecutive output columns f0 .. f0 + 3 of image row x, written as one 8- or
  // 16-byte store.
  constexpr int R = 8 * PAIRS;
  const int xx = threadIdx.x % EX_X, rq = threadIdx.x / EX_X;
  const int x = x0 + xx;
  float2 acc[2 * PAIRS];
#pragma unroll
  for (int i = 0; i < 2 * PAIRS; ++i) acc[i] = make_float2(0.f, 0.f);
  for (int j = 0; j < nph; ++j) {
    const float2 p = ph[j * EX_X + xx];
#pragma unroll
    for (int i = 0; i < 2 * PAIRS; ++i) acc[i] = sd_fma(acc[i], sd[(2 * PAIRS * rq + i) * nph + j], p.x, p.y);
  }
  if (x >= N) return;
#pragma unroll
  for (int q = 0; q < PAIRS; ++q) {
    const int ra = a0 + 2 * (PAIRS * rq + q), rb = ra + 1;
    const float ka = ra < nrows ? ((mode == 1 && ra > 0) ? 2.f : 1.f) : 0.f;
    const float kb = rb < nrows ? ((mode == 1 && rb > 0) ? 2.f : 1.f) : 0.f;
    const float4 v = make_float4(ka * acc[2 * q].x, ka * acc[2 * q].y, kb * acc[2 * q + 1].x,
                                 kb * acc[2 * q + 1].y);
    const int f0 = 2 * ra;
    if (f0 >= kp) continue;
    if (img) {
      uint8_t* tile = img + (size_t)(x / 128) * img_tile_bytes;
      const __nv_bfloat162 h01 = __floats2bfloat162_rn(v.x, v.y);
      const __nv_bfloat162 h23 = __floats2bfloat162_rn(v.z, v.w);
      const float2 f01 = __bfloat1622float2(h01), f23 = __bfloat1622float2(h23);
      const __nv_bfloat162 l01 = __floats2bfloat162_rn(v.x - f01.x, v.y - f01.y);
      const __nv_bfloat162 l23 = __floats2bfloat162_rn(v.z - f23.x, v.w - f23.y);
      uint2 hw, lw;
      hw.x = *reinterpret_cast<const uint32_t*>(&h01);
      hw.y = *reinterpret_cast<const uint32_t*>(&h23);
      lw.x = *reinterpret_cast<const uint32_t*>(&l01);
      lw.y = *reinterpret_cast<const uint32_t*>(&l23);
      *reinterpret_cast<uint2*>(tile + sw128_offset(128, x % 128, f0)) = hw;
      *reinterpret_cast<uint2*>(tile + sw128_offset(128, x % 128, kp + f0)) = lw;
    } else {
      *reinterpret_cast<float4*>(Ut + (size_t)x * kp + f0) = v;
    }
  }
  // Columns past the last row group are zero.
  if (blockIdx.y == gridDim.y - 1 && rq == 0) {
    for (int f = 2 * R * gridDim.y; f < kp; f += 4) {
      if (img) {
        uint8_t* tile = img + (size_t)(x / 128) * img_tile_bytes;
        *reinterpret_cast<uint2*>(tile + sw128_offset(128, x % 128, f)) = make_uint2(0u, 0u);
        *reinterpret_cast<uint2*>(tile + sw128_offset(128, x % 128, kp + f)) = make_uint2(0u, 0u);
      } else {
        *reinterpret_cast<float4*>(Ut + (size_t)x * kp + f) = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
  }
}

template <int PAIRS>
__global__ void __launch_bounds__(EX_NT)
expand_kernel(const float2* __restrict__ coef, int nrows, int ncoef, int ld,
              const float2* __restrict__ TX, int N, int mode, int nc, int kp,
              float* __restrict__ Ut, uint8_t* __restrict__ img, uint32_t img_tile_bytes) {
  constexpr int R = 8 * PAIRS;
  extern __shared__ __align__(16) float4 se[];
  const int nph = expand_nph(mode, ncoef, nc);
  float4* sd = se;                                         // [R][nph]
  float2* ph = reinterpret_cast<float2*>(se + R * nph);    // [nph][EX_X]
  const int x0 = blockIdx.x * EX_X, a0 = blockIdx.y * R;
  {  // image b of a batch
    const size_t b = blockIdx.z;
    coef += b * nrows * ld;
    if (img) img += b * ((N + 127) / 128) * (size_t)img_tile_bytes;
    else Ut += b * N * kp;
  }
  pdl_trigger();
  fill_batched<EX_NT>(ph, nph * EX_X, [&](int i) {
    const int j = i / EX_X, x = x0 + i % EX_X;
    return x < N ? TX[(size_t)j * N + x] : make_float2(0.f, 0.f);
  });
  pdl_wait();
  fill_batched<EX_NT>(sd, R * nph, [&](int i) {
    const int r = i / nph, j = i % nph;
    return (a0 + r < nrows) ? expand_sd(coef + (size_t)(a0 + r) * ld, mode, nc, j)
                            : make_float4(0.f, 0.f, 0.f, 0.f);
  });
  __syncthreads();
  expand_store<PAIRS>(sd, ph, nrows, nph, N, mode, kp, a0, x0, Ut, img, img_tile_bytes);
}

// The expansion with every band row of an x strip in one CTA (up to 64 rows): all 256
// threads stage the tables, then thread (xp, rg), rg < ceil(nrows / 8), computes image
// rows x0 + 2 xp and x0 + 2 xp + 1 for the eight band rows 8 rg .. 8 rg + 7, so each
// step over j takes one 16-byte phase load and eight 16-byte broadcast loads of
// coefficient pairs for 32 packed FMAs. The pairs are staged transposed
// (sdT[j][8 groups]); rows past nrows are zero. Same operands, order and scale as
// expand_store: bit-identical results.
constexpr int EXR_X = 64, EXR_NT = 256;
__global__ void __launch_bounds__(EXR_NT)
expand_rows_kernel(const float2* __restrict__ coef, int nrows, int ncoef, int ld,
                   const float2* __restrict__ TX, int N, int mode, int nc, int kp,
                   float* __restrict__ Ut, uint8_t* __restrict__ img, uint32_t img_tile_bytes) {
  extern __shared__ __align__(16) float4 sr4[];
  const int groups = (nrows + 7) / 8, R = 8 * groups;
  const int nph = expand_nph(mode, ncoef, nc);
  float4* sdT = sr4;                                             // [nph][R]
  float2* ph = reinterpret_cast<float2*>(sr4 + nph * R);         // [nph][EXR_X]
  const int x0 = blockIdx.x * EXR_X;
  {  // image b of a batch
    const size_t b = blockIdx.z;
    coef += b * nrows * ld;
    if (img) img += b * ((N + 127) / 128) * (size_t)img_tile_bytes;
    else Ut += b * N * kp;
  }
  pdl_trigger();
  fill_batched<EXR_NT>(ph, nph * EXR_X, [&](int i) {
    const int j = i / EXR_X, x = x0 + i % EXR_X;
    return x < N ? TX[(size_t)j * N + x] : make_float2(0.f, 0.f);
  });
  pdl_wait();
  // sdT[j][r] = the pair of band row r: coalesced reads of coef, a transposed store.
  for (int base = threadIdx.x; base < R * nph; base += EXR_NT * 4) {
    float4 v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = base + q * EXR_NT, r = i / nph;
      if (i < R * nph)
        v[q] = r < nrows ? expand_sd(coef + (size_t)r * ld, mode, nc, i % nph)
                         : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = base + q * EXR_NT;
      if (i < R * nph) sdT[(i % nph) * R + i / nph] = v[q];
    }
  }
  __syncthreads();
  const int xp = threadIdx.x % 32, rg = threadIdx.x / 32;
  if (rg >= groups) return;   // staging helpers only
  float2 acc[8][2];
#pragma unroll
  for (int i = 0; i < 8; ++i) acc[i][0] = acc[i][1] = make_float2(0.f, 0.f);
  for (int j = 0; j < nph; ++j) {
    const float4 p = *reinterpret_cast<const float4*>(ph + j * EXR_X + 2 * xp);
    const float4* cq = sdT + j * R + 8 * rg;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const float4 sd = cq[i];
      acc[i][0] = sd_fma(acc[i][0], sd, p.x, p.y);
      acc[i][1] = sd_fma(acc[i][1], sd, p.z, p.w);
    }
  }
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int x = x0 + 2 * xp + h;
    if (x >= N) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int ra = 8 * rg + 2 * q, rb = ra + 1;
      const float ka = ra < nrows ? ((mode == 1 && ra > 0) ? 2.f : 1.f) : 0.f;
      const float kb = rb < nrows ? ((mode == 1 && rb > 0) ? 2.f : 1.f) : 0.f;
      const float4 v = make_float4(ka * acc[2 * q][h].x, ka * acc[2 * q][h].y,
                                   kb * acc[2 * q + 1][h].x, kb * acc[2 * q + 1][h].y);
      const int f0 = 2 * ra;
      if (f0 >= kp) continue;
      if (img) {
        uint8_t* tile = img + (size_t)(x / 128) * img_tile_bytes;
        const __nv_bfloat162 h01 = __floats2bfloat162_rn(v.x, v.y);
        const __nv_bfloat162 h23 = __floats2bfloat162_rn(v.z, v.w);
        const float2 f01 = __bfloat1622float2(h01), f23 = __bfloat1622float2(h23);
        const __nv_bfloat162 l01 = __floats2bfloat162_rn(v.x - f01.x, v.y - f01.y);
        const __nv_bfloat162 l23 = __floats2bfloat162_rn(v.z - f23.x, v.w - f23.y);
        uint2 hw, lw;
        hw.x = *reinterpret_cast<const uint32_t*>(&h01);
        hw.y = *reinterpret_cast<const uint32_t*>(&h23);
        lw.x = *reinterpret_cast<const uint32_t*>(&l01);
        lw.y = *reinterpret_cast<const uint32_t*>(&l23);
        *reinterpret_cast<uint2*>(tile + sw128_offset(128, x % 128, f0)) = hw;
        *reinterpret_cast<uint2*>(tile + sw128_offset(128, x % 128, kp + f0)) = lw;
      } else {
        *reinterpret_cast<float4*>(Ut + (size_t)x * kp + f0) = v;
      }
    }
    // Columns past the last row group are zero.
    if (rg == 0) {
      for (int f = 2 * R; f < kp; f += 4) {
        if (img) {
          uint8_t* tile = img + (size_t)(x / 128) * img_tile_bytes;
          *reinterpret_cast<uint2*>(tile + sw128_offset(128, x % 128, f)) = make_uint2(0u, 0u);
          *reinterpret_cast<uint2*>(tile + sw128_offset(128, x % 128, kp + f)) = make_uint2(0u, 0u);
        } else {
          *reinterpret_cast<float4*>(Ut + (size_t)x * kp + f) = make_float4(0.f, 0.f, 0.f, 0.f);
        }
      }
    }
  }
}

template <int PAIRS>
static cudaError_t launch_expand_t(cudaStream_t s, const float2* coef, int nrows, int ncoef,
                                   int ld, const float2* TX, int N, int mode, int nc, int kp,
                                   float* Ut, void* img, int batch) {
  constexpr int R = 8 * PAIRS;
  // Split-BF16 image tile: 128 rows x [hi | lo] of kp columns, in 64-column atoms.
  const uint32_t img_tile_bytes = (uint32_t)((2 * kp + 63) / 64) * 128u * 128u;
  const int nph = expand_nph(mode, ncoef, nc);
  const size_t smem = (size_t)R * nph * sizeof(float4) + (size_t)nph * EX_X * sizeof(float2);
  cudaError_t e = cudaFuncSetAttribute(expand_kernel<PAIRS>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((N + EX_X - 1) / EX_X, (nrows + R - 1) / R, batch);
  return launch_pdl(expand_kernel<PAIRS>, grid, dim3(EX_NT), smem, s, coef, nrows, ncoef, ld, TX,
                    N, mode, nc, kp, Ut, static_cast<uint8_t*>(img), img_tile_bytes);
}

// Batches take 16 rows per CTA (fewer phase-table stagings, more reuse of each phase),
// single images 8 (more CTAs); the results are the same.
static cudaError_t launch_expand(cudaStream_t s, const float2* coef, int nrows, int ncoef, int ld,
                                 const float2* TX, int N, int mode, int nc, int kp, float* Ut,
                                 void* img, int batch) {
  if (batch >= 8 && nrows <= 64) {
    // Every band row of an x strip in one CTA (enough CTAs from 8 images on).
    const int R = 8 * ((nrows + 7) / 8);
    const uint32_t img_tile_bytes = (uint32_t)((2 * kp + 63) / 64) * 128u * 128u;
    const int nph = expand_nph(mode, ncoef, nc);
    const size_t smem = (size_t)nph * R * sizeof(float4) + (size_t)nph * EXR_X * sizeof(float2);
    cudaError_t e = cudaFuncSetAttribute(expand_rows_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return launch_pdl(expand_rows_kernel, dim3((N + EXR_X - 1) / EXR_X, 1, batch),
                      dim3(EXR_NT), smem, s, coef, nrows, ncoef, ld, TX, N, mode, nc, kp, Ut,
                      static_cast<uint8_t*>(img), img_tile_bytes);
  }
  return batch >= 4 ? launch_expand_t<2>(s, coef, nrows, ncoef, ld, TX, N, mode, nc, kp, Ut, img, batch)
                    : launch_expand_t<1>(s, coef, nrows, ncoef, ld, TX, N, mode, nc, kp, Ut, img, batch);
}

static size_t z_whole_smem(const BandGeom& g);

// Whole small grid per CTA (width BW_WHOLE, or by default from 8 images on) where both
// whole-grid kernels' tables fit in shared memory.
static bool band_whole(const BandGeom& g, int batch, int width) {
  if (fields_whole_smem(g) > SMEM_STAGE || z_whole_smem(g) > SMEM_STAGE) return false;
  return width > 0 ? width == BW_WHOLE : batch >= 8;
}

cudaError_t launch_band_forward(cudaStream_t s, const Cache& c, Field& f, float* ik, float* iP,
                                float2* chat, float* Ut, void* img, int batch, int width) {
  const BandGeom& g = c.g;
  auto fields = [&](auto wtag) -> cudaError_t {
    constexpr int W = decltype(wtag)::value;
    const bool staged = fields_smem<W>(g, true) <= SMEM_STAGE;
    const size_t sm1 = fields_smem<W>(g, staged);
    cudaError_t e1 = cudaFuncSetAttribute(band_fields_kernel<W>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1);
    if (e1 != cudaSuccess) return e1;
    return launch_pdl(band_fields_kernel<W>, dim3(g.K, (g.Pc + W - 1) / W, batch), dim3(BF_NT),
                      sm1, s, c.H, static_cast<const float2*>(f.mband), c.w, g.Nr, g.Nc, g.Pr,
                      g.Pc, g.row0, c.ESc_t, c.ESr_t, (int)staged, f.e, ik);
  };
  // Schedule: the autotuned one when set, else the whole small grid per CTA for large
  // batches (enough CTAs to fill the GPU) and column chunks otherwise.
  cudaError_t err;
  if (band_whole(g, batch, width)) {
    const size_t smw = fields_whole_smem(g);
    err = cudaFuncSetAttribute(band_fields_whole_kernel,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smw);
    if (err == cudaSuccess)
      err = launch_pdl(band_fields_whole_kernel, dim3(g.K, 1, batch), dim3(BG_NT), smw, s, c.H,
                       static_cast<const float2*>(f.mband), c.w, g.Nr, g.Nc, g.Pr, g.Pc, g.row0,
                       c.ESc_t, c.ESr_t, f.e, ik);
  } else {
    const bool wide = width > 0 ? width >= BW_BATCH : batch >= 4;
    err = wide ? fields(std::integral_constant<int, BW_BATCH>{})
               : fields(std::integral_constant<int, BW_ONE>{});
  }
  if (err != cudaSuccess) return err;
  const int n = g.Pr * g.Pc;
  err = launch_pdl(sum_k_kernel, dim3((n + 255) / 256, batch), dim3(256), 0, s,
                   static_cast<const float*>(ik), g.K, n, iP);
  if (err != cudaSuccess) return err;
  const int nd = 2 * g.Nc - 1;
  if (batch >= 4 && chat_rows_smem(g) <= SMEM_STAGE) {
    // BC_DR band rows per CTA (bit-identical to one row per CTA) once a batch fills the GPU.
    const size_t smc = chat_rows_smem(g);
    err = cudaFuncSetAttribute(band_chat_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smc);
    if (err != cudaSuccess) return err;
    err = launch_pdl(band_chat_rows_kernel, dim3((g.Nr + BC_DR - 1) / BC_DR, batch), dim3(256),
                     smc, s, static_cast<const float*>(iP), g.Nr, g.Nc, g.Pr, g.Pc, c.EDr_t, c.EDc,
                     1.f / ((float)g.Pr * (float)g.Pc), chat);
  } else {
    const size_t smc = chat_smem(g);
    err = cudaFuncSetAttribute(band_chat_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smc);
    if (err != cudaSuccess) return err;
    err = launch_pdl(band_chat_kernel, dim3(g.Nr, batch), dim3(BI_NT), smc, s,
                     static_cast<const float*>(iP), g.Nr, g.Nc, g.Pr, g.Pc, c.EDr_t, c.EDc,
                     1.f / ((float)g.Pr * (float)g.Pc), chat);
  }
  if (err != cudaSuccess) return err;
  return launch_expand(s, chat, g.Nr, nd, nd, c.TXDc, g.N, 1, g.Nc, g.kp_rows, Ut, img, batch);
}

// Adjoint 1 (one CTA per small-grid row jr):
//   wv[c] = sum_a EDr_t[a][jr] kappa(c) g'[a][c]   (a = dr + Nr - 1, c = dc >= 0)
//   gamma[jr][jc] = Re sum_c wv[c] EDc_t[c + Nc - 1][jc]   (gamma is real)
__global__ void __launch_bounds__(256)
band_gamma_kernel(const float2* __restrict__ gh, int Nr, int Nc, int Pr, int Pc,
                  const float2* __restrict__ EDr_t, const float2* __restrict__ EDc_t,
                  float* __restrict__ gam) {
  extern __shared__ float2 sg[];
  const int jr = blockIdx.x;
  const int na = 2 * Nr - 1;
  gh += (size_t)blockIdx.y * na * Nc;   // image b of a batch
  gam += (size_t)blockIdx.y * Pr * Pc;
  float2* wv = sg;               // [Nc]
  float2* edr = wv + Nc;         // [na]   column jr of EDr_t
  float2* ghs = edr + na;        // [na][Nc]
  float2* edc = ghs + na * Nc;   // [Nc][Pc] rows Nc-1 .. 2Nc-2 of EDc_t
  pdl_trigger();
  fill_batched<256>(edr, na, [&](int r) { return EDr_t[(size_t)r * Pr + jr]; });
  fill_batched<256>(edc, Nc * Pc, [&](int i) { return EDc_t[(size_t)(Nc - 1) * Pc + i]; });
  pdl_wait();
  fill_batched<256>(ghs, na * Nc, [&](int i) { return gh[i]; });
  __syncthreads();
  // SPLIT adjacent lanes per output, as in band_chat_kernel.
  constexpr int SPLIT = 4, GROUPS = 256 / SPLIT;
  const int sub = threadIdx.x % SPLIT, grp = threadIdx.x / SPLIT;
  for (int base = 0; base < Nc; base += GROUPS) {
    const int c = base + grp;
    float2 a = make_float2(0.f, 0.f);
    if (c < Nc)
      for (int r = sub; r < na; r += SPLIT) cfma(a, edr[r], ghs[r * Nc + c]);
    a = split_sum<SPLIT>(a);
    const float kc = c > 0 ? 2.f : 1.f;
    if (c < Nc && sub == 0) wv[c] = make_float2(kc * a.x, kc * a.y);
  }
  __syncthreads();
  for (int base = 0; base < Pc; base += GROUPS) {
    const int jc = base + grp;
    float acc = 0.f;
    if (jc < Pc)
      for (int c = sub; c < Nc; c += SPLIT) {
        const float2 t = edc[c * Pc + jc];
        acc = fmaf(wv[c].x, t.x, fmaf(-wv[c].y, t.y, acc));
      }
    acc = split_sum<SPLIT>(make_float2(acc, 0.f)).x;
    if (jc < Pc && sub == 0) gam[(size_t)jr * Pc + jc] = acc;
  }
}

// Adjoint 1 with BG_JR small-grid rows per CTA: grid (ceil(Pr / BG_JR), batch). The
// tables and the image's g' are staged once per BG_JR rows; one thread per output (wv)
// or pair of outputs (gamma) keeps the four interleaved partial sums of
// band_gamma_kernel and adds them in its order, so the results are bit-identical.
constexpr int BG_JR = 10;
__global__ void __launch_bounds__(256)
band_gamma_rows_kernel(const float2* __restrict__ gh, int Nr, int Nc, int Pr, int Pc,
                       const float2* __restrict__ EDr_t, const float2* __restrict__ EDc_t,
                       float* __restrict__ gam) {
  extern __shared__ __align__(16) float2 sg[];
  const int na = 2 * Nr - 1;
  const int jr0 = blockIdx.x * BG_JR, nj = min(BG_JR, Pr - jr0);
  gh += (size_t)blockIdx.y * na * Nc;   // image b of a batch
  gam += (size_t)blockIdx.y * Pr * Pc;
  float2* edc = sg;                  // [Nc][Pc] rows Nc-1 .. 2Nc-2 of EDc_t
  float2* ghs = edc + Nc * Pc;       // [na][Nc]
  float2* edr = ghs + na * Nc;       // [BG_JR][na]: EDr_t[a][jr0 + j]
  float2* wv = edr + BG_JR * na;     // [BG_JR][Nc]
  pdl_trigger();
  fill_batched<256>(edr, nj * na, [&](int i) {
    return EDr_t[(size_t)(i % na) * Pr + jr0 + i / na];
  });
  fill_batched<256>(edc, Nc * Pc, [&](int i) { return EDc_t[(size_t)(Nc - 1) * Pc + i]; });
  pdl_wait();
  fill_batched<256>(ghs, na * Nc, [&](int i) { return gh[i]; });
  __syncthreads();
  // wv[j][c] = kappa(c) sum_a EDr_t[a][jr] g'[a][c]
  for (int it = threadIdx.x; it < nj * Nc; it += 256) {
    const int j = it / Nc, c = it % Nc;
    float2 a[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) a[s] = make_float2(0.f, 0.f);
    for (int r0 = 0; r0 < na; r0 += 4) {
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int r = r0 + s;
        if (r < na) cfma(a[s], edr[j * na + r], ghs[r * Nc + c]);
      }
    }
    const float2 v = sum4(a);
    const float kc = c > 0 ? 2.f : 1.f;
    wv[j * Nc + c] = make_float2(kc * v.x, kc * v.y);
  }
  __syncthreads();
  // gamma[jr][jc] = Re sum_c wv[j][c] EDc_t[c + Nc - 1][jc], two columns per thread
  const int pc2 = Pc / 2;
  for (int it = threadIdx.x; it < nj * pc2; it += 256) {
    const int j = it / pc2, jc = 2 * (it % pc2);
    float a0[4] = {0.f, 0.f, 0.f, 0.f}, a1[4] = {0.f, 0.f, 0.f, 0.f};
    for (int c0 = 0; c0 < Nc; c0 += 4) {
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int c = c0 + s;
        if (c < Nc) {
          const float2 w = wv[j * Nc + c];
          const float4 t = *reinterpret_cast<const float4*>(edc + c * Pc + jc);
          a0[s] = fmaf(w.x, t.x, fmaf(-w.y, t.y, a0[s]));
          a1[s] = fmaf(w.x, t.z, fmaf(-w.y, t.w, a1[s]));
        }
      }
    }
    float* out = gam + (size_t)(jr0 + j) * Pc + jc;
    out[0] = (a0[0] + a0[1]) + (a0[2] + a0[3]);
    out[1] = (a1[0] + a1[1]) + (a1[2] + a1[3]);
  }
}

static size_t gamma_rows_smem(const BandGeom& g) {
  const int na = 2 * g.Nr - 1;
  return (size_t)(g.Nc * g.Pc + na * g.Nc + BG_JR * na + BG_JR * g.Nc) * sizeof(float2);
}

static size_t gamma_smem(const BandGeom& g) {
  const int na = 2 * g.Nr - 1;
  return (size_t)(g.Nc + na + na * g.Nc + g.Nc * g.Pc) * sizeof(float2);
}

// Largest dynamic shared memory any small-grid kernel needs for this band
// (the per-kernel CTAs fall back to unstaged tables above their staging limit).
size_t band_max_smem(const BandGeom& g) {
  constexpr int WMAX = BW_ONE > BW_BATCH ? BW_ONE : BW_BATCH;
  size_t m = band_fields_smem(g);
  m = std::max(m, (size_t)(g.Pr * WMAX + g.Pc * WMAX) * sizeof(float2));
  m = std::max(m, chat_smem(g));
  m = std::max(m, gamma_smem(g));
  m = std::max(m, (size_t)(16 + EX_X) * (2 * g.Nc - 1) * sizeof(float2));   // expand, 16 rows
  return m;
}

// The folded input of the Z transform over the small-grid columns: entry i = jr Pc + jc
// of [Pr][Pc] holds, for jc < Nc, q(jr, jc) + q(jr, jc + Nc) and, for jc >= Nc,
// q(jr, jc - Nc) - q(jr, jc), where q = e_k gamma (products rounded on their own).
__device__ __forceinline__ float2 z_fold_q(const float2* __restrict__ ek,
                                           const float* __restrict__ gam, int Nc, int Pc, int i) {
  const int jr = i / Pc, jc = i % Pc, j = jc < Nc ? jc : jc - Nc;
  const size_t o0 = (size_t)jr * Pc + j, o1 = o0 + Nc;
  const float2 t0 = ek[o0], t1 = ek[o1];
  const float g0 = gam[o0], g1 = gam[o1];
  const float2 a = make_float2(__fmul_rn(t0.x, g0), __fmul_rn(t0.y, g0));
  const float2 b = make_float2(__fmul_rn(t1.x, g1), __fmul_rn(t1.y, g1));
  return jc < Nc ? fold_sum(a, b) : fold_diff(a, b);
}

// The staged product q = e_k gamma ([Pr][Pc], products by __fmul_rn) folded in place into
// the layout of z_fold_q, with the same operations; one thread per (jr, jc < Nc) pair.
__device__ __forceinline__ float2 z_product(const float2* __restrict__ ek,
                                            const float* __restrict__ gam, int i) {
  const float2 t = ek[i];
  const float g = gam[i];
  return make_float2(__fmul_rn(t.x, g), __fmul_rn(t.y, g));
}
template <int NT>
__device__ __forceinline__ void z_fold_inplace(float2* q, int Pr, int Nc, int Pc) {
  for (int i = threadIdx.x; i < Pr * Nc; i += NT) {
    const int jr = i / Nc, jc = i - jr * Nc;
    float2* row = q + jr * Pc;
    const float2 a = row[jc], b = row[jc + Nc];
    row[jc] = fold_sum(a, b);
    row[jc + Nc] = fold_diff(a, b);
  }
}

// C = A B with a separate A operand per column of each pair (the transform over P = 2 n
// inputs, folded: column 2p reads a0, column 2p + 1 reads a1), K = Kd in increasing
// order with cfma; each thread owns RT rows x 2 columns.
template <int RT, int NT, class ALoad0, class ALoad1, class Store>
__device__ __forceinline__ void fold_cols_in(int M, int npairs, int Kd, ALoad0 a0, ALoad1 a1,
                                             const float2* __restrict__ B, int ldb, Store store) {
  const int rblocks = (M + RT - 1) / RT;
  for (int it = threadIdx.x; it < rblocks * npairs; it += NT) {
    const int m0 = (it / npairs) * RT, p = it % npairs;
    float2 acc[RT][2];
#pragma unroll
    for (int i = 0; i < RT; ++i) acc[i][0] = acc[i][1] = make_float2(0.f, 0.f);
    for (int k = 0; k < Kd; ++k) {
      const float4 b = *reinterpret_cast<const float4*>(B + (size_t)k * ldb + 2 * p);
      const float2 b0 = make_float2(b.x, b.y), b1 = make_float2(b.z, b.w);
#pragma unroll
      for (int i = 0; i < RT; ++i) {
        const int m = min(m0 + i, M - 1);
        cfma(acc[i][0], a0(m, k), b0);
        cfma(acc[i][1], a1(m, k), b1);
      }
    }
#pragma unroll
    for (int i = 0; i < RT; ++i) {
      if (m0 + i < M) {
        store(m0 + i, 2 * p, acc[i][0]);
        store(m0 + i, 2 * p + 1, acc[i][1]);
      }
    }
  }
}

// Adjoint 2: grid (K, band column chunks of W, batch). CTA (k, q) owns band columns
// uc in [q W, q W + W): q_k = e_k gamma (Pr x Pc, staged), Z1 = q_k conj(ESc)
// restricted to those columns (Pr x W), Zk = conj(ESr_t) Z1 / (Pr Pc) (Nr x W); four
// adjacent columns per thread as in the fields kernel.
template <int W>
__global__ void __launch_bounds__(BF_NT)
band_z_kernel(const float2* __restrict__ e, const float* __restrict__ gam, int Nr, int Nc, int Pr,
              int Pc, int col0, const float2* __restrict__ ESc, const float2* __restrict__ ESr_t,
              int stage_tables, float inv, float2* __restrict__ Zk) {
  static_assert(W % 4 == 0, "four columns per thread");
  constexpr int JB = W / 4;
  extern __shared__ __align__(16) float2 sz[];
  const int k = blockIdx.x;
  const int u0 = blockIdx.y * W;
  const int uw = min(W, Nc - u0);
  {  // image b of a batch
    const size_t b = blockIdx.z;
    e += b * gridDim.x * Pr * Pc;
    gam += b * Pr * Pc;
    Zk += b * gridDim.x * Nr * Nc;
  }
  float2* Z1 = sz;                  // [Pr][W]
  float2* esc = Z1 + Pr * W;        // [Pc][W] (rows jc < Nc used; columns past uw are zero)
  float2* q = esc + Pc * W;         // [Pr][Pc]   (staged: folded, z_fold_q)
  float2* esr = q + Pr * Pc;        // [Nr][Pr]   (staged)
  const float2* ek = e + (size_t)k * Pr * Pc;
  pdl_trigger();
  fill_batched<BF_NT>(esc, Nc * W, [&](int i) {
    const int jc = i / W, uu = i % W;
    return uu < uw ? conjf2(ESc[(size_t)jc * Nc + u0 + uu]) : make_float2(0.f, 0.f);
  });
  const float2* ESR = ESr_t;
  if (stage_tables) {
    fill_batched<BF_NT>(esr, Nr * Pr, [&](int i) { return ESr_t[i]; });
    ESR = esr;
  }
  pdl_wait();
  if (stage_tables) {
    fill_batched<BF_NT>(q, Pr * Pc, [&](int i) { return z_product(ek, gam, i); });
    __syncthreads();
    z_fold_inplace<BF_NT>(q, Pr, Nc, Pc);
  }
  __syncthreads();
  // Columns u0 + jb + {0, 2} have the parity of col0, {1, 3} the other (u0, jb multiples
  // of 4): the even class takes the folded sums, the odd class the differences.
  const int cpar = col0 & 1;
  for (int it = threadIdx.x; it < Pr * JB; it += BF_NT) {
    const int jr = it / JB, jb = 4 * (it % JB);
    float2 acc[4] = {};
    for (int jc = 0; jc < Nc; ++jc) {
      float2 va, vb;
      if (stage_tables) {
        va = q[jr * Pc + (cpar ? Nc : 0) + jc];
        vb = q[jr * Pc + (cpar ? 0 : Nc) + jc];
      } else {
        const float2 vs = z_fold_q(ek, gam, Nc, Pc, jr * Pc + jc);
        const float2 vd = z_fold_q(ek, gam, Nc, Pc, jr * Pc + Nc + jc);
        va = cpar ? vd : vs;
        vb = cpar ? vs : vd;
      }
      const float4 b01 = *reinterpret_cast<const float4*>(esc + jc * W + jb);
      const float4 b23 = *reinterpret_cast<const float4*>(esc + jc * W + jb + 2);
      cfma(acc[0], va, make_float2(b01.x, b01.y));
      cfma(acc[1], vb, make_float2(b01.z, b01.w));
      cfma(acc[2], va, make_float2(b23.x, b23.y));
      cfma(acc[3], vb, make_float2(b23.z, b23.w));
    }
    *reinterpret_cast<float4*>(Z1 + jr * W + jb) = make_float4(acc[0].x, acc[0].y, acc[1].x, acc[1].y);
    *reinterpret_cast<float4*>(Z1 + jr * W + jb + 2) =
        make_float4(acc[2].x, acc[2].y, acc[3].x, acc[3].y);
  }
  __syncthreads();
  for (int it = threadIdx.x; it < Nr * JB; it += BF_NT) {
    const int ur = it / JB, jb = 4 * (it % JB);
    float2 acc[4] = {};
    for (int jr = 0; jr < Pr; ++jr) cfma4(acc, conjf2(ESR[ur * Pr + jr]), Z1 + jr * W + jb);
#pragma unroll
    for (int qq = 0; qq < 4; ++qq) {
      if (jb + qq >= uw) break;
      Zk[((size_t)k * Nr + ur) * Nc + u0 + jb + qq] =
          make_float2(acc[qq].x * inv, acc[qq].y * inv);
    }
  }
}

// Adjoint 2, whole small grid per CTA: grid (K, 1, batch), CTA (k, b) computes all of
// Zk for image b, every table staged once. Same arithmetic as band_z_kernel
// (bit-identical results); the band columns are padded to an even count with zero
// table columns, whose outputs are not stored.
__global__ void __launch_bounds__(BG_NT)
band_z_whole_kernel(const float2* __restrict__ e, const float* __restrict__ gam, int Nr, int Nc,
                    int Pr, int Pc, int col0, const float2* __restrict__ ESc,
                    const float2* __restrict__ ESr_t, float inv, float2* __restrict__ Zk) {
  extern __shared__ __align__(16) float2 sz[];
  const int k = blockIdx.x;
  const int NcE = even_up(Nc);
  {  // image b of a batch
    const size_t b = blockIdx.z;
    e += b * gridDim.x * Pr * Pc;
    gam += b * Pr * Pc;
    Zk += b * gridDim.x * Nr * Nc;
  }
  float2* esc = sz;                   // [Pc][NcE]
  float2* esr = esc + Pc * NcE;       // [Nr][Pr]
  float2* q = esr + Nr * Pr;          // [Pr][Pc]
  float2* Z1 = q + Pr * Pc;           // [Pr][NcE]
  const float2* ek = e + (size_t)k * Pr * Pc;
  pdl_trigger();
  fill_batched<BG_NT>(esc, Nc * NcE, [&](int i) {
    const int jc = i / NcE, u = i % NcE;
    return u < Nc ? conjf2(ESc[(size_t)jc * Nc + u]) : make_float2(0.f, 0.f);
  });
  fill_batched<BG_NT>(esr, Nr * Pr, [&](int i) { return ESr_t[i]; });
  pdl_wait();
  fill_batched<BG_NT>(q, Pr * Pc, [&](int i) { return z_product(ek, gam, i); });
  __syncthreads();
  z_fold_inplace<BG_NT>(q, Pr, Nc, Pc);
  __syncthreads();
  // Column 2p has the parity of col0: sums for an even class, differences for an odd one.
  const int off0 = (col0 & 1) ? Nc : 0, off1 = Nc - off0;
  fold_cols_in<5, BG_NT>(Pr, NcE / 2, Nc, [&](int jr, int jc) { return q[jr * Pc + off0 + jc]; },
                         [&](int jr, int jc) { return q[jr * Pc + off1 + jc]; }, esc, NcE,
                         [&](int jr, int u, float2 v) { Z1[jr * NcE + u] = v; });
  __syncthreads();
  float2* zk = Zk + (size_t)k * Nr * Nc;
  cgemm_rt2<3, BG_NT>(Nr, NcE / 2, Pr, [&](int ur, int jr) { return conjf2(esr[ur * Pr + jr]); },
                      Z1, NcE, [&](int ur, int u, float2 v) {
                        if (u < Nc) zk[(size_t)ur * Nc + u] = make_float2(v.x * inv, v.y * inv);
                      });
}

static size_t z_whole_smem(const BandGeom& g) {
  const int NcE = even_up(g.Nc);
  return (size_t)(g.Pc * NcE + g.Nr * g.Pr + g.Pr * g.Pc + g.Pr * NcE) * sizeof(float2);
}

// Adjoint 3: X[u] = scale sum_k w_k conj(H_k(u)) Z_k(u). Four lanes per u: lane j
// sums k = j, j + 4, ... in order (the loads of up to 8 of its k issued together),
// then the four partial sums are added in a fixed order.
constexpr int BX_SPLIT = 4;
__global__ void band_x_kernel(const float2* __restrict__ Zk, const float2* __restrict__ H,
                              const float* __restrict__ w, int K, int nb, float scale,
                              float2* __restrict__ X) {
  pdl_trigger();
  pdl_wait();
  Zk += (size_t)blockIdx.y * K * nb;   // image b of a batch
  X += (size_t)blockIdx.y * nb;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int u = t / BX_SPLIT, j = t % BX_SPLIT;
  float2 acc = make_float2(0.f, 0.f);
  if (u < nb) {
    for (int k0 = j; k0 < K; k0 += 8 * BX_SPLIT) {
      float2 hv[8], zv[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int k = k0 + q * BX_SPLIT;
        if (k < K) {
          hv[q] = H[(size_t)k * nb + u];
          zv[q] = Zk[(size_t)k * nb + u];
        }
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int k = k0 + q * BX_SPLIT;
        if (k < K) {
          const float2 c = cmul(conjf2(hv[q]), zv[q]);
          acc.x = fmaf(w[k], c.x, acc.x);
          acc.y = fmaf(w[k], c.y, acc.y);
        }
      }
    }
  }
  // lanes 4u .. 4u + 3 are adjacent in one warp: (0 + 1) + (2 + 3)
#pragma unroll
  for (int o = 1; o < BX_SPLIT; o <<= 1) {
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
  }
  if (u < nb && j == 0) X[u] = make_float2(acc.x * scale, acc.y * scale);
}

cudaError_t launch_band_adjoint(cudaStream_t s, const Cache& c, const Field& f, const float2* gh,
                                double scale, float* gam, float2* Zk, float2* X, float* Vt,
                                void* img, int batch, int width) {
  const BandGeom& g = c.g;
  cudaError_t e0;
  if (batch >= 4 && gamma_rows_smem(g) <= SMEM_STAGE) {
    // BG_JR small-grid rows per CTA (bit-identical to one row per CTA) for batches.
    const size_t smg = gamma_rows_smem(g);
    e0 = cudaFuncSetAttribute(band_gamma_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smg);
    if (e0 != cudaSuccess) return e0;
    e0 = launch_pdl(band_gamma_rows_kernel, dim3((g.Pr + BG_JR - 1) / BG_JR, batch), dim3(256),
                    smg, s, gh, g.Nr, g.Nc, g.Pr, g.Pc, c.EDr_t, c.EDc_t, gam);
  } else {
    const size_t smg = gamma_smem(g);
    e0 = cudaFuncSetAttribute(band_gamma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smg);
    if (e0 != cudaSuccess) return e0;
    e0 = launch_pdl(band_gamma_kernel, dim3(g.Pr, batch), dim3(256), smg, s, gh, g.Nr, g.Nc, g.Pr,
                    g.Pc, c.EDr_t, c.EDc_t, gam);
  }
  if (e0 != cudaSuccess) return e0;
  auto zk = [&](auto wtag) -> cudaError_t {
    constexpr int W = decltype(wtag)::value;
    const size_t base = (size_t)(g.Pr * W + g.Pc * W) * sizeof(float2);
    const size_t full = base + (size_t)(g.Pr * g.Pc + g.Nr * g.Pr) * sizeof(float2);
    const int stage = full <= SMEM_STAGE;
    const size_t smz = stage ? full : base;
    cudaError_t e1 = cudaFuncSetAttribute(band_z_kernel<W>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smz);
    if (e1 != cudaSuccess) return e1;
    return launch_pdl(band_z_kernel<W>, dim3(g.K, (g.Nc + W - 1) / W, batch), dim3(BF_NT), smz, s,
                      static_cast<const float2*>(f.e), static_cast<const float*>(gam), g.Nr, g.Nc,
                      g.Pr, g.Pc, g.col0, c.ESc, c.ESr_t, stage, 1.f / ((float)g.Pr * (float)g.Pc),
                      Zk);
  };
  cudaError_t err;
  if (band_whole(g, batch, width)) {
    const size_t smw = z_whole_smem(g);
    err = cudaFuncSetAttribute(band_z_whole_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smw);
    if (err == cudaSuccess)
      err = launch_pdl(band_z_whole_kernel, dim3(g.K, 1, batch), dim3(BG_NT), smw, s,
                       static_cast<const float2*>(f.e), static_cast<const float*>(gam), g.Nr,
                       g.Nc, g.Pr, g.Pc, g.col0, c.ESc, c.ESr_t, 1.f / ((float)g.Pr * (float)g.Pc),
                       Zk);
  } else {
    const bool wide = width > 0 ? width >= BW_BATCH : batch >= 4;
    err = wide ? zk(std::integral_constant<int, BW_BATCH>{})
               : zk(std::integral_constant<int, BW_ONE>{});
  }
  if (err != cudaSuccess) return err;
  const int nb = g.Nr * g.Nc;
  err = launch_pdl(band_x_kernel, dim3((nb * BX_SPLIT + 127) / 128, batch), dim3(128), 0, s,
                   static_cast<const float2*>(Zk), c.H, c.w, g.K, nb, (float)scale, X);
  if (err != cudaSuccess) return err;
  return launch_expand(s, X, g.Nr, g.Nc, g.Nc, c.TXSc, g.N, 0, g.Nc, g.kp_rows, Vt, img, batch);
}

// ---------------------------------------------------------------- FP64 partial sums
__global__ void sum_partials_kernel(const double* __restrict__ part, int n, int stride,
                                    double* __restrict__ out) {
  // One warp per component; lanes stride over blocks, then a fixed shuffle tree.
  pdl_trigger();
  pdl_wait();
  const int comp = blockIdx.x;
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += 32) s += part[(size_t)i * stride + comp];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) out[comp] = s;
}

cudaError_t launch_sum_partials(cudaStream_t s, const double* part, int n, int stride,
                                double* out) {
  return launch_pdl(sum_partials_kernel, dim3(stride), dim3(32), 0, s, part, n, stride, out);
}

// Two partial sets in one launch: blocks [0, sa) sum a's components, the rest b's.
__global__ void sum_partials2_kernel(const double* __restrict__ a, int na, int sa,
                                     double* __restrict__ out_a, const double* __restrict__ b,
                                     int nb, int sb, double* __restrict__ out_b) {
  pdl_trigger();
  pdl_wait();
  const bool first = (int)blockIdx.x < sa;
  const int comp = first ? blockIdx.x : blockIdx.x - sa;
  const double* part = first ? a : b;
  const int n = first ? na : nb, stride = first ? sa : sb;
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += 32) s += part[(size_t)i * stride + comp];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) (first ? out_a : out_b)[comp] = s;
}

cudaError_t launch_sum_partials2(cudaStream_t s, const double* a, int na, int sa, double* out_a,
                                 const double* b, int nb, int sb, double* out_b) {
  return launch_pdl(sum_partials2_kernel, dim3(sa + sb), dim3(32), 0, s, a, na, sa, out_a, b, nb,
                    sb, out_b);
}

// Per image b of a batch: out[b][0..sa) from a + b na sa (sa components over na
// blocks) and out[b][sa..sa+sb) from b + b nb sb, each in the fixed shuffle order.
__global__ void sum_partials_batch_kernel(const double* __restrict__ a, int na, int sa,
                                          const double* __restrict__ b, int nb, int sb,
                                          double* __restrict__ out) {
  pdl_trigger();
  pdl_wait();
  const size_t img = blockIdx.y;
  const bool first = (int)blockIdx.x < sa;
  const int comp = first ? blockIdx.x : blockIdx.x - sa;
  const int n = first ? na : nb, stride = first ? sa : sb;
  const double* part = first ? a + img * na * sa : b + img * nb * sb;
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += 32) v += part[(size_t)i * stride + comp];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (threadIdx.x == 0) out[img * (sa + sb) + blockIdx.x] = v;
}

cudaError_t launch_sum_partials_batch(cudaStream_t s, const double* a, int na, int sa,
                                      const double* b, int nb, int sb, double* out, int batch) {
  return launch_pdl(sum_partials_batch_kernel, dim3(sa + sb, batch), dim3(32), 0, s, a, na, sa, b,
                    nb, sb, out);
}

// ---------------------------------------------------------------- field export
// B[r][x] = sum_c A[k][r][c] e^{2 pi i s_c x/N};  E[y][x] = sum_r e^{2 pi i s_r y/N} B[r][x].
__global__ void export_rows_kernel(const float2* __restrict__ H, const float2* __restrict__ mband,
                                   int k, int Nr, int Nc, int N, const float2* __restrict__ TXSc,
                                   float2* __restrict__ B) {
  const int r = blockIdx.y;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= N) return;
  float2 acc = make_float2(0.f, 0.f);
  for (int c = 0; c < Nc; ++c) {
    const float2 a = cmul(H[((size_t)k * Nr + r) * Nc + c], mband[(size_t)r * Nc + c]);
    cfma(acc, a, conjf2(TXSc[(size_t)c * N + x]));
  }
  B[(size_t)r * N + x] = acc;
}

__global__ void export_cols_kernel(const float2* __restrict__ B, int Nr, int N,
                                   const float2* __restrict__ TYS, float2* __restrict__ E) {
  const int y = blockIdx.y;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= N) return;
  float2 acc = make_float2(0.f, 0.f);
  for (int r = 0; r < Nr; ++r) cfma(acc, conjf2(TYS[(size_t)r * N + y]), B[(size_t)r * N + x]);
  E[(size_t)y * N + x] = acc;
}

cudaError_t launch_export_field(cudaStream_t s, const Cache& c, const Field& f, int k,
                                float2* tmp_rows, float2* out) {
  const BandGeom& g = c.g;
  export_rows_kernel<<<dim3((g.N + 127) / 128, g.Nr), 128, 0, s>>>(c.H, f.mband, k, g.Nr, g.Nc,
                                                                   g.N, c.TXSc, tmp_rows);
  export_cols_kernel<<<dim3((g.N + 127) / 128, g.N), 128, 0, s>>>(tmp_rows, g.Nr, g.N, c.TYS,
                                                                  out);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- PE loss and dL/dI
// Loss::pe_loss / background_penalty_loss partial sums (source/utils/loss.cpp:16-64)
// and, when dldi is set, the dL/dI of the pe_gradient* variants
// (source/utils/gradient.cpp:121-196) without the common 4 alpha.
constexpr int PL_NT = 256;
__global__ void __launch_bounds__(PL_NT)
pe_loss_kernel(const float* __restrict__ w, const float* __restrict__ t,
               const float* __restrict__ pe_win, const float* __restrict__ pen_win,
               float pe_weight, float penalty, float pen_thr, size_t n,
               float* __restrict__ dldi, double* __restrict__ partial) {
  __shared__ double sh[PL_NT / 32];
  double pe = 0.0, pen = 0.0;
  for (size_t i = (size_t)blockIdx.x * PL_NT + threadIdx.x; i < n; i += (size_t)gridDim.x * PL_NT) {
    const float W = w[i], T = t[i];
    const float pw = pe_win ? pe_win[i] : 1.f;
    const float r = W - T;
    pe += (double)r * (double)r * (double)pw;
    float s = pe_weight * r * pw;
    if (penalty != 0.f && T < 0.5f) {
      const float qw = pen_win ? pen_win[i] : pw;
      const float ex = fmaxf(W - pen_thr, 0.f);
      pen += (double)ex * (double)ex * (double)qw;
      s += penalty * ex * qw;
    }
    if (dldi) dldi[i] = s * W * (1.f - W);
  }
  const double a = block_sum<PL_NT>(pe, sh);
  const double b = block_sum<PL_NT>(pen, sh);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = a;
    partial[2 * blockIdx.x + 1] = b;
  }
}

static int pe_blocks(size_t n) {
  int nb = (int)((n + PL_NT - 1) / PL_NT);
  return nb > 592 ? 592 : nb;
}

cudaError_t launch_pe_loss(cudaStream_t s, const float* w, const float* t, const float* pe_win,
                           const float* pen_win, float penalty, float pen_thr, size_t n,
                           double* partial, int* nblocks) {
  *nblocks = pe_blocks(n);
  pe_loss_kernel<<<*nblocks, PL_NT, 0, s>>>(w, t, pe_win, pen_win, 1.f, penalty, pen_thr, n,
                                            nullptr, partial);
  return cudaGetLastError();
}

cudaError_t launch_pe_dldi(cudaStream_t s, const float* w, const float* t, const float* pe_win,
                           const float* pen_win, float pe_weight, float penalty, float pen_thr,
                           size_t n, float* dldi, double* partial, int* nblocks) {
  *nblocks = pe_blocks(n);
  pe_loss_kernel<<<*nblocks, PL_NT, 0, s>>>(w, t, pe_win, pen_win, pe_weight, penalty, pen_thr,
                                            n, dldi, partial);
  return cudaGetLastError();
}

}  // namespace litho_b200
