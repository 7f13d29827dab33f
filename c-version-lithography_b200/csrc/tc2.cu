// Split-BF16 tensor-core passes at full resolution (tcgen05, sm_100a): the tile
// analysis (row DFT and column contraction, both on the tensor cores) and the
// row synthesis with its fused epilogue.
//
// Operand images ("split2"): a tile of RB rows x K FP32 values (K % 16 == 0),
// v = hi + lo with hi = bf16(v), lo = bf16(v - hi), is stored as one K-major
// 128-byte-swizzle UMMA tile with 2K columns [hi | lo]: element (r, k) has hi at
// sw128_offset(RB, r, k) and lo at sw128_offset(RB, r, K + k). The three-pass
// product a_hi b_hi + a_hi b_lo + a_lo b_hi is three MMA sections over the same
// two tiles, (A+0, B+0), (A+0, B+K), (A+K, B+0), accumulated in FP32 in tensor
// memory. Images of constant operands (twiddle tables) are built once per
// optical cache; per-call operands are packed by pack_split2_kernel or written
// by the threads of the CTA that consumes them.
//
// Every mbarrier wait is bounded by a clock budget; on expiry the kernel records
// a code in *err, waits (bounded) for its own bulk copies, releases its tensor
// memory and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "tc_ptx.cuh"
#include "tc_split2.cuh"

namespace litho_b200 {

// First element of row m of image blockIdx.z (the images of a batched launch lie
// N * N apart).
__device__ __forceinline__ size_t img_row(int N, int m) {
  return ((size_t)blockIdx.z * N + m) * N;
}

// ---------------------------------------------------------------- image packing
// Logical real matrix of a pack source: kind 0 reads src[row * ld + col];
// kind 1 reads the complex src2[(row / 2) * ld + col] and gives its real part
// for even rows, its imaginary part for odd rows. Outside rows x cols it is 0.
struct Split2Src {
  const float* src;
  int kind;
  int rows, cols, ld;
};

__device__ __forceinline__ float s2_value(const Split2Src& s, int row, int col) {
  if (row >= s.rows || col >= s.cols) return 0.f;
  if (s.kind == 0) return s.src[(size_t)row * s.ld + col];
  const float2 z = reinterpret_cast<const float2*>(s.src)[(size_t)(row >> 1) * s.ld + col];
  return (row & 1) ? z.y : z.x;
}

// Tiles (rb, kb) of RB rows x K columns, stored in the order t = rb * nkb + kb.
// One thread per 16-byte chunk (8 bf16) of the destination.
__global__ void pack_split2_kernel(Split2Src s, int RB, int K, int nkb, uint4* __restrict__ dst,
                                   size_t n16) {
  pdl_trigger();
  pdl_wait();
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n16) return;
  const int atoms = (int)s2_atoms(K);
  const int j = (int)(idx % 8);          // logical 16-byte chunk within the atom row
  size_t rest = idx / 8;
  const int r = (int)(rest % RB);
  rest /= RB;
  const int a = (int)(rest % atoms);
  const size_t t = rest / atoms;
  const int rb = (int)(t / nkb), kb = (int)(t % nkb);
  const int row = rb * RB + r;
  __nv_bfloat16 out[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int kk = a * 64 + j * 8 + q;
    __nv_bfloat16 hi, lo;
    if (kk < 2 * K) {
      split_bf16(s2_value(s, row, kb * K + (kk < K ? kk : kk - K)), hi, lo);
      out[q] = kk < K ? hi : lo;
    } else {
      out[q] = __float2bfloat16_rn(0.f);
    }
  }
  const size_t off16 = (t * atoms + a) * (size_t)RB * 8 + (size_t)(r / 8) * 64 +
                       (size_t)(r % 8) * 8 + (size_t)(j ^ (r % 8));
  dst[off16] = *reinterpret_cast<const uint4*>(out);
}

size_t split2_image_bytes(int nrb, int RB, int nkb, int K) {
  return (size_t)nrb * nkb * s2_tile_bytes(RB, K);
}

cudaError_t launch_pack_split2(cudaStream_t st, const float* src, int kind, int rows, int cols,
                               int ld, int RB, int K, int nrb, int nkb, void* dst) {
  const size_t n16 = (size_t)nrb * nkb * s2_atoms(K) * (size_t)RB * 8;
  Split2Src s{src, kind, rows, cols, ld};
  return launch_pdl(pack_split2_kernel, dim3((unsigned)((n16 + 255) / 256)), dim3(256), 0, st, s,
                    RB, K, nkb, reinterpret_cast<uint4*>(dst), n16);
}

// ---------------------------------------------------------------- tile analysis
// For every 128 x 128 tile (rows y0.., columns x0..) of the image A:
//   stage 1  R[y][f] = sum_x A[y][x] TX[f][x]          (M = 128 y, N = BN f, K = 128 x)
//   stage 2  Q[n][f] = sum_y TY2[n][y] R[y][f]          (M = 128 n, N = BN f, K = 128 y)
// with TX rows f = 2c (Re) / 2c + 1 (Im) of the column twiddles e^{-2 pi i s_c x / N}
// and TY2 rows n = 2r (Re) / 2r + 1 (Im) of the row twiddles T[r][y]. The complex
// partial P[r][c] = sum_y T[r][y] R_c[y] is then
//   Re = Q[2r][2c] - Q[2r+1][2c+1],  Im = Q[2r][2c+1] + Q[2r+1][2c],
// and with sym the conjugate rows -r come from the same Q:
//   Re = Q[2r][2c] + Q[2r+1][2c+1],  Im = Q[2r][2c+1] - Q[2r+1][2c].
// Output: part[row][c][tile] (row = r, or r + nr - 1 for +r / nr - 1 - r for -r with sym).

constexpr int A2_NT = 256;

// Stages 1 and 2 of a tile analysis and the tile's partial, for a CTA whose 256
// threads have written the [hi | lo] image tile into sA (64 KiB) and whose thread
// 0 has issued the bulk copy of the TX image tile into sB on bars[0]. bars[1..3]
// are initialised and unused; tmem holds at least BN columns. Every thread calls
// it; on a bounded-wait expiry *fail is set and *err receives 3..6.
template <int BN>
__device__ __forceinline__ void analysis_stages(uint8_t* sA, uint8_t* sB, const uint64_t* bars,
                                                uint32_t tmem, volatile int* fail,
                                                const Tc2Analysis& a, const uint8_t* tyImg,
                                                int xt, int yt, int* err) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t uA = tc::smem_u32(sA), uB = tc::smem_u32(sB);
  const uint32_t barX = tc::smem_u32(&bars[0]), barM1 = tc::smem_u32(&bars[1]);
  const uint32_t barT = tc::smem_u32(&bars[2]), barM2 = tc::smem_u32(&bars[3]);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  constexpr uint32_t idesc = tc::idesc_bf16(128, BN);
  if (tid == 0 && !*fail) {
    if (!tc::mbar_wait(barX, 0)) {
      *fail = 1;
      atomicExch(err, 3);
      tc::mbar_wait(barX, 0);
    } else {
      tc::fence_after();
      s2_mma(tmem, uA, 128, uB, BN, 128, idesc);
      tc::mma_commit(barM1);
      if (!tc::mbar_wait(barM1, 0)) {
        *fail = 1;
        atomicExch(err, 4);
        tc::mbar_wait(barM1, 0);
      } else {
        // Stage 1 has read sA: bring this y tile's row-twiddle image into it.
        bulk_tile(uA, tyImg + (size_t)yt * A2_A_BYTES, A2_A_BYTES, barT);
      }
    }
  }
  __syncthreads();
  tc::fence_after();
  const int lane_base = (warp & 3) * 32;
  if (!*fail) {
    // R (TMEM lanes y, columns f) -> sB as the K-major [hi | lo] operand of stage 2.
    // Lanes y and y ^ 1 share the 4-byte words (f, y & ~1): the even lane stores
    // the hi pair, the odd lane the lo pair.
    const int y = lane_base + lane;
    const int ye = y & ~1;
    const bool odd = lane & 1;
    for (int q = warp >> 2; q < BN / 16; q += 2) {
      float rv[16];
      tmem_ld16x(tmem + ((uint32_t)lane_base << 16) + (uint32_t)(16 * q), rv);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float pv = __shfl_xor_sync(0xffffffffu, rv[i], 1);
        uint32_t h2, l2;
        split_pair(odd ? pv : rv[i], odd ? rv[i] : pv, h2, l2);
        *reinterpret_cast<uint32_t*>(sB + sw128_offset(BN, 16 * q + i, odd ? 128 + ye : ye)) =
            odd ? l2 : h2;
      }
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  if (tid == 0 && !*fail) {
    if (!tc::mbar_wait(barT, 0)) {
      *fail = 1;
      atomicExch(err, 5);
      tc::mbar_wait(barT, 0);
    } else {
      s2_mma(tmem, uA, 128, uB, BN, 128, idesc);
      tc::mma_commit(barM2);
      if (!tc::mbar_wait(barM2, 0)) {
        *fail = 1;
        atomicExch(err, 6);
        tc::mbar_wait(barM2, 0);
      }
    }
  }
  __syncthreads();
  tc::fence_after();
  // P (TMEM) -> the tile's partials, staged in sA (the row-twiddle tile is dead once
  // stage 2 has completed) as [row][c], then copied out as one contiguous block.
  const int count = a.nrows_out * a.ncols;
  float2* stage = reinterpret_cast<float2*>(sA);
  if (!*fail) {
    const int n = lane_base + lane;
    const int r = n >> 1, s = n & 1;
    for (int q = warp >> 2; q < BN / 16; q += 2) {
      float qv[16], pv[16];
      tmem_ld16x(tmem + ((uint32_t)lane_base << 16) + (uint32_t)(16 * q), qv);
#pragma unroll
      for (int i = 0; i < 16; ++i) pv[i] = __shfl_xor_sync(0xffffffffu, qv[i], 1);
      if (r >= a.nr) continue;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int c = 8 * q + i;
        if (c >= a.ncols) break;
        const float o0 = qv[2 * i], o1 = qv[2 * i + 1], p0 = pv[2 * i], p1 = pv[2 * i + 1];
        if (!a.sym) {
          if (s == 0) stage[r * a.ncols + c] = make_float2(o0 - p1, o1 + p0);
        } else if (s == 0) {
          stage[(a.nr - 1 + r) * a.ncols + c] = make_float2(o0 - p1, o1 + p0);
        } else if (r >= 1) {
          stage[(a.nr - 1 - r) * a.ncols + c] = make_float2(p0 + o1, p1 - o0);
        }
      }
    }
  }
  __syncthreads();
  if (!*fail) {
    // [image][tile][row][c]; the image of a batched launch is blockIdx.z
    float2* out = a.part + (((size_t)blockIdx.z * gridDim.y + yt) * gridDim.x + xt) * count;
    for (int e = tid; e < count; e += blockDim.x) out[e] = stage[e];
  }
}

template <int BN>
__global__ void __launch_bounds__(A2_NT, 2)
analysis_tc2_kernel(Tc2Analysis a, const uint8_t* __restrict__ txImg,
                    const uint8_t* __restrict__ tyImg, int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bars[4];  // TX landed, stage 1 done, TY landed, stage 2 done
  __shared__ uint32_t tmem_slot;
  __shared__ int fail;
  constexpr uint32_t B_BYTES = s2_tile_bytes(BN, 128);
  constexpr uint32_t TM_COLS = BN <= 32 ? 32 : (BN <= 64 ? 64 : 128);
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  uint8_t* sA = smem;
  uint8_t* sB = smem + A2_A_BYTES;
  const uint32_t uB = tc::smem_u32(sB);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int xt = blockIdx.x, yt = blockIdx.y;
  const int x0 = xt * 128, y0 = yt * 128;
  const uint32_t barX = tc::smem_u32(&bars[0]);
  pdl_trigger();
  if (tid == 0) {
    for (int i = 0; i < 4; ++i) tc::mbar_init(tc::smem_u32(&bars[i]), 1);
    fail = 0;
    tc::fence_mbar_init();
  }
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(&tmem_slot), TM_COLS);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tmem_slot;
  if (tid == 0) bulk_tile(uB, txImg + (size_t)xt * B_BYTES, B_BYTES, barX);
  pdl_wait();

  // Image tile -> sA as [hi | lo]; every load of the thread is issued first.
  float v[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int j = tid + i * A2_NT;
    const int r = j >> 4, c8 = (j & 15) * 8;
    const int m = y0 + r, x = x0 + c8;
    if (a.vec4 && m < a.N && x + 7 < a.N) {
      const float4 p = __ldg(reinterpret_cast<const float4*>(a.in + img_row(a.N, m) + x));
      const float4 q = __ldg(reinterpret_cast<const float4*>(a.in + img_row(a.N, m) + x + 4));
      v[i][0] = p.x; v[i][1] = p.y; v[i][2] = p.z; v[i][3] = p.w;
      v[i][4] = q.x; v[i][5] = q.y; v[i][6] = q.z; v[i][7] = q.w;
    } else {
#pragma unroll
      for (int e = 0; e < 8; ++e)
        v[i][e] = (m < a.N && x + e < a.N) ? __ldg(a.in + img_row(a.N, m) + x + e) : 0.f;
    }
  }
  bool bad = false;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int j = tid + i * A2_NT;
    const int r = j >> 4, c8 = (j & 15) * 8;
    const int m = y0 + r, x = x0 + c8;
    float u[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const bool in_range = m < a.N && x + e < a.N;
      u[e] = v[i][e];
      if (in_range) bad |= !isfinite(u[e]);
      if (a.mode == 1) {
        u[e] = in_range ? 0.5f * (1.f + fast_cos(u[e])) : 0.f;
        if (a.mask_out && in_range) a.mask_out[img_row(a.N, m) + x + e] = u[e];
      }
    }
    uint4 h4, l4;
    split_pair(u[0], u[1], h4.x, l4.x);
    split_pair(u[2], u[3], h4.y, l4.y);
    split_pair(u[4], u[5], h4.z, l4.z);
    split_pair(u[6], u[7], h4.w, l4.w);
    *reinterpret_cast<uint4*>(sA + sw128_offset(128, r, c8)) = h4;
    *reinterpret_cast<uint4*>(sA + sw128_offset(128, r, 128 + c8)) = l4;
  }
  if (bad) atomicOr(a.flag, 1);
  analysis_stages<BN>(sA, sB, bars, tmem, &fail, a, tyImg, xt, yt, err);
  tc::fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, TM_COLS);
}

template <int BN>
static cudaError_t analysis_tc2_t(cudaStream_t s, const Tc2Analysis& a, const void* tx,
                                  const void* ty, int* err, int batch) {
  const size_t smem = A2_A_BYTES + s2_tile_bytes(BN, 128) + 1024;
  cudaError_t e = cudaFuncSetAttribute(analysis_tc2_kernel<BN>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int t = (a.N + 127) / 128;
  return launch_pdl(analysis_tc2_kernel<BN>, dim3(t, t, batch), dim3(A2_NT), smem, s, a,
                    static_cast<const uint8_t*>(tx), static_cast<const uint8_t*>(ty), err);
}

int tc2_analysis_rows(int ncols) { return (2 * ncols + 15) / 16 * 16; }

// Images for the analysis: tx (rows f of the real table tw[2 ncols][N], K tiles of
// 128 x) and ty (rows n of the complex table T[nr][N], K tiles of 128 y).
size_t tc2_tx_image_bytes(int N, int ncols) {
  return split2_image_bytes(1, tc2_analysis_rows(ncols), (N + 127) / 128, 128);
}
size_t tc2_ty_image_bytes(int N) { return split2_image_bytes(1, 128, (N + 127) / 128, 128); }

cudaError_t launch_pack_tc2_tx(cudaStream_t s, const float* tw, int ncols, int N, void* dst) {
  return launch_pack_split2(s, tw, 0, 2 * ncols, N, N, tc2_analysis_rows(ncols), 128, 1,
                            (N + 127) / 128, dst);
}
cudaError_t launch_pack_tc2_ty(cudaStream_t s, const float2* T, int nr, int N, void* dst) {
  return launch_pack_split2(s, reinterpret_cast<const float*>(T), 1, 2 * nr, N, N, 128, 128, 1,
                            (N + 127) / 128, dst);
}

bool tc2_analysis_supported(int ncols, int nr) {
  return tc2_analysis_rows(ncols) <= 128 && 2 * nr <= 128;
}

cudaError_t launch_analysis_tc2(cudaStream_t s, int mode, const float* in, float* mask_out,
                                int* flag, int N, int ncols, int nrows_out, int nr, int sym,
                                float2* part, const void* tx_img, const void* ty_img, int* err,
                                int batch) {
  // The epilogue stages the tile's partials in the 64 KiB operand area.
  if ((size_t)nrows_out * ncols * sizeof(float2) > A2_A_BYTES) return cudaErrorInvalidValue;
  const int vec4 = (N % 4 == 0) && (reinterpret_cast<uintptr_t>(in) % 16 == 0);
  Tc2Analysis a{in, mask_out, flag, N, mode, vec4, ncols, nrows_out, nr, sym, part};
  switch (tc2_analysis_rows(ncols)) {
    case 16: return analysis_tc2_t<16>(s, a, tx_img, ty_img, err, batch);
    case 32: return analysis_tc2_t<32>(s, a, tx_img, ty_img, err, batch);
    case 48: return analysis_tc2_t<48>(s, a, tx_img, ty_img, err, batch);
    case 64: return analysis_tc2_t<64>(s, a, tx_img, ty_img, err, batch);
    case 80: return analysis_tc2_t<80>(s, a, tx_img, ty_img, err, batch);
    case 96: return analysis_tc2_t<96>(s, a, tx_img, ty_img, err, batch);
    case 112: return analysis_tc2_t<112>(s, a, tx_img, ty_img, err, batch);
    case 128: return analysis_tc2_t<128>(s, a, tx_img, ty_img, err, batch);
    default: return cudaErrorInvalidValue;
  }
}

// ---------------------------------------------------------------- row synthesis
//   out[y][x] = sum_f AY[y][f] Ut[x][f]   (f < kp, kp % 16 == 0, kp <= 128)
// per 128 x 128 output tile: A = split2 image of AY rows y0.. (K = kp), B = split2
// image of Ut rows x0.., 3 kp / 16 MMAs with M = N = 128. On interior tiles the
// epilogue's per-pixel input (target or theta) is fetched into registers while
// the operands load and the MMAs run; the accumulator is staged through shared
// memory (aliasing the dead operand tiles) so that every global access of the
// epilogue is coalesced.
constexpr int S2_NT = 256;
constexpr int S2_SS = 128 + 4;                          // staging row stride (floats)
constexpr int S2_CHUNKS = 128 * 128 / 4 / S2_NT;        // float4 chunks per thread (16)

size_t tc2_synth_smem(int kp) {
  const size_t ops = 2 * (size_t)s2_tile_bytes(128, kp);
  const size_t stage = (size_t)128 * S2_SS * sizeof(float);
  return (ops > stage ? ops : stage) + 1024;
}

template <class Epi>
__global__ void __launch_bounds__(S2_NT, 2)
synth_tc2_kernel(const uint8_t* __restrict__ Aimg, const uint8_t* __restrict__ Bimg, int N,
                 int kp, Epi epi, int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ uint32_t tmem_slot;
  __shared__ int fail;
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  const uint32_t tile_bytes = s2_tile_bytes(128, kp);
  const uint32_t uA = tc::smem_u32(smem), uB = uA + tile_bytes;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int xt = blockIdx.x, yt = blockIdx.y;
  const int x0 = xt * 128, y0 = yt * 128;
  const bool interior = epi.vec && y0 + 128 <= N && x0 + 128 <= N;
  const uint32_t barL = tc::smem_u32(&bars[0]), barM = tc::smem_u32(&bars[1]);
  pdl_trigger();
  if (tid == 0) {
    tc::mbar_init(barL, 1);
    tc::mbar_init(barM, 1);
    fail = 0;
    tc::fence_mbar_init();
  }
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(&tmem_slot), 128);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tmem_slot;
  // The twiddle operand (a cache table) loads before the dependency wait, the
  // band operand (written by the previous kernel) after it.
  if (tid == 0) {
    tc::mbar_expect_tx(barL, 2 * tile_bytes);
    const uint8_t* ga = Aimg + (size_t)yt * tile_bytes;
    for (uint32_t q = 0; q < tile_bytes; q += 16384)
      tc::bulk_g2s(uA + q, ga + q, tile_bytes - q < 16384u ? tile_bytes - q : 16384u, barL);
  }
  pdl_wait();
  if (tid == 0) {
    // The band operand image of this launch's image blockIdx.z.
    const uint8_t* gb = Bimg + ((size_t)blockIdx.z * gridDim.x + xt) * tile_bytes;
    for (uint32_t q = 0; q < tile_bytes; q += 16384)
      tc::bulk_g2s(uB + q, gb + q, tile_bytes - q < 16384u ? tile_bytes - q : 16384u, barL);
  }
  // Epilogue inputs of interior tiles, coalesced: chunk j covers row j / 32,
  // columns 4 (j % 32) .. + 3 (edge tiles read theirs in the epilogue).
  float4 pre[S2_CHUNKS];
  if (interior) {
#pragma unroll
    for (int i = 0; i < S2_CHUNKS; ++i) {
      const int j = tid + i * S2_NT;
      pre[i] = epi.pre4(y0 + (j >> 5), x0 + (j & 31) * 4, 4);
    }
  }
  if (tid == 0) {
    if (!tc::mbar_wait(barL, 0)) {
      fail = 1;
      atomicExch(err, 1);
      tc::mbar_wait(barL, 0);
    } else {
      tc::fence_after();
      s2_mma(tmem, uA, 128, uB, 128, kp, tc::idesc_bf16(128, 128));
      tc::mma_commit(barM);
      if (!tc::mbar_wait(barM, 0)) {
        fail = 1;
        atomicExch(err, 2);
        tc::mbar_wait(barM, 0);
      }
    }
  }
  __syncthreads();
  tc::fence_after();
  float* Ss = reinterpret_cast<float*>(smem);
  if (!fail) {
    const int lane_base = (warp & 3) * 32;
    const int row = lane_base + lane;
    for (int q = (warp >> 2) * 4; q < (warp >> 2) * 4 + 4; ++q) {
      float v[16];
      tmem_ld16x(tmem + ((uint32_t)lane_base << 16) + (uint32_t)(16 * q), v);
#pragma unroll
      for (int i = 0; i < 16; i += 4)
        *reinterpret_cast<float4*>(&Ss[row * S2_SS + 16 * q + i]) =
            make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
    }
  }
  tc::fence_before();
  __syncthreads();
  if (!fail) {
    if (interior) {
#pragma unroll
      for (int i = 0; i < S2_CHUNKS; ++i) {
        const int j = tid + i * S2_NT;
        const int r = j >> 5, c = (j & 31) * 4;
        epi.store4p(y0 + r, x0 + c, *reinterpret_cast<const float4*>(&Ss[r * S2_SS + c]),
                    pre[i], 4);
      }
    } else {
#pragma unroll 1
      for (int i = 0; i < S2_CHUNKS; ++i) {
        const int j = tid + i * S2_NT;
        const int r = j >> 5, c = (j & 31) * 4;
        const int m = y0 + r, n = x0 + c;
        const int nv = m < N ? min(4, N - n) : 0;
        if (nv > 0)
          epi.store4(m, n, *reinterpret_cast<const float4*>(&Ss[r * S2_SS + c]), nv);
      }
    }
  }
  epi.finish();
  if (warp == 0) tc::tmem_dealloc(tmem, 128);
}

template <class Epi>
static cudaError_t launch_tc2(cudaStream_t s, const void* Aimg, const void* Bimg, int N, int kp,
                              const Epi& e, int* err, int* nblocks, int batch) {
  const int smem = (int)tc2_synth_smem(kp);
  cudaError_t r = cudaFuncSetAttribute(synth_tc2_kernel<Epi>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (r != cudaSuccess) return r;
  dim3 grid((N + 127) / 128, (N + 127) / 128, batch);
  *nblocks = grid.x * grid.y;
  return launch_pdl(synth_tc2_kernel<Epi>, grid, dim3(S2_NT), (size_t)smem, s,
                    static_cast<const uint8_t*>(Aimg), static_cast<const uint8_t*>(Bimg), N, kp,
                    e, err);
}

// Images of the synthesis operands: rows of 128 (y for AY, x for Ut), K = kp.
size_t tc2_rows_image_bytes(int N, int kp) { return split2_image_bytes((N + 127) / 128, 128, 1, kp); }

cudaError_t launch_pack_tc2_rows(cudaStream_t s, const float* src, int N, int kp, void* dst) {
  return launch_pack_split2(s, src, 0, N, kp, kp, 128, kp, (N + 127) / 128, 1, dst);
}

cudaError_t launch_synth_resist_tc2(cudaStream_t s, const void* Aimg, const void* Bimg, int N,
                                    int kp, const ResistEpilogue& ep, int* err, int* nblocks,
                                    int batch) {
  const int vec = N % 4 == 0 && aligned16(ep.aerial) && aligned16(ep.wafer) &&
                  aligned16(ep.target) && aligned16(ep.pe_window) && aligned16(ep.pen_window) &&
                  aligned16(ep.dldi);
  return launch_tc2(s, Aimg, Bimg, N, kp, ResistEpiT<true>{ep, N, vec, 0.0, 0.0}, err,
                    nblocks, batch);
}

cudaError_t launch_synth_grad_tc2(cudaStream_t s, const void* Aimg, const void* Bimg, int N,
                                  int kp, const GradEpilogue& ep, int* err, int* nblocks,
                                  int batch) {
  const int vec = N % 4 == 0 && aligned16(ep.grad_mask) && aligned16(ep.theta) &&
                  aligned16(ep.grad_theta);
  return launch_tc2(s, Aimg, Bimg, N, kp, GradEpiT<true>{ep, N, vec, 0.0}, err, nblocks, batch);
}

// ---------------------------------------------------------------- fused resist + adjoint analysis
// For the CTM evaluation: per 128 x 128 tile, I = AYD . Ut^T in tensor memory; the
// resist epilogue (FP64 loss partials, optional aerial / wafer stores) turns I
// into dL/dI in registers, and dL/dI goes straight into shared memory as the
// [hi | lo] image operand of the adjoint tile analysis (TXD, TYD, conjugate rows),
// which leaves this tile's partial of the D-band spectrum of dL/dI. dL/dI is
// never written to global memory. Shared memory holds the synthesis operands,
// then the accumulator staging area with the TXD image tile behind it, then the
// dL/dI tile over the staging area, then the TYD image tile in its place.
constexpr uint32_t FUSED_TX_OFFSET = 68 * 1024;  // past the 128 x S2_SS float staging area
// dL/dI of an edge tile, written over this thread's own staging chunks. Kept out of
// line: inlined, its register demand spills the interior path.
__device__ __noinline__ void edge_dldi(ResistEpiT<true>& epi, float* Ss, int y0, int x0,
                                       int N) {
#pragma unroll 1
  for (int i = 0; i < S2_CHUNKS; ++i) {
    const int j = threadIdx.x + i * S2_NT;
    const int r = j >> 5, c = (j & 31) * 4;
    const int m = y0 + r, n = x0 + c;
    const int nv = m < N ? min(4, N - n) : 0;
    float4* sp = reinterpret_cast<float4*>(&Ss[r * S2_SS + c]);
    *sp = nv > 0 ? epi.dldi4(m, n, *sp, epi.pre4(m, n, nv), nv) : make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

template <int BN, bool PLAIN>
__global__ void __launch_bounds__(S2_NT, 2)
synth_resist_analysis_kernel(const uint8_t* __restrict__ Aimg, const uint8_t* __restrict__ Bimg,
                             int N, int kp, ResistEpiT<true> epi, Tc2Analysis a,
                             const uint8_t* __restrict__ txImg, const uint8_t* __restrict__ tyImg,
                             int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bars[6];  // [0..3] analysis stages, [4] operands, [5] synthesis
  __shared__ uint32_t tmem_slot;
  __shared__ int fail;
  constexpr uint32_t TX_BYTES = s2_tile_bytes(BN, 128);
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  uint8_t* sA = smem;                    // dL/dI tile, then the TYD image tile
  uint8_t* sB = smem + FUSED_TX_OFFSET;  // TXD image tile, then R
  float* Ss = reinterpret_cast<float*>(smem);  // accumulator staging [128][S2_SS]
  const uint32_t tile_bytes = s2_tile_bytes(128, kp);
  const uint32_t uA = tc::smem_u32(smem), uB = uA + tile_bytes;  // synthesis operands
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int xt = blockIdx.x, yt = blockIdx.y;
  const int x0 = xt * 128, y0 = yt * 128;
  const bool interior = epi.vec && y0 + 128 <= N && x0 + 128 <= N;
  const uint32_t barL = tc::smem_u32(&bars[4]), barM = tc::smem_u32(&bars[5]);
  pdl_trigger();
  if (tid == 0) {
    for (int i = 0; i < 6; ++i) tc::mbar_init(tc::smem_u32(&bars[i]), 1);
    fail = 0;
    tc::fence_mbar_init();
  }
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(&tmem_slot), 128);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tmem_slot;
  if (tid == 0) {
    tc::mbar_expect_tx(barL, 2 * tile_bytes);
    const uint8_t* ga = Aimg + (size_t)yt * tile_bytes;
    for (uint32_t q = 0; q < tile_bytes; q += 16384)
      tc::bulk_g2s(uA + q, ga + q, tile_bytes - q < 16384u ? tile_bytes - q : 16384u, barL);
  }
  pdl_wait();
  if (tid == 0) {
    // The band operand image of this launch's image blockIdx.z.
    const uint8_t* gb = Bimg + ((size_t)blockIdx.z * gridDim.x + xt) * tile_bytes;
    for (uint32_t q = 0; q < tile_bytes; q += 16384)
      tc::bulk_g2s(uB + q, gb + q, tile_bytes - q < 16384u ? tile_bytes - q : 16384u, barL);
  }
  // Targets of interior tiles, coalesced: chunk j covers row j / 32, columns
  // 4 (j % 32) .. + 3; the same registers later carry this thread's dL/dI.
  float4 pre[S2_CHUNKS];
  if (interior) {
#pragma unroll
    for (int i = 0; i < S2_CHUNKS; ++i) {
      const int j = tid + i * S2_NT;
      pre[i] = epi.pre4(y0 + (j >> 5), x0 + (j & 31) * 4, 4);
    }
  }
  if (tid == 0) {
    if (!tc::mbar_wait(barL, 0)) {
      fail = 1;
      atomicExch(err, 1);
      tc::mbar_wait(barL, 0);
    } else {
      tc::fence_after();
      s2_mma(tmem, uA, 128, uB, 128, kp, tc::idesc_bf16(128, 128));
      tc::mma_commit(barM);
      if (!tc::mbar_wait(barM, 0)) {
        fail = 1;
        atomicExch(err, 2);
        tc::mbar_wait(barM, 0);
      } else {
        // The synthesis operands are dead: the TXD tile loads behind the staging area.
        bulk_tile(tc::smem_u32(sB), txImg + (size_t)xt * TX_BYTES, TX_BYTES,
                  tc::smem_u32(&bars[0]));
      }
    }
  }
  __syncthreads();
  tc::fence_after();
  if (!fail) {
    const int lane_base = (warp & 3) * 32;
    const int row = lane_base + lane;
#pragma unroll 1
    for (int q = (warp >> 2) * 4; q < (warp >> 2) * 4 + 4; ++q) {
      float v[16];
      tmem_ld16x(tmem + ((uint32_t)lane_base << 16) + (uint32_t)(16 * q), v);
#pragma unroll
      for (int i = 0; i < 16; i += 4)
        *reinterpret_cast<float4*>(&Ss[row * S2_SS + 16 * q + i]) =
            make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
    }
  }
  tc::fence_before();
  __syncthreads();
  bool bad = false;
  if (!fail) {
    if (interior) {
#pragma unroll
      for (int i = 0; i < S2_CHUNKS; ++i) {
        const int j = tid + i * S2_NT;
        const int r = j >> 5, c = (j & 31) * 4;
        const float4 I4 = *reinterpret_cast<const float4*>(&Ss[r * S2_SS + c]);
        pre[i] = PLAIN ? epi.plain4(y0 + r, x0 + c, I4, pre[i])
                       : epi.dldi4(y0 + r, x0 + c, I4, pre[i], 4);
      }
    } else {
      // Edge tiles: dL/dI in place in the staging area, then into pre[] (a rolled
      // loop may not index pre[], which would move it to local memory).
      edge_dldi(epi, Ss, y0, x0, N);
#pragma unroll
      for (int i = 0; i < S2_CHUNKS; ++i) {
        const int j = tid + i * S2_NT;
        pre[i] = *reinterpret_cast<const float4*>(&Ss[(j >> 5) * S2_SS + (j & 31) * 4]);
      }
    }
  }
  __syncthreads();  // every read of the staging area is done: the dL/dI tile replaces it
  if (!fail) {
#pragma unroll
    for (int i = 0; i < S2_CHUNKS; ++i) {
      const int j = tid + i * S2_NT;
      const int r = j >> 5, c = (j & 31) * 4;
      const float4 g = pre[i];
      bad |= !(isfinite(g.x) && isfinite(g.y) && isfinite(g.z) && isfinite(g.w));
      uint2 h2, l2;
      split_pair(g.x, g.y, h2.x, l2.x);
      split_pair(g.z, g.w, h2.y, l2.y);
      *reinterpret_cast<uint2*>(sA + sw128_offset(128, r, c)) = h2;
      *reinterpret_cast<uint2*>(sA + sw128_offset(128, r, 128 + c)) = l2;
    }
  }
  if (bad) atomicOr(a.flag, 1);
  epi.finish();
  tc::fence_before();
  analysis_stages<BN>(sA, sB, bars, tmem, &fail, a, tyImg, xt, yt, err);
  tc::fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 128);
}

template <int BN, bool PLAIN>
static cudaError_t fused_v(cudaStream_t s, const void* Aimg, const void* Bimg, int N, int kp,
                          const ResistEpiT<true>& e, const Tc2Analysis& a, const void* tx,
                          const void* ty, int* err, int* nblocks, int batch) {
  const size_t ops = 2 * (size_t)s2_tile_bytes(128, kp);
  const size_t ana = (size_t)FUSED_TX_OFFSET + s2_tile_bytes(BN, 128);
  const size_t smem = (ops > ana ? ops : ana) + 1024;
  cudaError_t r = cudaFuncSetAttribute(synth_resist_analysis_kernel<BN, PLAIN>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (r != cudaSuccess) return r;
  dim3 grid((N + 127) / 128, (N + 127) / 128, batch);
  *nblocks = grid.x * grid.y;
  return launch_pdl(synth_resist_analysis_kernel<BN, PLAIN>, grid, dim3(S2_NT), smem, s,
                    static_cast<const uint8_t*>(Aimg), static_cast<const uint8_t*>(Bimg), N, kp, e,
                    a, static_cast<const uint8_t*>(tx), static_cast<const uint8_t*>(ty), err);
}

// No window and no penalty (the CTM evaluation) takes a leaner epilogue: the general one
// needs more than the 128 registers of two CTAs per SM.
template <int BN>
static cudaError_t fused_t(cudaStream_t s, const void* Aimg, const void* Bimg, int N, int kp,
                          const ResistEpiT<true>& e, const Tc2Analysis& a, const void* tx,
                          const void* ty, int* err, int* nblocks, int batch) {
  return e.plain() ? fused_v<BN, true>(s, Aimg, Bimg, N, kp, e, a, tx, ty, err, nblocks, batch)
                   : fused_v<BN, false>(s, Aimg, Bimg, N, kp, e, a, tx, ty, err, nblocks, batch);
}

cudaError_t launch_synth_resist_analysis_tc2(cudaStream_t s, const void* Aimg, const void* Bimg,
                                             int N, int kp, const ResistEpilogue& ep, int ncols,
                                             int nr, float2* part, int* flag, const void* tx_img,
                                             const void* ty_img, int* err, int* nblocks,
                                             int batch) {
  const int vec = N % 4 == 0 && aligned16(ep.aerial) && aligned16(ep.wafer) &&
                  aligned16(ep.target) && aligned16(ep.pe_window) && aligned16(ep.pen_window);
  if ((size_t)(2 * nr - 1) * ncols * sizeof(float2) > A2_A_BYTES) return cudaErrorInvalidValue;
  const ResistEpiT<true> e{ep, N, vec, 0.0, 0.0};
  const Tc2Analysis a{nullptr, nullptr, flag, N, 0, 0, ncols, 2 * nr - 1, nr, 1, part};
  switch (tc2_analysis_rows(ncols)) {
    case 16: return fused_t<16>(s, Aimg, Bimg, N, kp, e, a, tx_img, ty_img, err, nblocks, batch);
    case 32: return fused_t<32>(s, Aimg, Bimg, N, kp, e, a, tx_img, ty_img, err, nblocks, batch);
    case 48: return fused_t<48>(s, Aimg, Bimg, N, kp, e, a, tx_img, ty_img, err, nblocks, batch);
    case 64: return fused_t<64>(s, Aimg, Bimg, N, kp, e, a, tx_img, ty_img, err, nblocks, batch);
    case 80: return fused_t<80>(s, Aimg, Bimg, N, kp, e, a, tx_img, ty_img, err, nblocks, batch);
    case 96: return fused_t<96>(s, Aimg, Bimg, N, kp, e, a, tx_img, ty_img, err, nblocks, batch);
    case 112: return fused_t<112>(s, Aimg, Bimg, N, kp, e, a, tx_img, ty_img, err, nblocks, batch);
    case 128: return fused_t<128>(s, Aimg, Bimg, N, kp, e, a, tx_img, ty_img, err, nblocks, batch);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace litho_b200
