// Split-BF16 ("split2") operand images and their tcgen05 helpers, shared by the
// per-tile kernels (tc2.cu) and the persistent pipelined kernels (tc3.cu).
//
// A tile of RB rows x K FP32 values (K % 16 == 0), v = hi + lo with hi = bf16(v),
// lo = bf16(v - hi), is stored as one K-major 128-byte-swizzle UMMA tile with 2K
// columns [hi | lo]: element (r, k) has hi at sw128_offset(RB, r, k) and lo at
// sw128_offset(RB, r, K + k). The three-pass product a_hi b_hi + a_hi b_lo + a_lo b_hi
// is three MMA sections over the same two tiles, accumulated in FP32 in tensor memory.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "tc_ptx.cuh"

namespace litho_b200 {

__host__ __device__ constexpr uint32_t s2_atoms(int K) { return (uint32_t)(2 * K + 63) / 64; }
__host__ __device__ constexpr uint32_t s2_tile_bytes(int RB, int K) {
  return s2_atoms(K) * (uint32_t)RB * 128u;
}

// Descriptor of the 16-wide K step starting at column k of a split2 tile with RB rows.
__device__ __forceinline__ uint64_t s2_desc(uint32_t base, int RB, int k) {
  return tc::desc_sw128(base + (uint32_t)(k / 64) * (uint32_t)RB * 128u +
                        (uint32_t)((k % 64) / 16) * 32u);
}

// The three split-BF16 sections of D[M][N] = A[M][K] . B[N][K]^T (K % 16 == 0):
// 3 K / 16 tcgen05.mma instructions, issued by one thread.
__device__ __forceinline__ void s2_mma(uint32_t tmem, uint32_t sa, int ra, uint32_t sb, int rb,
                                       int K, uint32_t idesc) {
  const int aoff[3] = {0, 0, K}, boff[3] = {0, K, 0};
  bool first = true;
  for (int s = 0; s < 3; ++s)
    for (int k = 0; k < K; k += 16) {
      tc::mma_bf16(tmem, s2_desc(sa, ra, aoff[s] + k), s2_desc(sb, rb, boff[s] + k), idesc,
                   first ? 0u : 1u);
      first = false;
    }
}

__device__ __forceinline__ void split_bf16(float v, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(v);
  lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}
// The same split for two values with packed conversions: hi2 / lo2 hold (a, b)
// as consecutive bf16 (a at the lower address).
__device__ __forceinline__ void split_pair(float a, float b, uint32_t& hi2, uint32_t& lo2) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(a - hf.x, b - hf.y);
  hi2 = *reinterpret_cast<const uint32_t*>(&h);
  lo2 = *reinterpret_cast<const uint32_t*>(&l);
}

// The same three sections with the operands' roles exchanged: D = B . A^T from the
// tiles of D^T = A . B^T, D[M][N] = Bt[M][K] . At[N][K]^T with M from the tile sb and N
// from sa. Every element sums the same products in the same order as s2_mma on
// (sa, sb): a_hi b_hi, then a_hi b_lo, then a_lo b_hi.
__device__ __forceinline__ void s2_mma_swapped(uint32_t tmem, uint32_t sa, int ra, uint32_t sb,
                                               int rb, int K, uint32_t idesc) {
  const int aoff[3] = {0, 0, K}, boff[3] = {0, K, 0};
  bool first = true;
  for (int s = 0; s < 3; ++s)
    for (int k = 0; k < K; k += 16) {
      tc::mma_bf16(tmem, s2_desc(sb, rb, boff[s] + k), s2_desc(sa, ra, aoff[s] + k), idesc,
                   first ? 0u : 1u);
      first = false;
    }
}

// MN-major split tile of a 128 (M) x 128 (K) block, 128-byte swizzle: for each k the
// 128 rows m lie in two 64-row atoms (LBO = 1024 bytes apart), 8 consecutive k form
// one 1024-byte atom group (SBO = 2048 bytes apart). Element (m, k) of the hi part is
// at byte
//   (k / 8) * 2048 + (m / 64) * 1024 + (k % 8) * 128 + ((((m % 64) / 8) ^ (k % 8)) * 16)
//   + (m % 8) * 2,
// the lo part MN_LO bytes further; 64 KiB in all, base 1024-byte aligned. A thread
// that holds 8 consecutive rows m of one column k writes them as one 16-byte chunk.
constexpr uint32_t MN_LBO = 1024, MN_SBO = 2048, MN_LO = 32768;
__host__ __device__ constexpr uint32_t mn_chunk_offset(uint32_t m, uint32_t k) {
  return (k >> 3) * MN_SBO + (m >> 6) * MN_LBO + (k & 7u) * 128u +
         ((((m & 63u) >> 3) ^ (k & 7u)) << 4);
}
// Shared-memory descriptor of the MN-major layout above (sm_100 version bit, SW128).
__device__ __forceinline__ uint64_t desc_mn_sw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)(MN_LBO >> 4) << 16;
  d |= (uint64_t)(MN_SBO >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}
// Instruction-descriptor bit: operand A is MN-major.
constexpr uint32_t IDESC_A_MN = 1u << 15;

// s2_mma with A (M = 128 rows, K = 128) in the MN-major split layout at sa (hi) and
// sa + MN_LO (lo): the same three sections and K steps in the same order. idesc must
// carry IDESC_A_MN.
__device__ __forceinline__ void s2_mma_amn(uint32_t tmem, uint32_t sa, uint32_t sb, int rb, int K,
                                           uint32_t idesc) {
  const uint32_t aoff[3] = {0u, 0u, MN_LO};
  const int boff[3] = {0, K, 0};
  bool first = true;
  for (int s = 0; s < 3; ++s)
    for (int k = 0; k < K; k += 16) {
      tc::mma_bf16(tmem, desc_mn_sw128(sa + aoff[s] + (uint32_t)k * 256u),
                   s2_desc(sb, rb, boff[s] + k), idesc, first ? 0u : 1u);
      first = false;
    }
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16x(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Bulk copy of `bytes` (a multiple of 16) in pieces of at most 16 KiB onto mbarrier
// `bar`, without announcing the bytes (bulk_tile announces them).
__device__ __forceinline__ void bulk_chunks(uint32_t dst, const uint8_t* src, uint32_t bytes,
                                            uint32_t bar) {
  for (uint32_t q = 0; q < bytes; q += 16384) {
    const uint32_t n = bytes - q < 16384u ? bytes - q : 16384u;
    tc::bulk_g2s(dst + q, src + q, n, bar);
  }
}
__device__ __forceinline__ void bulk_tile(uint32_t dst, const uint8_t* src, uint32_t bytes,
                                          uint32_t bar) {
  tc::mbar_expect_tx(bar, bytes);
  bulk_chunks(dst, src, bytes, bar);
}

constexpr uint32_t A2_A_BYTES = s2_tile_bytes(128, 128);   // 64 KiB: a 128 x 128 image tile

// Arguments of a tile analysis (tc2.cu, tc3.cu): for every 128 x 128 tile of the image
// in (mode 1: theta, analysed as (1 + cos theta) / 2 and optionally stored to mask_out),
// the band partial part[image][yt][xt][row][c] (ncols complex columns, nrows_out rows;
// sym: rows -nr+1 .. nr-1 from the conjugate symmetry of a real image).
struct Tc2Analysis {
  const float* in;
  float* mask_out;
  int* flag;
  int N, mode, vec4;
  int ncols;           // complex band columns (BN >= 2 ncols)
  int nrows_out, nr, sym;
  float2* part;
};

// Rows of the tile-analysis operand TX for ncols complex columns (2 ncols rounded to 16).
int tc2_analysis_rows(int ncols);

}  // namespace litho_b200
