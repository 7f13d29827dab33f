// Row synthesis on the 5th-generation tensor cores (tcgen05, sm_100a).
//
//   out[y][x] = sum_f AY[y][f] Ut[x][f]          (f < kp, kp = 2 Nr rounded to 16)
//
// in split-BF16: every FP32 operand v = hi + lo with hi = bf16(v) and
// lo = bf16(v - hi); the three-pass product a_hi b_hi + a_hi b_lo + a_lo b_hi is
// one BF16 GEMM over a tripled inner dimension,
//   A3[y] = [AY_hi | AY_hi | AY_lo],   B3[x] = [Ut_hi | Ut_lo | Ut_hi],
// accumulated in FP32 in tensor memory. Operands live in global memory as
// "images" already in the UMMA canonical K-major 128-byte-swizzle layout, so
// each CTA fetches them with plain bulk copies (cp.async.bulk, the TMA engine)
// into shared memory; one thread issues the tcgen05.mma chain (M = 128,
// N = 256, K = 16 per instruction); after the commit barrier the 8 warps read
// the accumulator with tcgen05.ld, stage 32-column slices through shared
// memory and run the fused epilogue with coalesced global accesses.
//
// Every mbarrier wait is bounded by a clock budget; on expiry the kernel
// records a code in *err, skips the remaining work, releases its tensor memory
// and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "tc_ptx.cuh"

namespace litho_b200 {



constexpr int TC_M = 128, TC_N = 256, TC_KC = 256;  // tile rows, tile columns, K per chunk
constexpr int TC_NT = 256;
constexpr uint32_t TC_A_BYTES = TC_M * TC_KC * 2;   // 64 KiB
constexpr uint32_t TC_B_BYTES = TC_N * TC_KC * 2;   // 128 KiB
constexpr int TC_SS = TC_N + 4;                     // staging row stride (floats)

// ---------------------------------------------------------------- operand images
// Image of a [rows][kp] FP32 matrix as split-BF16 K-major SW128 tiles:
// tile t = rows [t*tile_rows, (t+1)*tile_rows), chunk ch = K [256 ch, 256 ch + 256),
// atom column kb (64 K each), 8-row groups 1024 bytes apart, 16-byte chunk c of
// row r stored at position c ^ (r % 8). order 0: [hi, hi, lo]; order 1: [hi, lo, hi];
// K beyond 3 kp is zero, rows beyond 'rows' are zero.
__global__ void pack_split_kernel(const float* __restrict__ src, int rows, int kp, int tile_rows,
                                  int nchunks, int order, uint4* __restrict__ dst,
                                  size_t n16) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n16) return;
  // idx enumerates (tile, chunk, kb, r, c) with c fastest.
  const int c = (int)(idx % 8);
  size_t rest = idx / 8;
  const int r = (int)(rest % tile_rows);
  rest /= tile_rows;
  const int kb = (int)(rest % 4);
  rest /= 4;
  const int ch = (int)(rest % nchunks);
  const int t = (int)(rest / nchunks);
  const int row = t * tile_rows + r;
  __nv_bfloat16 out[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int k = ch * TC_KC + kb * 64 + c * 8 + q;
    const int sec = k / kp, f = k % kp;
    float v = 0.f;
    if (sec < 3 && row < rows) v = src[(size_t)row * kp + f];
    const __nv_bfloat16 hi = __float2bfloat16_rn(v);
    const __nv_bfloat16 lo = __float2bfloat16_rn(v - __bfloat162float(hi));
    const bool want_lo = (order == 0) ? (sec == 2) : (sec == 1);
    out[q] = (sec < 3) ? (want_lo ? lo : hi) : __float2bfloat16_rn(0.f);
  }
  const size_t tile_base = ((size_t)t * nchunks + ch) * 4 + kb;
  const size_t off16 = tile_base * (size_t)tile_rows * 8 + (size_t)(r / 8) * 64 +
                       (size_t)(r % 8) * 8 + (size_t)(c ^ (r % 8));
  dst[off16] = *reinterpret_cast<const uint4*>(out);
}

int tc_chunks(int kp) { return (3 * kp + TC_KC - 1) / TC_KC; }

size_t tc_image_bytes(int rows, int kp, int tile_rows) {
  const size_t tiles = (size_t)(rows + tile_rows - 1) / tile_rows;
  return tiles * (size_t)tc_chunks(kp) * (size_t)tile_rows * TC_KC * 2;
}

cudaError_t launch_pack_split(cudaStream_t s, const float* src, int rows, int kp, int tile_rows,
                              int order, void* dst) {
  const int nch = tc_chunks(kp);
  const size_t tiles = (size_t)(rows + tile_rows - 1) / tile_rows;
  const size_t n16 = tiles * nch * 4 * (size_t)tile_rows * 8;
  pack_split_kernel<<<(unsigned)((n16 + 255) / 256), 256, 0, s>>>(
      src, rows, kp, tile_rows, nch, order, reinterpret_cast<uint4*>(dst), n16);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- the GEMM
template <class Epi>
__global__ void __launch_bounds__(TC_NT, 1)
synth_tc_kernel(const uint8_t* __restrict__ Aimg, const uint8_t* __restrict__ Bimg, int N,
                int nchunks, int ksteps_total, Epi epi, int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ uint32_t tmem_slot;
  __shared__ int fail;
  // 1024-byte alignment of the operand tiles (the swizzle pattern is anchored there).
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  uint8_t* sA = smem;
  uint8_t* sB = smem + TC_A_BYTES;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int xt = blockIdx.x, yt = blockIdx.y;
  const uint32_t barL = tc::smem_u32(&bars[0]), barM = tc::smem_u32(&bars[1]);
  if (tid == 0) {
    tc::mbar_init(barL, 1);
    tc::mbar_init(barM, 1);
    fail = 0;
    tc::fence_mbar_init();
  }
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(&tmem_slot), TC_N);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tmem_slot;
  constexpr uint32_t idesc = tc::idesc_bf16(TC_M, TC_N);

  for (int ch = 0; ch < nchunks; ++ch) {
    if (tid == 0) {
      tc::mbar_expect_tx(barL, TC_A_BYTES + TC_B_BYTES);
      const uint8_t* ga = Aimg + ((size_t)yt * nchunks + ch) * TC_A_BYTES;
      const uint8_t* gb = Bimg + ((size_t)xt * nchunks + ch) * TC_B_BYTES;
      for (uint32_t q = 0; q < TC_A_BYTES; q += 16384)
        tc::bulk_g2s(tc::smem_u32(sA) + q, ga + q, 16384, barL);
      for (uint32_t q = 0; q < TC_B_BYTES; q += 16384)
        tc::bulk_g2s(tc::smem_u32(sB) + q, gb + q, 16384, barL);
      if (!tc::mbar_wait(barL, ch & 1)) {
        fail = 1;
        atomicExch(err, 1);
      } else {
        tc::fence_after();
        const int ks = min(16, ksteps_total - 16 * ch);
        for (int st = 0; st < ks; ++st) {
          const int kb = st >> 2;
          const uint32_t ko = (uint32_t)(st & 3) * 32;
          const uint64_t ad = tc::desc_sw128(tc::smem_u32(sA) + kb * (TC_M * 128) + ko);
          const uint64_t bd = tc::desc_sw128(tc::smem_u32(sB) + kb * (TC_N * 128) + ko);
          tc::mma_bf16(tmem, ad, bd, idesc, (ch > 0 || st > 0) ? 1u : 0u);
        }
        tc::mma_commit(barM);
        if (!tc::mbar_wait(barM, ch & 1)) {
          fail = 2;
          atomicExch(err, 2);
          // The MMA may still be in flight: give it one more bounded wait before
          // the tensor memory is released below.
          tc::mbar_wait(barM, ch & 1);
        }
      }
    }
    __syncthreads();
    if (fail) break;
  }
  tc::fence_after();

  if (!fail) {
    // Epilogue. The whole 128 x 256 FP32 accumulator is staged in shared memory
    // (the operand tiles are dead): warps w and w + 4 read TMEM lanes 32 (w % 4)
    // .. + 31, warps 0-3 columns [0, 128), warps 4-7 [128, 256), and store rows
    // with 16-byte writes (row stride TC_SS, conflict-free per quarter warp).
    // Then all threads run the fused epilogue over 16-byte column chunks, four
    // chunks per batch so that their global loads overlap.
    float* stg = reinterpret_cast<float*>(smem);
    const int lane_base = (warp & 3) * 32;
    const int half = warp >> 2;
    const int y0 = yt * TC_M, x0 = xt * TC_N;
    for (int rd = 0; rd < 4; ++rd) {
      const int col = half * 128 + rd * 32;
      float v[32];
      tc::tmem_ld32(tmem + ((uint32_t)lane_base << 16) + (uint32_t)col, v);
      float* row = stg + (size_t)(lane_base + lane) * TC_SS + col;
#pragma unroll
      for (int i = 0; i < 32; i += 4)
        *reinterpret_cast<float4*>(row + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
    }
    __syncthreads();
    constexpr int CH = TC_N / 4;                 // float4 chunks per row
    constexpr int V = 4;
    for (int base = tid; base < TC_M * CH; base += TC_NT * V) {
      int m[V], n[V], nv[V];
      float4 val[V];
#pragma unroll
      for (int q = 0; q < V; ++q) {
        const int idx = base + q * TC_NT;
        const int r = idx / CH, c4 = (idx % CH) * 4;
        m[q] = y0 + r;
        n[q] = x0 + c4;
        nv[q] = (idx < TC_M * CH && m[q] < N && n[q] < N) ? min(4, N - n[q]) : 0;
        val[q] = nv[q] > 0 ? *reinterpret_cast<const float4*>(stg + (size_t)r * TC_SS + c4)
                           : make_float4(0.f, 0.f, 0.f, 0.f);
      }
      epi.template store4v<V>(m, n, val, nv);
    }
  }
  epi.finish();
  tc::fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, TC_N);
}

static size_t tc_smem_bytes() { return TC_A_BYTES + TC_B_BYTES + 1024; }

template <class Epi>
static cudaError_t launch_tc(cudaStream_t s, const void* Aimg, const void* Bimg, int N, int kp,
                             const Epi& e, int* err, int* nblocks) {
  const int smem = (int)tc_smem_bytes();
  cudaError_t r = cudaFuncSetAttribute(synth_tc_kernel<Epi>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (r != cudaSuccess) return r;
  dim3 grid((N + TC_N - 1) / TC_N, (N + TC_M - 1) / TC_M);
  *nblocks = grid.x * grid.y;
  const int nch = tc_chunks(kp);
  const int ksteps = (3 * kp + 15) / 16;
  synth_tc_kernel<Epi><<<grid, TC_NT, smem, s>>>(static_cast<const uint8_t*>(Aimg),
                                                 static_cast<const uint8_t*>(Bimg), N, nch,
                                                 ksteps, e, err);
  return cudaGetLastError();
}

cudaError_t launch_synth_resist_tc(cudaStream_t s, const void* Aimg, const void* Bimg, int N,
                                   int kp, const ResistEpilogue& ep, int* err, int* nblocks) {
  const int vec = N % 4 == 0 && aligned16(ep.aerial) && aligned16(ep.wafer) &&
                  aligned16(ep.target) && aligned16(ep.pe_window) && aligned16(ep.pen_window) &&
                  aligned16(ep.dldi);
  return launch_tc(s, Aimg, Bimg, N, kp, ResistEpi{ep, N, vec, 0.0, 0.0}, err, nblocks);
}

cudaError_t launch_synth_grad_tc(cudaStream_t s, const void* Aimg, const void* Bimg, int N, int kp,
                                 const GradEpilogue& ep, int* err, int* nblocks) {
  const int vec = N % 4 == 0 && aligned16(ep.grad_mask) && aligned16(ep.theta) &&
                  aligned16(ep.grad_theta);
  return launch_tc(s, Aimg, Bimg, N, kp, GradEpi{ep, N, vec, 0.0}, err, nblocks);
}

}  // namespace litho_b200
