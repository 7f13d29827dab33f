// Persistent, warp-specialised split-BF16 tensor-core passes (tcgen05, sm_100a).
//
// The per-tile kernels of tc2.cu run one 128 x 128 tile per CTA, two CTAs per SM,
// each CTA through its phases in order (operand copies, MMA, tensor-memory
// read-back, epilogue). The kernels here run one CTA per SM over a contiguous share
// of the work items (image z, tile row yt, tile column xt; images fastest, so
// consecutive items of a CTA share their tile's constant operand images, which
// stay in shared memory), with each phase in its own warps and the phases of
// neighbouring items overlapped:
//   * loader / epilogue warps move image data between global memory and shared or
//     tensor memory;
//   * one thread issues the bulk copies of the constant operand images and every
//     tcgen05.mma, and commits each MMA group to an mbarrier;
//   * the accumulators are double-buffered in tensor memory, so the epilogue of
//     item j runs while the MMAs of item j + 1 do.
// The roles hand buffers to each other through mbarriers (full / free per buffer,
// phase parity per use). Every wait is bounded: on expiry, or when another role has
// given up, a role records a code in *err (first failure only) and leaves its loop;
// the MMA thread then waits (bounded) for its own copies and MMAs in flight, the
// tensor memory is released and the kernel returns.
//
// The syntheses compute the transposed accumulator D[x][y] (tensor-memory lane =
// image column x) so that the 32 lanes of a warp touch 32 consecutive pixels of an
// image row: every global access of the epilogues is a fully used 128-byte line,
// with no staging through shared memory. Per element the products and their order
// are those of the per-tile kernels (s2_mma_swapped), so images agree bit for bit.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "tc_ptx.cuh"
#include "tc_split2.cuh"

namespace litho_b200 {

namespace {

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ uint8_t* align1024(uint8_t* p) {
  return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 1023) &
                                    ~static_cast<uintptr_t>(1023));
}

// Bounded wait for the completion of the phase of `bar` with parity `parity`. Gives
// up when another role has failed (*fail) or after about 2^31 SM cycles (one second),
// then records `code` in *err (first failure wins) and returns false.
__device__ __forceinline__ bool pwait(uint32_t bar, uint32_t parity, volatile int* fail, int* err,
                                      int code) {
  const long long t0 = clock64();
  while (!tc::mbar_try_wait(bar, parity)) {
    if (*fail) return false;
    if (clock64() - t0 > (1LL << 31)) {
      *fail = 1;
      atomicCAS(err, 0, code);
      return false;
    }
  }
  return true;
}

// This CTA's contiguous share [lo, hi) of `items` work items.
__device__ __forceinline__ void my_items(int items, int& lo, int& hi) {
  lo = (int)((long long)blockIdx.x * items / gridDim.x);
  hi = (int)((long long)(blockIdx.x + 1) * items / gridDim.x);
}
struct Item {
  int z, yt, xt;
};
// Item it of T x T tiles x B images, images fastest.
__device__ __forceinline__ Item item_at(int it, int T, int B) {
  Item r;
  r.z = it % B;
  const int t = it / B;
  r.xt = t % T;
  r.yt = t / T;
  return r;
}
// The item after it (no division: a role walks its items in order).
__device__ __forceinline__ Item item_next(Item it, int T, int B) {
  if (++it.z == B) {
    it.z = 0;
    if (++it.xt == T) {
      it.xt = 0;
      ++it.yt;
    }
  }
  return it;
}

// Per-item FP64 partial sums of the epilogue warps without a CTA barrier (a warp that
// leaves its loop on a failed wait must not strand the others): every warp adds its
// lanes' values in a fixed shuffle order and its lane 0 stores them in slot b = j & 3
// and arrives on red_bar[b] (count = epilogue warps); a collecting thread waits for
// the slot (bounded), adds the warps in order and writes the partials: thread 0 right
// after its own part (fused kernel), or, in the syntheses, one warp in turn during its
// item j + 1 (collect2). Either reads slot b before it reads the accumulator of item
// j + 2, and no warp reaches item j + 4, which writes slot b again, before every warp
// has read the accumulator of item j + 2 (the accumulators are double-buffered), so a
// slot is read before it is written again.
constexpr int EPI_SLOTS = 4;
template <int NV>
struct EpiSums {
  double v[EPI_SLOTS][16][NV];
};
template <int NV>
__device__ __forceinline__ void epi_put(EpiSums<NV>& sh, uint32_t red_bar, int b,
                                        const double (&v)[NV]) {
  double t[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    t[k] = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t[k] += __shfl_xor_sync(0xffffffffu, t[k], o);
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) sh.v[b][threadIdx.x >> 5][k] = t[k];
    mbar_arrive(red_bar);
  }
}
// The slot's sums over nw warps, added in warp order (false when the wait gave up).
template <int NV>
__device__ __forceinline__ bool epi_take(const EpiSums<NV>& sh, uint32_t red_bar, int b,
                                         uint32_t parity, int nw, volatile int* fail, int* err,
                                         int code, double (&out)[NV]) {
  if (!pwait(red_bar, parity, fail, err, code)) return false;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    out[k] = 0.0;
    for (int w = 0; w < nw; ++w) out[k] += sh.v[b][w][k];
  }
  return true;
}

// L2 prefetch of the row segment of this lane for a later item: the line holding row
// yb + lane, column x0 of image img (N x N floats), when columns x0 .. x0 + 31 lie
// inside the image and pf (N % 4 == 0, 16-byte aligned image base) holds.
__device__ __forceinline__ void prefetch_rows(const float* img, int N, int yb, int x0, bool pf) {
  const int y = yb + (int)(threadIdx.x & 31);
  if (pf && y < N && x0 + 32 <= N) tc::prefetch_l2_line(img + (size_t)y * N + x0);
}

// The sums of item j (slot j & 3) over nw warps into out[0 .. nv - 1], by lane 0 of the
// warp that collects item j (false when the wait gave up). Item j is collected by warp
// j % nw one item later, when every warp has normally stored its part, so that no warp
// waits for the others in the common case.
__device__ __forceinline__ bool collect2(const EpiSums<2>& sh, uint64_t* red_bar, int j, int nw,
                                         volatile int* fail, int* err, int code, double* out,
                                         int nv) {
  double t[2];
  if (!epi_take<2>(sh, tc::smem_u32(&red_bar[j & 3]), j & 3, (j >> 2) & 1, nw, fail, err, code,
                   t))
    return false;
  out[0] = t[0];
  if (nv > 1) out[1] = t[1];
  return true;
}

// R (tensor memory: lanes y = lane_base + lane, columns f) -> sR, the K-major
// [hi | lo] operand of stage 2 (rows f, K = y), for the 16-column groups q0, q0 + dq,
// .. of BN. The words (f, y & ~1) hold the pair of lanes y & ~1 and y | 1: for each
// pair of columns (f, f + 1) the even lane splits and stores column f (hi and lo
// word), the odd lane column f + 1, after one exchange of values between the two.
// acc: the accumulator's address with this warp's lane base.
template <int BN>
__device__ __forceinline__ void r_to_operand(uint32_t acc, uint8_t* sR, int lane_base, int q0,
                                             int dq) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t ye = ((uint32_t)lane_base + lane) & ~1u;
  const uint32_t odd = lane & 1u;
  // sw128_offset(BN, f, k) for f = 16 q + i + odd, k = ye (hi) or 128 + ye (lo): the
  // part that depends on (f % 8), and the 1024-byte groups of 8 rows f / 8
  uint32_t off[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint32_t f8 = 2u * i + odd;
    off[i] = (ye >> 6) * (uint32_t)BN * 128u + f8 * 128u + ((((ye & 63u) >> 3) ^ f8) << 4) +
             (ye & 7u) * 2u;
  }
  constexpr uint32_t LO = 2u * (uint32_t)BN * 128u;   // k + 128: two atoms further
#pragma unroll 1
  for (int q = q0; q < BN / 16; q += dq) {
    float rv[16];
    tmem_ld16x(acc + (uint32_t)(16 * q), rv);
    uint8_t* sq = sR + (uint32_t)q * 2048u;
#pragma unroll
    for (int i = 0; i < 16; i += 2) {
      // the even lane receives its partner's column i, the odd lane column i + 1
      const float got = __shfl_xor_sync(0xffffffffu, odd ? rv[i] : rv[i + 1], 1);
      uint32_t h2, l2;
      split_pair(odd ? got : rv[i], odd ? rv[i + 1] : got, h2, l2);
      uint8_t* w = sq + (uint32_t)(i >> 3) * 1024u + off[(i & 7) >> 1];
      *reinterpret_cast<uint32_t*>(w) = h2;
      *reinterpret_cast<uint32_t*>(w + LO) = l2;
    }
  }
}

// Q (tensor memory: lanes n = 2 r + s, columns f = 2 c + t) -> the tile's partials
// P[r][c] of the band (see analysis_stages in tc2.cu): Re = Q[2r][2c] - Q[2r+1][2c+1],
// Im = Q[2r][2c+1] + Q[2r+1][2c]; with sym also the conjugate rows -r (from the odd
// lane of the pair). The tile's block is stored column-major, P[c][row] at
// out + c nrows_out + row, so that a warp's store of one column touches two runs of
// consecutive rows instead of 32 rows ncols apart (reduce_tiles_kernel with trows =
// nrows_out reads this layout).
template <int BN>
__device__ __forceinline__ void q_to_partials(uint32_t acc, float2* out, const Tc2Analysis& a,
                                              int lane_base, int q0, int dq) {
  const int lane = threadIdx.x & 31;
  const int nn = lane_base + lane;
  const int r = nn >> 1, s = nn & 1;
  // the output row of this lane, or none
  float2* row = nullptr;
  if (r < a.nr) {
    if (!a.sym)
      row = s == 0 ? out + r : nullptr;
    else if (s == 0)
      row = out + (a.nr - 1 + r);
    else if (r >= 1)
      row = out + (a.nr - 1 - r);
  }
#pragma unroll 1
  for (int q = q0; q < BN / 16; q += dq) {
    float qv[16], pv[16];
    tmem_ld16x(acc + (uint32_t)(16 * q), qv);
#pragma unroll
    for (int i = 0; i < 16; ++i) pv[i] = __shfl_xor_sync(0xffffffffu, qv[i], 1);
    if (row == nullptr) continue;
    float2* rq = row + (size_t)(8 * q) * a.nrows_out;
    const int nc = a.ncols - 8 * q;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if (i >= nc) break;
      const float o0 = qv[2 * i], o1 = qv[2 * i + 1], p0 = pv[2 * i], p1 = pv[2 * i + 1];
      rq[(size_t)i * a.nrows_out] = s == 0 ? make_float2(o0 - p1, o1 + p0)
                                           : make_float2(p0 + o1, p1 - o0);
    }
  }
}

int sm_count() {
  static int count[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!count[dev]) {
    int c = 0;
    if (cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || c <= 0)
      c = 148;
    count[dev] = c;
  }
  return count[dev];
}

}  // namespace

// =============================================================== tile analysis
// The partials of launch_analysis_tc2 (same products, same order, same layout
// part[image][yt][xt][row][c]) from a persistent pipeline:
//   warps 0-15  load the image tile (theta -> mask for mode 1), split it into the
//               [hi | lo] operand sA;
//   warp 24     (one thread) copies the TX tile (per xt) and the TY tile (per yt),
//               issues stage 1 R = sA . TX^T into accR[j & 1] and stage 2
//               Q = TY . R^T into accQ[j & 1];
//   warps 16-23 turn R into the stage-2 operand sR, and Q into the item's partials
//               (two warps per lane quarter, each taking every other 16-column group).
// Shared memory: TY 64 KiB | sA 64 KiB | TX | sR (BN x 128 split tiles, BN <= 96).
// Tensor memory: 512 columns, accR[b] at 128 b, accQ[b] at 256 + 128 b.
// A3_TMW TMEM warps: warps A3_LOADW + i and A3_LOADW + i + 4 share the lane quarter i
// of the accumulators and split its 16-column groups (even / odd).
constexpr int A3_LOADW = 16, A3_TMW = 8, A3_MMAW = A3_LOADW + A3_TMW;
constexpr int A3_NT = (A3_MMAW + 1) * 32;
// chunks of 8 pixels per loader thread, rows between a thread's chunks
constexpr int A3_CH = 2048 / (32 * A3_LOADW), A3_RS = 2 * A3_LOADW;

template <int BN, int MODE>
__global__ void __launch_bounds__(A3_NT, 1)
analysis_tc3_kernel(Tc2Analysis a, int T, int B, const uint8_t* __restrict__ txImg,
                    const uint8_t* __restrict__ tyImg, int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 0 sA full (16 loader warps), 1-2 stage 1 done [b], 3 sR full (8 TMEM warps),
  // 4-5 stage 2 done [b], 6-7 accQ[b] free (8 TMEM warps), 8 TX landed, 9 TY landed
  __shared__ __align__(8) uint64_t bars[10];
  __shared__ uint32_t tmem_slot;
  __shared__ int fail;
  constexpr uint32_t TXB = s2_tile_bytes(BN, 128);
  uint8_t* smem = align1024(smem_raw);
  uint8_t* sA = smem + A2_A_BYTES;
  uint8_t* sR = smem + 2 * A2_A_BYTES + TXB;
  const uint32_t uTY = tc::smem_u32(smem), uA = tc::smem_u32(sA);
  const uint32_t uTX = uA + A2_A_BYTES, uR = tc::smem_u32(sR);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto bar = [&](int i) { return tc::smem_u32(&bars[i]); };
  int lo, hi;
  my_items(T * T * B, lo, hi);
  const int n = hi - lo;
  pdl_trigger();
  if (threadIdx.x == 0) {
    tc::mbar_init(bar(0), A3_LOADW);
    tc::mbar_init(bar(1), 1);
    tc::mbar_init(bar(2), 1);
    tc::mbar_init(bar(3), A3_TMW);
    tc::mbar_init(bar(4), 1);
    tc::mbar_init(bar(5), 1);
    tc::mbar_init(bar(6), A3_TMW);
    tc::mbar_init(bar(7), A3_TMW);
    tc::mbar_init(bar(8), 1);
    tc::mbar_init(bar(9), 1);
    fail = 0;
    tc::fence_mbar_init();
  }
  if (warp == A3_MMAW) tc::tmem_alloc(tc::smem_u32(&tmem_slot), 512);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tmem_slot;
  volatile int* vfail = &fail;
  constexpr uint32_t idesc = tc::idesc_bf16(128, BN);

  if (warp < A3_LOADW) {
    // ------------------------------------------------------------ loaders
    pdl_wait();
    const int tid = threadIdx.x;
    // chunk i of a thread: row (tid >> 4) + A3_RS i, columns c8 .. c8 + 7 of the tile;
    // its hi part at so + 128 A3_RS i of sA, its lo part 32 KiB further (sw128_offset)
    const int r0 = tid >> 4, c8 = (tid & 15) * 8;
    const uint32_t so = sw128_offset(128, r0, c8);
    constexpr int HALF = A3_CH / 2;
    float v[A3_CH][8];
    // chunks i0 .. i0 + HALF - 1 of item it into v
    auto load_half = [&](const Item& it, int i0) {
      const int m0 = it.yt * 128 + r0, x = it.xt * 128 + c8;
      const float* img = a.in + (size_t)it.z * a.N * a.N + (size_t)m0 * a.N + x;
#pragma unroll
      for (int i = i0; i < i0 + HALF; ++i) {
        const int m = m0 + A3_RS * i;
        const float* pi = img + (size_t)(A3_RS * i) * a.N;
        if (a.vec4 && m < a.N && x + 7 < a.N) {
          const float4 p = __ldg(reinterpret_cast<const float4*>(pi));
          const float4 q = __ldg(reinterpret_cast<const float4*>(pi + 4));
          v[i][0] = p.x; v[i][1] = p.y; v[i][2] = p.z; v[i][3] = p.w;
          v[i][4] = q.x; v[i][5] = q.y; v[i][6] = q.z; v[i][7] = q.w;
        } else {
#pragma unroll
          for (int e = 0; e < 8; ++e) v[i][e] = (m < a.N && x + e < a.N) ? __ldg(pi + e) : 0.f;
        }
      }
    };
    // chunks i0 .. i0 + HALF - 1 of item j: theta -> mask (mode 1), split into the hi /
    // lo words hw / lw of sA (stored by store_half); the non-finite inputs flagged in bad
    uint4 hw[HALF], lw[HALF];
    auto conv_half = [&](const Item& it, int i0, bool& bad) {
      const int m0 = it.yt * 128 + r0, x = it.xt * 128 + c8;
      float* mo = a.mask_out ? a.mask_out + (size_t)it.z * a.N * a.N + (size_t)m0 * a.N + x
                             : nullptr;
      const bool full = a.vec4 && it.yt * 128 + 127 < a.N && x + 7 < a.N;
#pragma unroll
      for (int i = i0; i < i0 + HALF; ++i) {
        const int m = m0 + A3_RS * i;
        float u[8];
        if (full) {
          // every input is finite exactly when chk stays 0
          float chk = 0.f;
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            chk = __fmaf_rn(v[i][e], 0.f, chk);
            u[e] = MODE == 1 ? 0.5f * (1.f + fast_cos(v[i][e])) : v[i][e];
          }
          bad |= chk != 0.f;
          if (mo) {
            float* po = mo + (size_t)(A3_RS * i) * a.N;
            *reinterpret_cast<float4*>(po) = make_float4(u[0], u[1], u[2], u[3]);
            *reinterpret_cast<float4*>(po + 4) = make_float4(u[4], u[5], u[6], u[7]);
          }
        } else {
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            const bool in_range = m < a.N && x + e < a.N;
            u[e] = v[i][e];
            if (in_range) bad |= !isfinite(u[e]);
            if (MODE == 1) {
              u[e] = in_range ? 0.5f * (1.f + fast_cos(u[e])) : 0.f;
              if (mo && in_range) mo[(size_t)(A3_RS * i) * a.N + e] = u[e];
            }
          }
        }
        split_pair(u[0], u[1], hw[i - i0].x, lw[i - i0].x);
        split_pair(u[2], u[3], hw[i - i0].y, lw[i - i0].y);
        split_pair(u[4], u[5], hw[i - i0].z, lw[i - i0].z);
        split_pair(u[6], u[7], hw[i - i0].w, lw[i - i0].w);
      }
    };
    auto store_half = [&](int i0) {
#pragma unroll
      for (int i = i0; i < i0 + HALF; ++i) {
        *reinterpret_cast<uint4*>(sA + so + (uint32_t)(128 * A3_RS) * i) = hw[i - i0];
        *reinterpret_cast<uint4*>(sA + so + 32768u + (uint32_t)(128 * A3_RS) * i) = lw[i - i0];
      }
    };
    // The loads run half an item ahead of the conversion: the second half of item j
    // loads while the first half converts, the first half of item j + 1 while the
    // second half of item j converts. The first half is converted before the wait for
    // sA to become free, so that only its stores follow stage 1 of the previous item.
    // the input tile of item i + 2 is fetched into L2 during item i: 512 segments of 128
    // bytes, one per loader thread (row tid / 4, columns 32 (tid % 4) ..)
    const bool pf = a.N % 4 == 0 && reinterpret_cast<uintptr_t>(a.in) % 16 == 0;
    auto prefetch_item = [&](const Item& i) {
      const int y = i.yt * 128 + (tid >> 2), x = i.xt * 128 + 32 * (tid & 3);
      static_assert(A3_LOADW * 32 == 512, "one 128-byte segment per loader thread");
      if (pf && y < a.N && x + 32 <= a.N)
        tc::prefetch_l2_line(a.in + (size_t)i.z * a.N * a.N + (size_t)y * a.N + x);
    };
    Item cur = item_at(lo, T, B);
    if (n > 0) load_half(cur, 0);
    if (n > 1) prefetch_item(item_next(cur, T, B));
    for (int j = 0; j < n; ++j, cur = item_next(cur, T, B)) {
      if (j + 2 < n) prefetch_item(item_next(item_next(cur, T, B), T, B));
      load_half(cur, HALF);
      bool bad = false;
      conv_half(cur, 0, bad);
      // sA is free once stage 1 of the previous item has completed
      if (j > 0 && !pwait(bar(1 + ((j - 1) & 1)), ((j - 1) >> 1) & 1, vfail, err, 11)) break;
      store_half(0);
      if (j + 1 < n) load_half(item_next(cur, T, B), 0);
      conv_half(cur, HALF, bad);
      store_half(HALF);
      if (bad) atomicOr(a.flag, 1);
      fence_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(bar(0));
    }
  } else if (warp < A3_MMAW) {
    // ------------------------------------------------------------ TMEM warps
    pdl_wait();
    const int lane_base = (warp & 3) * 32;
    constexpr int DQ = A3_TMW / 4;
    const int q0 = (warp - A3_LOADW) / 4;   // first 16-column group of this warp
    const int count = a.nrows_out * a.ncols;
    Item prv = item_at(lo, T, B), cur = prv;   // items j - 1 and j
    for (int j = 0; j <= n; ++j) {
      if (j > 0) {
        prv = cur;
        cur = item_next(cur, T, B);
      }
      if (j < n && !pwait(bar(1 + (j & 1)), (j >> 1) & 1, vfail, err, 12)) break;
      // stage 2 of the previous item done: sR is free and its Q is ready
      if (j > 0 && !pwait(bar(4 + ((j - 1) & 1)), ((j - 1) >> 1) & 1, vfail, err, 13)) break;
      tc::fence_after();
      if (j < n) {
        r_to_operand<BN>(tmem + (uint32_t)((j & 1) * 128) + ((uint32_t)lane_base << 16), sR,
                         lane_base, q0, DQ);
        fence_async_smem();
        tc::fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(bar(3));
      }
      if (j > 0) {
        // Q of the previous item -> its partials P[r][c] (see analysis_stages in tc2.cu)
        const int jp = j - 1;
        float2* out = a.part + (((size_t)prv.z * T + prv.yt) * T + prv.xt) * count;
        q_to_partials<BN>(tmem + 256u + (uint32_t)((jp & 1) * 128) + ((uint32_t)lane_base << 16),
                          out, a, lane_base, q0, DQ);
        tc::fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(bar(6 + (jp & 1)));
      }
    }
  } else if (lane == 0) {
    // ------------------------------------------------------------ MMA thread
    int pxt = -1, pyt = -1;
    uint32_t ntx = 0, nty = 0;
    int m1 = 0, m2 = 0;
    // Issue order MMA1(0), MMA1(1), MMA2(0), MMA1(2), MMA2(1), ...: stage 1 of item j
    // is issued as soon as its operand sA is full, before stage 2 of item j - 1 waits
    // for its operand sR, so the tensor pipe runs stage 1 of the next item while the
    // TMEM warps build sR.
    Item it = item_at(lo, T, B), prv = it;
    for (int j = 0; j <= n; ++j) {
      if (j < n) {
        const bool newx = it.xt != pxt;
        if (newx) {
          // the TX tile in use is read by stage 1 of the previous item
          if (j > 0 && !pwait(bar(1 + ((j - 1) & 1)), ((j - 1) >> 1) & 1, vfail, err, 14)) break;
          bulk_tile(uTX, txImg + (size_t)it.xt * TXB, TXB, bar(8));
          ++ntx;
          pxt = it.xt;
        }
        if (!pwait(bar(0), j & 1, vfail, err, 15)) break;
        if (newx && !pwait(bar(8), (ntx - 1) & 1, vfail, err, 16)) break;
        tc::fence_after();
        s2_mma(tmem + (uint32_t)((j & 1) * 128), uA, 128, uTX, BN, 128, idesc);
        tc::mma_commit(bar(1 + (j & 1)));
        ++m1;
      }
      if (j > 0) {
        // stage 2 of item jj = j - 1
        const int jj = j - 1;
        const bool newy = prv.yt != pyt;
        if (newy) {
          if (jj > 0 && !pwait(bar(4 + ((jj - 1) & 1)), ((jj - 1) >> 1) & 1, vfail, err, 17)) break;
          bulk_tile(uTY, tyImg + (size_t)prv.yt * A2_A_BYTES, A2_A_BYTES, bar(9));
          ++nty;
          pyt = prv.yt;
        }
        if (!pwait(bar(3), jj & 1, vfail, err, 18)) break;
        if (newy && !pwait(bar(9), (nty - 1) & 1, vfail, err, 19)) break;
        if (jj >= 2 && !pwait(bar(6 + (jj & 1)), ((jj - 2) >> 1) & 1, vfail, err, 20)) break;
        tc::fence_after();
        s2_mma(tmem + 256u + (uint32_t)((jj & 1) * 128), uTY, 128, uR, BN, 128, idesc);
        tc::mma_commit(bar(4 + (jj & 1)));
        ++m2;
        prv = item_next(prv, T, B);
      }
      if (j < n) it = item_next(it, T, B);
    }
    if (*vfail) {
      // nothing of this CTA may still be in flight when it exits
      if (ntx) tc::mbar_wait(bar(8), (ntx - 1) & 1);
      if (nty) tc::mbar_wait(bar(9), (nty - 1) & 1);
      if (m1) tc::mbar_wait(bar(1 + ((m1 - 1) & 1)), ((m1 - 1) >> 1) & 1);
      if (m2) tc::mbar_wait(bar(4 + ((m2 - 1) & 1)), ((m2 - 1) >> 1) & 1);
    }
  }
  tc::fence_before();
  __syncthreads();
  if (warp == A3_MMAW) tc::tmem_dealloc(tmem, 512);
}

template <int BN, int MODE>
static cudaError_t analysis_tc3_m(cudaStream_t s, const Tc2Analysis& a, const void* tx,
                                  const void* ty, int* err, int batch) {
  const size_t smem = 2 * (size_t)A2_A_BYTES + 2 * (size_t)s2_tile_bytes(BN, 128) + 1024;
  cudaError_t e = cudaFuncSetAttribute(analysis_tc3_kernel<BN, MODE>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int T = (a.N + 127) / 128;
  const int items = T * T * batch;
  const int grid = items < sm_count() ? items : sm_count();
  return launch_pdl(analysis_tc3_kernel<BN, MODE>, dim3(grid), dim3(A3_NT), smem, s, a, T, batch,
                    static_cast<const uint8_t*>(tx), static_cast<const uint8_t*>(ty), err);
}
template <int BN>
static cudaError_t analysis_tc3_t(cudaStream_t s, const Tc2Analysis& a, const void* tx,
                                  const void* ty, int* err, int batch) {
  return a.mode == 1 ? analysis_tc3_m<BN, 1>(s, a, tx, ty, err, batch)
                     : analysis_tc3_m<BN, 0>(s, a, tx, ty, err, batch);
}

bool tc3_analysis_supported(int ncols, int nr) {
  return tc2_analysis_supported(ncols, nr) && tc2_analysis_rows(ncols) <= 96;
}

cudaError_t launch_analysis_tc3(cudaStream_t s, int mode, const float* in, float* mask_out,
                                int* flag, int N, int ncols, int nrows_out, int nr, int sym,
                                float2* part, const void* tx_img, const void* ty_img, int* err,
                                int batch) {
  // vector loads of the input and vector stores of the mask
  const int vec4 = (N % 4 == 0) && (reinterpret_cast<uintptr_t>(in) % 16 == 0) &&
                   (reinterpret_cast<uintptr_t>(mask_out) % 16 == 0);
  Tc2Analysis a{in, mask_out, flag, N, mode, vec4, ncols, nrows_out, nr, sym, part};
  switch (tc2_analysis_rows(ncols)) {
    case 16: return analysis_tc3_t<16>(s, a, tx_img, ty_img, err, batch);
    case 32: return analysis_tc3_t<32>(s, a, tx_img, ty_img, err, batch);
    case 48: return analysis_tc3_t<48>(s, a, tx_img, ty_img, err, batch);
    case 64: return analysis_tc3_t<64>(s, a, tx_img, ty_img, err, batch);
    case 80: return analysis_tc3_t<80>(s, a, tx_img, ty_img, err, batch);
    case 96: return analysis_tc3_t<96>(s, a, tx_img, ty_img, err, batch);
    default: return cudaErrorInvalidValue;
  }
}


// =============================================================== epilogue arithmetic
// Per pixel exactly the FAST arithmetic of ResistEpiT<true> / GradEpiT<true>
// (device_common.cuh); loss and norm terms are summed in FP32 over a thread's 32
// pixels of an item and in FP64 from there on.
struct S3Resist {
  ResistEpilogue p;
  __device__ __forceinline__ float sigmoid(float I) const {
    const float z = -p.alpha * (I - p.thr);
    return __fdividef(1.f, 1.f + __expf(z));
  }
  // Mode 1 at in-range pixel i (image offset included): the stores of aerial / wafer,
  // the loss terms into pe / pen, and dL/dI returned.
  __device__ __forceinline__ float dldi(size_t i, float I, float T, bool plain, float& pe,
                                        float& pen) const {
    if (p.aerial) p.aerial[i] = I;
    const float W = sigmoid(I);
    if (p.wafer) p.wafer[i] = W;
    const float r = W - T;
    if (plain) {
      pe += r * r;
      return p.pe_weight * r * W * (1.f - W);
    }
    const float pw = p.pe_window ? __ldg(p.pe_window + i) : 1.f;
    const float qw = p.pen_window ? __ldg(p.pen_window + i) : pw;
    pe += r * r * pw;
    float s = p.pe_weight * r * pw;
    if ((p.penalty != 0.f || p.loss_penalty_term) && T < 0.5f) {
      const float ex = fmaxf(W - p.pen_thr, 0.f);
      pen += ex * ex * qw;
      s += p.penalty * ex * qw;
    }
    return s * W * (1.f - W);
  }
  __device__ __forceinline__ bool plain() const {
    return p.pe_window == nullptr && p.pen_window == nullptr && p.penalty == 0.f &&
           !p.loss_penalty_term;
  }
};

// =============================================================== row synthesis
// out[y][x] = sum_f AY[y][f] Bt[x][f] with the theta-chain (KIND 0, GradEpilogue) or
// the resist (KIND 1, ResistEpilogue) epilogue, as launch_synth_grad_tc2 /
// launch_synth_resist_tc2, from a persistent pipeline:
//   warp 16      (one thread) copies the AY tile (per yt), double-buffers the band
//                operand tile Bt (per image and xt) and issues D[x][y] into acc[j & 1];
//   warps 0-15   run the epilogue of item j while the MMA of item j + 1 runs: warp w
//                takes lanes x = 32 (w % 4) + lane and rows y = 32 (w / 4) .. + 31.
// The FP64 partial of an item (squared gradient norm, or the two loss terms) is
// written to [image][yt][xt] as the per-tile kernels write theirs. Shared memory:
// AY | Bt[0] | Bt[1] (split tiles of 128 x kp). Tensor memory: acc[b] at 128 b.
constexpr int S3_EPIW = 16, S3_MMAW = 16;
constexpr int S3_NT = (S3_EPIW + 1) * 32;

template <int KIND>
__global__ void __launch_bounds__(S3_NT, 1)
synth_tc3_kernel(const uint8_t* __restrict__ Aimg, const uint8_t* __restrict__ Bimg, int N,
                 int kp, int T, int B, GradEpilogue g, S3Resist r, int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 0-1 Bt[b] landed, 2 AY landed, 3-4 acc[b] full, 5-6 acc[b] free (epilogue warps)
  __shared__ __align__(8) uint64_t bars[7];
  __shared__ uint32_t tmem_slot;
  __shared__ int fail;
  __shared__ __align__(8) uint64_t red_bar[EPI_SLOTS];
  __shared__ EpiSums<2> red;
  const uint32_t tb = s2_tile_bytes(128, kp);
  uint8_t* smem = align1024(smem_raw);
  const uint32_t uAY = tc::smem_u32(smem);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto bar = [&](int i) { return tc::smem_u32(&bars[i]); };
  int lo, hi;
  my_items(T * T * B, lo, hi);
  const int n = hi - lo;
  pdl_trigger();
  if (threadIdx.x == 0) {
    for (int i = 0; i < 5; ++i) tc::mbar_init(bar(i), 1);
    tc::mbar_init(bar(5), S3_EPIW);
    tc::mbar_init(bar(6), S3_EPIW);
    for (int i = 0; i < EPI_SLOTS; ++i) tc::mbar_init(tc::smem_u32(&red_bar[i]), S3_EPIW);
    fail = 0;
    tc::fence_mbar_init();
  }
  if (warp == S3_MMAW) tc::tmem_alloc(tc::smem_u32(&tmem_slot), 256);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tmem_slot;
  volatile int* vfail = &fail;

  if (warp < S3_EPIW) {
    // ------------------------------------------------------------ epilogue warps
    pdl_wait();
    const int q = warp & 3, h = warp >> 2;
    const uint32_t lane_addr = (uint32_t)(32 * q) << 16;
    const float* src = KIND == 0 ? g.theta : (r.p.mode == 1 ? r.p.target : nullptr);
    const bool plain = KIND == 1 && r.plain();
    // theta chain without the dPE/dM output: the CTM evaluation
    const bool lean = KIND == 0 && g.theta != nullptr && g.grad_mask == nullptr;
    // per-pixel input, coalesced along x: rows e0 .. e0 + 15 of item j into pre[]
    float pre[32];
    auto load_rows = [&](const Item& it, int e0) {
      const int x = it.xt * 128 + 32 * q + lane, yb = it.yt * 128 + 32 * h;
      const float* sp = src + (size_t)it.z * N * N + (size_t)yb * N + x;
      if (x < N && yb + 31 < N) {
#pragma unroll
        for (int e = e0; e < e0 + 16; ++e) pre[e] = __ldg(sp + e * N);
      } else {
#pragma unroll
        for (int e = e0; e < e0 + 16; ++e) pre[e] = (x < N && yb + e < N) ? __ldg(sp + e * N) : 0.f;
      }
    };
    Item it = item_at(lo, T, B);
    // the input rows of item i + 2 are fetched into L2 during item i
    const bool pf = src && N % 4 == 0 && reinterpret_cast<uintptr_t>(src) % 16 == 0;
    auto prefetch_item = [&](const Item& i) {
      prefetch_rows(src + (size_t)i.z * N * N, N, i.yt * 128 + 32 * h, i.xt * 128 + 32 * q, pf);
    };
    if (src && n > 0) {
      load_rows(it, 0);
      load_rows(it, 16);
    }
    if (n > 1) prefetch_item(item_next(it, T, B));
    const bool sums = KIND == 0 ? g.theta != nullptr : r.p.mode == 1;
    // the partial sums of item i: the squared norm (KIND 0) or the two loss terms
    auto sums_out = [&](const Item& i) {
      const size_t bid = ((size_t)i.z * T + i.yt) * T + i.xt;
      return KIND == 0 ? g.norm_partial + bid : r.p.loss_partial + 2 * bid;
    };
    Item ip = it;   // item j - 1
    int done = 0;   // items finished
    for (int j = 0; j < n; ++j, ip = it, it = item_next(it, T, B)) {
      const Item nxt = item_next(it, T, B);
      if (j + 2 < n) prefetch_item(item_next(nxt, T, B));
      const int x = it.xt * 128 + 32 * q + lane;
      const int yb = it.yt * 128 + 32 * h;
      const bool xin = x < N;
      const bool full = xin && yb + 31 < N;
      const size_t base = (size_t)it.z * N * N;
      if (!pwait(bar(3 + (j & 1)), (j >> 1) & 1, vfail, err, 21)) break;
      tc::fence_after();
      float d[32];
      tc::tmem_ld32(tmem + (uint32_t)((j & 1) * 128) + lane_addr + (uint32_t)(32 * h), d);
      tc::fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(bar(5 + (j & 1)));
      float s0 = 0.f, s1 = 0.f;
      // rows e0 .. e0 + 15; the inputs of the next item load into the rows just used
      auto rows = [&](int e0) {
        if (lean && full) {
          float* gp = g.grad_theta + base + (size_t)yb * N + x;
#pragma unroll
          for (int e = e0; e < e0 + 16; ++e) {
            const float gt = -0.5f * d[e] * fast_sin(pre[e]);
            s0 += gt * gt;
            gp[e * N] = gt;
          }
        } else {
#pragma unroll
          for (int e = e0; e < e0 + 16; ++e) {
            const int y = yb + e;
            const bool in = xin && y < N;
            const size_t i = base + (size_t)y * N + x;
            if (KIND == 0) {
              const float G = d[e];
              if (in && g.grad_mask) g.grad_mask[i] = G;
              if (g.theta && in) {
                // pixels past the image edge are left out: the band operand's rows there
                // are not part of the image and may hold anything
                const float gt = -0.5f * G * fast_sin(pre[e]);
                s0 += gt * gt;
                g.grad_theta[i] = gt;
              }
            } else if (in) {
              const float I = d[e];
              if (r.p.mode == 0) {
                if (r.p.aerial) r.p.aerial[i] = I;
                if (r.p.wafer) r.p.wafer[i] = r.sigmoid(I);
              } else {
                r.p.dldi[i] = r.dldi(i, I, pre[e], plain, s0, s1);
              }
            }
          }
        }
        if (src && j + 1 < n) load_rows(nxt, e0);
      };
      rows(0);
      rows(16);
      if (sums) {
        const double v[2] = {(double)s0, (double)s1};
        epi_put<2>(red, tc::smem_u32(&red_bar[j & 3]), j & 3, v);
        // the sums of item j - 1, by one warp in turn
        if (j > 0 && lane == 0 && warp == (j - 1) % S3_EPIW &&
            !collect2(red, red_bar, j - 1, S3_EPIW, vfail, err, 27, sums_out(ip), KIND == 0 ? 1 : 2))
          break;
      }
      done = j + 1;
    }
    // the sums of the last item
    if (sums && n > 0 && done == n && lane == 0 && warp == (n - 1) % S3_EPIW)
      collect2(red, red_bar, n - 1, S3_EPIW, vfail, err, 28, sums_out(ip), KIND == 0 ? 1 : 2);
  } else if (warp == S3_MMAW && lane == 0) {
    // ------------------------------------------------------------ MMA thread
    // the band operand image is written by the previous kernel of the stream
    pdl_wait();
    constexpr uint32_t idesc = tc::idesc_bf16(128, 128);
    auto bt_src = [&](const Item& it) { return Bimg + ((size_t)it.z * T + it.xt) * tb; };
    int pyt = -1;
    uint32_t nay = 0;
    int nb = 0, nm = 0;
    Item it = item_at(lo, T, B);
    if (n > 0) {
      bulk_tile(uAY + tb, bt_src(it), tb, bar(0));
      nb = 1;
    }
    for (int j = 0; j < n; ++j, it = item_next(it, T, B)) {
      const bool newy = it.yt != pyt;
      if (newy) {
        // the AY tile in use is read by the previous item's MMA
        if (j > 0 && !pwait(bar(3 + ((j - 1) & 1)), ((j - 1) >> 1) & 1, vfail, err, 22)) break;
        bulk_tile(uAY, Aimg + (size_t)it.yt * tb, tb, bar(2));
        ++nay;
        pyt = it.yt;
      }
      if (!pwait(bar(j & 1), (j >> 1) & 1, vfail, err, 23)) break;
      if (newy && !pwait(bar(2), (nay - 1) & 1, vfail, err, 24)) break;
      if (j >= 2 && !pwait(bar(5 + (j & 1)), ((j - 2) >> 1) & 1, vfail, err, 25)) break;
      tc::fence_after();
      s2_mma_swapped(tmem + (uint32_t)((j & 1) * 128), uAY, 128, uAY + (uint32_t)(1 + (j & 1)) * tb,
                     128, kp, idesc);
      tc::mma_commit(bar(3 + (j & 1)));
      ++nm;
      if (j + 1 < n) {
        // Bt[(j + 1) & 1] is read by the MMA of item j - 1
        if (j >= 1 && !pwait(bar(3 + ((j - 1) & 1)), ((j - 1) >> 1) & 1, vfail, err, 26)) break;
        bulk_tile(uAY + (uint32_t)(1 + ((j + 1) & 1)) * tb, bt_src(item_next(it, T, B)), tb,
                  bar((j + 1) & 1));
        ++nb;
      }
    }
    if (*vfail) {
      if (nb) tc::mbar_wait(bar((nb - 1) & 1), ((nb - 1) >> 1) & 1);
      if (nay) tc::mbar_wait(bar(2), (nay - 1) & 1);
      if (nm) tc::mbar_wait(bar(3 + ((nm - 1) & 1)), ((nm - 1) >> 1) & 1);
    }
  }
  tc::fence_before();
  __syncthreads();
  if (warp == S3_MMAW) tc::tmem_dealloc(tmem, 256);
}

template <int KIND>
static cudaError_t synth_tc3_t(cudaStream_t s, const void* Aimg, const void* Bimg, int N, int kp,
                               const GradEpilogue& g, const ResistEpilogue& r, int* err,
                               int* nblocks, int batch) {
  const size_t smem = 3 * (size_t)s2_tile_bytes(128, kp) + 1024;
  cudaError_t e = cudaFuncSetAttribute(synth_tc3_kernel<KIND>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int T = (N + 127) / 128;
  const int items = T * T * batch;
  const int grid = items < sm_count() ? items : sm_count();
  *nblocks = T * T;
  return launch_pdl(synth_tc3_kernel<KIND>, dim3(grid), dim3(S3_NT), smem, s,
                    static_cast<const uint8_t*>(Aimg), static_cast<const uint8_t*>(Bimg), N, kp,
                    T, batch, g, S3Resist{r}, err);
}

bool tc3_synth_supported(int kp) { return kp % 16 == 0 && kp <= 128; }

cudaError_t launch_synth_grad_tc3(cudaStream_t s, const void* Aimg, const void* Bimg, int N,
                                  int kp, const GradEpilogue& ep, int* err, int* nblocks,
                                  int batch) {
  return synth_tc3_t<0>(s, Aimg, Bimg, N, kp, ep, ResistEpilogue{}, err, nblocks, batch);
}

cudaError_t launch_synth_resist_tc3(cudaStream_t s, const void* Aimg, const void* Bimg, int N,
                                    int kp, const ResistEpilogue& ep, int* err, int* nblocks,
                                    int batch) {
  return synth_tc3_t<1>(s, Aimg, Bimg, N, kp, GradEpilogue{}, ep, err, nblocks, batch);
}

// =============================================================== fused resist + adjoint analysis
// The CTM evaluation's resist synthesis and the adjoint tile analysis of its dL/dI
// (launch_synth_resist_analysis_tc2: same loss partials, same adjoint partials) from a
// persistent pipeline. Per item j:
//   SMMA(j)   I^T = Ut . AYD^T into accI[j & 1] (transposed: lanes x);
//   epi(j)    warps 0-15: resist, loss terms, dL/dI, written as the split operand sA
//             (M = y, K = x) in region X, while TXD(j) lands behind it. sA is MN-major
//             (mn_chunk_offset): a thread holds the 32 rows y of its column x and
//             writes them as 16-byte chunks, with no exchange between lanes;
//   MMA1(j)   R = sA . TXD^T into accR; once done, X takes the synthesis operands of
//             item j + 1 (Ut, AYD) and SMMA(j + 1) is issued;
//   R(j)      warps 0-15: R -> sR;  MMA2(j)  Q = TYD . R^T into accQ;
//   Q(j)      warps 0-15 (after epi(j + 1)): Q -> the item's adjoint partials.
// Shared memory: X = max(sA + TXD, Ut + AYD) | TYD 64 KiB (per yt) | sR.
// Tensor memory: accI[b] at 128 b, accR at 256, accQ at 384.
constexpr int F3_MW = 16, F3_MMAW = 16;
constexpr int F3_NT = (F3_MW + 1) * 32;

template <int BN>
__host__ __device__ constexpr uint32_t f3_x_bytes(uint32_t tb) {
  return (A2_A_BYTES + s2_tile_bytes(BN, 128)) > 2 * tb ? (A2_A_BYTES + s2_tile_bytes(BN, 128))
                                                          : 2 * tb;
}

template <int BN>
__global__ void __launch_bounds__(F3_NT, 1)
fused_tc3_kernel(const uint8_t* __restrict__ Aimg, const uint8_t* __restrict__ Bimg, int N,
                 int kp, int T, int B, S3Resist r, Tc2Analysis a,
                 const uint8_t* __restrict__ txImg, const uint8_t* __restrict__ tyImg,
                 int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 0 synthesis operands landed, 1-2 SMMA done [b], 3 sA full (math warps), 4 TXD landed,
  // 5 MMA1 done, 6 sR full (math warps), 7 TYD landed, 8 MMA2 done, 9 accQ free
  // (math warps), 10-11 accI[b] free (math warps)
  __shared__ __align__(8) uint64_t bars[12];
  __shared__ uint32_t tmem_slot;
  __shared__ int fail;
  __shared__ __align__(8) uint64_t red_bar[EPI_SLOTS];
  __shared__ EpiSums<2> red;
  constexpr uint32_t TXB = s2_tile_bytes(BN, 128);
  const uint32_t tb = s2_tile_bytes(128, kp);
  const uint32_t XB = f3_x_bytes<BN>(tb);
  uint8_t* smem = align1024(smem_raw);
  uint8_t* sA = smem;
  uint8_t* sR = smem + XB + A2_A_BYTES;
  const uint32_t uX = tc::smem_u32(smem);
  const uint32_t uUt = uX, uAYD = uX + tb, uTXD = uX + A2_A_BYTES, uTYD = uX + XB;
  const uint32_t uR = tc::smem_u32(sR);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto bar = [&](int i) { return tc::smem_u32(&bars[i]); };
  int lo, hi;
  my_items(T * T * B, lo, hi);
  const int n = hi - lo;
  pdl_trigger();
  if (threadIdx.x == 0) {
    for (int i = 0; i < 12; ++i) tc::mbar_init(bar(i), 1);
    tc::mbar_init(bar(3), F3_MW);
    tc::mbar_init(bar(6), F3_MW);
    tc::mbar_init(bar(9), F3_MW);
    tc::mbar_init(bar(10), F3_MW);
    tc::mbar_init(bar(11), F3_MW);
    for (int i = 0; i < EPI_SLOTS; ++i) tc::mbar_init(tc::smem_u32(&red_bar[i]), F3_MW);
    fail = 0;
    tc::fence_mbar_init();
  }
  if (warp == F3_MMAW) tc::tmem_alloc(tc::smem_u32(&tmem_slot), 512);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tmem_slot;
  volatile int* vfail = &fail;

  if (warp < F3_MW) {
    // ------------------------------------------------------------ math warps
    pdl_wait();
    const int q = warp & 3, h = warp >> 2;
    const int lane_base = 32 * q;
    const uint32_t lane_addr = (uint32_t)lane_base << 16;
    const int xl = lane_base + lane;
    // no window, no penalty, no aerial / wafer output: the CTM evaluation
    const bool lean = r.plain() && r.p.aerial == nullptr && r.p.wafer == nullptr;
    const int count = a.nrows_out * a.ncols;
    // this thread's four 16-byte chunks of sA (rows y = 32 h + 8 c .. + 7 of column xl)
    uint32_t aoff[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) aoff[c] = mn_chunk_offset((uint32_t)(32 * h + 8 * c), (uint32_t)xl);
    float pre[32];
    auto prefetch = [&](const Item& it) {
      const int x = it.xt * 128 + xl, yb = it.yt * 128 + 32 * h;
      const float* tp = r.p.target + (size_t)it.z * N * N + (size_t)yb * N + x;
      if (x < N && yb + 31 < N) {
#pragma unroll
        for (int e = 0; e < 32; ++e) pre[e] = __ldg(tp + e * N);
      } else {
#pragma unroll
        for (int e = 0; e < 32; ++e) pre[e] = (x < N && yb + e < N) ? __ldg(tp + e * N) : 0.f;
      }
    };
    // the target rows of item i + 2 are fetched into L2 during item i
    const bool pf = N % 4 == 0 && reinterpret_cast<uintptr_t>(r.p.target) % 16 == 0;
    Item it = item_at(lo, T, B), ip = it;   // items j and j - 1
    if (n > 0) prefetch(it);
    for (int j = 0; j < n; ++j, ip = it, it = item_next(it, T, B)) {
      if (j + 2 < n) {
        const Item i2 = item_next(item_next(it, T, B), T, B);
        prefetch_rows(r.p.target + (size_t)i2.z * N * N, N, i2.yt * 128 + 32 * h,
                      i2.xt * 128 + lane_base, pf);
      }
      const int x = it.xt * 128 + xl, yb = it.yt * 128 + 32 * h;
      const bool xin = x < N;
      const size_t base = (size_t)it.z * N * N;
      if (!pwait(bar(1 + (j & 1)), (j >> 1) & 1, vfail, err, 31)) break;
      tc::fence_after();
      float d[32];
      tc::tmem_ld32(tmem + (uint32_t)((j & 1) * 128) + lane_addr + (uint32_t)(32 * h), d);
      tc::fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(bar(10 + (j & 1)));
      // sA is free: the MMA thread issues SMMA(j) only after MMA1(j - 1) completed.
      // d[e] becomes dL/dI at (yb + e, x), 0 outside the image.
      float s0 = 0.f, s1 = 0.f;
      bool bad;
      if (lean && xin && yb + 31 < N) {
        // The window-free arithmetic of S3Resist::dldi on pixel pairs in packed FP32x2
        // (each lane rounded as the scalar operation, in the scalar order, so dL/dI is
        // the per-tile kernels' bit for bit; __expf and the reciprocal stay per lane).
        // Every dL/dI is non-finite exactly when its r is, and then so is the product
        // with 0 in chk. The loss terms are summed in two interleaved FP32 chains.
        float2 chk = make_float2(0.f, 0.f), se = chk;
        const float2 na = make_float2(-r.p.alpha, -r.p.alpha);
        const float2 nt = make_float2(-r.p.thr, -r.p.thr);
        const float2 one = make_float2(1.f, 1.f), pw = make_float2(r.p.pe_weight, r.p.pe_weight);
#pragma unroll
        for (int e = 0; e < 32; e += 2) {
          const float2 z = __fmul2_rn(na, __fadd2_rn(make_float2(d[e], d[e + 1]), nt));
          const float2 den = __fadd2_rn(one, make_float2(__expf(z.x), __expf(z.y)));
          const float2 W = make_float2(__fdividef(1.f, den.x), __fdividef(1.f, den.y));
          const float2 rr = __fadd2_rn(W, make_float2(-pre[e], -pre[e + 1]));
          se = __ffma2_rn(rr, rr, se);
          const float2 g = __fmul2_rn(__fmul2_rn(__fmul2_rn(pw, rr), W),
                                      __fadd2_rn(one, make_float2(-W.x, -W.y)));
          chk = __ffma2_rn(g, make_float2(0.f, 0.f), chk);
          d[e] = g.x;
          d[e + 1] = g.y;
        }
        s0 = se.x + se.y;
        bad = chk.x + chk.y != 0.f;
      } else {
        const bool plain = r.plain();
        bad = false;
#pragma unroll
        for (int e = 0; e < 32; ++e) {
          const int y = yb + e;
          float gd = 0.f;
          if (xin && y < N) gd = r.dldi(base + (size_t)y * N + x, d[e], pre[e], plain, s0, s1);
          bad |= !isfinite(gd);
          d[e] = gd;
        }
      }
      // rows 8 c .. 8 c + 7 of column xl: one 16-byte chunk of hi, one of lo
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        uint4 h4, l4;
        split_pair(d[8 * c + 0], d[8 * c + 1], h4.x, l4.x);
        split_pair(d[8 * c + 2], d[8 * c + 3], h4.y, l4.y);
        split_pair(d[8 * c + 4], d[8 * c + 5], h4.z, l4.z);
        split_pair(d[8 * c + 6], d[8 * c + 7], h4.w, l4.w);
        *reinterpret_cast<uint4*>(sA + aoff[c]) = h4;
        *reinterpret_cast<uint4*>(sA + aoff[c] + MN_LO) = l4;
      }
      if (bad) atomicOr(a.flag, 1);
      fence_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(bar(3));
      {
        const double v[2] = {(double)s0, (double)s1};
        const uint32_t rb = tc::smem_u32(&red_bar[j & 3]);
        epi_put<2>(red, rb, j & 3, v);
        double t[2];
        if (threadIdx.x == 0 &&
            epi_take<2>(red, rb, j & 3, (j >> 2) & 1, F3_MW, vfail, err, 46, t)) {
          const size_t bid = ((size_t)it.z * T + it.yt) * T + it.xt;
          r.p.loss_partial[2 * bid] = t[0];
          r.p.loss_partial[2 * bid + 1] = t[1];
        }
      }
      if (j + 1 < n) prefetch(item_next(it, T, B));
      if (j > 0) {
        // MMA2 of the previous item: its Q is ready and sR is free
        if (!pwait(bar(8), (j - 1) & 1, vfail, err, 32)) break;
        tc::fence_after();
        q_to_partials<BN>(tmem + 384u + lane_addr,
                          a.part + (((size_t)ip.z * T + ip.yt) * T + ip.xt) * count, a,
                          lane_base, h, 4);
        tc::fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(bar(9));
      }
      if (!pwait(bar(5), j & 1, vfail, err, 33)) break;
      tc::fence_after();
      r_to_operand<BN>(tmem + 256u + lane_addr, sR, lane_base, h, 4);
      fence_async_smem();
      tc::fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(bar(6));
      if (j + 1 == n) {
        if (!pwait(bar(8), j & 1, vfail, err, 34)) break;
        tc::fence_after();
        q_to_partials<BN>(tmem + 384u + lane_addr,
                          a.part + (((size_t)it.z * T + it.yt) * T + it.xt) * count, a,
                          lane_base, h, 4);
        tc::fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(bar(9));
      }
    }
  } else if (warp == F3_MMAW && lane == 0) {
    // ------------------------------------------------------------ MMA thread
    // the band operand image is written by the previous kernel of the stream
    pdl_wait();
    constexpr uint32_t idI = tc::idesc_bf16(128, 128), idA = tc::idesc_bf16(128, BN);
    auto load_ops = [&](const Item& it) {
      tc::mbar_expect_tx(bar(0), 2 * tb);
      bulk_chunks(uUt, Bimg + ((size_t)it.z * T + it.xt) * tb, tb, bar(0));
      bulk_chunks(uAYD, Aimg + (size_t)it.yt * tb, tb, bar(0));
    };
    int pyt = -1;
    uint32_t nty = 0;
    int nops = 0, ntx = 0;
    uint32_t last_bar = 0, last_par = 0;
    bool any = false;
    auto commit = [&](int b, uint32_t par) {
      tc::mma_commit(bar(b));
      last_bar = bar(b);
      last_par = par;
      any = true;
    };
    Item it = item_at(lo, T, B);
    if (n > 0) {
      load_ops(it);
      nops = 1;
    }
    for (int j = 0; j < n; ++j, it = item_next(it, T, B)) {
      if (j == 0) {
        if (!pwait(bar(0), 0, vfail, err, 35)) break;
        tc::fence_after();
        s2_mma_swapped(tmem, uAYD, 128, uUt, 128, kp, idI);
        commit(1, 0);
      }
      // synthesis of item j done: X's operands are dead, TXD(j) goes behind sA
      if (!pwait(bar(1 + (j & 1)), (j >> 1) & 1, vfail, err, 36)) break;
      bulk_tile(uTXD, txImg + (size_t)it.xt * TXB, TXB, bar(4));
      ++ntx;
      const bool newy = it.yt != pyt;
      if (newy) {
        if (j > 0 && !pwait(bar(8), (j - 1) & 1, vfail, err, 37)) break;
        bulk_tile(uTYD, tyImg + (size_t)it.yt * A2_A_BYTES, A2_A_BYTES, bar(7));
        ++nty;
        pyt = it.yt;
      }
      if (!pwait(bar(3), j & 1, vfail, err, 38)) break;
      if (!pwait(bar(4), j & 1, vfail, err, 39)) break;
      tc::fence_after();
      s2_mma_amn(tmem + 256u, uX, uTXD, BN, 128, idA | IDESC_A_MN);
      commit(5, j & 1);
      if (!pwait(bar(5), j & 1, vfail, err, 40)) break;
      if (j + 1 < n) {
        // X is free: the next item's synthesis operands, then its SMMA (accI[(j+1)&1]
        // was read by the epilogue of item j - 1)
        load_ops(item_next(it, T, B));
        ++nops;
        if (!pwait(bar(0), (j + 1) & 1, vfail, err, 41)) break;
        if (j >= 1 && !pwait(bar(10 + ((j + 1) & 1)), ((j - 1) >> 1) & 1, vfail, err, 42)) break;
        tc::fence_after();
        s2_mma_swapped(tmem + (uint32_t)(((j + 1) & 1) * 128), uAYD, 128, uUt, 128, kp, idI);
        commit(1 + ((j + 1) & 1), ((j + 1) >> 1) & 1);
      }
      if (!pwait(bar(6), j & 1, vfail, err, 43)) break;
      if (newy && !pwait(bar(7), (nty - 1) & 1, vfail, err, 44)) break;
      if (j >= 1 && !pwait(bar(9), (j - 1) & 1, vfail, err, 45)) break;
      tc::fence_after();
      s2_mma(tmem + 384u, uTYD, 128, uR, BN, 128, idA);
      commit(8, j & 1);
    }
    if (*vfail) {
      if (nops) tc::mbar_wait(bar(0), (nops - 1) & 1);
      if (ntx) tc::mbar_wait(bar(4), (ntx - 1) & 1);
      if (nty) tc::mbar_wait(bar(7), (nty - 1) & 1);
      if (any) tc::mbar_wait(last_bar, last_par);
    }
  }
  tc::fence_before();
  __syncthreads();
  if (warp == F3_MMAW) tc::tmem_dealloc(tmem, 512);
}

template <int BN>
static cudaError_t fused_tc3_t(cudaStream_t s, const void* Aimg, const void* Bimg, int N, int kp,
                               const ResistEpilogue& e, const Tc2Analysis& a, const void* tx,
                               const void* ty, int* err, int* nblocks, int batch) {
  const uint32_t tb = s2_tile_bytes(128, kp);
  const size_t smem = (size_t)f3_x_bytes<BN>(tb) + A2_A_BYTES + s2_tile_bytes(BN, 128) + 1024;
  if (smem > 232448 - 512) return cudaErrorInvalidValue;
  cudaError_t r = cudaFuncSetAttribute(fused_tc3_kernel<BN>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (r != cudaSuccess) return r;
  const int T = (N + 127) / 128;
  const int items = T * T * batch;
  const int grid = items < sm_count() ? items : sm_count();
  *nblocks = T * T;
  return launch_pdl(fused_tc3_kernel<BN>, dim3(grid), dim3(F3_NT), smem, s,
                    static_cast<const uint8_t*>(Aimg), static_cast<const uint8_t*>(Bimg), N, kp, T,
                    batch, S3Resist{e}, a, static_cast<const uint8_t*>(tx),
                    static_cast<const uint8_t*>(ty), err);
}

bool tc3_fused_supported(int kp, int ncols, int nr) {
  if (!tc3_analysis_supported(ncols, nr) || !tc3_synth_supported(kp)) return false;
  const uint32_t tb = s2_tile_bytes(128, kp);
  const uint32_t bn = (uint32_t)tc2_analysis_rows(ncols);
  const uint32_t txb = s2_tile_bytes((int)bn, 128);
  const uint32_t xb = A2_A_BYTES + txb > 2 * tb ? A2_A_BYTES + txb : 2 * tb;
  return (size_t)xb + A2_A_BYTES + txb + 1024 <= 232448 - 512;
}

cudaError_t launch_synth_resist_analysis_tc3(cudaStream_t s, const void* Aimg, const void* Bimg,
                                             int N, int kp, const ResistEpilogue& ep, int ncols,
                                             int nr, float2* part, int* flag, const void* tx_img,
                                             const void* ty_img, int* err, int* nblocks,
                                             int batch) {
  if (!tc3_fused_supported(kp, ncols, nr)) return cudaErrorInvalidValue;
  const Tc2Analysis a{nullptr, nullptr, flag, N, 0, 0, ncols, 2 * nr - 1, nr, 1, part};
  switch (tc2_analysis_rows(ncols)) {
    case 16: return fused_tc3_t<16>(s, Aimg, Bimg, N, kp, ep, a, tx_img, ty_img, err, nblocks, batch);
    case 32: return fused_tc3_t<32>(s, Aimg, Bimg, N, kp, ep, a, tx_img, ty_img, err, nblocks, batch);
    case 48: return fused_tc3_t<48>(s, Aimg, Bimg, N, kp, ep, a, tx_img, ty_img, err, nblocks, batch);
    case 64: return fused_tc3_t<64>(s, Aimg, Bimg, N, kp, ep, a, tx_img, ty_img, err, nblocks, batch);
    case 80: return fused_tc3_t<80>(s, Aimg, Bimg, N, kp, ep, a, tx_img, ty_img, err, nblocks, batch);
    case 96: return fused_tc3_t<96>(s, Aimg, Bimg, N, kp, ep, a, tx_img, ty_img, err, nblocks, batch);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace litho_b200
