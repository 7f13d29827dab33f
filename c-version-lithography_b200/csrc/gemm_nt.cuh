// FP32 SIMT "NT" GEMM tile engine:  C[m][n] = sum_k A[m][k] * B[n][k]
// with A and B both K-contiguous, a functor that produces A elements (so a
// prologue such as M = (1 + cos theta)/2 is fused into the load) and a functor
// that consumes every C element (so resist / loss / theta-chain epilogues are
// fused into the store). Used by the row analyses (A = image, B = twiddles,
// K = N, split over blockIdx.z) and the row syntheses (A = twiddles, B = band
// coefficients, K = 2*band rows).
//
// Thread (tx, ty), tid = ty * BNT + tx, owns rows ty*TM + i (i < TM, read as
// float4 from shared memory) and columns tx + j*BNT (j < TN, consecutive tx
// read consecutive words, so shared loads are conflict-free).
#pragma once
#include <cuda_runtime.h>

namespace litho_b200 {

template <int BMT, int BNT, int TM, int TN, int BK, class ALoad, class Epi>
__global__ void __launch_bounds__(BMT * BNT)
gemm_nt_kernel(int M, int Nn, int K, int k_per_split, ALoad aload_in, const float* __restrict__ B,
               int ldb, Epi epi_in) {
  ALoad aload = aload_in;  // per-thread mutable copies of the functors
  Epi epi = epi_in;
  constexpr int BM = BMT * TM;
  constexpr int BN = BNT * TN;
  constexpr int NT = BMT * BNT;
  constexpr int AS = BM + 4;  // row stride of the transposed tiles (keeps float4 alignment)
  constexpr int BS = BN + 1;
  static_assert(TM % 4 == 0, "TM must be a multiple of 4");
  static_assert(BK % 4 == 0, "BK must be a multiple of 4");
  __shared__ __align__(16) float As[BK * AS];
  __shared__ float Bs[BK * BS];

  const int tid = threadIdx.x;
  const int tx = tid % BNT;
  const int ty = tid / BNT;
  const int m0 = blockIdx.x * BM;
  const int n0 = blockIdx.y * BN;
  const int kbeg = blockIdx.z * k_per_split;
  const int kend = min(K, kbeg + k_per_split);

  float acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = 0.f;

  for (int kt = kbeg; kt < kend; kt += BK) {
    // A tile: BM rows x BK columns, four consecutive k per thread-step.
    constexpr int AQ = BM * (BK / 4);
    for (int e = tid; e < AQ; e += NT) {
      const int mm = e / (BK / 4);
      const int kq = (e % (BK / 4)) * 4;
      float v[4];
      aload.load4(m0 + mm, kt + kq, kend, v);
#pragma unroll
      for (int q = 0; q < 4; ++q) As[(kq + q) * AS + mm] = v[q];
    }
    constexpr int BQ = BN * BK;
    for (int e = tid; e < BQ; e += NT) {
      const int nn = e / BK;
      const int kk = e % BK;
      const int gn = n0 + nn, gk = kt + kk;
      Bs[kk * BS + nn] = (gn < Nn && gk < kend) ? __ldg(B + (size_t)gn * ldb + gk) : 0.f;
    }
    __syncthreads();
#pragma unroll
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

#pragma unroll
  for (int i = 0; i < TM; ++i) {
    const int m = m0 + ty * TM + i;
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const int n = n0 + tx + j * BNT;
      if (m < M && n < Nn) epi.store(m, n, acc[i][j]);
    }
  }
  epi.finish();
}

}  // namespace litho_b200
