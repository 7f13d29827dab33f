// Vector kernels of the L-BFGS driver of the CTM theta optimisation
// (CTM_Optimizer.cpp:189-227): the inner products of one vector with up to
// LB_KMAX stored vectors in one pass, accumulated in FP64, and the linear
// combination that forms the search direction. Together they let the two-loop
// recursion run on FP64 Gram matrices on the host with two passes over the
// history per iteration instead of one pass per inner product.
#include <cuda_runtime.h>

#include <algorithm>

#include "device_common.cuh"
#include "litho_internal.cuh"

namespace litho_b200 {

constexpr int LB_NT = 256;
constexpr int LB_KMAX = 64;

// partial[block][j] = sum over this block's elements of rows[j][i] * v[i] (FP64).
template <int KB>
__global__ void __launch_bounds__(LB_NT)
multi_dot_kernel(const float* __restrict__ rows, size_t ld, int k, size_t n,
                 const float* __restrict__ v, double* __restrict__ partial) {
  __shared__ double sh[LB_NT / 32];
  double acc[KB];
#pragma unroll
  for (int j = 0; j < KB; ++j) acc[j] = 0.0;
  for (size_t i = (size_t)blockIdx.x * LB_NT + threadIdx.x; i < n; i += (size_t)gridDim.x * LB_NT) {
    const double x = v[i];
#pragma unroll
    for (int j = 0; j < KB; ++j)
      if (j < k) acc[j] += (double)rows[(size_t)j * ld + i] * x;
  }
#pragma unroll
  for (int j = 0; j < KB; ++j) {
    if (j >= k) break;
    const double t = block_sum<LB_NT>(acc[j], sh);
    if (threadIdx.x == 0) partial[(size_t)blockIdx.x * k + j] = t;
  }
}

// out[j] = the partials of column j summed in block order.
__global__ void multi_dot_sum_kernel(const double* __restrict__ partial, int nb, int k,
                                     double* __restrict__ out) {
  const int j = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += 32) s += partial[(size_t)b * k + j];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) out[j] = s;
}

int multi_dot_blocks(size_t n) {
  const size_t b = (n + LB_NT - 1) / LB_NT;
  return (int)(b < 1 ? 1 : (b > 592 ? 592 : b));
}

cudaError_t launch_multi_dot(cudaStream_t s, const float* rows, size_t ld, int k, size_t n,
                             const float* v, double* partial, double* out) {
  if (k < 1 || k > LB_KMAX) return cudaErrorInvalidValue;
  const int nb = multi_dot_blocks(n);
  if (k <= 8)
    multi_dot_kernel<8><<<nb, LB_NT, 0, s>>>(rows, ld, k, n, v, partial);
  else if (k <= 24)
    multi_dot_kernel<24><<<nb, LB_NT, 0, s>>>(rows, ld, k, n, v, partial);
  else
    multi_dot_kernel<LB_KMAX><<<nb, LB_NT, 0, s>>>(rows, ld, k, n, v, partial);
  multi_dot_sum_kernel<<<k, 32, 0, s>>>(partial, nb, k, out);
  return cudaGetLastError();
}

// Inner products of the k rows with up to three vectors in one launch: CTA (bx, by)
// takes rows 8 by .. 8 by + 7 and a stride of the elements, so every row is read
// once and the three vectors once per group of 8 rows (three times for 20 rows);
// partial[((by * gridDim.x + bx) * 8 + r) * 3 + v].
__global__ void __launch_bounds__(LB_NT)
multi_dot3_kernel(const float* __restrict__ rows, size_t ld, int k, size_t n,
                  const float* __restrict__ v0, const float* __restrict__ v1,
                  const float* __restrict__ v2, double* __restrict__ partial) {
  __shared__ double sh[LB_NT / 32];
  const int j0 = blockIdx.y * 8;
  double acc[8][3];
#pragma unroll
  for (int r = 0; r < 8; ++r) acc[r][0] = acc[r][1] = acc[r][2] = 0.0;
  for (size_t i = (size_t)blockIdx.x * LB_NT + threadIdx.x; i < n; i += (size_t)gridDim.x * LB_NT) {
    const double a = v0[i], b = v1 ? (double)v1[i] : 0.0, c = v2 ? (double)v2[i] : 0.0;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      if (j0 + r >= k) break;
      const double x = rows[(size_t)(j0 + r) * ld + i];
      acc[r][0] += x * a;
      acc[r][1] += x * b;
      acc[r][2] += x * c;
    }
  }
  double* out = partial + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 24;
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const double t = block_sum<LB_NT>(acc[r][v], sh);
      if (threadIdx.x == 0) out[r * 3 + v] = t;
    }
}

// out[v * k + j] = the partials of (row j, vector v) summed in block order.
__global__ void multi_dot3_sum_kernel(const double* __restrict__ partial, int nbx, int k, int nv,
                                      double* __restrict__ out) {
  const int j = blockIdx.x, v = blockIdx.y;
  if (v >= nv) return;
  const double* p = partial + (size_t)(j / 8) * nbx * 24 + (j % 8) * 3 + v;
  double s = 0.0;
  for (int b = threadIdx.x; b < nbx; b += 32) s += p[(size_t)b * 24];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) out[(size_t)v * k + j] = s;
}

int multi_dot3_blocks(size_t n, int k) {
  const int ky = (k + 7) / 8;
  const size_t b = (n + LB_NT - 1) / LB_NT;
  const size_t cap = std::max<size_t>(1, 592 / ky);
  return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

cudaError_t launch_multi_dot3(cudaStream_t s, const float* rows, size_t ld, int k, size_t n,
                              const float* v0, const float* v1, const float* v2, double* partial,
                              double* out) {
  if (k < 1 || k > LB_KMAX || !v0) return cudaErrorInvalidValue;
  const int nv = v2 ? 3 : (v1 ? 2 : 1);
  const int nbx = multi_dot3_blocks(n, k);
  multi_dot3_kernel<<<dim3(nbx, (k + 7) / 8), LB_NT, 0, s>>>(rows, ld, k, n, v0, v1, v2, partial);
  multi_dot3_sum_kernel<<<dim3(k, nv), 32, 0, s>>>(partial, nbx, k, nv, out);
  return cudaGetLastError();
}

// out[i] = cv v[i] + sum_j coef[j] rows[j][i], in FP64 per element.
__global__ void __launch_bounds__(LB_NT)
combine_kernel(const float* __restrict__ rows, size_t ld, int k, size_t n,
               const double* __restrict__ coef, const float* __restrict__ v, double cv,
               float* __restrict__ out) {
  __shared__ double c[LB_KMAX];
  if (threadIdx.x < k) c[threadIdx.x] = coef[threadIdx.x];
  __syncthreads();
  for (size_t i = (size_t)blockIdx.x * LB_NT + threadIdx.x; i < n; i += (size_t)gridDim.x * LB_NT) {
    double a = cv * (double)v[i];
    for (int j = 0; j < k; ++j) a += c[j] * (double)rows[(size_t)j * ld + i];
    out[i] = (float)a;
  }
}

cudaError_t launch_combine(cudaStream_t s, const float* rows, size_t ld, int k, size_t n,
                           const double* coef, const float* v, double cv, float* out) {
  if (k < 0 || k > LB_KMAX) return cudaErrorInvalidValue;
  combine_kernel<<<multi_dot_blocks(n), LB_NT, 0, s>>>(rows, ld, k, n, coef, v, cv, out);
  return cudaGetLastError();
}

}  // namespace litho_b200
