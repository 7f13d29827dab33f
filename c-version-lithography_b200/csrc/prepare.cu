// One-time FP64 optical set-up: the SOCS kernels of a partially coherent source
// through an aberrated circular pupil, restated from the reference's LithoPrepare
// (source/litho_model/litho_prepare.cpp:16-385) with its grid (grid.cpp:27,38-48),
// pupil (pupil.cpp:14-46), Fringe Zernike wavefront (zernike.cpp:12-56) and annular
// source map (source.cpp:114-158):
//   * normalised frequency axis f_i = (i - N/2) / (N dx) / (NA / lambda), C integer N/2;
//   * source map: the axis values in [-2, 2], an upsample-times finer linspace grid
//     over the same range, the annulus sigma_in < rho < sigma_out (hard edges, or the
//     erf smooth step of width `smoothing`), averaged back in upsample^2 blocks and
//     clamped at 0; source points = entries above 1e-8 in row-major order (row: fy);
//   * A = [sqrt(w_s) P(f + f_s)] over the SOCS support (the full grid, or with
//     `compact` the pupil's extent grown by the source shifts), P(f + f_s) bilinear
//     between the four pixels around the sub-pixel shift, column-major flattening;
//   * the thin SVD A = U S V^H, kernels U_k with eigenvalues S_k^2 for the K largest.
// B200 form: the pupil, A, the Gram matrix A^H A and the kernels U_k = A v_k / S_k are
// FP64 kernels on the GPU; the Hermitian eigendecomposition A^H A = V S^2 V^H (Ns x Ns,
// Ns source points) is cuSOLVER's FP64 zheevd. The kernels agree with the SVD's up to a
// phase per kernel (and a basis within each degenerate eigenvalue), which no image
// depends on.
#include <cuComplex.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "litho_internal.cuh"

namespace litho_b200 {
namespace {

// Fringe Zernike polynomials Z1..Z11 on normalised pupil coordinates (zernike.cpp:24-38).
__device__ double fringe(int n, double f, double g) {
  const double r2 = f * f + g * g;
  switch (n) {
    case 1: return 1.0;
    case 2: return 2.0 * f;
    case 3: return 2.0 * g;
    case 4: return sqrt(3.0) * (2.0 * r2 - 1.0);
    case 5: return sqrt(6.0) * (2.0 * f * g);
    case 6: return sqrt(6.0) * (f * f - g * g);
    case 7: return sqrt(8.0) * (3.0 * r2 - 2.0) * g;
    case 8: return sqrt(8.0) * (3.0 * r2 - 2.0) * f;
    case 9: return sqrt(8.0) * (3.0 * f * f * g - g * g * g);
    case 10: return sqrt(8.0) * (f * f * f - 3.0 * f * g * g);
    case 11: return sqrt(5.0) * (6.0 * r2 * r2 - 6.0 * r2 + 1.0);
    default: return 0.0;
  }
}

struct Zernike {
  double c[12];   // c[1..11]
};

// P[row][col] = [rho^2 <= 1] exp(i 2 pi W), DC at (N/2, N/2).
__global__ void pupil_kernel(int N, double scale, Zernike z, cuDoubleComplex* P) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x, row = blockIdx.y;
  if (col >= N) return;
  const double f = (col - N / 2) * scale, g = (row - N / 2) * scale;
  cuDoubleComplex v = make_cuDoubleComplex(0.0, 0.0);
  if (f * f + g * g <= 1.0) {
    double w = 0.0;
    for (int n = 1; n <= 11; ++n)
      if (z.c[n] != 0.0) w += z.c[n] * fringe(n, f, g);
    double s, c;
    sincospi(2.0 * w, &s, &c);
    v = make_cuDoubleComplex(c, s);
  }
  P[(size_t)row * N + col] = v;
}

struct SourcePt {
  int r0, c0;
  double tr, tc, sw;   // row/column shift fractions, sqrt(weight)
};

// A[m + i M] (column-major, M = Nr Nc, m = r + c Nr): sqrt(w_i) times the pupil shifted
// by source point i, bilinear (litho_prepare.cpp:266-294).
__global__ void shifted_pupil_kernel(const cuDoubleComplex* __restrict__ P, int N, int oy, int ox,
                                     int Nr, int Nc, const SourcePt* __restrict__ pts,
                                     cuDoubleComplex* __restrict__ A) {
  const size_t M = (size_t)Nr * Nc;
  const size_t m = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (m >= M) return;
  const int r = (int)(m % Nr), c = (int)(m / Nr);
  const SourcePt s = pts[i];
  auto at = [&](int rr, int cc) {
    return (rr < 0 || rr >= N || cc < 0 || cc >= N) ? make_cuDoubleComplex(0.0, 0.0)
                                                    : P[(size_t)rr * N + cc];
  };
  const int ra = oy + r + s.r0, ca = ox + c + s.c0;
  const double w00 = (1 - s.tr) * (1 - s.tc), w01 = (1 - s.tr) * s.tc;
  const double w10 = s.tr * (1 - s.tc), w11 = s.tr * s.tc;
  const cuDoubleComplex p00 = at(ra, ca), p01 = at(ra, ca + 1);
  const cuDoubleComplex p10 = at(ra + 1, ca), p11 = at(ra + 1, ca + 1);
  const double re = w00 * p00.x + w01 * p01.x + w10 * p10.x + w11 * p11.x;
  const double im = w00 * p00.y + w01 * p01.y + w10 * p10.y + w11 * p11.y;
  A[m + (size_t)i * M] = make_cuDoubleComplex(s.sw * re, s.sw * im);
}

// G = A^H A (Ns x Ns, column-major, both triangles): 16 x 16 output tiles, the rows
// of A in chunks of 16 through shared memory, fixed summation order.
constexpr int GT = 16;
__global__ void gram_kernel(const cuDoubleComplex* __restrict__ A, size_t M, int Ns,
                            cuDoubleComplex* __restrict__ G) {
  __shared__ cuDoubleComplex sa[GT][GT + 1], sb[GT][GT + 1];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = blockIdx.y * GT + ty, j = blockIdx.x * GT + tx;
  double re = 0.0, im = 0.0;
  for (size_t m0 = 0; m0 < M; m0 += GT) {
    const size_t mr = m0 + tx;   // row of A loaded by this thread
    const int ci = blockIdx.y * GT + ty, cj = blockIdx.x * GT + ty;
    sa[ty][tx] = (mr < M && ci < Ns) ? A[mr + (size_t)ci * M] : make_cuDoubleComplex(0.0, 0.0);
    sb[ty][tx] = (mr < M && cj < Ns) ? A[mr + (size_t)cj * M] : make_cuDoubleComplex(0.0, 0.0);
    __syncthreads();
#pragma unroll
    for (int k = 0; k < GT; ++k) {
      const cuDoubleComplex a = sa[ty][k], b = sb[tx][k];   // conj(a) b
      re = fma(a.x, b.x, fma(a.y, b.y, re));
      im = fma(a.x, b.y, fma(-a.y, b.x, im));
    }
    __syncthreads();
  }
  if (i < Ns && j < Ns) G[i + (size_t)j * Ns] = make_cuDoubleComplex(re, im);
}

// U[m + k M] = (A v_k)[m] / sigma_k for the K kept eigenpairs (column Ns - 1 - k of V).
__global__ void kernels_kernel(const cuDoubleComplex* __restrict__ A, size_t M, int Ns,
                               const cuDoubleComplex* __restrict__ V, const double* __restrict__ ev,
                               int K, cuDoubleComplex* __restrict__ U) {
  const size_t m = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (m >= M) return;
  const int col = Ns - 1 - k;
  const double lam = ev[col];
  double re = 0.0, im = 0.0;
  for (int i = 0; i < Ns; ++i) {
    const cuDoubleComplex a = A[m + (size_t)i * M], v = V[i + (size_t)col * Ns];
    re = fma(a.x, v.x, fma(-a.y, v.y, re));
    im = fma(a.x, v.y, fma(a.y, v.x, im));
  }
  const double inv = lam > 0.0 ? 1.0 / sqrt(lam) : 0.0;
  U[m + (size_t)k * M] = make_cuDoubleComplex(re * inv, im * inv);
}

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { cudaFree(p); }
  bool alloc(size_t bytes) { return cudaMalloc(&p, bytes) == cudaSuccess; }
  template <class T>
  T* as() const { return static_cast<T*>(p); }
};

}  // namespace
}  // namespace litho_b200

using namespace litho_b200;

extern "C" int litho_socs_prepare(litho_ctx* ctx, const litho_socs_params* p, litho_cache** out,
                                  litho_socs_info* info, double* eigenvalues,
                                  double* band_kernels) {
  if (!ctx || !p || !out) return LITHO_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  const int N = p->N, up = p->upsample > 0 ? p->upsample : 10;
  if (N < 4 || !(p->pixel_nm > 0) || !(p->wavelength_nm > 0) || !(p->na > 0) ||
      !(p->sigma_out > p->sigma_in) || p->sigma_in < 0 || !(p->smoothing >= 0))
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT,
                     "socs_prepare: N >= 4, positive pixel size, wavelength and NA, "
                     "0 <= sigma_in < sigma_out and smoothing >= 0 are required");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx->fail(LITHO_ERR_CUDA, "cudaSetDevice");
  cudaStream_t s = ctx->stream;
  // normalised frequency axis (grid.cpp:27, 38-48)
  const double scale = (1.0 / (N * p->pixel_nm)) / (p->na / p->wavelength_nm);
  std::vector<double> f(N);
  for (int i = 0; i < N; ++i) f[i] = (i - N / 2) * scale;
  const double df = f[1] - f[0];
  // source map (source.cpp:114-158)
  std::vector<double> ff;
  for (double v : f)
    if (v >= -2.0 && v <= 2.0) ff.push_back(v);
  const int num = (int)ff.size();
  if (num < 2) return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "socs_prepare: source axis has < 2 points");
  const int hn = num * up;
  std::vector<double> hi(hn);
  const double hstep = (ff[num - 1] - ff[0]) / (double)(hn - 1);   // LinSpaced(hn, ff0, ff_end)
  for (int i = 0; i < hn; ++i) hi[i] = ff[0] + i * hstep;
  auto step = [&](double x) {
    return p->smoothing == 0.0 ? (x > 0.0 ? 1.0 : 0.0) : 0.5 * (1.0 + std::erf(x / p->smoothing));
  };
  std::vector<double> smap((size_t)num * num, 0.0);
  for (int R = 0; R < num; ++R)
    for (int C = 0; C < num; ++C) {
      double acc = 0.0;
      for (int a = 0; a < up; ++a)
        for (int b = 0; b < up; ++b) {
          const double gy = hi[R * up + a], gx = hi[C * up + b];
          const double rho = std::sqrt(gx * gx + gy * gy);
          acc += step(p->sigma_out - rho) * step(rho - p->sigma_in);
        }
      smap[(size_t)R * num + C] = std::max(acc / (up * up), 0.0);
    }
  // source points (litho_prepare.cpp:65-102): row -> gs (y), column -> fs (x)
  std::vector<double> fs, gs, ws;
  for (int R = 0; R < num; ++R)
    for (int C = 0; C < num; ++C)
      if (smap[(size_t)R * num + C] > 1e-8) {
        fs.push_back(ff[C]);
        gs.push_back(ff[R]);
        ws.push_back(smap[(size_t)R * num + C]);
      }
  const int Ns = (int)ws.size();
  if (Ns == 0) return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "socs_prepare: the source map is empty");
  double ws_sum = 0.0;
  for (double w : ws) ws_sum += w;
  // SOCS support (litho_prepare.cpp:239-255): the pupil's nonzero extent (rho^2 <= 1)
  int oy = 0, ox = 0, ey = N, ex = N;
  if (p->compact) {
    int py0 = N, px0 = N, py1 = -1, px1 = -1;
    for (int r = 0; r < N; ++r)
      for (int c = 0; c < N; ++c)
        if (f[c] * f[c] + f[r] * f[r] <= 1.0) {
          py0 = std::min(py0, r); px0 = std::min(px0, c);
          py1 = std::max(py1, r); px1 = std::max(px1, c);
        }
    if (py1 < 0) return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "socs_prepare: the pupil is empty");
    const double gmax = *std::max_element(gs.begin(), gs.end());
    const double gmin = *std::min_element(gs.begin(), gs.end());
    const double fmax = *std::max_element(fs.begin(), fs.end());
    const double fmin = *std::min_element(fs.begin(), fs.end());
    oy = std::max(0, py0 - (int)std::floor(gmax / df) - 1);
    ox = std::max(0, px0 - (int)std::floor(fmax / df) - 1);
    ey = std::min(N, py1 - (int)std::floor(gmin / df) + 1);
    ex = std::min(N, px1 - (int)std::floor(fmin / df) + 1);
  }
  const int Nr = ey - oy, Nc = ex - ox;
  const size_t M = (size_t)Nr * Nc;
  if (M * Ns * sizeof(cuDoubleComplex) > ((size_t)8 << 30))
    return ctx->fail(LITHO_ERR_UNSUPPORTED,
                     "socs_prepare: the SOCS matrix (support x source points) exceeds 8 GiB; "
                     "use the compact support");
  const int K = std::min(p->num_socs > 0 ? p->num_socs : Ns, Ns);
  // device work
  std::vector<SourcePt> pts(Ns);
  for (int i = 0; i < Ns; ++i) {
    const double dc = fs[i] / df, dr = gs[i] / df;
    pts[i].c0 = (int)std::floor(dc);
    pts[i].r0 = (int)std::floor(dr);
    pts[i].tc = dc - pts[i].c0;
    pts[i].tr = dr - pts[i].r0;
    pts[i].sw = std::sqrt(ws[i]);
  }
  Zernike z{};
  if (p->zernike)
    for (int n = 1; n <= 11; ++n) z.c[n] = p->zernike[n - 1];
  DevBuf dP, dPts, dA, dG, dW, dU, dWork, dInfo;
  if (!dP.alloc((size_t)N * N * sizeof(cuDoubleComplex)) ||
      !dPts.alloc(Ns * sizeof(SourcePt)) || !dA.alloc(M * Ns * sizeof(cuDoubleComplex)) ||
      !dG.alloc((size_t)Ns * Ns * sizeof(cuDoubleComplex)) || !dW.alloc(Ns * sizeof(double)) ||
      !dU.alloc(M * K * sizeof(cuDoubleComplex)) || !dInfo.alloc(sizeof(int))) {
    cudaGetLastError();
    return ctx->fail(LITHO_ERR_OOM, "socs_prepare: device allocation failed");
  }
  LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(dPts.p, pts.data(), Ns * sizeof(SourcePt),
                                      cudaMemcpyHostToDevice, s));
  pupil_kernel<<<dim3((N + 127) / 128, N), 128, 0, s>>>(N, scale, z, dP.as<cuDoubleComplex>());
  shifted_pupil_kernel<<<dim3((unsigned)((M + 255) / 256), Ns), 256, 0, s>>>(
      dP.as<cuDoubleComplex>(), N, oy, ox, Nr, Nc, dPts.as<SourcePt>(), dA.as<cuDoubleComplex>());
  gram_kernel<<<dim3((Ns + GT - 1) / GT, (Ns + GT - 1) / GT), dim3(GT, GT), 0, s>>>(
      dA.as<cuDoubleComplex>(), M, Ns, dG.as<cuDoubleComplex>());
  LITHO_CUDA_TRY(ctx, cudaGetLastError());
  // Hermitian eigendecomposition, FP64 (eigenvalues ascending, eigenvectors in dG)
  cusolverDnHandle_t h = nullptr;
  if (cusolverDnCreate(&h) != CUSOLVER_STATUS_SUCCESS)
    return ctx->fail(LITHO_ERR_CUDA, "socs_prepare: cusolverDnCreate failed");
  struct HandleGuard {
    cusolverDnHandle_t h;
    ~HandleGuard() { cusolverDnDestroy(h); }
  } guard{h};
  cusolverDnSetStream(h, s);
  int lwork = 0;
  if (cusolverDnZheevd_bufferSize(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, Ns,
                                  dG.as<cuDoubleComplex>(), Ns, dW.as<double>(), &lwork) !=
          CUSOLVER_STATUS_SUCCESS ||
      !dWork.alloc((size_t)std::max(lwork, 1) * sizeof(cuDoubleComplex)))
    return ctx->fail(LITHO_ERR_CUDA, "socs_prepare: eigensolver workspace");
  if (cusolverDnZheevd(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, Ns,
                       dG.as<cuDoubleComplex>(), Ns, dW.as<double>(),
                       dWork.as<cuDoubleComplex>(), lwork, dInfo.as<int>()) !=
      CUSOLVER_STATUS_SUCCESS)
    return ctx->fail(LITHO_ERR_CUDA, "socs_prepare: eigensolver failed to launch");
  kernels_kernel<<<dim3((unsigned)((M + 255) / 256), K), 256, 0, s>>>(
      dA.as<cuDoubleComplex>(), M, Ns, dG.as<cuDoubleComplex>(), dW.as<double>(), K,
      dU.as<cuDoubleComplex>());
  LITHO_CUDA_TRY(ctx, cudaGetLastError());
  std::vector<double> evals(Ns);
  std::vector<cuDoubleComplex> U(M * K);
  int solver_info = 0;
  LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(evals.data(), dW.p, Ns * sizeof(double),
                                      cudaMemcpyDeviceToHost, s));
  LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(U.data(), dU.p, M * K * sizeof(cuDoubleComplex),
                                      cudaMemcpyDeviceToHost, s));
  LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(&solver_info, dInfo.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  LITHO_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  if (solver_info != 0)
    return ctx->fail(LITHO_ERR_CUDA, "socs_prepare: the eigensolver did not converge (info " +
                                         std::to_string(solver_info) + ")");
  // kept eigenvalues, largest first; the band [k][r][c] of each kernel
  std::vector<double> lam(K);
  double total = 0.0, kept = 0.0;
  for (int i = 0; i < Ns; ++i) total += std::max(evals[i], 0.0);
  for (int k = 0; k < K; ++k) {
    lam[k] = std::max(evals[Ns - 1 - k], 0.0);
    kept += lam[k];
  }
  // The kernels vanish outside the union of the shifted pupils (rows of A that are zero
  // for every source point): the band is the window of their nonzero coefficients.
  int r0 = Nr, r1 = -1, c0 = Nc, c1 = -1;
  for (int k = 0; k < K; ++k)
    for (int c = 0; c < Nc; ++c)
      for (int r = 0; r < Nr; ++r) {
        const cuDoubleComplex v = U[(size_t)r + (size_t)c * Nr + (size_t)k * M];
        if (v.x != 0.0 || v.y != 0.0) {
          r0 = std::min(r0, r); r1 = std::max(r1, r);
          c0 = std::min(c0, c); c1 = std::max(c1, c);
        }
      }
  if (r1 < 0) return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "socs_prepare: every kernel is zero");
  const int Br = r1 - r0 + 1, Bc = c1 - c0 + 1;
  std::vector<double> band((size_t)K * Br * Bc * 2);
  for (int k = 0; k < K; ++k)
    for (int r = 0; r < Br; ++r)
      for (int c = 0; c < Bc; ++c) {
        const cuDoubleComplex v = U[(size_t)(r0 + r) + (size_t)(c0 + c) * Nr + (size_t)k * M];
        const size_t o = (((size_t)k * Br + r) * Bc + c) * 2;
        band[o] = v.x;
        band[o + 1] = v.y;
      }
  // centred row oy + r is integer frequency oy + r - N/2 (ifftshift to DC at the corner)
  const int row0 = oy + r0 - N / 2, col0 = ox + c0 - N / 2;
  const int st = litho_cache_create_band(ctx, N, K, Br, Bc, row0, col0, band.data(), lam.data(),
                                         ws_sum, out);
  if (st) return st;
  if (info) {
    info->K = K;
    info->Ns = Ns;
    info->Nr = Br;
    info->Nc = Bc;
    info->row0 = row0;
    info->col0 = col0;
    info->ws_sum = ws_sum;
    info->energy_captured = total > 0.0 ? kept / total : 0.0;
  }
  if (eigenvalues) std::copy(lam.begin(), lam.end(), eigenvalues);
  if (band_kernels) std::copy(band.begin(), band.end(), band_kernels);
  return LITHO_OK;
}
