// Sparse edge-placement error at selected edge points (EPs): Loss::evaluate_sparse_epe
// (source/utils/loss.cpp:125-163) and the dL/dI of Gradient::epe_gradient
// (source/utils/gradient.cpp:198-227). EP selection stays on the host; the points
// (subpixel (y, x)) and weights arrive per call. One thread per EP, FP64 arithmetic
// on the FP32 aerial image. The dL/dI scatter is deterministic: every EP emits its
// stencil's (pixel, value) pairs, a stable radix sort groups them by pixel with the EP
// order kept, and each pixel's contributions are added in FP64 in that order, as the
// reference's serial loop adds them into its double-precision dL/dI.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include "device_common.cuh"

namespace litho_b200 {

// make_bilinear_stencil (source/utils/epe_utils.cpp:39-67): the point clamped to the
// pixel-centre range, the four corners of its cell with bilinear weights; a repeated
// edge pixel carries the merged weight (its partner's weight is zero).
struct Stencil {
  int y0, y1, x0, x1;
  double wy1, wx1;
};

__device__ __forceinline__ Stencil make_stencil(int rows, int cols, double y, double x) {
  const double yy = fmin(fmax(y, 0.0), rows - 1.0), xx = fmin(fmax(x, 0.0), cols - 1.0);
  Stencil s;
  s.y0 = (int)floor(yy);
  s.x0 = (int)floor(xx);
  s.y1 = min(s.y0 + 1, rows - 1);
  s.x1 = min(s.x0 + 1, cols - 1);
  s.wy1 = s.y1 == s.y0 ? 0.0 : yy - s.y0;
  s.wx1 = s.x1 == s.x0 ? 0.0 : xx - s.x0;
  return s;
}

// |grad I| at (y, x) with LevelSetUtils::_gradient_1d (central differences, second-order
// one-sided at the borders, d = 1), floored at 1e-6.
__device__ __forceinline__ double grad_mag(const float* I, int rows, int cols, int y, int x) {
  auto at = [&](int yy, int xx) { return (double)__ldg(I + (size_t)yy * cols + xx); };
  double gx, gy;
  if (x == 0) gx = (-3.0 * at(y, 0) + 4.0 * at(y, 1) - at(y, 2)) / 2.0;
  else if (x == cols - 1) gx = (3.0 * at(y, x) - 4.0 * at(y, x - 1) + at(y, x - 2)) / 2.0;
  else gx = (at(y, x + 1) - at(y, x - 1)) / 2.0;
  if (y == 0) gy = (-3.0 * at(0, x) + 4.0 * at(1, x) - at(2, x)) / 2.0;
  else if (y == rows - 1) gy = (3.0 * at(y, x) - 4.0 * at(y - 1, x) + at(y - 2, x)) / 2.0;
  else gy = (at(y + 1, x) - at(y - 1, x)) / 2.0;
  return fmax(sqrt(gx * gx + gy * gy), 1e-6);
}

// Bilinear sample of f(y, x) over the stencil (weights in the reference's order).
template <class F>
__device__ __forceinline__ double sample(const Stencil& s, F f) {
  const double a = (1.0 - s.wy1) * (1.0 - s.wx1), b = (1.0 - s.wy1) * s.wx1;
  const double c = s.wy1 * (1.0 - s.wx1), d = s.wy1 * s.wx1;
  double v = 0.0;
  if (a > 0.0) v += a * f(s.y0, s.x0);
  if (b > 0.0) v += b * f(s.y0, s.x1);
  if (c > 0.0) v += c * f(s.y1, s.x0);
  if (d > 0.0) v += d * f(s.y1, s.x1);
  return v;
}

// eps: n x 2 (y, x); w: n weights. Per EP: signed EPE (pixels; NaN when inactive) and,
// per CTA, FP64 partial sums (weighted squared loss, |EPE| nm, active count). With
// keys set, EP i writes its stencil's contributions scatter_scale x 2 w (I - thr) / G^2
// x weight to keys / vals [4 i .. 4 i + 3] (pixel index, or NO_PIXEL for an empty slot).
constexpr int EPE_NT = 256;
constexpr uint32_t NO_PIXEL = 0xFFFFFFFFu;
__global__ void __launch_bounds__(EPE_NT)
epe_kernel(const float* __restrict__ I, int rows, int cols, const double* __restrict__ eps,
           const double* __restrict__ w, int n, double thr, double pixel_nm,
           double* __restrict__ signed_epe, double* __restrict__ partial,
           uint32_t* __restrict__ keys, double* __restrict__ vals, double scatter_scale) {
  pdl_trigger();
  pdl_wait();
  __shared__ double sh[EPE_NT / 32];
  const int i = blockIdx.x * EPE_NT + threadIdx.x;
  double loss = 0.0, absn = 0.0, active = 0.0;
  if (i < n) {
    const double wi = w[i];
    double se = nan("");
    if (keys)
      for (int c = 0; c < 4; ++c) keys[4 * (size_t)i + c] = NO_PIXEL;
    if (wi > 0.0) {
      const Stencil s = make_stencil(rows, cols, eps[2 * i], eps[2 * i + 1]);
      const double a = sample(s, [&](int y, int x) { return (double)__ldg(I + (size_t)y * cols + x); });
      const double m = fmax(sample(s, [&](int y, int x) { return grad_mag(I, rows, cols, y, x); }), 1e-6);
      se = (a - thr) / m;
      loss = wi * se * se;
      absn = fabs(se) * pixel_nm;
      active = 1.0;
      if (keys) {
        // bilinear_scatter (epe_utils.cpp:76-80): the stencil's corners in the reference's
        // order; a repeated edge pixel appears twice with its partner's weight 0, and
        // zero-weight slots stay empty
        const double g = scatter_scale * (2.0 * wi * (a - thr) / (m * m));
        const double wt[4] = {(1.0 - s.wy1) * (1.0 - s.wx1), (1.0 - s.wy1) * s.wx1,
                              s.wy1 * (1.0 - s.wx1), s.wy1 * s.wx1};
        const int py[4] = {s.y0, s.y0, s.y1, s.y1}, px[4] = {s.x0, s.x1, s.x0, s.x1};
        for (int c = 0; c < 4; ++c)
          if (wt[c] > 0.0) {
            keys[4 * (size_t)i + c] = (uint32_t)py[c] * (uint32_t)cols + (uint32_t)px[c];
            vals[4 * (size_t)i + c] = wt[c] * g;
          }
      }
    }
    if (signed_epe) signed_epe[i] = se;
  }
  const double l = block_sum<EPE_NT>(loss, sh);
  const double an = block_sum<EPE_NT>(absn, sh);
  const double ac = block_sum<EPE_NT>(active, sh);
  if (threadIdx.x == 0) {
    partial[3 * blockIdx.x] = l;
    partial[3 * blockIdx.x + 1] = an;
    partial[3 * blockIdx.x + 2] = ac;
  }
}

// The sorted contributions of pixel keys[t] summed in order by the first entry of its
// run (each pixel written by one thread) and added to dldi once.
__global__ void epe_runs_kernel(const uint32_t* __restrict__ keys, const double* __restrict__ vals,
                                int m, uint32_t npix, float* __restrict__ dldi) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m) return;
  const uint32_t k = keys[t];
  if (k >= npix || (t > 0 && keys[t - 1] == k)) return;
  double sum = 0.0;
  for (int u = t; u < m && keys[u] == k; ++u) sum += vals[u];
  dldi[k] += (float)sum;
}

namespace {
struct ScatterWork {
  uint32_t *k_in, *k_out;
  double *v_in, *v_out;
  void* temp;
  size_t temp_bytes, total;
};
size_t align256(size_t v) { return (v + 255) / 256 * 256; }
ScatterWork scatter_layout(int n, void* base) {
  ScatterWork w{};
  const size_t m = 4 * (size_t)(n > 0 ? n : 1);
  cub::DeviceRadixSort::SortPairs(nullptr, w.temp_bytes, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                  (double*)nullptr, (double*)nullptr, (int)m);
  char* p = static_cast<char*>(base);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = align256(off + bytes);
    return p ? p + o : nullptr;
  };
  w.k_in = reinterpret_cast<uint32_t*>(take(m * sizeof(uint32_t)));
  w.k_out = reinterpret_cast<uint32_t*>(take(m * sizeof(uint32_t)));
  w.v_in = reinterpret_cast<double*>(take(m * sizeof(double)));
  w.v_out = reinterpret_cast<double*>(take(m * sizeof(double)));
  w.temp = take(w.temp_bytes);
  w.total = off;
  return w;
}
}  // namespace

size_t epe_scatter_work_bytes(int n) { return scatter_layout(n, nullptr).total; }

cudaError_t launch_epe(cudaStream_t s, const float* I, int rows, int cols, const double* eps,
                       const double* w, int n, double thr, double pixel_nm, double* signed_epe,
                       double* partial, float* dldi, double scatter_scale, int* nblocks,
                       void* work, size_t work_bytes) {
  *nblocks = (n + EPE_NT - 1) / EPE_NT;
  if (*nblocks == 0) *nblocks = 1;
  ScatterWork sw{};
  const bool scatter = dldi && n > 0;
  if (scatter) {
    sw = scatter_layout(n, work);
    if (!work || work_bytes < sw.total) return cudaErrorInvalidValue;
  }
  cudaError_t e = launch_pdl(epe_kernel, dim3(*nblocks), dim3(EPE_NT), 0, s, I, rows, cols, eps, w,
                             n, thr, pixel_nm, signed_epe, partial, scatter ? sw.k_in : nullptr,
                             scatter ? sw.v_in : nullptr, scatter_scale);
  if (e != cudaSuccess || !scatter) return e;
  const int m = 4 * n;
  size_t tb = sw.temp_bytes;
  e = cub::DeviceRadixSort::SortPairs(sw.temp, tb, sw.k_in, sw.k_out, sw.v_in, sw.v_out, m, 0,
                                      32, s);
  if (e != cudaSuccess) return e;
  epe_runs_kernel<<<(m + 255) / 256, 256, 0, s>>>(sw.k_out, sw.v_out, m,
                                                  (uint32_t)rows * (uint32_t)cols, dldi);
  return cudaGetLastError();
}

}  // namespace litho_b200
