// WENO5-Godunov level-set kernels (source/utils/level_set_utils.cpp of the
// reference) as shared-memory-tiled stencils.
//
// Boundary handling: the reference edge-pads phi by 3 on both axes and
// der_weno5 pads by 3 more along the derivative axis; edge padding twice is
// edge padding once by 6, and after cropping the output pixel (i, j) reads
// phi[i][clamp(j-3 .. j+3)] and phi[clamp(i-3 .. i+3)][j]. The tile loader
// therefore clamps every halo index into the image.
#include <cuda_runtime.h>
#include <algorithm>
#include <cfloat>

#include "litho_internal.cuh"

namespace litho_b200 {

constexpr int LS_TX = 32;      // tile width (x, columns)
constexpr int LS_TY = 8;       // rows per pass of the CTA; each thread computes LS_RPT rows
constexpr int LS_RPT = 4;
constexpr int LS_H = 3;        // halo
constexpr int LS_SW = LS_TX + 2 * LS_H;
constexpr int LS_SH = LS_TY * LS_RPT + 2 * LS_H;
constexpr int LS_NT = LS_TX * LS_TY;
static_assert(LS_TX == 32 && LS_SW <= 64, "the tile loader maps one warp to one tile row");

// WENO5-JS one-sided derivative from the five differences v1..v5 (already divided by
// the spacing), level_set_utils.cpp:45-113, for two stencils at once: lane x of the
// result is the derivative of (v1.x .. v5.x), lane y that of (v1.y .. v5.y). The
// arithmetic is packed FP32x2 (sm_100 FFMA2 / FMUL2 / FADD2: one instruction for both
// lanes, each lane rounded as the scalar operation), which halves the instructions of
// this part of an issue-bound stencil. The smoothness indicators are scaled by
// 1/max(v^2) before forming the weights: the weights are invariant under that scaling
// (eps = 1e-6 max v^2 scales the same way) and the scaled values stay inside FP32
// range. alpha_i = gamma_i / S_i^2 and the result sum(alpha_i d_i) / sum(alpha_i) are
// both multiplied by S1^2 S2^2 S3^2 (one division instead of four; the scaled S_i lie
// in [1e-6, 34], so the products stay well inside FP32 range). __fdividef (within 2
// ulp) serves the reciprocal and the division: max v^2 and the weight sum stay far
// inside the range where it is accurate.
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 weno5x2(float2 v1, float2 v2, float2 v3, float2 v4, float2 v5) {
  const float2 d1 = __ffma2_rn(f2(11.f / 6.f), v3, __ffma2_rn(f2(-7.f / 6.f), v2, __fmul2_rn(f2(1.f / 3.f), v1)));
  const float2 d2 = __ffma2_rn(f2(1.f / 3.f), v4, __ffma2_rn(f2(5.f / 6.f), v3, __fmul2_rn(f2(-1.f / 6.f), v2)));
  const float2 d3 = __ffma2_rn(f2(-1.f / 6.f), v5, __ffma2_rn(f2(5.f / 6.f), v4, __fmul2_rn(f2(1.f / 3.f), v3)));
  const float2 s1 = __fmul2_rn(v1, v1), s2 = __fmul2_rn(v2, v2), s3 = __fmul2_rn(v3, v3);
  const float2 s4 = __fmul2_rn(v4, v4), s5 = __fmul2_rn(v5, v5);
  const float mx = fmaxf(fmaxf(fmaxf(s1.x, s2.x), fmaxf(s3.x, s4.x)), s5.x);
  const float my = fmaxf(fmaxf(fmaxf(s1.y, s2.y), fmaxf(s3.y, s4.y)), s5.y);
  // all differences of a lane zero: its candidates are zero, and so is its result
  // (inv = 0 keeps its weights finite)
  const float2 inv = make_float2(mx > 0.f ? __fdividef(1.f, mx) : 0.f,
                                 my > 0.f ? __fdividef(1.f, my) : 0.f);
  const float2 t1 = __fadd2_rn(__ffma2_rn(f2(-2.f), v2, v1), v3);
  const float2 t2 = __fadd2_rn(__ffma2_rn(f2(-2.f), v3, v2), v4);
  const float2 t3 = __fadd2_rn(__ffma2_rn(f2(-2.f), v4, v3), v5);
  const float2 q1 = __ffma2_rn(f2(3.f), v3, __ffma2_rn(f2(-4.f), v2, v1));
  const float2 q2 = __ffma2_rn(f2(-1.f), v4, v2);
  const float2 q3 = __fadd2_rn(__ffma2_rn(f2(-4.f), v4, __fmul2_rn(f2(3.f), v3)), v5);
  auto smooth = [&](float2 t, float2 q) {
    const float2 a = __fmul2_rn(__fmul2_rn(f2(13.f / 12.f), t), t);
    return __ffma2_rn(__ffma2_rn(__fmul2_rn(f2(0.25f), q), q, a), inv, f2(1e-6f));
  };
  const float2 S1 = smooth(t1, q1), S2 = smooth(t2, q2), S3 = smooth(t3, q3);
  const float2 w1 = __fmul2_rn(S1, S1), w2 = __fmul2_rn(S2, S2), w3 = __fmul2_rn(S3, S3);
  const float2 b1 = __fmul2_rn(f2(0.1f), __fmul2_rn(w2, w3));
  const float2 b2 = __fmul2_rn(f2(0.6f), __fmul2_rn(w1, w3));
  const float2 b3 = __fmul2_rn(f2(0.3f), __fmul2_rn(w1, w2));
  const float2 num = __ffma2_rn(b3, d3, __ffma2_rn(b2, d2, __fmul2_rn(b1, d1)));
  const float2 den = __fadd2_rn(__fadd2_rn(b1, b2), b3);
  return make_float2(__fdividef(num.x, den.x), __fdividef(num.y, den.y));
}

// Godunov |grad phi| for the sign of the normal speed (level_set_utils.cpp:180-213).
__device__ __forceinline__ float godunov(float speed, float xm, float xp, float ym, float yp) {
  float gx2 = 0.f, gy2 = 0.f;
  if (speed > 0.f) {
    const float a = fmaxf(xm, 0.f), b = fminf(xp, 0.f);
    const float c = fmaxf(ym, 0.f), d = fminf(yp, 0.f);
    gx2 = fmaxf(a * a, b * b);
    gy2 = fmaxf(c * c, d * d);
  } else if (speed < 0.f) {
    const float a = fminf(xm, 0.f), b = fmaxf(xp, 0.f);
    const float c = fminf(ym, 0.f), d = fmaxf(yp, 0.f);
    gx2 = fmaxf(a * a, b * b);
    gy2 = fmaxf(c * c, d * d);
  }
  return sqrtf(gx2 + gy2);
}

__device__ __forceinline__ void load_tile(float (*t)[LS_SW], const float* __restrict__ phi,
                                          int rows, int cols, int y0, int x0) {
  // warp w loads tile rows w, w + 8, ...; each lane columns lane and lane + 32
  const int lane = threadIdx.x & 31;
  const int xa = min(max(x0 - LS_H + lane, 0), cols - 1);
  const int xb = min(max(x0 - LS_H + lane + 32, 0), cols - 1);
  for (int ty = threadIdx.x >> 5; ty < LS_SH; ty += LS_NT / 32) {
    const float* row = phi + (size_t)min(max(y0 - LS_H + ty, 0), rows - 1) * cols;
    t[ty][lane] = __ldg(row + xa);
    if (lane + 32 < LS_SW) t[ty][lane + 32] = __ldg(row + xb);
  }
}

// delta = Vn |grad phi|_G at tile pixel (ly, lx) (tile coordinates include the halo).
__device__ __forceinline__ float weno_delta(const float (*t)[LS_SW], int ly, int lx, float speed,
                                            float idx, float idy) {
  float d[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) d[q] = (t[ly][lx - 2 + q] - t[ly][lx - 3 + q]) * idx;
  // minus: D(j-3..j+1) = d[0..4]; plus: mirrored d[5..1]; both in one packed call
  const float2 xmp = weno5x2(make_float2(d[0], d[5]), make_float2(d[1], d[4]),
                             make_float2(d[2], d[3]), make_float2(d[3], d[2]),
                             make_float2(d[4], d[1]));
#pragma unroll
  for (int q = 0; q < 6; ++q) d[q] = (t[ly - 2 + q][lx] - t[ly - 3 + q][lx]) * idy;
  const float2 ymp = weno5x2(make_float2(d[0], d[5]), make_float2(d[1], d[4]),
                             make_float2(d[2], d[3]), make_float2(d[3], d[2]),
                             make_float2(d[4], d[1]));
  return speed * godunov(speed, xmp.x, xmp.y, ymp.x, ymp.y);
}

// _gradient_1d along x (level_set_utils.cpp:228-255) at global column x of row ly.
__device__ __forceinline__ float grad_x(const float (*t)[LS_SW], int ly, int lx, int x, int cols,
                                        float inv2d) {
  if (x == 0) return (-3.f * t[ly][lx] + 4.f * t[ly][lx + 1] - t[ly][lx + 2]) * inv2d;
  if (x == cols - 1) return (3.f * t[ly][lx] - 4.f * t[ly][lx - 1] + t[ly][lx - 2]) * inv2d;
  return (t[ly][lx + 1] - t[ly][lx - 1]) * inv2d;
}
__device__ __forceinline__ float grad_y(const float (*t)[LS_SW], int ly, int lx, int y, int rows,
                                        float inv2d) {
  if (y == 0) return (-3.f * t[ly][lx] + 4.f * t[ly + 1][lx] - t[ly + 2][lx]) * inv2d;
  if (y == rows - 1) return (3.f * t[ly][lx] - 4.f * t[ly - 1][lx] + t[ly - 2][lx]) * inv2d;
  return (t[ly + 1][lx] - t[ly - 1][lx]) * inv2d;
}

// b * kappa |grad phi| (level_set_utils.cpp:257-278) at global (y, x).
__device__ float kappa_term(const float (*t)[LS_SW], int ly, int lx, int y, int x, int rows,
                            int cols, float dx, float dy, float b) {
  const float ix = 1.f / (2.f * dx), iy = 1.f / (2.f * dy);
  float px, py, pxy, pxx, pyy;
  if (x >= 2 && x < cols - 2 && y >= 2 && y < rows - 2) {
    // Away from the image border every difference below is the central one: the
    // same arithmetic as the general path, without its border tests.
    auto cx = [&](int oy, int ox) { return (t[ly + oy][lx + ox + 1] - t[ly + oy][lx + ox - 1]) * ix; };
    auto cy = [&](int oy) { return (t[ly + oy + 1][lx] - t[ly + oy - 1][lx]) * iy; };
    px = cx(0, 0);
    py = cy(0);
    pxy = (cx(1, 0) - cx(-1, 0)) * iy;
    pxx = (cx(0, 1) - cx(0, -1)) * ix;
    pyy = (cy(1) - cy(-1)) * iy;
    const float g2 = px * px + py * py;
    const float num = pxx * py * py - 2.f * px * py * pxy + pyy * px * px;
    return g2 > (float)DBL_EPSILON ? b * __fdividef(num, g2) : 0.f;
  }
  // phi_x at (y, x) and its row/column neighbours used by the second derivatives.
  auto px_at = [&](int oy, int ox) { return grad_x(t, ly + oy, lx + ox, x + ox, cols, ix); };
  auto py_at = [&](int oy) { return grad_y(t, ly + oy, lx, y + oy, rows, iy); };
  px = px_at(0, 0);
  py = py_at(0);
  if (y == 0) pxy = (-3.f * px + 4.f * px_at(1, 0) - px_at(2, 0)) * iy;
  else if (y == rows - 1) pxy = (3.f * px - 4.f * px_at(-1, 0) + px_at(-2, 0)) * iy;
  else pxy = (px_at(1, 0) - px_at(-1, 0)) * iy;
  if (x == 0) pxx = (-3.f * px + 4.f * px_at(0, 1) - px_at(0, 2)) * ix;
  else if (x == cols - 1) pxx = (3.f * px - 4.f * px_at(0, -1) + px_at(0, -2)) * ix;
  else pxx = (px_at(0, 1) - px_at(0, -1)) * ix;
  if (y == 0) pyy = (-3.f * py + 4.f * py_at(1) - py_at(2)) * iy;
  else if (y == rows - 1) pyy = (3.f * py - 4.f * py_at(-1) + py_at(-2)) * iy;
  else pyy = (py_at(1) - py_at(-1)) * iy;
  const float g2 = px * px + py * py;
  const float num = pxx * py * py - 2.f * px * py * pxy + pyy * px * px;
  return g2 > (float)DBL_EPSILON ? b * __fdividef(num, g2) : 0.f;
}

__device__ float block_max(float v, float* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  float r = 0.f;
  if (threadIdx.x == 0)
    for (int w = 0; w < LS_NT / 32; ++w) r = fmaxf(r, sh[w]);
  __syncthreads();
  return r;
}

// what: 0 = delta (+ habs), 1 = kappa term, 2 = normal = kappa - delta,
// 3 = RK2 stage 1: out = phi0 + dt N(phi0), 4 = RK2 stage 2:
// out = 0.5 phi0 + 0.5 (phi1 + dt N(phi1)), mask_out = out >= 0.
struct LsArgs {
  int rows, cols, what;
  const float* phi;   // field whose stencil is evaluated
  const float* phi0;  // stage 2: the step's starting phi
  const float* vn;
  float dx, dy, b;
  const float* dt;    // device scalar (stages)
  float* out;
  float* out2;        // habs (what 0) or mask (what 4)
  int wy0, wy1, wx0, wx1;  // update window [wy0, wy1) x [wx0, wx1) (stages 3, 4 and what 6, 8)
  // Batched launches: image blockIdx.z of rows x cols images back to back; its dt at
  // dt[blockIdx.z * dt_stride]; its window from wins[4 blockIdx.z ..] when wins is set.
  const int* wins;
  int dt_stride;
};

// WHAT (the mode, LsArgs::what) is a template parameter so that the per-pixel loop
// carries no mode tests.
template <int WHAT>
__global__ void __launch_bounds__(LS_NT) levelset_kernel(LsArgs a) {
  const size_t img = (size_t)blockIdx.z * a.rows * a.cols;
  const float* phi = a.phi + img;
  float* out = a.out + img;
  int wy0 = a.wy0, wy1 = a.wy1, wx0 = a.wx0, wx1 = a.wx1;
  if (a.wins) {
    const int* w = a.wins + 4 * (size_t)blockIdx.z;
    wy0 = w[0]; wy1 = w[1]; wx0 = w[2]; wx1 = w[3];
  }
  if (WHAT >= 5) {  // elementwise modes
    const int x = blockIdx.x * LS_TX + threadIdx.x % LS_TX;
    for (int r = 0; r < LS_RPT; ++r) {
      const int y = blockIdx.y * LS_TY * LS_RPT + threadIdx.x / LS_TX + r * LS_TY;
      if (y < a.rows && x < a.cols) {
        const size_t i = (size_t)y * a.cols + x;
        const bool in = y >= wy0 && y < wy1 && x >= wx0 && x < wx1;
        if (WHAT == 5)         // printed mask: phi >= 0 (LSM_Optimizer.cpp:128)
          out[i] = phi[i] >= 0.f ? 1.f : 0.f;
        else if (WHAT == 6)    // speed restricted to the update window
          out[i] = in ? a.vn[img + i] : 0.f;
        else if (WHAT == 7)    // +-0.5 sign image of phi >= 0 (full_chip_lsm.cpp:229-230)
          out[i] = phi[i] >= 0.f ? 0.5f : -0.5f;
        else if (WHAT == 9)    // mask - 0.5 (full_chip_lsm.cpp:143)
          out[i] = phi[i] - 0.5f;
        else                     // commit phi inside the window over phi0 (out may be phi0)
          out[i] = in ? phi[i] : a.phi0[img + i];
      }
    }
    return;
  }
  __shared__ float t[LS_SH][LS_SW];
  const int x0 = blockIdx.x * LS_TX;
  const int y0 = blockIdx.y * LS_TY * LS_RPT;
  load_tile(t, phi, a.rows, a.cols, y0, x0);
  __syncthreads();
  const float idx = 1.f / a.dx, idy = 1.f / a.dy;
  const float dt = (WHAT >= 3) ? a.dt[(size_t)blockIdx.z * a.dt_stride] : 0.f;
  const float* phi0 = a.phi0 ? a.phi0 + img : nullptr;
  const float* vn = a.vn ? a.vn + img : nullptr;
  float* out2 = a.out2 ? a.out2 + img : nullptr;
  const int lx = threadIdx.x % LS_TX;
  for (int r = 0; r < LS_RPT; ++r) {
    const int ly = threadIdx.x / LS_TX + r * LS_TY;
    const int y = y0 + ly, x = x0 + lx;
    if (y >= a.rows || x >= a.cols) continue;
    const size_t i = (size_t)y * a.cols + x;
    if (WHAT >= 3 && !(y >= wy0 && y < wy1 && x >= wx0 && x < wx1)) {
      // Outside the update window the step keeps phi (stage 1) / the starting phi (stage 2).
      const float keep = WHAT == 3 ? t[ly + LS_H][lx + LS_H] : __ldg(phi0 + i);
      if (WHAT == 4 && out2) out2[i] = keep >= 0.f ? 1.f : 0.f;
      out[i] = keep;
      continue;
    }
    const float speed = WHAT == 1 ? 0.f : __ldg(vn + i);
    float v;
    if (WHAT == 0) {
      v = weno_delta(t, ly + LS_H, lx + LS_H, speed, idx, idy);
      if (out2) out2[i] = fabsf(speed);
    } else if (WHAT == 1) {
      v = kappa_term(t, ly + LS_H, lx + LS_H, y, x, a.rows, a.cols, a.dx, a.dy, a.b);
    } else {
      const float n = kappa_term(t, ly + LS_H, lx + LS_H, y, x, a.rows, a.cols, a.dx, a.dy, a.b) -
                      weno_delta(t, ly + LS_H, lx + LS_H, speed, idx, idy);
      if (WHAT == 2) {
        v = n;
      } else if (WHAT == 3) {
        v = t[ly + LS_H][lx + LS_H] + dt * n;
      } else {
        v = 0.5f * __ldg(phi0 + i) + 0.5f * (t[ly + LS_H][lx + LS_H] + dt * n);
        if (out2) out2[i] = v >= 0.f ? 1.f : 0.f;
      }
    }
    out[i] = v;
  }
}

static dim3 ls_grid(int rows, int cols) {
  return dim3((cols + LS_TX - 1) / LS_TX, (rows + LS_TY * LS_RPT - 1) / (LS_TY * LS_RPT));
}

cudaError_t launch_levelset(cudaStream_t s, int what, int rows, int cols, const float* phi,
                            const float* phi0, const float* vn, float dx, float dy, float b,
                            const float* dt, float* out, float* out2, const int* window,
                            int nimg, const int* d_windows, int dt_stride) {
  if (nimg < 1 || nimg > 65535) return cudaErrorInvalidValue;
  LsArgs a{rows, cols, what, phi, phi0, vn, dx, dy, b, dt, out, out2, 0, rows, 0, cols,
           d_windows, dt_stride};
  if (window) {
    a.wy0 = window[0]; a.wy1 = window[1]; a.wx0 = window[2]; a.wx1 = window[3];
  }
  dim3 g = ls_grid(rows, cols);
  g.z = nimg;
  switch (what) {
    case 0: levelset_kernel<0><<<g, LS_NT, 0, s>>>(a); break;
    case 1: levelset_kernel<1><<<g, LS_NT, 0, s>>>(a); break;
    case 2: levelset_kernel<2><<<g, LS_NT, 0, s>>>(a); break;
    case 3: levelset_kernel<3><<<g, LS_NT, 0, s>>>(a); break;
    case 4: levelset_kernel<4><<<g, LS_NT, 0, s>>>(a); break;
    case 5: levelset_kernel<5><<<g, LS_NT, 0, s>>>(a); break;
    case 6: levelset_kernel<6><<<g, LS_NT, 0, s>>>(a); break;
    case 7: levelset_kernel<7><<<g, LS_NT, 0, s>>>(a); break;
    case 8: levelset_kernel<8><<<g, LS_NT, 0, s>>>(a); break;
    case 9: levelset_kernel<9><<<g, LS_NT, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// max |Vn| partials then dt = get_dt_normal_kappa (level_set_utils.cpp:280-288).
__global__ void __launch_bounds__(LS_NT) absmax_kernel(const float* __restrict__ v, size_t n,
                                                       float* __restrict__ part, int* bad) {
  __shared__ float sh[LS_NT / 32];
  v += (size_t)blockIdx.y * n;                 // image blockIdx.y of a batched launch
  part += (size_t)blockIdx.y * gridDim.x;
  float m = 0.f;
  bool nonfinite = false;
  for (size_t i = (size_t)blockIdx.x * LS_NT + threadIdx.x; i < n; i += (size_t)gridDim.x * LS_NT) {
    const float a = v[i];
    nonfinite |= !isfinite(a);
    m = fmaxf(m, fabsf(a));
  }
  if (nonfinite && bad) atomicOr(bad, 1);
  const float r = block_max(m, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = r;
}

__global__ void dt_kernel(const float* __restrict__ part, int n, float dx, float dy, float cfl,
                          float b, float* __restrict__ vmax, float* __restrict__ dt) {
  if (threadIdx.x != 0) return;
  float m = 0.f;
  for (int i = 0; i < n; ++i) m = fmaxf(m, part[i]);
  const double normal = (double)m / dx + (double)m / dy;
  const double kap = (double)b * (1.0 / ((double)dx * dx) + 1.0 / ((double)dy * dy)) * 2.0;
  const double den = normal + kap;
  *vmax = m;
  *dt = den < 1e-9 ? 1e-3f : (float)(cfl / den);
}

// dt of every image of a batched launch: vd[2 i] = max |Vn|, vd[2 i + 1] = dt.
__global__ void dt_batch_kernel(const float* __restrict__ part, int nb, float dx, float dy,
                                float cfl, float b, float* __restrict__ vd) {
  const float* p = part + (size_t)blockIdx.x * nb;
  float m = 0.f;
  for (int i = threadIdx.x; i < nb; i += 32) m = fmaxf(m, p[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (threadIdx.x != 0) return;
  const double normal = (double)m / dx + (double)m / dy;
  const double kap = (double)b * (1.0 / ((double)dx * dx) + 1.0 / ((double)dy * dy)) * 2.0;
  const double den = normal + kap;
  vd[2 * (size_t)blockIdx.x] = m;
  vd[2 * (size_t)blockIdx.x + 1] = den < 1e-9 ? 1e-3f : (float)(cfl / den);
}

int dt_batch_blocks(size_t n, int nimg) {
  const size_t want = (n + LS_NT - 1) / LS_NT;
  const size_t cap = std::max<size_t>(1, 1184 / (size_t)std::max(nimg, 1));
  return (int)std::max<size_t>(1, std::min(want, cap));
}

cudaError_t launch_dt_batch(cudaStream_t s, const float* vn, size_t n, int nimg, float dx,
                            float dy, float cfl, float b, float* part, float* vd, int* bad) {
  if (nimg < 1 || nimg > 65535) return cudaErrorInvalidValue;
  const int nb = dt_batch_blocks(n, nimg);
  absmax_kernel<<<dim3(nb, nimg), LS_NT, 0, s>>>(vn, n, part, bad);
  dt_batch_kernel<<<nimg, 32, 0, s>>>(part, nb, dx, dy, cfl, b, vd);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- mask rendering
// render_levelset_mask (levelset_mask_renderer.cpp:7-33), Gray mode: phi (float32)
// upsampled by `scale` with pixel-centre bilinear interpolation and edge
// replication (the cv::resize INTER_LINEAR convention), then the fraction of each
// source pixel's scale x scale subpixels with phi >= 0. Upsampled coordinate X
// samples the source at u = (X + 0.5) / scale - 0.5: columns floor(u) and
// floor(u) + 1 with weights 1 - t and t, t = u - floor(u); before the first and
// from the last source column on the edge value is used alone (t = 0). The two
// passes are separable: rows first, then columns, each a product sum in FP32.
// nimg images of rows x cols lie back to back; one thread per source pixel.
__device__ __forceinline__ void bilinear_coord(int X, int n, double inv, int& i0, int& i1,
                                               float& w0, float& w1) {
  float u = (float)((X + 0.5) * inv - 0.5);
  int i = (int)floorf(u);
  float t = u - (float)i;
  if (i < 0) { i = 0; t = 0.f; }
  if (i >= n - 1) { i = n - 1; t = 0.f; }
  i0 = i;
  i1 = min(i + 1, n - 1);
  w0 = 1.f - t;
  w1 = t;
}

__global__ void render_gray_kernel(const float* __restrict__ phi, int rows, int cols, int nimg,
                                   int scale, float* __restrict__ mask) {
  const size_t per = (size_t)rows * cols;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= per * nimg) return;
  const int img = (int)(idx / per);
  const int y = (int)((idx % per) / cols), x = (int)(idx % cols);
  const float* p = phi + (size_t)img * per;
  const double inv = 1.0 / scale;
  int inside = 0;
  for (int sy = 0; sy < scale; ++sy) {
    int r0, r1;
    float b0, b1;
    bilinear_coord(y * scale + sy, rows, inv, r0, r1, b0, b1);
    for (int sx = 0; sx < scale; ++sx) {
      int c0, c1;
      float a0, a1;
      bilinear_coord(x * scale + sx, cols, inv, c0, c1, a0, a1);
      const float h0 = __fadd_rn(__fmul_rn(p[(size_t)r0 * cols + c0], a0),
                                 __fmul_rn(p[(size_t)r0 * cols + c1], a1));
      const float h1 = __fadd_rn(__fmul_rn(p[(size_t)r1 * cols + c0], a0),
                                 __fmul_rn(p[(size_t)r1 * cols + c1], a1));
      const float v = __fadd_rn(__fmul_rn(h0, b0), __fmul_rn(h1, b1));
      inside += v >= 0.f;
    }
  }
  mask[idx] = (float)((double)inside / ((double)scale * scale));
}

__global__ void render_binary_kernel(const float* __restrict__ phi, size_t n,
                                     float* __restrict__ mask) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) mask[i] = phi[i] >= 0.f ? 1.f : 0.f;
}

cudaError_t launch_render_mask(cudaStream_t s, const float* phi, int rows, int cols, int nimg,
                               int gray, int scale, float* mask) {
  const size_t n = (size_t)rows * cols * nimg;
  const unsigned nb = (unsigned)((n + 255) / 256);
  if (gray)
    render_gray_kernel<<<nb, 256, 0, s>>>(phi, rows, cols, nimg, scale, mask);
  else
    render_binary_kernel<<<nb, 256, 0, s>>>(phi, n, mask);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- reinit_sdf
// LevelSetUtils::reinit_sdf (level_set_utils.cpp:290-319): two OpenCV
// distanceTransform(DIST_L2, 5) calls, i.e. the 5x5 chamfer distance with
// weights a = 1, b = 1.4, c = 2.1969 (float32) to the nearest feature pixel,
// computed by a forward raster pass (rows top to bottom, left to right) and a
// backward pass, each pixel taking the minimum of its own value and its already
// final neighbours plus the weights. Within a row the only dependency is
// d(j) = min(g(j), d(j-1) + a), g being the minimum over the rows above (below)
// plus the pixel's own value. A CTA splits a row into one contiguous segment per
// thread: each thread runs the recurrence over its segment from +inf, the segment
// results are combined by a block scan with the composition
//   (A1, L1) then (A2, L2)  ->  (min(A2, A1 + L2), L1 + L2)
// (A: the value at the segment's last column, L: its length), and each thread reruns
// its segment from the carry it receives. Float throughout, in a fixed order.
//
// One CTA runs one transform of one image (blockIdx.y): blockIdx.x = 0 measures
// inside pixels to the outside and writes +d dx at the inside pixels, blockIdx.x = 1
// measures outside pixels to the inside and writes -d dx at the outside pixels. A
// transform's distance is 0 at its feature pixels (the other class), so each CTA keeps
// its forward-pass values in the output at its own pixels only: the two CTAs of an
// image touch disjoint pixels and need no other buffer. Inside means phi > level
// (phi >= level when `inclusive`). With no feature pixel at all the distance stays
// FLT_MAX, as OpenCV returns.
//
// PMAX > 0: a thread owns at most PMAX columns and holds their classification (and,
// backward, their forward-pass values) in registers, loading the following rows'
// while the current row is processed, so that the row loop waits on no global load.
// PMAX == 0: the same transform with direct loads (very long rows).
constexpr float DT_A = 1.0f, DT_B = 1.4f, DT_C = 2.1969f;

template <int NT, int PMAX>
__global__ void __launch_bounds__(NT)
chamfer_sdf_kernel(const float* __restrict__ phi_all, int rows, int cols, float level,
                   int inclusive, float dx, float* __restrict__ sdf_all) {
  extern __shared__ float rowbuf[];  // ring of 3 rows of W = cols + 4 floats, column j at j + 2
  __shared__ float wtot[32];
  constexpr int NW = NT / 32;
  constexpr int QN = PMAX > 0 ? PMAX : 1;
  const float FMAX = 3.402823466e38f;
  const int W = cols + 4;
  const bool inside_pass = blockIdx.x == 0;
  const size_t img = (size_t)blockIdx.y * rows * cols;
  const float* phi = phi_all + img;
  float* sdf = sdf_all + img;
  const int per = (cols + NT - 1) / NT;  // columns per thread
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int j0 = min((int)threadIdx.x * per, cols);
  const int nq = min(per, cols - j0);    // columns this thread owns (0 past the row end)
  auto seg_end = [&](int t) { return min((t + 1) * per, cols); };   // one past the last column
  auto seg_start = [&](int t) { return min(t * per, cols); };
  if (threadIdx.x < 3) {  // +inf pads: two columns on each side of every ring row
    float* r = rowbuf + threadIdx.x * W;
    r[0] = r[1] = r[W - 2] = r[W - 1] = FMAX;
  }
  auto cls = [&](float p) { return (inclusive ? p >= level : p > level) == inside_pass; };
  auto load_bits = [&](int i) {
    unsigned b = 0;
#pragma unroll
    for (int q = 0; q < QN; ++q)
      if (q < nq && cls(phi[(size_t)i * cols + j0 + q])) b |= 1u << q;
    return b;
  };
  unsigned bits0 = 0, bits1 = 0;   // own-pixel bits of the current row and the next one
  float pf[QN];                    // phi of a following row, in flight
  float fv[QN];                    // backward: forward-pass values of the current row
  auto own = [&](int i, int q) -> bool {
    if constexpr (PMAX > 0) return ((bits0 >> q) & 1u) != 0u;
    else return cls(phi[(size_t)i * cols + j0 + q]);
  };
  const int qn = PMAX > 0 ? QN : per;

  // ---- forward pass
  if constexpr (PMAX > 0) bits0 = load_bits(0);
  for (int i = 0; i < rows; ++i) {
    float* r0 = rowbuf + (i % 3) * W + 2;
    const float* r1 = rowbuf + ((i + 2) % 3) * W + 2;  // row i-1
    const float* r2 = rowbuf + ((i + 1) % 3) * W + 2;  // row i-2
    float a = FMAX;
#pragma unroll
    for (int q = 0; q < qn; ++q) {
      if (q >= nq) break;
      const int j = j0 + q;
      float g = 0.f;   // a feature pixel of this transform
      if (own(i, q)) {
        g = FMAX;
        if (i >= 1)
          g = fminf(fminf(fminf(r1[j] + DT_A, r1[j - 1] + DT_B), fminf(r1[j + 1] + DT_B, r1[j - 2] + DT_C)),
                    r1[j + 2] + DT_C);
        if (i >= 2) g = fminf(g, fminf(r2[j - 1] + DT_C, r2[j + 1] + DT_C));
      }
      a = fminf(g, a + DT_A);
      r0[j] = g;
    }
    if constexpr (PMAX > 0) {
      if (i + 1 < rows) {
#pragma unroll
        for (int q = 0; q < QN; ++q) pf[q] = q < nq ? phi[(size_t)(i + 1) * cols + j0 + q] : 0.f;
      }
    }
    // inclusive scan over the threads of the segment results
    float v = a;
    const int e = seg_end(threadIdx.x);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const float u = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v = fminf(v, u + (float)(e - seg_end(threadIdx.x - o)));
    }
    if (lane == 31) wtot[warp] = v;
    __syncthreads();
    if (warp == 0) {
      float x = lane < NW ? wtot[lane] : FMAX;
      const int ew = seg_end(32 * lane + 31);
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const float u = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o && lane < NW) x = fminf(x, u + (float)(ew - seg_end(32 * (lane - o) + 31)));
      }
      if (lane < NW) wtot[lane] = x;
    }
    __syncthreads();
    // carry: the value at column j0 - 1
    float c = __shfl_up_sync(0xffffffffu, v, 1);
    if (lane == 0) c = FMAX;
    if (warp > 0) {
      const int wend = seg_end(32 * warp - 1);   // end of the previous warp's segments
      const float wc = wtot[warp - 1] + (float)(j0 - wend);
      c = lane == 0 ? wtot[warp - 1] : fminf(c, wc);
    }
    float d = c;
#pragma unroll
    for (int q = 0; q < qn; ++q) {
      if (q >= nq) break;
      const int j = j0 + q;
      d = fminf(r0[j], d + DT_A);
      r0[j] = d;
      if (own(i, q)) sdf[(size_t)i * cols + j] = d;
    }
    if constexpr (PMAX > 0) {
      if (i + 1 < rows) {
        unsigned b = 0;
#pragma unroll
        for (int q = 0; q < QN; ++q)
          if (q < nq && cls(pf[q])) b |= 1u << q;
        bits0 = b;
      }
    }
    __syncthreads();
  }
  // ---- backward pass
  if constexpr (PMAX > 0) {
    bits0 = load_bits(rows - 1);
    bits1 = rows >= 2 ? load_bits(rows - 2) : 0u;
#pragma unroll
    for (int q = 0; q < QN; ++q)
      fv[q] = (q < nq && ((bits0 >> q) & 1u)) ? sdf[(size_t)(rows - 1) * cols + j0 + q] : 0.f;
  }
  for (int i = rows - 1; i >= 0; --i) {
    const int slot = (rows - 1 - i);
    float* r0 = rowbuf + (slot % 3) * W + 2;
    const float* r1 = rowbuf + ((slot + 2) % 3) * W + 2;  // row i+1 (final)
    const float* r2 = rowbuf + ((slot + 1) % 3) * W + 2;  // row i+2 (final)
    float a = FMAX;
#pragma unroll
    for (int qq = 0; qq < qn; ++qq) {
      const int q = qn - 1 - qq;   // right to left
      if (q >= nq) continue;
      const int j = j0 + q;
      float g;   // the forward-pass value (0 at a feature pixel)
      if constexpr (PMAX > 0) g = fv[q];
      else g = own(i, q) ? sdf[(size_t)i * cols + j] : 0.f;
      if (g > DT_A) {
        if (i + 1 < rows)
          g = fminf(g, fminf(fminf(fminf(r1[j] + DT_A, r1[j + 1] + DT_B), fminf(r1[j - 1] + DT_B, r1[j + 2] + DT_C)),
                             r1[j - 2] + DT_C));
        if (i + 2 < rows) g = fminf(g, fminf(r2[j + 1] + DT_C, r2[j - 1] + DT_C));
      }
      a = fminf(g, a + DT_A);
      r0[j] = g;
    }
    if constexpr (PMAX > 0) {
      // forward values of row i - 1 (its bits are known), phi of row i - 2
      if (i >= 1) {
#pragma unroll
        for (int q = 0; q < QN; ++q)
          fv[q] = (q < nq && ((bits1 >> q) & 1u)) ? sdf[(size_t)(i - 1) * cols + j0 + q] : 0.f;
      }
      if (i >= 2) {
#pragma unroll
        for (int q = 0; q < QN; ++q) pf[q] = q < nq ? phi[(size_t)(i - 2) * cols + j0 + q] : 0.f;
      }
    }
    // inclusive scan from the right of the segment results (value at a segment's first column)
    float v = a;
    const int st = seg_start(threadIdx.x);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const float u = __shfl_down_sync(0xffffffffu, v, o);
      if (lane + o < 32) v = fminf(v, u + (float)(seg_start(threadIdx.x + o) - st));
    }
    if (lane == 0) wtot[warp] = v;
    __syncthreads();
    if (warp == 0) {
      float x = lane < NW ? wtot[lane] : FMAX;
      const int sw = seg_start(32 * lane);
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const float u = __shfl_down_sync(0xffffffffu, x, o);
        if (lane + o < NW) x = fminf(x, u + (float)(seg_start(32 * (lane + o)) - sw));
      }
      if (lane < NW) wtot[lane] = x;
    }
    __syncthreads();
    // carry: the value at column j0 + nq (the next segment's first column)
    float c = __shfl_down_sync(0xffffffffu, v, 1);
    if (lane == 31) c = FMAX;
    if (warp < NW - 1) {
      const int wst = seg_start(32 * (warp + 1));   // first column of the next warp's segments
      const float wc = wtot[warp + 1] + (float)(wst - seg_start(threadIdx.x + 1));
      c = lane == 31 ? wtot[warp + 1] : fminf(c, wc);
    }
    float d = c;
#pragma unroll
    for (int qq = 0; qq < qn; ++qq) {
      const int q = qn - 1 - qq;
      if (q >= nq) continue;
      const int j = j0 + q;
      d = fminf(r0[j], d + DT_A);
      r0[j] = d;
      if (own(i, q)) {
        if (inside_pass) sdf[(size_t)i * cols + j] = d >= FMAX ? FMAX : d * dx;
        else sdf[(size_t)i * cols + j] = d >= FMAX ? -FMAX : -d * dx;
      }
    }
    if constexpr (PMAX > 0) {
      unsigned b = 0;
      if (i >= 2) {
#pragma unroll
        for (int q = 0; q < QN; ++q)
          if (q < nq && cls(pf[q])) b |= 1u << q;
      }
      bits0 = bits1;
      bits1 = b;
    }
    __syncthreads();
  }
}

// A smooth test pattern (sin x cos y with a per-image phase) whose zero set crosses
// every row: the input of the chamfer timing of litho_ctx_autotune.
__global__ void chamfer_probe_kernel(float* __restrict__ p, int rows, int cols, int nimg) {
  const size_t n = (size_t)rows * cols * nimg;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % cols), y = (int)((i / cols) % rows), k = (int)(i / ((size_t)rows * cols));
    p[i] = sinf(0.031f * x + k) * cosf(0.027f * y) - 0.1f;
  }
}

cudaError_t launch_chamfer_probe(cudaStream_t s, float* p, int rows, int cols, int nimg) {
  chamfer_probe_kernel<<<1184, 256, 0, s>>>(p, rows, cols, nimg);
  return cudaGetLastError();
}

template <int NT, int PMAX>
static cudaError_t chamfer_launch(cudaStream_t s, int rows, int cols, const float* phi,
                                  float level, int inclusive, float dx, float* sdf, int nimg) {
  const size_t smem = (size_t)3 * (cols + 4) * sizeof(float);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(chamfer_sdf_kernel<NT, PMAX>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  chamfer_sdf_kernel<NT, PMAX><<<dim3(2, nimg), NT, smem, s>>>(phi, rows, cols, level, inclusive,
                                                               dx, sdf);
  return cudaGetLastError();
}

cudaError_t launch_reinit_sdf(cudaStream_t s, int rows, int cols, const float* phi, float level,
                              int inclusive, float dx, float* sdf, int nimg, int threads) {
  if (nimg < 1 || nimg > 65535 || rows < 1 || cols < 1) return cudaErrorInvalidValue;
  // Many images: small CTAs (long segments, little scan overhead, many CTAs per SM).
  // Few images: the row latency decides, so short segments over more threads.
  if (threads <= 0) {
    if (nimg >= 64) threads = cols <= 4096 ? 128 : cols <= 8192 ? 256 : 1024;
    else threads = cols <= 1536 ? 512 : 1024;
  }
  const int per = (cols + threads - 1) / threads;
  // the register arrays hold the smallest of 8, 16, 32 columns that covers a segment
  switch (threads) {
    case 128:
      if (per <= 8) return chamfer_launch<128, 8>(s, rows, cols, phi, level, inclusive, dx, sdf, nimg);
      if (per <= 16) return chamfer_launch<128, 16>(s, rows, cols, phi, level, inclusive, dx, sdf, nimg);
      if (per <= 32) return chamfer_launch<128, 32>(s, rows, cols, phi, level, inclusive, dx, sdf, nimg);
      return cudaErrorInvalidValue;
    case 256:
      if (per <= 32) return chamfer_launch<256, 32>(s, rows, cols, phi, level, inclusive, dx, sdf, nimg);
      return cudaErrorInvalidValue;
    case 512:
      if (per <= 8) return chamfer_launch<512, 8>(s, rows, cols, phi, level, inclusive, dx, sdf, nimg);
      if (per <= 16) return chamfer_launch<512, 16>(s, rows, cols, phi, level, inclusive, dx, sdf, nimg);
      return cudaErrorInvalidValue;
    case 1024:
      return chamfer_launch<1024, 0>(s, rows, cols, phi, level, inclusive, dx, sdf, nimg);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_dt(cudaStream_t s, const float* vn, size_t n, float dx, float dy, float cfl,
                      float b, float* part, float* vmax, float* dt, int* bad) {
  int nb = (int)((n + LS_NT - 1) / LS_NT);
  if (nb > 296) nb = 296;
  absmax_kernel<<<nb, LS_NT, 0, s>>>(vn, n, part, bad);
  dt_kernel<<<1, 32, 0, s>>>(part, nb, dx, dy, cfl, b, vmax, dt);
  return cudaGetLastError();
}

}  // namespace litho_b200
