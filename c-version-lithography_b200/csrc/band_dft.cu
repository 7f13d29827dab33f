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
// So the full-resolution work is four K-independent separable passes (row
// analysis / column contraction / column expansion / row synthesis); the
// K-dependent work lives on the small grid.
#include <cuda_runtime.h>
#include <math_constants.h>

#include "gemm_nt.cuh"
#include "litho_internal.cuh"

namespace litho_b200 {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ void cfma(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, fmaf(-a.y, b.y, acc.x));
  acc.y = fmaf(a.x, b.y, fmaf(a.y, b.x, acc.y));
}

// ---------------------------------------------------------------- FP64 block reduce
template <int NT>
__device__ double block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    for (int w = 0; w < NT / 32; ++w) r += sh[w];  // fixed order: deterministic
  }
  __syncthreads();
  return r;
}

// ---------------------------------------------------------------- row analysis
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
      float4 t = __ldg(reinterpret_cast<const float4*>(in + (size_t)m * N + k));
      v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else {
#pragma unroll
      for (int q = 0; q < 4; ++q)
        v[q] = (m < N && k + q < kend) ? __ldg(in + (size_t)m * N + k + q) : 0.f;
    }
    bool bad = false;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (m < N && k + q < kend) bad |= !isfinite(v[q]);
    }
    if (bad) atomicOr(flag, 1);
    if (mode == 1) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        v[q] = 0.5f * (1.f + cosf(v[q]));
        if (mask_out && m < N && k + q < kend) mask_out[(size_t)m * N + k + q] = v[q];
      }
    }
  }
};

struct PartialStore {
  float* out;  // [gridDim.z][M][ld]
  int M, ld;
  __device__ __forceinline__ void store(int m, int n, float v) {
    out[((size_t)blockIdx.z * M + m) * ld + n] = v;
  }
  __device__ __forceinline__ void finish() {}
};

template <int TN>
static cudaError_t analysis_rows_t(cudaStream_t s, const ImageLoad& ld, const float* tw, int N,
                                   int ncols2, int ksplit, float* out) {
  constexpr int BMT = 32, BNT = 8, TM = 4, BK = 16;
  int kps, zs;
  row_split(N, ksplit, &kps, &zs);
  dim3 grid((N + BMT * TM - 1) / (BMT * TM), (ncols2 + BNT * TN - 1) / (BNT * TN), zs);
  PartialStore st{out, N, ncols2};
  gemm_nt_kernel<BMT, BNT, TM, TN, BK><<<grid, BMT * BNT, 0, s>>>(N, ncols2, N, kps, ld, tw,
                                                                 N, st);
  return cudaGetLastError();
}

// in: N x N image (mode 0) or theta (mode 1). tw: [2*ncols][N] real rows
// (Re, Im interleaved by row). out: [zs][N][2*ncols] partial sums, where
// row_split(N, ksplit) gives zs (the number of x chunks actually used).
cudaError_t launch_analysis_rows(cudaStream_t s, int mode, const float* in, float* mask_out,
                                 int* flag, const float* tw, int N, int ncols, int ksplit,
                                 float* out) {
  const int vec4 = (N % 4 == 0) && (reinterpret_cast<uintptr_t>(in) % 16 == 0);
  ImageLoad ld{in, mask_out, flag, N, mode, vec4};
  const int n2 = 2 * ncols;
  if (n2 <= 16) return analysis_rows_t<2>(s, ld, tw, N, n2, ksplit, out);
  if (n2 <= 32) return analysis_rows_t<4>(s, ld, tw, N, n2, ksplit, out);
  if (n2 <= 48) return analysis_rows_t<6>(s, ld, tw, N, n2, ksplit, out);
  if (n2 <= 64) return analysis_rows_t<8>(s, ld, tw, N, n2, ksplit, out);
  if (n2 <= 72) return analysis_rows_t<9>(s, ld, tw, N, n2, ksplit, out);
  if (n2 <= 80) return analysis_rows_t<10>(s, ld, tw, N, n2, ksplit, out);
  if (n2 <= 96) return analysis_rows_t<12>(s, ld, tw, N, n2, ksplit, out);
  return analysis_rows_t<16>(s, ld, tw, N, n2, ksplit, out);
}

// ---------------------------------------------------------------- column contraction
// out[ys][a][c] = scale * sum_{y in chunk ys} T(a, y) * sum_z R[z][y][c]
// sym == 0: a in [0, nrows), T(a, y) = TY[a][y].
// sym == 1: a in [0, 2*nr - 1), d = a - (nr - 1), T = d >= 0 ? TY[d][y] : conj(TY[-d][y]).
constexpr int AC_RB = 8;    // rows a per block
constexpr int AC_YT = 32;   // y tile staged in shared memory
__global__ void __launch_bounds__(128)
analysis_cols_kernel(const float2* __restrict__ R, int ksplit, int N, int ncols,
                     const float2* __restrict__ TY, int nrows_out, int nr, int sym, int ychunk,
                     float scale, float2* __restrict__ out) {
  __shared__ float2 tys[AC_RB][AC_YT];
  const int a0 = blockIdx.x * AC_RB;
  const int ys = blockIdx.y;
  const int y0 = ys * ychunk;
  const int y1 = min(N, y0 + ychunk);
  for (int c0 = 0; c0 < ncols; c0 += blockDim.x) {
    const int c = c0 + threadIdx.x;
    float2 acc[AC_RB];
#pragma unroll
    for (int r = 0; r < AC_RB; ++r) acc[r] = make_float2(0.f, 0.f);
    for (int yt = y0; yt < y1; yt += AC_YT) {
      __syncthreads();
      for (int e = threadIdx.x; e < AC_RB * AC_YT; e += blockDim.x) {
        const int r = e / AC_YT, yy = e % AC_YT;
        const int a = a0 + r, y = yt + yy;
        float2 t = make_float2(0.f, 0.f);
        if (a < nrows_out && y < y1) {
          if (!sym) {
            t = TY[(size_t)a * N + y];
          } else {
            const int d = a - (nr - 1);
            t = d >= 0 ? TY[(size_t)d * N + y] : conjf2(TY[(size_t)(-d) * N + y]);
          }
        }
        tys[r][yy] = t;
      }
      __syncthreads();
      if (c < ncols) {
        const int ye = min(AC_YT, y1 - yt);
        for (int yy = 0; yy < ye; ++yy) {
          const int y = yt + yy;
          float2 v = make_float2(0.f, 0.f);
          for (int z = 0; z < ksplit; ++z) {
            const float2 p = R[((size_t)z * N + y) * ncols + c];
            v.x += p.x; v.y += p.y;
          }
#pragma unroll
          for (int r = 0; r < AC_RB; ++r) cfma(acc[r], tys[r][yy], v);
        }
      }
    }
    if (c < ncols) {
#pragma unroll
      for (int r = 0; r < AC_RB; ++r) {
        const int a = a0 + r;
        if (a < nrows_out)
          out[((size_t)ys * nrows_out + a) * ncols + c] =
              make_float2(acc[r].x * scale, acc[r].y * scale);
      }
    }
  }
}

cudaError_t launch_analysis_cols(cudaStream_t s, const float* R, int ksplit, int N, int ncols,
                                 const float2* TY, int nrows_out, int nr, int sym, int ysplit,
                                 float scale, float2* out_partial) {
  const int ychunk = (N + ysplit - 1) / ysplit;
  dim3 grid((nrows_out + AC_RB - 1) / AC_RB, ysplit);
  const int threads = ncols <= 64 ? 64 : 128;
  analysis_cols_kernel<<<grid, threads, 0, s>>>(reinterpret_cast<const float2*>(R), ksplit, N,
                                                ncols, TY, nrows_out, nr, sym, ychunk, scale,
                                                out_partial);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- column expansion
// Ut[x][2a + {0,1}] = kappa(a) * sum_c coef[a][c] * phase(c, x), ld = kp (columns
// 2*nrows..kp-1 are zero-filled by the a == 0 blocks).
// mode 0 (band S): phase = conj(TX[c][x]) (TX = e^{-2 pi i s_c x/N}), kappa = 1.
// mode 1 (difference set D): c in [0, 2*nc-1), d = c - (nc-1),
//   phase = d >= 0 ? conj(TX[d][x]) : TX[-d][x], kappa(a) = a > 0 ? 2 : 1.
__global__ void __launch_bounds__(128)
expand_cols_kernel(const float2* __restrict__ coef, int ncoef, int coef_ld,
                   const float2* __restrict__ TX, int N, int nrows, int mode, int nc, int kp,
                   float* __restrict__ Ut) {
  extern __shared__ float2 crow[];
  const int a = blockIdx.y;
  for (int c = threadIdx.x; c < ncoef; c += blockDim.x) crow[c] = coef[(size_t)a * coef_ld + c];
  __syncthreads();
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= N) return;
  float2 acc = make_float2(0.f, 0.f);
  if (mode == 0) {
    for (int c = 0; c < ncoef; ++c) cfma(acc, crow[c], conjf2(TX[(size_t)c * N + x]));
  } else {
    for (int c = 0; c < ncoef; ++c) {
      const int d = c - (nc - 1);
      const float2 t = d >= 0 ? conjf2(TX[(size_t)d * N + x]) : TX[(size_t)(-d) * N + x];
      cfma(acc, crow[c], t);
    }
    if (a > 0) { acc.x *= 2.f; acc.y *= 2.f; }
  }
  Ut[(size_t)x * kp + 2 * a] = acc.x;
  Ut[(size_t)x * kp + 2 * a + 1] = acc.y;
  if (a == 0)
    for (int f = 2 * nrows; f < kp; ++f) Ut[(size_t)x * kp + f] = 0.f;
}

cudaError_t launch_expand_cols(cudaStream_t s, const float2* coef, int nrows, int ncoef,
                               int coef_ld, const float2* TX, int N, int mode, int nc, int kp,
                               float* Ut) {
  dim3 grid((N + 127) / 128, nrows);
  expand_cols_kernel<<<grid, 128, ncoef * sizeof(float2), s>>>(coef, ncoef, coef_ld, TX, N,
                                                               nrows, mode, nc, kp, Ut);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- row synthesis
// out[y][x] = sum_f AY[y][f] * Bt[x][f]; the functor is the fused epilogue.
struct AYLoad {
  const float* AY;
  int N, kp;
  __device__ __forceinline__ void load4(int m, int k, int kend, float* v) {
    if (m < N && k + 3 < kend) {
      float4 t = __ldg(reinterpret_cast<const float4*>(AY + (size_t)m * kp + k));
      v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else {
#pragma unroll
      for (int q = 0; q < 4; ++q) v[q] = (m < N && k + q < kend) ? AY[(size_t)m * kp + k + q] : 0.f;
    }
  }
};

constexpr int SY_BMT = 16, SY_BNT = 16, SY_TM = 8, SY_TN = 8, SY_BK = 16;
constexpr int SY_NT = SY_BMT * SY_BNT;

struct ResistEpi {
  ResistEpilogue p;
  int N;
  double pe, pen;
  __device__ __forceinline__ void store(int m, int n, float I) {
    const size_t i = (size_t)m * N + n;
    const float W = 1.f / (1.f + expf(-p.alpha * (I - p.thr)));
    if (p.aerial) p.aerial[i] = I;
    if (p.wafer) p.wafer[i] = W;
    if (p.mode == 1) {
      const float T = p.target[i];
      const float pw = p.pe_window ? p.pe_window[i] : 1.f;
      const float r = W - T;
      pe += (double)r * (double)r * (double)pw;
      float s = p.pe_weight * r * pw;
      if (p.penalty != 0.f && T < 0.5f) {
        const float qw = p.pen_window ? p.pen_window[i] : pw;
        const float ex = fmaxf(W - p.pen_thr, 0.f);
        pen += (double)ex * (double)ex * (double)qw;
        s += p.penalty * ex * qw;
      }
      p.dldi[i] = s * W * (1.f - W);
    }
  }
  __device__ __forceinline__ void finish() {
    if (p.mode != 1) return;
    __shared__ double sh[SY_NT / 32];
    const double a = block_sum<SY_NT>(pe, sh);
    const double b = block_sum<SY_NT>(pen, sh);
    if (threadIdx.x == 0) {
      const int bid = blockIdx.y * gridDim.x + blockIdx.x;
      p.loss_partial[2 * bid] = a;
      p.loss_partial[2 * bid + 1] = b;
    }
  }
};

struct GradEpi {
  GradEpilogue p;
  int N;
  double nrm;
  __device__ __forceinline__ void store(int m, int n, float G) {
    const size_t i = (size_t)m * N + n;
    if (p.grad_mask) p.grad_mask[i] = G;
    if (p.theta) {
      const float gt = -0.5f * G * sinf(p.theta[i]);
      p.grad_theta[i] = gt;
      nrm += (double)gt * (double)gt;
    }
  }
  __device__ __forceinline__ void finish() {
    if (!p.theta) return;
    __shared__ double sh[SY_NT / 32];
    const double a = block_sum<SY_NT>(nrm, sh);
    if (threadIdx.x == 0) p.norm_partial[blockIdx.y * gridDim.x + blockIdx.x] = a;
  }
};

static dim3 synth_grid(int N) {
  return dim3((N + SY_BMT * SY_TM - 1) / (SY_BMT * SY_TM),
              (N + SY_BNT * SY_TN - 1) / (SY_BNT * SY_TN), 1);
}

cudaError_t launch_synth_resist(cudaStream_t s, const float* AY, const float* Bt, int N, int kp,
                                const ResistEpilogue& ep, int* nblocks) {
  const dim3 grid = synth_grid(N);
  *nblocks = grid.x * grid.y;
  ResistEpi e{ep, N, 0.0, 0.0};
  AYLoad ld{AY, N, kp};
  gemm_nt_kernel<SY_BMT, SY_BNT, SY_TM, SY_TN, SY_BK>
      <<<grid, SY_NT, 0, s>>>(N, N, kp, kp, ld, Bt, kp, e);
  return cudaGetLastError();
}

cudaError_t launch_synth_grad(cudaStream_t s, const float* AY, const float* Bt, int N, int kp,
                              const GradEpilogue& ep, int* nblocks) {
  const dim3 grid = synth_grid(N);
  *nblocks = grid.x * grid.y;
  GradEpi e{ep, N, 0.0};
  AYLoad ld{AY, N, kp};
  gemm_nt_kernel<SY_BMT, SY_BNT, SY_TM, SY_TN, SY_BK>
      <<<grid, SY_NT, 0, s>>>(N, N, kp, kp, ld, Bt, kp, e);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- small-grid band stage
// Forward 1: T[k][r][jc] = sum_c H[k][r][c] m[r][c] ESc_t[c][jc],  m = sum_ys mpart[ys][r][c].
__global__ void band_fwd1_kernel(const float2* __restrict__ H, const float2* __restrict__ mpart,
                                 int ysplit, int Nr, int Nc, int Pc,
                                 const float2* __restrict__ ESc_t, float2* __restrict__ mband,
                                 float2* __restrict__ T) {
  extern __shared__ float2 ah[];
  const int r = blockIdx.x, k = blockIdx.y;
  for (int c = threadIdx.x; c < Nc; c += blockDim.x) {
    float2 m = make_float2(0.f, 0.f);
    for (int ys = 0; ys < ysplit; ++ys) {
      const float2 p = mpart[((size_t)ys * Nr + r) * Nc + c];
      m.x += p.x; m.y += p.y;
    }
    if (k == 0 && mband) mband[(size_t)r * Nc + c] = m;
    ah[c] = cmul(H[((size_t)k * Nr + r) * Nc + c], m);
  }
  __syncthreads();
  for (int jc = threadIdx.x; jc < Pc; jc += blockDim.x) {
    float2 acc = make_float2(0.f, 0.f);
    for (int c = 0; c < Nc; ++c) cfma(acc, ah[c], ESc_t[(size_t)c * Pc + jc]);
    T[((size_t)k * Nr + r) * Pc + jc] = acc;
  }
}

// Forward 2: e[k][jr][jc] = sum_r ESr_t[r][jr] T[k][r][jc]; ik[k][jr][jc] = w_k |e|^2.
__global__ void band_fwd2_kernel(const float2* __restrict__ T, const float2* __restrict__ ESr_t,
                                 const float* __restrict__ w, int Nr, int Pr, int Pc,
                                 float2* __restrict__ e, float* __restrict__ ik) {
  extern __shared__ float2 er[];
  const int jr = blockIdx.x, k = blockIdx.y;
  for (int r = threadIdx.x; r < Nr; r += blockDim.x) er[r] = ESr_t[(size_t)r * Pr + jr];
  __syncthreads();
  const float wk = w[k];
  for (int jc = threadIdx.x; jc < Pc; jc += blockDim.x) {
    float2 acc = make_float2(0.f, 0.f);
    for (int r = 0; r < Nr; ++r) cfma(acc, er[r], T[((size_t)k * Nr + r) * Pc + jc]);
    const size_t o = ((size_t)k * Pr + jr) * Pc + jc;
    e[o] = acc;
    ik[o] = wk * (acc.x * acc.x + acc.y * acc.y);
  }
}

// Forward 3: Q[jr][dc] = sum_jc i[jr][jc] conj(EDc_t[dc][jc]),  i = sum_k ik[k] (k order).
__global__ void band_fwd3_kernel(const float* __restrict__ ik, int K, int Pr, int Pc, int nd,
                                 const float2* __restrict__ EDc_t, float2* __restrict__ Q) {
  extern __shared__ float irow[];
  const int jr = blockIdx.x;
  for (int jc = threadIdx.x; jc < Pc; jc += blockDim.x) {
    float s = 0.f;
    for (int k = 0; k < K; ++k) s += ik[((size_t)k * Pr + jr) * Pc + jc];
    irow[jc] = s;
  }
  __syncthreads();
  for (int dc = threadIdx.x; dc < nd; dc += blockDim.x) {
    float2 acc = make_float2(0.f, 0.f);
    for (int jc = 0; jc < Pc; ++jc) {
      const float2 t = EDc_t[(size_t)dc * Pc + jc];
      acc.x = fmaf(irow[jc], t.x, acc.x);
      acc.y = fmaf(-irow[jc], t.y, acc.y);
    }
    Q[(size_t)jr * nd + dc] = acc;
  }
}

// Forward 4: chat[dr][dc] = sum_jr conj(EDr_t[dr + Nr - 1][jr]) Q[jr][dc] / (Pr Pc), dr >= 0.
__global__ void band_fwd4_kernel(const float2* __restrict__ Q, int Nr, int Pr, int nd,
                                 const float2* __restrict__ EDr_t, float inv,
                                 float2* __restrict__ chat) {
  const int dr = blockIdx.x;
  const float2* ed = EDr_t + (size_t)(dr + Nr - 1) * Pr;
  for (int dc = threadIdx.x; dc < nd; dc += blockDim.x) {
    float2 acc = make_float2(0.f, 0.f);
    for (int jr = 0; jr < Pr; ++jr) cfma(acc, conjf2(ed[jr]), Q[(size_t)jr * nd + dc]);
    chat[(size_t)dr * nd + dc] = make_float2(acc.x * inv, acc.y * inv);
  }
}

static int pick_threads(int n) {
  int t = 32;
  while (t < n && t < 256) t <<= 1;
  return t;
}

cudaError_t launch_band_forward(cudaStream_t s, const Cache& c, const float2* mpart,
                                int ysplit, Field& f, float* ik, float2* T, float2* Q,
                                float2* chat, float* Ut) {
  const BandGeom& g = c.g;
  band_fwd1_kernel<<<dim3(g.Nr, g.K), pick_threads(g.Pc), g.Nc * sizeof(float2), s>>>(
      c.H, mpart, ysplit, g.Nr, g.Nc, g.Pc, c.ESc_t, f.mband, T);
  band_fwd2_kernel<<<dim3(g.Pr, g.K), pick_threads(g.Pc), g.Nr * sizeof(float2), s>>>(
      T, c.ESr_t, c.w, g.Nr, g.Pr, g.Pc, f.e, ik);
  const int nd = 2 * g.Nc - 1;
  band_fwd3_kernel<<<g.Pr, pick_threads(nd), g.Pc * sizeof(float), s>>>(ik, g.K, g.Pr, g.Pc,
                                                                         nd, c.EDc_t, Q);
  band_fwd4_kernel<<<g.Nr, pick_threads(nd), 0, s>>>(Q, g.Nr, g.Pr, nd, c.EDr_t,
                                                     1.f / ((float)g.Pr * (float)g.Pc), chat);
  // U[dr][x] (dr = 0..Nr-1, Hermitian half with kappa) for the row synthesis.
  return launch_expand_cols(s, chat, g.Nr, nd, nd, c.TXDc, g.N, 1, g.Nc, g.kp_rows, Ut);
}

// Adjoint 1: Gam[a][jc] = sum_{c < Nc} kappa(c) g'[a][c] EDc_t[c + Nc - 1][jc],
//            g' = sum_ys gpart[ys][a][c], a = dr + Nr - 1 in [0, 2Nr - 1).
__global__ void band_adj1_kernel(const float2* __restrict__ gpart, int ysplit, int na, int Nc,
                                 int Pc, const float2* __restrict__ EDc_t,
                                 float2* __restrict__ Gam) {
  extern __shared__ float2 grow[];
  const int a = blockIdx.x;
  for (int c = threadIdx.x; c < Nc; c += blockDim.x) {
    float2 v = make_float2(0.f, 0.f);
    for (int ys = 0; ys < ysplit; ++ys) {
      const float2 p = gpart[((size_t)ys * na + a) * Nc + c];
      v.x += p.x; v.y += p.y;
    }
    const float kc = c > 0 ? 2.f : 1.f;
    grow[c] = make_float2(v.x * kc, v.y * kc);
  }
  __syncthreads();
  for (int jc = threadIdx.x; jc < Pc; jc += blockDim.x) {
    float2 acc = make_float2(0.f, 0.f);
    for (int c = 0; c < Nc; ++c) cfma(acc, grow[c], EDc_t[(size_t)(c + Nc - 1) * Pc + jc]);
    Gam[(size_t)a * Pc + jc] = acc;
  }
}

// Adjoint 2: gam[jr][jc] = Re sum_a EDr_t[a][jr] Gam[a][jc]   (gamma is real).
__global__ void band_adj2_kernel(const float2* __restrict__ Gam, int na, int Pr, int Pc,
                                 const float2* __restrict__ EDr_t, float* __restrict__ gam) {
  extern __shared__ float2 ed[];
  const int jr = blockIdx.x;
  for (int a = threadIdx.x; a < na; a += blockDim.x) ed[a] = EDr_t[(size_t)a * Pr + jr];
  __syncthreads();
  for (int jc = threadIdx.x; jc < Pc; jc += blockDim.x) {
    float acc = 0.f;
    for (int a = 0; a < na; ++a) {
      const float2 t = Gam[(size_t)a * Pc + jc];
      acc = fmaf(ed[a].x, t.x, fmaf(-ed[a].y, t.y, acc));
    }
    gam[(size_t)jr * Pc + jc] = acc;
  }
}

// Adjoint 3: Z1[k][jr][uc] = sum_jc e[k][jr][jc] gam[jr][jc] conj(ESc[jc][uc]).
__global__ void band_adj3_kernel(const float2* __restrict__ e, const float* __restrict__ gam,
                                 int Pr, int Pc, int Nc, const float2* __restrict__ ESc,
                                 float2* __restrict__ Z1) {
  extern __shared__ float2 q[];
  const int jr = blockIdx.x, k = blockIdx.y;
  for (int jc = threadIdx.x; jc < Pc; jc += blockDim.x) {
    const float2 v = e[((size_t)k * Pr + jr) * Pc + jc];
    const float gv = gam[(size_t)jr * Pc + jc];
    q[jc] = make_float2(v.x * gv, v.y * gv);
  }
  __syncthreads();
  for (int uc = threadIdx.x; uc < Nc; uc += blockDim.x) {
    float2 acc = make_float2(0.f, 0.f);
    for (int jc = 0; jc < Pc; ++jc) cfma(acc, q[jc], conjf2(ESc[(size_t)jc * Nc + uc]));
    Z1[((size_t)k * Pr + jr) * Nc + uc] = acc;
  }
}

// Adjoint 4: Zk[k][ur][uc] = sum_jr conj(ESr_t[ur][jr]) Z1[k][jr][uc] / (Pr Pc).
__global__ void band_adj4_kernel(const float2* __restrict__ Z1, int Pr, int Nc,
                                 const float2* __restrict__ ESr_t, float inv,
                                 float2* __restrict__ Zk, int Nr) {
  const int ur = blockIdx.x, k = blockIdx.y;
  const float2* es = ESr_t + (size_t)ur * Pr;
  for (int uc = threadIdx.x; uc < Nc; uc += blockDim.x) {
    float2 acc = make_float2(0.f, 0.f);
    for (int jr = 0; jr < Pr; ++jr) cfma(acc, conjf2(es[jr]), Z1[((size_t)k * Pr + jr) * Nc + uc]);
    Zk[((size_t)k * Nr + ur) * Nc + uc] = make_float2(acc.x * inv, acc.y * inv);
  }
}

// Adjoint 5: X[u] = scale * sum_k w_k conj(H[k][u]) Zk[k][u]  (k order).
__global__ void band_adj5_kernel(const float2* __restrict__ Zk, const float2* __restrict__ H,
                                 const float* __restrict__ w, int K, int nb, float scale,
                                 float2* __restrict__ X) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nb) return;
  float2 acc = make_float2(0.f, 0.f);
  for (int k = 0; k < K; ++k) {
    const float2 t = cmul(conjf2(H[(size_t)k * nb + u]), Zk[(size_t)k * nb + u]);
    acc.x = fmaf(w[k], t.x, acc.x);
    acc.y = fmaf(w[k], t.y, acc.y);
  }
  X[u] = make_float2(acc.x * scale, acc.y * scale);
}

cudaError_t launch_band_adjoint(cudaStream_t s, const Cache& c, const Field& f,
                                const float2* gpart, int ysplit, double scale, float2* Gam,
                                float* gam, float2* Z1, float2* Zk, float2* X, float* Vt) {
  const BandGeom& g = c.g;
  const int na = 2 * g.Nr - 1;
  band_adj1_kernel<<<na, pick_threads(g.Pc), g.Nc * sizeof(float2), s>>>(gpart, ysplit, na, g.Nc,
                                                                         g.Pc, c.EDc_t, Gam);
  band_adj2_kernel<<<g.Pr, pick_threads(g.Pc), na * sizeof(float2), s>>>(Gam, na, g.Pr, g.Pc,
                                                                         c.EDr_t, gam);
  band_adj3_kernel<<<dim3(g.Pr, g.K), pick_threads(g.Nc), g.Pc * sizeof(float2), s>>>(
      f.e, gam, g.Pr, g.Pc, g.Nc, c.ESc, Z1);
  band_adj4_kernel<<<dim3(g.Nr, g.K), pick_threads(g.Nc), 0, s>>>(
      Z1, g.Pr, g.Nc, c.ESr_t, 1.f / ((float)g.Pr * (float)g.Pc), Zk, g.Nr);
  const int nb = g.Nr * g.Nc;
  band_adj5_kernel<<<(nb + 127) / 128, 128, 0, s>>>(Zk, c.H, c.w, g.K, nb, (float)scale, X);
  return launch_expand_cols(s, X, g.Nr, g.Nc, g.Nc, c.TXSc, g.N, 0, g.Nc, g.kp_rows, Vt);
}

// ---------------------------------------------------------------- FP64 partial sums
__global__ void sum_partials_kernel(const double* __restrict__ part, int n, int stride,
                                    double* __restrict__ out) {
  // One thread per component, fixed order (deterministic).
  const int comp = threadIdx.x;
  if (comp >= stride) return;
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += part[(size_t)i * stride + comp];
  out[comp] = s;
}

cudaError_t launch_sum_partials(cudaStream_t s, const double* part, int n, int stride,
                                double* out) {
  sum_partials_kernel<<<1, 32, 0, s>>>(part, n, stride, out);
  return cudaGetLastError();
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
