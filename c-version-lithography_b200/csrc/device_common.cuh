// Device helpers shared by the band-DFT kernels: complex arithmetic, FP64
// block reductions, vector load/store helpers and the fused epilogues of the
// row syntheses (resist + PE + dL/dI, and the theta chain + gradient norm).
#pragma once
#include <cuda_runtime.h>

#include "litho_internal.cuh"

namespace litho_b200 {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ void cfma(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, fmaf(-a.y, b.y, acc.x));
  acc.y = fmaf(a.x, b.y, fmaf(a.y, b.x, acc.y));
}

// FP64 sum over a CTA of NT threads, fixed order (deterministic); result in thread 0.
template <int NT>
__device__ double block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    for (int w = 0; w < NT / 32; ++w) r += sh[w];
  }
  __syncthreads();
  return r;
}

template <class T>
__device__ __forceinline__ float4 ld4(const T* p, size_t i, int vec, int nvalid) {
  if (vec && nvalid == 4) return __ldg(reinterpret_cast<const float4*>(p + i));
  float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
  if (nvalid > 0) r.x = p[i];
  if (nvalid > 1) r.y = p[i + 1];
  if (nvalid > 2) r.z = p[i + 2];
  if (nvalid > 3) r.w = p[i + 3];
  return r;
}
__device__ __forceinline__ void st4(float* p, size_t i, float4 v, int vec, int nvalid) {
  if (vec && nvalid == 4) {
    *reinterpret_cast<float4*>(p + i) = v;
    return;
  }
  if (nvalid > 0) p[i] = v.x;
  if (nvalid > 1) p[i + 1] = v.y;
  if (nvalid > 2) p[i + 2] = v.z;
  if (nvalid > 3) p[i + 3] = v.w;
}

constexpr int EPI_NT = 256;  // threads of every CTA that runs a synthesis epilogue

// Resist + PE + dL/dI (imaging.cpp:165-168, loss.cpp:16-64, gradient.cpp:121-196).
struct ResistEpi {
  ResistEpilogue p;
  int N, vec;
  double pe, pen;
  __device__ __forceinline__ float sigmoid(float I) const {
    return 1.f / (1.f + expf(-p.alpha * (I - p.thr)));
  }
  __device__ __forceinline__ void one(float I, float T, float pw, float qw, float& W, float& g) {
    W = sigmoid(I);
    const float r = W - T;
    pe += (double)r * (double)r * (double)pw;
    float s = p.pe_weight * r * pw;
    if (p.penalty != 0.f && T < 0.5f) {
      const float ex = fmaxf(W - p.pen_thr, 0.f);
      pen += (double)ex * (double)ex * (double)qw;
      s += p.penalty * ex * qw;
    }
    g = s * W * (1.f - W);
  }
  __device__ __forceinline__ void store1(int m, int n, float I) {
    const size_t i = (size_t)m * N + n;
    if (p.aerial) p.aerial[i] = I;
    if (p.mode == 0) {
      if (p.wafer) p.wafer[i] = sigmoid(I);
      return;
    }
    const float T = __ldg(p.target + i);
    const float pw = p.pe_window ? __ldg(p.pe_window + i) : 1.f;
    const float qw = p.pen_window ? __ldg(p.pen_window + i) : pw;
    float W, g;
    one(I, T, pw, qw, W, g);
    if (p.wafer) p.wafer[i] = W;
    p.dldi[i] = g;
  }
  __device__ __forceinline__ void store4(int m, int n, float4 I, int nvalid) {
    const size_t i = (size_t)m * N + n;
    if (p.aerial) st4(p.aerial, i, I, vec, nvalid);
    if (p.mode == 0) {
      if (p.wafer) {
        const float4 W = make_float4(sigmoid(I.x), sigmoid(I.y), sigmoid(I.z), sigmoid(I.w));
        st4(p.wafer, i, W, vec, nvalid);
      }
      return;
    }
    const float4 T = ld4(p.target, i, vec, nvalid);
    const float4 one4 = make_float4(1.f, 1.f, 1.f, 1.f);
    const float4 pw = p.pe_window ? ld4(p.pe_window, i, vec, nvalid) : one4;
    const float4 qw = p.pen_window ? ld4(p.pen_window, i, vec, nvalid) : pw;
    float4 W = make_float4(0.f, 0.f, 0.f, 0.f), g = W;
    if (nvalid > 0) one(I.x, T.x, pw.x, qw.x, W.x, g.x);
    if (nvalid > 1) one(I.y, T.y, pw.y, qw.y, W.y, g.y);
    if (nvalid > 2) one(I.z, T.z, pw.z, qw.z, W.z, g.z);
    if (nvalid > 3) one(I.w, T.w, pw.w, qw.w, W.w, g.w);
    if (p.wafer) st4(p.wafer, i, W, vec, nvalid);
    st4(p.dldi, i, g, vec, nvalid);
  }
  // V float4 chunks at once: every input load is issued before any store, so
  // the loads of the batch overlap instead of waiting on one another.
  template <int V>
  __device__ __forceinline__ void store4v(const int (&m)[V], const int (&n)[V],
                                          const float4 (&I)[V], const int (&nv)[V]) {
    if (p.mode == 0) {
#pragma unroll
      for (int q = 0; q < V; ++q)
        if (nv[q] > 0) store4(m[q], n[q], I[q], nv[q]);
      return;
    }
    float4 T[V], pw[V], qw[V];
    const float4 one4 = make_float4(1.f, 1.f, 1.f, 1.f);
#pragma unroll
    for (int q = 0; q < V; ++q) {
      const size_t i = (size_t)m[q] * N + n[q];
      T[q] = nv[q] > 0 ? ld4(p.target, i, vec, nv[q]) : one4;
      pw[q] = (p.pe_window && nv[q] > 0) ? ld4(p.pe_window, i, vec, nv[q]) : one4;
      qw[q] = (p.pen_window && nv[q] > 0) ? ld4(p.pen_window, i, vec, nv[q]) : pw[q];
    }
#pragma unroll
    for (int q = 0; q < V; ++q) {
      if (nv[q] <= 0) continue;
      const size_t i = (size_t)m[q] * N + n[q];
      float4 W = make_float4(0.f, 0.f, 0.f, 0.f), g = W;
      if (nv[q] > 0) one(I[q].x, T[q].x, pw[q].x, qw[q].x, W.x, g.x);
      if (nv[q] > 1) one(I[q].y, T[q].y, pw[q].y, qw[q].y, W.y, g.y);
      if (nv[q] > 2) one(I[q].z, T[q].z, pw[q].z, qw[q].z, W.z, g.z);
      if (nv[q] > 3) one(I[q].w, T[q].w, pw[q].w, qw[q].w, W.w, g.w);
      if (p.aerial) st4(p.aerial, i, I[q], vec, nv[q]);
      if (p.wafer) st4(p.wafer, i, W, vec, nv[q]);
      st4(p.dldi, i, g, vec, nv[q]);
    }
  }
  // All EPI_NT threads of the CTA must call finish.
  __device__ __forceinline__ void finish() {
    if (p.mode != 1) return;
    __shared__ double sh[EPI_NT / 32];
    const double a = block_sum<EPI_NT>(pe, sh);
    const double b = block_sum<EPI_NT>(pen, sh);
    if (threadIdx.x == 0) {
      const int bid = blockIdx.y * gridDim.x + blockIdx.x;
      p.loss_partial[2 * bid] = a;
      p.loss_partial[2 * bid + 1] = b;
    }
  }
};

// dPE/dM, the theta chain -1/2 G sin(theta) and its FP64 squared norm
// (CTM_Optimizer.cpp:151-152).
struct GradEpi {
  GradEpilogue p;
  int N, vec;
  double nrm;
  __device__ __forceinline__ void store1(int m, int n, float G) {
    const size_t i = (size_t)m * N + n;
    if (p.grad_mask) p.grad_mask[i] = G;
    if (!p.theta) return;
    const float gt = -0.5f * G * sinf(__ldg(p.theta + i));
    nrm += (double)gt * gt;
    p.grad_theta[i] = gt;
  }
  __device__ __forceinline__ void store4(int m, int n, float4 G, int nvalid) {
    const size_t i = (size_t)m * N + n;
    if (p.grad_mask) st4(p.grad_mask, i, G, vec, nvalid);
    if (!p.theta) return;
    const float4 th = ld4(p.theta, i, vec, nvalid);
    float4 gt;
    gt.x = -0.5f * G.x * sinf(th.x);
    gt.y = -0.5f * G.y * sinf(th.y);
    gt.z = -0.5f * G.z * sinf(th.z);
    gt.w = -0.5f * G.w * sinf(th.w);
    if (nvalid > 0) nrm += (double)gt.x * gt.x;
    if (nvalid > 1) nrm += (double)gt.y * gt.y;
    if (nvalid > 2) nrm += (double)gt.z * gt.z;
    if (nvalid > 3) nrm += (double)gt.w * gt.w;
    st4(p.grad_theta, i, gt, vec, nvalid);
  }
  template <int V>
  __device__ __forceinline__ void store4v(const int (&m)[V], const int (&n)[V],
                                          const float4 (&G)[V], const int (&nv)[V]) {
    float4 th[V];
#pragma unroll
    for (int q = 0; q < V; ++q)
      th[q] = (p.theta && nv[q] > 0) ? ld4(p.theta, (size_t)m[q] * N + n[q], vec, nv[q])
                                     : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int q = 0; q < V; ++q) {
      if (nv[q] <= 0) continue;
      const size_t i = (size_t)m[q] * N + n[q];
      if (p.grad_mask) st4(p.grad_mask, i, G[q], vec, nv[q]);
      if (!p.theta) continue;
      float4 gt;
      gt.x = -0.5f * G[q].x * sinf(th[q].x);
      gt.y = -0.5f * G[q].y * sinf(th[q].y);
      gt.z = -0.5f * G[q].z * sinf(th[q].z);
      gt.w = -0.5f * G[q].w * sinf(th[q].w);
      if (nv[q] > 0) nrm += (double)gt.x * gt.x;
      if (nv[q] > 1) nrm += (double)gt.y * gt.y;
      if (nv[q] > 2) nrm += (double)gt.z * gt.z;
      if (nv[q] > 3) nrm += (double)gt.w * gt.w;
      st4(p.grad_theta, i, gt, vec, nv[q]);
    }
  }
  __device__ __forceinline__ void finish() {
    if (!p.theta) return;
    __shared__ double sh[EPI_NT / 32];
    const double a = block_sum<EPI_NT>(nrm, sh);
    if (threadIdx.x == 0) p.norm_partial[blockIdx.y * gridDim.x + blockIdx.x] = a;
  }
};

inline int aligned16(const void* p) {
  return p == nullptr || reinterpret_cast<uintptr_t>(p) % 16 == 0;
}

}  // namespace litho_b200
