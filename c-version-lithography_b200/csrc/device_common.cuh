// Device helpers shared by the band-DFT kernels: complex arithmetic, FP64
// block reductions, vector load/store helpers and the fused epilogues of the
// row syntheses (resist + PE + dL/dI, and the theta chain + gradient norm).
#pragma once
#include <cuda_runtime.h>

#include "litho_internal.cuh"

namespace litho_b200 {

// Programmatic dependent launch. Every kernel of an imaging / adjoint chain calls
// pdl_trigger() first, so that its stream successor may be scheduled while it runs,
// and pdl_wait() before its first access to global data that an earlier kernel of
// the stream writes or reads (only the optical cache's constant tables may be
// touched before it), and before its first global write. pdl_wait returns once the
// predecessor grid has completed and its memory is visible; both are no-ops for a
// kernel launched without the programmatic-serialization attribute.
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

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

// sin / cos for the split-BF16 tensor-core path: Cody-Waite reduction of x by
// 2 pi with a two-term constant (6.28125, exact in 9 bits so that k * 6.28125 is
// exact for |k| < 2^15, plus the remainder 2 pi - 6.28125), then the SFU sine
// or cosine on [-pi, pi]. Absolute error below about 1e-6 for |x| < 1e3: far
// inside the 1e-3 budget of that path, and a few instructions instead of the
// full-range library routine, which keeps the unrolled epilogues compact.
__device__ __forceinline__ float reduce_2pi(float x) {
  const float k = rintf(x * 0.15915494309189535f);
  return fmaf(-k, 1.9353071795864769e-3f, fmaf(-k, 6.28125f, x));
}
__device__ __forceinline__ float fast_cos(float x) { return __cosf(reduce_2pi(x)); }
__device__ __forceinline__ float fast_sin(float x) { return __sinf(reduce_2pi(x)); }

// Resist + PE + dL/dI (imaging.cpp:165-168, loss.cpp:16-64, gradient.cpp:121-196).
// FAST (tensor-core path) uses the SFU exponential and reciprocal and rounds each
// pixel's loss term to FP32 before the FP64 accumulation.
template <bool FAST>
struct ResistEpiT {
  ResistEpilogue p;
  int N, vec;
  double pe, pen;
  // Pixel (m, n) of image blockIdx.z: the images of a batched launch lie N * N apart.
  __device__ __forceinline__ size_t pix(int m, int n) const {
    return ((size_t)blockIdx.z * N + m) * N + n;
  }
  __device__ __forceinline__ float sigmoid(float I) const {
    const float z = -p.alpha * (I - p.thr);
    return FAST ? __fdividef(1.f, 1.f + __expf(z)) : 1.f / (1.f + expf(z));
  }
  __device__ __forceinline__ void one(float I, float T, float pw, float qw, float& W, float& g) {
    W = sigmoid(I);
    const float r = W - T;
    pe += FAST ? (double)(r * r * pw) : (double)r * (double)r * (double)pw;
    float s = p.pe_weight * r * pw;
    if ((p.penalty != 0.f || p.loss_penalty_term) && T < 0.5f) {
      const float ex = fmaxf(W - p.pen_thr, 0.f);
      pen += FAST ? (double)(ex * ex * qw) : (double)ex * (double)ex * (double)qw;
      s += p.penalty * ex * qw;
    }
    g = s * W * (1.f - W);
  }
  __device__ __forceinline__ void store4(int m, int n, float4 I, int nvalid) {
    store4p(m, n, I, pre4(m, n, nvalid), nvalid);
  }
  // The per-pixel input (target) fetched before the accumulator is ready, and the
  // store that consumes it.
  __device__ __forceinline__ float4 pre4(int m, int n, int nvalid) const {
    if (p.mode == 0 || nvalid <= 0) return make_float4(0.f, 0.f, 0.f, 0.f);
    return ld4(p.target, pix(m, n), vec, nvalid);
  }
  __device__ __forceinline__ void store4p(int m, int n, float4 I, float4 T, int nvalid) {
    const size_t i = pix(m, n);
    if (p.mode == 0) {
      if (p.aerial) st4(p.aerial, i, I, vec, nvalid);
      if (p.wafer) {
        const float4 W = make_float4(sigmoid(I.x), sigmoid(I.y), sigmoid(I.z), sigmoid(I.w));
        st4(p.wafer, i, W, vec, nvalid);
      }
      return;
    }
    st4(p.dldi, i, dldi4(m, n, I, T, nvalid), vec, nvalid);
  }
  // Mode 1 without the dL/dI store: aerial / wafer stores and loss terms as in
  // store4p, dL/dI returned (0 in lanes past nvalid).
  __device__ __forceinline__ float4 dldi4(int m, int n, float4 I, float4 T, int nvalid) {
    const size_t i = pix(m, n);
    if (p.aerial) st4(p.aerial, i, I, vec, nvalid);
    const float4 one4 = make_float4(1.f, 1.f, 1.f, 1.f);
    const float4 pw = p.pe_window ? ld4(p.pe_window, i, vec, nvalid) : one4;
    const float4 qw = p.pen_window ? ld4(p.pen_window, i, vec, nvalid) : pw;
    float4 W = make_float4(0.f, 0.f, 0.f, 0.f), g = W;
    if (nvalid > 0) one(I.x, T.x, pw.x, qw.x, W.x, g.x);
    if (nvalid > 1) one(I.y, T.y, pw.y, qw.y, W.y, g.y);
    if (nvalid > 2) one(I.z, T.z, pw.z, qw.z, W.z, g.z);
    if (nvalid > 3) one(I.w, T.w, pw.w, qw.w, W.w, g.w);
    if (p.wafer) st4(p.wafer, i, W, vec, nvalid);
    return g;
  }
  // dldi4 for four in-range pixels when there is no window and no penalty (the CTM
  // evaluation): the same arithmetic with pw = qw = 1, which x * 1.f leaves exact.
  __device__ __forceinline__ float4 plain4(int m, int n, float4 I, float4 T) {
    const size_t i = pix(m, n);
    if (p.aerial) st4(p.aerial, i, I, vec, 4);
    float4 W, g;
    auto one_plain = [&](float x, float t, float& w, float& d) {
      w = sigmoid(x);
      const float r = w - t;
      pe += FAST ? (double)(r * r) : (double)r * (double)r;
      d = p.pe_weight * r * w * (1.f - w);
    };
    one_plain(I.x, T.x, W.x, g.x);
    one_plain(I.y, T.y, W.y, g.y);
    one_plain(I.z, T.z, W.z, g.z);
    one_plain(I.w, T.w, W.w, g.w);
    if (p.wafer) st4(p.wafer, i, W, vec, 4);
    return g;
  }
  __host__ __device__ bool plain() const {
    return p.pe_window == nullptr && p.pen_window == nullptr && p.penalty == 0.f &&
           !p.loss_penalty_term;
  }
  // All EPI_NT threads of the CTA must call finish.
  __device__ __forceinline__ void finish() {
    if (p.mode != 1) return;
    __shared__ double sh[EPI_NT / 32];
    const double a = block_sum<EPI_NT>(pe, sh);
    const double b = block_sum<EPI_NT>(pen, sh);
    if (threadIdx.x == 0) {
      const size_t bid = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
      p.loss_partial[2 * bid] = a;
      p.loss_partial[2 * bid + 1] = b;
    }
  }
};

// dPE/dM, the theta chain -1/2 G sin(theta) and its FP64 squared norm
// (CTM_Optimizer.cpp:151-152). FAST selects fast_sin and per-chunk FP32 norms
// (tensor-core path).
template <bool FAST>
struct GradEpiT {
  GradEpilogue p;
  int N, vec;
  double nrm;
  __device__ __forceinline__ size_t pix(int m, int n) const {
    return ((size_t)blockIdx.z * N + m) * N + n;
  }
  __device__ __forceinline__ float sn(float t) const { return FAST ? fast_sin(t) : sinf(t); }
  __device__ __forceinline__ void store4(int m, int n, float4 G, int nvalid) {
    store4p(m, n, G, pre4(m, n, nvalid), nvalid);
  }
  __device__ __forceinline__ float4 pre4(int m, int n, int nvalid) const {
    if (!p.theta || nvalid <= 0) return make_float4(0.f, 0.f, 0.f, 0.f);
    return ld4(p.theta, pix(m, n), vec, nvalid);
  }
  __device__ __forceinline__ void store4p(int m, int n, float4 G, float4 th, int nvalid) {
    const size_t i = pix(m, n);
    if (p.grad_mask) st4(p.grad_mask, i, G, vec, nvalid);
    if (!p.theta) return;
    float4 gt;
    gt.x = -0.5f * G.x * sn(th.x);
    gt.y = -0.5f * G.y * sn(th.y);
    gt.z = -0.5f * G.z * sn(th.z);
    gt.w = -0.5f * G.w * sn(th.w);
    if (FAST) {
      // lanes past the edge hold theta = 0 and G = 0, so they add nothing
      nrm += (double)(gt.x * gt.x + gt.y * gt.y + gt.z * gt.z + gt.w * gt.w);
    } else {
      if (nvalid > 0) nrm += (double)gt.x * gt.x;
      if (nvalid > 1) nrm += (double)gt.y * gt.y;
      if (nvalid > 2) nrm += (double)gt.z * gt.z;
      if (nvalid > 3) nrm += (double)gt.w * gt.w;
    }
    st4(p.grad_theta, i, gt, vec, nvalid);
  }
  __device__ __forceinline__ void finish() {
    if (!p.theta) return;
    __shared__ double sh[EPI_NT / 32];
    const double a = block_sum<EPI_NT>(nrm, sh);
    if (threadIdx.x == 0)   // [image][tile] over a batched launch
      p.norm_partial[((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = a;
  }
};

using ResistEpi = ResistEpiT<false>;
using GradEpi = GradEpiT<false>;

inline int aligned16(const void* p) {
  return p == nullptr || reinterpret_cast<uintptr_t>(p) % 16 == 0;
}

}  // namespace litho_b200
