// A C++ consumer of the C ABI (include/litho_b200.h), built by g++ against the header
// and linked to liblitho_b200.so, the way a maintainer's shim in the reference code
// base would use it: the reference's class names (Imaging, Gradient, CTM objective,
// one LSM step) over plain row-major host matrices, with device buffers from the CUDA
// runtime. It writes every result to a binary file for the test that compares them
// with the package's own calls (the kernels it generated included, so that both sides
// image with the same cache).
//
//   consumer <out.bin>
//
// Exit status: 0 done, 3 no usable GPU (litho_ctx_create failed), 1 an ABI call failed.
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "litho_b200.h"

namespace shim {

using Mat = std::vector<float>;   // N x N, row-major

struct Error : std::runtime_error {
  int status;
  Error(int st, const std::string& m) : std::runtime_error(m), status(st) {}
};

inline void check(int st, litho_ctx* ctx, const char* what) {
  if (st != LITHO_OK)
    throw Error(st, std::string(what) + ": " + litho_status_string(st) + " (" +
                        (ctx ? litho_ctx_last_error(ctx) : "") + ")");
}

struct DeviceBuffer {
  float* p = nullptr;
  explicit DeviceBuffer(size_t n) {
    if (cudaMalloc(&p, n * sizeof(float)) != cudaSuccess) throw Error(LITHO_ERR_OOM, "cudaMalloc");
  }
  ~DeviceBuffer() { cudaFree(p); }
  void up(const Mat& m) { cudaMemcpy(p, m.data(), m.size() * sizeof(float), cudaMemcpyHostToDevice); }
  Mat down(size_t n) const {
    Mat m(n);
    cudaMemcpy(m.data(), p, n * sizeof(float), cudaMemcpyDeviceToHost);
    return m;
  }
};

// ImagingCache (litho_prepare.h:18-47) on the device: K dense N x N kernels, DC at (0, 0).
class Cache {
 public:
  Cache(litho_ctx* ctx, int N, const std::vector<std::complex<double>>& kernels,
        const std::vector<double>& eigenvalues, double ws_sum)
      : ctx_(ctx), N_(N) {
    const int K = (int)eigenvalues.size();
    std::vector<double> flat(2 * kernels.size());
    for (size_t i = 0; i < kernels.size(); ++i) {
      flat[2 * i] = kernels[i].real();
      flat[2 * i + 1] = kernels[i].imag();
    }
    check(litho_cache_create_dense(ctx, N, K, flat.data(), eigenvalues.data(), ws_sum, &c_), ctx,
          "litho_cache_create_dense");
  }
  ~Cache() { litho_cache_destroy(c_); }
  litho_cache* get() const { return c_; }
  int N() const { return N_; }

 private:
  litho_ctx* ctx_;
  int N_;
  litho_cache* c_ = nullptr;
};

// Imaging (include/litho_model/imaging.h:16-53): compute() keeps the field for Gradient.
class Imaging {
 public:
  Imaging(litho_ctx* ctx, const Cache& cache)
      : ctx_(ctx), cache_(cache), buf_(3 * (size_t)cache.N() * cache.N()) {
    check(litho_field_create(ctx, cache.get(), &field_), ctx, "litho_field_create");
  }
  ~Imaging() { litho_field_destroy(field_); }
  void compute(const Mat& mask, double thr, double alpha, Mat& aerial, Mat& wafer) {
    const size_t n = (size_t)cache_.N() * cache_.N();
    cudaMemcpy(buf_.p, mask.data(), n * sizeof(float), cudaMemcpyHostToDevice);
    check(litho_imaging_compute(ctx_, cache_.get(), buf_.p, thr, alpha, buf_.p + n,
                                buf_.p + 2 * n, field_),
          ctx_, "litho_imaging_compute");
    aerial.resize(n);
    wafer.resize(n);
    cudaMemcpy(aerial.data(), buf_.p + n, n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaMemcpy(wafer.data(), buf_.p + 2 * n, n * sizeof(float), cudaMemcpyDeviceToHost);
  }
  litho_field* get_electric_field() const { return field_; }

 private:
  litho_ctx* ctx_;
  const Cache& cache_;
  DeviceBuffer buf_;
  litho_field* field_ = nullptr;
};

// Gradient::pe_gradient (gradient.cpp:121-141) on the field of an Imaging call.
inline Mat pe_gradient(litho_ctx* ctx, int N, const Mat& wafer, const Mat& target,
                       litho_field* field, double alpha, double* loss) {
  const size_t n = (size_t)N * N;
  DeviceBuffer w(n), t(n), g(n);
  w.up(wafer);
  t.up(target);
  check(litho_pe_gradient(ctx, field, w.p, t.p, nullptr, alpha, g.p, loss), ctx,
        "litho_pe_gradient");
  return g.down(n);
}

}  // namespace shim

int main(int argc, char** argv) {
  if (argc != 2) {
    std::fprintf(stderr, "usage: consumer <out.bin>\n");
    return 2;
  }
  litho_ctx* ctx = nullptr;
  const int cst = litho_ctx_create(0, nullptr, &ctx);
  if (cst != LITHO_OK) {
    std::printf("litho_ctx_create: %s\n", litho_status_string(cst));
    return 3;
  }
  int rc = 0;
  try {
    // Two smooth kernels on a 96 x 96 grid (the synthetic cache of the reference's
    // micro-gradient tests: exp(-(12 + 8k)|f|^2) with a linear phase, f in cycles/pixel).
    const int N = 96, K = 2;
    std::vector<std::complex<double>> ker((size_t)K * N * N);
    for (int k = 0; k < K; ++k)
      for (int r = 0; r < N; ++r)
        for (int c = 0; c < N; ++c) {
          const double fy = (r <= N / 2 ? r : r - N) / (double)N;
          const double fx = (c <= N / 2 ? c : c - N) / (double)N;
          const double amp = std::exp(-(12.0 + 8.0 * k) * (fx * fx + fy * fy) * 900.0);
          ker[((size_t)k * N + r) * N + c] = std::polar(amp, k * (0.35 * fx - 0.2 * fy) * 30.0);
        }
    shim::Cache cache(ctx, N, ker, {0.7, 0.3}, 1.2);
    const double pi = 3.14159265358979323846, thr = 0.25, alpha = 50.0;
    shim::Mat target((size_t)N * N, 0.f), theta((size_t)N * N), mask((size_t)N * N);
    for (int r = 30; r < 66; ++r)
      for (int c = 24; c < 40; ++c) target[(size_t)r * N + c] = 1.f;
    for (int r = 30; r < 42; ++r)
      for (int c = 40; c < 72; ++c) target[(size_t)r * N + c] = 1.f;
    for (size_t i = 0; i < target.size(); ++i) {
      theta[i] = (float)(target[i] > 0.f ? 0.3 * pi : 0.7 * pi);   // CTM_Optimizer.cpp:55-64
      mask[i] = 0.5f * (1.f + std::cos(theta[i]));
    }
    // Imaging::compute, then Gradient::pe_gradient on its field
    shim::Imaging imaging(ctx, cache);
    shim::Mat aerial, wafer;
    imaging.compute(mask, thr, alpha, aerial, wafer);
    double pe = 0.0;
    const shim::Mat grad_mask =
        shim::pe_gradient(ctx, N, wafer, target, imaging.get_electric_field(), alpha, &pe);
    // CTM_Optimizer::_evaluate_theta_objective in one call
    const size_t n = (size_t)N * N;
    shim::DeviceBuffer d_theta(n), d_target(n), d_gt(n), d_phi(n), d_vn(n), d_out(n);
    d_theta.up(theta);
    d_target.up(target);
    double loss = 0.0, norm = 0.0;
    shim::check(litho_ctm_evaluate(ctx, cache.get(), nullptr, d_theta.p, d_target.p, thr, alpha,
                                   nullptr, nullptr, nullptr, nullptr, d_gt.p, &loss, &norm),
                ctx, "litho_ctm_evaluate");
    const shim::Mat grad_theta = d_gt.down(n);
    // one LSM RK2 step (LSM_Optimizer.cpp:109-115) with the PE gradient as the speed
    shim::Mat phi(n);
    for (int r = 0; r < N; ++r)
      for (int c = 0; c < N; ++c)
        phi[(size_t)r * N + c] = (float)(20.0 - std::hypot(r - 48.0, c - 45.0));
    d_phi.up(phi);
    d_vn.up(grad_mask);
    double dt = 0.0;
    shim::check(litho_lsm_rk2_update(ctx, N, N, d_phi.p, d_vn.p, 1.0, 1.0, 0.5, 0.01, d_out.p,
                                     nullptr, &dt),
                ctx, "litho_lsm_rk2_update");
    const shim::Mat phi_next = d_out.down(n);
    // errors come back as status codes, not exceptions across the ABI
    shim::Mat bad = mask;
    bad[5] = NAN;
    shim::Mat a2, w2;
    int nonfinite = 0;
    try {
      imaging.compute(bad, thr, alpha, a2, w2);
    } catch (const shim::Error& e) {
      nonfinite = e.status;
    }
    FILE* f = std::fopen(argv[1], "wb");
    if (!f) throw std::runtime_error("cannot write the output file");
    const int hdr[3] = {N, K, nonfinite};
    std::fwrite(hdr, sizeof(int), 3, f);
    const double sc[4] = {pe, loss, norm, dt};
    std::fwrite(sc, sizeof(double), 4, f);
    std::fwrite(ker.data(), sizeof(std::complex<double>), ker.size(), f);
    const shim::Mat* outs[] = {&target, &theta,      &mask, &aerial,  &wafer,
                               &grad_mask, &grad_theta, &phi, &phi_next};
    for (const shim::Mat* m : outs) std::fwrite(m->data(), sizeof(float), m->size(), f);
    std::fclose(f);
    std::printf("consumer ok: PE %.9g, CTM loss %.9g, |dPE/dtheta| %.9g, dt %.9g, NaN mask -> %s\n",
                pe, loss, norm, dt, litho_status_string(nonfinite));
  } catch (const std::exception& e) {
    std::fprintf(stderr, "consumer failed: %s\n", e.what());
    rc = 1;
  }
  litho_ctx_destroy(ctx);
  return rc;
}
