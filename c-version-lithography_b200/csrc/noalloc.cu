// RK2 level-set update without any device allocation: the same kernels as
// litho_lsm_rk2_update, with the intermediate stage and the dt reduction held
// in one file-scope device array instead of a context's scratch memory.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "litho_internal.cuh"

using namespace litho_b200;

namespace {

// Layout of the static scratch, in floats: [0] non-finite flag (int, cleared by
// every call), [64, 64 + 296) per-block |Vn| maxima, [360] max |Vn|, [361] dt,
// [512, 512 + LITHO_RK2_NOALLOC_MAX_PIXELS) the first RK2 stage phi1.
constexpr size_t kFlag = 0, kPart = 64, kVmax = 360, kDt = 361, kPhi1 = 512;
static __device__ __align__(256) float g_rk2_scratch[kPhi1 + LITHO_RK2_NOALLOC_MAX_PIXELS];

constexpr int kMaxDevices = 64;
float* g_scratch_ptr[kMaxDevices] = {};
std::mutex g_setup_mutex;

// Address of this device's copy of the scratch (looked up once per device).
int scratch_for_device(int dev, float** out) {
  if (dev < 0 || dev >= kMaxDevices) return LITHO_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_rk2_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return LITHO_ERR_CUDA;
    }
    g_scratch_ptr[dev] = static_cast<float*>(p);
  }
  *out = g_scratch_ptr[dev];
  return LITHO_OK;
}

}  // namespace

extern "C" int litho_lsm_rk2_update_noalloc(void* stream, int rows, int cols, const float* d_phi,
                                            const float* d_vn, double dx, double dy, double cfl,
                                            double b, float* d_phi_out, float* d_mask,
                                            double* dt) {
  if (!d_phi || !d_vn || !d_phi_out || rows <= 0 || cols <= 0 || !(dx > 0.0) || !(dy > 0.0))
    return LITHO_ERR_INVALID_ARGUMENT;
  if (rows < 3 || cols < 3) return LITHO_ERR_SHAPE;
  const size_t n = (size_t)rows * cols;
  if (n > (size_t)LITHO_RK2_NOALLOC_MAX_PIXELS) return LITHO_ERR_UNSUPPORTED;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return LITHO_ERR_CUDA;
  }
  float* base = nullptr;
  int st = scratch_for_device(dev, &base);
  if (st) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int* flag = reinterpret_cast<int*>(base + kFlag);
  float* dt_dev = base + kDt;
  if (cudaMemsetAsync(flag, 0, sizeof(int), s) != cudaSuccess ||
      launch_dt(s, d_vn, n, (float)dx, (float)dy, (float)cfl, (float)b, base + kPart,
                base + kVmax, dt_dev, flag) != cudaSuccess ||
      launch_levelset(s, 3, rows, cols, d_phi, nullptr, d_vn, (float)dx, (float)dy, (float)b,
                      dt_dev, base + kPhi1, nullptr) != cudaSuccess ||
      launch_levelset(s, 4, rows, cols, base + kPhi1, d_phi, d_vn, (float)dx, (float)dy,
                      (float)b, dt_dev, d_phi_out, d_mask) != cudaSuccess) {
    cudaGetLastError();
    return LITHO_ERR_CUDA;
  }
  float head[kDt + 1];
  if (cudaMemcpyAsync(head, base, sizeof(head), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return LITHO_ERR_CUDA;
  }
  int bad;
  static_assert(sizeof(bad) == sizeof(float), "flag shares a float slot");
  std::memcpy(&bad, head + kFlag, sizeof(bad));
  if (bad) return LITHO_ERR_NONFINITE;
  if (dt) *dt = head[kDt];
  return LITHO_OK;
}
