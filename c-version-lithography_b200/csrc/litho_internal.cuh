// Internal declarations shared by the CUDA translation units of the
// imaging-and-gradient library. Not part of the public C ABI.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/litho_b200.h"

namespace litho_b200 {

// ---------------------------------------------------------------- status
struct Status {
  int code = LITHO_OK;
  std::string msg;
};

#define LITHO_CUDA_TRY(ctx, expr)                                              \
  do {                                                                         \
    cudaError_t _e = (expr);                                                   \
    if (_e != cudaSuccess) {                                                   \
      return (ctx)->fail(LITHO_ERR_CUDA, std::string(#expr) + ": " +           \
                                             cudaGetErrorString(_e));          \
    }                                                                          \
  } while (0)

// ---------------------------------------------------------------- band geometry
// Integer frequencies of the kernels' support: rows s_r = row0 + r (r < Nr),
// cols s_c = col0 + c (c < Nc); both wrap modulo N. The aerial image is then
// band-limited to the difference set D = [-(Nr-1), Nr-1] x [-(Nc-1), Nc-1].
// The small grid has Pr >= 2Nr-1, Pc >= 2Nc-1 points so that neither D nor
// S - S + D aliases onto the frequencies that are read back.
struct BandGeom {
  int N = 0, K = 0;
  int Nr = 0, Nc = 0;
  int row0 = 0, col0 = 0;
  int Pr = 0, Pc = 0;
  int kp_rows = 0;   // 2*Nr rounded up to 16: inner dimension of the row syntheses
  int kp_cols = 0;   // 2*Nc rounded up to 16: output width of the row analyses
};

// Device-resident optical cache (one per ImagingCache).
struct Cache {
  BandGeom g;
  float2* H = nullptr;        // K x Nr x Nc band kernels
  float* w = nullptr;         // K weights already divided by the source-weight sum
  std::vector<double> w_host; // same, FP64 on the host
  // Full-resolution twiddle tables (float2 rows of length N):
  float* TXS = nullptr;   // [2Nc][N]: rows 2c, 2c+1 = Re, Im e^{-2 pi i s_c x / N}
  float* TXD = nullptr;   // [2Nc][N]: same for d_c = 0..Nc-1
  float2* TYS = nullptr;  // [Nr][N]: e^{-2 pi i s_r y / N}
  float2* TYD = nullptr;  // [Nr][N]: e^{-2 pi i d_r y / N}, d_r = 0..Nr-1
  float* AYS = nullptr;   // [N][kp_rows]: (Re, Im) of TYS[r][y] interleaved per y
  float* AYD = nullptr;   // [N][kp_rows]: (Re, Im) of TYD[d][y] interleaved per y
  float2* TXSc = nullptr; // [Nc][N]: e^{-2 pi i s_c x / N} (complex rows)
  float2* TXDc = nullptr; // [Nc][N]: e^{-2 pi i d_c x / N}
  // Small-grid tables (Pr x Pc grid, P >= 2 * band - 1):
  float2* ESr_t = nullptr;  // [Nr][Pr]: e^{+2 pi i s_r j / Pr}
  float2* ESc_t = nullptr;  // [Nc][Pc]: e^{+2 pi i s_c j / Pc}
  float2* ESc = nullptr;    // [Pc][Nc]: the same, transposed
  float2* EDr_t = nullptr;  // [2Nr-1][Pr]: e^{+2 pi i d j / Pr}, d = -(Nr-1)..Nr-1
  float2* EDc_t = nullptr;  // [2Nc-1][Pc]: e^{+2 pi i d j / Pc}, d = -(Nc-1)..Nc-1
  int device = 0;
};

// Band-domain state of one imaging call: replaces the K full-resolution
// electric fields the reference caches (imaging.h:45-47) by the exact
// band representation from which any E_k can be re-synthesised.
struct Field {
  const Cache* cache = nullptr;
  float2* mband = nullptr;   // Nr x Nc: DFT of the mask on S divided by N^2
  float2* e = nullptr;       // K x Pr x Pc small-grid fields
  bool valid = false;
};

struct Scratch {
  void* base = nullptr;
  size_t bytes = 0;
};

struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int precision = LITHO_PRECISION_FP32;
  Scratch scratch;
  double* d_red = nullptr;       // FP64 reduction partials
  size_t red_cap = 0;
  double* h_red = nullptr;       // pinned host mirror for results
  std::string last_error;
  long long launches = 0;        // kernel launches issued by the library
  // Optional per-stage CUDA-event timing (litho_ctx_enable_stage_timing).
  bool timing = false;
  cudaEvent_t ev[LITHO_NUM_STAGES][2] = {};
  bool ev_pending[LITHO_NUM_STAGES] = {};
  double stage_ms[LITHO_NUM_STAGES] = {};
  long long stage_count[LITHO_NUM_STAGES] = {};
  void stage_begin(int st) {
    if (timing) cudaEventRecord(ev[st][0], stream);
  }
  void stage_end(int st) {
    if (timing) { cudaEventRecord(ev[st][1], stream); ev_pending[st] = true; }
  }
  void collect_stages();  // after a stream synchronize

  int fail(int code, const std::string& m) {
    last_error = m;
    return code;
  }
  int ensure_scratch(size_t bytes);
  int ensure_red(size_t n);
};

// Split of a length-N contraction into chunks of kps (a multiple of 16) for a
// requested number of splits; zs is the number of chunks actually produced.
inline void row_split(int N, int ksplit, int* kps, int* zs) {
  if (ksplit < 1) ksplit = 1;
  *kps = ((N + ksplit - 1) / ksplit + 15) / 16 * 16;
  *zs = (N + *kps - 1) / *kps;
}

// ---------------------------------------------------------------- kernels
// All launchers return cudaGetLastError() of their launches.
// Row analysis: out[z][y][2c+{0,1}] = sum_{x in split z} A[y][x] tw[2c+{0,1}][x],
// A = in (mode 0) or (1 + cos in)/2 (mode 1, optionally stored to mask_out).
cudaError_t launch_analysis_rows(cudaStream_t s, int mode, const float* in, float* mask_out,
                                 int* flag, const float* tw, int N, int ncols, int ksplit,
                                 float* out);
// Column contraction over y of the row-analysis partials (see band_dft.cu).
cudaError_t launch_analysis_cols(cudaStream_t s, const float* R, int ksplit, int N, int ncols,
                                 const float2* TY, int nrows_out, int nr, int sym, int ysplit,
                                 float scale, float2* out_partial);
cudaError_t launch_band_forward(cudaStream_t s, const Cache& c, const float2* mpart, int ysplit,
                                Field& f, float* ik, float2* T, float2* Q, float2* chat,
                                float* Ut);
cudaError_t launch_band_adjoint(cudaStream_t s, const Cache& c, const Field& f,
                                const float2* gpart, int ysplit, double scale, float2* Gam,
                                float* gam, float2* Z1, float2* Zk, float2* X, float* Vt);
cudaError_t launch_expand_cols(cudaStream_t s, const float2* coef, int nrows, int ncoef,
                               int coef_ld, const float2* TX, int N, int mode, int nc, int kp,
                               float* Ut);

// Row synthesis: out[y][x] = sum_f AY[y][f] * Bt[x][f] with a fused epilogue.
struct ResistEpilogue {
  int mode;                 // 0: image only; 1: resist + loss + dL/dI
  float thr, alpha;
  float* aerial;            // nullable
  float* wafer;             // nullable
  const float* target;      // mode 1
  const float* pe_window;   // nullable
  const float* pen_window;  // nullable
  float pe_weight, penalty, pen_thr;
  float* dldi;              // mode 1
  double* loss_partial;     // mode 1: per-block (pe, penalty) FP64 partial sums
};
struct GradEpilogue {
  float* grad_mask;         // nullable
  const float* theta;       // nullable: theta chain when set
  float* grad_theta;        // with theta
  double* norm_partial;     // with theta: per-block partial of sum grad_theta^2
};
cudaError_t launch_synth_resist(cudaStream_t s, const float* AY, const float* Bt, int N, int kp,
                                const ResistEpilogue& ep, int* nblocks);
cudaError_t launch_synth_grad(cudaStream_t s, const float* AY, const float* Bt, int N, int kp,
                              const GradEpilogue& ep, int* nblocks);
cudaError_t launch_sum_partials(cudaStream_t s, const double* part, int n, int stride,
                                double* out);
cudaError_t launch_export_field(cudaStream_t s, const Cache& c, const Field& f, int k,
                                float2* tmp_rows, float2* out);
cudaError_t launch_pe_loss(cudaStream_t s, const float* w, const float* t, const float* pe_win,
                           const float* pen_win, float penalty, float pen_thr, size_t n,
                           double* partial, int* nblocks);
cudaError_t launch_pe_dldi(cudaStream_t s, const float* w, const float* t, const float* pe_win,
                           const float* pen_win, float pe_weight, float penalty, float pen_thr,
                           size_t n, float* dldi, double* partial, int* nblocks);

// Level set (levelset.cu). what: 0 delta (+|Vn|), 1 kappa term, 2 normal,
// 3 RK2 stage 1, 4 RK2 stage 2 (+ mask).
cudaError_t launch_levelset(cudaStream_t s, int what, int rows, int cols, const float* phi,
                            const float* phi0, const float* vn, float dx, float dy, float b,
                            const float* dt, float* out, float* out2);
cudaError_t launch_dt(cudaStream_t s, const float* vn, size_t n, float dx, float dy, float cfl,
                      float b, float* part, float* vmax, float* dt, int* bad);

}  // namespace litho_b200
