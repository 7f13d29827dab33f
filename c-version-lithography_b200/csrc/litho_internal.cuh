// Internal declarations shared by the CUDA translation units of the
// imaging-and-gradient library. Not part of the public C ABI.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <map>
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
  float2* EDc = nullptr;    // [Pc][2Nc-1]: the same, transposed
  // Split-BF16 tensor-core operand images (tc2.cu), built when tc2_supported:
  // the row-synthesis twiddles AYS / AYD (rows y), the row-analysis column
  // twiddles TXS / TXD (rows f, K tiles of x) and the row twiddles TYS / TYD
  // (rows 2r / 2r + 1 = Re / Im, K tiles of y).
  void* AYS_img = nullptr;
  void* AYD_img = nullptr;
  void* TXS_img = nullptr;
  void* TXD_img = nullptr;
  void* TYS_img = nullptr;
  void* TYD_img = nullptr;
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

// Identity of one CTM evaluation's launch chain: every device pointer it
// touches, the band geometry and the scalars baked into its kernels.
struct EvalKey {
  const void* ptr[16] = {};
  int geom[6] = {};
  double thr = 0.0, alpha = 0.0;
  bool operator==(const EvalKey& o) const {
    for (int i = 0; i < 16; ++i)
      if (ptr[i] != o.ptr[i]) return false;
    for (int i = 0; i < 6; ++i)
      if (geom[i] != o.geom[i]) return false;
    return thr == o.thr && alpha == o.alpha;
  }
};

struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int precision = LITHO_PRECISION_FP32;
  Scratch scratch;
  Scratch host_stage;            // device staging of the host-buffer entry points
  cudaStream_t aux = nullptr;    // upload stream of the host-buffer entry points
  cudaEvent_t ev_aux[2] = {};    // [0] theta uploaded (main stream), [1] target uploaded (aux)
  // Pipelined host-buffer batches: download stream and per-slot events (uploaded,
  // computed, downloaded) of the two device staging slots.
  Scratch pipe_stage;
  cudaStream_t dn = nullptr;
  cudaEvent_t ev_pipe[2][3] = {};
  // CUDA graph of the last repeated CTM evaluation (litho_ctm_evaluate): captured
  // on the second consecutive call with the same key, replayed while it stays.
  bool graphs = true;
  cudaGraphExec_t eval_graph = nullptr;
  EvalKey eval_graph_key, eval_last_key;
  bool eval_last_valid = false;
  long long eval_graph_launches = 0;
  // The same for the batched split-BF16 evaluation (litho_ctm_evaluate_batch), kept
  // apart so that a loop alternating single-tile and batched calls replays both.
  cudaGraphExec_t batch_graph = nullptr;
  EvalKey batch_graph_key, batch_last_key;
  bool batch_last_valid = false;
  long long batch_graph_launches = 0;
  double* d_red = nullptr;       // FP64 reduction partials
  // Deferred status of the device-resident entry points ([0] a non-finite input was
  // seen, [1] the first tensor-core wait code), read by litho_ctx_deferred_status.
  int* d_deferred = nullptr;
  int ensure_deferred();
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
  // Schedules chosen by litho_ctx_autotune: the small-grid chunk width per (N, batch)
  // and the chamfer CTA size per (columns, images); 0 where nothing was tuned.
  std::map<std::pair<int, int>, int> tuned_band, tuned_chamfer;
  int band_width(int N, int batch) const {
    const auto it = tuned_band.find({N, batch});
    return it == tuned_band.end() ? 0 : it->second;
  }
  int chamfer_threads(int cols, int nimg) const {
    const auto it = tuned_chamfer.find({cols, nimg});
    return it == tuned_chamfer.end() ? 0 : it->second;
  }
  // Schedule of the split-BF16 tensor-core passes (LITHO_TC_SCHEDULE_*): per-tile CTAs
  // (tc2.cu) or the persistent pipelines (tc3.cu, the default where supported). A
  // batched call and a single-image call take the same schedule, so every image's
  // results are the same alone and in a batch, bit for bit.
  int tc_schedule = LITHO_TC_SCHEDULE_AUTO;
  // Largest number of micro tiles per batched pass of the exchange (0: as many as the
  // scratch budget allows); litho_ctx_set_exchange_group.
  int exchange_group_max = 0;
  // Layout of the tile partials the last analysis launch left in the scratch, for
  // the reduction that follows it: 0 row-major, else column-major with this many rows
  // (forward and adjoint analyses; the adjoint's may come from the fused synthesis).
  int fwd_part_trows = 0, adj_part_trows = 0;
  // The schedule used for `batch` images of size N: the set one, or under
  // LITHO_TC_SCHEDULE_AUTO the one litho_ctx_autotune chose for (N, batch), else the
  // persistent pipelines.
  std::map<std::pair<int, int>, int> tuned_tc;
  bool tc_persistent(int N, int batch) const {
    if (tc_schedule != LITHO_TC_SCHEDULE_AUTO) return tc_schedule == LITHO_TC_SCHEDULE_PERSISTENT;
    const auto it = tuned_tc.find({N, batch});
    return it == tuned_tc.end() || it->second == LITHO_TC_SCHEDULE_PERSISTENT;
  }
};

// ---------------------------------------------------------------- launch helper
// Launch with programmatic stream serialization (the kernel must follow the
// pdl_trigger / pdl_wait protocol of device_common.cuh).
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                       cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  // On the legacy default stream every launch keeps the plain stream order.
  cfg.numAttrs = (s == nullptr || s == cudaStreamLegacy) ? 0 : 1;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// ---------------------------------------------------------------- kernels
// All launchers return cudaGetLastError() of their launches.
// Tile analysis: for every 128 x 128 tile t of the image A (A = in for mode 0,
// (1 + cos in)/2 for mode 1, optionally stored to mask_out)
//   part[a][c][t] = sum_{(y, x) in t} T(a, y) A[y][x] tw(c, x)
// with tw = [2 ncols][N] real rows (Re, Im) and T(a, y) = TY[a][y] (sym 0,
// a < nrows_out) or, for sym 1, d = a - (nr - 1), TY[d][y] / conj(TY[-d][y]).
int analysis_tiles(int N);
cudaError_t launch_analysis(cudaStream_t s, int mode, const float* in, float* mask_out,
                            int* flag, const float* tw, int N, int ncols, const float2* TY,
                            int nrows_out, int nr, int sym, float2* part);
// out[o] = scale * sum_t part[o][t] (fixed order). Tile blocks are row-major [row][c],
// or column-major [c][row] with trows rows when trows > 0 (the persistent tensor-core
// analyses); out is row-major either way.
cudaError_t launch_reduce_tiles(cudaStream_t s, const float2* part, int tiles, int count,
                                float scale, float2* out, int batch = 1, int trows = 0);
// Small-grid stage of the forward: f.mband -> f.e, ik, iP and Ut (the row
// synthesis operand), or, with img set, Ut's split-BF16 operand image for the
// tensor-core synthesis (launch_pack_tc2_rows layout) instead of Ut.
// Shared memory of its per-kernel CTA: band_fields_smem.
size_t band_fields_smem(const BandGeom& g);
size_t band_max_smem(const BandGeom& g);
// width: the schedule of the small-grid field and Z kernels: column chunks of 8 or 16
// columns per CTA, or BW_WHOLE (the whole small grid per CTA, where its tables fit in
// shared memory); 0: whole from 8 images on, else 16 for batches of 4 or more images,
// else 8. The results do not depend on it, bit for bit.
constexpr int BW_WHOLE = 128;
cudaError_t launch_band_forward(cudaStream_t s, const Cache& c, Field& f, float* ik, float* iP,
                                float2* chat, float* Ut, void* img, int batch = 1,
                                int width = 0);
// Small-grid stage of the adjoint: gh (the D-band DFT of dL/dI) -> gam, Zk, X and Vt
// (or Vt's operand image, as for the forward).
cudaError_t launch_band_adjoint(cudaStream_t s, const Cache& c, const Field& f, const float2* gh,
                                double scale, float* gam, float2* Zk, float2* X, float* Vt,
                                void* img, int batch = 1, int width = 0);

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
  // mode 1: sum the background-penalty term (threshold pen_thr) into the loss partials
  // even when penalty is 0 (it then adds nothing to dL/dI), for the loss the
  // reference's LSM loop tracks (LSM_Optimizer.cpp:87-90).
  int loss_penalty_term;
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
cudaError_t launch_sum_partials2(cudaStream_t s, const double* a, int na, int sa, double* out_a,
                                 const double* b, int nb, int sb, double* out_b);
// Batched sums: per image b, sa components over na blocks of a (stride na sa per
// image) then sb over nb blocks of b, into out[b][sa + sb].
cudaError_t launch_sum_partials_batch(cudaStream_t s, const double* a, int na, int sa,
                                      const double* b, int nb, int sb, double* out, int batch);
cudaError_t launch_export_field(cudaStream_t s, const Cache& c, const Field& f, int k,
                                float2* tmp_rows, float2* out);
cudaError_t launch_pe_loss(cudaStream_t s, const float* w, const float* t, const float* pe_win,
                           const float* pen_win, float penalty, float pen_thr, size_t n,
                           double* partial, int* nblocks);
cudaError_t launch_pe_dldi(cudaStream_t s, const float* w, const float* t, const float* pe_win,
                           const float* pen_win, float pe_weight, float penalty, float pen_thr,
                           size_t n, float* dldi, double* partial, int* nblocks);

// Split-BF16 tensor-core passes (tc2.cu). err receives a code (1..6) when a
// bounded wait of a kernel expires.
// Tile analysis, same partials as launch_analysis: tx_img / ty_img are the
// images of tw and TY (launch_pack_tc2_tx / _ty); needs tc2_analysis_supported.
bool tc2_analysis_supported(int ncols, int nr);
size_t tc2_tx_image_bytes(int N, int ncols);
size_t tc2_ty_image_bytes(int N);
cudaError_t launch_pack_tc2_tx(cudaStream_t s, const float* tw, int ncols, int N, void* dst);
cudaError_t launch_pack_tc2_ty(cudaStream_t s, const float2* T, int nr, int N, void* dst);
cudaError_t launch_analysis_tc2(cudaStream_t s, int mode, const float* in, float* mask_out,
                                int* flag, int N, int ncols, int nrows_out, int nr, int sym,
                                float2* part, const void* tx_img, const void* ty_img, int* err,
                                int batch = 1);
// Row synthesis: Aimg = image of AY ([N][kp], launch_pack_tc2_rows), Bimg = image
// of the band operand Bt ([N][kp]); kp % 16 == 0 and kp <= 128.
size_t tc2_rows_image_bytes(int N, int kp);
cudaError_t launch_pack_tc2_rows(cudaStream_t s, const float* src, int N, int kp, void* dst);
cudaError_t launch_synth_resist_tc2(cudaStream_t s, const void* Aimg, const void* Bimg, int N,
                                    int kp, const ResistEpilogue& ep, int* err, int* nblocks,
                                    int batch = 1);
cudaError_t launch_synth_grad_tc2(cudaStream_t s, const void* Aimg, const void* Bimg, int N,
                                  int kp, const GradEpilogue& ep, int* err, int* nblocks,
                                  int batch = 1);
// Resist synthesis fused with the adjoint tile analysis (CTM evaluation): loss
// partials as launch_synth_resist_tc2 (ep.dldi unused), and the adjoint partials
// part[tile][2 nr - 1][ncols] of dL/dI as launch_analysis_tc2 with the TXD / TYD
// images; a non-finite dL/dI raises flag[0].
cudaError_t launch_synth_resist_analysis_tc2(cudaStream_t s, const void* Aimg, const void* Bimg,
                                             int N, int kp, const ResistEpilogue& ep, int ncols,
                                             int nr, float2* part, int* flag, const void* tx_img,
                                             const void* ty_img, int* err, int* nblocks,
                                             int batch = 1);
// The same passes as persistent, warp-specialised pipelines (tc3.cu): one CTA per SM
// over a contiguous share of the (image, tile) items. Same arguments and results
// (image values bit for bit; FP64 partial sums in another order). Supported for tile
// analyses with 2 Nc rounded to 16 at most 96 and syntheses with kp <= 128; the fused
// kernel also needs its shared-memory plan to fit.
bool tc3_analysis_supported(int ncols, int nr);
bool tc3_synth_supported(int kp);
bool tc3_fused_supported(int kp, int ncols, int nr);
cudaError_t launch_analysis_tc3(cudaStream_t s, int mode, const float* in, float* mask_out,
                                int* flag, int N, int ncols, int nrows_out, int nr, int sym,
                                float2* part, const void* tx_img, const void* ty_img, int* err,
                                int batch = 1);
cudaError_t launch_synth_resist_tc3(cudaStream_t s, const void* Aimg, const void* Bimg, int N,
                                    int kp, const ResistEpilogue& ep, int* err, int* nblocks,
                                    int batch = 1);
cudaError_t launch_synth_grad_tc3(cudaStream_t s, const void* Aimg, const void* Bimg, int N,
                                  int kp, const GradEpilogue& ep, int* err, int* nblocks,
                                  int batch = 1);
cudaError_t launch_synth_resist_analysis_tc3(cudaStream_t s, const void* Aimg, const void* Bimg,
                                             int N, int kp, const ResistEpilogue& ep, int ncols,
                                             int nr, float2* part, int* flag, const void* tx_img,
                                             const void* ty_img, int* err, int* nblocks,
                                             int batch = 1);
// The tensor-core path needs kp <= 128 and 2 Nc <= 128 (bands up to 64 x 64).
inline bool tc2_supported(const BandGeom& g) {
  return g.kp_rows <= 128 && tc2_analysis_supported(g.Nc, g.Nr);
}

// Level set (levelset.cu). what: 0 delta (+|Vn|), 1 kappa term, 2 normal,
// 3 RK2 stage 1, 4 RK2 stage 2 (+ mask), 5 mask phi >= 0, 6 speed restricted to the
// window, 7 +-0.5 sign image of phi >= 0, 8 out = phi inside the window, phi0 outside,
// 9 phi - 0.5.
// window (host, nullable): {y0, y1, x0, x1}; stages 3 and 4 update only inside it
// (outside they keep phi / phi0). NULL = the whole grid.
cudaError_t launch_levelset(cudaStream_t s, int what, int rows, int cols, const float* phi,
                            const float* phi0, const float* vn, float dx, float dy, float b,
                            const float* dt, float* out, float* out2,
                            const int* window = nullptr, int nimg = 1,
                            const int* d_windows = nullptr, int dt_stride = 0);
// render_levelset_mask for nimg images of rows x cols: gray = 0 -> phi >= 0,
// gray = 1 -> subpixel coverage of the scale-times bilinear upsampling.
cudaError_t launch_render_mask(cudaStream_t s, const float* phi, int rows, int cols, int nimg,
                               int gray, int scale, float* mask);
cudaError_t launch_dt(cudaStream_t s, const float* vn, size_t n, float dx, float dy, float cfl,
                      float b, float* part, float* vmax, float* dt, int* bad);
// Chamfer signed distance of reinit_sdf over nimg rows x cols images back to back:
// inside = phi > level (phi >= level when inclusive); sdf must not alias phi.
// threads: CTA size (128 or 256 for rows of up to 32 columns per thread, 1024; 0 picks
// by the row length).
cudaError_t launch_reinit_sdf(cudaStream_t s, int rows, int cols, const float* phi, float level,
                              int inclusive, float dx, float* sdf, int nimg = 1, int threads = 0);
// Fills nimg rows x cols images with a pattern whose zero set crosses every row.
cudaError_t launch_chamfer_probe(cudaStream_t s, float* p, int rows, int cols, int nimg);
// max |Vn| and dt of nimg images of n pixels: vd[2 i] = max |Vn_i|, vd[2 i + 1] = dt_i;
// part holds nimg * dt_batch_blocks(n, nimg) floats.
int dt_batch_blocks(size_t n, int nimg);
cudaError_t launch_dt_batch(cudaStream_t s, const float* vn, size_t n, int nimg, float dx,
                            float dy, float cfl, float b, float* part, float* vd, int* bad);

// Sparse EPE at host-selected edge points (epe.cu): eps n x 2 (y, x) and weights n,
// device FP64. signed_epe (nullable) per point; partial: 3 FP64 sums per block
// (weighted squared loss, |EPE| nm, active count); dldi (nullable): scatter of
// 2 w (I - thr) / G^2 onto each point's bilinear stencil (atomic adds).
// With dldi set, each EP's dL/dI (scatter_scale x 2 w (I - thr) / G^2) is added onto its
// bilinear stencil deterministically: the (pixel, weighted value) pairs of all EPs are
// sorted by pixel with a stable radix sort (EP order kept within a pixel) and each
// pixel's run is summed in FP64 in that order, then added to dldi once. That needs
// `work` of at least epe_scatter_work_bytes(n) bytes (device, 256-byte aligned).
size_t epe_scatter_work_bytes(int n);
cudaError_t launch_epe(cudaStream_t s, const float* I, int rows, int cols, const double* eps,
                       const double* w, int n, double thr, double pixel_nm, double* signed_epe,
                       double* partial, float* dldi, double scatter_scale, int* nblocks,
                       void* work = nullptr, size_t work_bytes = 0);

// Full-chip micro tiles (fullchip.cu). Rects are 4 ints (y0, y1, x0, x1) per tile;
// origins 2 ints (y, x) per tile; rel holds max_rel entries of FC_REL_INTS ints
// per tile: {neighbour, direction, my_guard[4], neighbour_overlap[4],
// my_overlap[4], neighbour_guard[4]}.
constexpr int FC_REL_INTS = 18;
cudaError_t launch_tiles_extract(cudaStream_t s, const float* g, int H, int W, int ntiles,
                                 const int* origins, int ts, float* out);
cudaError_t launch_tiles_assemble(cudaStream_t s, const float* loc, int ntiles, int ts,
                                  const int* core_g, const int* core_l, int W, float* g);
cudaError_t launch_loss_windows(cudaStream_t s, const float* target, int ntiles, int ts,
                                const int* region, int loss_type, const float* main_dil,
                                float* pe_w, float* pen_w, float* epe_w);
cudaError_t launch_dilate_main(cudaStream_t s, const float* target, int ntiles, int ts,
                               int iterations, float* tmp, float* out);
// grect: the region as a global half-open rect (y0, y1, x0, x1); oy, ox the tile origin.
cudaError_t launch_ep_candidates(cudaStream_t s, const double* eps, const double* w, int n,
                                 int periods, int H, int W, int oy, int ox, const int* grect,
                                 int ts, const float* win, double* out_eps, double* out_w);
// L-BFGS vector kernels (lbfgs.cu): out[j] = rows[j] . v in FP64 (k <= 64 rows of
// length n, row stride ld; partial holds multi_dot_blocks(n) * k doubles), and
// out = cv v + sum_j coef[j] rows[j] (coef: k device doubles).
int multi_dot_blocks(size_t n);
cudaError_t launch_multi_dot(cudaStream_t s, const float* rows, size_t ld, int k, size_t n,
                             const float* v, double* partial, double* out);
cudaError_t launch_combine(cudaStream_t s, const float* rows, size_t ld, int k, size_t n,
                           const double* coef, const float* v, double cv, float* out);
// The inner products of k rows with up to three vectors (v1, v2 nullable) in one pass:
// out[v k + j]; partial holds multi_dot3_blocks(n, k) * ((k + 7) / 8) * 24 doubles.
int multi_dot3_blocks(size_t n, int k);
cudaError_t launch_multi_dot3(cudaStream_t s, const float* rows, size_t ld, int k, size_t n,
                              const float* v0, const float* v1, const float* v2, double* partial,
                              double* out);
// Loss-region and Core sums of nimg tiles in one launch (rectangles: device, 4 ints
// per tile); partial holds nimg * rect_losses_batch_blocks(ts) * 6 doubles.
int rect_losses_batch_blocks(int ts);
cudaError_t launch_rect_losses_batch(cudaStream_t s, const float* Wf, const float* T,
                                     const float* pe_w, const float* pen_w, int ts,
                                     const int* d_regions, const int* d_cores, float pen_thr,
                                     double* partial, int nimg);
cudaError_t launch_exchange(cudaStream_t s, const float* masks, const float* raw, int ntiles,
                            int ts, const int* nrel, const int* rel, int max_rel,
                            const litho_exchange_options& o, float* grad, double* cept_loss,
                            double* part);
// CTAs per tile and relation of launch_exchange; part holds ntiles * max_rel * that.
int exchange_chunks(int ntiles);
cudaError_t launch_theta_update(cudaStream_t s, float* theta, const float* grad, int ntiles,
                                int ts, const int* win, float lr, float* mask);

}  // namespace litho_b200

// The ABI's opaque handles are the library's own objects.
struct litho_ctx : public litho_b200::Context {};
struct litho_cache : public litho_b200::Cache {};
struct litho_field : public litho_b200::Field {};
