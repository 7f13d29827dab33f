/*
 * litho_b200.h - C ABI of the B200 imaging-and-gradient library.
 *
 * Drop-in boundary for the hot path of wyhcoder/C-version-Lithography:
 *   SOCS/Abbe aerial image  I = sum_k w_k |IFFT(H_k . FFT(M))|^2 / sum(ws),
 *   sigmoid resist          W = 1 / (1 + exp(-alpha (I - thr))),
 *   pattern-error loss      PE = sum (W - T)^2 (+ background penalty),
 *   its adjoint             dPE/dM and dPE/dtheta through M = (1 + cos theta)/2,
 *   WENO5-Godunov level-set update (RK2) used by LSM and full-chip LSM.
 *
 * Conventions
 *   - Every entry point returns an int status (LITHO_OK == 0) and never throws.
 *     litho_ctx_last_error() gives a message for the last failure on a context.
 *   - Images are float32, row-major (row = y, col = x), N x N, in DEVICE memory
 *     unless the name ends in _host. Eigen's default column-major matrices map
 *     onto these by transposition (Eigen::Map<Matrix<float,-1,-1,RowMajor>>).
 *   - Kernels and weights cross the boundary in float64, as the reference's
 *     ImagingCache holds them; the library keeps them in float32 on the device.
 *   - A context owns one CUDA stream and its scratch memory and is used by one
 *     host thread at a time (the reference uses one Imaging/Gradient object per
 *     thread, include/utils/micro_gradient_exchange.h:131-138).
 *   - Caches must outlive the fields created from them (the reference's
 *     Imaging holds a const reference to its ImagingCache, imaging.h:42).
 */
#ifndef LITHO_B200_H
#define LITHO_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define LITHO_OK 0
#define LITHO_ERR_INVALID_ARGUMENT 1 /* std::invalid_argument in the reference */
#define LITHO_ERR_SHAPE 2            /* dimension mismatch */
#define LITHO_ERR_NONFINITE 3        /* NaN/Inf in an input that must be finite */
#define LITHO_ERR_OOM 4              /* device allocation failed */
#define LITHO_ERR_CUDA 5             /* CUDA runtime error */
#define LITHO_ERR_NOT_READY 6        /* a field used before imaging filled it */
#define LITHO_ERR_UNSUPPORTED 7      /* size or option outside what is built */

#define LITHO_PRECISION_FP32 0       /* plain FP32 DFT passes (SIMT) */
#define LITHO_PRECISION_BF16X3 1     /* full-resolution analyses and syntheses on the tcgen05
                                        tensor cores in split BF16 (hi*hi + hi*lo + lo*hi,
                                        FP32 accumulation) */

#define LITHO_TC_SCHEDULE_AUTO 0       /* the one litho_ctx_autotune chose for the size
                                          and batch, else persistent; per tile where the
                                          band does not fit the persistent kernels'
                                          shared-memory plan (the default) */
#define LITHO_TC_SCHEDULE_PER_TILE 1   /* one CTA per 128 x 128 tile, phases in order */
#define LITHO_TC_SCHEDULE_PERSISTENT 2 /* one CTA per SM over a share of the (image, tile)
                                          items, warp-specialised and pipelined */

typedef struct litho_ctx litho_ctx;
typedef struct litho_cache litho_cache;
typedef struct litho_field litho_field;

int litho_version(void);
const char* litho_status_string(int status);
const char* litho_ctx_last_error(const litho_ctx* ctx);

/* ------------------------------------------------------------ context
 * stream: a cudaStream_t to run on (cudaStreamLegacy for the legacy default stream), or
 * NULL for a stream the context creates. On the legacy default stream the kernels keep
 * the plain stream order (no programmatic dependent launch) and litho_ctm_evaluate
 * launches its chain directly (that stream cannot be captured into a graph).
 */
int litho_ctx_create(int device, void* stream, litho_ctx** out);
int litho_ctx_destroy(litho_ctx* ctx);
int litho_ctx_synchronize(litho_ctx* ctx);
int litho_ctx_set_precision(litho_ctx* ctx, int precision);
/* Kernels this context has launched so far (a counter, for benchmarks). */
long long litho_ctx_launch_count(const litho_ctx* ctx);
/* CUDA-graph replay of litho_ctm_evaluate and of the split-BF16
 * litho_ctm_evaluate_batch (on by default, one graph for each): the second
 * consecutive call with the same buffers, cache, precision, batch and scalars
 * captures its launch chain into a graph; later identical calls replay it with one
 * launch. Contexts on the legacy default stream never capture. Turn it off
 * when the context's stream is itself being captured by the caller, or under
 * tools that cannot follow a stream capture. */
int litho_ctx_enable_graphs(litho_ctx* ctx, int on);
/* Schedule of the split-BF16 tensor-core passes (LITHO_TC_SCHEDULE_*). The schedules
 * compute the same products per pixel; the loss and norm partial sums are added in
 * another order, so they may differ in their last bits. This choice has no
 * counterpart in the reference (whose passes are FFTs on the CPU). */
int litho_ctx_set_tc_schedule(litho_ctx* ctx, int schedule);
/* Largest number of micro tiles the split-BF16 exchange (litho_exchange_compute*)
 * images in one batched pass; 0 (the default): every tile of the partition while the
 * pass's scratch stays within 4 GiB, at least 16. Results do not depend on it. */
int litho_ctx_set_exchange_group(litho_ctx* ctx, int max_tiles);

/* Per-stage device timing with CUDA events on the context's stream. Stages:
 * 0 tile analysis of the mask (row DFT + column contraction per 128 x 128 tile),
 * 1 tile reduction, 2 band forward (small grid), 3 row synthesis + resist/loss
 * epilogue, 4 tile analysis of dL/dI, 5 its tile reduction, 6 band adjoint,
 * 7 row synthesis + theta chain, 8 level-set kernels (RK2 update, reinit).
 * ms[i] accumulates milliseconds, counts[i] calls of stage i since timing was
 * enabled (enabling resets both). */
#define LITHO_NUM_STAGES 9
int litho_ctx_enable_stage_timing(litho_ctx* ctx, int on);
int litho_ctx_stage_times(const litho_ctx* ctx, double* ms, long long* counts);

/* ------------------------------------------------------------ optical set-up
 * litho_socs_prepare replaces LithoPrepare's SOCS path (source/litho_model/
 * litho_prepare.cpp:16-385 with grid.cpp:27,38-48, pupil.cpp:14-46, zernike.cpp:12-56
 * and source.cpp:114-158): from the optics it builds, in FP64, the annular source map
 * and its points, the shifted-pupil matrix A = [sqrt(w_s) P(f + f_s)] over the SOCS
 * support, and the K strongest coherent modes of A (eigenvalues sigma_k^2), then
 * creates the device cache from them (as litho_cache_create_band). The kernels equal
 * the reference's up to a phase per kernel (and a basis within each degenerate
 * eigenvalue), which the image does not depend on when K keeps whole degenerate groups.
 * info (nullable) receives the sizes; eigenvalues (nullable, K doubles) and
 * band_kernels (nullable, K x Nr x Nc interleaved complex doubles, band row r at integer
 * frequency row0 + r) receive the kernels; size them from a first call with info only
 * and num_socs fixed, or generously (K <= number of source points). */
typedef struct litho_socs_params {
  int N;                  /* optical grid (pixels per side) */
  double pixel_nm;        /* pixel size */
  double wavelength_nm;
  double na;
  double sigma_in, sigma_out; /* annulus, normalised to NA / lambda */
  double smoothing;       /* source edge width (0: hard edges, the reference's default) */
  int upsample;           /* source oversampling per axis (<= 0: 10, the reference's) */
  int num_socs;           /* kernels kept (<= 0: all source points; the reference keeps 36) */
  int compact;            /* 1: support cropped to the shifted pupils (compact_socs) */
  const double* zernike;  /* nullable: Fringe coefficients Z1..Z11 (11 doubles, waves) */
} litho_socs_params;
typedef struct litho_socs_info {
  int K, Ns;              /* kernels kept, source points */
  int Nr, Nc, row0, col0; /* band of the kernels (integer frequencies row0.., col0..) */
  double ws_sum;          /* sum of the source weights (the image normaliser) */
  double energy_captured; /* kept eigenvalues / all eigenvalues */
} litho_socs_info;
int litho_socs_prepare(litho_ctx* ctx, const litho_socs_params* params, litho_cache** out,
                       litho_socs_info* info, double* eigenvalues, double* band_kernels);

/* ------------------------------------------------------------ optical cache
 * Replaces ImagingCache (include/litho_model/litho_prepare.h:18-47) as consumed
 * by Imaging (source/litho_model/imaging.cpp:60-107) and Gradient
 * (source/utils/gradient.cpp:34-55).
 *
 * litho_cache_create_dense: the reference's own layout. kernels = K full N x N
 *   complex frequency kernels with DC at index (0,0) (the layout of
 *   ImagingCache::optical_kernels_frequency), interleaved (re, im) float64,
 *   row-major [k][row][col][2]. weights = socs_eigenvalues (SOCS) or source_ws
 *   (Abbe), ws_sum = source_ws.sum(). The band support (the smallest wrapped
 *   row and column ranges holding every nonzero coefficient) is detected here.
 * litho_cache_create_band: the same kernels given only on their support, K x Nr
 *   x Nc, where band row r holds integer frequency row0 + r (mod N) and band
 *   column c holds col0 + c (mod N); row0/col0 may be negative.
 * Errors mirror imaging.cpp:68-107: K == 0, non-finite or negative weights,
 * ws_sum <= 0 give LITHO_ERR_INVALID_ARGUMENT.
 */
int litho_cache_create_dense(litho_ctx* ctx, int N, int K, const double* kernels,
                             const double* weights, double ws_sum, litho_cache** out);
int litho_cache_create_band(litho_ctx* ctx, int N, int K, int Nr, int Nc, int row0, int col0,
                            const double* kernels_band, const double* weights, double ws_sum,
                            litho_cache** out);
int litho_cache_info(const litho_cache* cache, int* N, int* K, int* Nr, int* Nc, int* row0,
                     int* col0);
int litho_cache_destroy(litho_cache* cache);

/* ------------------------------------------------------------ field
 * The band-domain electric-field state of one imaging call. It replaces
 * Imaging::get_electric_field() (include/litho_model/imaging.h:34-36): the
 * reference hands K full N x N complex fields to Gradient::pe_gradient; here
 * the exact band representation is kept and litho_field_export rebuilds E_k
 * (centred exactly like the reference's fields) when a caller needs it.
 */
int litho_field_create(litho_ctx* ctx, const litho_cache* cache, litho_field** out);
int litho_field_destroy(litho_field* field);
/* E_k as interleaved (re, im) float32, N x N row-major, device memory. */
int litho_field_export(litho_ctx* ctx, const litho_field* field, int k, float* d_E);

/* ------------------------------------------------------------ imaging
 * Imaging::compute (source/litho_model/imaging.cpp:60-171). aerial / wafer may
 * be NULL. field (may be NULL) receives the state Gradient needs.
 */
int litho_imaging_compute(litho_ctx* ctx, const litho_cache* cache, const float* d_mask,
                          double threshold, double alpha, float* d_aerial, float* d_wafer,
                          litho_field* field);

/* ------------------------------------------------------------ adjoint
 * Gradient::_backpropagate (source/utils/gradient.cpp:34-109):
 *   grad = output_scale / sum(ws) * sum_k w_k Re IFFT(conj(H_k) FFT(E_k dLdI)).
 */
int litho_backpropagate(litho_ctx* ctx, const litho_field* field, const float* d_dLdI,
                        double output_scale, float* d_grad);

/* Options shared by the pe_gradient* and pe_loss* variants
 * (source/utils/gradient.cpp:121-196, source/utils/loss.cpp:16-64):
 *   dL/dI = [pe_weight (W-T) pe_window + penalty [T<0.5] max(W - pen_thr, 0)
 *            penalty_window] W (1-W),  output_scale = 4 alpha.
 * A NULL window is all ones; a NULL penalty_window uses pe_window, as the
 * reference's single-window overloads do.
 */
typedef struct litho_pe_options {
  const float* pe_window;
  const float* penalty_window;
  double pe_weight;         /* 1.0 for Gradient::pe_gradient */
  double penalty;           /* 0.0 disables the background penalty */
  double penalty_threshold; /* 0.01 is the reference's default */
} litho_pe_options;

/* pe_gradient / pe_gradient_with_penalty (gradient.cpp:121-196). opt may be
 * NULL (plain PE). loss (host, nullable) receives the matching
 * Loss::pe_loss / pe_loss_with_penalty value. */
int litho_pe_gradient(litho_ctx* ctx, const litho_field* field, const float* d_wafer,
                      const float* d_target, const litho_pe_options* opt, double alpha,
                      float* d_grad, double* loss);

/* Loss::pe_loss / pe_loss_with_penalty (source/utils/loss.cpp:16-51). */
int litho_pe_loss(litho_ctx* ctx, const float* d_wafer, const float* d_target, int rows,
                  int cols, const litho_pe_options* opt, double* loss);

/* One CTM objective evaluation, fused (CTM_Optimizer::_evaluate_theta_objective,
 * source/optimizer/CTM_Optimizer.cpp:175-187): M = (1 + cos theta)/2, imaging,
 * PE, dPE/dM, dPE/dtheta = -1/2 dPE/dM sin theta and ||dPE/dtheta||_2.
 * Every output pointer except d_grad_theta may be NULL. */
int litho_ctm_evaluate(litho_ctx* ctx, const litho_cache* cache, litho_field* field,
                       const float* d_theta, const float* d_target, double threshold,
                       double alpha, float* d_mask, float* d_aerial, float* d_wafer,
                       float* d_grad_mask, float* d_grad_theta, double* loss,
                       double* grad_norm);

/* Same, through host buffers (copies inside): the call a CPU caller makes. */
int litho_ctm_evaluate_host(litho_ctx* ctx, const litho_cache* cache, litho_field* field,
                            const float* h_theta, const float* h_target, double threshold,
                            double alpha, float* h_grad_theta, double* loss,
                            double* grad_norm);

/* Batched CTM objective: `batch` images of the cache's size N (theta, target and
 * d_grad_theta hold them back to back, [batch][N][N]) in one pass of the chain,
 * every kernel covering all images at once, so the per-image latency of the
 * small-grid stages and of each tile's pipeline overlaps across images. losses and
 * norms (host, nullable) receive one value per image, as litho_ctm_evaluate's loss
 * and grad_norm. In LITHO_PRECISION_FP32 the images are evaluated one after another.
 * Repeated calls on the same buffers replay a CUDA graph (litho_ctx_enable_graphs). */
int litho_ctm_evaluate_batch(litho_ctx* ctx, const litho_cache* cache, int batch,
                             const float* d_theta, const float* d_target, double threshold,
                             double alpha, float* d_grad_theta, double* losses, double* norms);

/* Batched imaging + Gradient::pe_gradient (gradient.cpp:121-133) for the level-set
 * path: `batch` binary or gray masks ([batch][N][N]) through imaging, the sigmoid
 * resist and the PE loss against their targets, and dPE/dM of each into
 * d_grad_masks (the normal speed of LSM_Optimizer). losses (host, nullable): the PE
 * of each image. In LITHO_PRECISION_BF16X3 all images share one pass of the chain;
 * in LITHO_PRECISION_FP32 they are evaluated one after another. Each image's results
 * equal its own evaluation in a batch of one. */
int litho_pe_gradient_batch(litho_ctx* ctx, const litho_cache* cache, int batch,
                            const float* d_masks, const float* d_targets, double threshold,
                            double alpha, float* d_grad_masks, double* losses);

/* litho_ctm_evaluate_batch through host buffers ([batch][N][N] theta, target and
 * h_grad_theta): in LITHO_PRECISION_BF16X3 the images go through in groups whose
 * uploads, batched evaluation and downloads overlap on three streams, so the call
 * is bound by the host link rather than by the sum of copies and compute; pass
 * page-locked (pinned) host buffers, or the copies cannot overlap. In
 * LITHO_PRECISION_FP32 it calls litho_ctm_evaluate_host image after image. */
int litho_ctm_evaluate_host_batch(litho_ctx* ctx, const litho_cache* cache, int batch,
                                  const float* h_theta, const float* h_target, double threshold,
                                  double alpha, float* h_grad_theta, double* losses,
                                  double* norms);

/* ------------------------------------------------------------ sparse EPE
 * Edge points (EPs) are chosen on the host (EpSelect, source/utils/ep_select.cpp);
 * eps is n x 2 host doubles (y, x) in subpixel image coordinates, weights n host
 * doubles (points with weight <= 0 are inactive).
 * Loss::evaluate_sparse_epe (source/utils/loss.cpp:125-163): per active point the
 * bilinear samples of I and of |grad I| (LevelSetUtils::_gradient_1d, floored at
 * 1e-6) give the signed EPE (I - threshold) / |grad I| in pixels. signed_epe (host,
 * nullable, n) receives it (NaN for inactive points); totals (host, nullable, 3)
 * receives {sum w EPE^2, sum |EPE| * pixel_size_nm, active count}. */
int litho_evaluate_sparse_epe(litho_ctx* ctx, int rows, int cols, const float* d_aerial,
                              int n_eps, const double* eps, const double* weights,
                              double threshold, double pixel_size_nm, double* signed_epe,
                              double* totals);
/* Gradient::epe_gradient (source/utils/gradient.cpp:198-227): with |grad I| frozen,
 * dL/dI = 2 w (I - threshold) / |grad I|^2 scattered onto each point's bilinear
 * stencil, back-propagated with output scale 2. The scatter uses atomic adds, so
 * points whose stencils share a pixel may round differently from run to run. */
int litho_epe_gradient(litho_ctx* ctx, const litho_field* field, const float* d_aerial,
                       int n_eps, const double* eps, const double* weights, double threshold,
                       float* d_grad);

/* ------------------------------------------------------------ level set
 * LevelSetUtils::evolve_normal_WENO_godunov (source/utils/level_set_utils.cpp:150-225):
 * delta = Vn |grad phi|_Godunov with WENO5-JS one-sided derivatives and edge
 * replication. h_abs (nullable) = |Vn| (the reference's H1_abs == H2_abs).
 */
int litho_weno_godunov(litho_ctx* ctx, int rows, int cols, const float* d_phi,
                       const float* d_vn, double dy, double dx, float* d_delta, float* d_habs);
/* LevelSetUtils::evolve_kappa (level_set_utils.cpp:257-278). */
int litho_kappa(litho_ctx* ctx, int rows, int cols, const float* d_phi, double dx, double dy,
                double b, float* d_out);
/* LSM_Optimizer::_caculate_evolution_term (source/optimizer/LSM_Optimizer.cpp:47-58):
 * normal = kappa term - delta, dt = get_dt_normal_kappa (level_set_utils.cpp:280-288). */
int litho_evolution_term(litho_ctx* ctx, int rows, int cols, const float* d_phi,
                         const float* d_vn, double dx, double dy, double cfl, double b,
                         float* d_normal, double* dt);
/* LevelSetUtils::reinit_sdf (level_set_utils.cpp:290-319): signed distance
 * dist_in * dx - dist_out * dx with the 5x5 chamfer metric of OpenCV's
 * distanceTransform(DIST_L2, 5) (weights 1, 1.4, 2.1969), inside = phi > 0.
 * With no boundary in the tile the magnitude is FLT_MAX (OpenCV's no-feature
 * value). d_mask (nullable) receives the printed mask sdf >= 0 as 1/0 floats. */
int litho_reinit_sdf(litho_ctx* ctx, int rows, int cols, const float* d_phi, double dx,
                     double dy, float* d_sdf, float* d_mask);
/* Grows the context's device scratch to what the batched calls on `batch` images of
 * this cache need (the CTM / PE-gradient chain and the batched RK2 update), so that a
 * serving loop never allocates between its steps. */
int litho_ctx_reserve(litho_ctx* ctx, const litho_cache* cache, int batch);
/* Autotuner: times the candidate schedules on this device and keeps the fastest in
 * the context for the calls that follow. With a cache: the schedule of the
 * small-grid field and Z kernels for `batch` images of that cache (8 or 16 columns
 * per CTA, or 128: the whole small grid per CTA), timed on the forward and adjoint
 * band stages (results do not depend on it, bit for bit); in
 * LITHO_PRECISION_BF16X3 under LITHO_TC_SCHEDULE_AUTO also the schedule of the
 * tensor-core passes for that batch (per-tile CTAs or the persistent pipelines), timed
 * on the whole batched CTM chain (images agree bit for bit between the schedules; the
 * loss sums may differ in their last bits). With
 * nimg > 0: the CTA size (128, 256, 512 or 1024 threads) of the chamfer transform of
 * reinit_sdf for nimg images of rows x cols (the batched re-initialisations of that
 * many images use it; the result may differ from another CTA size's in the last
 * bit). Writes the choices (0: not tuned) to band_width / chamfer_threads (nullable). */
int litho_ctx_autotune(litho_ctx* ctx, const litho_cache* cache, int batch, int rows, int cols,
                       int nimg, int* band_width, int* chamfer_threads);
/* The schedules the autotuner chose for `batch` images of size N (0: not tuned):
 * band_width as litho_ctx_autotune reports it, tc_schedule a LITHO_TC_SCHEDULE_* value. */
int litho_ctx_tuned_schedule(const litho_ctx* ctx, int N, int batch, int* band_width,
                             int* tc_schedule);
/* Vector kernels of the CTM L-BFGS driver (CTM_Optimizer.cpp:189-227, LBFGS++'s
 * two-loop recursion evaluated on FP64 Gram matrices of the stored pairs).
 * litho_lbfgs_dots: out[j] = sum_i rows[j][i] v[i] accumulated in FP64 for the k
 * (1..64) float32 device rows of length n, row j at d_rows + j * ld; out is k host
 * doubles (the call waits for them). litho_lbfgs_combine: d_out[i] = cv v[i] +
 * sum_j coef[j] rows[j][i], in FP64 per element, stored float32 (coef: k host doubles,
 * k may be 0; d_out must not alias d_v). */
int litho_lbfgs_dots(litho_ctx* ctx, int k, long long n, const float* d_rows, long long ld,
                     const float* d_v, double* out);
int litho_lbfgs_combine(litho_ctx* ctx, int k, long long n, const float* d_rows, long long ld,
                        const double* coef, const float* d_v, double cv, float* d_out);
/* litho_lbfgs_dots against up to three vectors in one pass over the rows (d_v1, d_v2
 * nullable, d_v2 only with d_v1): out[v * k + j] = rows[j] . v_v, nv * k host doubles. */
int litho_lbfgs_dots3(litho_ctx* ctx, int k, long long n, const float* d_rows, long long ld,
                      const float* d_v0, const float* d_v1, const float* d_v2, double* out);
/* litho_reinit_sdf for `batch` images ([batch][rows][cols]) in one launch, inside =
 * phi > level: level 0.5 on a binary mask gives reinit_sdf(mask - 0.5), the LSM
 * initialisation (LSM_Optimizer.cpp:62), without the shifted copy. d_sdf and d_mask
 * must not alias d_phi. It only enqueues work on the context's stream (no wait). */
int litho_reinit_sdf_batch(litho_ctx* ctx, int batch, int rows, int cols, const float* d_phi,
                           double level, double dx, double dy, float* d_sdf, float* d_mask);
/* One RK2 level-set update (LSM_Optimizer.cpp:109-115, the second stage reuses
 * the first stage's dt) and the printed mask (phi >= 0) (LSM_Optimizer.cpp:128).
 * d_phi_out may alias nothing else; d_mask (nullable) receives 1/0 floats. */
int litho_lsm_rk2_update(litho_ctx* ctx, int rows, int cols, const float* d_phi,
                         const float* d_vn, double dx, double dy, double cfl, double b,
                         float* d_phi_out, float* d_mask, double* dt);
/* litho_lsm_rk2_update for `batch` images ([batch][rows][cols] phi, Vn, phi_out, mask),
 * each with its own CFL dt (dts, host, nullable: one per image); the dt of each image
 * stays on the device between its stages, so the whole batch costs one host
 * round trip. phi_out must not alias phi. */
int litho_lsm_rk2_update_batch(litho_ctx* ctx, int batch, int rows, int cols, const float* d_phi,
                               const float* d_vn, double dx, double dy, double cfl, double b,
                               float* d_phi_out, float* d_mask, double* dts);

/* ------------------------------------------------------------ device-resident serving
 * The batched calls above return their per-image scalars to the host and so wait for
 * the stream. A server that keeps many solves on the GPU uses these forms instead:
 * they only enqueue work on the context's stream, leave every result on the device and
 * report a non-finite input (or an expired tensor-core wait) through the context's
 * deferred status, read with litho_ctx_deferred_status. No counterpart in the
 * reference (its LSM_Optimizer runs one solve per call).
 *
 * litho_pe_gradient_batch_device: litho_pe_gradient_batch with d_losses (device,
 *   [batch][2] doubles) = {PE, background-penalty term at penalty_threshold}; the
 *   term adds nothing to dPE/dM (LSM_Optimizer.cpp:87-90 tracks PE + 1.0 x that term
 *   while its speed is the plain PE gradient).
 * litho_lsm_rk2_update_batch_device: litho_lsm_rk2_update_batch with d_dts (device,
 *   nullable, batch doubles).
 * litho_lsm_track_batch: the best-state bookkeeping of LSM_Optimizer.cpp:93-100 for
 *   `batch` solves: l_b = d_losses[2b] + pen_weight d_losses[2b + 1];
 *   d_history[b][d_iters[b]] = l_b (when d_history is set and the column exists),
 *   d_iters[b] += 1, and when l_b < d_best[b]: d_best[b] = l_b and image b of d_masks
 *   (n_pixels floats each) is copied to d_best_masks.
 * litho_ctx_deferred_status: waits for the stream, returns and clears the first
 *   deferred error (LITHO_OK if none). */
int litho_pe_gradient_batch_device(litho_ctx* ctx, const litho_cache* cache, int batch,
                                   const float* d_masks, const float* d_targets, double threshold,
                                   double alpha, double penalty_threshold, float* d_grad_masks,
                                   double* d_losses);
int litho_lsm_rk2_update_batch_device(litho_ctx* ctx, int batch, int rows, int cols,
                                      const float* d_phi, const float* d_vn, double dx, double dy,
                                      double cfl, double b, float* d_phi_out, float* d_mask,
                                      double* d_dts);
int litho_lsm_track_batch(litho_ctx* ctx, int batch, long long n_pixels, const double* d_losses,
                          double pen_weight, double* d_best, const float* d_masks,
                          float* d_best_masks, double* d_history, int history_cols, int* d_iters);
int litho_ctx_deferred_status(litho_ctx* ctx);

/* ------------------------------------------------------------ full chip
 * Partition (include/utils/partition.h, source/utils/partition.cpp:21-120): the
 * height x width layout is split into grid_rows x grid_cols Cores (boundaries
 * at i * height / grid_rows); each Core grows by halo pixels into a square
 * local tile of tile_size = max Core side + 2 halo, rounded up to even, read
 * with periodic wrap at the layout edge. Core + guard pixels is the update
 * window; the guard strips over the left/right/top/bottom neighbours' Cores are
 * what the micro-gradient exchange compares and fuses.
 * Local tiles live contiguously in device memory as [tile][tile_size][tile_size]
 * float32, tile id = row * grid_cols + col (PartitionMeta::tiles order).
 */
typedef struct litho_partition litho_partition;
int litho_partition_create(litho_ctx* ctx, int height, int width, int grid_rows, int grid_cols,
                           int halo, int guard, litho_partition** out);
/* The same geometry over given, possibly uneven Core boundaries (Partition::build,
 * partition.cpp:21-80, with its i * extent / count cuts replaced by the caller's):
 * row_cuts[0..grid_rows] and col_cuts[0..grid_cols] run from 0 to height / width,
 * each Core at least max(1, guard) pixels wide. As in the reference, every tile
 * takes the one tile_size = largest Core side + 2 halo (rounded up to even), so
 * smaller Cores carry a wider margin beyond their halo on the bottom / right side. */
int litho_partition_create_cuts(litho_ctx* ctx, int height, int width, int grid_rows,
                                const int* row_cuts, int grid_cols, const int* col_cuts, int halo,
                                int guard, litho_partition** out);
int litho_partition_destroy(litho_partition* partition);
int litho_partition_info(const litho_partition* partition, int* num_tiles, int* tile_size);
/* Rectangles of one tile, each (y0, y1, x0, x1) half-open: rects[0..3]
 * core_global, [4..7] tile_global, [8..11] core_local, [12..15] update_local
 * (PartitionTile, include/utils/partition.h). */
int litho_partition_tile_rects(const litho_partition* partition, int tile, int* rects);
/* Partition::extract_all (partition.cpp:83-103): global (height x width) -> tiles. */
int litho_partition_extract(litho_ctx* ctx, const litho_partition* partition,
                            const float* d_global, float* d_tiles);
/* Partition::assemble_global (partition.cpp:105-113): every tile's Core -> global. */
int litho_partition_assemble(litho_ctx* ctx, const litho_partition* partition,
                             const float* d_tiles, float* d_global);

/* MicroGradientOptions (include/utils/micro_gradient_exchange.h:19-40); the
 * reference's defaults are given beside each field. The EPE terms are in
 * litho_exchange_epe below. */
#define LITHO_MICRO_LOSS_PE 0
#define LITHO_MICRO_LOSS_PE_PENALTY 1
#define LITHO_MICRO_LOSS_EPE 2
#define LITHO_MICRO_LOSS_PE_EPE 3
#define LITHO_MICRO_REGION_CORE 0
#define LITHO_MICRO_REGION_CORE_GUARD 1
#define LITHO_FUSION_AVERAGE 0
#define LITHO_FUSION_LINEAR 1
typedef struct litho_exchange_options {
  int loss_type;                 /* LITHO_MICRO_LOSS_PE */
  int loss_region;               /* LITHO_MICRO_REGION_CORE */
  double pe_weight;              /* 1.0 */
  double penalty_weight;         /* 2.0 (PEPenalty only) */
  double penalty_threshold;      /* 0.01 */
  int enable_cept;               /* 0 */
  int cept_guard_only;           /* 0 */
  double cept_weight;            /* 1.1 */
  int enable_grad_fusion;        /* 0 */
  int fusion_mode;               /* LITHO_FUSION_AVERAGE */
  double fusion_weight_owner;    /* 0.5; fusion weights must be >= 0 with a positive sum */
  double fusion_weight_neighbor; /* 0.5 */
} litho_exchange_options;

/* MicroGradientExchange::compute (source/utils/micro_gradient_exchange.cpp:134-334)
 * for the PE loss types: per tile imaging, the windowed data loss over the loss
 * region and its raw mask gradient (phase one, tiles in sequence on the
 * context's stream), then one launch for every tile's neighbour exchange: CEPT
 * against the neighbours' Cores and Average/Linear guard-gradient fusion.
 * cache N must equal tile_size. d_masks: local masks [tile][ts][ts];
 * d_global_target: height x width; d_raw (nullable): raw per-tile gradients;
 * d_grad: exchanged gradients. tile_losses (host, nullable): 5 doubles per tile
 * {pe_loss_raw, bg_penalty_raw, data_loss, cept_loss, loss}; totals (host,
 * nullable): {loss, data_loss, cept_loss} (MicroGradientExchangeResult). */
int litho_exchange_compute(litho_ctx* ctx, const litho_partition* partition,
                           const litho_cache* cache, const float* d_masks,
                           const float* d_global_target, double threshold, double alpha,
                           const litho_exchange_options* opt, float* d_raw, float* d_grad,
                           double* tile_losses, double* totals);

/* The EPE side of MicroGradientOptions (micro_gradient_exchange.h:22-32) and the edge
 * points (EPs) it evaluates. EP selection (select_micro_epe_points, ep_select.cpp)
 * stays with the caller: eps (host, n_eps x 2) holds each selected EP's global
 * subpixel (y, x) on the layout and weights (host, n_eps) its weight_epe. */
typedef struct litho_exchange_epe {
  double epe_weight;                /* 1.0: EPE and PE_EPE */
  int main_region_dilation_pixels;  /* 2: PE_EPE, 3 x 3 dilations of target > 0.5 */
  double epe_pixel_size;            /* 1.0 nm per pixel: absolute EPE statistics only */
  int collect_core_metrics;         /* 0 */
  const double* eps;
  const double* weights;
  int n_eps;
} litho_exchange_epe;

/* Per-tile results of litho_exchange_compute_epe (MicroGradientData and its
 * CoreLossMetrics, micro_gradient_exchange.h:66-99), LITHO_EXCHANGE_TILE_METRICS
 * doubles per tile in this order. */
#define LITHO_EXCHANGE_TILE_METRICS 17
enum {
  LITHO_TM_PE_LOSS = 0,        /* unweighted PE over the PE window of the loss region */
  LITHO_TM_BG_PENALTY_RAW,     /* PEPenalty or core metrics, else 0 */
  LITHO_TM_PENALTY_LOSS,       /* penalty weight x raw background penalty (PEPenalty) */
  LITHO_TM_EPE_LOSS,           /* sum weight_epe x EPE^2 (pixel^2) over the region's EPs */
  LITHO_TM_EPE_ABS_SUM_NM,
  LITHO_TM_EPE_COUNT,
  LITHO_TM_DATA_LOSS,
  LITHO_TM_CEPT_LOSS,
  LITHO_TM_LOSS,
  LITHO_TM_CORE_PE_LOSS,       /* core metrics (collect_core_metrics), else 0 */
  LITHO_TM_CORE_BG_PENALTY_RAW,
  LITHO_TM_CORE_PE_PENALTY_LOSS,
  LITHO_TM_CORE_EPE_LOSS,
  LITHO_TM_CORE_EPE_ABS_SUM_NM,
  LITHO_TM_CORE_EP_COUNT,
  LITHO_TM_CORE_EPE_MEAN,
  LITHO_TM_CORE_DATA_LOSS
};

/* MicroGradientExchange::compute with every loss type (PE, PEPenalty, EPE,
 * PE_EPE) and the optional Core metrics. EPs of the loss region come with their
 * periodic copies when the region is Core + Guard; Core metrics use the EPs of
 * the Core alone. The EPE data gradient (Gradient::epe_gradient, gradient.cpp:198-227)
 * joins the PE gradient in one adjoint pass per tile. epe == NULL means
 * no EPs and the defaults above. tile_metrics (host, nullable):
 * LITHO_EXCHANGE_TILE_METRICS doubles per tile; totals as for litho_exchange_compute. */
int litho_exchange_compute_epe(litho_ctx* ctx, const litho_partition* partition,
                               const litho_cache* cache, const float* d_masks,
                               const float* d_global_target, double threshold, double alpha,
                               const litho_exchange_options* opt, const litho_exchange_epe* epe,
                               float* d_raw, float* d_grad, double* tile_metrics,
                               double* totals);
/* One fixed-step theta update of FullChipCTMOptimizer (source/optimizer/full_chip_ctm.cpp:127-147):
 * inside each tile's update window theta -= lr * (-1/2 grad sin theta); the
 * whole tile's mask = (1 + cos theta) / 2. d_grad == NULL only refreshes the
 * masks from theta. */
int litho_fullchip_theta_step(litho_ctx* ctx, const litho_partition* partition,
                              float* d_theta, const float* d_grad, double learning_rate,
                              float* d_masks);

/* render_levelset_mask (source/utils/levelset_mask_renderer.cpp:7-33): Binary = phi >= 0;
 * Gray = fraction of the scale x scale subpixels of each pixel with phi >= 0 after a
 * pixel-centre bilinear upsampling (edge replicated) of the float32 phi by scale. */
#define LITHO_MASK_BINARY 0
#define LITHO_MASK_GRAY 1
int litho_render_levelset_mask(litho_ctx* ctx, int rows, int cols, const float* d_phi,
                               int mask_type, int scale, float* d_mask);

/* Full-chip LSM (source/optimizer/full_chip_lsm.cpp:25-254) on a partition's tiles.
 * init (:138-146): every tile's phi = reinit_sdf(extracted initial mask - 0.5, dx, dy)
 * and its mask = render_levelset_mask(phi). step (:208-244): per tile, with the
 * exchanged mask gradient restricted to the Core + Guard window as normal speed,
 * the two-stage RK2 update (one CFL dt per tile, evolution term = curvature term -
 * WENO/Godunov term) inside the window only; with reinit set, the window is then
 * replaced by reinit_sdf of the +-0.5 sign image of phi >= 0; finally every tile's
 * mask is rendered. dt_min / dt_max (host, nullable) receive the range of the
 * tiles' steps. Tiles as for litho_exchange_compute. */
int litho_fullchip_lsm_init(litho_ctx* ctx, const litho_partition* partition,
                            const float* d_global_mask, double dx, double dy, int mask_type,
                            int scale, float* d_phi, float* d_masks);
int litho_fullchip_lsm_step(litho_ctx* ctx, const litho_partition* partition, const float* d_phi,
                            const float* d_grad, double dx, double dy, double cfl, double b,
                            int reinit, int mask_type, int scale, float* d_phi_out,
                            float* d_masks, double* dt_min, double* dt_max);

/* ------------------------------------------------------------ no-allocation variant
 * litho_lsm_rk2_update_noalloc: the RK2 level-set update of litho_lsm_rk2_update
 * (same kernels, same results) for callers that must not allocate device
 * memory at call time, e.g. a service whose device memory budget is fully
 * reserved up front, or code interleaved with other streams' work where a
 * cudaMalloc would implicitly synchronise the device. It takes a plain
 * cudaStream_t (NULL = default stream) instead of a litho_ctx and never calls
 * cudaMalloc/cudaFree: its scratch (the first RK2 stage and the dt reduction)
 * is one static device array of 2048 * 2048 + 512 floats (about 16 MiB) per
 * device, so rows * cols must not exceed LITHO_RK2_NOALLOC_MAX_PIXELS; larger
 * grids return LITHO_ERR_UNSUPPORTED without launching anything (use
 * litho_lsm_rk2_update for them). Nothing has to be zero beforehand: each call
 * clears the non-finite flag it uses. The first call on each device looks up
 * the scratch address (cudaGetSymbolAddress) and loads the module. Every call
 * copies dt and the flag back and waits on its stream, so it must never be
 * called while that stream is being captured into a CUDA graph (the wait
 * would invalidate the capture). The calling thread's current device must be
 * the stream's device. Calls share the one scratch array per device, so two
 * calls that overlap in time (different host threads or streams) race:
 * serialise them. dt (host, nullable) receives the step used.
 * Status as litho_lsm_rk2_update; LITHO_ERR_NONFINITE for non-finite Vn.
 * This entry point has no counterpart in the reference.
 */
#define LITHO_RK2_NOALLOC_MAX_PIXELS (2048 * 2048)
int litho_lsm_rk2_update_noalloc(void* stream, int rows, int cols, const float* d_phi,
                                 const float* d_vn, double dx, double dy, double cfl, double b,
                                 float* d_phi_out, float* d_mask, double* dt);

#ifdef __cplusplus
}
#endif

#endif /* LITHO_B200_H */
