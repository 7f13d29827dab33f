// C ABI of the imaging-and-gradient library: contexts, optical caches, fields
// and the entry points declared in include/litho_b200.h. Host-side
// orchestration of the band-DFT kernels (band_dft.cu) and the level-set
// kernels (levelset.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "litho_internal.cuh"

using namespace litho_b200;

namespace {

constexpr double kTwoPi = 6.283185307179586476925286766559;

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }
int round16(int v) { return (v + 15) / 16 * 16; }

// e^{sign 2 pi i (f * j mod P) / P}, exact integer phase reduction in FP64.
void twiddle(long long f, long long j, long long P, double sign, double* re, double* im) {
  long long p = ((f % P) + P) % P;
  p = (p * (j % P)) % P;
  const double a = sign * kTwoPi * (double)p / (double)P;
  *re = std::cos(a);
  *im = std::sin(a);
}

template <class T>
int upload(Context* ctx, T** dst, const std::vector<T>& src) {
  if (cudaMalloc(reinterpret_cast<void**>(dst), src.size() * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    return ctx->fail(LITHO_ERR_OOM, "device allocation of an optical table failed");
  }
  if (cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice) !=
      cudaSuccess)
    return ctx->fail(LITHO_ERR_CUDA, "upload of an optical table failed");
  return LITHO_OK;
}

void free_cache(Cache* c) {
  void* ptrs[] = {c->H,     c->w,       c->TXS,     c->TXD,     c->TYS,     c->TYD,
                  c->AYS,   c->AYD,     c->TXSc,    c->TXDc,    c->ESr_t,   c->ESc_t,
                  c->ESc,   c->EDr_t,   c->EDc_t,   c->EDc,     c->AYS_img, c->AYD_img,
                  c->TXS_img, c->TXD_img, c->TYS_img, c->TYD_img};
  for (void* p : ptrs)
    if (p) cudaFree(p);
}

// Scratch layout of one imaging + adjoint evaluation.
struct Layout {
  size_t part, gh, ik, iP, chat, X, Ut, Vt, dldi, gam, Zk, rows_tmp, img, fm, fe, total;
  int tiles;
};

// batch > 1 (the batched CTM evaluation): every per-image buffer repeated batch times
// back to back, plus the band state of the batch (fm: m on the band, fe: the K
// small-grid fields per image).
Layout make_layout(const BandGeom& g, int batch = 1, bool own_field = false) {
  Layout L{};
  const size_t B = (size_t)batch;
  const int N = g.N;
  L.tiles = analysis_tiles(N);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = align_up(off + bytes, 256);
    return o;
  };
  L.part = take(B * L.tiles * (2 * g.Nr - 1) * g.Nc * sizeof(float2));
  L.gh = take(B * (2 * g.Nr - 1) * g.Nc * sizeof(float2));
  L.ik = take(B * g.K * g.Pr * g.Pc * sizeof(float));
  L.iP = take(B * g.Pr * g.Pc * sizeof(float));
  L.Ut = take(B * N * g.kp_rows * sizeof(float));
  L.Vt = take(B * N * g.kp_rows * sizeof(float));
  L.dldi = take((size_t)N * N * sizeof(float));
  L.gam = take(B * g.Pr * g.Pc * sizeof(float));
  L.Zk = take(B * g.K * g.Nr * g.Nc * sizeof(float2));
  L.chat = take(B * g.Nr * (2 * g.Nc - 1) * sizeof(float2));
  L.X = take(B * g.Nr * g.Nc * sizeof(float2));
  L.rows_tmp = take((size_t)g.Nr * N * sizeof(float2));
  L.img = take(B * (tc2_supported(g) ? tc2_rows_image_bytes(N, g.kp_rows) : 16));  // band operand images
  const bool field = batch > 1 || own_field;
  L.fm = field ? take(B * g.Nr * g.Nc * sizeof(float2)) : 0;
  L.fe = field ? take(B * g.K * g.Pr * g.Pc * sizeof(float2)) : 0;
  L.total = off;
  return L;
}

template <class T>
T* at(const Context* ctx, size_t off) {
  return reinterpret_cast<T*>(static_cast<char*>(ctx->scratch.base) + off);
}

bool finite_all(const double* p, size_t n) {
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(p[i])) return false;
  return true;
}

// Reduction slots in ctx->d_red: [0] flag (as int), partial sums after 8.
constexpr int RED_FLAG = 0;
constexpr int RED_SUM = 2;    // summed results (up to 4 doubles)
constexpr int RED_PART = 8;   // per-block partials

}  // namespace

int Context::ensure_scratch(size_t bytes) {
  if (scratch.bytes >= bytes) return LITHO_OK;
  if (scratch.base) {
    cudaStreamSynchronize(stream);
    cudaFree(scratch.base);
    scratch.base = nullptr;
    scratch.bytes = 0;
  }
  if (cudaMalloc(&scratch.base, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(LITHO_ERR_OOM, "scratch allocation of " + std::to_string(bytes) + " bytes failed");
  }
  scratch.bytes = bytes;
  return LITHO_OK;
}

int Context::ensure_deferred() {
  if (d_deferred) return LITHO_OK;
  if (cudaMalloc(&d_deferred, 2 * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    d_deferred = nullptr;
    return fail(LITHO_ERR_OOM, "deferred status allocation failed");
  }
  if (cudaMemsetAsync(d_deferred, 0, 2 * sizeof(int), stream) != cudaSuccess)
    return fail(LITHO_ERR_CUDA, "deferred status");
  return LITHO_OK;
}

int Context::ensure_red(size_t n) {
  if (red_cap >= n) return LITHO_OK;
  if (d_red) {
    cudaStreamSynchronize(stream);
    cudaFree(d_red);
    d_red = nullptr;
  }
  if (cudaMalloc(&d_red, n * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    red_cap = 0;
    return fail(LITHO_ERR_OOM, "reduction buffer allocation failed");
  }
  red_cap = n;
  return LITHO_OK;
}

void Context::collect_stages() {
  for (int i = 0; i < LITHO_NUM_STAGES; ++i) {
    if (!ev_pending[i]) continue;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ev[i][0], ev[i][1]) == cudaSuccess) {
      stage_ms[i] += ms;
      stage_count[i] += 1;
    } else {
      cudaGetLastError();
    }
    ev_pending[i] = false;
  }
}

// ============================================================== ABI
extern "C" {

int litho_version(void) { return 1; }

const char* litho_status_string(int s) {
  switch (s) {
    case LITHO_OK: return "ok";
    case LITHO_ERR_INVALID_ARGUMENT: return "invalid argument";
    case LITHO_ERR_SHAPE: return "shape mismatch";
    case LITHO_ERR_NONFINITE: return "non-finite input";
    case LITHO_ERR_OOM: return "out of device memory";
    case LITHO_ERR_CUDA: return "CUDA error";
    case LITHO_ERR_NOT_READY: return "field not computed";
    case LITHO_ERR_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
  }
}

const char* litho_ctx_last_error(const litho_ctx* ctx) {
  return ctx ? ctx->last_error.c_str() : "null context";
}

int litho_ctx_create(int device, void* stream, litho_ctx** out) {
  if (!out) return LITHO_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return LITHO_ERR_CUDA;
  }
  if (cudaSetDevice(device) != cudaSuccess) return LITHO_ERR_CUDA;
  litho_ctx* c = new (std::nothrow) litho_ctx();
  if (!c) return LITHO_ERR_OOM;
  c->device = device;
  if (stream) {
    c->stream = static_cast<cudaStream_t>(stream);
  } else {
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete c;
      return LITHO_ERR_CUDA;
    }
    c->own_stream = true;
  }
  if (cudaMallocHost(reinterpret_cast<void**>(&c->h_red), 64 * sizeof(double)) != cudaSuccess) {
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    return LITHO_ERR_OOM;
  }
  *out = c;
  return LITHO_OK;
}

int litho_ctx_destroy(litho_ctx* ctx) {
  if (!ctx) return LITHO_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->scratch.base) cudaFree(ctx->scratch.base);
  if (ctx->d_red) cudaFree(ctx->d_red);
  if (ctx->d_deferred) cudaFree(ctx->d_deferred);
  if (ctx->h_red) cudaFreeHost(ctx->h_red);
  if (ctx->host_stage.base) cudaFree(ctx->host_stage.base);
  if (ctx->eval_graph) cudaGraphExecDestroy(ctx->eval_graph);
  if (ctx->batch_graph) cudaGraphExecDestroy(ctx->batch_graph);
  for (cudaEvent_t e : ctx->ev_aux)
    if (e) cudaEventDestroy(e);
  if (ctx->aux) cudaStreamDestroy(ctx->aux);
  if (ctx->pipe_stage.base) cudaFree(ctx->pipe_stage.base);
  for (auto& slot : ctx->ev_pipe)
    for (cudaEvent_t e : slot)
      if (e) cudaEventDestroy(e);
  if (ctx->dn) cudaStreamDestroy(ctx->dn);
  for (int i = 0; i < LITHO_NUM_STAGES; ++i)
    for (int j = 0; j < 2; ++j)
      if (ctx->ev[i][j]) cudaEventDestroy(ctx->ev[i][j]);
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return LITHO_OK;
}

int litho_ctx_synchronize(litho_ctx* ctx) {
  if (!ctx) return LITHO_ERR_INVALID_ARGUMENT;
  LITHO_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return LITHO_OK;
}

int litho_ctx_set_precision(litho_ctx* ctx, int precision) {
  if (!ctx) return LITHO_ERR_INVALID_ARGUMENT;
  if (precision != LITHO_PRECISION_FP32 && precision != LITHO_PRECISION_BF16X3)
    return ctx->fail(LITHO_ERR_UNSUPPORTED, "precision mode not built");
  ctx->precision = precision;
  return LITHO_OK;
}

long long litho_ctx_launch_count(const litho_ctx* ctx) { return ctx ? ctx->launches : 0; }

int litho_ctx_enable_graphs(litho_ctx* ctx, int on) {
  if (!ctx) return LITHO_ERR_INVALID_ARGUMENT;
  ctx->graphs = on != 0;
  ctx->eval_last_valid = false;
  ctx->batch_last_valid = false;
  if (!ctx->graphs && (ctx->eval_graph || ctx->batch_graph)) {
    cudaStreamSynchronize(ctx->stream);
    if (ctx->eval_graph) cudaGraphExecDestroy(ctx->eval_graph);
    if (ctx->batch_graph) cudaGraphExecDestroy(ctx->batch_graph);
    ctx->eval_graph = nullptr;
    ctx->batch_graph = nullptr;
  }
  return LITHO_OK;
}

int litho_ctx_tuned_schedule(const litho_ctx* ctx, int N, int batch, int* band_width,
                             int* tc_schedule) {
  if (!ctx) return LITHO_ERR_INVALID_ARGUMENT;
  if (band_width) *band_width = ctx->band_width(N, batch);
  if (tc_schedule) {
    const auto it = ctx->tuned_tc.find({N, batch});
    *tc_schedule = it == ctx->tuned_tc.end() ? 0 : it->second;
  }
  return LITHO_OK;
}

int litho_ctx_set_exchange_group(litho_ctx* ctx, int max_tiles) {
  if (!ctx || max_tiles < 0) return LITHO_ERR_INVALID_ARGUMENT;
  ctx->exchange_group_max = max_tiles;
  return LITHO_OK;
}

int litho_ctx_set_tc_schedule(litho_ctx* ctx, int schedule) {
  if (!ctx) return LITHO_ERR_INVALID_ARGUMENT;
  if (schedule != LITHO_TC_SCHEDULE_AUTO && schedule != LITHO_TC_SCHEDULE_PER_TILE &&
      schedule != LITHO_TC_SCHEDULE_PERSISTENT)
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "unknown tensor-core schedule");
  ctx->tc_schedule = schedule;
  return LITHO_OK;
}

int litho_ctx_enable_stage_timing(litho_ctx* ctx, int on) {
  if (!ctx) return LITHO_ERR_INVALID_ARGUMENT;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return LITHO_ERR_CUDA;
  if (on && !ctx->ev[0][0]) {
    for (int i = 0; i < LITHO_NUM_STAGES; ++i)
      for (int j = 0; j < 2; ++j)
        if (cudaEventCreate(&ctx->ev[i][j]) != cudaSuccess)
          return ctx->fail(LITHO_ERR_CUDA, "cudaEventCreate failed");
  }
  ctx->timing = on != 0;
  for (int i = 0; i < LITHO_NUM_STAGES; ++i) {
    ctx->stage_ms[i] = 0.0;
    ctx->stage_count[i] = 0;
    ctx->ev_pending[i] = false;
  }
  return LITHO_OK;
}

int litho_ctx_stage_times(const litho_ctx* ctx, double* ms, long long* counts) {
  if (!ctx) return LITHO_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < LITHO_NUM_STAGES; ++i) {
    if (ms) ms[i] = ctx->stage_ms[i];
    if (counts) counts[i] = ctx->stage_count[i];
  }
  return LITHO_OK;
}

// ---------------------------------------------------------------- cache
int litho_cache_create_band(litho_ctx* ctx, int N, int K, int Nr, int Nc, int row0, int col0,
                            const double* kb, const double* weights, double ws_sum,
                            litho_cache** out) {
  if (!ctx || !out) return LITHO_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (N <= 0) return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "Imaging: cache.N must be positive");
  if (K <= 0 || !kb || !weights)
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "Imaging: no optical kernels available");
  if (Nr <= 0 || Nc <= 0 || Nr > N || Nc > N)
    return ctx->fail(LITHO_ERR_SHAPE, "band size must be within 1..N");
  if (!std::isfinite(ws_sum) || ws_sum <= 0.0)
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT,
                     "Imaging: source weights must be finite, nonnegative, and have a positive sum");
  for (int k = 0; k < K; ++k)
    if (!std::isfinite(weights[k]) || weights[k] < 0.0)
      return ctx->fail(LITHO_ERR_INVALID_ARGUMENT,
                       "Imaging: SOCS values must be finite and nonnegative");
  if (!finite_all(kb, (size_t)K * Nr * Nc * 2))
    return ctx->fail(LITHO_ERR_NONFINITE, "optical kernels must be finite");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return LITHO_ERR_CUDA;

  litho_cache* c = new (std::nothrow) litho_cache();
  if (!c) return LITHO_ERR_OOM;
  c->device = ctx->device;
  BandGeom& g = c->g;
  g.N = N; g.K = K; g.Nr = Nr; g.Nc = Nc; g.row0 = row0; g.col0 = col0;
  g.Pr = 2 * Nr; g.Pc = 2 * Nc;
  g.kp_rows = round16(2 * Nr);
  g.kp_cols = 2 * Nc;

  std::vector<float2> H((size_t)K * Nr * Nc);
  for (size_t i = 0; i < H.size(); ++i) H[i] = make_float2((float)kb[2 * i], (float)kb[2 * i + 1]);
  c->w_host.resize(K);
  std::vector<float> w(K);
  for (int k = 0; k < K; ++k) {
    c->w_host[k] = weights[k] / ws_sum;
    w[k] = (float)c->w_host[k];
  }
  double re, im;
  std::vector<float> TXS((size_t)2 * Nc * N), TXD((size_t)2 * Nc * N);
  std::vector<float2> TXSc((size_t)Nc * N), TXDc((size_t)Nc * N);
  for (int cidx = 0; cidx < Nc; ++cidx)
    for (int x = 0; x < N; ++x) {
      twiddle(col0 + cidx, x, N, -1.0, &re, &im);
      TXS[(size_t)(2 * cidx) * N + x] = (float)re;
      TXS[(size_t)(2 * cidx + 1) * N + x] = (float)im;
      TXSc[(size_t)cidx * N + x] = make_float2((float)re, (float)im);
      twiddle(cidx, x, N, -1.0, &re, &im);
      TXD[(size_t)(2 * cidx) * N + x] = (float)re;
      TXD[(size_t)(2 * cidx + 1) * N + x] = (float)im;
      TXDc[(size_t)cidx * N + x] = make_float2((float)re, (float)im);
    }
  std::vector<float2> TYS((size_t)Nr * N), TYD((size_t)Nr * N);
  std::vector<float> AYS((size_t)N * g.kp_rows, 0.f), AYD((size_t)N * g.kp_rows, 0.f);
  for (int r = 0; r < Nr; ++r)
    for (int y = 0; y < N; ++y) {
      twiddle(row0 + r, y, N, -1.0, &re, &im);
      TYS[(size_t)r * N + y] = make_float2((float)re, (float)im);
      AYS[(size_t)y * g.kp_rows + 2 * r] = (float)re;
      AYS[(size_t)y * g.kp_rows + 2 * r + 1] = (float)im;
      twiddle(r, y, N, -1.0, &re, &im);
      TYD[(size_t)r * N + y] = make_float2((float)re, (float)im);
      AYD[(size_t)y * g.kp_rows + 2 * r] = (float)re;
      AYD[(size_t)y * g.kp_rows + 2 * r + 1] = (float)im;
    }
  std::vector<float2> ESr_t((size_t)Nr * g.Pr), ESc_t((size_t)Nc * g.Pc), ESc((size_t)g.Pc * Nc);
  std::vector<float2> EDr_t((size_t)(2 * Nr - 1) * g.Pr), EDc_t((size_t)(2 * Nc - 1) * g.Pc);
  std::vector<float2> EDc((size_t)g.Pc * (2 * Nc - 1));
  for (int r = 0; r < Nr; ++r)
    for (int j = 0; j < g.Pr; ++j) {
      twiddle(row0 + r, j, g.Pr, 1.0, &re, &im);
      ESr_t[(size_t)r * g.Pr + j] = make_float2((float)re, (float)im);
    }
  for (int cidx = 0; cidx < Nc; ++cidx)
    for (int j = 0; j < g.Pc; ++j) {
      twiddle(col0 + cidx, j, g.Pc, 1.0, &re, &im);
      ESc_t[(size_t)cidx * g.Pc + j] = make_float2((float)re, (float)im);
      ESc[(size_t)j * Nc + cidx] = make_float2((float)re, (float)im);
    }
  for (int a = 0; a < 2 * Nr - 1; ++a)
    for (int j = 0; j < g.Pr; ++j) {
      twiddle(a - (Nr - 1), j, g.Pr, 1.0, &re, &im);
      EDr_t[(size_t)a * g.Pr + j] = make_float2((float)re, (float)im);
    }
  for (int a = 0; a < 2 * Nc - 1; ++a)
    for (int j = 0; j < g.Pc; ++j) {
      twiddle(a - (Nc - 1), j, g.Pc, 1.0, &re, &im);
      EDc_t[(size_t)a * g.Pc + j] = make_float2((float)re, (float)im);
      EDc[(size_t)j * (2 * Nc - 1) + a] = make_float2((float)re, (float)im);
    }
  // The per-kernel CTAs of the small-grid stage keep a band (and a band-by-grid
  // product) in shared memory; larger bands are not built.
  if (band_max_smem(g) > 220 * 1024) {
    delete c;
    return ctx->fail(LITHO_ERR_UNSUPPORTED,
                     "kernel band too large for the small-grid kernels' shared memory "
                     "(supported up to about 70 x 70 frequencies)");
  }
  int st = LITHO_OK;
  if (st == LITHO_OK) st = upload(ctx, &c->H, H);
  if (st == LITHO_OK) st = upload(ctx, &c->w, w);
  if (st == LITHO_OK) st = upload(ctx, &c->TXS, TXS);
  if (st == LITHO_OK) st = upload(ctx, &c->TXD, TXD);
  if (st == LITHO_OK) st = upload(ctx, &c->TXSc, TXSc);
  if (st == LITHO_OK) st = upload(ctx, &c->TXDc, TXDc);
  if (st == LITHO_OK) st = upload(ctx, &c->TYS, TYS);
  if (st == LITHO_OK) st = upload(ctx, &c->TYD, TYD);
  if (st == LITHO_OK) st = upload(ctx, &c->AYS, AYS);
  if (st == LITHO_OK) st = upload(ctx, &c->AYD, AYD);
  if (st == LITHO_OK) st = upload(ctx, &c->ESr_t, ESr_t);
  if (st == LITHO_OK) st = upload(ctx, &c->ESc_t, ESc_t);
  if (st == LITHO_OK) st = upload(ctx, &c->ESc, ESc);
  if (st == LITHO_OK) st = upload(ctx, &c->EDr_t, EDr_t);
  if (st == LITHO_OK) st = upload(ctx, &c->EDc_t, EDc_t);
  if (st == LITHO_OK) st = upload(ctx, &c->EDc, EDc);
  // Split-BF16 images of the twiddle tables for the tensor-core passes.
  if (tc2_supported(g)) {
    struct ImageJob {
      void** dst;
      size_t bytes;
      int what;
    } jobs[] = {{&c->TXS_img, tc2_tx_image_bytes(N, Nc), 0}, {&c->TXD_img, tc2_tx_image_bytes(N, Nc), 1},
                {&c->TYS_img, tc2_ty_image_bytes(N), 2},     {&c->TYD_img, tc2_ty_image_bytes(N), 3},
                {&c->AYS_img, tc2_rows_image_bytes(N, g.kp_rows), 4},
                {&c->AYD_img, tc2_rows_image_bytes(N, g.kp_rows), 5}};
    for (const ImageJob& j : jobs) {
      if (st != LITHO_OK) break;
      if (cudaMalloc(j.dst, j.bytes) != cudaSuccess) {
        cudaGetLastError();
        st = ctx->fail(LITHO_ERR_OOM, "tensor-core operand image allocation failed");
        break;
      }
      cudaError_t e;
      switch (j.what) {
        case 0: e = launch_pack_tc2_tx(ctx->stream, c->TXS, Nc, N, *j.dst); break;
        case 1: e = launch_pack_tc2_tx(ctx->stream, c->TXD, Nc, N, *j.dst); break;
        case 2: e = launch_pack_tc2_ty(ctx->stream, c->TYS, Nr, N, *j.dst); break;
        case 3: e = launch_pack_tc2_ty(ctx->stream, c->TYD, Nr, N, *j.dst); break;
        case 4: e = launch_pack_tc2_rows(ctx->stream, c->AYS, N, g.kp_rows, *j.dst); break;
        default: e = launch_pack_tc2_rows(ctx->stream, c->AYD, N, g.kp_rows, *j.dst); break;
      }
      if (e != cudaSuccess || cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        st = ctx->fail(LITHO_ERR_CUDA, "tensor-core operand packing failed");
    }
  }
  if (st != LITHO_OK) {
    free_cache(c);
    delete c;
    return st;
  }
  *out = c;
  return LITHO_OK;
}

// Smallest wrapped range of indices holding every flagged entry: the
// complement of the longest circular run of unflagged entries.
static void wrapped_range(const std::vector<char>& nz, int N, int* start, int* len) {
  int best = 0, best_end = -1, run = 0;
  for (int j = 0; j < 2 * N; ++j) {
    if (!nz[j % N]) {
      ++run;
      if (run > best && run < N) { best = run; best_end = j; }
    } else {
      run = 0;
    }
  }
  if (best == 0) {  // every index used
    *start = -(N / 2);
    *len = N;
    return;
  }
  int s = (best_end + 1) % N;
  *len = N - best;
  *start = s <= N / 2 ? s : s - N;
}

int litho_cache_create_dense(litho_ctx* ctx, int N, int K, const double* kernels,
                             const double* weights, double ws_sum, litho_cache** out) {
  if (!ctx || !out) return LITHO_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (N <= 0) return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "Imaging: cache.N must be positive");
  if (K <= 0 || !kernels)
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "Imaging: no optical kernels available");
  const size_t nn = (size_t)N * N;
  if (!finite_all(kernels, (size_t)K * nn * 2))
    return ctx->fail(LITHO_ERR_NONFINITE, "optical kernels must be finite");
  // Coefficients below 1e-12 of the largest magnitude (SVD round-off outside the
  // pupil support) are treated as zero; float32 cannot resolve them anyway.
  double amax = 0.0;
  for (size_t i = 0; i < (size_t)K * nn; ++i)
    amax = std::max(amax, std::hypot(kernels[2 * i], kernels[2 * i + 1]));
  const double tol = amax * 1e-12;
  std::vector<char> nzr(N, 0), nzc(N, 0);
  for (int k = 0; k < K; ++k)
    for (int r = 0; r < N; ++r)
      for (int cc = 0; cc < N; ++cc) {
        const size_t i = ((size_t)k * N + r) * N + cc;
        if (std::hypot(kernels[2 * i], kernels[2 * i + 1]) > tol) { nzr[r] = 1; nzc[cc] = 1; }
      }
  int row0, Nr, col0, Nc;
  wrapped_range(nzr, N, &row0, &Nr);
  wrapped_range(nzc, N, &col0, &Nc);
  if (Nr == 0 || Nc == 0) { row0 = 0; Nr = 1; col0 = 0; Nc = 1; }
  std::vector<double> band((size_t)K * Nr * Nc * 2);
  for (int k = 0; k < K; ++k)
    for (int r = 0; r < Nr; ++r)
      for (int cc = 0; cc < Nc; ++cc) {
        const int R = ((row0 + r) % N + N) % N, C = ((col0 + cc) % N + N) % N;
        const size_t src = ((size_t)k * N + R) * N + C;
        const size_t dst = ((size_t)k * Nr + r) * Nc + cc;
        band[2 * dst] = kernels[2 * src];
        band[2 * dst + 1] = kernels[2 * src + 1];
      }
  return litho_cache_create_band(ctx, N, K, Nr, Nc, row0, col0, band.data(), weights, ws_sum,
                                 out);
}

int litho_cache_info(const litho_cache* c, int* N, int* K, int* Nr, int* Nc, int* row0,
                     int* col0) {
  if (!c) return LITHO_ERR_INVALID_ARGUMENT;
  if (N) *N = c->g.N;
  if (K) *K = c->g.K;
  if (Nr) *Nr = c->g.Nr;
  if (Nc) *Nc = c->g.Nc;
  if (row0) *row0 = c->g.row0;
  if (col0) *col0 = c->g.col0;
  return LITHO_OK;
}

int litho_cache_destroy(litho_cache* c) {
  if (!c) return LITHO_OK;
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  free_cache(c);
  delete c;
  return LITHO_OK;
}

// ---------------------------------------------------------------- field
int litho_field_create(litho_ctx* ctx, const litho_cache* cache, litho_field** out) {
  if (!ctx || !cache || !out) return LITHO_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  litho_field* f = new (std::nothrow) litho_field();
  if (!f) return LITHO_ERR_OOM;
  f->cache = cache;
  const BandGeom& g = cache->g;
  if (cudaMalloc(&f->mband, (size_t)g.Nr * g.Nc * sizeof(float2)) != cudaSuccess ||
      cudaMalloc(&f->e, (size_t)g.K * g.Pr * g.Pc * sizeof(float2)) != cudaSuccess) {
    cudaGetLastError();
    if (f->mband) cudaFree(f->mband);
    delete f;
    return ctx->fail(LITHO_ERR_OOM, "field allocation failed");
  }
  *out = f;
  return LITHO_OK;
}

int litho_field_destroy(litho_field* f) {
  if (!f) return LITHO_OK;
  cudaDeviceSynchronize();
  if (f->mband) cudaFree(f->mband);
  if (f->e) cudaFree(f->e);
  delete f;
  return LITHO_OK;
}

}  // extern "C"

// ============================================================== orchestration
namespace {

int check_launch(Context* ctx, cudaError_t e, const char* what) {
  if (e != cudaSuccess) return ctx->fail(LITHO_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return LITHO_OK;
}

// Forward: tile analysis -> tile reduction -> small-grid band stage -> row
// synthesis with the fused resist epilogue. input_mode 1 reads theta. With
// fuse_adjoint (tensor-core path, ep.mode 1) the synthesis also runs the adjoint
// tile analysis of dL/dI, leaving its tile partials in L.part for run_adjoint
// with analysed set; dL/dI is then not stored.
int run_forward(Context* ctx, const Cache& c, Field& f, const Layout& L, int input_mode,
                const float* input, float* mask_out, ResistEpilogue ep, int* nblocks,
                cudaEvent_t before_synthesis = nullptr, bool fuse_adjoint = false,
                int batch = 1) {
  const BandGeom& g = c.g;
  cudaStream_t s = ctx->stream;
  int* flag = reinterpret_cast<int*>(ctx->d_red + RED_FLAG);
  int st;
  ctx->stage_begin(0);
  const bool tc = ctx->precision == LITHO_PRECISION_BF16X3 && c.TXS_img;
  const bool pers = tc && ctx->tc_persistent(g.N, batch);
  const bool fwd_tc3 = tc && pers && tc3_analysis_supported(g.Nc, g.Nr);
  ctx->fwd_part_trows = fwd_tc3 ? g.Nr : 0;   // the persistent analysis stores [c][row]
  if (fwd_tc3)
    st = check_launch(ctx, launch_analysis_tc3(s, input_mode, input, mask_out, flag, g.N, g.Nc,
                                               g.Nr, g.Nr, 0, at<float2>(ctx, L.part), c.TXS_img,
                                               c.TYS_img, flag + 1, batch),
                      "tensor-core tile analysis (persistent)");
  else if (tc)
    st = check_launch(ctx, launch_analysis_tc2(s, input_mode, input, mask_out, flag, g.N, g.Nc,
                                               g.Nr, g.Nr, 0, at<float2>(ctx, L.part), c.TXS_img,
                                               c.TYS_img, flag + 1, batch),
                      "tensor-core tile analysis");
  else
    st = check_launch(ctx, launch_analysis(s, input_mode, input, mask_out, flag, c.TXS, g.N, g.Nc,
                                           c.TYS, g.Nr, g.Nr, 0, at<float2>(ctx, L.part)),
                      "tile analysis");
  ctx->stage_end(0);
  if (st) return st;
  ctx->stage_begin(1);
  st = check_launch(ctx, launch_reduce_tiles(s, at<float2>(ctx, L.part), L.tiles, g.Nr * g.Nc,
                                             1.f / ((float)g.N * g.N), f.mband, batch,
                                             ctx->fwd_part_trows),
                    "tile reduction");
  ctx->stage_end(1);
  if (st) return st;
  ctx->stage_begin(2);
  st = check_launch(ctx, launch_band_forward(s, c, f, at<float>(ctx, L.ik), at<float>(ctx, L.iP),
                                             at<float2>(ctx, L.chat), at<float>(ctx, L.Ut),
                                             tc ? at<void>(ctx, L.img) : nullptr, batch,
                                             ctx->band_width(g.N, batch)),
                    "band forward");
  ctx->stage_end(2);
  if (st) return st;
  // The epilogue's inputs may still be arriving on another stream.
  if (before_synthesis) LITHO_CUDA_TRY(ctx, cudaStreamWaitEvent(s, before_synthesis, 0));
  ctx->stage_begin(3);
  if (tc) {
    int* err = reinterpret_cast<int*>(ctx->d_red + RED_FLAG) + 1;
    const bool fused_tc3 = fuse_adjoint && pers && tc3_fused_supported(g.kp_rows, g.Nc, g.Nr);
    if (fuse_adjoint) ctx->adj_part_trows = fused_tc3 ? 2 * g.Nr - 1 : 0;
    if (fused_tc3)
      st = check_launch(ctx, launch_synth_resist_analysis_tc3(
                                 s, c.AYD_img, at<void>(ctx, L.img), g.N, g.kp_rows, ep, g.Nc,
                                 g.Nr, at<float2>(ctx, L.part), flag, c.TXD_img, c.TYD_img, err,
                                 nblocks, batch),
                        "tensor-core row synthesis with adjoint tile analysis (persistent)");
    else if (fuse_adjoint)
      st = check_launch(ctx, launch_synth_resist_analysis_tc2(
                                 s, c.AYD_img, at<void>(ctx, L.img), g.N, g.kp_rows, ep, g.Nc,
                                 g.Nr, at<float2>(ctx, L.part), flag, c.TXD_img, c.TYD_img, err,
                                 nblocks, batch),
                        "tensor-core row synthesis with adjoint tile analysis");
    else if (pers && tc3_synth_supported(g.kp_rows))
      st = check_launch(ctx, launch_synth_resist_tc3(s, c.AYD_img, at<void>(ctx, L.img), g.N,
                                                     g.kp_rows, ep, err, nblocks, batch),
                        "tensor-core row synthesis (persistent)");
    else
      st = check_launch(ctx, launch_synth_resist_tc2(s, c.AYD_img, at<void>(ctx, L.img), g.N,
                                                     g.kp_rows, ep, err, nblocks, batch),
                        "tensor-core row synthesis");
  } else {
    st = check_launch(ctx, launch_synth_resist(s, c.AYD, at<float>(ctx, L.Ut), g.N, g.kp_rows, ep,
                                               nblocks),
                      "row synthesis");
  }
  ctx->stage_end(3);
  ctx->launches += 7;  // analysis, reduction, fields, sum over k, chat, expansion, synthesis
  f.valid = (st == LITHO_OK);
  return st;
}

int run_adjoint(Context* ctx, const Cache& c, const Field& f, const Layout& L, const float* dldi,
                double scale, GradEpilogue ep, int* nblocks, bool analysed = false,
                int batch = 1) {
  const BandGeom& g = c.g;
  cudaStream_t s = ctx->stream;
  int* flag = reinterpret_cast<int*>(ctx->d_red + RED_FLAG);
  const int na = 2 * g.Nr - 1;
  int st;
  ctx->stage_begin(4);
  const bool tc = ctx->precision == LITHO_PRECISION_BF16X3 && c.TXD_img;
  const bool pers = tc && ctx->tc_persistent(g.N, batch);
  if (!analysed) ctx->adj_part_trows = tc && pers && tc3_analysis_supported(g.Nc, g.Nr) ? na : 0;
  if (analysed)
    st = LITHO_OK;  // the partials are already in L.part
  else if (tc && pers && tc3_analysis_supported(g.Nc, g.Nr))
    st = check_launch(ctx, launch_analysis_tc3(s, 0, dldi, nullptr, flag, g.N, g.Nc, na, g.Nr, 1,
                                               at<float2>(ctx, L.part), c.TXD_img, c.TYD_img,
                                               flag + 1, batch),
                      "tensor-core adjoint tile analysis (persistent)");
  else if (tc)
    st = check_launch(ctx, launch_analysis_tc2(s, 0, dldi, nullptr, flag, g.N, g.Nc, na, g.Nr, 1,
                                               at<float2>(ctx, L.part), c.TXD_img, c.TYD_img,
                                               flag + 1, batch),
                      "tensor-core adjoint tile analysis");
  else
    st = check_launch(ctx, launch_analysis(s, 0, dldi, nullptr, flag, c.TXD, g.N, g.Nc, c.TYD, na,
                                           g.Nr, 1, at<float2>(ctx, L.part)),
                      "adjoint tile analysis");
  ctx->stage_end(4);
  if (st) return st;
  ctx->stage_begin(5);
  st = check_launch(ctx, launch_reduce_tiles(s, at<float2>(ctx, L.part), L.tiles, na * g.Nc,
                                             1.f / ((float)g.N * g.N), at<float2>(ctx, L.gh), batch,
                                             ctx->adj_part_trows),
                    "adjoint tile reduction");
  ctx->stage_end(5);
  if (st) return st;
  ctx->stage_begin(6);
  st = check_launch(ctx, launch_band_adjoint(s, c, f, at<float2>(ctx, L.gh), scale,
                                             at<float>(ctx, L.gam), at<float2>(ctx, L.Zk),
                                             at<float2>(ctx, L.X), at<float>(ctx, L.Vt),
                                             tc ? at<void>(ctx, L.img) : nullptr, batch,
                                             ctx->band_width(g.N, batch)),
                    "band adjoint");
  ctx->stage_end(6);
  if (st) return st;
  ctx->stage_begin(7);
  if (tc) {
    int* err = reinterpret_cast<int*>(ctx->d_red + RED_FLAG) + 1;
    if (pers && tc3_synth_supported(g.kp_rows))
      st = check_launch(ctx, launch_synth_grad_tc3(s, c.AYS_img, at<void>(ctx, L.img), g.N,
                                                   g.kp_rows, ep, err, nblocks, batch),
                        "tensor-core adjoint row synthesis (persistent)");
    else
      st = check_launch(ctx, launch_synth_grad_tc2(s, c.AYS_img, at<void>(ctx, L.img), g.N,
                                                   g.kp_rows, ep, err, nblocks, batch),
                        "tensor-core adjoint row synthesis");
  } else {
    st = check_launch(ctx, launch_synth_grad(s, c.AYS, at<float>(ctx, L.Vt), g.N, g.kp_rows, ep,
                                             nblocks),
                      "adjoint row synthesis");
  }
  ctx->stage_end(7);
  ctx->launches += analysed ? 6 : 7;  // analysis, reduction, gamma, Z, X, expansion, synthesis
  return st;
}

int prepare(Context* ctx, const Cache& c, Layout* L, int batch = 1, bool own_field = false) {
  if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx->fail(LITHO_ERR_CUDA, "cudaSetDevice");
  *L = make_layout(c.g, batch, own_field);
  int st = ctx->ensure_scratch(L->total);
  if (st) return st;
  const int blocks = ((c.g.N + 127) / 128) * ((c.g.N + 127) / 128);
  st = ctx->ensure_red(RED_PART + (3 * (size_t)blocks + 3) * batch + 1200);
  if (st) return st;
  LITHO_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_red, 0, RED_PART * sizeof(double), ctx->stream));
  return LITHO_OK;
}

// Copies n summed doubles (and the flag) back to the host and waits.
int fetch(Context* ctx, int n) {
  LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_red, ctx->d_red, (RED_SUM + n) * sizeof(double),
                                      cudaMemcpyDeviceToHost, ctx->stream));
  LITHO_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->collect_stages();
  int tc_err;
  std::memcpy(&tc_err, reinterpret_cast<const char*>(ctx->h_red + RED_FLAG) + sizeof(int),
              sizeof(int));
  if (tc_err)
    return ctx->fail(LITHO_ERR_CUDA, "tensor-core synthesis: a bounded wait expired (code " +
                                         std::to_string(tc_err) + ")");
  return LITHO_OK;
}

int* flag_word(const Context* ctx) { return reinterpret_cast<int*>(ctx->d_red + RED_FLAG); }

// deferred[0] |= the call's non-finite flag; deferred[1] keeps the first wait code.
__global__ void merge_deferred_kernel(const int* __restrict__ flag, int* __restrict__ deferred) {
  if (threadIdx.x == 0) {
    if (flag[0]) deferred[0] = 1;
    if (flag[1] && !deferred[1]) deferred[1] = flag[1];
  }
}
cudaError_t launch_merge_deferred(cudaStream_t s, const int* flag, int* deferred) {
  merge_deferred_kernel<<<1, 32, 0, s>>>(flag, deferred);
  return cudaGetLastError();
}

// dts[i] = the step of image i ((max |Vn|, dt) float pairs).
__global__ void dt_export_kernel(const float* __restrict__ vd, int batch, double* __restrict__ dts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < batch) dts[i] = vd[2 * i + 1];
}

// Per image b: tracked loss l = losses[2b] + pen_weight losses[2b + 1]; history[b][iters[b]]
// = l when there is a column for it; iters[b] += 1; improved[b] = l < best[b], and then
// best[b] = l.
__global__ void track_scalars_kernel(int batch, const double* __restrict__ losses, double pen_weight,
                                     double* __restrict__ best, double* __restrict__ history,
                                     int history_cols, int* __restrict__ iters,
                                     int* __restrict__ improved) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  const double l = losses[2 * b] + pen_weight * losses[2 * b + 1];
  const int it = iters[b];
  if (history && it >= 0 && it < history_cols) history[(size_t)b * history_cols + it] = l;
  iters[b] = it + 1;
  const int up = l < best[b];
  improved[b] = up;
  if (up) best[b] = l;
}
// best_masks[b] = masks[b] where improved[b]; vec: n % 4 == 0 and both bases 16-byte
// aligned, so every image's float4 view is aligned.
__global__ void track_masks_kernel(long long n, int vec, const int* __restrict__ improved,
                                   const float* __restrict__ masks, float* __restrict__ best_masks) {
  const int b = blockIdx.y;
  if (!improved[b]) return;
  const float* src = masks + (size_t)b * n;
  float* dst = best_masks + (size_t)b * n;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (vec) {
    const float4* s4 = reinterpret_cast<const float4*>(src);
    float4* d4 = reinterpret_cast<float4*>(dst);
    for (long long i = i0; i < n / 4; i += stride) d4[i] = s4[i];
  } else {
    for (long long i = i0; i < n; i += stride) dst[i] = src[i];
  }
}

bool flag_set(const Context* ctx) {
  int v;
  std::memcpy(&v, ctx->h_red + RED_FLAG, sizeof(int));
  return v != 0;
}

}  // namespace

extern "C" {

int litho_imaging_compute(litho_ctx* ctx, const litho_cache* cache, const float* d_mask,
                          double threshold, double alpha, float* d_aerial, float* d_wafer,
                          litho_field* field) {
  if (!ctx || !cache || !d_mask) return LITHO_ERR_INVALID_ARGUMENT;
  if (!std::isfinite(threshold) || !std::isfinite(alpha))
    return ctx->fail(LITHO_ERR_NONFINITE, "Imaging: mask, threshold, and alpha must be finite");
  if (field && field->cache != cache)
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "field belongs to another cache");
  // Without a caller's field the band state of this call lives in the context's
  // scratch (no allocation per call once the scratch has grown to this cache).
  Layout L;
  int st = prepare(ctx, *cache, &L, 1, field == nullptr);
  if (st) return st;
  Field tmp;
  Field* f = field;
  if (!f) {
    tmp.cache = cache;
    tmp.e = at<float2>(ctx, L.fe);
    tmp.mband = at<float2>(ctx, L.fm);
    f = &tmp;
  }
  f->valid = false;
  ResistEpilogue ep{};
  ep.mode = 0;
  ep.thr = (float)threshold;
  ep.alpha = (float)alpha;
  ep.aerial = d_aerial;
  ep.wafer = d_wafer;
  int nb = 0;
  st = run_forward(ctx, *cache, *f, L, 0, d_mask, nullptr, ep, &nb);
  if (!st) st = fetch(ctx, 0);
  if (st) return st;
  if (flag_set(ctx)) {
    f->valid = false;
    return ctx->fail(LITHO_ERR_NONFINITE, "Imaging: mask, threshold, and alpha must be finite");
  }
  return LITHO_OK;
}

int litho_backpropagate(litho_ctx* ctx, const litho_field* field, const float* d_dLdI,
                        double output_scale, float* d_grad) {
  if (!ctx || !field || !d_dLdI || !d_grad) return LITHO_ERR_INVALID_ARGUMENT;
  if (!field->valid) return ctx->fail(LITHO_ERR_NOT_READY, "Gradient: field not computed");
  const Cache& c = *field->cache;
  Layout L;
  int st = prepare(ctx, c, &L);
  if (st) return st;
  GradEpilogue ep{};
  ep.grad_mask = d_grad;
  int nb = 0;
  st = run_adjoint(ctx, c, *field, L, d_dLdI, output_scale, ep, &nb);
  if (!st) st = fetch(ctx, 0);
  if (st) return st;
  if (flag_set(ctx)) return ctx->fail(LITHO_ERR_NONFINITE, "Gradient: dLdI must be finite");
  return LITHO_OK;
}

int litho_pe_loss(litho_ctx* ctx, const float* d_wafer, const float* d_target, int rows,
                  int cols, const litho_pe_options* opt, double* loss) {
  if (!ctx || !d_wafer || !d_target || !loss || rows <= 0 || cols <= 0)
    return LITHO_ERR_INVALID_ARGUMENT;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return LITHO_ERR_CUDA;
  int st = ctx->ensure_red(RED_PART + 2 * 600);
  if (st) return st;
  litho_pe_options o{nullptr, nullptr, 1.0, 0.0, 0.01};
  if (opt) o = *opt;
  int nb = 0;
  st = check_launch(ctx,
                    launch_pe_loss(ctx->stream, d_wafer, d_target, o.pe_window, o.penalty_window,
                                   (float)o.penalty, (float)o.penalty_threshold,
                                   (size_t)rows * cols, ctx->d_red + RED_PART, &nb),
                    "pe loss");
  if (st) return st;
  st = check_launch(ctx, launch_sum_partials(ctx->stream, ctx->d_red + RED_PART, nb, 2,
                                             ctx->d_red + RED_SUM),
                    "sum");
  if (st) return st;
  ctx->launches += 2;
  st = fetch(ctx, 2);
  if (st) return st;
  // pe_weight * Loss::pe_loss + penalty * Loss::background_penalty_loss; with
  // pe_weight 1 this is Loss::pe_loss_with_penalty (loss.cpp:25-51).
  *loss = o.pe_weight * ctx->h_red[RED_SUM] + o.penalty * ctx->h_red[RED_SUM + 1];
  return LITHO_OK;
}

int litho_pe_gradient(litho_ctx* ctx, const litho_field* field, const float* d_wafer,
                      const float* d_target, const litho_pe_options* opt, double alpha,
                      float* d_grad, double* loss) {
  if (!ctx || !field || !d_wafer || !d_target || !d_grad) return LITHO_ERR_INVALID_ARGUMENT;
  if (!field->valid) return ctx->fail(LITHO_ERR_NOT_READY, "Gradient: field not computed");
  const Cache& c = *field->cache;
  Layout L;
  int st = prepare(ctx, c, &L);
  if (st) return st;
  litho_pe_options o{nullptr, nullptr, 1.0, 0.0, 0.01};
  if (opt) o = *opt;
  const int N = c.g.N;
  int nb = 0;
  st = check_launch(ctx,
                    launch_pe_dldi(ctx->stream, d_wafer, d_target, o.pe_window, o.penalty_window,
                                   (float)o.pe_weight, (float)o.penalty,
                                   (float)o.penalty_threshold, (size_t)N * N,
                                   at<float>(ctx, L.dldi), ctx->d_red + RED_PART, &nb),
                    "dL/dI");
  if (st) return st;
  st = check_launch(ctx, launch_sum_partials(ctx->stream, ctx->d_red + RED_PART, nb, 2,
                                             ctx->d_red + RED_SUM),
                    "sum");
  if (st) return st;
  ctx->launches += 2;
  GradEpilogue ep{};
  ep.grad_mask = d_grad;
  int nb2 = 0;
  st = run_adjoint(ctx, c, *field, L, at<float>(ctx, L.dldi), 4.0 * alpha, ep, &nb2);
  if (!st) st = fetch(ctx, 2);
  if (st) return st;
  if (loss) *loss = o.pe_weight * ctx->h_red[RED_SUM] + o.penalty * ctx->h_red[RED_SUM + 1];
  return LITHO_OK;
}

static int ctm_evaluate_impl(litho_ctx* ctx, const litho_cache* cache, litho_field* field,
                             const float* d_theta, const float* d_target, double threshold,
                             double alpha, float* d_mask, float* d_aerial, float* d_wafer,
                             float* d_grad_mask, float* d_grad_theta, double* loss,
                             double* grad_norm, cudaEvent_t target_ready) {
  if (!ctx || !cache || !d_theta || !d_target || !d_grad_theta) return LITHO_ERR_INVALID_ARGUMENT;
  if (!std::isfinite(threshold) || !std::isfinite(alpha))
    return ctx->fail(LITHO_ERR_NONFINITE, "Imaging: mask, threshold, and alpha must be finite");
  if (field && field->cache != cache)
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "field belongs to another cache");
  // Without a caller's field the band state lives in the context's scratch.
  Layout L;
  int st = prepare(ctx, *cache, &L, 1, field == nullptr);
  if (st) return st;
  Field tmp;
  Field* f = field;
  if (!f) {
    tmp.cache = cache;
    tmp.e = at<float2>(ctx, L.fe);
    tmp.mband = at<float2>(ctx, L.fm);
    f = &tmp;
  }
  ResistEpilogue ep{};
  ep.mode = 1;
  ep.thr = (float)threshold;
  ep.alpha = (float)alpha;
  ep.aerial = d_aerial;
  ep.wafer = d_wafer;
  ep.target = d_target;
  ep.pe_weight = 1.f;
  ep.penalty = 0.f;
  ep.pen_thr = 0.01f;
  ep.dldi = at<float>(ctx, L.dldi);
  ep.loss_partial = ctx->d_red + RED_PART;
  // Tensor-core path: the resist synthesis also runs the adjoint tile analysis.
  const bool fuse = ctx->precision == LITHO_PRECISION_BF16X3 && cache->TXD_img != nullptr;
  // The whole chain of launches, on ctx->stream.
  auto launch_chain = [&]() -> int {
    int nb = 0;
    int r = run_forward(ctx, *cache, *f, L, 1, d_theta, d_mask, ep, &nb, target_ready, fuse);
    GradEpilogue gp{};
    gp.grad_mask = d_grad_mask;
    gp.theta = d_theta;
    gp.grad_theta = d_grad_theta;
    gp.norm_partial = ctx->d_red + RED_PART + 2 * (size_t)nb;
    int nb2 = 0;
    if (!r)
      r = run_adjoint(ctx, *cache, *f, L, at<float>(ctx, L.dldi), 4.0 * alpha, gp, &nb2, fuse);
    // Both FP64 sums (loss terms and the gradient norm) in one launch at the end, off
    // the path between the forward and the adjoint.
    if (!r)
      r = check_launch(ctx, launch_sum_partials2(ctx->stream, ctx->d_red + RED_PART, nb, 2,
                                                 ctx->d_red + RED_SUM, gp.norm_partial, nb2, 1,
                                                 ctx->d_red + RED_SUM + 2),
                       "sum");
    ctx->launches += 1;
    return r;
  };
  // Repeated evaluations on the same buffers replay a CUDA graph of the chain.
  const BandGeom& g = cache->g;
  EvalKey key;
  const void* ptrs[16] = {cache,       f->e,          f->mband,          d_theta,
                          d_target,    d_mask,        d_aerial,          d_wafer,
                          d_grad_mask, d_grad_theta,  ctx->scratch.base, ctx->d_red,
                          cache->H,    cache->AYD_img, cache->TXS,
                          reinterpret_cast<const void*>(
                              (uintptr_t)ctx->precision |
                              ((uintptr_t)ctx->tc_persistent(cache->g.N, 1) << 4))};
  for (int i = 0; i < 16; ++i) key.ptr[i] = ptrs[i];
  const int geom[6] = {g.N, g.K, g.Nr, g.Nc, g.row0, g.col0};
  for (int i = 0; i < 6; ++i) key.geom[i] = geom[i];
  key.thr = threshold;
  key.alpha = alpha;
  const bool graphable = ctx->graphs && field != nullptr && target_ready == nullptr &&
                         !ctx->timing && ctx->stream != nullptr &&
                         ctx->stream != cudaStreamLegacy;   // the legacy stream cannot be captured
  if (graphable && ctx->eval_graph && key == ctx->eval_graph_key) {
    LITHO_CUDA_TRY(ctx, cudaGraphLaunch(ctx->eval_graph, ctx->stream));
    ctx->launches += ctx->eval_graph_launches;
    f->valid = true;
  } else if (graphable && ctx->eval_last_valid && key == ctx->eval_last_key) {
    if (ctx->eval_graph) {
      cudaGraphExecDestroy(ctx->eval_graph);
      ctx->eval_graph = nullptr;
    }
    const long long launches0 = ctx->launches;
    cudaGraph_t graph = nullptr;
    bool captured = false;
    if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      st = launch_chain();
      const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
      captured = st == LITHO_OK && e == cudaSuccess && graph &&
                 cudaGraphInstantiate(&ctx->eval_graph, graph, 0) == cudaSuccess;
      if (graph) cudaGraphDestroy(graph);
    }
    cudaGetLastError();
    if (captured) {
      ctx->eval_graph_key = key;
      ctx->eval_graph_launches = ctx->launches - launches0;
      LITHO_CUDA_TRY(ctx, cudaGraphLaunch(ctx->eval_graph, ctx->stream));
    } else {
      // Capture is not available here: launch the chain directly.
      if (ctx->eval_graph) cudaGraphExecDestroy(ctx->eval_graph);
      ctx->eval_graph = nullptr;
      ctx->launches = launches0;
      st = launch_chain();
    }
  } else {
    st = launch_chain();
  }
  ctx->eval_last_key = key;
  ctx->eval_last_valid = graphable;
  if (!st) st = fetch(ctx, 3);
  if (st) return st;
  if (flag_set(ctx)) {
    f->valid = false;
    return ctx->fail(LITHO_ERR_NONFINITE, "theta must be finite");
  }
  if (loss) *loss = ctx->h_red[RED_SUM];
  if (grad_norm) *grad_norm = std::sqrt(ctx->h_red[RED_SUM + 2]);
  return LITHO_OK;
}

int litho_ctm_evaluate(litho_ctx* ctx, const litho_cache* cache, litho_field* field,
                       const float* d_theta, const float* d_target, double threshold,
                       double alpha, float* d_mask, float* d_aerial, float* d_wafer,
                       float* d_grad_mask, float* d_grad_theta, double* loss,
                       double* grad_norm) {
  return ctm_evaluate_impl(ctx, cache, field, d_theta, d_target, threshold, alpha, d_mask,
                           d_aerial, d_wafer, d_grad_mask, d_grad_theta, loss, grad_norm,
                           nullptr);
}

// The batched tensor-core chain on ctx->stream, without a host round trip: per
// image {PE, penalty term, ||dPE/dtheta||^2} into d_sums ([batch][3], device). L
// comes from prepare(ctx, c, &L, batch, true) (band state of every image included;
// batch > 1 includes it anyway); the partials use the reduction area.
static int ctm_batch_chain(Context* ctx, const Cache& c, const Layout& L, int batch,
                           const float* d_theta, const float* d_target, double threshold,
                           double alpha, float* d_grad_theta, double* d_sums) {
  Field f;
  f.cache = &c;
  f.e = at<float2>(ctx, L.fe);
  f.mband = at<float2>(ctx, L.fm);
  ResistEpilogue ep{};
  ep.mode = 1;
  ep.thr = (float)threshold;
  ep.alpha = (float)alpha;
  ep.target = d_target;
  ep.pe_weight = 1.f;
  ep.penalty = 0.f;
  ep.pen_thr = 0.01f;
  ep.loss_partial = ctx->d_red + RED_PART;
  int nb = 0, nb2 = 0;
  int st = run_forward(ctx, c, f, L, 1, d_theta, nullptr, ep, &nb, nullptr, true, batch);
  GradEpilogue gp{};
  gp.theta = d_theta;
  gp.grad_theta = d_grad_theta;
  gp.norm_partial = ctx->d_red + RED_PART + 2 * (size_t)nb * batch;
  if (!st) st = run_adjoint(ctx, c, f, L, nullptr, 4.0 * alpha, gp, &nb2, true, batch);
  if (!st)
    st = check_launch(ctx, launch_sum_partials_batch(ctx->stream, ctx->d_red + RED_PART, nb, 2,
                                                     gp.norm_partial, nb2, 1, d_sums, batch),
                      "sum");
  ctx->launches += 1;
  return st;
}

int litho_ctm_evaluate_batch(litho_ctx* ctx, const litho_cache* cache, int batch,
                             const float* d_theta, const float* d_target, double threshold,
                             double alpha, float* d_grad_theta, double* losses, double* norms) {
  if (!ctx || !cache || batch < 1 || !d_theta || !d_target || !d_grad_theta)
    return LITHO_ERR_INVALID_ARGUMENT;
  if (!std::isfinite(threshold) || !std::isfinite(alpha))
    return ctx->fail(LITHO_ERR_NONFINITE, "Imaging: mask, threshold, and alpha must be finite");
  const BandGeom& g = cache->g;
  const size_t px = (size_t)g.N * g.N;
  const bool tc = ctx->precision == LITHO_PRECISION_BF16X3 && cache->TXD_img != nullptr;
  if (!tc || batch == 1) {
    // One image after another (FP32 parity mode, or a single image).
    for (int b = 0; b < batch; ++b) {
      double lo = 0.0, no = 0.0;
      const int st = ctm_evaluate_impl(ctx, cache, nullptr, d_theta + b * px, d_target + b * px,
                                       threshold, alpha, nullptr, nullptr, nullptr, nullptr,
                                       d_grad_theta + b * px, &lo, &no, nullptr);
      if (st) return st;
      if (losses) losses[b] = lo;
      if (norms) norms[b] = no;
    }
    return LITHO_OK;
  }
  Layout L;
  int st = prepare(ctx, *cache, &L, batch);
  if (st) return st;
  double* d_sums = ctx->d_red + RED_PART + 3 * (size_t)L.tiles * batch;
  auto chain = [&]() {
    return ctm_batch_chain(ctx, *cache, L, batch, d_theta, d_target, threshold, alpha,
                           d_grad_theta, d_sums);
  };
  // Repeated calls on the same buffers replay a CUDA graph of the chain (captured on
  // the second consecutive call with the same key), as the single-image evaluation does.
  EvalKey key;
  const void* ptrs[16] = {cache, d_theta, d_target, d_grad_theta, ctx->scratch.base, ctx->d_red,
                          cache->H, cache->AYD_img, cache->TXS_img, cache->TXD_img,
                          reinterpret_cast<const void*>((uintptr_t)batch),
                          reinterpret_cast<const void*>(
                              (uintptr_t)ctx->precision | ((uintptr_t)ctx->tc_persistent(g.N, batch) << 4) |
                              ((uintptr_t)ctx->band_width(g.N, batch) << 8))};
  for (int i = 0; i < 16; ++i) key.ptr[i] = ptrs[i];
  const int geom[6] = {g.N, g.K, g.Nr, g.Nc, g.row0, g.col0};
  for (int i = 0; i < 6; ++i) key.geom[i] = geom[i];
  key.thr = threshold;
  key.alpha = alpha;
  const bool graphable = ctx->graphs && !ctx->timing && ctx->stream != nullptr &&
                         ctx->stream != cudaStreamLegacy;   // the legacy stream cannot be captured
  if (graphable && ctx->batch_graph && key == ctx->batch_graph_key) {
    LITHO_CUDA_TRY(ctx, cudaGraphLaunch(ctx->batch_graph, ctx->stream));
    ctx->launches += ctx->batch_graph_launches;
  } else if (graphable && ctx->batch_last_valid && key == ctx->batch_last_key) {
    if (ctx->batch_graph) {
      cudaGraphExecDestroy(ctx->batch_graph);
      ctx->batch_graph = nullptr;
    }
    const long long launches0 = ctx->launches;
    cudaGraph_t graph = nullptr;
    bool captured = false;
    if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      st = chain();
      const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
      captured = st == LITHO_OK && e == cudaSuccess && graph &&
                 cudaGraphInstantiate(&ctx->batch_graph, graph, 0) == cudaSuccess;
      if (graph) cudaGraphDestroy(graph);
    }
    cudaGetLastError();
    if (captured) {
      ctx->batch_graph_key = key;
      ctx->batch_graph_launches = ctx->launches - launches0;
      LITHO_CUDA_TRY(ctx, cudaGraphLaunch(ctx->batch_graph, ctx->stream));
    } else {
      // Capture is not available here: launch the chain directly.
      if (ctx->batch_graph) cudaGraphExecDestroy(ctx->batch_graph);
      ctx->batch_graph = nullptr;
      ctx->launches = launches0;
      st = chain();
    }
  } else {
    st = chain();
  }
  ctx->batch_last_key = key;
  ctx->batch_last_valid = graphable;
  std::vector<double> sums(3 * (size_t)batch);
  if (!st)
    LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(sums.data(), d_sums, sums.size() * sizeof(double),
                                        cudaMemcpyDeviceToHost, ctx->stream));
  if (!st) st = fetch(ctx, 0);
  if (st) return st;
  if (flag_set(ctx)) return ctx->fail(LITHO_ERR_NONFINITE, "theta must be finite");
  for (int b = 0; b < batch; ++b) {
    if (losses) losses[b] = sums[3 * (size_t)b];
    if (norms) norms[b] = std::sqrt(sums[3 * (size_t)b + 2]);
  }
  return LITHO_OK;
}

// Batched imaging + PE + dPE/dM. losses (host, nullable): PE per image, after a host
// round trip. d_losses (device, nullable): {PE, background-penalty term} per image with
// no host round trip (pen_term also sums that term at threshold pen_thr; a non-finite
// input goes to the deferred status).
static int pe_gradient_batch_impl(litho_ctx* ctx, const litho_cache* cache, int batch,
                                  const float* d_masks, const float* d_targets, double threshold,
                                  double alpha, float* d_grad_masks, double* losses,
                                  double* d_losses, bool pen_term, double pen_thr) {
  if (!ctx || !cache || batch < 1 || !d_masks || !d_targets || !d_grad_masks)
    return LITHO_ERR_INVALID_ARGUMENT;
  if (!std::isfinite(threshold) || !std::isfinite(alpha))
    return ctx->fail(LITHO_ERR_NONFINITE, "Imaging: mask, threshold, and alpha must be finite");
  const BandGeom& g = cache->g;
  const size_t px = (size_t)g.N * g.N;
  const bool tc = ctx->precision == LITHO_PRECISION_BF16X3 && cache->TXD_img != nullptr;
  Layout L;
  int st = prepare(ctx, *cache, &L, tc ? batch : 1, true);
  if (st) return st;
  Field f;
  f.cache = cache;
  f.e = at<float2>(ctx, L.fe);
  f.mband = at<float2>(ctx, L.fm);
  ResistEpilogue ep{};
  ep.mode = 1;
  ep.thr = (float)threshold;
  ep.alpha = (float)alpha;
  ep.pe_weight = 1.f;
  ep.penalty = 0.f;
  ep.pen_thr = (float)pen_thr;
  ep.loss_penalty_term = pen_term ? 1 : 0;
  ep.loss_partial = ctx->d_red + RED_PART;
  GradEpilogue gp{};
  cudaStream_t s = ctx->stream;
  const bool device_out = d_losses != nullptr;
  if (device_out) {
    st = ctx->ensure_deferred();
    if (st) return st;
  }
  if (tc) {
    // Every image in one pass: the resist synthesis runs the adjoint tile analysis.
    ep.target = d_targets;
    gp.grad_mask = d_grad_masks;
    int nb = 0, nb2 = 0;
    st = run_forward(ctx, *cache, f, L, 0, d_masks, nullptr, ep, &nb, nullptr, true, batch);
    if (!st) st = run_adjoint(ctx, *cache, f, L, nullptr, 4.0 * alpha, gp, &nb2, true, batch);
    double* d_sums = ctx->d_red + RED_PART + 2 * (size_t)nb * batch;
    if (!st)
      st = check_launch(ctx, launch_sum_partials_batch(s, ctx->d_red + RED_PART, nb, 2,
                                                       ctx->d_red + RED_PART, 0, 0, d_sums, batch),
                        "sum");
    ctx->launches += 1;
    if (device_out) {
      if (!st)
        LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(d_losses, d_sums, 2 * (size_t)batch * sizeof(double),
                                            cudaMemcpyDeviceToDevice, s));
      if (!st) st = check_launch(ctx, launch_merge_deferred(s, flag_word(ctx), ctx->d_deferred),
                                 "deferred status");
      return st;
    }
    std::vector<double> sums(2 * (size_t)batch);
    if (!st)
      LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(sums.data(), d_sums, sums.size() * sizeof(double),
                                          cudaMemcpyDeviceToHost, s));
    if (!st) st = fetch(ctx, 0);
    if (st) return st;
    if (flag_set(ctx)) return ctx->fail(LITHO_ERR_NONFINITE, "mask must be finite");
    for (int b = 0; b < batch && losses; ++b) losses[b] = sums[2 * (size_t)b];
    return LITHO_OK;
  }
  // FP32: one image after another through the same chain with dL/dI stored between
  // the resist synthesis and the adjoint.
  for (int b = 0; b < batch; ++b) {
    ep.target = d_targets + b * px;
    ep.dldi = at<float>(ctx, L.dldi);
    gp.grad_mask = d_grad_masks + b * px;
    int nb = 0, nb2 = 0;
    st = run_forward(ctx, *cache, f, L, 0, d_masks + b * px, nullptr, ep, &nb);
    if (!st)
      st = check_launch(ctx, launch_sum_partials(s, ctx->d_red + RED_PART, nb, 2,
                                                 ctx->d_red + RED_SUM),
                        "sum");
    ctx->launches += 1;
    if (!st) st = run_adjoint(ctx, *cache, f, L, at<float>(ctx, L.dldi), 4.0 * alpha, gp, &nb2);
    if (device_out) {
      if (!st)
        LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(d_losses + 2 * (size_t)b, ctx->d_red + RED_SUM,
                                            2 * sizeof(double), cudaMemcpyDeviceToDevice, s));
      if (st) return st;
      continue;
    }
    if (!st) st = fetch(ctx, 2);
    if (st) return st;
    if (flag_set(ctx)) return ctx->fail(LITHO_ERR_NONFINITE, "mask must be finite");
    if (losses) losses[b] = ctx->h_red[RED_SUM];
  }
  if (device_out)
    return check_launch(ctx, launch_merge_deferred(s, flag_word(ctx), ctx->d_deferred),
                        "deferred status");
  return LITHO_OK;
}

int litho_pe_gradient_batch(litho_ctx* ctx, const litho_cache* cache, int batch,
                            const float* d_masks, const float* d_targets, double threshold,
                            double alpha, float* d_grad_masks, double* losses) {
  return pe_gradient_batch_impl(ctx, cache, batch, d_masks, d_targets, threshold, alpha,
                                d_grad_masks, losses, nullptr, false, 0.01);
}

int litho_pe_gradient_batch_device(litho_ctx* ctx, const litho_cache* cache, int batch,
                                   const float* d_masks, const float* d_targets, double threshold,
                                   double alpha, double penalty_threshold, float* d_grad_masks,
                                   double* d_losses) {
  if (!ctx || !d_losses) return LITHO_ERR_INVALID_ARGUMENT;
  if (!std::isfinite(penalty_threshold))
    return ctx->fail(LITHO_ERR_NONFINITE, "penalty threshold must be finite");
  return pe_gradient_batch_impl(ctx, cache, batch, d_masks, d_targets, threshold, alpha,
                                d_grad_masks, nullptr, d_losses, true, penalty_threshold);
}

// Host buffers: theta goes up first on the context's stream; the target follows on
// an upload stream while the analysis and the small-grid stage run, and the
// resist epilogue waits for it. The staging buffer and the upload stream persist
// in the context.
int litho_ctm_evaluate_host(litho_ctx* ctx, const litho_cache* cache, litho_field* field,
                            const float* h_theta, const float* h_target, double threshold,
                            double alpha, float* h_grad_theta, double* loss,
                            double* grad_norm) {
  if (!ctx || !cache || !h_theta || !h_target || !h_grad_theta) return LITHO_ERR_INVALID_ARGUMENT;
  const size_t n = (size_t)cache->g.N * cache->g.N;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return LITHO_ERR_CUDA;
  if (ctx->host_stage.bytes < 3 * n * sizeof(float)) {
    cudaStreamSynchronize(ctx->stream);
    if (ctx->host_stage.base) cudaFree(ctx->host_stage.base);
    ctx->host_stage.base = nullptr;
    ctx->host_stage.bytes = 0;
    if (cudaMalloc(&ctx->host_stage.base, 3 * n * sizeof(float)) != cudaSuccess) {
      cudaGetLastError();
      return ctx->fail(LITHO_ERR_OOM, "host-call staging allocation failed");
    }
    ctx->host_stage.bytes = 3 * n * sizeof(float);
  }
  if (!ctx->aux) {
    if (cudaStreamCreateWithFlags(&ctx->aux, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_aux[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_aux[1], cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return ctx->fail(LITHO_ERR_CUDA, "upload stream creation failed");
    }
  }
  float* d = static_cast<float*>(ctx->host_stage.base);
  int st = LITHO_OK;
  if (cudaMemcpyAsync(d, h_theta, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream) !=
          cudaSuccess ||
      cudaEventRecord(ctx->ev_aux[0], ctx->stream) != cudaSuccess ||
      cudaStreamWaitEvent(ctx->aux, ctx->ev_aux[0], 0) != cudaSuccess ||
      cudaMemcpyAsync(d + n, h_target, n * sizeof(float), cudaMemcpyHostToDevice, ctx->aux) !=
          cudaSuccess ||
      cudaEventRecord(ctx->ev_aux[1], ctx->aux) != cudaSuccess)
    st = ctx->fail(LITHO_ERR_CUDA, "host to device copy failed");
  if (!st)
    st = ctm_evaluate_impl(ctx, cache, field, d, d + n, threshold, alpha, nullptr, nullptr,
                           nullptr, nullptr, d + 2 * n, loss, grad_norm, ctx->ev_aux[1]);
  if (!st && cudaMemcpyAsync(h_grad_theta, d + 2 * n, n * sizeof(float), cudaMemcpyDeviceToHost,
                             ctx->stream) != cudaSuccess)
    st = ctx->fail(LITHO_ERR_CUDA, "device to host copy failed");
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess && !st)
    st = ctx->fail(LITHO_ERR_CUDA, "stream synchronize failed");
  if (cudaStreamSynchronize(ctx->aux) != cudaSuccess && !st)
    st = ctx->fail(LITHO_ERR_CUDA, "upload stream synchronize failed");
  return st;
}

int litho_ctm_evaluate_host_batch(litho_ctx* ctx, const litho_cache* cache, int batch,
                                  const float* h_theta, const float* h_target, double threshold,
                                  double alpha, float* h_grad_theta, double* losses,
                                  double* norms) {
  if (!ctx || !cache || batch < 1 || !h_theta || !h_target || !h_grad_theta)
    return LITHO_ERR_INVALID_ARGUMENT;
  if (!std::isfinite(threshold) || !std::isfinite(alpha))
    return ctx->fail(LITHO_ERR_NONFINITE, "Imaging: mask, threshold, and alpha must be finite");
  const size_t n = (size_t)cache->g.N * cache->g.N;
  const bool tc = ctx->precision == LITHO_PRECISION_BF16X3 && cache->TXD_img != nullptr;
  if (!tc) {
    // FP32 parity mode: the single-image host call, image after image.
    for (int b = 0; b < batch; ++b) {
      double lo = 0.0, no = 0.0;
      const int st = litho_ctm_evaluate_host(ctx, cache, nullptr, h_theta + b * n,
                                             h_target + b * n, threshold, alpha,
                                             h_grad_theta + b * n, &lo, &no);
      if (st) return st;
      if (losses) losses[b] = lo;
      if (norms) norms[b] = no;
    }
    return LITHO_OK;
  }
  if (cudaSetDevice(ctx->device) != cudaSuccess) return LITHO_ERR_CUDA;
  // Groups of G images through two device slots: the upload of group g + 1, the
  // batched chain of group g and the download of group g - 1 run on three streams.
  // Large images are link-bound (a 2048^2 image takes about 0.6 ms to upload and
  // 0.13 ms to evaluate alone): one per group keeps the pipeline's fill and drain
  // short. Small ones are grouped so that the chain keeps up with the copies.
  const int G = std::min(batch, cache->g.N >= 1024 ? 1 : 4);
  const int ngroups = (batch + G - 1) / G;
  const size_t slot_floats = 3 * (size_t)G * n;                 // theta | target | gradient
  const size_t need = 2 * slot_floats * sizeof(float) + 3 * (size_t)batch * sizeof(double);
  if (ctx->pipe_stage.bytes < need) {
    cudaStreamSynchronize(ctx->stream);
    if (ctx->dn) cudaStreamSynchronize(ctx->dn);
    if (ctx->pipe_stage.base) cudaFree(ctx->pipe_stage.base);
    ctx->pipe_stage.base = nullptr;
    ctx->pipe_stage.bytes = 0;
    if (cudaMalloc(&ctx->pipe_stage.base, need) != cudaSuccess) {
      cudaGetLastError();
      return ctx->fail(LITHO_ERR_OOM, "host-batch staging allocation failed");
    }
    ctx->pipe_stage.bytes = need;
  }
  if (!ctx->aux) {
    if (cudaStreamCreateWithFlags(&ctx->aux, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_aux[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_aux[1], cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return ctx->fail(LITHO_ERR_CUDA, "upload stream creation failed");
    }
  }
  if (!ctx->dn) {
    bool ok = cudaStreamCreateWithFlags(&ctx->dn, cudaStreamNonBlocking) == cudaSuccess;
    for (auto& slot : ctx->ev_pipe)
      for (cudaEvent_t& e : slot)
        ok = ok && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      return ctx->fail(LITHO_ERR_CUDA, "download stream creation failed");
    }
  }
  Layout L;
  int st = prepare(ctx, *cache, &L, G, true);   // with the band state of G images
  if (st) return st;
  float* base = static_cast<float*>(ctx->pipe_stage.base);
  double* d_sums = reinterpret_cast<double*>(base + 2 * slot_floats);
  cudaStream_t up = ctx->aux, cp = ctx->stream, dn = ctx->dn;
  enum { UP = 0, CP = 1, DN = 2 };
  // The uploads must not start before work already queued on the compute stream.
  if (cudaEventRecord(ctx->ev_aux[0], cp) != cudaSuccess ||
      cudaStreamWaitEvent(up, ctx->ev_aux[0], 0) != cudaSuccess)
    st = ctx->fail(LITHO_ERR_CUDA, "stream ordering failed");
  for (int g = 0; g < ngroups && !st; ++g) {
    const int s = g & 1;
    const int t0 = g * G, m = batch - t0 < G ? batch - t0 : G;
    float* th = base + s * slot_floats;
    float* tg = th + (size_t)G * n;
    float* gr = tg + (size_t)G * n;
    cudaEvent_t* ev = ctx->ev_pipe[s];
    bool ok = true;
    if (g >= 2) ok = cudaStreamWaitEvent(up, ev[CP], 0) == cudaSuccess;   // slot's inputs read
    ok = ok && cudaMemcpyAsync(th, h_theta + t0 * n, m * n * sizeof(float),
                               cudaMemcpyHostToDevice, up) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(tg, h_target + t0 * n, m * n * sizeof(float),
                               cudaMemcpyHostToDevice, up) == cudaSuccess;
    ok = ok && cudaEventRecord(ev[UP], up) == cudaSuccess;
    ok = ok && cudaStreamWaitEvent(cp, ev[UP], 0) == cudaSuccess;
    if (g >= 2) ok = ok && cudaStreamWaitEvent(cp, ev[DN], 0) == cudaSuccess;   // slot's gradients out
    if (!ok) {
      st = ctx->fail(LITHO_ERR_CUDA, "host batch: copy scheduling failed");
      break;
    }
    st = ctm_batch_chain(ctx, *cache, L, m, th, tg, threshold, alpha, gr, d_sums + 3 * (size_t)t0);
    if (st) break;
    ok = cudaEventRecord(ev[CP], cp) == cudaSuccess &&
         cudaStreamWaitEvent(dn, ev[CP], 0) == cudaSuccess &&
         cudaMemcpyAsync(h_grad_theta + t0 * n, gr, m * n * sizeof(float), cudaMemcpyDeviceToHost,
                         dn) == cudaSuccess &&
         cudaEventRecord(ev[DN], dn) == cudaSuccess;
    if (!ok) st = ctx->fail(LITHO_ERR_CUDA, "host batch: download failed");
  }
  std::vector<double> sums(3 * (size_t)batch);
  if (!st)
    LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(sums.data(), d_sums, sums.size() * sizeof(double),
                                        cudaMemcpyDeviceToHost, cp));
  if (cudaStreamSynchronize(dn) != cudaSuccess && !st)
    st = ctx->fail(LITHO_ERR_CUDA, "download stream synchronize failed");
  if (cudaStreamSynchronize(up) != cudaSuccess && !st)
    st = ctx->fail(LITHO_ERR_CUDA, "upload stream synchronize failed");
  if (!st) st = fetch(ctx, 0);
  if (st) return st;
  if (flag_set(ctx)) return ctx->fail(LITHO_ERR_NONFINITE, "theta must be finite");
  for (int b = 0; b < batch; ++b) {
    if (losses) losses[b] = sums[3 * (size_t)b];
    if (norms) norms[b] = std::sqrt(sums[3 * (size_t)b + 2]);
  }
  return LITHO_OK;
}

int litho_field_export(litho_ctx* ctx, const litho_field* field, int k, float* d_E) {
  if (!ctx || !field || !d_E) return LITHO_ERR_INVALID_ARGUMENT;
  if (!field->valid) return ctx->fail(LITHO_ERR_NOT_READY, "field not computed");
  const Cache& c = *field->cache;
  if (k < 0 || k >= c.g.K) return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "kernel index out of range");
  Layout L;
  int st = prepare(ctx, c, &L);
  if (st) return st;
  st = check_launch(ctx, launch_export_field(ctx->stream, c, *field, k, at<float2>(ctx, L.rows_tmp),
                                             reinterpret_cast<float2*>(d_E)),
                    "field export");
  ctx->launches += 2;
  if (!st) LITHO_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return st;
}

// ---------------------------------------------------------------- level set
static int ls_check(litho_ctx* ctx, int rows, int cols, double dx, double dy, int minsz) {
  if (rows <= 0 || cols <= 0 || !(dx > 0.0) || !(dy > 0.0))
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT,
                     "evolve_normal_WENO_godunov: grid must be non-empty and dx/dy must be positive");
  if (rows < minsz || cols < minsz)
    return ctx->fail(LITHO_ERR_SHAPE, "curvature needs at least 3 rows and 3 columns");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx->fail(LITHO_ERR_CUDA, "cudaSetDevice");
  return LITHO_OK;
}

int litho_weno_godunov(litho_ctx* ctx, int rows, int cols, const float* d_phi, const float* d_vn,
                       double dy, double dx, float* d_delta, float* d_habs) {
  if (!ctx || !d_phi || !d_vn || !d_delta) return LITHO_ERR_INVALID_ARGUMENT;
  int st = ls_check(ctx, rows, cols, dx, dy, 1);
  if (st) return st;
  st = check_launch(ctx, launch_levelset(ctx->stream, 0, rows, cols, d_phi, nullptr, d_vn,
                                         (float)dx, (float)dy, 0.f, nullptr, d_delta, d_habs),
                    "weno godunov");
  ctx->launches += 1;
  if (!st) LITHO_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return st;
}

int litho_kappa(litho_ctx* ctx, int rows, int cols, const float* d_phi, double dx, double dy,
                double b, float* d_out) {
  if (!ctx || !d_phi || !d_out) return LITHO_ERR_INVALID_ARGUMENT;
  int st = ls_check(ctx, rows, cols, dx, dy, 3);
  if (st) return st;
  st = check_launch(ctx, launch_levelset(ctx->stream, 1, rows, cols, d_phi, nullptr, nullptr,
                                         (float)dx, (float)dy, (float)b, nullptr, d_out, nullptr),
                    "kappa");
  ctx->launches += 1;
  if (!st) LITHO_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return st;
}

static int ls_dt(litho_ctx* ctx, int rows, int cols, const float* d_vn, double dx, double dy,
                 double cfl, double b, float** dt_dev) {
  int st = ctx->ensure_red(RED_PART + 2 * 600);
  if (st) return st;
  LITHO_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_red, 0, RED_PART * sizeof(double), ctx->stream));
  float* part = reinterpret_cast<float*>(ctx->d_red + RED_PART);
  float* vmax = reinterpret_cast<float*>(ctx->d_red + RED_SUM);
  float* dt = vmax + 1;
  st = check_launch(ctx, launch_dt(ctx->stream, d_vn, (size_t)rows * cols, (float)dx, (float)dy,
                                   (float)cfl, (float)b, part, vmax, dt,
                                   reinterpret_cast<int*>(ctx->d_red + RED_FLAG)),
                    "dt");
  ctx->launches += 2;
  *dt_dev = dt;
  return st;
}

int litho_evolution_term(litho_ctx* ctx, int rows, int cols, const float* d_phi,
                         const float* d_vn, double dx, double dy, double cfl, double b,
                         float* d_normal, double* dt) {
  if (!ctx || !d_phi || !d_vn || !d_normal) return LITHO_ERR_INVALID_ARGUMENT;
  int st = ls_check(ctx, rows, cols, dx, dy, 3);
  if (st) return st;
  float* dtd = nullptr;
  st = ls_dt(ctx, rows, cols, d_vn, dx, dy, cfl, b, &dtd);
  if (st) return st;
  st = check_launch(ctx, launch_levelset(ctx->stream, 2, rows, cols, d_phi, nullptr, d_vn,
                                         (float)dx, (float)dy, (float)b, dtd, d_normal, nullptr),
                    "evolution");
  ctx->launches += 1;
  if (!st) st = fetch(ctx, 1);
  if (st) return st;
  if (flag_set(ctx)) return ctx->fail(LITHO_ERR_NONFINITE, "normal speed must be finite");
  float h[2];
  std::memcpy(h, ctx->h_red + RED_SUM, sizeof(h));
  if (dt) *dt = h[1];
  return LITHO_OK;
}

int litho_reinit_sdf(litho_ctx* ctx, int rows, int cols, const float* d_phi, double dx,
                     double dy, float* d_sdf, float* d_mask) {
  if (!ctx || !d_phi || !d_sdf) return LITHO_ERR_INVALID_ARGUMENT;
  int st = ls_check(ctx, rows, cols, dx, dy, 1);
  if (st) return st;
  if ((size_t)3 * cols * sizeof(float) > 200 * 1024)
    return ctx->fail(LITHO_ERR_UNSUPPORTED, "reinit_sdf supports at most 17066 columns");
  if (d_sdf == d_phi) return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "reinit_sdf: sdf must not alias phi");
  ctx->stage_begin(8);
  st = check_launch(ctx, launch_reinit_sdf(ctx->stream, rows, cols, d_phi, 0.f, 0, (float)dx, d_sdf,
                                           1, ctx->chamfer_threads(cols, 1)),
                    "reinit_sdf");
  if (!st && d_mask)
    st = check_launch(ctx, launch_levelset(ctx->stream, 5, rows, cols, d_sdf, nullptr, nullptr,
                                           (float)dx, (float)dy, 0.f, nullptr, d_mask, nullptr),
                      "mask");
  ctx->stage_end(8);
  ctx->launches += d_mask ? 2 : 1;
  if (!st) LITHO_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (!st) ctx->collect_stages();
  return st;
}

int litho_ctx_reserve(litho_ctx* ctx, const litho_cache* cache, int batch) {
  if (!ctx || !cache || batch < 1) return LITHO_ERR_INVALID_ARGUMENT;
  Layout L;
  int st = prepare(ctx, *cache, &L, batch, true);
  if (st) return st;
  // The batched RK2 update of `batch` images of this size (its stage-1 images).
  const size_t n = (size_t)cache->g.N * cache->g.N;
  st = ctx->ensure_scratch(std::max(L.total, n * batch * sizeof(float)));
  if (st) return st;
  st = ctx->ensure_red(RED_PART + ((size_t)batch * dt_batch_blocks(n, batch) + 1) / 2 + 8 +
                       (size_t)batch + 8);
  if (!st) st = ctx->ensure_deferred();
  if (st) return st;
  LITHO_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return LITHO_OK;
}

int litho_ctx_autotune(litho_ctx* ctx, const litho_cache* cache, int batch, int rows, int cols,
                       int nimg, int* band_width, int* chamfer_threads) {
  if (!ctx || (cache && batch < 1) || (nimg > 0 && (rows < 3 || cols < 3)))
    return LITHO_ERR_INVALID_ARGUMENT;
  if (band_width) *band_width = 0;
  if (chamfer_threads) *chamfer_threads = 0;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx->fail(LITHO_ERR_CUDA, "cudaSetDevice");
  cudaStream_t s = ctx->stream;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return ctx->fail(LITHO_ERR_CUDA, "cudaEventCreate");
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return ctx->fail(LITHO_ERR_CUDA, "cudaEventCreate");
  }
  // Mean time of three runs after one warm-up run, on the context's stream.
  auto timed = [&](auto&& run, float* ms) -> int {
    cudaError_t e = run();
    if (e == cudaSuccess) e = cudaEventRecord(e0, s);
    for (int r = 0; r < 3 && e == cudaSuccess; ++r) e = run();
    if (e == cudaSuccess) e = cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
    return check_launch(ctx, e, "autotune timing");
  };
  int st = LITHO_OK;
  if (cache) {
    // Schedule of the small-grid field and Z kernels (8- or 16-column chunks, or the
    // whole small grid per CTA; the results do not depend on it): the forward and
    // adjoint band stages of `batch` images, on zeroed inputs.
    Layout L;
    st = prepare(ctx, *cache, &L, batch, true);
    if (!st) LITHO_CUDA_TRY(ctx, cudaMemsetAsync(ctx->scratch.base, 0, L.total, s));
    const bool tc = ctx->precision == LITHO_PRECISION_BF16X3 && cache->TXS_img;
    Field f;
    f.cache = cache;
    f.e = at<float2>(ctx, L.fe);
    f.mband = at<float2>(ctx, L.fm);
    float best = 0.f;
    int bw = 0;
    for (const int w : {8, 16, BW_WHOLE}) {
      if (st) break;
      float ms = 0.f;
      st = timed([&]() -> cudaError_t {
        cudaError_t e = launch_band_forward(s, *cache, f, at<float>(ctx, L.ik), at<float>(ctx, L.iP),
                                            at<float2>(ctx, L.chat), at<float>(ctx, L.Ut),
                                            tc ? at<void>(ctx, L.img) : nullptr, batch, w);
        if (e != cudaSuccess) return e;
        return launch_band_adjoint(s, *cache, f, at<float2>(ctx, L.gh), 1.0, at<float>(ctx, L.gam),
                                   at<float2>(ctx, L.Zk), at<float2>(ctx, L.X),
                                   at<float>(ctx, L.Vt), tc ? at<void>(ctx, L.img) : nullptr,
                                   batch, w);
      }, &ms);
      if (!st && (bw == 0 || ms < best)) { best = ms; bw = w; }
    }
    if (!st) {
      ctx->tuned_band[{cache->g.N, batch}] = bw;
      if (band_width) *band_width = bw;
    }
    // Schedule of the split-BF16 tensor-core passes (per-tile CTAs or the persistent
    // pipelines) for `batch` images, when the context leaves it to the tuner: the
    // whole batched CTM chain timed with each, on zero theta and target images.
    if (!st && tc && ctx->tc_schedule == LITHO_TC_SCHEDULE_AUTO) {
      const size_t px = (size_t)cache->g.N * cache->g.N * batch;
      float* buf = nullptr;
      if (cudaMalloc(&buf, 3 * px * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        st = ctx->fail(LITHO_ERR_OOM, "autotune buffers");
      }
      if (!st) LITHO_CUDA_TRY(ctx, cudaMemsetAsync(buf, 0, 3 * px * sizeof(float), s));
      double* d_sums = ctx->d_red + RED_PART + 3 * (size_t)L.tiles * batch;
      float best_tc = 0.f;
      int pick = LITHO_TC_SCHEDULE_PERSISTENT;
      for (const int sched : {LITHO_TC_SCHEDULE_PERSISTENT, LITHO_TC_SCHEDULE_PER_TILE}) {
        if (st) break;
        ctx->tuned_tc[{cache->g.N, batch}] = sched;
        float ms = 0.f;
        int cst = LITHO_OK;
        st = timed([&]() -> cudaError_t {
          cst = ctm_batch_chain(ctx, *cache, L, batch, buf, buf + px, 0.225, 50.0, buf + 2 * px,
                                d_sums);
          return cst ? cudaErrorUnknown : cudaSuccess;
        }, &ms);
        if (!st && ms > 0.f && (best_tc == 0.f || ms < best_tc)) { best_tc = ms; pick = sched; }
      }
      if (buf) {
        cudaStreamSynchronize(s);
        cudaFree(buf);
      }
      ctx->tuned_tc[{cache->g.N, batch}] = pick;
    }
  }
  if (!st && nimg > 0) {
    // Chamfer CTA size for nimg images of rows x cols (timed on at most 512 MB of them).
    if ((size_t)3 * (cols + 4) * sizeof(float) > 200 * 1024) {
      st = ctx->fail(LITHO_ERR_UNSUPPORTED, "reinit_sdf supports at most 17066 columns");
    } else {
      const size_t px = (size_t)rows * cols;
      const int nt = (int)std::max<size_t>(1, std::min<size_t>(nimg, ((size_t)512 << 20) / (8 * px)));
      st = ctx->ensure_scratch(2 * px * nt * sizeof(float));
      float* phi = static_cast<float*>(ctx->scratch.base);
      float* out = phi + px * nt;
      if (!st) st = check_launch(ctx, launch_chamfer_probe(s, phi, rows, cols, nt), "autotune pattern");
      float best = 0.f;
      int bt = 0;
      for (const int t : {128, 256, 512, 1024}) {
        if (st) break;
        const int per = (cols + t - 1) / t;
        if ((t <= 256 && per > 32) || (t == 512 && per > 16)) continue;
        float ms = 0.f;
        st = timed([&]() {
          return launch_reinit_sdf(s, rows, cols, phi, 0.f, 0, 1.f, out, nt, t);
        }, &ms);
        if (!st && (bt == 0 || ms < best)) { best = ms; bt = t; }
      }
      if (!st) {
        ctx->tuned_chamfer[{cols, nimg}] = bt;
        if (chamfer_threads) *chamfer_threads = bt;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st;
}

int litho_lbfgs_dots(litho_ctx* ctx, int k, long long n, const float* d_rows, long long ld,
                     const float* d_v, double* out) {
  if (!ctx || k < 1 || k > 64 || n < 1 || ld < n || !d_rows || !d_v || !out)
    return LITHO_ERR_INVALID_ARGUMENT;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx->fail(LITHO_ERR_CUDA, "cudaSetDevice");
  const int nb = multi_dot_blocks((size_t)n);
  int st = ctx->ensure_red(RED_PART + (size_t)nb * k + (size_t)k + 8);
  if (st) return st;
  double* part = ctx->d_red + RED_PART;
  double* res = part + (size_t)nb * k;
  st = check_launch(ctx, launch_multi_dot(ctx->stream, d_rows, (size_t)ld, k, (size_t)n, d_v, part,
                                          res),
                    "L-BFGS inner products");
  ctx->launches += 2;
  if (st) return st;
  LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(out, res, (size_t)k * sizeof(double), cudaMemcpyDeviceToHost,
                                      ctx->stream));
  LITHO_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return LITHO_OK;
}

int litho_lbfgs_dots3(litho_ctx* ctx, int k, long long n, const float* d_rows, long long ld,
                      const float* d_v0, const float* d_v1, const float* d_v2, double* out) {
  if (!ctx || k < 1 || k > 64 || n < 1 || ld < n || !d_rows || !d_v0 || !out || (d_v2 && !d_v1))
    return LITHO_ERR_INVALID_ARGUMENT;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx->fail(LITHO_ERR_CUDA, "cudaSetDevice");
  const int nv = d_v2 ? 3 : (d_v1 ? 2 : 1);
  const size_t npart = (size_t)multi_dot3_blocks((size_t)n, k) * ((k + 7) / 8) * 24;
  int st = ctx->ensure_red(RED_PART + npart + (size_t)nv * k + 8);
  if (st) return st;
  double* part = ctx->d_red + RED_PART;
  double* res = part + npart;
  st = check_launch(ctx, launch_multi_dot3(ctx->stream, d_rows, (size_t)ld, k, (size_t)n, d_v0, d_v1,
                                           d_v2, part, res),
                    "L-BFGS inner products");
  ctx->launches += 2;
  if (st) return st;
  LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(out, res, (size_t)nv * k * sizeof(double),
                                      cudaMemcpyDeviceToHost, ctx->stream));
  LITHO_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return LITHO_OK;
}

int litho_lbfgs_combine(litho_ctx* ctx, int k, long long n, const float* d_rows, long long ld,
                        const double* coef, const float* d_v, double cv, float* d_out) {
  if (!ctx || k < 0 || k > 64 || n < 1 || !d_v || !d_out ||
      (k > 0 && (!d_rows || ld < n || !coef)))
    return LITHO_ERR_INVALID_ARGUMENT;
  if (d_out == d_v) return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "L-BFGS combine: out must not alias v");
  if (!std::isfinite(cv) || (k > 0 && !finite_all(coef, (size_t)k)))
    return ctx->fail(LITHO_ERR_NONFINITE, "L-BFGS combine: coefficients must be finite");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx->fail(LITHO_ERR_CUDA, "cudaSetDevice");
  int st = ctx->ensure_red(RED_PART + 64 + 8);
  if (st) return st;
  double* dc = ctx->d_red + RED_PART;
  if (k > 0)
    LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(dc, coef, (size_t)k * sizeof(double), cudaMemcpyHostToDevice,
                                        ctx->stream));
  ctx->launches += 1;
  return check_launch(ctx, launch_combine(ctx->stream, d_rows, (size_t)ld, k, (size_t)n, dc, d_v,
                                          cv, d_out),
                      "L-BFGS direction");
}

int litho_reinit_sdf_batch(litho_ctx* ctx, int batch, int rows, int cols, const float* d_phi,
                           double level, double dx, double dy, float* d_sdf, float* d_mask) {
  if (!ctx || batch < 1 || !d_phi || !d_sdf) return LITHO_ERR_INVALID_ARGUMENT;
  int st = ls_check(ctx, rows, cols, dx, dy, 1);
  if (st) return st;
  if (!std::isfinite(level)) return ctx->fail(LITHO_ERR_NONFINITE, "reinit_sdf: level must be finite");
  if ((size_t)3 * cols * sizeof(float) > 200 * 1024)
    return ctx->fail(LITHO_ERR_UNSUPPORTED, "reinit_sdf supports at most 17066 columns");
  if (d_sdf == d_phi || (d_mask && (d_mask == d_phi || d_mask == d_sdf)))
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "reinit_sdf: sdf, mask and phi must not alias");
  const size_t n = (size_t)rows * cols;
  for (int b0 = 0; b0 < batch && !st; b0 += 65535) {
    const int B = std::min(batch - b0, 65535);
    st = check_launch(ctx, launch_reinit_sdf(ctx->stream, rows, cols, d_phi + b0 * n, (float)level,
                                             0, (float)dx, d_sdf + b0 * n, B,
                                             ctx->chamfer_threads(cols, B)),
                      "reinit_sdf");
    if (!st && d_mask)
      st = check_launch(ctx, launch_levelset(ctx->stream, 5, rows, cols, d_sdf + b0 * n, nullptr,
                                             nullptr, (float)dx, (float)dy, 0.f, nullptr,
                                             d_mask + b0 * n, nullptr, nullptr, B),
                        "mask");
    ctx->launches += d_mask ? 2 : 1;
  }
  return st;
}

int litho_lsm_rk2_update(litho_ctx* ctx, int rows, int cols, const float* d_phi,
                         const float* d_vn, double dx, double dy, double cfl, double b,
                         float* d_phi_out, float* d_mask, double* dt) {
  if (!ctx || !d_phi || !d_vn || !d_phi_out) return LITHO_ERR_INVALID_ARGUMENT;
  int st = ls_check(ctx, rows, cols, dx, dy, 3);
  if (st) return st;
  const size_t n = (size_t)rows * cols;
  st = ctx->ensure_scratch(n * sizeof(float));
  if (st) return st;
  float* phi1 = static_cast<float*>(ctx->scratch.base);
  float* dtd = nullptr;
  st = ls_dt(ctx, rows, cols, d_vn, dx, dy, cfl, b, &dtd);
  if (st) return st;
  ctx->stage_begin(8);
  st = check_launch(ctx, launch_levelset(ctx->stream, 3, rows, cols, d_phi, nullptr, d_vn,
                                         (float)dx, (float)dy, (float)b, dtd, phi1, nullptr),
                    "rk2 stage 1");
  if (!st)
    st = check_launch(ctx, launch_levelset(ctx->stream, 4, rows, cols, phi1, d_phi, d_vn,
                                           (float)dx, (float)dy, (float)b, dtd, d_phi_out, d_mask),
                      "rk2 stage 2");
  ctx->stage_end(8);
  ctx->launches += 2;
  if (!st) st = fetch(ctx, 1);
  if (st) return st;
  if (flag_set(ctx)) return ctx->fail(LITHO_ERR_NONFINITE, "normal speed must be finite");
  float h[2];
  std::memcpy(h, ctx->h_red + RED_SUM, sizeof(h));
  if (dt) *dt = h[1];
  return LITHO_OK;
}

static int rk2_update_batch_impl(litho_ctx* ctx, int batch, int rows, int cols,
                                 const float* d_phi, const float* d_vn, double dx, double dy,
                                 double cfl, double b, float* d_phi_out, float* d_mask,
                                 double* dts, bool device_out, double* d_dts) {
  if (!ctx || batch < 1 || !d_phi || !d_vn || !d_phi_out) return LITHO_ERR_INVALID_ARGUMENT;
  if (d_phi_out == d_phi) return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "phi_out must not alias phi");
  int st = ls_check(ctx, rows, cols, dx, dy, 3);
  if (!st && device_out) st = ctx->ensure_deferred();
  if (st) return st;
  if (batch > 65535) return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "at most 65535 images per call");
  const size_t n = (size_t)rows * cols;
  st = ctx->ensure_scratch(n * batch * sizeof(float));
  if (st) return st;
  // Per-image absmax partials, then the per-image (max |Vn|, dt) pairs.
  const size_t nparts = (size_t)batch * dt_batch_blocks(n, batch);
  const size_t part_dbl = (nparts + 1) / 2 + 8;
  st = ctx->ensure_red(RED_PART + part_dbl + (size_t)batch + 8);
  if (st) return st;
  LITHO_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_red, 0, RED_PART * sizeof(double), ctx->stream));
  float* phi1 = static_cast<float*>(ctx->scratch.base);
  float* part = reinterpret_cast<float*>(ctx->d_red + RED_PART);
  float* vd = reinterpret_cast<float*>(ctx->d_red + RED_PART + part_dbl);   // [batch][2]
  int* bad = reinterpret_cast<int*>(ctx->d_red + RED_FLAG);
  cudaStream_t s = ctx->stream;
  // Every image in each launch: dt per image, then the two RK2 stages with dt[2 i + 1].
  st = check_launch(ctx, launch_dt_batch(s, d_vn, n, batch, (float)dx, (float)dy, (float)cfl,
                                         (float)b, part, vd, bad),
                    "dt");
  if (!st)
    st = check_launch(ctx, launch_levelset(s, 3, rows, cols, d_phi, nullptr, d_vn, (float)dx,
                                           (float)dy, (float)b, vd + 1, phi1, nullptr, nullptr,
                                           batch, nullptr, 2),
                      "rk2 stage 1");
  if (!st)
    st = check_launch(ctx, launch_levelset(s, 4, rows, cols, phi1, d_phi, d_vn, (float)dx,
                                           (float)dy, (float)b, vd + 1, d_phi_out, d_mask, nullptr,
                                           batch, nullptr, 2),
                      "rk2 stage 2");
  ctx->launches += 4;
  if (device_out) {
    if (!st && d_dts) {
      dt_export_kernel<<<(batch + 255) / 256, 256, 0, s>>>(vd, batch, d_dts);
      st = check_launch(ctx, cudaGetLastError(), "dt export");
      ctx->launches += 1;
    }
    if (!st) st = check_launch(ctx, launch_merge_deferred(s, bad, ctx->d_deferred), "deferred status");
    return st;
  }
  std::vector<float> h(2 * (size_t)batch);
  if (!st)
    LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(h.data(), vd, h.size() * sizeof(float),
                                        cudaMemcpyDeviceToHost, s));
  if (!st) st = fetch(ctx, 0);
  if (st) return st;
  if (flag_set(ctx)) return ctx->fail(LITHO_ERR_NONFINITE, "normal speed must be finite");
  for (int i = 0; i < batch && dts; ++i) dts[i] = h[2 * (size_t)i + 1];
  return LITHO_OK;
}

int litho_lsm_rk2_update_batch(litho_ctx* ctx, int batch, int rows, int cols, const float* d_phi,
                               const float* d_vn, double dx, double dy, double cfl, double b,
                               float* d_phi_out, float* d_mask, double* dts) {
  return rk2_update_batch_impl(ctx, batch, rows, cols, d_phi, d_vn, dx, dy, cfl, b, d_phi_out,
                               d_mask, dts, false, nullptr);
}

int litho_lsm_rk2_update_batch_device(litho_ctx* ctx, int batch, int rows, int cols,
                                      const float* d_phi, const float* d_vn, double dx, double dy,
                                      double cfl, double b, float* d_phi_out, float* d_mask,
                                      double* d_dts) {
  return rk2_update_batch_impl(ctx, batch, rows, cols, d_phi, d_vn, dx, dy, cfl, b, d_phi_out,
                               d_mask, nullptr, true, d_dts);
}

int litho_lsm_track_batch(litho_ctx* ctx, int batch, long long n_pixels, const double* d_losses,
                          double pen_weight, double* d_best, const float* d_masks,
                          float* d_best_masks, double* d_history, int history_cols, int* d_iters) {
  if (!ctx || batch < 1 || n_pixels < 1 || !d_losses || !d_best || !d_masks || !d_best_masks ||
      !d_iters || (d_history && history_cols < 1))
    return LITHO_ERR_INVALID_ARGUMENT;
  if (batch > 65535) return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "at most 65535 images per call");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx->fail(LITHO_ERR_CUDA, "cudaSetDevice");
  int st = ctx->ensure_red(RED_PART + (size_t)batch + 8);
  if (st) return st;
  int* improved = reinterpret_cast<int*>(ctx->d_red + RED_PART);
  cudaStream_t s = ctx->stream;
  track_scalars_kernel<<<(batch + 127) / 128, 128, 0, s>>>(batch, d_losses, pen_weight, d_best,
                                                            d_history, history_cols, d_iters,
                                                            improved);
  const long long blocks = std::min<long long>((n_pixels / 4 + 255) / 256 + 1, 148);
  const int vec = n_pixels % 4 == 0 && reinterpret_cast<uintptr_t>(d_masks) % 16 == 0 &&
                  reinterpret_cast<uintptr_t>(d_best_masks) % 16 == 0;
  track_masks_kernel<<<dim3((unsigned)blocks, batch), 256, 0, s>>>(n_pixels, vec, improved,
                                                                  d_masks, d_best_masks);
  ctx->launches += 2;
  return check_launch(ctx, cudaGetLastError(), "LSM best-state tracking");
}

int litho_ctx_deferred_status(litho_ctx* ctx) {
  if (!ctx) return LITHO_ERR_INVALID_ARGUMENT;
  if (!ctx->d_deferred) return LITHO_OK;
  int h[2] = {0, 0};
  LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(h, ctx->d_deferred, sizeof(h), cudaMemcpyDeviceToHost,
                                      ctx->stream));
  LITHO_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  LITHO_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_deferred, 0, sizeof(h), ctx->stream));
  if (h[1])
    return ctx->fail(LITHO_ERR_CUDA, "tensor-core pass: a bounded wait expired (code " +
                                         std::to_string(h[1]) + ")");
  if (h[0]) return ctx->fail(LITHO_ERR_NONFINITE, "a deferred call saw a non-finite input");
  return LITHO_OK;
}

}  // extern "C"

// ============================================================== full chip
struct litho_partition {
  int device = 0;
  int height = 0, width = 0, grid_rows = 0, grid_cols = 0, halo = 0, guard = 0;
  int ts = 0, ntiles = 0;
  static constexpr int kMaxRel = 4;
  std::vector<int> rects;  // 16 per tile: core_global, tile_global, core_local, update_local
  // Device metadata: origins (2/tile) | core_global | core_local | update_local (4/tile
  // each) | neighbour count (1/tile) | relations (kMaxRel * FC_REL_INTS per tile).
  int* d_meta = nullptr;
  size_t off_origin = 0, off_core_g = 0, off_core_l = 0, off_update = 0, off_nrel = 0, off_rel = 0;
  // Exchange work, allocated on first use: targets | pe windows | penalty windows |
  // raw gradients (ntiles * ts * ts floats each), the imaging field, loss sums.
  float* d_work = nullptr;
  float2* fe = nullptr;
  float2* fm = nullptr;
  size_t fe_n = 0, fm_n = 0;
  // Loss sums: kSlots per tile (see litho_exchange_compute_epe), then 1 per tile (CEPT).
  static constexpr int kSlots = 14;
  double* d_loss = nullptr;
  double* d_xpart = nullptr;   // exchange partial sums: ntiles * kMaxRel * 32

  std::vector<double> h_loss;
  // EPE work, allocated when an EPE term or the Core metrics are asked for: EPE
  // windows, the PE_EPE main region and its row-pass temporary (ntiles * ts * ts
  // each), then one tile each of aerial and wafer image.
  float* d_epe_work = nullptr;
  size_t epe_work_n = 0;
  // EPs as uploaded (y, x | w) and one tile's candidates (y, x | w), in doubles.
  double* d_ep = nullptr;
  size_t ep_n = 0;
  void* d_epe_sort = nullptr;   // work of the deterministic dL/dI scatter
  size_t epe_sort_bytes = 0;
};

namespace {

struct IRect {
  int y0, y1, x0, x1;
};
IRect irect_intersect(IRect a, IRect b) {
  return {std::max(a.y0, b.y0), std::min(a.y1, b.y1), std::max(a.x0, b.x0), std::min(a.x1, b.x1)};
}
IRect irect_grow(IRect a, int w) { return {a.y0 - w, a.y1 + w, a.x0 - w, a.x1 + w}; }
IRect irect_shift(IRect a, int dy, int dx) { return {a.y0 + dy, a.y1 + dy, a.x0 + dx, a.x1 + dx}; }
void put(std::vector<int>& v, size_t at, IRect r) {
  v[at] = r.y0; v[at + 1] = r.y1; v[at + 2] = r.x0; v[at + 3] = r.x1;
}

void free_partition(litho_partition* p) {
  cudaSetDevice(p->device);
  if (p->d_meta) cudaFree(p->d_meta);
  if (p->d_work) cudaFree(p->d_work);
  if (p->fe) cudaFree(p->fe);
  if (p->fm) cudaFree(p->fm);
  if (p->d_loss) cudaFree(p->d_loss);
  if (p->d_xpart) cudaFree(p->d_xpart);
  if (p->d_epe_work) cudaFree(p->d_epe_work);
  if (p->d_ep) cudaFree(p->d_ep);
  if (p->d_epe_sort) cudaFree(p->d_epe_sort);
}

}  // namespace


namespace {

// Partition::build (partition.cpp:21-80) over given Core boundaries: row r of the
// tile grid covers rows [row_cuts[r], row_cuts[r + 1]), column c columns
// [col_cuts[c], col_cuts[c + 1]); one square tile size = largest Core side + 2 halo,
// rounded up to even; tiles keyed row-major with their four-neighbour relations.
int partition_build(litho_ctx* ctx, int height, int width, const std::vector<int>& row_cuts,
                    const std::vector<int>& col_cuts, int halo, int guard, litho_partition** out) {
  const int grid_rows = (int)row_cuts.size() - 1, grid_cols = (int)col_cuts.size() - 1;
  auto* p = new (std::nothrow) litho_partition();
  if (!p) return ctx->fail(LITHO_ERR_OOM, "host allocation failed");
  p->device = ctx->device;
  p->height = height; p->width = width; p->grid_rows = grid_rows; p->grid_cols = grid_cols;
  p->halo = halo; p->guard = guard;
  int max_side = 0;
  for (int r = 0; r < grid_rows; ++r) max_side = std::max(max_side, row_cuts[r + 1] - row_cuts[r]);
  for (int c = 0; c < grid_cols; ++c) max_side = std::max(max_side, col_cuts[c + 1] - col_cuts[c]);
  int ts = max_side + 2 * halo;
  ts += ts % 2;
  p->ts = ts;
  const int n = grid_rows * grid_cols;
  p->ntiles = n;
  std::vector<IRect> core(n), tile(n);
  for (int r = 0; r < grid_rows; ++r)
    for (int c = 0; c < grid_cols; ++c) {
      const int id = r * grid_cols + c;
      core[id] = {row_cuts[r], row_cuts[r + 1], col_cuts[c], col_cuts[c + 1]};
      tile[id] = {core[id].y0 - halo, core[id].y0 - halo + ts, core[id].x0 - halo,
                  core[id].x0 - halo + ts};
    }
  const int R = litho_partition::kMaxRel;
  p->off_origin = 0;
  p->off_core_g = 2 * (size_t)n;
  p->off_core_l = p->off_core_g + 4 * (size_t)n;
  p->off_update = p->off_core_l + 4 * (size_t)n;
  p->off_nrel = p->off_update + 4 * (size_t)n;
  p->off_rel = p->off_nrel + (size_t)n;
  std::vector<int> meta(p->off_rel + (size_t)n * R * FC_REL_INTS, 0);
  p->rects.assign(16 * (size_t)n, 0);
  const int dirs[4][3] = {{0, -1, 0}, {0, 1, 1}, {-1, 0, 2}, {1, 0, 3}};  // left, right, top, bottom
  for (int id = 0; id < n; ++id) {
    const int r = id / grid_cols, c = id % grid_cols;
    const IRect cl = irect_shift(core[id], -tile[id].y0, -tile[id].x0);
    const IRect up = irect_grow(cl, guard);
    put(p->rects, 16 * (size_t)id, core[id]);
    put(p->rects, 16 * (size_t)id + 4, tile[id]);
    put(p->rects, 16 * (size_t)id + 8, cl);
    put(p->rects, 16 * (size_t)id + 12, up);
    meta[p->off_origin + 2 * id] = tile[id].y0;
    meta[p->off_origin + 2 * id + 1] = tile[id].x0;
    put(meta, p->off_core_g + 4 * (size_t)id, core[id]);
    put(meta, p->off_core_l + 4 * (size_t)id, cl);
    put(meta, p->off_update + 4 * (size_t)id, up);
    int k = 0;
    for (const auto& d : dirs) {
      const int rr = r + d[0], cc = c + d[1];
      if (rr < 0 || rr >= grid_rows || cc < 0 || cc >= grid_cols) continue;
      const int nb = rr * grid_cols + cc;
      const IRect gg = irect_intersect(irect_grow(core[id], guard), core[nb]);
      const IRect og = irect_intersect(core[id], irect_grow(core[nb], guard));
      const size_t at = p->off_rel + ((size_t)id * R + k) * FC_REL_INTS;
      meta[at] = nb;
      meta[at + 1] = d[2];
      put(meta, at + 2, irect_shift(gg, -tile[id].y0, -tile[id].x0));
      put(meta, at + 6, irect_shift(gg, -tile[nb].y0, -tile[nb].x0));
      put(meta, at + 10, irect_shift(og, -tile[id].y0, -tile[id].x0));
      put(meta, at + 14, irect_shift(og, -tile[nb].y0, -tile[nb].x0));
      ++k;
    }
    meta[p->off_nrel + id] = k;
  }
  if (cudaSetDevice(ctx->device) != cudaSuccess) {
    delete p;
    return ctx->fail(LITHO_ERR_CUDA, "cudaSetDevice");
  }
  int st = upload(ctx, &p->d_meta, meta);
  if (st) {
    free_partition(p);
    delete p;
    return st;
  }
  *out = p;
  return LITHO_OK;
}

}  // namespace

extern "C" {

int litho_partition_create(litho_ctx* ctx, int height, int width, int grid_rows, int grid_cols,
                           int halo, int guard, litho_partition** out) {
  if (!ctx || !out) return LITHO_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (height <= 0 || width <= 0 || grid_rows <= 0 || grid_cols <= 0 || grid_rows > height ||
      grid_cols > width || halo < 0 || guard < 0)
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "Partition: invalid layout or grid size");
  if (guard > halo)
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "Partition: guard must not exceed halo");
  // Core boundaries at i * extent / count (partition.cpp:37-38).
  std::vector<int> rc(grid_rows + 1), cc(grid_cols + 1);
  for (int r = 0; r <= grid_rows; ++r) rc[r] = (int)((long long)r * height / grid_rows);
  for (int c = 0; c <= grid_cols; ++c) cc[c] = (int)((long long)c * width / grid_cols);
  return partition_build(ctx, height, width, rc, cc, halo, guard, out);
}

int litho_partition_create_cuts(litho_ctx* ctx, int height, int width, int grid_rows,
                                const int* row_cuts, int grid_cols, const int* col_cuts, int halo,
                                int guard, litho_partition** out) {
  if (!ctx || !out || !row_cuts || !col_cuts) return LITHO_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (height <= 0 || width <= 0 || grid_rows <= 0 || grid_cols <= 0 || halo < 0 || guard < 0)
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "Partition: invalid layout or grid size");
  if (guard > halo)
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "Partition: guard must not exceed halo");
  std::vector<int> rc(row_cuts, row_cuts + grid_rows + 1), cc(col_cuts, col_cuts + grid_cols + 1);
  auto valid = [&](const std::vector<int>& cuts, int extent) {
    if (cuts.front() != 0 || cuts.back() != extent) return false;
    for (size_t i = 0; i + 1 < cuts.size(); ++i)
      if (cuts[i + 1] - cuts[i] < std::max(1, guard)) return false;
    return true;
  };
  // Every Core at least as wide as the guard: a tile's guard band then reaches only its
  // four neighbours' Cores, the relations the exchange evaluates.
  if (!valid(rc, height) || !valid(cc, width))
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT,
                     "Partition: cuts must run from 0 to the extent, each Core at least the guard wide");
  return partition_build(ctx, height, width, rc, cc, halo, guard, out);
}

int litho_partition_destroy(litho_partition* p) {
  if (!p) return LITHO_OK;
  free_partition(p);
  delete p;
  return LITHO_OK;
}

int litho_partition_info(const litho_partition* p, int* num_tiles, int* tile_size) {
  if (!p) return LITHO_ERR_INVALID_ARGUMENT;
  if (num_tiles) *num_tiles = p->ntiles;
  if (tile_size) *tile_size = p->ts;
  return LITHO_OK;
}

int litho_partition_tile_rects(const litho_partition* p, int tile, int* rects) {
  if (!p || !rects || tile < 0 || tile >= p->ntiles) return LITHO_ERR_INVALID_ARGUMENT;
  std::memcpy(rects, p->rects.data() + 16 * (size_t)tile, 16 * sizeof(int));
  return LITHO_OK;
}

int litho_partition_extract(litho_ctx* ctx, const litho_partition* p, const float* d_global,
                            float* d_tiles) {
  if (!ctx || !p || !d_global || !d_tiles) return LITHO_ERR_INVALID_ARGUMENT;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx->fail(LITHO_ERR_CUDA, "cudaSetDevice");
  ctx->launches += 1;
  return check_launch(ctx, launch_tiles_extract(ctx->stream, d_global, p->height, p->width,
                                                p->ntiles, p->d_meta + p->off_origin, p->ts,
                                                d_tiles),
                      "tile extraction");
}

int litho_partition_assemble(litho_ctx* ctx, const litho_partition* p, const float* d_tiles,
                             float* d_global) {
  if (!ctx || !p || !d_global || !d_tiles) return LITHO_ERR_INVALID_ARGUMENT;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx->fail(LITHO_ERR_CUDA, "cudaSetDevice");
  ctx->launches += 1;
  return check_launch(ctx, launch_tiles_assemble(ctx->stream, d_tiles, p->ntiles, p->ts,
                                                 p->d_meta + p->off_core_g,
                                                 p->d_meta + p->off_core_l, p->width, d_global),
                      "tile assembly");
}

// Tiles per batched pass of the exchange (tensor-core path): every tile of the
// partition in one pass while the pass's scratch stays within kExchangeBudget bytes
// (about 4.6 MB per 1280^2 tile at K = 24: 256 such tiles take 1.2 GB), and at least
// kExchangeGroup tiles.
constexpr int kExchangeGroup = 16;
constexpr size_t kExchangeBudget = (size_t)4 << 30;
int exchange_group(const Context* ctx, const BandGeom& g, int n) {
  if (ctx->exchange_group_max > 0) return std::min(n, ctx->exchange_group_max);
  const size_t per = make_layout(g, 2, true).total - make_layout(g, 1, true).total;
  const size_t fit = kExchangeBudget / std::max<size_t>(per, 1);
  return (int)std::min<size_t>((size_t)n, std::max<size_t>(kExchangeGroup, fit));
}

int litho_exchange_compute_epe(litho_ctx* ctx, const litho_partition* cp, const litho_cache* cache,
                               const float* d_masks, const float* d_global_target, double threshold,
                               double alpha, const litho_exchange_options* opt,
                               const litho_exchange_epe* epe_in, float* d_raw, float* d_grad,
                               double* tile_metrics, double* totals) {
  if (!ctx || !cp || !cache || !d_masks || !d_global_target || !d_grad)
    return LITHO_ERR_INVALID_ARGUMENT;
  auto* p = const_cast<litho_partition*>(cp);  // owns mutable work buffers only
  litho_exchange_options o{LITHO_MICRO_LOSS_PE, LITHO_MICRO_REGION_CORE, 1.0, 2.0, 0.01, 0, 0,
                           1.1, 0, LITHO_FUSION_AVERAGE, 0.5, 0.5};
  if (opt) o = *opt;
  litho_exchange_epe e{1.0, 2, 1.0, 0, nullptr, nullptr, 0};
  if (epe_in) e = *epe_in;
  if (o.loss_type < LITHO_MICRO_LOSS_PE || o.loss_type > LITHO_MICRO_LOSS_PE_EPE ||
      (o.loss_region != LITHO_MICRO_REGION_CORE && o.loss_region != LITHO_MICRO_REGION_CORE_GUARD) ||
      (o.fusion_mode != LITHO_FUSION_AVERAGE && o.fusion_mode != LITHO_FUSION_LINEAR))
    return ctx->fail(LITHO_ERR_UNSUPPORTED, "MicroGradientOptions: unsupported loss type, region or fusion mode");
  const double w10[] = {o.pe_weight, o.penalty_weight, o.penalty_threshold, o.cept_weight,
                        o.fusion_weight_owner, o.fusion_weight_neighbor, threshold, alpha,
                        e.epe_weight, e.epe_pixel_size};
  if (!finite_all(w10, 10))
    return ctx->fail(LITHO_ERR_NONFINITE, "MicroGradientOptions: weights must be finite");
  if (o.enable_grad_fusion && (o.fusion_weight_owner < 0.0 || o.fusion_weight_neighbor < 0.0 ||
                               o.fusion_weight_owner + o.fusion_weight_neighbor <= 0.0))
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT,
                     "MicroGradientOptions: fusion weights must be non-negative with a positive sum");
  if (e.n_eps < 0 || (e.n_eps > 0 && (!e.eps || !e.weights)) || e.main_region_dilation_pixels < 0)
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT,
                     "MicroGradientOptions: EPs need coordinates and weights; dilation must be >= 0");
  if (!finite_all(e.eps, 2 * (size_t)e.n_eps) || !finite_all(e.weights, (size_t)e.n_eps))
    return ctx->fail(LITHO_ERR_NONFINITE, "MicroGradientExchange: EP coordinates and weights must be finite");
  if (cache->g.N != p->ts)
    return ctx->fail(LITHO_ERR_SHAPE, "MicroGradientExchange: cache N must equal the tile size");
  if (d_raw && d_raw == d_grad)
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "raw and exchanged gradients must not alias");
  const int n = p->ntiles, ts = p->ts;
  const size_t tt = (size_t)ts * ts;
  const int S = litho_partition::kSlots;
  const bool epe_terms = o.loss_type == LITHO_MICRO_LOSS_EPE || o.loss_type == LITHO_MICRO_LOSS_PE_EPE;
  const bool core = e.collect_core_metrics != 0;
  const bool eval_epe = epe_terms || core;   // micro_gradient_exchange.cpp:144-148
  // Tensor-core path: the tiles go through the imaging + adjoint chain in groups
  // (exchange_group: normally all of them), one batched pass per group (the EP work
  // stays per tile between the forward and the adjoint pass).
  const bool batched = ctx->precision == LITHO_PRECISION_BF16X3 && cache->TXD_img != nullptr &&
                       n > 1;
  const int group = batched ? exchange_group(ctx, cache->g, n) : 1;
  Layout L;
  int st = prepare(ctx, *cache, &L, group, batched);
  if (st) return st;
  const bool guard_region = o.loss_region == LITHO_MICRO_REGION_CORE_GUARD;
  const int periods = guard_region ? 1 : 0;
  const size_t ncand = (size_t)e.n_eps * (2 * periods + 1) * (2 * periods + 1);
  if (ncand > (size_t)1 << 28)   // the sorted scatter takes 4 entries per candidate
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "MicroGradientExchange: too many EPs");
  if (!p->d_work) {
    if (cudaMalloc(&p->d_work, 4 * n * tt * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&p->d_loss, (size_t)(S + 1) * n * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&p->d_xpart, (size_t)litho_partition::kMaxRel * n * 32 * sizeof(double)) !=
            cudaSuccess) {
      cudaGetLastError();
      return ctx->fail(LITHO_ERR_OOM, "full-chip work allocation failed");
    }
    p->h_loss.assign((size_t)(S + 1) * n, 0.0);
  }
  // EP work: EPE window, main region, dilation scratch (n tiles each), then the
  // aerial and wafer images and the dL/dI of a group of tiles.
  const size_t epe_work_n = eval_epe ? (3 * (size_t)n + 3 * (size_t)group) * tt : 0;
  const size_t ep_n = eval_epe ? 3 * ((size_t)e.n_eps + ncand) : 0;
  if (p->epe_work_n < epe_work_n || p->ep_n < ep_n) {
    LITHO_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (p->epe_work_n < epe_work_n) {
      if (p->d_epe_work) cudaFree(p->d_epe_work);
      p->d_epe_work = nullptr; p->epe_work_n = 0;
      if (cudaMalloc(&p->d_epe_work, epe_work_n * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        return ctx->fail(LITHO_ERR_OOM, "full-chip EPE work allocation failed");
      }
      p->epe_work_n = epe_work_n;
    }
    if (p->ep_n < ep_n) {
      if (p->d_ep) cudaFree(p->d_ep);
      p->d_ep = nullptr; p->ep_n = 0;
      if (cudaMalloc(&p->d_ep, ep_n * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return ctx->fail(LITHO_ERR_OOM, "full-chip EP allocation failed");
      }
      p->ep_n = ep_n;
    }
  }
  const size_t sort_bytes = eval_epe ? epe_scatter_work_bytes((int)ncand) : 0;
  if (p->epe_sort_bytes < sort_bytes) {
    LITHO_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (p->d_epe_sort) cudaFree(p->d_epe_sort);
    p->d_epe_sort = nullptr; p->epe_sort_bytes = 0;
    if (cudaMalloc(&p->d_epe_sort, sort_bytes) != cudaSuccess) {
      cudaGetLastError();
      return ctx->fail(LITHO_ERR_OOM, "full-chip EPE scatter allocation failed");
    }
    p->epe_sort_bytes = sort_bytes;
  }
  const BandGeom& g = cache->g;
  const size_t fe_n = (size_t)g.K * g.Pr * g.Pc, fm_n = (size_t)g.Nr * g.Nc;
  if (p->fe_n < fe_n || p->fm_n < fm_n) {
    LITHO_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (p->fe) cudaFree(p->fe);
    if (p->fm) cudaFree(p->fm);
    p->fe = nullptr; p->fm = nullptr; p->fe_n = p->fm_n = 0;
    if (cudaMalloc(&p->fe, fe_n * sizeof(float2)) != cudaSuccess ||
        cudaMalloc(&p->fm, fm_n * sizeof(float2)) != cudaSuccess) {
      cudaGetLastError();
      return ctx->fail(LITHO_ERR_OOM, "full-chip field allocation failed");
    }
    p->fe_n = fe_n; p->fm_n = fm_n;
  }
  // Per-block partials of the EPE and rectangle sums share the reduction area.
  const int epe_blocks = ncand == 0 ? 1 : (int)((ncand + 255) / 256);
  st = ctx->ensure_red(RED_PART + std::max<size_t>(3 * (size_t)std::max(epe_blocks, 64) + 8,
                                                   6 * ((size_t)rect_losses_batch_blocks(ts) + 1) *
                                                           group + 8));
  if (st) return st;
  LITHO_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_red, 0, RED_PART * sizeof(double), ctx->stream));
  float* targets = p->d_work;
  float* pe_w = targets + n * tt;
  float* pen_w = pe_w + n * tt;
  float* raw = d_raw ? d_raw : pen_w + n * tt;
  float* epe_w = eval_epe ? p->d_epe_work : nullptr;
  float* main_dil = eval_epe ? epe_w + n * tt : nullptr;
  float* dil_tmp = eval_epe ? main_dil + n * tt : nullptr;
  float* aerial = eval_epe ? dil_tmp + n * tt : nullptr;
  float* wafer = eval_epe ? aerial + group * tt : nullptr;
  float* dldi_group = eval_epe ? wafer + group * tt : nullptr;
  double* ep_in = p->d_ep;                                   // 2 n_eps coordinates | n_eps weights
  double* cand = eval_epe ? ep_in + 3 * (size_t)e.n_eps : nullptr;   // 2 ncand | ncand
  Field f;
  f.cache = cache; f.e = p->fe; f.mband = p->fm;
  cudaStream_t s = ctx->stream;
  float* dldi = at<float>(ctx, L.dldi);
  double* part = ctx->d_red + RED_PART;
  LITHO_CUDA_TRY(ctx, cudaMemsetAsync(p->d_loss, 0, (size_t)(S + 1) * n * sizeof(double), s));
  if (eval_epe && e.n_eps > 0) {
    LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(ep_in, e.eps, 2 * (size_t)e.n_eps * sizeof(double),
                                        cudaMemcpyHostToDevice, s));
    LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(ep_in + 2 * (size_t)e.n_eps, e.weights,
                                        (size_t)e.n_eps * sizeof(double), cudaMemcpyHostToDevice, s));
  }
  st = check_launch(ctx, launch_tiles_extract(s, d_global_target, p->height, p->width, n,
                                              p->d_meta + p->off_origin, ts, targets),
                    "target extraction");
  const bool pe_epe = o.loss_type == LITHO_MICRO_LOSS_PE_EPE;
  if (!st && pe_epe)
    st = check_launch(ctx, launch_dilate_main(s, targets, n, ts, e.main_region_dilation_pixels,
                                              dil_tmp, main_dil),
                      "main-region dilation");
  if (!st)
    st = check_launch(ctx, launch_loss_windows(s, targets, n, ts,
                                               p->d_meta + (guard_region ? p->off_update : p->off_core_l),
                                               o.loss_type, pe_epe ? main_dil : nullptr, pe_w, pen_w,
                                               epe_w),
                      "loss windows");
  ctx->launches += 2 + (pe_epe ? 2 : 0);
  // micro_loss_weights (micro_gradient_exchange.cpp:95-99).
  const double wpe = o.loss_type == LITHO_MICRO_LOSS_EPE ? 0.0 : o.pe_weight;
  const double wepe = epe_terms ? e.epe_weight : 0.0;
  const double wpen = o.loss_type == LITHO_MICRO_LOSS_PE_PENALTY ? o.penalty_weight : 0.0;
  // One adjoint per tile: dL/dI = PE part (written by the resist epilogue, adjoint scale
  // 4 alpha) + wepe * EPE part (adjoint scale 2), the latter pre-scaled onto 4 alpha.
  const bool epe_grad = epe_terms && wepe != 0.0;
  double adj_scale = 4.0 * alpha, epe_fac = 0.0;
  bool zero_pe_dldi = false;
  if (epe_grad) {
    if (adj_scale != 0.0) {
      epe_fac = 2.0 * wepe / adj_scale;
    } else {
      adj_scale = 2.0 * wepe;   // alpha = 0: the PE part is multiplied by 0 anyway
      epe_fac = 1.0;
      zero_pe_dldi = true;
    }
  }
  // Per-tile EP work after the forward pass of tile t (aerial / wafer images and dL/dI
  // of that tile at the given pointers): loss-region EPs (periodic copies with a
  // Core + Guard region) give the EPE sums and, for the EPE types, the scatter of
  // their dL/dI; with the Core metrics, the loss-region and Core sums from the wafer
  // image and the Core EPs without copies.
  auto ep_work = [&](int t, const float* aer, const float* waf, float* dl, bool rects) -> int {
    const int* R = &p->rects[16 * (size_t)t];   // core_global | tile_global | core_local | update_local
    const int* region = guard_region ? R + 12 : R + 8;
    const int oy = R[4], ox = R[6];
    double* slot = p->d_loss + (size_t)S * t;
    const int grect[4] = {region[0] + oy, region[1] + oy, region[2] + ox, region[3] + ox};
    int used = 0;
    int r = LITHO_OK;
    // Without EPs the EPE sums and counts stay at their zeroed slots.
    const bool eps_any = e.n_eps > 0;
    if (eps_any) {
      r = check_launch(ctx, launch_ep_candidates(s, ep_in, ep_in + 2 * (size_t)e.n_eps, e.n_eps,
                                                 periods, p->height, p->width, oy, ox, grect, ts,
                                                 epe_w + t * tt, cand, cand + 2 * ncand),
                       "EP candidates");
      if (!r)
        r = check_launch(ctx, launch_epe(s, aer, ts, ts, cand, cand + 2 * ncand, (int)ncand,
                                         threshold, e.epe_pixel_size, nullptr, part,
                                         epe_grad ? dl : nullptr, epe_fac, &used, p->d_epe_sort,
                                         p->epe_sort_bytes),
                         "sparse EPE");
      if (!r) r = check_launch(ctx, launch_sum_partials(s, part, used, 3, slot + 2), "sum");
      ctx->launches += 3;
    }
    if (r || !core) return r;
    if (rects) {
      // Loss-region and Core sums of this tile in one pass, straight to slots 5..10.
      r = check_launch(ctx, launch_rect_losses_batch(
                                s, waf, targets + t * tt, pe_w + t * tt, pen_w + t * tt, ts,
                                p->d_meta + (guard_region ? p->off_update : p->off_core_l) + 4 * t,
                                p->d_meta + p->off_core_l + 4 * t, (float)o.penalty_threshold,
                                part, 1),
                       "region and core losses");
      if (!r)
        r = check_launch(ctx, launch_sum_partials_batch(s, part, rect_losses_batch_blocks(ts), 6,
                                                        part, 0, 0, slot + 5, 1),
                         "sum");
      ctx->launches += 2;
    }
    const int crect[4] = {R[0], R[1], R[2], R[3]};   // core_global
    if (!r && eps_any) {
      r = check_launch(ctx, launch_ep_candidates(s, ep_in, ep_in + 2 * (size_t)e.n_eps, e.n_eps,
                                                 0, p->height, p->width, oy, ox, crect, ts,
                                                 epe_w + t * tt, cand, cand + 2 * ncand),
                       "core EP candidates");
      if (!r)
        r = check_launch(ctx, launch_epe(s, aer, ts, ts, cand, cand + 2 * ncand, e.n_eps,
                                         threshold, e.epe_pixel_size, nullptr, part, nullptr, 0.0,
                                         &used),
                         "core sparse EPE");
      if (!r) r = check_launch(ctx, launch_sum_partials(s, part, used, 3, slot + 11), "sum");
      ctx->launches += 3;
    }
    return r;
  };
  // With an EPE gradient the adjoint needs dL/dI after the EP scatter, so the resist
  // synthesis stores it; otherwise it stays on chip (fused adjoint tile analysis).
  const bool fuse = !epe_grad;
  for (int t0 = 0; batched && t0 < n && !st; t0 += group) {
    // Tiles t0 .. t0 + B - 1 in one pass: windows and penalty in the resist epilogue,
    // raw gradients straight to their slots, per-tile {PE, penalty} sums to the
    // first two loss slots.
    const int B = std::min(group, n - t0);
    Field fb;
    fb.cache = cache;
    fb.e = at<float2>(ctx, L.fe);
    fb.mband = at<float2>(ctx, L.fm);
    ResistEpilogue ep{};
    ep.mode = 1;
    ep.thr = (float)threshold;
    ep.alpha = (float)alpha;
    ep.aerial = eval_epe ? aerial : nullptr;
    ep.wafer = core ? wafer : nullptr;
    ep.target = targets + t0 * tt;
    ep.pe_window = pe_w + t0 * tt;
    ep.pen_window = pen_w + t0 * tt;
    ep.pe_weight = (float)wpe;
    ep.penalty = (float)wpen;
    ep.pen_thr = (float)o.penalty_threshold;
    ep.dldi = fuse ? nullptr : dldi_group;
    ep.loss_partial = part;
    int nb = 0, nb2 = 0;
    st = run_forward(ctx, *cache, fb, L, 0, d_masks + t0 * tt, nullptr, ep, &nb, nullptr, fuse, B);
    double* sums = part + 2 * (size_t)nb * B;
    if (!st)
      st = check_launch(ctx, launch_sum_partials_batch(s, part, nb, 2, part, 0, 0, sums, B), "sum");
    ctx->launches += 1;
    if (!st)
      LITHO_CUDA_TRY(ctx, cudaMemcpy2DAsync(p->d_loss + (size_t)S * t0, S * sizeof(double), sums,
                                            2 * sizeof(double), 2 * sizeof(double), B,
                                            cudaMemcpyDeviceToDevice, s));
    if (!st && zero_pe_dldi)
      LITHO_CUDA_TRY(ctx, cudaMemsetAsync(dldi_group, 0, B * tt * sizeof(float), s));
    if (!st && core) {
      // Loss-region and Core sums of the group's tiles in one launch, to slots 5..10.
      const int nbr = rect_losses_batch_blocks(ts);
      double* sums6 = part + 6 * (size_t)nbr * B;
      st = check_launch(ctx, launch_rect_losses_batch(
                                 s, wafer, targets + t0 * tt, pe_w + t0 * tt, pen_w + t0 * tt, ts,
                                 p->d_meta + (guard_region ? p->off_update : p->off_core_l) + 4 * t0,
                                 p->d_meta + p->off_core_l + 4 * t0, (float)o.penalty_threshold,
                                 part, B),
                        "region and core losses");
      if (!st)
        st = check_launch(ctx, launch_sum_partials_batch(s, part, nbr, 6, part, 0, 0, sums6, B),
                          "sum");
      if (!st)
        LITHO_CUDA_TRY(ctx, cudaMemcpy2DAsync(p->d_loss + (size_t)S * t0 + 5, S * sizeof(double),
                                              sums6, 6 * sizeof(double), 6 * sizeof(double), B,
                                              cudaMemcpyDeviceToDevice, s));
      ctx->launches += 2;
    }
    for (int b = 0; eval_epe && b < B && !st; ++b)
      st = ep_work(t0 + b, aerial + b * tt, core ? wafer + b * tt : nullptr,
                   fuse ? nullptr : dldi_group + b * tt, false);
    GradEpilogue gp{};
    gp.grad_mask = raw + t0 * tt;
    if (!st)
      st = run_adjoint(ctx, *cache, fb, L, fuse ? nullptr : dldi_group, adj_scale, gp, &nb2, fuse, B);
  }
  for (int t = 0; !batched && t < n && !st; ++t) {
    ResistEpilogue ep{};
    ep.mode = 1;
    ep.thr = (float)threshold;
    ep.alpha = (float)alpha;
    ep.aerial = eval_epe ? aerial : nullptr;
    ep.wafer = core ? wafer : nullptr;
    ep.target = targets + t * tt;
    ep.pe_window = pe_w + t * tt;
    ep.pen_window = pen_w + t * tt;
    ep.pe_weight = (float)wpe;
    ep.penalty = (float)wpen;
    ep.pen_thr = (float)o.penalty_threshold;
    ep.dldi = dldi;
    ep.loss_partial = part;
    double* slot = p->d_loss + (size_t)S * t;
    int nb = 0;
    st = run_forward(ctx, *cache, f, L, 0, d_masks + t * tt, nullptr, ep, &nb);
    if (!st) st = check_launch(ctx, launch_sum_partials(s, part, nb, 2, slot), "sum");
    ctx->launches += 1;
    if (!st && zero_pe_dldi) LITHO_CUDA_TRY(ctx, cudaMemsetAsync(dldi, 0, tt * sizeof(float), s));
    if (!st && eval_epe) st = ep_work(t, aerial, wafer, dldi, true);
    GradEpilogue gp{};
    gp.grad_mask = raw + t * tt;
    int nb2 = 0;
    if (!st) st = run_adjoint(ctx, *cache, f, L, dldi, adj_scale, gp, &nb2);
  }
  if (!st)
    LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(d_grad, raw, n * tt * sizeof(float),
                                        cudaMemcpyDeviceToDevice, s));
  if (!st)
    st = check_launch(ctx, launch_exchange(s, d_masks, raw, n, ts, p->d_meta + p->off_nrel,
                                           p->d_meta + p->off_rel, litho_partition::kMaxRel, o,
                                           d_grad, p->d_loss + (size_t)S * n, p->d_xpart),
                      "micro-gradient exchange");
  ctx->launches += 1;
  if (!st)
    LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(p->h_loss.data(), p->d_loss,
                                        (size_t)(S + 1) * n * sizeof(double),
                                        cudaMemcpyDeviceToHost, s));
  if (!st) st = fetch(ctx, 0);
  if (st) return st;
  if (flag_set(ctx)) return ctx->fail(LITHO_ERR_NONFINITE, "Imaging: mask, threshold, and alpha must be finite");
  double tot[3] = {0.0, 0.0, 0.0};
  const bool report_bg = o.loss_type == LITHO_MICRO_LOSS_PE_PENALTY || core;
  for (int t = 0; t < n; ++t) {
    const double* h = &p->h_loss[(size_t)S * t];
    // With the wafer image at hand the loss-region sums come from it; otherwise from
    // the resist epilogue (whose background sum runs only under a penalty).
    const double pe = core ? h[5] : h[0];
    const double bg = core ? h[6] : h[1];
    const double cept = p->h_loss[(size_t)S * n + t];
    const double epe_loss = eval_epe ? h[2] : 0.0;
    const double data = wpe * pe + wpen * bg + wepe * epe_loss;
    const double loss = data + (o.enable_cept ? o.cept_weight * cept : 0.0);
    if (tile_metrics) {
      double* r = tile_metrics + (size_t)LITHO_EXCHANGE_TILE_METRICS * t;
      std::fill(r, r + LITHO_EXCHANGE_TILE_METRICS, 0.0);
      r[LITHO_TM_PE_LOSS] = pe;
      r[LITHO_TM_BG_PENALTY_RAW] = report_bg ? bg : 0.0;
      r[LITHO_TM_PENALTY_LOSS] = wpen * bg;
      r[LITHO_TM_EPE_LOSS] = epe_loss;
      r[LITHO_TM_EPE_ABS_SUM_NM] = eval_epe ? h[3] : 0.0;
      r[LITHO_TM_EPE_COUNT] = eval_epe ? h[4] : 0.0;
      r[LITHO_TM_DATA_LOSS] = data;
      r[LITHO_TM_CEPT_LOSS] = cept;
      r[LITHO_TM_LOSS] = loss;
      if (core) {
        const double cnt = h[13];
        r[LITHO_TM_CORE_PE_LOSS] = h[8];
        r[LITHO_TM_CORE_BG_PENALTY_RAW] = h[9];
        r[LITHO_TM_CORE_PE_PENALTY_LOSS] = o.pe_weight * h[10] + o.penalty_weight * h[9];
        r[LITHO_TM_CORE_EPE_LOSS] = h[11];
        r[LITHO_TM_CORE_EPE_ABS_SUM_NM] = h[12];
        r[LITHO_TM_CORE_EP_COUNT] = cnt;
        r[LITHO_TM_CORE_EPE_MEAN] = cnt == 0.0 ? 0.0 : h[12] / cnt;
        r[LITHO_TM_CORE_DATA_LOSS] = wpe * h[8] + wpen * h[9] + wepe * h[11];
      }
    }
    tot[0] += loss; tot[1] += data; tot[2] += cept;
  }
  if (totals) std::memcpy(totals, tot, sizeof(tot));
  return LITHO_OK;
}

int litho_exchange_compute(litho_ctx* ctx, const litho_partition* cp, const litho_cache* cache,
                           const float* d_masks, const float* d_global_target, double threshold,
                           double alpha, const litho_exchange_options* opt, float* d_raw,
                           float* d_grad, double* tile_losses, double* totals) {
  if (!ctx || !cp) return LITHO_ERR_INVALID_ARGUMENT;
  std::vector<double> m((size_t)LITHO_EXCHANGE_TILE_METRICS * cp->ntiles);
  const int st = litho_exchange_compute_epe(ctx, cp, cache, d_masks, d_global_target, threshold,
                                            alpha, opt, nullptr, d_raw, d_grad, m.data(), totals);
  if (st || !tile_losses) return st;
  for (int t = 0; t < cp->ntiles; ++t) {
    const double* r = &m[(size_t)LITHO_EXCHANGE_TILE_METRICS * t];
    double* o = tile_losses + 5 * (size_t)t;
    o[0] = r[LITHO_TM_PE_LOSS]; o[1] = r[LITHO_TM_BG_PENALTY_RAW]; o[2] = r[LITHO_TM_DATA_LOSS];
    o[3] = r[LITHO_TM_CEPT_LOSS]; o[4] = r[LITHO_TM_LOSS];
  }
  return LITHO_OK;
}

int litho_fullchip_theta_step(litho_ctx* ctx, const litho_partition* p, float* d_theta,
                              const float* d_grad, double learning_rate, float* d_masks) {
  if (!ctx || !p || !d_theta || !d_masks) return LITHO_ERR_INVALID_ARGUMENT;
  if (!std::isfinite(learning_rate))
    return ctx->fail(LITHO_ERR_NONFINITE, "learning rate must be finite");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx->fail(LITHO_ERR_CUDA, "cudaSetDevice");
  ctx->launches += 1;
  return check_launch(ctx, launch_theta_update(ctx->stream, d_theta, d_grad, p->ntiles, p->ts,
                                               p->d_meta + p->off_update, (float)learning_rate,
                                               d_masks),
                      "theta update");
}

}  // extern "C"

extern "C" {

int litho_render_levelset_mask(litho_ctx* ctx, int rows, int cols, const float* d_phi,
                               int mask_type, int scale, float* d_mask) {
  if (!ctx || !d_phi || !d_mask || rows <= 0 || cols <= 0) return LITHO_ERR_INVALID_ARGUMENT;
  if (mask_type != LITHO_MASK_BINARY && mask_type != LITHO_MASK_GRAY)
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "render_levelset_mask: unknown mask type");
  if (mask_type == LITHO_MASK_GRAY && (scale < 1 || scale > 64))
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "render_levelset_mask: scale must be in 1..64");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx->fail(LITHO_ERR_CUDA, "cudaSetDevice");
  ctx->launches += 1;
  int st = check_launch(ctx, launch_render_mask(ctx->stream, d_phi, rows, cols, 1,
                                                mask_type == LITHO_MASK_GRAY, scale, d_mask),
                        "render_levelset_mask");
  if (!st) LITHO_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return st;
}

int litho_fullchip_lsm_init(litho_ctx* ctx, const litho_partition* p, const float* d_global_mask,
                            double dx, double dy, int mask_type, int scale, float* d_phi,
                            float* d_masks) {
  if (!ctx || !p || !d_global_mask || !d_phi || !d_masks) return LITHO_ERR_INVALID_ARGUMENT;
  if (!(dx > 0.0) || !(dy > 0.0))
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "full-chip LSM: dx and dy must be positive");
  if ((mask_type != LITHO_MASK_BINARY && mask_type != LITHO_MASK_GRAY) ||
      (mask_type == LITHO_MASK_GRAY && (scale < 1 || scale > 64)))
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "full-chip LSM: bad mask type or scale");
  if ((size_t)3 * p->ts * sizeof(float) > 200 * 1024)
    return ctx->fail(LITHO_ERR_UNSUPPORTED, "reinit_sdf supports at most 17066 columns");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx->fail(LITHO_ERR_CUDA, "cudaSetDevice");
  if (d_phi == d_masks) return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "full-chip LSM: phi must not alias the masks");
  cudaStream_t s = ctx->stream;
  // The extracted masks go to d_masks first (they are replaced by the renders below).
  int st = check_launch(ctx, launch_tiles_extract(s, d_global_mask, p->height, p->width, p->ntiles,
                                                  p->d_meta + p->off_origin, p->ts, d_masks),
                        "tile extraction");
  // reinit_sdf(mask - 0.5) of every tile at once: mask - 0.5 > 0 exactly when mask > 0.5.
  for (int t0 = 0; t0 < p->ntiles && !st; t0 += 65535)
    st = check_launch(ctx, launch_reinit_sdf(s, p->ts, p->ts, d_masks + (size_t)t0 * p->ts * p->ts,
                                             0.5f, 0, (float)dx, d_phi + (size_t)t0 * p->ts * p->ts,
                                             std::min(p->ntiles - t0, 65535),
                                             ctx->chamfer_threads(p->ts,
                                                                  std::min(p->ntiles - t0, 65535))),
                      "reinit_sdf");
  if (!st)
    st = check_launch(ctx, launch_render_mask(s, d_phi, p->ts, p->ts, p->ntiles,
                                              mask_type == LITHO_MASK_GRAY, scale, d_masks),
                      "render_levelset_mask");
  ctx->launches += 3;
  if (!st) LITHO_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  return st;
}

int litho_fullchip_lsm_step(litho_ctx* ctx, const litho_partition* p, const float* d_phi,
                            const float* d_grad, double dx, double dy, double cfl, double b,
                            int reinit, int mask_type, int scale, float* d_phi_out,
                            float* d_masks, double* dt_min, double* dt_max) {
  if (!ctx || !p || !d_phi || !d_grad || !d_phi_out || !d_masks) return LITHO_ERR_INVALID_ARGUMENT;
  if (d_phi_out == d_phi || d_masks == d_phi || d_masks == d_phi_out)
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT,
                     "full-chip LSM: phi, phi_out and the masks must not alias");
  if (!(dx > 0.0) || !(dy > 0.0) || !std::isfinite(cfl) || !std::isfinite(b))
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "full-chip LSM: dx, dy must be positive");
  if ((mask_type != LITHO_MASK_BINARY && mask_type != LITHO_MASK_GRAY) ||
      (mask_type == LITHO_MASK_GRAY && (scale < 1 || scale > 64)))
    return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "full-chip LSM: bad mask type or scale");
  if (p->ts < 3) return ctx->fail(LITHO_ERR_SHAPE, "curvature needs at least 3 rows and 3 columns");
  if ((size_t)3 * p->ts * sizeof(float) > 200 * 1024)
    return ctx->fail(LITHO_ERR_UNSUPPORTED, "reinit_sdf supports at most 17066 columns");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx->fail(LITHO_ERR_CUDA, "cudaSetDevice");
  const size_t tt = (size_t)p->ts * p->ts;
  const int n = p->ntiles, ts = p->ts;
  // Tiles per chunk: the chunk's windowed speed and RK2 stage-1 images live in scratch
  // (512 MB at most); every launch below covers the whole chunk.
  const int G = (int)std::max<size_t>(
      1, std::min<size_t>({(size_t)n, (size_t)65535, ((size_t)512 << 20) / (2 * tt * sizeof(float))}));
  int st = ctx->ensure_scratch(2 * (size_t)G * tt * sizeof(float));
  if (st) return st;
  const size_t part_dbl = (std::max<size_t>(1184, (size_t)G) + 1) / 2 + 8;  // absmax partials
  st = ctx->ensure_red(RED_PART + part_dbl + (size_t)n + 8);
  if (st) return st;
  float* vw = static_cast<float*>(ctx->scratch.base);  // windowed speed of the chunk
  float* phi1 = vw + (size_t)G * tt;                   // RK2 stage 1, then the reinit distance
  cudaStream_t s = ctx->stream;
  LITHO_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_red, 0, RED_PART * sizeof(double), s));
  float* part = reinterpret_cast<float*>(ctx->d_red + RED_PART);
  float* vd = reinterpret_cast<float*>(ctx->d_red + RED_PART + part_dbl);  // [tile][max |V|, dt]
  int* bad = reinterpret_cast<int*>(ctx->d_red + RED_FLAG);
  const int* wins = p->d_meta + p->off_update;                            // update_local per tile
  for (int t0 = 0; t0 < n && !st; t0 += G) {
    const int B = std::min(G, n - t0);
    const float* ph = d_phi + t0 * tt;
    float* out = d_phi_out + t0 * tt;
    const int* w = wins + 4 * (size_t)t0;
    float* dtd = vd + 2 * (size_t)t0 + 1;
    st = check_launch(ctx, launch_levelset(s, 6, ts, ts, ph, nullptr, d_grad + t0 * tt, (float)dx,
                                           (float)dy, 0.f, nullptr, vw, nullptr, nullptr, B, w, 0),
                      "windowed speed");
    if (!st)
      st = check_launch(ctx, launch_dt_batch(s, vw, tt, B, (float)dx, (float)dy, (float)cfl,
                                             (float)b, part, vd + 2 * (size_t)t0, bad),
                        "dt");
    if (!st)
      st = check_launch(ctx, launch_levelset(s, 3, ts, ts, ph, nullptr, vw, (float)dx, (float)dy,
                                             (float)b, dtd, phi1, nullptr, nullptr, B, w, 2),
                        "rk2 stage 1");
    if (!st)
      st = check_launch(ctx, launch_levelset(s, 4, ts, ts, phi1, ph, vw, (float)dx, (float)dy,
                                             (float)b, dtd, out, nullptr, nullptr, B, w, 2),
                        "rk2 stage 2");
    ctx->launches += 5;
  }
  // reinit_sdf of the +-0.5 sign image of phi >= 0 (full_chip_lsm.cpp:229-230) of every
  // tile at once: the chamfer transform with inside = phi >= 0, into the mask buffer
  // (rendered afresh below), then phi inside each tile's window only.
  for (int t0 = 0; reinit && t0 < n && !st; t0 += 65535) {
    const int B = std::min(n - t0, 65535);
    st = check_launch(ctx, launch_reinit_sdf(s, ts, ts, d_phi_out + t0 * tt, 0.f, 1, (float)dx,
                                             d_masks + t0 * tt, B, ctx->chamfer_threads(ts, B)),
                      "reinit_sdf");
    if (!st)
      st = check_launch(ctx, launch_levelset(s, 8, ts, ts, d_masks + t0 * tt, d_phi_out + t0 * tt,
                                             nullptr, (float)dx, (float)dy, 0.f, nullptr,
                                             d_phi_out + t0 * tt, nullptr, nullptr, B,
                                             wins + 4 * (size_t)t0, 0),
                        "window commit");
    ctx->launches += 2;
  }
  if (!st)
    st = check_launch(ctx, launch_render_mask(s, d_phi_out, p->ts, p->ts, n,
                                              mask_type == LITHO_MASK_GRAY, scale, d_masks),
                      "render_levelset_mask");
  ctx->launches += 1;
  if (st) return st;
  std::vector<float> h(2 * (size_t)n);
  LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(h.data(), vd, h.size() * sizeof(float),
                                      cudaMemcpyDeviceToHost, s));
  st = fetch(ctx, 0);
  if (st) return st;
  if (flag_set(ctx)) return ctx->fail(LITHO_ERR_NONFINITE, "normal speed must be finite");
  float lo = h[1], hi = h[1];
  for (int t = 1; t < n; ++t) {
    lo = std::min(lo, h[2 * (size_t)t + 1]);
    hi = std::max(hi, h[2 * (size_t)t + 1]);
  }
  if (dt_min) *dt_min = lo;
  if (dt_max) *dt_max = hi;
  return LITHO_OK;
}

}  // extern "C"

// ============================================================== sparse EPE
extern "C" {

int litho_evaluate_sparse_epe(litho_ctx* ctx, int rows, int cols, const float* d_aerial,
                              int n_eps, const double* eps, const double* weights,
                              double threshold, double pixel_size_nm, double* signed_epe,
                              double* totals) {
  if (!ctx || !d_aerial || n_eps < 0 || (n_eps > 0 && (!eps || !weights)))
    return LITHO_ERR_INVALID_ARGUMENT;
  if (rows < 3 || cols < 3)
    return ctx->fail(LITHO_ERR_SHAPE, "evaluate_sparse_epe: the image needs at least 3 x 3 pixels");
  if (!std::isfinite(threshold) || !std::isfinite(pixel_size_nm))
    return ctx->fail(LITHO_ERR_NONFINITE, "evaluate_sparse_epe: threshold and pixel size must be finite");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx->fail(LITHO_ERR_CUDA, "cudaSetDevice");
  const int n = n_eps;
  int st = ctx->ensure_scratch((size_t)(4 * n + 4) * sizeof(double));
  if (st) return st;
  const int nb = n == 0 ? 1 : (n + 255) / 256;
  st = ctx->ensure_red(RED_PART + 3 * (size_t)nb + 8);
  if (st) return st;
  double* d_eps = static_cast<double*>(ctx->scratch.base);
  double* d_w = d_eps + 2 * n;
  double* d_se = d_w + n;
  cudaStream_t s = ctx->stream;
  LITHO_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_red, 0, RED_PART * sizeof(double), s));
  if (n > 0) {
    LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(d_eps, eps, 2 * n * sizeof(double), cudaMemcpyHostToDevice, s));
    LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(d_w, weights, n * sizeof(double), cudaMemcpyHostToDevice, s));
  }
  int used = 0;
  st = check_launch(ctx, launch_epe(s, d_aerial, rows, cols, d_eps, d_w, n, threshold,
                                    pixel_size_nm, d_se, ctx->d_red + RED_PART, nullptr, 1.0,
                                    &used),
                    "sparse EPE");
  if (!st)
    st = check_launch(ctx, launch_sum_partials(s, ctx->d_red + RED_PART, used, 3,
                                               ctx->d_red + RED_SUM),
                      "sum");
  ctx->launches += 2;
  if (st) return st;
  if (signed_epe && n > 0)
    LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(signed_epe, d_se, n * sizeof(double),
                                        cudaMemcpyDeviceToHost, s));
  st = fetch(ctx, 3);
  if (st) return st;
  if (totals) std::memcpy(totals, ctx->h_red + RED_SUM, 3 * sizeof(double));
  return LITHO_OK;
}

int litho_epe_gradient(litho_ctx* ctx, const litho_field* field, const float* d_aerial,
                       int n_eps, const double* eps, const double* weights, double threshold,
                       float* d_grad) {
  if (!ctx || !field || !d_aerial || !d_grad || n_eps < 0 || (n_eps > 0 && (!eps || !weights)))
    return LITHO_ERR_INVALID_ARGUMENT;
  if (n_eps > (1 << 28)) return ctx->fail(LITHO_ERR_INVALID_ARGUMENT, "epe_gradient: too many EPs");
  if (!field->valid) return ctx->fail(LITHO_ERR_NOT_READY, "Gradient: field not computed");
  if (!std::isfinite(threshold))
    return ctx->fail(LITHO_ERR_NONFINITE, "epe_gradient: threshold must be finite");
  const Cache& c = *field->cache;
  const int N = c.g.N;
  if (N < 3) return ctx->fail(LITHO_ERR_SHAPE, "epe_gradient: the image needs at least 3 x 3 pixels");
  Layout L;
  int st = prepare(ctx, c, &L);
  if (st) return st;
  const int n = n_eps;
  const size_t ep_off = align_up(L.total, 256);
  const size_t sort_off = align_up(ep_off + (size_t)(3 * n + 4) * sizeof(double), 256);
  const size_t sort_bytes = epe_scatter_work_bytes(n);
  st = ctx->ensure_scratch(sort_off + sort_bytes);
  if (st) return st;
  const int nb = n == 0 ? 1 : (n + 255) / 256;
  st = ctx->ensure_red(RED_PART + 3 * (size_t)nb + 8);
  if (st) return st;
  LITHO_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_red, 0, RED_PART * sizeof(double), ctx->stream));
  double* d_eps = at<double>(ctx, ep_off);
  double* d_w = d_eps + 2 * n;
  cudaStream_t s = ctx->stream;
  float* dldi = at<float>(ctx, L.dldi);
  LITHO_CUDA_TRY(ctx, cudaMemsetAsync(dldi, 0, (size_t)N * N * sizeof(float), s));
  if (n > 0) {
    LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(d_eps, eps, 2 * n * sizeof(double), cudaMemcpyHostToDevice, s));
    LITHO_CUDA_TRY(ctx, cudaMemcpyAsync(d_w, weights, n * sizeof(double), cudaMemcpyHostToDevice, s));
  }
  int used = 0;
  st = check_launch(ctx, launch_epe(s, d_aerial, N, N, d_eps, d_w, n, threshold, 1.0, nullptr,
                                    ctx->d_red + RED_PART, dldi, 1.0, &used,
                                    at<void>(ctx, sort_off), sort_bytes),
                    "sparse EPE scatter");
  ctx->launches += n > 0 ? 3 : 1;   // EPE, sort, per-pixel sums
  if (st) return st;
  // dL/dI already holds the 2 of the squared EPE; |E|^2 gives another 2 (gradient.cpp:225-226).
  GradEpilogue ep{};
  ep.grad_mask = d_grad;
  int nb2 = 0;
  st = run_adjoint(ctx, c, *field, L, dldi, 2.0, ep, &nb2);
  if (!st) st = fetch(ctx, 0);
  if (st) return st;
  if (flag_set(ctx)) return ctx->fail(LITHO_ERR_NONFINITE, "epe_gradient: dL/dI must be finite");
  return LITHO_OK;
}

}  // extern "C"
