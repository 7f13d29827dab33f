// Full-chip micro-tile kernels: periodic Halo extraction and Core assembly
// (source/utils/partition.cpp:83-113), the neighbour exchange of
// MicroGradientExchange::compute phase two (source/utils/micro_gradient_exchange.cpp:253-326:
// CEPT against the frozen neighbour Core, optional two-sided CEPT, Average or
// Linear guard-gradient fusion) and the windowed CTM theta update of
// FullChipCTMOptimizer (source/optimizer/full_chip_ctm.cpp:127-147).
//
// All tiles of a partition share one tile size ts and live contiguously as
// [tile][ts][ts] float32 arrays.
#include <cuda_runtime.h>
#include <algorithm>

#include "device_common.cuh"

namespace litho_b200 {

// out[t][y][x] = global[(oy_t + y) mod H][(ox_t + x) mod W]
// Tile t's rows are spread over the CTAs of grid row t, the threads over the columns;
// the periodic wrap of a row start is taken once per row and column once per thread.
__global__ void tiles_extract_kernel(const float* __restrict__ g, int H, int W,
                                     const int* __restrict__ origins, int ts,
                                     float* __restrict__ out) {
  const int t = blockIdx.y;
  const int oy = origins[2 * t], ox = origins[2 * t + 1];
  const int gx0 = ((ox % W) + W) % W;
  for (int y = blockIdx.x; y < ts; y += gridDim.x) {
    const float* grow = g + (size_t)(((oy + y) % H + H) % H) * W;
    float* orow = out + ((size_t)t * ts + y) * ts;
    for (int x = threadIdx.x; x < ts; x += blockDim.x) {
      int gx = gx0 + x;
      if (gx >= W) gx = gx - W < W ? gx - W : gx % W;
      orow[x] = __ldg(grow + gx);
    }
  }
}

cudaError_t launch_tiles_extract(cudaStream_t s, const float* g, int H, int W, int ntiles,
                                 const int* origins, int ts, float* out) {
  dim3 grid(ts < 256 ? ts : 256, ntiles);
  tiles_extract_kernel<<<grid, 256, 0, s>>>(g, H, W, origins, ts, out);
  return cudaGetLastError();
}

// global[core_global] = local[core_local]; rects as (y0, y1, x0, x1).
__global__ void tiles_assemble_kernel(const float* __restrict__ loc, int ts,
                                      const int* __restrict__ core_g,
                                      const int* __restrict__ core_l, int W,
                                      float* __restrict__ g) {
  const int t = blockIdx.y;
  const int gy0 = core_g[4 * t], gx0 = core_g[4 * t + 2];
  const int rows = core_g[4 * t + 1] - gy0, cols = core_g[4 * t + 3] - gx0;
  const int ly0 = core_l[4 * t], lx0 = core_l[4 * t + 2];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows * cols; i += gridDim.x * blockDim.x) {
    const int y = i / cols, x = i % cols;
    g[(size_t)(gy0 + y) * W + gx0 + x] = loc[((size_t)t * ts + ly0 + y) * ts + lx0 + x];
  }
}

cudaError_t launch_tiles_assemble(cudaStream_t s, const float* loc, int ntiles, int ts,
                                  const int* core_g, const int* core_l, int W, float* g) {
  dim3 grid(64, ntiles);
  tiles_assemble_kernel<<<grid, 256, 0, s>>>(loc, ts, core_g, core_l, W, g);
  return cudaGetLastError();
}

// build_micro_loss_windows (micro_gradient_exchange.cpp:65-93), every tile at once.
// Inside the tile's loss region: pen = [T < 0.5]; epe = 1, or for PE_EPE the dilated
// main region; pe = [T > 0.5] for PEPenalty, 1 - epe for PE_EPE, else 1. All three are
// 0 outside the region. main_dil (PE_EPE only) and epe_w are nullable.
__global__ void loss_windows_kernel(const float* __restrict__ target, int ts,
                                    const int* __restrict__ region, int loss_type,
                                    const float* __restrict__ main_dil, float* __restrict__ pe_w,
                                    float* __restrict__ pen_w, float* __restrict__ epe_w) {
  const int t = blockIdx.y;
  const int y0 = region[4 * t], y1 = region[4 * t + 1], x0 = region[4 * t + 2],
            x1 = region[4 * t + 3];
  for (int y = blockIdx.x; y < ts; y += gridDim.x) {
    const bool row_in = y >= y0 && y < y1;
    for (int x = threadIdx.x; x < ts; x += blockDim.x) {
      const size_t k = ((size_t)t * ts + y) * ts + x;
      const bool in = row_in && x >= x0 && x < x1;
      const float T = target[k];
      const float e = loss_type == LITHO_MICRO_LOSS_PE_EPE ? main_dil[k] : 1.f;
      float pe = loss_type == LITHO_MICRO_LOSS_PE_PENALTY ? (T > 0.5f ? 1.f : 0.f) : 1.f;
      if (loss_type == LITHO_MICRO_LOSS_PE_EPE) pe = 1.f - e;
      pe_w[k] = in ? pe : 0.f;
      pen_w[k] = in && T < 0.5f ? 1.f : 0.f;
      if (epe_w) epe_w[k] = in ? e : 0.f;
    }
  }
}

cudaError_t launch_loss_windows(cudaStream_t s, const float* target, int ntiles, int ts,
                                const int* region, int loss_type, const float* main_dil,
                                float* pe_w, float* pen_w, float* epe_w) {
  dim3 grid(ts < 256 ? ts : 256, ntiles);
  loss_windows_kernel<<<grid, 256, 0, s>>>(target, ts, region, loss_type, main_dil, pe_w, pen_w,
                                           epe_w);
  return cudaGetLastError();
}

// The PE_EPE main region: [T > 0.5] dilated `iterations` times by a 3 x 3 square
// with zeros outside the tile (cv::dilate with BORDER_CONSTANT 0,
// micro_gradient_exchange.cpp:71-80), i.e. a Chebyshev-distance dilation by
// `iterations`, done as a row pass then a column pass.
__global__ void dilate_main_kernel(const float* __restrict__ src, int ts, int r, int rows_pass,
                                   float* __restrict__ dst) {
  const int t = blockIdx.y;
  const float* a = src + (size_t)t * ts * ts;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ts * ts; i += gridDim.x * blockDim.x) {
    const int y = i / ts, x = i % ts;
    float m = 0.f;
    if (rows_pass) {
      for (int d = max(0, x - r); d <= min(ts - 1, x + r) && m == 0.f; ++d)
        m = a[(size_t)y * ts + d] > 0.5f ? 1.f : 0.f;
    } else {
      for (int d = max(0, y - r); d <= min(ts - 1, y + r) && m == 0.f; ++d) m = a[(size_t)d * ts + x];
    }
    dst[(size_t)t * ts * ts + i] = m;
  }
}

cudaError_t launch_dilate_main(cudaStream_t s, const float* target, int ntiles, int ts,
                               int iterations, float* tmp, float* out) {
  dim3 grid((ts * ts + 255) / 256 < 128 ? (ts * ts + 255) / 256 : 128, ntiles);
  dilate_main_kernel<<<grid, 256, 0, s>>>(target, ts, iterations, 1, tmp);
  dilate_main_kernel<<<grid, 256, 0, s>>>(tmp, ts, iterations, 0, out);
  return cudaGetLastError();
}

// region_eps_local (micro_gradient_exchange.cpp:18-50) for one tile: candidate
// c = (i * P + py') * P + px' (P = 2 periods + 1) is EP i shifted by (py, px) whole
// layouts; it is kept, at local (y, x) with EP i's weight, when it lies in the
// region (global half-open rect) and any pixel of its bilinear stencil on the tile
// has a nonzero EPE window. Dropped candidates get weight 0 (inactive).
__global__ void ep_candidates_kernel(const double* __restrict__ eps, const double* __restrict__ w,
                                     int n, int periods, int H, int W, int oy, int ox, int gy0,
                                     int gy1, int gx0, int gx1, int ts,
                                     const float* __restrict__ win, double* __restrict__ out_eps,
                                     double* __restrict__ out_w) {
  const int P = 2 * periods + 1;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n * P * P) return;
  const int i = c / (P * P), py = (c / P) % P - periods, px = c % P - periods;
  const double y = eps[2 * i] + (double)py * H, x = eps[2 * i + 1] + (double)px * W;
  double ly = 0.0, lx = 0.0, wc = 0.0;
  if (y >= gy0 && y < gy1 && x >= gx0 && x < gx1) {
    ly = y - oy;
    lx = x - ox;
    const double yy = fmin(fmax(ly, 0.0), ts - 1.0), xx = fmin(fmax(lx, 0.0), ts - 1.0);
    const int y0 = (int)floor(yy), x0 = (int)floor(xx);
    const int y1 = min(y0 + 1, ts - 1), x1 = min(x0 + 1, ts - 1);
    const double wy1 = y1 == y0 ? 0.0 : yy - y0, wx1 = x1 == x0 ? 0.0 : xx - x0;
    const bool touch = ((1.0 - wy1) * (1.0 - wx1) > 0.0 && win[(size_t)y0 * ts + x0] != 0.f) ||
                       ((1.0 - wy1) * wx1 > 0.0 && win[(size_t)y0 * ts + x1] != 0.f) ||
                       (wy1 * (1.0 - wx1) > 0.0 && win[(size_t)y1 * ts + x0] != 0.f) ||
                       (wy1 * wx1 > 0.0 && win[(size_t)y1 * ts + x1] != 0.f);
    if (touch) wc = w[i];
  }
  out_eps[2 * (size_t)c] = ly;
  out_eps[2 * (size_t)c + 1] = lx;
  out_w[c] = wc;
}

cudaError_t launch_ep_candidates(cudaStream_t s, const double* eps, const double* w, int n,
                                 int periods, int H, int W, int oy, int ox, const int* grect,
                                 int ts, const float* win, double* out_eps, double* out_w) {
  const int P = 2 * periods + 1;
  const long long nc = (long long)n * P * P;
  if (nc == 0) return cudaSuccess;
  ep_candidates_kernel<<<(unsigned)((nc + 255) / 256), 256, 0, s>>>(
      eps, w, n, periods, H, W, oy, ox, grect[0], grect[1], grect[2], grect[3], ts, win, out_eps,
      out_w);
  return cudaGetLastError();
}

// Loss sums over the loss region and the Core of a group of tiles in one launch
// (the Core metrics of micro_gradient_exchange.cpp:224-233), per CTA in FP64:
// sum pe_w (W - T)^2, sum_{T < 0.5} pen_w max(W - pen_thr, 0)^2 and
// sum_{T > 0.5} (W - T)^2. Tile blockIdx.y (images ts x ts back to back, rectangles
// {y0, y1, x0, x1} 4 ints per tile), the Core being inside the region.
// partial[(tile * gridDim.x + block) * 6 + k]: k = 0..2 the three sums over the
// region, 3..5 over the Core.
constexpr int RL_NT = 256;
__global__ void __launch_bounds__(RL_NT)
rect_losses_batch_kernel(const float* __restrict__ Wf, const float* __restrict__ T,
                         const float* __restrict__ pe_w, const float* __restrict__ pen_w, int ts,
                         const int* __restrict__ regions, const int* __restrict__ cores,
                         float pen_thr, double* __restrict__ partial) {
  __shared__ double sh[RL_NT / 32];
  const size_t img = (size_t)blockIdx.y * ts * ts;
  const int* rg = regions + 4 * (size_t)blockIdx.y;
  const int* cr = cores + 4 * (size_t)blockIdx.y;
  const int cy0 = cr[0], cy1 = cr[1], cx0 = cr[2], cx1 = cr[3];
  double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  // block b takes rows rg[0] + b, + gridDim.x, ...; the threads sweep the columns
  for (int y = rg[0] + blockIdx.x; y < rg[1]; y += gridDim.x)
  for (int x = rg[2] + threadIdx.x; x < rg[3]; x += RL_NT) {
    const size_t k = img + (size_t)y * ts + x;
    const double w = Wf[k], t = T[k], r = w - t;
    const double pe = r * r * (double)pe_w[k];
    double bg = 0.0;
    if (t < 0.5) {
      const double ex = fmax(0.0, w - (double)pen_thr);
      bg = (double)pen_w[k] * ex * ex;
    }
    const double mainpe = t > 0.5 ? r * r : 0.0;
    v[0] += pe; v[1] += bg; v[2] += mainpe;
    if (y >= cy0 && y < cy1 && x >= cx0 && x < cx1) {
      v[3] += pe; v[4] += bg; v[5] += mainpe;
    }
  }
  double* out = partial + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 6;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const double a = block_sum<RL_NT>(v[k], sh);
    if (threadIdx.x == 0) out[k] = a;
  }
}

int rect_losses_batch_blocks(int ts) { return ts < 1 ? 1 : (ts > 96 ? 96 : ts); }

cudaError_t launch_rect_losses_batch(cudaStream_t s, const float* Wf, const float* T,
                                     const float* pe_w, const float* pen_w, int ts,
                                     const int* d_regions, const int* d_cores, float pen_thr,
                                     double* partial, int nimg) {
  if (nimg < 1 || nimg > 65535) return cudaErrorInvalidValue;
  rect_losses_batch_kernel<<<dim3(rect_losses_batch_blocks(ts), nimg), RL_NT, 0, s>>>(
      Wf, T, pe_w, pen_w, ts, d_regions, d_cores, pen_thr, partial);
  return cudaGetLastError();
}

// Neighbour relations of one tile come in the reference's order (left, right,
// top, bottom; absent neighbours omitted).
constexpr int REL_INTS = FC_REL_INTS;
constexpr int EX_NT = 256;

__device__ __forceinline__ float linear_strength(int dir, int y, int x, int rows, int cols) {
  switch (dir) {
    case 0: return cols == 1 ? 1.f : 1.f - (float)x / (float)(cols - 1);   // left
    case 1: return cols == 1 ? 1.f : (float)x / (float)(cols - 1);         // right
    case 2: return rows == 1 ? 1.f : 1.f - (float)y / (float)(rows - 1);   // top
    default: return rows == 1 ? 1.f : (float)y / (float)(rows - 1);        // bottom
  }
}

// Relation slot j of every tile (tile blockIdx.y; its j-th neighbour in the
// reference's order), spread over gridDim.x CTAs per tile. grad holds a copy of raw
// before slot 0 and leaves the last slot as raw (fused on guards) + cept_weight *
// cept_grad. A relation's guard strip (outside the Core) and, two-sided, its
// overlap strip (inside the Core) are disjoint, so one launch covers both; the
// overlap strips of different relations share Core corners, so the slots run as
// separate launches in the reference's order. part[(tile * max_rel + j) * gridDim.x +
// block] = this block's sum of (A guard mask - B core mask)^2.
__global__ void __launch_bounds__(EX_NT)
exchange_rel_kernel(const float* __restrict__ masks, const float* __restrict__ raw, int ts,
                    const int* __restrict__ nrel, const int* __restrict__ rel, int max_rel, int j,
                    litho_exchange_options o, float* __restrict__ grad,
                    double* __restrict__ part) {
  __shared__ double sh[EX_NT / 32];
  const int t = blockIdx.y, nch = gridDim.x;
  double* out = part + ((size_t)t * max_rel + j) * nch + blockIdx.x;
  if (j >= nrel[t]) {
    if (threadIdx.x == 0) *out = 0.0;
    return;
  }
  const size_t tt = (size_t)ts * ts;
  const float* mA = masks + t * tt;
  const float* rA = raw + t * tt;
  float* gA = grad + t * tt;
  const int* R = rel + ((size_t)t * max_rel + j) * REL_INTS;
  const int nb = R[0], dir = R[1];
  const int gy0 = R[2], gy1 = R[3], gx0 = R[4], gx1 = R[5];       // my guard (local A)
  const int sy0 = R[6], sx0 = R[8];                                // neighbour overlap (local B)
  const float* mB = masks + (size_t)nb * tt;
  const float* rB = raw + (size_t)nb * tt;
  const int rows = gy1 - gy0, cols = gx1 - gx0;
  double acc = 0.0;
  for (int i = blockIdx.x * EX_NT + threadIdx.x; i < rows * cols; i += nch * EX_NT) {
    const int y = i / cols, x = i % cols;
    const size_t ia = (size_t)(gy0 + y) * ts + gx0 + x;
    const size_t ib = (size_t)(sy0 + y) * ts + sx0 + x;
    float g = gA[ia];
    if (o.enable_grad_fusion) {
      const float st = o.fusion_mode == 0 ? 1.f : linear_strength(dir, y, x, rows, cols);
      const float wn = (float)o.fusion_weight_neighbor * st;
      if (wn != 0.f)
        g = ((float)o.fusion_weight_owner * rA[ia] + wn * rB[ib]) /
            ((float)o.fusion_weight_owner + wn);
    }
    if (o.enable_cept) {
      const float d = mA[ia] - mB[ib];
      acc += (double)d * (double)d;
      g += (float)o.cept_weight * 2.f * d;
    }
    gA[ia] = g;
  }
  if (o.enable_cept && !o.cept_guard_only) {
    // The neighbour's guard over this tile's Core edge drives the Core side too.
    const int oy0 = R[10], oy1 = R[11], ox0 = R[12], ox1 = R[13];   // my overlap (local A)
    const int ny0 = R[14], nx0 = R[16];                              // neighbour guard (local B)
    const int orows = oy1 - oy0, ocols = ox1 - ox0;
    for (int i = blockIdx.x * EX_NT + threadIdx.x; i < orows * ocols; i += nch * EX_NT) {
      const int y = i / ocols, x = i % ocols;
      const size_t ia = (size_t)(oy0 + y) * ts + ox0 + x;
      const size_t ib = (size_t)(ny0 + y) * ts + nx0 + x;
      gA[ia] += (float)o.cept_weight * 2.f * (mA[ia] - mB[ib]);
    }
  }
  const double total = block_sum<EX_NT>(acc, sh);
  if (threadIdx.x == 0) *out = total;
}

// cept_loss[t] = the tile's partial sums in a fixed order.
__global__ void exchange_sum_kernel(const double* __restrict__ part, int per_tile, int ntiles,
                                    double* __restrict__ cept_loss) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntiles) return;
  double s = 0.0;
  for (int k = 0; k < per_tile; ++k) s += part[(size_t)t * per_tile + k];
  cept_loss[t] = s;
}

int exchange_chunks(int ntiles) {
  const int c = (4 * 148 + ntiles - 1) / std::max(ntiles, 1);
  return c < 4 ? 4 : (c > 32 ? 32 : c);
}

cudaError_t launch_exchange(cudaStream_t s, const float* masks, const float* raw, int ntiles,
                            int ts, const int* nrel, const int* rel, int max_rel,
                            const litho_exchange_options& o, float* grad, double* cept_loss,
                            double* part) {
  if (ntiles < 1 || ntiles > 65535) return cudaErrorInvalidValue;
  const int nch = exchange_chunks(ntiles);
  for (int j = 0; j < max_rel; ++j) {
    exchange_rel_kernel<<<dim3(nch, ntiles), EX_NT, 0, s>>>(masks, raw, ts, nrel, rel, max_rel, j,
                                                           o, grad, part);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  exchange_sum_kernel<<<(ntiles + 127) / 128, 128, 0, s>>>(part, max_rel * nch, ntiles, cept_loss);
  return cudaGetLastError();
}

// theta -= lr * (-1/2 G sin theta) inside the update window (y0, y1, x0, x1) of each
// tile; mask = (1 + cos theta) / 2 over the whole tile. grad == nullptr only
// refreshes the masks.
__global__ void theta_update_kernel(float* __restrict__ theta, const float* __restrict__ grad,
                                    int ts, const int* __restrict__ win, float lr,
                                    float* __restrict__ mask) {
  const int t = blockIdx.y;
  const int y0 = win[4 * t], y1 = win[4 * t + 1], x0 = win[4 * t + 2], x1 = win[4 * t + 3];
  for (int y = blockIdx.x; y < ts; y += gridDim.x) {
    const bool row_in = grad && y >= y0 && y < y1;
    for (int x = threadIdx.x; x < ts; x += blockDim.x) {
      const size_t k = ((size_t)t * ts + y) * ts + x;
      float th = theta[k];
      if (row_in && x >= x0 && x < x1) {
        th -= lr * (-0.5f * grad[k] * sinf(th));
        theta[k] = th;
      }
      mask[k] = 0.5f * (1.f + cosf(th));
    }
  }
}

cudaError_t launch_theta_update(cudaStream_t s, float* theta, const float* grad, int ntiles,
                                int ts, const int* win, float lr, float* mask) {
  dim3 grid(ts < 256 ? ts : 256, ntiles);
  theta_update_kernel<<<grid, 256, 0, s>>>(theta, grad, ts, win, lr, mask);
  return cudaGetLastError();
}

}  // namespace litho_b200
