"""Seeded synthetic workloads of the imaging-and-gradient benchmark.

No public dataset belongs to this path; the benchmark inputs are generated
here with ``numpy.random.default_rng(seed)``:

* Manhattan targets: axis-aligned rectangles (widths 30-120 nm, minimum
  space 40 nm on a 2 nm grid) plus optional L/T shapes, binary {0, 1}.
* SOCS kernels: the top-K coherent modes of a partially coherent annular
  source (sigma 0.6-0.9 sampled on a 21 x 21 grid) through a circular pupil,
  restricted to an Nk x Nk frequency support centred on DC and computed in
  FP64 (thin SVD of the shifted-pupil matrix, as
  source/litho_model/litho_prepare.cpp:258-328 does), with eigen-weights
  replaced by a geometric sequence lambda_k = 0.8^k.

Everything here is FP64 host set-up, done once per workload; the timed path
runs in the CUDA library.
"""
from __future__ import annotations

import math
from typing import Tuple

import numpy as np


def synthetic_socs_band(K: int = 24, nk: int = 35, ratio: float = 0.8, sigma_in: float = 0.6,
                        sigma_out: float = 0.9, src_grid: int = 21):
    """K band kernels (K, nk, nk) complex128 on integer frequencies
    [-(nk//2), nk - 1 - nk//2]^2, their weights and the source-weight sum."""
    half = nk // 2
    f = np.arange(nk) - half
    fx = f[None, :].astype(np.float64)
    fy = f[:, None].astype(np.float64)
    r_pupil = (half + 0.5) / (1.0 + sigma_out)   # shifted pupils stay inside the support
    s = np.linspace(-1.0, 1.0, src_grid)
    sx, sy = np.meshgrid(s, s)
    rho = np.hypot(sx, sy)
    on = (rho >= sigma_in) & (rho <= sigma_out)
    pts = np.stack([sx[on], sy[on]], axis=1)
    cols = []
    for px, py in pts:
        pupil = ((fx + px * r_pupil) ** 2 + (fy + py * r_pupil) ** 2 <= r_pupil ** 2)
        cols.append(pupil.astype(np.complex128).reshape(-1))
    A = np.stack(cols, axis=1) / math.sqrt(len(cols))
    U, S, _ = np.linalg.svd(A, full_matrices=False)
    K = min(K, U.shape[1])
    band = U[:, :K].T.reshape(K, nk, nk).copy()
    weights = ratio ** np.arange(K, dtype=np.float64)
    return band, -half, -half, weights, 1.0


def band_to_dense(band: np.ndarray, row0: int, col0: int, N: int) -> np.ndarray:
    """Embed band kernels into K x N x N DC-at-corner frequency kernels."""
    K, nr, nc = band.shape
    out = np.zeros((K, N, N), dtype=np.complex128)
    rows = (row0 + np.arange(nr)) % N
    cols = (col0 + np.arange(nc)) % N
    out[:, rows[:, None], cols[None, :]] = band
    return out


def _place(canvas, occ, rects, space):
    for (y0, y1, x0, x1) in rects:
        if y0 < 0 or x0 < 0 or y1 > canvas.shape[0] or x1 > canvas.shape[1]:
            return False
        if occ[max(0, y0 - space):y1 + space, max(0, x0 - space):x1 + space].any():
            return False
    for (y0, y1, x0, x1) in rects:
        canvas[y0:y1, x0:x1] = 1.0
    for (y0, y1, x0, x1) in rects:
        occ[y0:y1, x0:x1] = True
    return True


def manhattan_target(N: int, n_rect: int, seed: int, pixel_nm: float = 2.0, wmin_nm: float = 30.0,
                     wmax_nm: float = 120.0, space_nm: float = 40.0, n_lt: int = 0,
                     lmax_nm: float = None, max_tries: int = 200000) -> np.ndarray:
    """Binary target of n_rect rectangles and n_lt L/T shapes (float64 {0,1})."""
    rng = np.random.default_rng(seed)
    wmin = max(1, int(round(wmin_nm / pixel_nm)))
    wmax = max(wmin, int(round(wmax_nm / pixel_nm)))
    space = int(round(space_nm / pixel_nm))
    lmax = int(round((lmax_nm if lmax_nm else 6 * wmax_nm) / pixel_nm))
    canvas = np.zeros((N, N), dtype=np.float64)
    occ = np.zeros((N, N), dtype=bool)
    placed = lt = tries = 0
    margin = space
    while (placed < n_rect or lt < n_lt) and tries < max_tries:
        tries += 1
        w = int(rng.integers(wmin, wmax + 1))
        L = int(rng.integers(wmin, max(wmin + 1, min(lmax, N // 3))))
        horiz = bool(rng.integers(0, 2))
        h_, w_ = (w, L) if horiz else (L, w)
        y0 = int(rng.integers(margin, max(margin + 1, N - margin - h_)))
        x0 = int(rng.integers(margin, max(margin + 1, N - margin - w_)))
        if placed < n_rect:
            if _place(canvas, occ, [(y0, y0 + h_, x0, x0 + w_)], space):
                placed += 1
            continue
        # L or T: a bar plus a perpendicular arm touching it
        w2 = int(rng.integers(wmin, wmax + 1))
        L2 = int(rng.integers(wmin, max(wmin + 1, min(lmax, N // 4))))
        if horiz:
            ax = x0 if rng.integers(0, 2) == 0 else x0 + (w_ - w2) // 2
            arm = (y0 + h_, y0 + h_ + L2, ax, ax + w2)
        else:
            ay = y0 if rng.integers(0, 2) == 0 else y0 + (h_ - w2) // 2
            arm = (ay, ay + w2, x0 + w_, x0 + w_ + L2)
        if _place(canvas, occ, [(y0, y0 + h_, x0, x0 + w_), arm], space):
            lt += 1
    return canvas


def density_target(N: int, density: float, seed: int, pixel_nm: float = 2.0) -> np.ndarray:
    """Rectangles added until the pattern density reaches ``density``."""
    rng = np.random.default_rng(seed)
    wmin, wmax, space = int(15 / (pixel_nm / 2)), int(60 / (pixel_nm / 2)), int(20 / (pixel_nm / 2))
    canvas = np.zeros((N, N), dtype=np.float64)
    occ = np.zeros((N, N), dtype=bool)
    tries = 0
    while canvas.mean() < density and tries < 50 * N:
        tries += 1
        w = int(rng.integers(wmin, wmax + 1))
        L = int(rng.integers(wmin, 8 * wmax))
        h_, w_ = (w, L) if rng.integers(0, 2) else (L, w)
        y0 = int(rng.integers(0, max(1, N - h_)))
        x0 = int(rng.integers(0, max(1, N - w_)))
        _place(canvas, occ, [(y0, y0 + h_, x0, x0 + w_)], space)
    return canvas


def cell_layout(H: int, W: int, seed: int, cell: int = 64, wmin: int = 18, wmax: int = 57,
                margin: int = 4) -> np.ndarray:
    """A large binary layout (float32 {0,1}) built fast: one rectangle of seeded width
    and height in [wmin, wmax] pixels per cell x cell block, at a seeded offset that
    keeps it `margin` pixels inside its block (so neighbours stay at least 2 margin
    apart). With the defaults (2 nm pixels: 36-114 nm features in 128 nm cells) the
    pattern density is about 34 %."""
    rng = np.random.default_rng(seed)
    gy, gx = -(-H // cell), -(-W // cell)
    h = rng.integers(wmin, wmax + 1, size=(gy, gx))
    w = rng.integers(wmin, wmax + 1, size=(gy, gx))
    oy = margin + (rng.random((gy, gx)) * (cell - 2 * margin - h + 1)).astype(np.int64)
    ox = margin + (rng.random((gy, gx)) * (cell - 2 * margin - w + 1)).astype(np.int64)
    # rows / columns inside each cell's rectangle, as two separable indicator tables
    r = np.arange(cell)
    in_y = (r[None, None, :] >= oy[..., None]) & (r[None, None, :] < (oy + h)[..., None])
    in_x = (r[None, None, :] >= ox[..., None]) & (r[None, None, :] < (ox + w)[..., None])
    out = np.empty((gy * cell, gx * cell), dtype=np.float32)
    for i in range(gy):
        blk = in_y[i][:, :, None] & in_x[i][:, None, :]          # (gx, cell, cell)
        out[i * cell:(i + 1) * cell] = blk.transpose(1, 0, 2).reshape(cell, gx * cell)
    return out[:H, :W]


def theta_init_from_target(target: np.ndarray) -> np.ndarray:
    """theta = pi (1 - target): the benchmark's binary-mask initialisation."""
    return np.pi * (1.0 - target)


def theta_init_reference(target: np.ndarray) -> np.ndarray:
    """CTM_Optimizer::_initialize_theta (CTM_Optimizer.cpp:55-64): 0.3 pi / 0.7 pi."""
    pi = 3.14159265358979323846
    return np.where(target > 0.0, 0.3 * pi, 0.7 * pi)


def uneven_cuts(extent: int, lo: int, hi: int, seed: int) -> list:
    """Seeded Core boundaries 0 = c_0 < c_1 < ... < c_n = extent with every Core side
    c_{i+1} - c_i in [lo, hi] (requires extent >= lo and hi >= 2 lo): sides drawn
    uniformly from [lo, hi] while the rest exceeds hi, then the rest split into one or
    two Cores inside the range."""
    if extent < lo or hi < 2 * lo:
        raise ValueError("uneven_cuts needs extent >= lo and hi >= 2 lo")
    rng = np.random.default_rng(seed)
    cuts = [0]
    while extent - cuts[-1] > hi:
        rest = extent - cuts[-1]
        side = int(rng.integers(lo, hi + 1))
        if rest - side < lo:          # keep a last Core of at least lo
            side = rest - lo
        cuts.append(cuts[-1] + side)
    cuts.append(extent)
    return cuts
