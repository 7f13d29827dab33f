"""FP64 restatement of the reference SOCS/Abbe imaging, losses, adjoint and CTM.

Test infrastructure only (see ``oracle/__init__.py``). Arrays are row-major
NumPy float64 / complex128 with (row=y, col=x), the same orientation as the
reference's Eigen matrices.

An ``OracleCache`` mirrors ``ImagingCache`` (include/litho_model/litho_prepare.h:18-47):
``kernels`` are the K full N x N frequency kernels with DC at the corner,
``eigenvalues`` are the SOCS weights (empty tuple for Abbe), ``source_ws``
the source weights whose sum normalises the image.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Sequence

import numpy as np
import scipy.fft as sfft

FFT_WORKERS = 8


def set_fft_workers(n: int) -> None:
    global FFT_WORKERS
    FFT_WORKERS = int(n)


@dataclasses.dataclass
class OracleCache:
    N: int
    kernels: List[np.ndarray]          # K x (N x N complex128), DC at corner
    source_ws: np.ndarray              # Ns (Abbe: == K) float64
    eigenvalues: Sequence[float] = ()  # K (SOCS) or empty (Abbe)

    @property
    def weights(self) -> np.ndarray:
        # imaging.cpp:157: weight = use_socs ? socs_eigenvalues[k] : source_weights(k)
        if len(self.eigenvalues):
            return np.asarray(self.eigenvalues, dtype=np.float64)
        return np.asarray(self.source_ws, dtype=np.float64)

    @property
    def ws_sum(self) -> float:
        return float(np.sum(self.source_ws))


# ---------------------------------------------------------------- shifts / FFT
def fftshift(x: np.ndarray) -> np.ndarray:
    """fft.cpp:152-157: roll by floor(N/2) along both axes."""
    return np.roll(x, (x.shape[0] // 2, x.shape[1] // 2), axis=(0, 1))


def ifftshift(x: np.ndarray) -> np.ndarray:
    """fft.cpp:159-163: roll by ceil(N/2) along both axes."""
    return np.roll(x, ((x.shape[0] + 1) // 2, (x.shape[1] + 1) // 2), axis=(0, 1))


def _fft2(x):
    return sfft.fft2(x, workers=FFT_WORKERS)


def _ifft2_unnormalised(x):
    # FFTW_BACKWARD is unnormalised; scipy's ifft2 divides by N^2.
    return sfft.ifft2(x, norm="forward", workers=FFT_WORKERS)


# ------------------------------------------------------------------- imaging
def imaging_compute(mask: np.ndarray, cache: OracleCache, threshold: float = 0.25,
                    alpha: float = 50.0, keep_fields: bool = True):
    """Imaging::compute (source/litho_model/imaging.cpp:60-171).

    Returns (aerial, wafer, fields). fields[k] = E_k (N x N complex128),
    centred exactly as the reference's ``get_electric_field()``.
    """
    N = cache.N
    mask = np.asarray(mask, dtype=np.float64)
    if mask.shape != (N, N):
        raise ValueError("Imaging: mask dimensions must match cache.N")     # imaging.cpp:68-70
    if not (np.all(np.isfinite(mask)) and math.isfinite(threshold) and math.isfinite(alpha)):
        raise ValueError("Imaging: mask, threshold, and alpha must be finite")  # :71-73
    if len(cache.kernels) == 0:
        raise ValueError("Imaging: no optical kernels available")             # :74-76
    ws_sum = cache.ws_sum
    if not (np.all(np.isfinite(cache.source_ws)) and np.all(np.asarray(cache.source_ws) >= 0)
            and math.isfinite(ws_sum) and ws_sum > 0):
        raise ValueError("Imaging: source weights must be finite, nonnegative, and have a positive sum")
    weights = cache.weights
    inv = 1.0 / float(N * N)
    # imaging.cpp:114-118: M_f = FFT(ifftshift(M))
    mask_frequency = _fft2(ifftshift(mask.astype(np.complex128)))
    aerial = np.zeros((N, N), dtype=np.float64)
    fields = []
    # imaging.cpp:137-148 then fixed-k-order sum :156-164
    for k, kernel in enumerate(cache.kernels):
        e = fftshift(_ifft2_unnormalised(mask_frequency * kernel) * inv)
        aerial += weights[k] * (e.real ** 2 + e.imag ** 2)
        if keep_fields:
            fields.append(e)
    aerial /= ws_sum
    wafer = 1.0 / (1.0 + np.exp(-alpha * (aerial - threshold)))             # :165-168
    return aerial, wafer, fields


# ---------------------------------------------------------------- losses
def pe_loss(wafer, target, window=None) -> float:
    """Loss::pe_loss (source/utils/loss.cpp:16-23)."""
    d = (np.asarray(wafer) - np.asarray(target)) ** 2
    if window is not None:
        d = d * window
    return float(d.sum())


def background_penalty_loss(wafer, target, penalty_threshold, window=None) -> float:
    """Loss::background_penalty_loss (source/utils/loss.cpp:53-64)."""
    excess = np.maximum(0.0, wafer - penalty_threshold)
    bg = (target < 0.5)
    v = excess * excess * bg
    if window is not None:
        v = v * window
    return float(v.sum())


def pe_loss_with_penalty(wafer, target, penalty, penalty_threshold, window=None) -> float:
    """Loss::pe_loss_with_penalty (source/utils/loss.cpp:25-51)."""
    return pe_loss(wafer, target, window) + penalty * background_penalty_loss(
        wafer, target, penalty_threshold, window)


# ---------------------------------------------------------------- adjoint
def backpropagate(dLdI: np.ndarray, fields: Sequence[np.ndarray], cache: OracleCache,
                  output_scale: float) -> np.ndarray:
    """Gradient::_backpropagate (source/utils/gradient.cpp:34-109)."""
    N = cache.N
    if dLdI.shape != (N, N):
        raise ValueError("Gradient: dLdI dimensions do not match cache")
    inv = 1.0 / float(N * N)
    weights = cache.weights
    grad = np.zeros((N, N), dtype=np.float64)
    for k, e in enumerate(fields):
        buf = _fft2(ifftshift(e * dLdI))                                      # :72-76
        buf *= np.conj(cache.kernels[k])                                     # :78
        buf = fftshift(_ifft2_unnormalised(buf))                             # :80-84
        grad += output_scale * weights[k] * inv * buf.real                   # :86-87
    return grad / cache.ws_sum                                               # :98-107


def pe_dLdI(wafer, target, pe_window=None, pe_weight=1.0, penalty=0.0,
            penalty_threshold=0.01, penalty_window=None):
    """dL/dI of every pe_gradient* variant (source/utils/gradient.cpp:121-196).

    The common 4*alpha factor is applied by the caller via output_scale.
    """
    residual = wafer - target
    if pe_window is not None:
        residual = residual * pe_window
    s = pe_weight * residual
    if penalty != 0.0:
        bg = (target < 0.5).astype(np.float64)
        excess = np.maximum(wafer - penalty_threshold, 0.0)
        pen = penalty * bg * excess
        pw = penalty_window if penalty_window is not None else pe_window
        if pw is not None:
            pen = pen * pw
        s = s + pen
    return s * wafer * (1.0 - wafer)


def pe_gradient(wafer, target, fields, cache, alpha, **kw):
    """Gradient::pe_gradient / pe_gradient_with_penalty (gradient.cpp:121-196)."""
    return backpropagate(pe_dLdI(wafer, target, **kw), fields, cache, 4.0 * alpha)


# ---------------------------------------------------------------- CTM
def initialize_theta(target: np.ndarray) -> np.ndarray:
    """CTM_Optimizer::_initialize_theta (source/optimizer/CTM_Optimizer.cpp:55-64)."""
    pi = 3.14159265358979323846
    return np.where(target > 0.0, 0.3 * pi, 0.7 * pi)


def theta_to_mask(theta):
    """CTM_Optimizer.cpp:81: mask = 0.5 (1 + cos theta)."""
    return 0.5 * (1.0 + np.cos(theta))


def ctm_evaluate(theta, target, cache, threshold, alpha):
    """CTM_Optimizer::_evaluate_theta_objective (CTM_Optimizer.cpp:175-187).

    Returns dict(loss, mask, aerial, wafer, grad_mask, grad_theta, grad_norm).
    """
    mask = theta_to_mask(theta)
    aerial, wafer, fields = imaging_compute(mask, cache, threshold, alpha)
    gm = pe_gradient(wafer, target, fields, cache, alpha)
    gt = -0.5 * gm * np.sin(theta)                                           # :151, :183
    return dict(loss=pe_loss(wafer, target), mask=mask, aerial=aerial, wafer=wafer,
                grad_mask=gm, grad_theta=gt, grad_norm=float(np.linalg.norm(gt)))


def pe_evaluate_streamed(mask, target, kernel_at, weights, ws_sum, threshold, alpha):
    """Imaging::compute then Gradient::pe_gradient (imaging.cpp:60-171,
    gradient.cpp:34-133) with the kernels produced one at a time by kernel_at(k)
    (an N x N DC-at-corner array) and no field kept: the forward accumulates
    sum_k w_k |E_k|^2 in k order; the adjoint recomputes E_k from the cached mask
    spectrum before its two FFTs. The FFTs, shifts and sums are the reference's;
    only the storage differs, so that 4096^2 x 48 kernels fits in host memory.

    Returns dict(aerial, wafer, loss, grad_mask)."""
    mask = np.asarray(mask, dtype=np.float64)
    N = mask.shape[0]
    inv = 1.0 / float(N * N)
    K = len(weights)
    mask_frequency = _fft2(ifftshift(mask.astype(np.complex128)))
    aerial = np.zeros((N, N), dtype=np.float64)
    for k in range(K):
        e = fftshift(_ifft2_unnormalised(mask_frequency * kernel_at(k)) * inv)
        aerial += weights[k] * (e.real ** 2 + e.imag ** 2)
        del e
    aerial /= ws_sum
    wafer = 1.0 / (1.0 + np.exp(-alpha * (aerial - threshold)))
    dldi = pe_dLdI(wafer, target)
    grad = np.zeros((N, N), dtype=np.float64)
    scale = 4.0 * alpha
    for k in range(K):
        h = kernel_at(k)
        e = fftshift(_ifft2_unnormalised(mask_frequency * h) * inv)
        buf = _fft2(ifftshift(e * dldi))
        del e
        buf *= np.conj(h)
        buf = fftshift(_ifft2_unnormalised(buf))
        grad += scale * weights[k] * inv * buf.real
        del buf
    grad /= ws_sum
    return dict(aerial=aerial, wafer=wafer, loss=pe_loss(wafer, target), grad_mask=grad)


def ctm_gradient_descent(target, cache, threshold, alpha, iterations, learning_rate,
                         tolerance):
    """CTM_Optimizer::_optimize_gradient_descent (CTM_Optimizer.cpp:109-173)."""
    theta = initialize_theta(target)
    mask = theta_to_mask(theta)
    history = []
    best_mask, min_pe = mask, float("inf")
    for _ in range(iterations):
        r = ctm_evaluate(theta, target, cache, threshold, alpha)
        pe = r["loss"]
        history.append(pe)
        if pe < min_pe:
            min_pe, best_mask = pe, r["mask"]
        if r["grad_norm"] <= tolerance:
            break
        theta = theta - learning_rate * r["grad_theta"]
    return best_mask, history, theta


# ---------------------------------------------------------------- EPE metric
def bilinear_stencil(rows, cols, y, x):
    """make_bilinear_stencil (source/utils/epe_utils.cpp:39-67).

    Clamp to pixel centres, up to four (y, x, weight) entries, zero weights
    dropped and repeated edge pixels merged.
    """
    yy = min(max(y, 0.0), rows - 1.0)
    xx = min(max(x, 0.0), cols - 1.0)
    y0 = int(math.floor(yy)); x0 = int(math.floor(xx))
    y1 = min(y0 + 1, rows - 1); x1 = min(x0 + 1, cols - 1)
    wy1 = 0.0 if y1 == y0 else yy - y0
    wx1 = 0.0 if x1 == x0 else xx - x0
    out = []
    for py, wy in ((y0, 1.0 - wy1), (y1, wy1)):
        for px, wx in ((x0, 1.0 - wx1), (x1, wx1)):
            w = wy * wx
            if w <= 0.0:
                continue
            for i, (ey, ex, ew) in enumerate(out):
                if ey == py and ex == px:
                    out[i] = (ey, ex, ew + w)
                    break
            else:
                out.append((py, px, w))
    return out


def bilinear_sample(field, stencil):
    return sum(w * field[y, x] for (y, x, w) in stencil)


def evaluate_sparse_epe(aerial, eps, weights, threshold, pixel_size_nm):
    """Loss::evaluate_sparse_epe (source/utils/loss.cpp:125-163)."""
    from .levelset_oracle import gradient_1d
    gx = gradient_1d(aerial, 1.0, 1)
    gy = gradient_1d(aerial, 1.0, 0)
    mag = np.maximum(np.sqrt(gx * gx + gy * gy), 1e-6)
    n = len(weights)
    signed = np.full(n, np.nan)
    loss = 0.0; abs_nm = 0.0; active = 0
    for i in range(n):
        if weights[i] <= 0.0:
            continue
        st = bilinear_stencil(aerial.shape[0], aerial.shape[1], eps[i][0], eps[i][1])
        a = bilinear_sample(aerial, st)
        m = max(bilinear_sample(mag, st), 1e-6)
        s = (a - threshold) / m
        signed[i] = s
        loss += weights[i] * s * s
        abs_nm += abs(s) * pixel_size_nm
        active += 1
    return dict(signed_epe_pixel=signed, weighted_squared_loss=loss,
                absolute_sum_nm=abs_nm, active_count=active)


def epe_gradient(aerial, fields, cache, eps, weights, threshold):
    """Gradient::epe_gradient (source/utils/gradient.cpp:198-227): frozen |grad I|,
    dL/dI = 2 w (I - thr) / G^2 scattered onto the bilinear stencil (bilinear_scatter,
    source/utils/epe_utils.cpp:76-80), back-propagated with output scale 2."""
    from .levelset_oracle import gradient_1d
    gx = gradient_1d(aerial, 1.0, 1)
    gy = gradient_1d(aerial, 1.0, 0)
    mag = np.maximum(np.sqrt(gx * gx + gy * gy), 1e-6)
    N = cache.N
    dldi = np.zeros((N, N))
    for i in range(len(weights)):
        if weights[i] <= 0.0:
            continue
        st = bilinear_stencil(N, N, eps[i][0], eps[i][1])
        a = bilinear_sample(aerial, st)
        m = max(bilinear_sample(mag, st), 1e-6)
        g = 2.0 * weights[i] * (a - threshold) / (m * m)
        for (y, x, w) in st:
            dldi[y, x] += w * g
    return backpropagate(dldi, fields, cache, 2.0)
