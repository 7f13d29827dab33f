"""Host-side file formats and the CTM -> LSM hand-off of the reference.

* :func:`save_mat`, :func:`save_mat_int`, :func:`load_txt` - ``SaveTxt``
  (source/utils/save_txt.cpp:23-105): whitespace-separated text matrices with a
  ``# rows=R cols=C`` header; ``load_txt`` skips blank and ``#`` lines and requires a
  constant column count.
* :func:`load_target_image` - the demos' target bitmap load (cv::imread grayscale / 255).
* :func:`binarize`, :func:`binarize_otsu` - ``Imbinarize::binarize`` /
  ``binarize_OTSU`` (source/utils/imbinarize.cpp:12-37): the gray CTM mask scaled to
  8 bits and thresholded with OpenCV's adaptive Gaussian or Otsu threshold, the
  same library calls the reference makes.
* :func:`binarize_advanced` - ``Imbinarize::binarize_advanced``
  (source/utils/imbinarize.cpp:84-189), the CTM -> LSM hand-off of the demos: peak
  quantile threshold, small-component removal, SRAFs kept outside a keep-out disk
  around the target, final small-component pass.
* :func:`write_lsm_history_csv`, :func:`write_core_metrics_csv`,
  :func:`write_summary_csv` - the ``history.csv``, ``core_metrics_best.csv`` and
  ``summary.csv`` of a full-chip LSM run (demo/demo_full_chip_lsm.cpp:170-201): the
  same columns, values printed with 17 significant digits.

These run once per optimisation on the host; they accept NumPy arrays or tensors.
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np


def _numpy(m):
    if hasattr(m, "detach"):
        m = m.detach().cpu().numpy()
    return np.asarray(m, dtype=np.float64)


def save_mat(m, path: str, precision: int = 6) -> None:
    """SaveTxt::save_mat (save_txt.cpp:23-36): fixed-point values, one row per line."""
    a = _numpy(m)
    with open(path, "w") as f:
        f.write(f"# rows={a.shape[0]} cols={a.shape[1]}\n")
        for row in a:
            f.write(" ".join(f"{v:.{precision}f}" for v in row) + "\n")


def save_mat_int(m, path: str) -> None:
    """SaveTxt::save_mat_int (save_txt.cpp:38-50): values rounded half away from zero."""
    a = _numpy(m)
    r = np.where(a >= 0, np.floor(a + 0.5), np.ceil(a - 0.5)).astype(np.int64)
    with open(path, "w") as f:
        f.write(f"# rows={a.shape[0]} cols={a.shape[1]}\n")
        for row in r:
            f.write(" ".join(str(int(v)) for v in row) + "\n")


def load_txt(path: str) -> np.ndarray:
    """SaveTxt::load_txt (save_txt.cpp:57-105)."""
    if not os.path.exists(path):
        raise ValueError(f"load_txt: cannot open {path}")
    rows = []
    with open(path) as f:
        for line in f:
            s = line.strip()
            if not s or s.startswith("#"):
                continue
            vals = [float(t) for t in s.split()]
            if rows and len(vals) != len(rows[0]):
                raise ValueError(f"load_txt: inconsistent column count at row {len(rows) + 1} "
                                 f"in {path}")
            rows.append(vals)
    if not rows:
        raise ValueError(f"load_txt: empty matrix in {path}")
    return np.array(rows, dtype=np.float64)


def load_target_image(path: str) -> np.ndarray:
    """A target bitmap as the demos read it (demo/demo_full_chip_ctm.cpp:62-66,
    demo/demo_full_chip_lsm.cpp:93-97): cv::imread(IMREAD_GRAYSCALE), then each 8-bit
    pixel / 255 as float64."""
    import cv2
    img = cv2.imread(path, cv2.IMREAD_GRAYSCALE)
    if img is None:
        raise ValueError(f"load_target_image: cannot read {path}")
    return img.astype(np.float64) / 255.0


def _gray_u8(gray_mask):
    a = _numpy(gray_mask)
    # cv::Mat::convertTo(CV_8U, 255): round to nearest, saturate to [0, 255]
    return np.clip(np.rint(a * 255.0), 0, 255).astype(np.uint8)


def binarize(gray_mask, block_size: int = 51, c: float = -0.5) -> np.ndarray:
    """Imbinarize::binarize (imbinarize.cpp:12-26): adaptive Gaussian threshold."""
    import cv2
    bw = cv2.adaptiveThreshold(_gray_u8(gray_mask), 255, cv2.ADAPTIVE_THRESH_GAUSSIAN_C,
                               cv2.THRESH_BINARY, block_size, c)
    return bw.astype(np.float64) / 255.0


def binarize_otsu(gray_mask) -> np.ndarray:
    """Imbinarize::binarize_OTSU (imbinarize.cpp:28-37): Otsu threshold."""
    import cv2
    _, bw = cv2.threshold(_gray_u8(gray_mask), 0, 255, cv2.THRESH_BINARY | cv2.THRESH_OTSU)
    return bw.astype(np.float64) / 255.0


@dataclass
class BinarizeResult:
    """BinarizeResult (include/utils/imbinarize.h:13-20): 0/1 float64 masks."""
    initial_binary_mask: np.ndarray
    filtered_binary_mask: np.ndarray
    sraf_mask_initial: np.ndarray
    sraf_mask_final: np.ndarray
    final_mask: np.ndarray
    keep_out_zone: np.ndarray


def _quantile_linear(vals: np.ndarray, q: float) -> float:
    """_quantile (imbinarize.cpp:50-63): order statistics at floor/ceil of q (n - 1),
    then v_lo + (v_hi - v_lo) (pos - lo)."""
    if vals.size == 0:
        return 0.0
    q = min(max(q, 0.0), 1.0)
    pos = q * (vals.size - 1)
    lo, hi = int(np.floor(pos)), int(np.ceil(pos))
    v = np.sort(vals)
    if lo == hi:
        return float(v[lo])
    return float(v[lo] + (v[hi] - v[lo]) * (pos - lo))


def _drop_small_components(bin01: np.ndarray, area_threshold: int) -> np.ndarray:
    """8-connected components (OpenCV, CV_32S labels) with area < area_threshold cleared."""
    import cv2
    n, labels, stats, _ = cv2.connectedComponentsWithStats(bin01, connectivity=8, ltype=cv2.CV_32S)
    small = np.zeros(n, dtype=bool)
    small[1:] = stats[1:, cv2.CC_STAT_AREA] < area_threshold
    out = bin01.copy()
    out[small[labels]] = 0
    return out


def binarize_advanced(gray_mask, target_pattern, peak_min_intensity: float = 0.1,
                      quantile_val: float = 0.2, area_threshold: int = 50,
                      min_spacing_pixels: int = 15) -> BinarizeResult:
    """Imbinarize::binarize_advanced (imbinarize.cpp:84-189)."""
    import cv2
    gray = _numpy(gray_mask)
    tgt = _numpy(target_pattern)
    if gray.shape != tgt.shape:
        raise ValueError("binarize_advanced: gray mask and target sizes must match")
    H, W = gray.shape
    # peak_local_max(min_distance=1): >= its 3x3 dilation and > peak_min_intensity.
    dil = cv2.dilate(gray, cv2.getStructuringElement(cv2.MORPH_RECT, (3, 3)))
    peaks = gray[(gray >= dil) & (gray > peak_min_intensity)]
    if peaks.size == 0:
        z = np.zeros((H, W))
        return BinarizeResult(z, z.copy(), z.copy(), z.copy(), z.copy(), z.copy())
    thr = _quantile_linear(peaks, quantile_val)
    initial = (gray >= thr).astype(np.uint8)
    filtered = _drop_small_components(initial, area_threshold)
    tgt_bin = (tgt > 0.5).astype(np.uint8)
    sraf_initial = filtered * (1 - tgt_bin)
    sraf_final = sraf_initial.copy()
    keep_out = np.zeros((H, W), dtype=np.uint8)
    if min_spacing_pixels > 0:
        k = 2 * min_spacing_pixels + 1
        keep_out = cv2.dilate(tgt_bin, cv2.getStructuringElement(cv2.MORPH_ELLIPSE, (k, k)))
        sraf_final = sraf_initial * (1 - keep_out)
    final = _drop_small_components(np.bitwise_or(tgt_bin, sraf_final), area_threshold)
    f = lambda m: m.astype(np.float64)
    return BinarizeResult(f(initial), f(filtered), f(sraf_initial), f(sraf_final), f(final),
                          f(keep_out))


def _g17(v) -> str:
    """An ostream value under std::setprecision(17): integers as integers, else %.17g."""
    if isinstance(v, (int, np.integer)) and not isinstance(v, bool):
        return str(int(v))
    return "%.17g" % float(v)


LSM_HISTORY_COLUMNS = (
    "iteration,loss,data_loss,cept_loss,min_dt,max_dt,pe_contribution,penalty_contribution,"
    "epe_contribution,cept_contribution,core_pe,core_bg_penalty_raw,core_pe_penalty,"
    "core_epe_squared_pixel,core_epe_abs_sum_nm,core_ep_count,core_epe_mean_nm,core_data_loss,"
    "total_pe,total_bg_penalty_raw,total_epe_squared_pixel,total_epe_abs_sum_nm,total_ep_count,"
    "epe_mean_nm")


def write_lsm_history_csv(history, path: str) -> None:
    """history.csv (demo_full_chip_lsm.cpp:170-186): one row per FullChipLSMIteration."""
    with open(path, "w") as f:
        f.write(LSM_HISTORY_COLUMNS + "\n")
        for r in history:
            c = r.core
            row = (r.iteration, r.loss, r.data_loss, r.cept_loss, r.min_dt, r.max_dt,
                   r.pe_contribution, r.penalty_contribution, r.epe_contribution,
                   r.cept_contribution, c.pe_loss, c.bg_penalty_raw, c.pe_penalty_loss, c.epe_loss,
                   c.epe_abs_sum_nm, int(c.ep_count), c.epe_mean, c.data_loss, r.total_pe_loss,
                   r.total_bg_penalty_raw, r.total_epe_loss, r.total_epe_abs_sum_nm,
                   int(r.total_ep_count), r.epe_mean)
            f.write(",".join(_g17(v) for v in row) + "\n")


CORE_METRICS_COLUMNS = (
    "best_iteration,micro_id,y0,y1,x0,x1,core_pe,core_bg_penalty_raw,core_pe_penalty,"
    "core_epe_squared_pixel,core_epe_abs_sum_nm,core_ep_count,core_epe_mean_nm,core_data_loss")


def write_core_metrics_csv(result, partition, path: str) -> None:
    """core_metrics_best.csv (demo_full_chip_lsm.cpp:187-196): the best round's Core
    metrics per Micro, with its global Core rectangle."""
    with open(path, "w") as f:
        f.write(CORE_METRICS_COLUMNS + "\n")
        for tile, m in zip(partition.tiles, result.best_core_metrics):
            c = tile.core_global
            row = (int(result.best_iteration), int(tile.id), c.y0, c.y1, c.x0, c.x1, m.pe_loss,
                   m.bg_penalty_raw, m.pe_penalty_loss, m.epe_loss, m.epe_abs_sum_nm,
                   int(m.ep_count), m.epe_mean, m.data_loss)
            f.write(",".join(_g17(v) for v in row) + "\n")


def write_summary_csv(result, seconds: float, path: str) -> None:
    """summary.csv (demo_full_chip_lsm.cpp:197-201)."""
    last = result.history[-1]
    with open(path, "w") as f:
        f.write("best_iteration,best_loss,final_iteration,final_loss,seconds\n")
        row = (int(result.best_iteration), result.best_loss, int(last.iteration), last.loss,
               float(seconds))
        f.write(",".join(_g17(v) for v in row) + "\n")
