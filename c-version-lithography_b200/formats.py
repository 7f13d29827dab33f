"""Host-side file formats and the CTM -> LSM hand-off of the reference.

* :func:`save_mat`, :func:`save_mat_int`, :func:`load_txt` - ``SaveTxt``
  (source/utils/save_txt.cpp:23-105): whitespace-separated text matrices with a
  ``# rows=R cols=C`` header; ``load_txt`` skips blank and ``#`` lines and requires a
  constant column count.
* :func:`binarize`, :func:`binarize_otsu` - ``Imbinarize::binarize`` /
  ``binarize_OTSU`` (source/utils/imbinarize.cpp:12-37): the gray CTM mask scaled to
  8 bits and thresholded with OpenCV's adaptive Gaussian or Otsu threshold, the
  same library calls the reference makes, giving the 0/1 mask that seeds LSM.

These run once per optimisation on the host; they accept NumPy arrays or tensors.
"""
from __future__ import annotations

import os

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
