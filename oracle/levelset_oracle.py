"""FP64 restatement of the reference WENO5-Godunov level-set path.

Test infrastructure only (see ``oracle/__init__.py``). Follows
source/utils/level_set_utils.cpp and source/optimizer/LSM_Optimizer.cpp of
the reference; vectorised over rows/columns but with the same arithmetic
per element.
"""
from __future__ import annotations

import numpy as np

EPS_DBL = np.finfo(np.float64).eps


def pad_edge(data: np.ndarray, pad: int, axis: int) -> np.ndarray:
    """LevelSetUtils::pad_edge (level_set_utils.cpp:19-43): edge replication."""
    widths = [(0, 0), (0, 0)]
    widths[axis] = (pad, pad)
    return np.pad(data, widths, mode="edge")


def weno5_rows(v: np.ndarray, n_orig: int, dx: float, direction: str) -> np.ndarray:
    """LevelSetUtils::weno5_1d (level_set_utils.cpp:45-113) applied to every row of v."""
    D1 = (v[:, 1:] - v[:, :-1]) / dx
    if direction == "plus":
        v1, v2, v3, v4, v5 = (D1[:, 5:5 + n_orig], D1[:, 4:4 + n_orig], D1[:, 3:3 + n_orig],
                              D1[:, 2:2 + n_orig], D1[:, 1:1 + n_orig])
    else:
        v1, v2, v3, v4, v5 = (D1[:, 0:n_orig], D1[:, 1:1 + n_orig], D1[:, 2:2 + n_orig],
                              D1[:, 3:3 + n_orig], D1[:, 4:4 + n_orig])
    c13, c76, c116, c16, c56 = 1.0 / 3.0, 7.0 / 6.0, 11.0 / 6.0, 1.0 / 6.0, 5.0 / 6.0
    cS1, cS2 = 13.0 / 12.0, 0.25
    d1 = c13 * v1 - c76 * v2 + c116 * v3
    d2 = -c16 * v2 + c56 * v3 + c13 * v4
    d3 = c13 * v3 + c56 * v4 - c16 * v5
    t1 = v1 - 2 * v2 + v3
    t2 = v2 - 2 * v3 + v4
    t3 = v3 - 2 * v4 + v5
    S1 = cS1 * t1 * t1 + cS2 * (v1 - 4 * v2 + 3 * v3) ** 2
    S2 = cS1 * t2 * t2 + cS2 * (v2 - v4) ** 2
    S3 = cS1 * t3 * t3 + cS2 * (3 * v3 - 4 * v4 + v5) ** 2
    vmax2 = np.maximum.reduce([v1 * v1, v2 * v2, v3 * v3, v4 * v4, v5 * v5])
    eps = 1e-6 * vmax2 + 1e-99
    a1 = 0.1 / ((S1 + eps) * (S1 + eps))
    a2 = 0.6 / ((S2 + eps) * (S2 + eps))
    a3 = 0.3 / ((S3 + eps) * (S3 + eps))
    return (a1 * d1 + a2 * d2 + a3 * d3) / (a1 + a2 + a3)


def der_weno5(M: np.ndarray, dx: float, direction: str, axis: int = -1) -> np.ndarray:
    """LevelSetUtils::der_weno5 (level_set_utils.cpp:115-148)."""
    if direction not in ("plus", "minus"):
        raise ValueError("direction must be plus or minus")
    is_2d = M.shape[0] > 1 and M.shape[1] > 1
    ax = (1 if is_2d else 0) if axis == -1 else axis
    padded = pad_edge(M, 3, ax)
    if ax == 0:
        return weno5_rows(padded.T, M.shape[0], dx, direction).T
    return weno5_rows(padded, M.shape[1], dx, direction)


def evolve_normal_weno_godunov(phi: np.ndarray, Vn: np.ndarray, dy: float, dx: float):
    """LevelSetUtils::evolve_normal_WENO_godunov (level_set_utils.cpp:150-225).

    Returns (delta, H1_abs, H2_abs).
    """
    if phi.shape != Vn.shape:
        raise ValueError("evolve_normal_WENO_godunov: phi and Vn sizes must match")
    if phi.size == 0 or dx <= 0.0 or dy <= 0.0:
        raise ValueError("evolve_normal_WENO_godunov: grid must be non-empty and dx/dy must be positive")
    data_ext = pad_edge(pad_edge(phi, 3, 0), 3, 1)
    vn_ext = pad_edge(pad_edge(Vn, 3, 0), 3, 1)
    pxm = der_weno5(data_ext, dx, "minus", 1)
    pxp = der_weno5(data_ext, dx, "plus", 1)
    pym = der_weno5(data_ext.T, dy, "minus", 1).T
    pyp = der_weno5(data_ext.T, dy, "plus", 1).T
    pos = vn_ext > 0.0
    neg = vn_ext < 0.0
    gx_pos = np.maximum(np.maximum(pxm, 0.0) ** 2, np.minimum(pxp, 0.0) ** 2)
    gy_pos = np.maximum(np.maximum(pym, 0.0) ** 2, np.minimum(pyp, 0.0) ** 2)
    gx_neg = np.maximum(np.minimum(pxm, 0.0) ** 2, np.maximum(pxp, 0.0) ** 2)
    gy_neg = np.maximum(np.minimum(pym, 0.0) ** 2, np.maximum(pyp, 0.0) ** 2)
    gsq = np.where(pos, gx_pos + gy_pos, np.where(neg, gx_neg + gy_neg, 0.0))
    delta_ext = vn_ext * np.sqrt(gsq)
    r, c = phi.shape
    delta = delta_ext[3:3 + r, 3:3 + c]
    h = np.abs(vn_ext)[3:3 + r, 3:3 + c]
    return delta, h.copy(), h.copy()


def gradient_1d(M: np.ndarray, d: float, axis: int) -> np.ndarray:
    """LevelSetUtils::_gradient_1d (level_set_utils.cpp:228-255)."""
    out = np.empty_like(M, dtype=np.float64)
    if axis == 0:
        out[0] = (-3 * M[0] + 4 * M[1] - M[2]) / (2 * d)
        out[-1] = (3 * M[-1] - 4 * M[-2] + M[-3]) / (2 * d)
        out[1:-1] = (M[2:] - M[:-2]) / (2 * d)
    else:
        out[:, 0] = (-3 * M[:, 0] + 4 * M[:, 1] - M[:, 2]) / (2 * d)
        out[:, -1] = (3 * M[:, -1] - 4 * M[:, -2] + M[:, -3]) / (2 * d)
        out[:, 1:-1] = (M[:, 2:] - M[:, :-2]) / (2 * d)
    return out


def evolve_kappa(phi: np.ndarray, dx: float, dy: float, b: float) -> np.ndarray:
    """LevelSetUtils::evolve_kappa (level_set_utils.cpp:257-278)."""
    px = gradient_1d(phi, dx, 1)
    py = gradient_1d(phi, dy, 0)
    pxy = gradient_1d(px, dy, 0)
    pxx = gradient_1d(px, dx, 1)
    pyy = gradient_1d(py, dy, 0)
    g2 = px * px + py * py
    num = pxx * py * py - 2.0 * px * py * pxy + pyy * px * px
    out = np.zeros_like(phi, dtype=np.float64)
    m = g2 > EPS_DBL
    out[m] = num[m] / g2[m]
    return b * out


def get_dt_normal_kappa(cfl, dx, dy, H1, H2, b) -> float:
    """LevelSetUtils::get_dt_normal_kappa (level_set_utils.cpp:280-288)."""
    normal = float(np.max(H1)) / dx + float(np.max(H2)) / dy
    kappa = b * (1.0 / (dx * dx) + 1.0 / (dy * dy)) * 2
    den = normal + kappa
    if den < 1e-9:
        return 1e-3
    return cfl / den


def reinit_sdf(phi: np.ndarray, dx: float, dy: float) -> np.ndarray:
    """LevelSetUtils::reinit_sdf (level_set_utils.cpp:290-319) via cv2 (same library)."""
    import cv2
    inside = phi > 0
    mask_out = np.where(inside, 0, 255).astype(np.uint8)
    mask_in = np.where(inside, 255, 0).astype(np.uint8)
    d_out = cv2.distanceTransform(mask_out, cv2.DIST_L2, 5)
    d_in = cv2.distanceTransform(mask_in, cv2.DIST_L2, 5)
    return d_in.astype(np.float64) * dx - d_out.astype(np.float64) * dx


def evolution_term(phi, Gm, dx, dy, cfl, b):
    """LSM_Optimizer::_caculate_evolution_term (LSM_Optimizer.cpp:47-58)."""
    delta, h1, h2 = evolve_normal_weno_godunov(phi, Gm, dy, dx)
    normal = evolve_kappa(phi, dx, dy, b) - delta
    return normal, get_dt_normal_kappa(cfl, dx, dy, h1, h2, b)


def lsm_rk2_update(phi, Gm, dx, dy, cfl, b):
    """One RK2 update (LSM_Optimizer.cpp:109-115); the second stage reuses dt."""
    n0, dt = evolution_term(phi, Gm, dx, dy, cfl, b)
    phi1 = phi + dt * n0
    n1, _ = evolution_term(phi1, Gm, dx, dy, cfl, b)
    return 0.5 * phi + 0.5 * (phi1 + dt * n1), dt


def render_levelset_mask(phi: np.ndarray, mask_type: str = "Gray", scale: int = 4) -> np.ndarray:
    """render_levelset_mask (source/utils/levelset_mask_renderer.cpp:7-33).

    Binary: phi >= 0. Gray: float32 phi bilinearly upsampled by `scale` with
    cv2.resize(INTER_LINEAR) (the library the reference calls), each scale x scale
    block of subpixels counted where phi >= 0, divided by scale^2."""
    phi = np.asarray(phi)
    if mask_type == "Binary":
        return (phi >= 0.0).astype(np.float64)
    import cv2
    h, w = phi.shape
    hi = cv2.resize(phi.astype(np.float32), (w * scale, h * scale), interpolation=cv2.INTER_LINEAR)
    inside = (hi >= 0.0).reshape(h, scale, w, scale).sum(axis=(1, 3))
    return inside / float(scale * scale)
