"""FP64 restatement of the reference's one-time optical set-up.

Test infrastructure only (see ``oracle/__init__.py``). Grid, pupil, Zernike
wavefront, annular source and the SOCS / Abbe kernel generation of
source/litho_model/{grid,pupil,zernike,source,litho_prepare}.cpp, used to
build the real-optics caches of the reference's own tests.
"""
from __future__ import annotations

import math
from typing import Dict, Optional

import numpy as np

from .imaging_oracle import OracleCache, ifftshift


def fft_freq_axis(N: int, pixel_nm: float) -> np.ndarray:
    """Grid::fftF (source/litho_model/grid.cpp:38-48): (i - N/2) / (N dx), C integer N/2."""
    df = 1.0 / (N * pixel_nm)
    return (np.arange(N) - N // 2) * df


def normalised_axis(N: int, pixel_nm: float, na: float, wavelength: float) -> np.ndarray:
    """Grid ctor (grid.cpp:27): Fx_1d = fftF / (NA / lambda)."""
    return fft_freq_axis(N, pixel_nm) / (na / wavelength)


def zernike_wavefront(fx: np.ndarray, fy: np.ndarray, coeffs: Dict[int, float]) -> np.ndarray:
    """ZernikeGenerator::wavefront (source/litho_model/zernike.cpp:12-56), Fringe 1-11."""
    r2 = fx * fx + fy * fy
    s3, s5, s6, s8 = math.sqrt(3), math.sqrt(5), math.sqrt(6), math.sqrt(8)
    table = {
        1: lambda: np.ones_like(fx), 2: lambda: 2.0 * fx, 3: lambda: 2.0 * fy,
        4: lambda: s3 * (2.0 * r2 - 1.0), 5: lambda: s6 * (2.0 * fx * fy),
        6: lambda: s6 * (fx * fx - fy * fy), 7: lambda: s8 * (3.0 * r2 - 2.0) * fy,
        8: lambda: s8 * (3.0 * r2 - 2.0) * fx, 9: lambda: s8 * (3.0 * fx * fx * fy - fy ** 3),
        10: lambda: s8 * (fx ** 3 - 3.0 * fx * fy * fy),
        11: lambda: s5 * (6.0 * r2 * r2 - 6.0 * r2 + 1.0),
    }
    W = np.zeros_like(fx)
    for idx, c in coeffs.items():
        if c == 0.0:
            continue
        W = W + c * (table[idx]() if idx in table else 0.0)
    return W


def pupil(N, pixel_nm, na, wavelength, aberrations: Optional[Dict[int, float]] = None):
    """Pupil (source/litho_model/pupil.cpp:14-46): circ(rho<=1) * exp(i 2 pi W), DC centred."""
    f = normalised_axis(N, pixel_nm, na, wavelength)
    fx = np.broadcast_to(f[None, :], (N, N))
    fy = np.broadcast_to(f[:, None], (N, N))
    amp = ((fx * fx + fy * fy) <= 1.0).astype(np.float64)
    W = zernike_wavefront(fx, fy, aberrations or {})
    return amp * np.exp(1j * 2.0 * np.pi * W)


def source_map(freq_coords: np.ndarray, sigma_in: float, sigma_out: float, upsample: int = 10):
    """Source::compute_source_map (source/litho_model/source.cpp:114-158), smoothing 0."""
    ff = freq_coords[(freq_coords >= -2.0) & (freq_coords <= 2.0)]
    num = ff.size
    hi = np.linspace(ff[0], ff[-1], num * upsample)
    ffx = hi[None, :]
    ffy = hi[:, None]
    rho = np.sqrt(ffx * ffx + ffy * ffy)
    pat = ((sigma_out - rho) > 0.0).astype(np.float64) * ((rho - sigma_in) > 0.0).astype(np.float64)
    if upsample > 1:
        pat = pat.reshape(num, upsample, num, upsample).mean(axis=(1, 3))
    pat = np.maximum(pat, 0.0)
    if pat.max() <= 0:
        raise RuntimeError("source map is all zero")
    return ff, pat


def extract_source_points(coords, weight_map, min_weight=1e-8):
    """LithoPrepare::_extract_source_points (litho_prepare.cpp:65-102), row-major order."""
    ii, jj = np.nonzero(weight_map > min_weight)
    return coords[jj].copy(), coords[ii].copy(), weight_map[ii, jj].copy()


def _bilinear_shift(P, rows, cols, r0, c0, tr, tc):
    N = P.shape[0]

    def at(r, c):
        ok = (r >= 0) & (r < N) & (c >= 0) & (c < N)
        out = np.zeros(np.broadcast(r, c).shape, dtype=np.complex128)
        rr = np.clip(r, 0, N - 1); cc = np.clip(c, 0, N - 1)
        out[ok] = P[rr, cc][ok]
        return out

    ra = rows[:, None] + r0; rb = ra + 1
    ca = cols[None, :] + c0; cb = ca + 1
    return ((1 - tr) * (1 - tc) * at(ra, ca) + (1 - tr) * tc * at(ra, cb)
            + tr * (1 - tc) * at(rb, ca) + tr * tc * at(rb, cb))


def prepare(N, pixel_nm, wavelength, na, sigma_in, sigma_out, use_socs=True,
            compact=False, num_socs=36, aberrations=None) -> OracleCache:
    """LithoPrepare (source/litho_model/litho_prepare.cpp:16-385)."""
    P = pupil(N, pixel_nm, na, wavelength, aberrations)
    fnorm = normalised_axis(N, pixel_nm, na, wavelength)
    coords, wmap = source_map(fnorm, sigma_in, sigma_out)
    fs, gs, ws = extract_source_points(coords, wmap)
    dfx = fnorm[1] - fnorm[0]
    dfy = dfx
    Ns = fs.size
    if not use_socs:
        kernels = []
        allr = np.arange(N)
        for i in range(Ns):
            dc = fs[i] / dfx; dr = gs[i] / dfy
            c0 = int(math.floor(dc)); r0 = int(math.floor(dr))
            sp = _bilinear_shift(P, allr, allr, r0, c0, dr - r0, dc - c0)
            kernels.append(ifftshift(sp))                                   # :217-218
        return OracleCache(N=N, kernels=kernels, source_ws=ws, eigenvalues=())
    oy, ox, ey, ex = 0, 0, N, N
    if compact:                                                             # :239-255
        nz = np.argwhere(P != 0)
        py0, px0 = nz.min(axis=0)
        py1, px1 = nz.max(axis=0)
        oy = max(0, int(py0) - int(math.floor(gs.max() / dfy)) - 1)
        ox = max(0, int(px0) - int(math.floor(fs.max() / dfx)) - 1)
        ey = min(N, int(py1) - int(math.floor(gs.min() / dfy)) + 1)
        ex = min(N, int(px1) - int(math.floor(fs.min() / dfx)) + 1)
    Nr, Nc = ey - oy, ex - ox
    A = np.empty((Nr * Nc, Ns), dtype=np.complex128)
    rows = np.arange(oy, ey); cols = np.arange(ox, ex)
    for i in range(Ns):                                                     # :266-294
        dc = fs[i] / dfx; dr = gs[i] / dfy
        c0 = int(math.floor(dc)); r0 = int(math.floor(dr))
        sp = _bilinear_shift(P, rows, cols, r0, c0, dr - r0, dc - c0)
        A[:, i] = math.sqrt(ws[i]) * sp.reshape(-1, order="F")
    U, S, _ = np.linalg.svd(A, full_matrices=False)                         # :298 (thin SVD)
    K = min(num_socs if num_socs > 0 else Ns, S.size)
    kernels = []
    for k in range(K):                                                      # :319-345
        kf = np.zeros((N, N), dtype=np.complex128)
        kf[oy:ey, ox:ex] = U[:, k].reshape((Nr, Nc), order="F")
        kernels.append(ifftshift(kf))
    return OracleCache(N=N, kernels=kernels, source_ws=ws,
                       eigenvalues=tuple(float(s * s) for s in S[:K]))


def synthetic_gaussian_cache(n: int, socs: bool) -> OracleCache:
    """make_cache of tests/test_micro_gradient_exchange.cpp:27-45 (K=2 smooth kernels)."""
    kernels = []
    idx = np.arange(n)
    f = np.where(idx <= n // 2, idx, idx - n) / n
    fx = f[None, :]; fy = f[:, None]
    for k in range(2):
        amp = np.exp(-(12.0 + 8.0 * k) * (fx * fx + fy * fy))
        kernels.append(amp * np.exp(1j * k * (0.35 * fx - 0.2 * fy)))
    return OracleCache(N=n, kernels=kernels, source_ws=np.array([0.5, 0.5]),
                       eigenvalues=(0.7, 0.3) if socs else ())
