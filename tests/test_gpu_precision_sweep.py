"""Precision sweep of the SOCS forward + adjoint (48 SOCS kernels of 35 x 35).

At 1024^2, for a mask uniform in [0, 1] and a binary Manhattan mask, the FP32 and the
split-BF16 paths are each compared with the FP64 oracle (the reference's FFT
algorithm): max|dI| / max I of the aerial image, the relative L2 error of dPE/dM, and
the EPE difference at 64 seeded edge points of the target (Loss::evaluate_sparse_epe on
each path's own aerial image). The EPE divides by |grad I|, so the points are drawn
among the target's edge points where the FP64 |grad I| is at least 0.01 per pixel (an
EPE of one pixel moves I by 0.01 or more; for a low-contrast image, the 64 steepest);
where the image is flat the EPE is not defined by the image to any precision. At 4096^2 the split-BF16 path is compared with the FP32
path (the oracle's 145 FFTs of 4096^2 complex fields do not fit a test's budget; FP32
against FP64 is pinned at 1024^2).

The EPE of a point is (I - threshold) / |grad I|: an image error dI moves it by about
dI / |grad I| plus EPE times the relative error of |grad I|, so points far from the
printed contour (large EPE) carry proportionally larger differences. The EPE difference
is therefore stated relative, |dEPE| / max(|EPE|, 1 px), and absolute over the points
within 2 px of the contour. EPE is evaluated for the binary masks, whose images have
their edges at the target's; the uniform masks' images have no edges to measure.

Bounds: FP32 1e-5 of peak, gradient 1e-4, EPE 1e-3 (relative); split-BF16 1e-3 of peak
(the stated bound for split-BF16), gradient 1e-3, EPE 1e-2 (relative). Each case prints
its measured errors.
"""
import importlib

import numpy as np
import pytest

from oracle import imaging_oracle as io

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

THR, ALPHA, K = 0.225, 50.0, 48
BOUNDS = {"fp32": (1e-5, 1e-4, 1e-3), "bf16x3": (1e-3, 1e-3, 1e-2)}


@pytest.fixture(scope="module")
def L():
    p = importlib.import_module("c-version-lithography_b200")
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    p.load_library()
    return p


@pytest.fixture(scope="module")
def wl():
    return importlib.import_module("c-version-lithography_b200.workloads")


def cpu(t):
    return t.detach().cpu().numpy().astype(np.float64)


def edge_points(target, n, seed, aerial=None, min_grad=0.01):
    """n seeded points on the 0.5 contour of a binary target (pixel-edge midlines);
    with `aerial`, only points whose nearest pixel has |grad aerial| >= min_grad."""
    from oracle.levelset_oracle import gradient_1d
    rng = np.random.default_rng(seed)
    ys, xs = np.nonzero(np.diff(target, axis=0))
    pts = [(y + 0.5, x + rng.uniform(-0.3, 0.3)) for y, x in zip(ys, xs)]
    ys, xs = np.nonzero(np.diff(target, axis=1))
    pts += [(y + rng.uniform(-0.3, 0.3), x + 0.5) for y, x in zip(ys, xs)]
    pts = np.array(pts)
    if aerial is not None:
        mag = np.hypot(gradient_1d(aerial, 1.0, 1), gradient_1d(aerial, 1.0, 0))
        iy = np.clip(np.rint(pts[:, 0]).astype(int), 0, aerial.shape[0] - 1)
        ix = np.clip(np.rint(pts[:, 1]).astype(int), 0, aerial.shape[1] - 1)
        m = mag[iy, ix]
        keep = m >= min_grad
        if keep.sum() < n:   # a low-contrast image: the n steepest edge points
            keep = np.zeros(len(pts), bool)
            keep[np.argsort(-m)[:n]] = True
        pts = pts[keep]
    return pts[rng.choice(len(pts), size=n, replace=False)]


def device_eval(L, cache, mask, target, eps):
    imaging = L.Imaging(cache)
    r = imaging.compute(mask, THR, ALPHA)
    g = L.Gradient(cache, THR, ALPHA).pe_gradient(r.wafer_image, target, imaging.get_electric_field())
    e = L.Loss.evaluate_sparse_epe(r.aerial_image, eps, np.ones(len(eps)), THR, 1.0, ctx=cache.ctx)
    return cpu(r.aerial_image), cpu(g), np.asarray(e.signed_epe_pixel, dtype=np.float64)


@pytest.fixture(scope="module")
def case1024(wl):
    N = 1024
    band, r0, c0, w, wss = wl.synthetic_socs_band(K=K)
    target = wl.manhattan_target(N, 40, seed=31)
    rng = np.random.default_rng(32)
    masks = {"uniform": rng.uniform(0.0, 1.0, (N, N)), "binary": target.copy()}
    oc = io.OracleCache(N=N, kernels=list(wl.band_to_dense(band, r0, c0, N)),
                        source_ws=np.array([wss]), eigenvalues=tuple(w))
    ref, eps = {}, {}
    for name, m in masks.items():
        m32 = m.astype(np.float32).astype(np.float64)
        a, wafer, fields = io.imaging_compute(m32, oc, THR, ALPHA)
        g = io.pe_gradient(wafer, target, fields, oc, ALPHA)
        eps[name] = edge_points(target, 64, 33, aerial=a)
        e = io.evaluate_sparse_epe(a, eps[name], np.ones(64), THR, 1.0)["signed_epe_pixel"]
        ref[name] = (a, g, e)
        del fields
    return N, (band, r0, c0, w, wss), target, masks, eps, ref


@pytest.mark.parametrize("prec", ["fp32", "bf16x3"])
@pytest.mark.parametrize("mask_kind", ["uniform", "binary"])
def test_precision_1024_against_oracle(L, case1024, prec, mask_kind):
    N, (band, r0, c0, w, wss), target, masks, eps, ref = case1024
    ctx = L.Context()
    ctx.set_precision(prec)
    cache = L.ImagingCache.from_band(N, band, r0, c0, w, wss, ctx=ctx)
    a, g, e = device_eval(L, cache, masks[mask_kind], target, eps[mask_kind])
    ra, rg, re_ = ref[mask_kind]
    di = float(np.max(np.abs(a - ra)) / np.max(np.abs(ra)))
    dg = float(np.linalg.norm(g - rg) / np.linalg.norm(rg))
    bi, bg, be = BOUNDS[prec]
    msg = f"\n1024^2 K={K} {mask_kind} {prec}: max|dI|/max I {di:.2e}, grad rel L2 {dg:.2e}"
    if mask_kind == "binary":
        de_rel, de_abs = epe_errors(e, re_)
        msg += f", EPE rel {de_rel:.2e}, |dEPE| within 2 px of the contour {de_abs}"
        assert de_rel <= be
    print(msg)
    assert di <= bi and dg <= bg
    ctx.close()


def epe_errors(e, ref):
    """max |dEPE| / max(|EPE|, 1) and, as text, max |dEPE| over the points with |EPE| <= 2 px."""
    d = np.abs(e - ref)
    near = np.abs(ref) <= 2.0
    return (float(np.max(d / np.maximum(np.abs(ref), 1.0))),
            f"{float(np.max(d[near])):.2e} px ({int(near.sum())} points)" if near.any() else "n/a")


def test_precision_4096_bf16_against_fp32(L, wl):
    N = 4096
    band, r0, c0, w, wss = wl.synthetic_socs_band(K=K)
    target = wl.manhattan_target(N, 120, seed=41)
    out = {}
    eps = None
    for prec in ("fp32", "bf16x3"):
        ctx = L.Context()
        ctx.set_precision(prec)
        cache = L.ImagingCache.from_band(N, band, r0, c0, w, wss, ctx=ctx)
        if eps is None:   # well-conditioned edge points of the FP32 image
            a32 = cpu(L.Imaging(cache).compute(target, THR, ALPHA).aerial_image)
            eps = edge_points(target, 64, 42, aerial=a32)
        out[prec] = device_eval(L, cache, target, target, eps)
        ctx.close()
    (a32, g32, e32), (a16, g16, e16) = out["fp32"], out["bf16x3"]
    di = float(np.max(np.abs(a16 - a32)) / np.max(np.abs(a32)))
    dg = float(np.linalg.norm(g16 - g32) / np.linalg.norm(g32))
    de_rel, de_abs = epe_errors(e16, e32)
    print(f"\n4096^2 K={K} binary bf16x3 vs fp32: max|dI|/max I {di:.2e}, grad rel L2 {dg:.2e}, "
          f"EPE rel {de_rel:.2e}, |dEPE| within 2 px of the contour {de_abs}")
    assert di <= 1e-3 and dg <= 1e-3 and de_rel <= 1e-2
