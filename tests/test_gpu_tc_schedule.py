"""The persistent, warp-specialised tensor-core pipelines (tc3) against the per-tile
kernels (tc2), both split-BF16, through the C ABI.

Both schedules form the same split-BF16 products per pixel in the same order, so the
images (aerial, wafer, dPE/dM, dPE/dtheta) must agree bit for bit; the FP64 loss and
norm sums are added in another order (FP32 over 32 pixels in the pipelines), so they
must agree to 1e-6 relative. Cases: ragged sizes (the last tile row and column only
partly inside the image), batches whose items split unevenly over the SMs, the fused
CTM evaluation, the unfused imaging call (resist synthesis only), the batched PE
gradient with the fused adjoint analysis, and a windowed, penalised gradient.
"""
import importlib

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

LOSS_TOL = 1e-6


@pytest.fixture(scope="module")
def L():
    p = importlib.import_module("c-version-lithography_b200")
    assert torch.cuda.is_available()
    p.load_library()
    return p


@pytest.fixture(scope="module")
def wl():
    return importlib.import_module("c-version-lithography_b200.workloads")


def contexts(L):
    out = {}
    for sched in ("per_tile", "persistent"):
        ctx = L.Context()
        ctx.set_precision("bf16x3")
        ctx.set_tc_schedule(sched)
        out[sched] = ctx
    return out


def close(ctxs):
    for c in ctxs.values():
        c.close()


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


@pytest.mark.parametrize("N,B", [(300, 3), (2048, 4), (520, 7)])
def test_batched_ctm_evaluation_same_on_both_schedules(L, wl, N, B):
    band, r0, c0, w, wss = wl.synthetic_socs_band()
    rng = np.random.default_rng(N + B)
    targets = np.stack([wl.manhattan_target(N, max(4, N // 20), seed=N + b) for b in range(B)])
    thetas = np.stack([wl.theta_init_reference(t) for t in targets])
    thetas = thetas + 0.2 * rng.standard_normal(thetas.shape)
    th = torch.tensor(thetas, dtype=torch.float32, device="cuda")
    tg = torch.tensor(targets, dtype=torch.float32, device="cuda")
    ctxs = contexts(L)
    out = {}
    for sched, ctx in ctxs.items():
        cache = L.ImagingCache.from_band(N, band, r0, c0, w, wss, ctx=ctx)
        losses, grads, norms = L.ctm_evaluate_batch(cache, th, tg, 0.225, 50.0)
        out[sched] = (losses, grads.clone(), norms)
    (l0, g0, n0), (l1, g1, n1) = out["per_tile"], out["persistent"]
    diff = (g0 - g1).abs().max().item()
    print(f"\n{B} x {N}^2: max |dgrad| {diff:.3e} (max |grad| {g0.abs().max().item():.3e}), "
          f"loss rel {max(rel(a, b) for a, b in zip(l1, l0)):.2e}, "
          f"norm rel {max(rel(a, b) for a, b in zip(n1, n0)):.2e}")
    assert torch.equal(g0, g1)
    for b in range(B):
        assert rel(l1[b], l0[b]) <= LOSS_TOL and rel(n1[b], n0[b]) <= LOSS_TOL, b
    close(ctxs)


@pytest.mark.parametrize("N", [130, 1024])
def test_imaging_and_pe_gradient_same_on_both_schedules(L, wl, N):
    band, r0, c0, w, wss = wl.synthetic_socs_band()
    rng = np.random.default_rng(N)
    mask = rng.uniform(0.0, 1.0, (N, N)).astype(np.float32)
    target = wl.manhattan_target(N, max(4, N // 20), seed=3 * N)
    win = np.zeros((N, N), dtype=np.float32)
    win[N // 8:N - N // 5, N // 6:N - N // 9] = 1.0
    ctxs = contexts(L)
    out = {}
    for sched, ctx in ctxs.items():
        cache = L.ImagingCache.from_band(N, band, r0, c0, w, wss, ctx=ctx)
        imaging = L.Imaging(cache)
        r = imaging.compute(mask, 0.225, 50.0)
        grad = L.Gradient(cache, 0.225, 50.0)
        g = grad.pe_gradient_with_penalty(r.wafer_image, target, imaging.get_electric_field(),
                                          1.5, 0.05, loss_window=win)
        masks = torch.tensor(np.stack([mask, target.astype(np.float32)]), device="cuda")
        tgts = torch.tensor(np.stack([target, target]).astype(np.float32), device="cuda")
        bl, bg = L.pe_gradient_batch(cache, masks, tgts, 0.225, 50.0)
        out[sched] = (r.aerial_image.clone(), r.wafer_image.clone(), g.clone(), grad.last_loss,
                      bl, bg.clone())
    a, b = out["per_tile"], out["persistent"]
    for i, name in enumerate(("aerial", "wafer", "windowed penalised gradient")):
        assert torch.equal(a[i], b[i]), name
    assert rel(b[3], a[3]) <= LOSS_TOL
    assert torch.equal(a[5], b[5]), "batched PE gradient"
    for x, y in zip(a[4], b[4]):
        assert rel(y, x) <= LOSS_TOL
    close(ctxs)


def test_schedule_argument_is_checked(L):
    ctx = L.Context()
    assert ctx.lib.litho_ctx_set_tc_schedule(ctx.handle, 3) == 1
    assert ctx.lib.litho_ctx_set_tc_schedule(ctx.handle, 2) == 0
    ctx.close()
