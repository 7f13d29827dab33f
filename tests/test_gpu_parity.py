"""GPU parity of the imaging / loss / adjoint / CTM path against the FP64 oracle.

Tolerances (FP32 path): aerial image max|dI| <= 1e-5 * max(I); gradients
relative L2 <= 1e-4; PE loss relative 1e-5. Every call goes through the C ABI
of liblitho_b200.so (via the package's ctypes layer).
"""
import glob
import importlib
import os

import numpy as np
import pytest

from oracle import imaging_oracle as io
from oracle import optics_oracle as oo

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
I_TOL = 1e-5
G_TOL = 1e-4


@pytest.fixture(scope="module")
def L():
    p = importlib.import_module("c-version-lithography_b200")
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    p.load_library()
    return p


@pytest.fixture(scope="module")
def wl():
    return importlib.import_module("c-version-lithography_b200.workloads")


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64); b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def peak_err(a, b):
    a = np.asarray(a, dtype=np.float64); b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def cpu(t):
    return t.detach().cpu().numpy().astype(np.float64)


def fixture_cache(name, wl):
    if name.startswith("ctm_real_"):
        n = int(name.split("_")[2].split(".")[0])
        return oo.prepare(n, 4.0, 193.0, 1.35, 0.6, 0.9, use_socs=True)
    if name.startswith("ctm_gauss_"):
        n = int(name.split("_")[2]); socs = "socs" in name
        c = oo.synthetic_gaussian_cache(n, socs)
        c.source_ws = np.array([0.3, 0.9])
        return c
    band, r0, c0, w, wss = wl.synthetic_socs_band()
    return io.OracleCache(N=128, kernels=list(wl.band_to_dense(band, r0, c0, 128)),
                          source_ws=np.array([wss]), eigenvalues=tuple(w))


def device_cache(L, oc):
    return L.ImagingCache.from_kernels(np.stack(oc.kernels), oc.source_ws, oc.eigenvalues)


FIXTURES = sorted(os.path.basename(p) for p in glob.glob(os.path.join(GOLDEN, "ctm_*.npz")))


@pytest.mark.parametrize("name", FIXTURES)
def test_imaging_matches_golden(L, wl, name):
    z = np.load(os.path.join(GOLDEN, name))
    oc = fixture_cache(name, wl)
    cache = device_cache(L, oc)
    imaging = L.Imaging(cache)
    mask = io.theta_to_mask(z["theta"].astype(np.float64))
    r = imaging.compute(mask, float(z["thr"]), float(z["alpha"]))
    assert peak_err(cpu(r.aerial_image), z["aerial"]) <= I_TOL, name
    assert np.max(np.abs(cpu(r.wafer_image) - z["wafer"])) <= float(z["alpha"]) * I_TOL * np.max(z["aerial"])


@pytest.mark.parametrize("name", FIXTURES)
def test_ctm_evaluate_matches_golden(L, wl, name):
    z = np.load(os.path.join(GOLDEN, name))
    cache = device_cache(L, fixture_cache(name, wl))
    opt = L.CTMOptimizer(cache, z["target"], float(z["thr"]), float(z["alpha"]), iterations=1)
    theta = torch.tensor(z["theta"], dtype=torch.float32, device="cuda")
    loss, gt, norm = opt.evaluate(theta, want_mask=True)
    assert abs(loss - float(z["loss"])) <= 1e-5 * max(1.0, abs(float(z["loss"]))), (loss, float(z["loss"]))
    assert rel_l2(cpu(gt), z["grad_theta"]) <= G_TOL, name
    assert abs(norm - float(z["grad_norm"])) <= G_TOL * float(z["grad_norm"])
    assert np.max(np.abs(cpu(opt.mask) - io.theta_to_mask(z["theta"].astype(np.float64)))) < 1e-6


@pytest.mark.parametrize("name", [f for f in FIXTURES if "real" in f])
def test_pe_gradient_variants_match_golden(L, wl, name):
    z = np.load(os.path.join(GOLDEN, name))
    cache = device_cache(L, fixture_cache(name, wl))
    imaging = L.Imaging(cache)
    grad = L.Gradient(cache, float(z["thr"]), float(z["alpha"]))
    mask = io.theta_to_mask(z["theta"].astype(np.float64))
    r = imaging.compute(mask, float(z["thr"]), float(z["alpha"]))
    gm = grad.pe_gradient(z["wafer"], z["target"], imaging.get_electric_field())
    assert rel_l2(cpu(gm), z["grad_mask"]) <= G_TOL
    assert abs(grad.last_loss - float(z["loss"])) <= 1e-6 * float(z["loss"])
    gp = grad.pe_gradient_with_penalty(z["wafer"], z["target"], imaging.get_electric_field(), 2.0, 0.01)
    assert rel_l2(cpu(gp), z["grad_mask_penalty"]) <= G_TOL
    assert abs(grad.last_loss - float(z["loss_penalty"])) <= 1e-6 * float(z["loss_penalty"])
    # Loss statics on the device.
    assert abs(L.Loss.pe_loss(z["wafer"], z["target"]) - float(z["loss"])) <= 1e-6 * float(z["loss"])


def test_windowed_and_weighted_gradient(L):
    """pe_gradient(W,T,E,window) and the (pe_weight, penalty_window) overload vs the oracle."""
    oc = oo.prepare(65, 4.0, 193.0, 1.35, 0.6, 0.9, use_socs=True)
    rng = np.random.default_rng(11)
    n = 65
    mask = rng.random((n, n)); target = (rng.random((n, n)) > 0.5).astype(np.float64)
    win = np.zeros((n, n)); win[8:50, 5:60] = 1.0
    pwin = np.zeros((n, n)); pwin[3:40, 10:64] = 1.0
    a, w, E = io.imaging_compute(mask, oc, 0.25, 30.0)
    cache = device_cache(L, oc)
    imaging = L.Imaging(cache)
    imaging.compute(mask, 0.25, 30.0)
    grad = L.Gradient(cache, 0.25, 30.0)
    g1 = grad.pe_gradient(w, target, imaging.get_electric_field(), loss_window=win)
    ref1 = io.pe_gradient(w, target, E, oc, 30.0, pe_window=win)
    assert rel_l2(cpu(g1), ref1) <= G_TOL
    g2 = grad.pe_gradient_with_penalty(w, target, imaging.get_electric_field(), 1.5, 0.05,
                                       loss_window=win, pe_weight=0.7, penalty_window=pwin)
    ref2 = io.pe_gradient(w, target, E, oc, 30.0, pe_window=win, pe_weight=0.7, penalty=1.5,
                          penalty_threshold=0.05, penalty_window=pwin)
    assert rel_l2(cpu(g2), ref2) <= G_TOL


def test_backpropagate_generic_dldi(L):
    """Gradient::_backpropagate with an arbitrary dL/dI and output scale."""
    oc = oo.synthetic_gaussian_cache(13, True)
    rng = np.random.default_rng(2)
    mask = rng.random((13, 13)); dldi = rng.standard_normal((13, 13))
    _, _, E = io.imaging_compute(mask, oc, 0.2, 5.0)
    ref = io.backpropagate(dldi, E, oc, 2.0)
    cache = device_cache(L, oc)
    imaging = L.Imaging(cache); imaging.compute(mask, 0.2, 5.0)
    got = L.Gradient(cache, 0.2, 5.0).backpropagate(dldi, imaging.get_electric_field(), 2.0)
    assert rel_l2(cpu(got), ref) <= G_TOL


@pytest.mark.parametrize("n", [64, 65])
def test_field_export_matches_reference_fields(L, n):
    """get_electric_field(): exported E_k equal the reference's centred fields."""
    oc = oo.prepare(n, 4.0, 193.0, 1.35, 0.6, 0.9, use_socs=True)
    mask = np.random.default_rng(n).random((n, n))
    _, _, E = io.imaging_compute(mask, oc, 0.25, 85.0)
    cache = device_cache(L, oc)
    imaging = L.Imaging(cache); imaging.compute(mask, 0.25, 85.0)
    field = imaging.get_electric_field()
    for k in (0, 1, len(E) - 1):
        got = field.export(k).cpu().numpy().astype(np.complex128)
        assert np.max(np.abs(got - E[k])) <= 1e-5 * np.max(np.abs(E[0]))


def test_large_tile_matches_oracle(L, wl):
    """2048^2, K = 24 band kernels, benchmark target: image and dPE/dtheta vs FP64."""
    N = 2048
    band, r0, c0, w, wss = wl.synthetic_socs_band()
    target = wl.manhattan_target(N, 100, seed=1, n_lt=10)
    theta = wl.theta_init_reference(target)
    oc = io.OracleCache(N=N, kernels=list(wl.band_to_dense(band, r0, c0, N)),
                        source_ws=np.array([wss]), eigenvalues=tuple(w))
    ref = io.ctm_evaluate(theta, target, oc, 0.225, 50.0)
    cache = L.ImagingCache.from_band(N, band, r0, c0, w, wss)
    assert (cache.Nr, cache.Nc) == (35, 35)
    opt = L.CTMOptimizer(cache, target, 0.225, 50.0, iterations=1)
    th = torch.tensor(theta, dtype=torch.float32, device="cuda")
    aerial = torch.empty_like(th)
    loss, gt, norm = opt.evaluate(th)
    imaging = L.Imaging(cache)
    r = imaging.compute(io.theta_to_mask(theta), 0.225, 50.0)
    assert peak_err(cpu(r.aerial_image), ref["aerial"]) <= I_TOL
    assert rel_l2(cpu(gt), ref["grad_theta"]) <= G_TOL
    assert abs(loss - ref["loss"]) <= 1e-5 * ref["loss"]
    # Printed binary image identical except pixels within 1e-4 of threshold.
    printed = cpu(r.aerial_image) >= 0.225
    printed_ref = ref["aerial"] >= 0.225
    differ = printed != printed_ref
    assert np.all(np.abs(ref["aerial"][differ] - 0.225) <= 1e-4)
    del aerial


def test_shift_equivariance_4096(L, wl):
    """Full-size property: a circular shift of the mask shifts image and gradient (N = 4096, K = 48)."""
    N = 4096
    band, r0, c0, w, wss = wl.synthetic_socs_band(K=48)
    cache = L.ImagingCache.from_band(N, band, r0, c0, w, wss)
    target = torch.tensor(wl.manhattan_target(N, 200, seed=5), dtype=torch.float32, device="cuda")
    rng = np.random.default_rng(9)
    theta = torch.tensor(rng.uniform(0.2, 2.9, (N, N)), dtype=torch.float32, device="cuda")
    opt = L.CTMOptimizer(cache, target, 0.225, 50.0, iterations=1)
    loss0, g0, _ = opt.evaluate(theta)
    g0 = g0.clone()
    dy, dx = 517, 1234
    opt2 = L.CTMOptimizer(cache, torch.roll(target, (dy, dx), (0, 1)), 0.225, 50.0, iterations=1)
    loss1, g1, _ = opt2.evaluate(torch.roll(theta, (dy, dx), (0, 1)))
    assert abs(loss1 - loss0) <= 1e-5 * loss0
    assert rel_l2(cpu(g1), cpu(torch.roll(g0, (dy, dx), (0, 1)))) <= G_TOL


def test_constant_mask_gives_dc_intensity(L, wl):
    """A constant mask c images to c^2 sum_k w'_k |H_k(0)|^2 everywhere."""
    band, r0, c0, w, wss = wl.synthetic_socs_band()
    cache = L.ImagingCache.from_band(1024, band, r0, c0, w, wss)
    r = L.Imaging(cache).compute(np.full((1024, 1024), 0.7), 0.225, 50.0)
    h0 = band[:, -r0, -c0]
    want = 0.49 * float(np.sum(w * np.abs(h0) ** 2) / wss)
    got = cpu(r.aerial_image)
    assert np.max(np.abs(got - want)) <= 1e-5 * want


def test_fd_gradient_on_gpu(L):
    """check_pe_gradient (tests/test_ctm_optimizer.cpp:61-96) through the GPU path.

    FP32 losses need a larger step than the reference's 1e-3: h = 1e-2, relative
    tolerance 1e-2 (the FD truncation error at h = 1e-2 is far below it).
    """
    n = 64
    oc = oo.prepare(n, 4.0, 193.0, 1.35, 0.6, 0.9, use_socs=True)
    target = np.zeros((n, n)); target[23:42, 23:42] = 1.0
    cache = device_cache(L, oc)
    opt = L.CTMOptimizer(cache, target, 0.25, 85.0, iterations=1)
    theta = torch.tensor(io.initialize_theta(target), dtype=torch.float32, device="cuda")
    _, gt, norm = opt.evaluate(theta)
    d = -gt.clone() / norm
    h = 1e-2
    fp, _, _ = opt.evaluate(theta + h * d)
    fm, _, _ = opt.evaluate(theta - h * d)
    num = (fp - fm) / (2 * h)
    assert abs(num + norm) <= 1e-2 * max(1.0, abs(num))


def test_errors_are_reported(L, wl):
    band, r0, c0, w, wss = wl.synthetic_socs_band(K=4)
    cache = L.ImagingCache.from_band(64, band, r0, c0, w, wss)
    imaging = L.Imaging(cache)
    bad = np.zeros((64, 64)); bad[3, 4] = np.nan
    with pytest.raises(L.LithoError) as e:
        imaging.compute(bad, 0.25, 50.0)
    assert e.value.status == 3
    with pytest.raises(L.LithoError):
        imaging.compute(np.zeros((64, 63)), 0.25, 50.0)
    with pytest.raises(L.LithoError) as e:
        imaging.compute(np.zeros((64, 64)), float("nan"), 50.0)
    grad = L.Gradient(cache, 0.25, 50.0)
    fresh = L.Field(cache)
    with pytest.raises(L.LithoError) as e:
        grad.pe_gradient(np.zeros((64, 64)), np.zeros((64, 64)), fresh)
    assert e.value.status == 6
    with pytest.raises(L.LithoError):
        L.ImagingCache.from_band(64, band, r0, c0, -w, wss)
    with pytest.raises(L.LithoError):
        L.ImagingCache.from_band(64, band, r0, c0, w, 0.0)


def test_repeat_is_bitwise_deterministic(L, wl):
    band, r0, c0, w, wss = wl.synthetic_socs_band()
    cache = L.ImagingCache.from_band(512, band, r0, c0, w, wss)
    target = wl.manhattan_target(512, 8, seed=3)
    opt = L.CTMOptimizer(cache, target, 0.225, 50.0, iterations=1)
    theta = torch.tensor(wl.theta_init_reference(target), dtype=torch.float32, device="cuda")
    l0, g0, n0 = opt.evaluate(theta)
    g0 = g0.clone()
    l1, g1, n1 = opt.evaluate(theta)
    assert l0 == l1 and n0 == n1
    assert torch.equal(g0, g1)


def test_ctm_gd_and_lbfgs_stopping(L):
    """tests/test_ctm_optimizer.cpp:170-196: tol 1e100 stops after one evaluation;
    one L-BFGS iteration with tol 0 lowers PE."""
    n = 64
    oc = oo.prepare(n, 4.0, 193.0, 1.35, 0.6, 0.9, use_socs=True)
    target = np.zeros((n, n)); target[23:42, 23:42] = 1.0
    cache = device_cache(L, oc)
    gd = L.CTMOptimizer(cache, target, 0.25, 85.0, 3, 0.9, "gradient_descent", 10, 1e100)
    m_gd = gd.optimize()
    assert len(gd.error_history) == 1 and torch.isfinite(m_gd).all()
    lb = L.CTMOptimizer(cache, target, 0.25, 85.0, 3, 0.9, "lbfgs", 10, 1e100)
    m_lb = lb.optimize()
    assert len(lb.error_history) == 1
    assert torch.allclose(m_gd, m_lb, atol=1e-6)
    step = L.CTMOptimizer(cache, target, 0.25, 85.0, 1, 0.9, "lbfgs", 10, 0.0)
    m = step.optimize()
    assert len(step.error_history) >= 2
    assert step.error_history[-1] <= step.error_history[0]
    assert torch.isfinite(m).all()
    # GD trajectory vs the oracle's GD for three iterations.
    gd3 = L.CTMOptimizer(cache, target, 0.25, 85.0, 3, 0.9, "gradient_descent", 10, 0.0)
    gd3.optimize()
    _, hist, _ = io.ctm_gradient_descent(target, oc, 0.25, 85.0, 3, 0.9, 0.0)
    for a, b in zip(gd3.error_history, hist):
        assert abs(a - b) <= 1e-4 * b


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_ctm_evaluate_host_buffers(L, wl, precision):
    """litho_ctm_evaluate_host (host buffers, overlapped uploads) equals the device-buffer call."""
    import ctypes
    N = 256
    band, r0, c0, w, wss = wl.synthetic_socs_band()
    ctx = L.Context()
    ctx.set_precision(precision)
    cache = L.ImagingCache.from_band(N, band, r0, c0, w, wss, ctx=ctx)
    rng = np.random.default_rng(5)
    theta = (rng.random((N, N)) * 3.0).astype(np.float32)
    target = (rng.random((N, N)) > 0.5).astype(np.float32)
    opt = L.CTMOptimizer(cache, target, 0.02, 50.0, iterations=1)
    loss_d, g_d, norm_d = opt.evaluate(torch.from_numpy(theta).cuda())
    g_d = g_d.cpu().numpy()
    field = L.Field(cache)
    for _ in range(2):
        h_theta = torch.from_numpy(theta).pin_memory()
        h_target = torch.from_numpy(target).pin_memory()
        h_grad = torch.empty((N, N), dtype=torch.float32).pin_memory()
        loss, norm = ctypes.c_double(), ctypes.c_double()
        ctx._check(ctx.lib.litho_ctm_evaluate_host(
            ctx.handle, cache.handle, field.handle, h_theta.data_ptr(), h_target.data_ptr(),
            0.02, 50.0, h_grad.data_ptr(), ctypes.byref(loss), ctypes.byref(norm)))
        assert loss.value == loss_d and norm.value == norm_d
        assert np.array_equal(h_grad.numpy(), g_d)


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_ctm_evaluate_graph_replay(L, wl, precision):
    """Repeated litho_ctm_evaluate calls on the same buffers are captured once and
    replayed as a CUDA graph: results equal the direct launches, and in-place
    changes of theta are seen by the replay."""
    N = 256
    band, r0, c0, w, wss = wl.synthetic_socs_band()
    stream = torch.cuda.Stream()      # a capturable stream (the legacy default is not)
    ctx = L.Context(stream=stream)
    ctx.set_precision(precision)
    cache = L.ImagingCache.from_band(N, band, r0, c0, w, wss, ctx=ctx)
    rng = np.random.default_rng(11)
    theta0 = (rng.random((N, N)) * 3.0).astype(np.float32)
    theta1 = (rng.random((N, N)) * 3.0).astype(np.float32)
    target = (rng.random((N, N)) > 0.5).astype(np.float32)
    with torch.cuda.stream(stream):
        _graph_replay_steps(L, cache, ctx, theta0, theta1, target)


def _graph_replay_steps(L, cache, ctx, theta0, theta1, target):
    fresh = L.CTMOptimizer(cache, target, 0.02, 50.0, iterations=1)
    ref0 = fresh.evaluate(torch.from_numpy(theta0).cuda())
    ref0 = (ref0[0], ref0[1].cpu().numpy(), ref0[2])
    fresh2 = L.CTMOptimizer(cache, target, 0.02, 50.0, iterations=1)
    ref1 = fresh2.evaluate(torch.from_numpy(theta1).cuda())
    ref1 = (ref1[0], ref1[1].cpu().numpy(), ref1[2])
    opt = L.CTMOptimizer(cache, target, 0.02, 50.0, iterations=1)
    th = torch.from_numpy(theta0).cuda()
    counts = []
    for i in range(5):
        if i == 3:
            th.copy_(torch.from_numpy(theta1))   # same buffer, new content
        c0 = ctx.launch_count
        loss, g, norm = opt.evaluate(th)
        counts.append(ctx.launch_count - c0)
        ref = ref1 if i >= 3 else ref0
        assert loss == ref[0] and norm == ref[2]
        assert np.array_equal(g.cpu().numpy(), ref[1])
    assert len(set(counts)) == 1   # replays count the kernels they launch


def _edge_points(target, rng, n_extra=20):
    """Points on the target's 0.5 contour (midpoints between unequal neighbours) plus a
    few random interior points; weights in [0, 1] with some inactive (0) points."""
    pts = []
    ys, xs = np.nonzero(target[:, 1:] != target[:, :-1])
    pts += [(y + rng.uniform(-0.3, 0.3), x + 0.5) for y, x in zip(ys, xs)]
    ys, xs = np.nonzero(target[1:, :] != target[:-1, :])
    pts += [(y + 0.5, x + rng.uniform(-0.3, 0.3)) for y, x in zip(ys, xs)]
    n = target.shape[0]
    pts += [(rng.uniform(-1, n), rng.uniform(-1, n)) for _ in range(n_extra)]   # clamped too
    eps = np.array(pts, dtype=np.float64)
    w = rng.uniform(0.2, 1.0, len(eps))
    w[rng.random(len(eps)) < 0.1] = 0.0
    return eps, w


def test_sparse_epe_and_gradient_match_oracle(L, wl):
    """Loss::evaluate_sparse_epe and Gradient::epe_gradient (loss.cpp:125-163,
    gradient.cpp:198-227) on real optics at 64 x 64 against the FP64 oracle, the same
    FP32 aerial image fed to both. Tolerances: signed EPE and totals 1e-9 relative
    (both FP64 on the same input); gradient relative L2 1e-4."""
    oc = oo.prepare(64, 4.0, 193.0, 1.35, 0.6, 0.9, use_socs=True)
    cache = device_cache(L, oc)
    rng = np.random.default_rng(21)
    target = np.zeros((64, 64))
    target[14:40, 20:34] = 1.0
    target[44:52, 10:50] = 1.0
    mask = io.theta_to_mask(io.initialize_theta(target) + 0.2 * rng.standard_normal((64, 64)))
    imaging = L.Imaging(cache)
    r = imaging.compute(mask, 0.1, 50.0)
    aerial = r.aerial_image
    a64 = cpu(aerial)
    eps, w = _edge_points(target, rng)
    ev = L.Loss.evaluate_sparse_epe(aerial, eps, w, 0.1, 4.0)
    ref = io.evaluate_sparse_epe(a64, eps, w, 0.1, 4.0)
    assert np.array_equal(np.isnan(ev.signed_epe_pixel), np.isnan(ref["signed_epe_pixel"]))
    ok = ~np.isnan(ref["signed_epe_pixel"])
    assert np.allclose(ev.signed_epe_pixel[ok], ref["signed_epe_pixel"][ok], rtol=1e-9, atol=1e-12)
    assert abs(ev.weighted_squared_loss - ref["weighted_squared_loss"]) <= 1e-9 * ref["weighted_squared_loss"]
    assert abs(ev.absolute_sum_nm - ref["absolute_sum_nm"]) <= 1e-9 * ref["absolute_sum_nm"]
    assert ev.active_count == ref["active_count"]
    _, _, fields = io.imaging_compute(mask, oc, 0.1, 50.0, keep_fields=True)
    g = L.Gradient(cache, 0.1, 50.0).epe_gradient(aerial, imaging.get_electric_field(), eps, w, 0.1)
    gref = io.epe_gradient(a64, fields, oc, eps, w, 0.1)
    assert rel_l2(cpu(g), gref) < 1e-4


def test_epe_gradient_is_bitwise_repeatable(L, wl):
    """The EPE dL/dI scatter (Gradient::epe_gradient, gradient.cpp:198-227) sums each
    pixel's contributions in EP order after a stable sort, so repeated calls give the
    same gradient bit for bit, with many EPs sharing pixels (the reference's serial loop
    is deterministic too, demo/demo_CTM_parallel_benchmark.cpp:193-196)."""
    oc = oo.prepare(64, 4.0, 193.0, 1.35, 0.6, 0.9, use_socs=True)
    cache = device_cache(L, oc)
    rng = np.random.default_rng(4)
    target = np.zeros((64, 64))
    target[14:40, 20:34] = 1.0
    mask = io.theta_to_mask(io.initialize_theta(target) + 0.2 * rng.standard_normal((64, 64)))
    imaging = L.Imaging(cache)
    r = imaging.compute(mask, 0.1, 50.0)
    eps, w = _edge_points(target, rng, n_extra=200)
    eps = np.concatenate([eps, eps[::3] + rng.uniform(-0.2, 0.2, eps[::3].shape)])  # shared pixels
    w = np.concatenate([w, rng.uniform(0.2, 1.0, len(eps) - len(w))])
    grad = L.Gradient(cache, 0.1, 50.0)
    g0 = grad.epe_gradient(r.aerial_image, imaging.get_electric_field(), eps, w, 0.1).clone()
    for _ in range(3):
        g1 = grad.epe_gradient(r.aerial_image, imaging.get_electric_field(), eps, w, 0.1)
        assert torch.equal(g0, g1)
    _, _, fields = io.imaging_compute(mask, oc, 0.1, 50.0, keep_fields=True)
    gref = io.epe_gradient(cpu(r.aerial_image), fields, oc, eps, w, 0.1)
    assert rel_l2(cpu(g0), gref) < 1e-4
