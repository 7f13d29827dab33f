"""Batched level-set gradients and the continuous-batching tile server on the GPU.

* litho_pe_gradient_batch: every image equals its own batch-of-one evaluation bit for
  bit, and matches the single-image Imaging + Gradient.pe_gradient path within the
  split-BF16 tolerance (gradient relative L2 <= 1e-3, PE relative 1e-4); the FP32
  mode (one image after another) matches it within the FP32 tolerance (1e-4, 1e-5).
* litho_lsm_rk2_update_batch: every image equals its own litho_lsm_rk2_update.
* TileServer (device-resident, no host round trip per step): a solve's results are the
  same alone and in a mix of other solves of other sizes that arrive while it runs (bit
  for bit); its loss history follows LSMOptimizer; a non-finite input is reported;
  slot and HBM-budget admission; a seeded Poisson stream reports latency percentiles.
"""
import importlib

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

THR, ALPHA = 0.225, 50.0


@pytest.fixture(scope="module")
def L():
    p = importlib.import_module("c-version-lithography_b200")
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    p.load_library()
    return p


@pytest.fixture(scope="module")
def S():
    return importlib.import_module("c-version-lithography_b200.serving")


@pytest.fixture(scope="module")
def wl():
    return importlib.import_module("c-version-lithography_b200.workloads")


def rel_l2(a, b):
    a = a.double().cpu(); b = b.double().cpu()
    return float((a - b).norm() / b.norm())


def tile(wl, N, seed):
    t = wl.manhattan_target(N, max(3, N // 40), seed=seed)
    return (torch.tensor(t, dtype=torch.float32, device="cuda"),
            torch.tensor(t, dtype=torch.float32, device="cuda"))


@pytest.fixture(scope="module")
def setup(L, wl):
    ctx = L.Context()
    ctx.set_precision("bf16x3")
    band, r0, c0, w, wss = wl.synthetic_socs_band()
    caches = {N: L.ImagingCache.from_band(N, band, r0, c0, w, wss, ctx=ctx) for N in (128, 256)}
    yield ctx, caches, (band, r0, c0, w, wss)
    ctx.close()


def test_pe_gradient_batch(L, wl, setup):
    ctx, caches, _ = setup
    cache = caches[256]
    rng = np.random.default_rng(1)
    tg = torch.stack([tile(wl, 256, s)[0] for s in range(5)])
    m = torch.tensor((rng.random((5, 256, 256)) > 0.5), dtype=torch.float32, device="cuda")
    m[0] = tg[0]
    losses, grads = L.pe_gradient_batch(cache, m, tg, THR, ALPHA)
    imaging, grad = L.Imaging(cache), L.Gradient(cache, THR, ALPHA)
    for b in range(5):
        one, g1 = L.pe_gradient_batch(cache, m[b:b + 1], tg[b:b + 1], THR, ALPHA)
        assert one[0] == losses[b] and torch.equal(g1[0], grads[b]), b
        r = imaging.compute(m[b], THR, ALPHA)
        ref = grad.pe_gradient(r.wafer_image, tg[b], imaging.get_electric_field())
        pe = L.Loss.pe_loss(r.wafer_image, tg[b], ctx=ctx)
        assert rel_l2(grads[b], ref) <= 1e-3, b
        assert abs(losses[b] - pe) <= 1e-4 * pe, b
    # FP32 parity mode: the images one after another through the FP32 chain
    c32 = L.Context()
    band, r0, c0, w, wss = setup[2]
    cache32 = L.ImagingCache.from_band(256, band, r0, c0, w, wss, ctx=c32)
    l32, g32 = L.pe_gradient_batch(cache32, m[:2], tg[:2], THR, ALPHA)
    im32, gr32 = L.Imaging(cache32), L.Gradient(cache32, THR, ALPHA)
    for b in range(2):
        r = im32.compute(m[b], THR, ALPHA)
        ref = gr32.pe_gradient(r.wafer_image, tg[b], im32.get_electric_field())
        assert rel_l2(g32[b], ref) <= 1e-4
        assert abs(l32[b] - L.Loss.pe_loss(r.wafer_image, tg[b], ctx=c32)) <= 1e-5 * l32[b]
    bad = m[:1].clone()
    bad[0, 5, 5] = float("nan")
    with pytest.raises(L.LithoError) as e:
        L.pe_gradient_batch(cache, bad, tg[:1], THR, ALPHA)
    assert e.value.status == 3
    c32.close()


def _run_alone(S, caches, tgt, m, its):
    srv = S.TileServer(caches, THR, ALPHA, reinit_interval=4)
    s = srv.submit(tgt, m, its)
    srv.drain()
    return s


def test_server_same_alone_and_in_the_mix(L, S, wl, setup):
    """Continuous batching: solves of two sizes arrive while others run; each
    solve's losses, best mask, final phi and mask equal its solo run bit for bit."""
    ctx, caches, _ = setup
    reqs = [(256, 1, 9), (128, 2, 6), (256, 3, 7), (128, 4, 11), (256, 5, 3)]
    tiles = {sd: tile(wl, N, sd) for N, sd, _ in reqs}
    srv = S.TileServer(caches, THR, ALPHA, reinit_interval=4, max_batch=3)
    mixed = {}
    # two at once, the rest arriving one per step while the first ones run
    for N, sd, its in reqs[:2]:
        mixed[sd] = srv.submit(*tiles[sd], its)
    for N, sd, its in reqs[2:]:
        srv.step()
        mixed[sd] = srv.submit(*tiles[sd], its)
    srv.drain()
    assert srv.active == 0 and not srv.queue and len(srv.finished) == len(reqs)
    for N, sd, its in reqs:
        a = _run_alone(S, caches, *tiles[sd], its)
        b = mixed[sd]
        assert b.done_iterations == its and len(b.losses) == its
        assert a.losses == b.losses, sd
        assert torch.equal(a.phi, b.phi) and torch.equal(a.mask, b.mask), sd
        assert torch.equal(a.best_mask, b.best_mask) and a.best_loss == b.best_loss, sd


def test_server_first_iteration_matches_lsm_step(L, S, wl, setup):
    """The server's first iteration is LSM_Optimizer's: the tracked loss PE + 1.0 x the
    background-penalty term at 0.01 of the initial mask (LSM_Optimizer.cpp:87-90) and
    one RK2 update with dPE/dM as the speed (single-image path, same tolerance as the
    batched gradient)."""
    ctx, caches, _ = setup
    cache = caches[128]
    tgt, m = tile(wl, 128, 9)
    s = _run_alone(S, caches, tgt, m, 1)
    r = L.Imaging(cache).compute(m, THR, ALPHA)
    pe = L.Loss.pe_loss_with_penalty(r.wafer_image, tgt, 1.0, 0.01, ctx=ctx)
    assert abs(s.losses[0] - pe) <= 1e-4 * pe and s.best_loss == s.losses[0]
    phi0 = L.LevelSetUtils.reinit_sdf(m - 0.5, 1.0, 1.0, ctx=ctx)
    imaging = L.Imaging(cache)
    r = imaging.compute(m, THR, ALPHA)
    gm = L.Gradient(cache, THR, ALPHA).pe_gradient(r.wafer_image, tgt, imaging.get_electric_field())
    phi1, _, _ = L.LevelSetUtils.rk2_update(phi0, gm, 1.0, 1.0, 0.5, 0.01, ctx=ctx)
    assert rel_l2(s.phi, phi1) <= 1e-4


def test_server_slots_and_budget(L, S, wl, setup):
    ctx, caches, _ = setup
    one = S.TileServer.solve_bytes(256)
    srv = S.TileServer(caches, THR, ALPHA, max_batch=4, hbm_budget=2.5 * one)
    solves = [srv.submit(*tile(wl, 256, 20 + i), 3) for i in range(4)]
    srv.step()
    assert srv.active == 2 and len(srv.queue) == 2     # the budget holds two solves
    srv.drain()
    assert all(s.done_iterations == 3 for s in solves)
    assert [s.id for s in sorted(solves, key=lambda s: s.t_admit)] == [0, 1, 2, 3]
    assert srv.held == pytest.approx(0.0, abs=1.0)
    srv = S.TileServer(caches, THR, ALPHA, max_batch=2)
    for i in range(3):
        srv.submit(*tile(wl, 128, 30 + i), 2)
    srv.step()
    assert srv.active == 2 and len(srv.queue) == 1     # two slots per size
    srv.drain()
    with pytest.raises(L.LithoError):
        srv.submit(torch.zeros((64, 64), device="cuda"), torch.zeros((64, 64), device="cuda"), 2)


def test_server_matches_lsm_optimizer(L, S, wl, setup):
    """A solve of 25 iterations (a re-initialisation after iteration 20) against
    LSMOptimizer (the single-image LSM_Optimizer loop) on the same cache: the loss
    history within the split-BF16 tolerance (1e-4 relative per iteration)."""
    ctx, caches, _ = setup
    cache = caches[128]
    tgt, m = tile(wl, 128, 12)
    srv = S.TileServer(caches, THR, ALPHA, reinit_interval=20)
    s = srv.submit(tgt, m, 25)
    srv.drain()
    lsm = L.LSMOptimizer(cache, tgt, THR, ALPHA, 1.0, 1.0, cfl=0.5, b=0.01, iterations=25)
    lsm.optimize(m)
    assert len(s.losses) == 25
    for a, b in zip(s.losses, lsm.error_history):
        assert abs(a - b) <= 1e-4 * b
    assert s.best_loss == min(s.losses)


def test_server_reports_a_nonfinite_target(L, S, wl, setup):
    ctx, caches, _ = setup
    tgt, m = tile(wl, 128, 13)
    bad = tgt.clone()
    bad[3, 3] = float("nan")
    srv = S.TileServer(caches, THR, ALPHA)
    srv.submit(bad, m, 2)
    with pytest.raises(L.LithoError) as e:
        srv.drain()
    assert e.value.status == 3


def test_server_poisson_stream(L, S, wl, setup):
    ctx, caches, _ = setup

    def make(N, rng):
        t = wl.manhattan_target(N, max(3, N // 40), seed=int(rng.integers(1 << 30)))
        return t, t

    arr = S.poisson_arrivals(400.0, 12, [128, 256], [2, 1], make, iterations=4, seed=3)
    srv = S.TileServer(caches, THR, ALPHA, max_batch=8)
    st = srv.serve(arr)
    assert st["requests"] == 12 and st["completed"] == 12
    assert st["latency_p99_s"] >= st["latency_p50_s"] > 0.0
    assert st["tile_iterations_per_s"] > 0.0


def test_rk2_update_batch_equals_single(L, wl, setup):
    """litho_lsm_rk2_update_batch: each image's phi, mask and dt equal those of
    litho_lsm_rk2_update on that image alone (same kernels, one host round trip)."""
    ctx, _, _ = setup
    rng = np.random.default_rng(4)
    B, n = 3, 96
    m = torch.tensor(rng.random((B, n, n)) > 0.5, dtype=torch.float32, device="cuda")
    phi = torch.stack([L.LevelSetUtils.reinit_sdf(m[b] - 0.5, 1.0, 1.0, ctx=ctx) for b in range(B)])
    vn = torch.tensor(rng.standard_normal((B, n, n)) * (1.0 + np.arange(B))[:, None, None],
                      dtype=torch.float32, device="cuda")
    out, mask = torch.empty_like(phi), torch.empty_like(phi)
    dts = L.LevelSetUtils.rk2_update_batch(phi, vn, 1.0, 1.0, 0.5, 0.01, out, mask, ctx=ctx)
    for b in range(B):
        p1, m1, dt = L.LevelSetUtils.rk2_update(phi[b], vn[b], 1.0, 1.0, 0.5, 0.01, ctx=ctx)
        assert dts[b] == dt and torch.equal(out[b], p1) and torch.equal(mask[b], m1), b
    assert len(set(dts)) == B      # each image its own CFL step
    with pytest.raises(L.LithoError):
        L.LevelSetUtils.rk2_update_batch(phi, vn, 1.0, 1.0, 0.5, 0.01, phi, mask, ctx=ctx)
