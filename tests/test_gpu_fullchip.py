"""GPU parity of the full-chip micro-tile path (Partition, MicroGradientExchange,
FullChipCTMOptimizer) against the FP64 full-chip oracle, through the C ABI.

Tolerances (FP32 path): tile copies bit-exact; raw and exchanged gradients
relative L2 <= 1e-4 per tile; data and CEPT losses relative 1e-5; full-chip CTM
loss history relative 1e-5 at the start and 1e-3 after three fixed steps, best
global mask max|d| <= 1e-3. Optics: the 193 nm / NA 1.35 annular SOCS cache
(36 kernels) on 128 x 128 tiles of 4 nm pixels.
"""
import importlib

import numpy as np
import pytest

from oracle import fullchip_oracle as fc
from oracle import imaging_oracle as io
from oracle import optics_oracle as oo

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

THR, ALPHA = 0.1, 50.0


@pytest.fixture(scope="module")
def L():
    p = importlib.import_module("c-version-lithography_b200")
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    p.load_library()
    return p


@pytest.fixture(scope="module")
def FC():
    return importlib.import_module("c-version-lithography_b200.fullchip")


@pytest.fixture(scope="module")
def band128():
    return oo.prepare(128, 4.0, 193.0, 1.35, 0.6, 0.9, use_socs=True), None


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64); b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def cpu(t):
    return t.detach().cpu().numpy().astype(np.float64)


def rect(r):
    return (r.y0, r.y1, r.x0, r.x1)


@pytest.mark.parametrize("cfg", [(24, 24, 2, 2, 4, 2), (25, 31, 2, 3, 3, 1), (280, 190, 3, 2, 16, 6),
                                 (40, 40, 1, 1, 0, 0)])
def test_partition_matches_oracle(L, FC, cfg):
    meta = fc.build(*cfg)
    part = FC.Partition(*cfg)
    assert part.tile_size == meta.tile_size and part.num_tiles == len(meta.tiles)
    for a, b in zip(part.tiles, meta.tiles):
        assert (a.row, a.col) == (b.row, b.col)
        assert rect(a.core_global) == rect(b.core_global)
        assert rect(a.tile_global) == rect(b.tile_global)
        assert rect(a.core_local) == rect(b.core_local)
        assert rect(a.update_local) == rect(b.update_local)
    g = np.random.default_rng(3).random((cfg[0], cfg[1])).astype(np.float32)
    tiles = part.extract_all(torch.from_numpy(g).cuda())
    ref = [fc.extract_local_tile(g, t) for t in meta.tiles]
    assert np.array_equal(tiles.cpu().numpy(), np.stack(ref))
    back = part.assemble_global(tiles).cpu().numpy()
    assert np.array_equal(back, g)


UNEVEN = [
    # (height, width, row_cuts, col_cuts, halo, guard)
    (300, 260, [0, 40, 96, 150, 200, 300], [0, 33, 100, 181, 260], 14, 6),
    (97, 120, [0, 12, 97], [0, 50, 51, 120], 5, 1),
]


@pytest.mark.parametrize("cfg", UNEVEN)
def test_partition_cuts_matches_oracle(L, FC, cfg):
    """litho_partition_create_cuts: uneven Cores, one tile size = largest Core + 2 halo
    (even), geometry and neighbour relations as the oracle's Partition::build over the
    same cuts; tile copies and the Core stitch are exact."""
    H, W, rc, cc, halo, guard = cfg
    meta = fc.build(H, W, len(rc) - 1, len(cc) - 1, halo, guard, row_cuts=rc, col_cuts=cc)
    part = FC.Partition(H, W, len(rc) - 1, len(cc) - 1, halo, guard, row_cuts=rc, col_cuts=cc)
    assert part.tile_size == meta.tile_size and part.num_tiles == len(meta.tiles)
    for a, b in zip(part.tiles, meta.tiles):
        assert (a.row, a.col) == (b.row, b.col)
        assert rect(a.core_global) == rect(b.core_global)
        assert rect(a.tile_global) == rect(b.tile_global)
        assert rect(a.core_local) == rect(b.core_local)
        assert rect(a.update_local) == rect(b.update_local)
    g = np.random.default_rng(4).random((H, W)).astype(np.float32)
    tiles = part.extract_all(torch.from_numpy(g).cuda())
    assert np.array_equal(tiles.cpu().numpy(), np.stack([fc.extract_local_tile(g, t)
                                                          for t in meta.tiles]))
    assert np.array_equal(part.assemble_global(tiles).cpu().numpy(), g)
    # equal cuts give the default partition
    eq = FC.Partition(H, W, 2, 3, halo, guard, row_cuts=[0, H // 2, H],
                      col_cuts=[0, W // 3, 2 * W // 3, W])
    ref = FC.Partition(H, W, 2, 3, halo, guard)
    assert [rect(t.tile_global) for t in eq.tiles] == [rect(t.tile_global) for t in ref.tiles]
    with pytest.raises(L.LithoError):
        FC.Partition(H, W, 2, 1, halo, guard, row_cuts=[1, 40, H], col_cuts=[0, W])
    with pytest.raises(L.LithoError):   # a Core narrower than the guard
        FC.Partition(H, W, 2, 1, halo, 6, row_cuts=[0, 3, H], col_cuts=[0, W])


@pytest.mark.parametrize("prec", ["fp32", "bf16x3"])
def test_uneven_layout_exchange_and_lsm_match_oracle(L, FC, band128, prec):
    """Micro tiles over uneven Cores (33-100 px, 20 tiles of 128^2): the exchange and
    three full-chip LSM steps against the FP64 oracle over the same cuts, the stitched
    Core mask included. Tolerances as the even-layout tests of each precision; the
    split-BF16 exchange runs all 20 tiles in one batched pass and in passes of at most 8
    tiles, with the same results bit for bit."""
    oc, _ = band128
    H, W, rc, cc, halo, guard = UNEVEN[0]
    meta = fc.build(H, W, len(rc) - 1, len(cc) - 1, halo, guard, row_cuts=rc, col_cuts=cc)
    assert meta.tile_size == oc.N
    ctx = L.Context()
    ctx.set_precision(prec)
    part = FC.Partition(H, W, len(rc) - 1, len(cc) - 1, halo, guard, ctx=ctx, row_cuts=rc,
                        col_cuts=cc)
    cache = L.ImagingCache.from_kernels(np.stack(oc.kernels), oc.source_ws, oc.eigenvalues, ctx=ctx)
    target = make_target(H, W, 71)
    rng = np.random.default_rng(72)
    theta_g = io.initialize_theta(target) + 0.3 * rng.standard_normal(target.shape)
    masks32 = [io.theta_to_mask(fc.extract_local_tile(theta_g, t)
                                + 0.05 * rng.standard_normal((meta.tile_size,) * 2)).astype(np.float32)
               for t in meta.tiles]
    opts = OPTION_SETS[1]
    ev = fc.exchange([m.astype(np.float64) for m in masks32], target, meta, oc, THR, ALPHA,
                     fc.ExchangeOptions(**opts))
    ex = FC.MicroGradientExchange(part, cache, THR, ALPHA)
    gpu_masks = torch.from_numpy(np.stack(masks32)).cuda()
    gpu_target = torch.from_numpy(target.astype(np.float32)).cuda()
    res = ex.compute(gpu_masks, gpu_target, FC.MicroGradientOptions(**opts))
    tol = 1e-4 if prec == "fp32" else 1e-3
    raw, grad = cpu(res.raw_gradients), cpu(res.mask_gradients)
    for t in meta.tiles:
        o = ev["locals"][t.id]
        assert rel_l2(raw[t.id], o["raw"]) < tol, t.id
        assert rel_l2(grad[t.id], o["grad"]) < tol, t.id
    assert abs(res.loss - ev["loss"]) <= 10 * tol * ev["loss"]
    if prec == "bf16x3":
        ctx.set_exchange_group(8)
        res8 = ex.compute(gpu_masks, gpu_target, FC.MicroGradientOptions(**opts))
        assert np.array_equal(cpu(res8.mask_gradients), grad) and res8.loss == res.loss
        ctx.set_exchange_group(0)
    lopts = dict(enable_cept=True, enable_grad_fusion=True)
    kw = dict(dx=1.0, dy=1.0, cfl=0.7, b=0.01, reinit_interval=2, mask_type="Binary",
              render_scale=4)
    ref = fc.full_chip_lsm(target, target, meta, oc, THR, ALPHA, fc.ExchangeOptions(**lopts), 3,
                           **kw)
    optz = FC.FullChipLSMOptimizer(part, cache, THR, ALPHA)
    out = optz.optimize(gpu_target, gpu_target,
                        FC.FullChipLSMOptions(iterations=3, cfl=0.7, curvature_weight=0.01,
                                              reinit_interval=2, mask_type="Binary",
                                              render_scale=4,
                                              gradient_options=FC.MicroGradientOptions(**lopts)))
    for a, b in zip(out.history, ref["history"]):
        assert abs(a.loss - b["loss"]) <= 1e-3 * b["loss"]
    assert out.best_iteration == ref["best"]["iteration"]
    gm = cpu(out.global_mask)
    assert gm.shape == (H, W)
    assert (np.abs(gm - ref["global_mask"]) > 1e-6).mean() <= 0.005
    part.close()
    ctx.close()


def make_target(H, W, seed):
    rng = np.random.default_rng(seed)
    t = np.zeros((H, W))
    for _ in range(10):
        y, x = rng.integers(0, H - 20), rng.integers(0, W - 20)
        t[y:y + rng.integers(6, 20), x:x + rng.integers(6, 20)] = 1.0
    return t


OPTION_SETS = [
    dict(),
    dict(loss_type="PEPenalty", loss_region="CoreGuard", pe_weight=0.7, penalty_weight=2.0,
         enable_cept=True, cept_guard_only=False, cept_weight=1.1, enable_grad_fusion=True,
         fusion_mode="Linear", fusion_weight_owner=0.5, fusion_weight_neighbor=0.5),
    dict(enable_cept=True, cept_guard_only=True, enable_grad_fusion=True, fusion_mode="Average",
         fusion_weight_owner=0.25, fusion_weight_neighbor=0.75),
]


@pytest.mark.parametrize("oi", range(len(OPTION_SETS)))
def test_exchange_matches_oracle(L, FC, band128, oi):
    oc, _ = band128
    cfg = (280, 190, 3, 2, 16, 6)
    meta = fc.build(*cfg)
    assert meta.tile_size == oc.N
    part = FC.Partition(*cfg)
    cache = L.ImagingCache.from_kernels(np.stack(oc.kernels), oc.source_ws, oc.eigenvalues)
    target = make_target(cfg[0], cfg[1], oi)
    rng = np.random.default_rng(10 + oi)
    theta_g = io.initialize_theta(target) + 0.3 * rng.standard_normal(target.shape)
    # independent per-tile perturbations, so guards and neighbour Cores disagree
    masks32 = [io.theta_to_mask(fc.extract_local_tile(theta_g, t)
                                + 0.05 * rng.standard_normal((meta.tile_size,) * 2)).astype(np.float32)
               for t in meta.tiles]
    masks = [m.astype(np.float64) for m in masks32]
    opts = OPTION_SETS[oi]
    ev = fc.exchange(masks, target, meta, oc, THR, ALPHA, fc.ExchangeOptions(**opts))
    ex = FC.MicroGradientExchange(part, cache, THR, ALPHA)
    res = ex.compute(torch.from_numpy(np.stack(masks32)).cuda(),
                     torch.from_numpy(target.astype(np.float32)).cuda(),
                     FC.MicroGradientOptions(**opts))
    raw, grad = cpu(res.raw_gradients), cpu(res.mask_gradients)
    for t in meta.tiles:
        o = ev["locals"][t.id]
        assert rel_l2(raw[t.id], o["raw"]) < 1e-4, t.id
        assert rel_l2(grad[t.id], o["grad"]) < 1e-4, t.id
        g = res.locals[t.id]
        assert abs(g.pe_loss - o["pe_loss"]) <= 1e-5 * max(o["pe_loss"], 1e-12)
        assert abs(g.bg_penalty_raw - o["bg_penalty_raw"]) <= 1e-5 * max(o["bg_penalty_raw"], 1e-9)
        assert abs(g.cept_loss - o["cept_loss"]) <= 1e-6 * max(o["cept_loss"], 1e-9)
    assert abs(res.loss - ev["loss"]) <= 1e-5 * ev["loss"]
    assert abs(res.data_loss - ev["data_loss"]) <= 1e-5 * ev["data_loss"]
    assert abs(res.cept_loss - ev["cept_loss"]) <= 1e-5 * max(ev["cept_loss"], 1e-9)
    if opts.get("enable_cept"):
        assert res.cept_loss > 0.0


@pytest.mark.parametrize("oi", range(len(OPTION_SETS)))
def test_exchange_bf16x3_batched_matches_oracle(L, FC, band128, oi):
    """Split-BF16 mode: the exchange images the tiles in batched passes (20 tiles here:
    one pass of all of them, or, for the even option sets, passes of at most 16 tiles,
    the second partial). Raw and exchanged gradients within the split-BF16 tolerance
    (relative L2 <= 1e-3 per tile), PE and penalty sums relative 1e-4, CEPT (mask-only)
    relative 1e-6."""
    oc, _ = band128
    cfg = (480, 384, 5, 4, 16, 6)
    meta = fc.build(*cfg)
    assert meta.tile_size == oc.N and len(meta.tiles) == 20
    ctx = L.Context()
    ctx.set_precision("bf16x3")
    ctx.set_exchange_group(16 if oi % 2 == 0 else 0)
    part = FC.Partition(*cfg, ctx=ctx)
    cache = L.ImagingCache.from_kernels(np.stack(oc.kernels), oc.source_ws, oc.eigenvalues, ctx=ctx)
    target = make_target(cfg[0], cfg[1], 40 + oi)
    rng = np.random.default_rng(20 + oi)
    theta_g = io.initialize_theta(target) + 0.3 * rng.standard_normal(target.shape)
    masks32 = [io.theta_to_mask(fc.extract_local_tile(theta_g, t)
                                + 0.05 * rng.standard_normal((meta.tile_size,) * 2)).astype(np.float32)
               for t in meta.tiles]
    opts = OPTION_SETS[oi]
    ev = fc.exchange([m.astype(np.float64) for m in masks32], target, meta, oc, THR, ALPHA,
                     fc.ExchangeOptions(**opts))
    ex = FC.MicroGradientExchange(part, cache, THR, ALPHA)
    res = ex.compute(torch.from_numpy(np.stack(masks32)).cuda(),
                     torch.from_numpy(target.astype(np.float32)).cuda(),
                     FC.MicroGradientOptions(**opts))
    raw, grad = cpu(res.raw_gradients), cpu(res.mask_gradients)
    for t in meta.tiles:
        o = ev["locals"][t.id]
        assert rel_l2(raw[t.id], o["raw"]) < 1e-3, t.id
        assert rel_l2(grad[t.id], o["grad"]) < 1e-3, t.id
        g = res.locals[t.id]
        assert abs(g.pe_loss - o["pe_loss"]) <= 1e-4 * max(o["pe_loss"], 1e-12), t.id
        assert abs(g.bg_penalty_raw - o["bg_penalty_raw"]) <= 1e-4 * max(o["bg_penalty_raw"], 1e-9)
        assert abs(g.cept_loss - o["cept_loss"]) <= 1e-6 * max(o["cept_loss"], 1e-9)
    assert abs(res.loss - ev["loss"]) <= 1e-4 * ev["loss"]
    # repeatable: the same call again gives the same bits
    res2 = ex.compute(torch.from_numpy(np.stack(masks32)).cuda(),
                      torch.from_numpy(target.astype(np.float32)).cuda(),
                      FC.MicroGradientOptions(**opts))
    assert np.array_equal(cpu(res2.mask_gradients), grad) and res2.loss == res.loss
    part.close()
    ctx.close()


def test_fullchip_ctm_matches_oracle(L, FC, band128):
    oc, _ = band128
    cfg = (192, 192, 2, 2, 16, 6)
    meta = fc.build(*cfg)
    part = FC.Partition(*cfg)
    cache = L.ImagingCache.from_kernels(np.stack(oc.kernels), oc.source_ws, oc.eigenvalues)
    target = make_target(192, 192, 7)
    opts = dict(enable_cept=True, enable_grad_fusion=True)
    ref = fc.full_chip_ctm(target, target, meta, oc, THR, ALPHA, fc.ExchangeOptions(**opts), 3, 0.9)
    optz = FC.FullChipCTMOptimizer(part, cache, THR, ALPHA)
    res = optz.optimize(torch.from_numpy(target.astype(np.float32)).cuda(),
                        FC.FullChipCTMOptions(iterations=3, learning_rate=0.9,
                                              gradient_options=FC.MicroGradientOptions(**opts)))
    hist = [h.loss for h in res.history]
    assert len(hist) == 4
    assert abs(hist[0] - ref["history"][0]) <= 1e-5 * ref["history"][0]
    for a, b in zip(hist, ref["history"]):
        assert abs(a - b) <= 1e-3 * b
    assert res.best_iteration == ref["best"]["iteration"]
    assert np.max(np.abs(cpu(res.global_mask) - ref["global_mask"])) < 1e-3
    # theta outside each tile's update window keeps its initial value
    init = part.extract_all(optz.initialize_theta(torch.from_numpy(target.astype(np.float32)).cuda(),
                                                  torch))
    th, th0 = cpu(res.local_theta), cpu(init)
    for t in part.tiles:
        w = t.update_local
        out = np.ones((part.tile_size, part.tile_size), bool)
        out[w.y0:w.y1, w.x0:w.x1] = False
        assert np.array_equal(th[t.id][out], th0[t.id][out])


def test_fullchip_errors(L, FC, band128):
    oc, _ = band128
    with pytest.raises(L.LithoError) as e:
        FC.Partition(24, 24, 2, 2, 2, 4)          # guard > halo
    assert e.value.status == 1
    with pytest.raises(L.LithoError):
        FC.Partition(4, 24, 5, 2, 2, 1)           # more grid rows than layout rows
    part = FC.Partition(24, 24, 2, 2, 4, 2)       # tile 20 != cache 128
    cache = L.ImagingCache.from_kernels(np.stack(oc.kernels), oc.source_ws, oc.eigenvalues)
    with pytest.raises(L.LithoError) as e:
        FC.MicroGradientExchange(part, cache)
    assert e.value.status == 2
    cfg = (192, 192, 2, 2, 16, 6)
    part = FC.Partition(*cfg)
    ex = FC.MicroGradientExchange(part, cache, THR, ALPHA)
    masks = torch.full((4, 128, 128), 0.5, device="cuda")
    tgt = torch.zeros((192, 192), device="cuda")
    with pytest.raises(L.LithoError) as e:
        ex.compute(masks, tgt, FC.MicroGradientOptions(enable_grad_fusion=True,
                                                       fusion_weight_owner=-1.0))
    assert e.value.status == 1
    with pytest.raises(L.LithoError) as e:
        ex.compute(masks, tgt, FC.MicroGradientOptions(loss_type="Contour"))
    assert e.value.status == 7
    with pytest.raises(L.LithoError) as e:
        ex.compute(masks, tgt, FC.MicroGradientOptions(loss_type="EPE"),
                   eps=np.array([[1.0, float("nan")]]))
    assert e.value.status == 3
    with pytest.raises(L.LithoError) as e:
        ex.compute(masks, tgt, FC.MicroGradientOptions(loss_type="PE_EPE",
                                                       main_region_dilation_pixels=-1))
    assert e.value.status == 1
    masks[1, 5, 7] = float("nan")
    with pytest.raises(L.LithoError) as e:
        ex.compute(masks, tgt)
    assert e.value.status == 3


@pytest.mark.parametrize("mask_type", ["Binary", "Gray"])
def test_fullchip_lsm_matches_oracle(L, FC, band128, mask_type):
    """FullChipLSMOptimizer (full_chip_lsm.cpp:38-254) against the FP64 oracle: three steps
    with a reinitialisation after the second, guard-only CEPT and fusion on. FP32 phi
    differs from FP64 by ~1e-5, so a rendered pixel whose phi is within that of 0 may
    flip: the loss history is compared to 1e-3 and the best masks to 0.5 % of pixels."""
    oc, _ = band128
    cfg = (192, 192, 2, 2, 16, 6)
    meta = fc.build(*cfg)
    part = FC.Partition(*cfg)
    cache = L.ImagingCache.from_kernels(np.stack(oc.kernels), oc.source_ws, oc.eigenvalues)
    target = make_target(192, 192, 5)
    opts = dict(enable_cept=True, enable_grad_fusion=True)
    kw = dict(dx=1.0, dy=1.0, cfl=0.7, b=0.01, reinit_interval=2, mask_type=mask_type,
              render_scale=4)
    ref = fc.full_chip_lsm(target, target, meta, oc, THR, ALPHA, fc.ExchangeOptions(**opts), 3, **kw)
    optz = FC.FullChipLSMOptimizer(part, cache, THR, ALPHA)
    res = optz.optimize(torch.from_numpy(target.astype(np.float32)).cuda(),
                        torch.from_numpy(target.astype(np.float32)).cuda(),
                        FC.FullChipLSMOptions(iterations=3, cfl=0.7, curvature_weight=0.01,
                                              reinit_interval=2, mask_type=mask_type,
                                              render_scale=4,
                                              gradient_options=FC.MicroGradientOptions(**opts)))
    assert np.allclose(cpu(res.initial_global_phi), ref["initial_global_phi"], atol=1e-5)
    hist = [h.loss for h in res.history]
    assert len(hist) == 4
    assert abs(hist[0] - ref["history"][0]["loss"]) <= 1e-5 * ref["history"][0]["loss"]
    for a, b in zip(res.history, ref["history"]):
        assert abs(a.loss - b["loss"]) <= 1e-3 * b["loss"]
        assert abs(a.min_dt - b["min_dt"]) <= 1e-4 * max(b["min_dt"], 1e-12)
        assert abs(a.max_dt - b["max_dt"]) <= 1e-4 * max(b["max_dt"], 1e-12)
    assert res.best_iteration == ref["best"]["iteration"]
    gm = cpu(res.global_mask)
    assert (np.abs(gm - ref["global_mask"]) > 1e-6).mean() <= 0.005
    # phi outside each tile's Core + Guard window keeps its initial SDF values
    init = [fc.extract_local_tile(target, t) for t in meta.tiles]
    from oracle import levelset_oracle as lo
    lp = cpu(res.local_phi)
    for t in meta.tiles:
        w = t.update_local
        out = np.ones((meta.tile_size,) * 2, bool)
        out[w.y0:w.y1, w.x0:w.x1] = False
        phi0 = lo.reinit_sdf(init[t.id] - 0.5, 1.0, 1.0)
        assert np.allclose(lp[t.id][out], phi0[out], atol=1e-5)
        # the returned masks are the renders of the returned phi
        assert np.array_equal(cpu(res.local_masks)[t.id],
                              cpu(L.render_levelset_mask(res.local_phi[t.id], mask_type, 4)))


THR_E = 0.17   # about the aerial intensity at the edges of big_target's features


def big_target(H, W, seed):
    """Rectangles of 80-160 nm (20-40 px): resolved edges, |grad I| ~ 0.015 / px. Two
    of them have an edge 3 px from the layout border, so that the periodic copies of
    their edge points fall into the Guards across the border."""
    rng = np.random.default_rng(seed)
    t = np.zeros((H, W))
    for _ in range(6):
        h, w = rng.integers(20, 40), rng.integers(20, 40)
        y, x = rng.integers(8, H - h - 8), rng.integers(8, W - w - 8)
        t[y:y + h, x:x + w] = 1.0
    t[3:30, W // 3:W // 3 + 30] = 1.0
    t[H // 2:H // 2 + 26, 3:28] = 1.0
    return t


def contour_eps(target, seed, stride=3):
    """Synthetic edge points on the 0.5 contour of a binary layout (pixel-edge midlines,
    jittered along the edge), every stride-th kept; every seventh has weight 0
    (inactive)."""
    rng = np.random.default_rng(seed)
    H, W = target.shape
    pts = []
    ys, xs = np.nonzero(np.diff(target, axis=0))
    pts += [(y + 0.5, x + rng.uniform(-0.3, 0.3)) for y, x in zip(ys, xs)]
    ys, xs = np.nonzero(np.diff(target, axis=1))
    pts += [(y + rng.uniform(-0.3, 0.3), x + 0.5) for y, x in zip(ys, xs)]
    eps = np.clip(np.array(pts[::stride]), 0.0, [H - 1e-6, W - 1e-6])
    w = np.ones(len(eps))
    w[::7] = 0.0
    return eps, w


EPE_OPTION_SETS = [
    dict(loss_type="EPE", epe_weight=0.3, epe_pixel_size=2.0),
    dict(loss_type="PE_EPE", loss_region="CoreGuard", main_region_dilation_pixels=2,
         pe_weight=0.8, epe_weight=0.05, collect_core_metrics=True, enable_cept=True,
         cept_guard_only=True, enable_grad_fusion=True, fusion_mode="Linear"),
    dict(loss_type="PEPenalty", loss_region="Core", collect_core_metrics=True, epe_pixel_size=4.0),
]


@pytest.mark.parametrize("prec", ["fp32", "bf16x3"])
@pytest.mark.parametrize("oi", range(len(EPE_OPTION_SETS)))
def test_exchange_epe_matches_oracle(L, FC, band128, oi, prec):
    """EPE / PE_EPE loss types and Core metrics (micro_gradient_exchange.cpp:144-245)
    against the oracle, with caller-supplied EPs. EP counts are exact. The EPE divides
    by |grad I| (~0.015 / px here), so the FP32 image error (~1e-6 absolute) reaches
    ~1e-4 relative per point: EPE sums and EPE-driven gradients are held to 1e-3
    relative, PE terms to 1e-5. Split-BF16 (the tiles in one batched pass, the EP
    work per tile between the forward and the adjoint pass; image error ~1e-5
    absolute): EPE terms and gradients 1e-2, PE terms 1e-4."""
    oc, _ = band128
    cfg = (280, 190, 3, 2, 16, 6)
    meta = fc.build(*cfg)
    ctx = L.Context()
    ctx.set_precision(prec)
    part = FC.Partition(*cfg, ctx=ctx)
    cache = L.ImagingCache.from_kernels(np.stack(oc.kernels), oc.source_ws, oc.eigenvalues, ctx=ctx)
    t_epe, t_pe = (1e-3, 1e-5) if prec == "fp32" else (1e-2, 1e-4)
    target = big_target(cfg[0], cfg[1], 20 + oi)
    eps, w = contour_eps(target, oi)
    rng = np.random.default_rng(30 + oi)
    theta_g = io.initialize_theta(target)     # edges where the EPs are
    masks32 = [io.theta_to_mask(fc.extract_local_tile(theta_g, t)
                                + 0.02 * rng.standard_normal((meta.tile_size,) * 2)).astype(np.float32)
               for t in meta.tiles]
    masks = [m.astype(np.float64) for m in masks32]
    opts = EPE_OPTION_SETS[oi]
    ev = fc.exchange(masks, target, meta, oc, THR_E, ALPHA, fc.ExchangeOptions(**opts), eps, w)
    ex = FC.MicroGradientExchange(part, cache, THR_E, ALPHA)
    res = ex.compute(torch.from_numpy(np.stack(masks32)).cuda(),
                     torch.from_numpy(target.astype(np.float32)).cuda(),
                     FC.MicroGradientOptions(**opts), eps=eps, eps_weights=w)
    raw, grad = cpu(res.raw_gradients), cpu(res.mask_gradients)

    def close(a, b, tol=1e-4, floor=1e-9):
        return abs(a - b) <= tol * max(abs(b), floor)

    n_active = 0
    for t in meta.tiles:
        o, g = ev["locals"][t.id], res.locals[t.id]
        assert rel_l2(raw[t.id], o["raw"]) < t_epe, t.id
        assert rel_l2(grad[t.id], o["grad"]) < t_epe, t.id
        assert g.epe_count == o["epe_count"], t.id
        n_active += g.epe_count
        assert close(g.epe_loss, o["epe_loss"], t_epe) and close(g.epe_abs_sum_nm, o["epe_abs_sum_nm"], t_epe)
        assert close(g.pe_loss, o["pe_loss"], t_pe) and close(g.bg_penalty_raw, o["bg_penalty_raw"], t_pe)
        assert close(g.data_loss, o["data_loss"], t_epe) and close(g.loss, o["loss"], t_epe)
        c, oc_ = g.core, o["core"]
        assert c.ep_count == oc_["ep_count"]
        for k in ("pe_loss", "bg_penalty_raw", "pe_penalty_loss"):
            assert close(getattr(c, k), oc_[k], t_pe), (t.id, k)
        for k in ("epe_loss", "epe_abs_sum_nm", "epe_mean", "data_loss"):
            assert close(getattr(c, k), oc_[k], t_epe), (t.id, k)
    if opts["loss_type"] in ("EPE", "PE_EPE") or opts.get("collect_core_metrics"):
        assert n_active > 0
    assert close(res.loss, ev["loss"], t_epe) and close(res.data_loss, ev["data_loss"], t_epe)
    if opts.get("collect_core_metrics"):
        assert sum(l.core.ep_count for l in res.locals) > 0
    part.close()
    ctx.close()


def test_fullchip_lsm_pe_epe_history(L, FC, band128):
    """FullChipLSMOptimizer with the PE_EPE loss type: history rows (contributions, Core
    sums, EP totals; full_chip_lsm.cpp:152-186) and best Core metrics against the oracle
    over two steps."""
    oc, _ = band128
    cfg = (192, 192, 2, 2, 16, 6)
    meta = fc.build(*cfg)
    part = FC.Partition(*cfg)
    cache = L.ImagingCache.from_kernels(np.stack(oc.kernels), oc.source_ws, oc.eigenvalues)
    target = big_target(192, 192, 9)
    eps, _ = contour_eps(target, 9)
    opts = dict(loss_type="PE_EPE", epe_weight=0.02, enable_cept=True)
    kw = dict(dx=1.0, dy=1.0, cfl=0.7, b=0.01, reinit_interval=0, mask_type="Binary",
              render_scale=4)
    ones = np.ones(len(eps))     # the LSM default epe_all_eps = true
    ref = fc.full_chip_lsm(target, target, meta, oc, THR_E, ALPHA, fc.ExchangeOptions(**opts), 2,
                           eps=eps, eps_weights=ones, **kw)
    optz = FC.FullChipLSMOptimizer(part, cache, THR_E, ALPHA)
    res = optz.optimize(torch.from_numpy(target.astype(np.float32)).cuda(),
                        torch.from_numpy(target.astype(np.float32)).cuda(),
                        FC.FullChipLSMOptions(iterations=2, cfl=0.7, curvature_weight=0.01,
                                              reinit_interval=0,
                                              gradient_options=FC.MicroGradientOptions(
                                                  **opts, epe_all_eps=True)),
                        eps=eps)
    assert len(res.history) == 3
    for a, b in zip(res.history, ref["history"]):
        tol = 1e-3
        for k in ("loss", "data_loss", "pe_contribution", "epe_contribution", "total_pe_loss",
                  "total_epe_loss", "total_epe_abs_sum_nm", "epe_mean"):
            assert abs(getattr(a, k) - b[k]) <= tol * max(abs(b[k]), 1e-9), (a.iteration, k)
        assert a.total_ep_count == b["total_ep_count"] and a.core.ep_count == b["core"]["ep_count"]
        for k in ("pe_loss", "epe_loss", "epe_mean", "data_loss"):
            assert abs(getattr(a.core, k) - b["core"][k]) <= tol * max(abs(b["core"][k]), 1e-9), k
    assert res.history[0].total_ep_count > 0 and res.history[0].epe_contribution > 0.0
    assert res.best_iteration == ref["best"]["iteration"]
    assert len(res.best_core_metrics) == part.num_tiles
