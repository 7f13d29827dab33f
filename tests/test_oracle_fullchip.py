"""Pins the full-chip oracle to the reference's known answers (CPU only):
tests/test_full_chip_ctm.cpp:50-187 (single-micro == standalone GD, guard-only
CEPT with fusion) and the partition geometry of partition.cpp:21-120."""
import numpy as np

from oracle import fullchip_oracle as fc
from oracle import imaging_oracle as io
from oracle import optics_oracle as oo


def make_target():
    t = np.zeros((24, 24))
    t[7:17, 5:19] = 1.0
    t[10:14, 10:14] = 0.0
    return t


def test_partition_geometry():
    meta = fc.build(24, 24, 2, 2, 4, 2)
    assert meta.tile_size == 20
    t0 = meta.tiles[0]
    assert t0.core_global == fc.Rect(0, 12, 0, 12)
    assert t0.tile_global == fc.Rect(-4, 16, -4, 16)
    assert t0.update_local == fc.Rect(2, 18, 2, 18)
    # right neighbour of tile 0: guard strip of tile 0 is neighbour core columns 12..14
    right = [n for n in t0.neighbors if n.direction == fc.RIGHT][0]
    assert right.guard_global == fc.Rect(0, 12, 12, 14)
    assert right.my_guard_local == fc.Rect(4, 16, 16, 18)
    assert right.neighbor_overlap_local == fc.Rect(4, 16, 4, 6)
    # uneven split: 25 rows into 2 -> cores of 12 and 13, tile size max+2 halo rounded even
    meta = fc.build(25, 31, 2, 3, 3, 1)
    assert meta.tile_size == (13 + 6) + 1
    rng = np.random.default_rng(0)
    g = rng.random((25, 31))
    locs = [fc.extract_local_tile(g, t) for t in meta.tiles]
    assert np.array_equal(fc.assemble_global(locs, meta), g)


def test_single_micro_equals_standalone_gd():
    """check_single_micro (tests/test_full_chip_ctm.cpp:50-97), SOCS and Abbe."""
    for socs in (True, False):
        meta = fc.build(24, 24, 1, 1, 0, 0)
        cache = oo.synthetic_gaussian_cache(meta.tile_size, socs)
        target = make_target()
        res = fc.full_chip_ctm(target, target, meta, cache, 0.25, 8.0, fc.ExchangeOptions(), 4, 0.01)
        theta = io.initialize_theta(target)
        best_loss, best_mask = np.inf, None
        for it in range(5):
            mask = io.theta_to_mask(theta)
            _, w, E = io.imaging_compute(mask, cache, 0.25, 8.0)
            loss = io.pe_loss(w, target)
            assert abs(loss - res["history"][it]) < 1e-11
            if loss < best_loss:
                best_loss, best_mask = loss, mask
            if it < 4:
                gm = io.pe_gradient(w, target, E, cache, 8.0)
                theta = theta + 0.5 * 0.01 * gm * np.sin(theta)
        assert np.allclose(best_mask, res["global_mask"], atol=1e-12)
        assert best_loss < res["history"][0]


def test_guard_only_cept_and_fusion():
    """check_guard_only_update (tests/test_full_chip_ctm.cpp:99-187)."""
    meta = fc.build(24, 24, 2, 2, 4, 2)
    cache = oo.synthetic_gaussian_cache(meta.tile_size, True)
    target = make_target()
    opt = fc.ExchangeOptions(enable_cept=True, enable_grad_fusion=True, cept_guard_only=False)
    res = fc.full_chip_ctm(target, target, meta, cache, 0.25, 8.0, opt, 2, 0.01)
    init = [fc.extract_local_tile(io.initialize_theta(target), t) for t in meta.tiles]
    for t in meta.tiles:
        w = t.update_local
        outside = np.ones((meta.tile_size, meta.tile_size), bool)
        outside[w.y0:w.y1, w.x0:w.x1] = False
        assert np.array_equal(res["thetas"][t.id][outside], init[t.id][outside])
    # guard-only CEPT leaves Core pixels of the CEPT gradient at zero
    masks = [io.theta_to_mask(th) for th in res["thetas"]]
    ev = fc.exchange(masks, target, meta, cache, 0.25, 8.0,
                     fc.ExchangeOptions(enable_cept=True, cept_guard_only=True))
    assert ev["cept_loss"] > 0.0
    for t in meta.tiles:
        c = t.core_local
        assert np.linalg.norm(ev["locals"][t.id]["cept_grad"][c.y0:c.y1, c.x0:c.x1]) == 0.0
    assert res["best"]["iteration"] > 0


def _literal_windows(target, region, radius, loss_type):
    """The independent window restatement of test_micro_gradient_exchange.cpp:497-518:
    the PE_EPE main region as "a target pixel > 0.5 within L-infinity distance radius"."""
    pe = np.zeros_like(target); epe = np.zeros_like(target); pen = np.zeros_like(target)
    H, W = target.shape
    for y in range(region.y0, region.y1):
        for x in range(region.x0, region.x1):
            main = bool(np.any(target[max(0, y - radius):min(H - 1, y + radius) + 1,
                                      max(0, x - radius):min(W - 1, x + radius) + 1] > 0.5))
            epe[y, x] = main if loss_type == "PE_EPE" else 1.0
            pe[y, x] = (not main) if loss_type == "PE_EPE" else \
                (target[y, x] > 0.5 if loss_type == "PEPenalty" else 1.0)
            pen[y, x] = target[y, x] < 0.5
    return pe, pen, epe


def test_loss_windows_match_reference_known_answer():
    """check_loss_windows (test_micro_gradient_exchange.cpp:520-546): dilation before the
    region cut, zero border, strict > 0.5, mutually exclusive PE / EPE windows."""
    target = np.zeros((12, 15))
    target[0, 0] = 1.0
    target[2, 2] = 0.5
    target[4:8, 5:9] = 1.0
    target[5, 6] = 0.0
    target[1, 8] = 1.0
    region = fc.Rect(2, 11, 3, 14)
    for radius in (0, 1, 2, 4):
        opt = fc.ExchangeOptions(loss_type="PE_EPE", main_region_dilation_pixels=radius)
        pe, pen, epe = fc.loss_windows(target, region, opt)
        rpe, rpen, repe = _literal_windows(target, region, radius, "PE_EPE")
        assert np.array_equal(pe, rpe) and np.array_equal(epe, repe) and np.array_equal(pen, rpen)
        assert np.sum(pe * epe) == 0.0 and pe.sum() + epe.sum() == region.rows * region.cols
    for lt in ("PE", "PEPenalty", "EPE"):
        pe, pen, epe = fc.loss_windows(target, region, fc.ExchangeOptions(loss_type=lt))
        rpe, rpen, repe = _literal_windows(target, region, 0, lt)
        assert np.array_equal(pe, rpe) and np.array_equal(epe, repe) and np.array_equal(pen, rpen)


def test_region_eps_local_periodic_copies():
    """region_eps_local (micro_gradient_exchange.cpp:18-50): half-open global region,
    periodic copies only for Core + Guard, window test on the clamped bilinear stencil."""
    meta = fc.build(32, 32, 2, 2, 8, 3)
    t0 = meta.tiles[0]                      # Core [0,16) x [0,16), tile origin (-8, -8)
    win = np.zeros((meta.tile_size,) * 2)
    r = t0.update_local
    win[r.y0:r.y1, r.x0:r.x1] = 1.0
    eps = np.array([[5.25, 6.5], [31.5, 4.0], [16.0, 3.0], [15.99, 15.5], [2.0, 30.6]])
    w = np.array([1.0, 0.5, 1.0, 0.0, 2.0])
    le, lw = fc.region_eps_local(eps, w, t0, t0.core_local, 32, 32, False, win)
    # (16.0, 3.0) is on the Core's open edge; the periodic points stay out without copies
    assert np.allclose(le, [[13.25, 14.5], [23.99, 23.5]]) and np.allclose(lw, [1.0, 0.0])
    le, lw = fc.region_eps_local(eps, w, t0, t0.update_local, 32, 32, True, win)
    got = {(round(a, 3), round(b, 3)) for a, b in le}
    # copies one layout up / left land in the Guard: y 31.5 - 32 = -0.5, x 30.6 - 32 = -1.4
    assert (7.5, 12.0) in got and (10.0, 6.6) in got and (24.0, 11.0) in got
    assert len(le) == len(lw) == 5


def test_partition_geometry_with_cuts():
    """Partition::build over caller-given Core boundaries: the reference's own cuts
    reproduce the default partition; uneven cuts keep one tile size (largest Core +
    2 halo, rounded even), Core + halo origins, and a Core stitch that is exact."""
    a = fc.build(25, 31, 2, 3, 3, 1)
    b = fc.build(25, 31, 2, 3, 3, 1, row_cuts=[0, 12, 25], col_cuts=[0, 10, 20, 31])
    assert a == b
    meta = fc.build(60, 50, 3, 2, 4, 2, row_cuts=[0, 5, 45, 60], col_cuts=[0, 17, 50])
    assert meta.tile_size == 40 + 8
    t = meta.tiles[1 * 2 + 1]
    assert t.core_global == fc.Rect(5, 45, 17, 50)
    assert t.tile_global == fc.Rect(1, 49, 13, 61)
    top = [n for n in t.neighbors if n.direction == fc.TOP][0]
    assert top.guard_global == fc.Rect(3, 5, 17, 50)
    g = np.random.default_rng(1).random((60, 50))
    locs = [fc.extract_local_tile(g, tt) for tt in meta.tiles]
    assert np.array_equal(fc.assemble_global(locs, meta), g)
