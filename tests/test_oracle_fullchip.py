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
