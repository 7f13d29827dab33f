"""Host-side arithmetic of bench.py on CPU (no GPU): the algorithmic bytes and FLOPs
its roofline and tensor-core fractions divide by, the parser of the clock record that
decides whether a run stands, and the seeded edge points of the accuracy statement."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402

N, K, NR, NC = 2048, 24, 35, 35


def test_stage_bytes_of_the_headline_tile():
    """Per 2048^2 tile: theta in for the tile analysis, the target in for the resist
    synthesis, theta in and dPE/dtheta out for the theta chain (4 x 4 N^2 = 67 MB), plus
    the complex64 band partials of the 256 tiles of 128^2 (35 x 35 forward, 69 x 35
    adjoint)."""
    px = 4 * N * N
    sb = bench.stage_bytes(N, NR, NC, fused=True)
    assert sb["tile_analysis"] == px + 8 * 256 * 35 * 35
    assert sb["row_synthesis_resist"] == px + 8 * 256 * 69 * 35
    assert sb["adjoint_row_synthesis_theta"] == 2 * px
    assert sb["tile_analysis"] + sb["row_synthesis_resist"] + sb["adjoint_row_synthesis_theta"] \
        - 8 * 256 * 35 * (35 + 69) == 4 * px == 67_108_864
    # 16 tiles per launch: the algorithmic bytes of the headline roofline
    assert 16 * sb["row_synthesis_resist"] == 347_570_176
    # the unfused chain writes dL/dI and reads it back
    un = bench.stage_bytes(N, NR, NC, fused=False)
    assert un["row_synthesis_resist"] == 2 * px
    assert un["adjoint_tile_analysis"] == px + 8 * 256 * 69 * 35


def test_mma_flops_count_the_three_split_passes_with_padding():
    """Tile analysis: two 128 x 80 x 128 products per 128^2 tile (2 Nc = 70 padded to 80),
    three split-BF16 passes each; synthesis: 128 x 128 x 80 per tile (2 Nr padded)."""
    mf = bench.mma_flops(N, NR, NC)
    tiles = 256
    ana = tiles * 3 * 2 * 2 * 128 * 128 * 80
    syn = tiles * 3 * 2 * 128 * 128 * 80
    assert mf == {"tile_analysis": ana, "row_synthesis_resist": syn + ana,
                  "adjoint_row_synthesis_theta": syn}
    assert bench.round16(70) == 80 and bench.round16(80) == 80 and bench.round16(1) == 16


def test_equivalent_pruned_dft_flops():
    """(16K + 12) N^2 Nk + (16K + 16) N Nk^2 per tile-iteration: 5.91e10 at 2048^2,
    K = 24, Nk = 35."""
    f = bench.algorithmic_flops(N, K, NR)
    assert f == (16 * 24 + 12) * N * N * 35 + (16 * 24 + 16) * N * 35 * 35
    assert abs(f / 5.91e10 - 1) < 1e-3


def test_clock_summary_reports_median_and_active_reasons():
    s = bench.ClockSampler(0)
    s.lines = [
        "1965, 1965, 812.3, Not Active, Not Active, Not Active, Not Active",
        "1950, 1965, 990.1, Not Active, Not Active, Not Active, Active",
        "1965, 1965, 995.0, Not Active, Not Active, Not Active, Active",
        "garbage",
        "[N/A], 1965, 0, Not Active, Not Active, Not Active, Not Active",
    ]
    out = s.summary()
    assert out == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"],
                   "samples": 3}
    s.lines = ["1400, 1965, 700, Active, Not Active, Active, Not Active"]
    assert s.summary()["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]
    s.lines = []
    assert s.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}


def test_edge_points_lie_on_target_edges_and_are_seeded():
    """Points sit on the 0.5 contour of the binary target (one coordinate at a pixel-edge
    midline, the other within 0.3 px of a pixel centre), at most n, and the same seed
    gives the same points."""
    t = np.zeros((64, 64))
    t[16:40, 20:50] = 1.0
    yy, xx = np.mgrid[0:64, 0:64]
    aerial = np.exp(-((yy - 28) ** 2 + (xx - 35) ** 2) / 300.0)
    p = bench.edge_points(t, aerial, n=32, seed=5)
    assert p.shape == (32, 2)
    for y, x in p:
        on_row_edge = abs(y - np.floor(y) - 0.5) < 1e-12 and abs(x - np.rint(x)) <= 0.3
        on_col_edge = abs(x - np.floor(x) - 0.5) < 1e-12 and abs(y - np.rint(y)) <= 0.3
        assert on_row_edge or on_col_edge
        # the midline lies between a printed and an unprinted pixel
        if on_row_edge:
            a, b = int(np.floor(y)), int(np.rint(x))
            assert t[a, b] != t[a + 1, b]
        else:
            a, b = int(np.rint(y)), int(np.floor(x))
            assert t[a, b] != t[a, b + 1]
    assert np.array_equal(p, bench.edge_points(t, aerial, n=32, seed=5))
    # fewer qualifying points than n: the n steepest are taken
    flat = np.full((64, 64), 0.5)
    q = bench.edge_points(t, flat, n=16, seed=5)
    assert q.shape == (16, 2)
