"""Seeded workload generators of the benchmark (CPU only): the uneven Core cuts of the
full-chip layout and the reference's theta initialisation."""
import importlib

import numpy as np
import pytest

wl = importlib.import_module("c-version-lithography_b200.workloads")


@pytest.mark.parametrize("extent,lo,hi", [(16384, 256, 1024), (4096, 256, 1024), (300, 40, 100),
                                          (256, 256, 1024)])
def test_uneven_cuts_cover_the_extent_within_bounds(extent, lo, hi):
    for seed in range(20):
        cuts = wl.uneven_cuts(extent, lo, hi, seed)
        sides = np.diff(cuts)
        assert cuts[0] == 0 and cuts[-1] == extent
        assert sides.min() >= lo and sides.max() <= hi
    # seeded: the same seed gives the same cuts, another seed other cuts
    assert wl.uneven_cuts(extent, lo, hi, 3) == wl.uneven_cuts(extent, lo, hi, 3)
    if extent > 2 * hi:
        assert wl.uneven_cuts(extent, lo, hi, 3) != wl.uneven_cuts(extent, lo, hi, 4)


def test_uneven_cuts_reject_impossible_bounds():
    with pytest.raises(ValueError):
        wl.uneven_cuts(100, 256, 1024, 0)      # extent below the smallest Core
    with pytest.raises(ValueError):
        wl.uneven_cuts(4096, 300, 500, 0)      # hi < 2 lo: a remainder may not split


def test_theta_init_reference_values():
    """CTM_Optimizer::_initialize_theta (CTM_Optimizer.cpp:55-64): 0.3 pi on the target,
    0.7 pi off it."""
    t = np.array([[0.0, 1.0], [1.0, 0.0]])
    th = wl.theta_init_reference(t)
    assert np.allclose(th, np.pi * np.array([[0.7, 0.3], [0.3, 0.7]]))
