"""The on-disk formats against the reference's own asset files (CPU).

The reference ships its inputs as text matrices written in the SaveTxt format
(source/utils/save_txt.cpp:23-105; assets/lsm_mask/*.txt, 257 x 257 LSM masks, and
assets/target_pattern/*_1024.txt, 1024 x 1024 targets) and as bitmaps read by the demos
with cv::imread (assets/target_pattern/*.bmp). These tests read those files where the
reference tree is present (they are skipped elsewhere): load_txt gives the matrices
with their shapes and binary values, the 1024 x 1024 text targets equal their bitmaps
read as the demos read them, save_mat_int writes the same values back, and
binarize_advanced (imbinarize.cpp:84-189) runs on a reference target with its
invariants checked and its peak threshold against NumPy's linear quantile.
"""
import glob
import importlib
import os

import numpy as np
import pytest

REF = "/root/reference/assets"
pytestmark = pytest.mark.skipif(not os.path.isdir(REF), reason="reference assets not present")


@pytest.fixture(scope="module")
def F():
    return importlib.import_module("c-version-lithography_b200.formats")


def lsm_masks():
    return sorted(glob.glob(os.path.join(REF, "lsm_mask", "*.txt")))


def test_lsm_mask_assets_load_and_round_trip(F, tmp_path):
    paths = lsm_masks()
    assert len(paths) >= 10
    for p in paths:
        m = F.load_txt(p)
        assert m.shape == (257, 257), p
        assert set(np.unique(m)) <= {0.0, 1.0}, p
        assert 0.0 < m.mean() < 1.0, p
    # save_mat_int writes the same values, one row per line after its header
    m = F.load_txt(paths[0])
    out = tmp_path / "rt.txt"
    F.save_mat_int(m, str(out))
    lines = out.read_text().splitlines()
    assert lines[0] == "# rows=257 cols=257"
    with open(paths[0]) as f:
        ref_rows = [ln.split() for ln in f if ln.strip() and not ln.lstrip().startswith("#")]
    assert [ln.split() for ln in lines[1:]] == ref_rows
    assert np.array_equal(F.load_txt(str(out)), m)


@pytest.mark.parametrize("name", ["contact_1_0_only_1024", "metal_3_0_only_1024"])
def test_1024_text_targets_equal_their_bitmaps(F, name):
    t = F.load_txt(os.path.join(REF, "target_pattern", name + ".txt"))
    b = F.load_target_image(os.path.join(REF, "target_pattern", name + ".bmp"))
    assert t.shape == (1024, 1024) and b.shape == (1024, 1024)
    assert np.array_equal(t, b)
    assert set(np.unique(t)) == {0.0, 1.0}


def test_load_txt_errors_like_the_reference(F, tmp_path):
    bad = tmp_path / "bad.txt"
    bad.write_text("# rows=2 cols=3\n1 2 3\n4 5\n")
    with pytest.raises(ValueError, match="inconsistent column count at row 2"):
        F.load_txt(str(bad))
    empty = tmp_path / "empty.txt"
    empty.write_text("# only a comment\n\n")
    with pytest.raises(ValueError, match="empty matrix"):
        F.load_txt(str(empty))
    with pytest.raises(ValueError, match="cannot open"):
        F.load_txt(str(tmp_path / "missing.txt"))


def test_binarize_advanced_on_a_reference_target(F):
    import cv2
    target = F.load_txt(os.path.join(REF, "target_pattern", "contact_1_0_only_1024.txt"))
    # A CTM-like gray mask: the blurred target plus a weaker halo ring where sub-resolution
    # assist features would grow.
    t8 = target.astype(np.uint8)
    ring = (cv2.dilate(t8, cv2.getStructuringElement(cv2.MORPH_ELLIPSE, (51, 51)))
            - cv2.dilate(t8, cv2.getStructuringElement(cv2.MORPH_ELLIPSE, (25, 25))))
    gray = (0.8 * cv2.GaussianBlur(target, (0, 0), 4.0)
            + 0.5 * cv2.GaussianBlur(ring.astype(np.float64), (0, 0), 3.0))
    r = F.binarize_advanced(gray, target, 0.1, 0.15, area_threshold=5, min_spacing_pixels=5)
    for m in (r.initial_binary_mask, r.filtered_binary_mask, r.sraf_mask_initial,
              r.sraf_mask_final, r.final_mask, r.keep_out_zone):
        assert m.shape == target.shape and set(np.unique(m)) <= {0.0, 1.0}
    # peak threshold: NumPy's linear quantile of the 3x3 local maxima above 0.1
    dil = cv2.dilate(gray, cv2.getStructuringElement(cv2.MORPH_RECT, (3, 3)))
    peaks = gray[(gray >= dil) & (gray > 0.1)]
    thr = np.quantile(peaks, 0.15, method="linear")
    assert np.array_equal(r.initial_binary_mask, (gray >= thr).astype(np.float64))
    assert np.all(r.filtered_binary_mask <= r.initial_binary_mask)
    assert np.array_equal(r.sraf_mask_initial, r.filtered_binary_mask * (target <= 0.5))
    assert np.all(r.keep_out_zone >= target)
    assert not np.any((r.sraf_mask_final > 0) & (r.keep_out_zone > 0))
    assert np.all(r.final_mask <= np.maximum(target, r.sraf_mask_final))
    assert r.sraf_mask_final.sum() > 0          # the halo survives as assist features
    # every target component of at least area_threshold pixels is kept
    n, lab, st, _ = cv2.connectedComponentsWithStats(t8, connectivity=8)
    for i in range(1, n):
        if st[i, cv2.CC_STAT_AREA] >= 5:
            assert np.all(r.final_mask[lab == i] == 1.0)
