"""Host file formats and the CTM -> LSM hand-off (save_txt.cpp, imbinarize.cpp); CPU only."""
import importlib

import numpy as np
import pytest

F = importlib.import_module("c-version-lithography_b200.formats")


def test_save_load_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    m = rng.standard_normal((5, 7))
    p = tmp_path / "m.txt"
    F.save_mat(m, str(p), precision=9)
    lines = p.read_text().splitlines()
    assert lines[0] == "# rows=5 cols=7"
    assert len(lines[1].split()) == 7
    back = F.load_txt(str(p))
    assert back.shape == (5, 7) and np.max(np.abs(back - m)) <= 5e-10
    F.save_mat_int(np.array([[0.5, -0.5, 1.49], [2.5, -2.5, 3.0]]), str(p))
    assert F.load_txt(str(p)).tolist() == [[1, -1, 1], [3, -3, 3]]   # half away from zero


def test_load_txt_rules(tmp_path):
    p = tmp_path / "a.txt"
    p.write_text("# header\n\n1 2 3\n   # indented comment\n4 5 6\n")
    assert F.load_txt(str(p)).tolist() == [[1, 2, 3], [4, 5, 6]]
    p.write_text("1 2\n3\n")
    with pytest.raises(ValueError, match="inconsistent column count at row 2"):
        F.load_txt(str(p))
    p.write_text("# only comments\n\n")
    with pytest.raises(ValueError, match="empty matrix"):
        F.load_txt(str(p))
    with pytest.raises(ValueError, match="cannot open"):
        F.load_txt(str(tmp_path / "missing.txt"))


def test_binarize_hand_off():
    cv2 = pytest.importorskip("cv2")
    yy, xx = np.mgrid[0:96, 0:96]
    gray = np.clip(0.5 + 0.4 * np.sin(xx / 9.0) * np.cos(yy / 11.0), 0, 1)
    b = F.binarize(gray)
    o = F.binarize_otsu(gray)
    assert set(np.unique(b)) <= {0.0, 1.0} and set(np.unique(o)) <= {0.0, 1.0}
    u8 = np.clip(np.rint(gray * 255.0), 0, 255).astype(np.uint8)
    _, ref = cv2.threshold(u8, 0, 255, cv2.THRESH_BINARY | cv2.THRESH_OTSU)
    assert np.array_equal(o, ref / 255.0)
    assert 0.2 < o.mean() < 0.8


def test_binarize_advanced_stages():
    """Imbinarize::binarize_advanced (imbinarize.cpp:84-189) on a hand-built case."""
    pytest.importorskip("cv2")
    tgt = np.zeros((200, 200))
    tgt[80:120, 80:120] = 1.0
    tgt[10:15, 180:186] = 1.0              # 30-pixel target island: dropped by the final pass
    gray = 0.8 * tgt
    gray[20:40, 20:40] = 0.7               # far SRAF, area 400: kept
    gray[150:153, 150:153] = 0.9           # 3 x 3 blob: below the area threshold
    gray[76:79, 90:110] = 0.7              # SRAF 1-4 px above the target: inside the keep-out
    r = F.binarize_advanced(gray, tgt, peak_min_intensity=0.1, quantile_val=0.2,
                            area_threshold=50, min_spacing_pixels=5)
    # Peaks: 0.7 x 460 (+ 0.8 x 1630, 0.9 x 9); the 0.2 quantile is 0.7.
    assert r.initial_binary_mask.sum() == 1600 + 30 + 400 + 9 + 60
    assert r.filtered_binary_mask.sum() == 1600 + 400 + 60          # blob and island < 50 px
    assert r.sraf_mask_initial.sum() == 400 + 60
    assert r.sraf_mask_final.sum() == 400
    assert np.all(r.keep_out_zone[tgt > 0.5] == 1.0)
    assert not np.any((r.sraf_mask_final > 0) & (r.keep_out_zone > 0))
    expect = np.zeros_like(tgt)
    expect[80:120, 80:120] = 1.0
    expect[20:40, 20:40] = 1.0
    assert np.array_equal(r.final_mask, expect)
    for m in (r.initial_binary_mask, r.final_mask, r.keep_out_zone):
        assert m.dtype == np.float64 and set(np.unique(m)) <= {0.0, 1.0}


def test_binarize_advanced_no_peaks_and_quantile():
    pytest.importorskip("cv2")
    z = F.binarize_advanced(np.zeros((16, 16)), np.ones((16, 16)))
    assert all(np.count_nonzero(m) == 0 for m in (z.initial_binary_mask, z.final_mask,
                                                  z.keep_out_zone))
    v = np.array([3.0, 1.0, 2.0, 10.0])
    assert F._quantile_linear(v, 0.5) == 2.5 and F._quantile_linear(v, 1.0) == 10.0
    assert F._quantile_linear(v, -1.0) == 1.0 and F._quantile_linear(np.array([]), 0.3) == 0.0
    with pytest.raises(ValueError, match="sizes must match"):
        F.binarize_advanced(np.zeros((4, 4)), np.zeros((4, 5)))
