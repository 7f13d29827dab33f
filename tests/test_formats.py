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
