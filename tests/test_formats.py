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


def test_full_chip_lsm_csv_schemas(tmp_path):
    """history.csv / core_metrics_best.csv / summary.csv (demo_full_chip_lsm.cpp:170-201)."""
    from types import SimpleNamespace as NS
    core = NS(pe_loss=1.25, bg_penalty_raw=0.5, pe_penalty_loss=2.25, epe_loss=3.0 / 7.0,
              epe_abs_sum_nm=12.0, ep_count=5, epe_mean=2.4, data_loss=1.0 / 3.0)
    rows = [NS(iteration=i, loss=10.0 - i, data_loss=9.0 - i, cept_loss=0.1 * i, min_dt=0.01 * i,
               max_dt=0.02 * i, pe_contribution=1.0, penalty_contribution=0.0,
               epe_contribution=0.2, cept_contribution=0.11 * i, core=core, total_pe_loss=2.0,
               total_bg_penalty_raw=0.0, total_epe_loss=0.5, total_epe_abs_sum_nm=20.0,
               total_ep_count=9, epe_mean=20.0 / 9.0) for i in range(3)]
    p = tmp_path / "history.csv"
    F.write_lsm_history_csv(rows, str(p))
    lines = p.read_text().splitlines()
    assert lines[0].split(",")[:4] == ["iteration", "loss", "data_loss", "cept_loss"]
    assert len(lines[0].split(",")) == 24 and len(lines) == 4
    v = lines[2].split(",")
    assert v[0] == "1" and float(v[1]) == 9.0 and v[15] == "5" and v[22] == "9"
    assert float(v[13]) == 3.0 / 7.0 and float(v[23]) == 20.0 / 9.0     # 17 digits round-trip
    tiles = [NS(id=t, core_global=NS(y0=10 * t, y1=10 * t + 10, x0=0, x1=16)) for t in range(2)]
    res = NS(best_iteration=2, best_loss=8.0, history=rows, best_core_metrics=[core, core])
    p = tmp_path / "core.csv"
    F.write_core_metrics_csv(res, NS(tiles=tiles), str(p))
    lines = p.read_text().splitlines()
    assert lines[0].startswith("best_iteration,micro_id,y0,y1,x0,x1,core_pe")
    assert lines[2].split(",")[:6] == ["2", "1", "10", "20", "0", "16"]
    p = tmp_path / "summary.csv"
    F.write_summary_csv(res, 1.5, str(p))
    assert p.read_text().splitlines() == ["best_iteration,best_loss,final_iteration,final_loss,seconds",
                                          "2,8,2,8,1.5"]
