"""Pins the FP64 oracle to the reference's own known-answer tests (CPU only).

The reference cannot be built here, so its tests are restated against the
oracle: tests/test_ctm_optimizer.cpp (FD gradient checks on real optics,
frequency axis), tests/test_level_set_godunov.cpp (planar, extremum, circle
symmetry, invalid input), tests/test_full_chip_imaging_compare.cpp:83-103
(compact SOCS == dense SOCS) and the golden fixtures of tests/golden/.
"""
import glob
import os

import numpy as np
import pytest

from oracle import imaging_oracle as io
from oracle import levelset_oracle as lo
from oracle import optics_oracle as oo

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("n", [64, 65])
@pytest.mark.parametrize("with_penalty", [False, True])
def test_fd_gradient_real_optics(n, with_penalty):
    """check_pe_gradient (tests/test_ctm_optimizer.cpp:61-96)."""
    cache = oo.prepare(n, 4.0, 193.0, 1.35, 0.6, 0.9, use_socs=True)
    target = np.zeros((n, n)); target[23:42, 23:42] = 1.0
    thr, alpha = 0.25, (10.0 if with_penalty else 85.0)
    theta = io.initialize_theta(target)
    a, w, E = io.imaging_compute(io.theta_to_mask(theta), cache, thr, alpha)
    kw = dict(penalty=2.0, penalty_threshold=0.01) if with_penalty else {}
    if with_penalty:
        assert io.pe_loss_with_penalty(w, target, 2.0, 0.01) > io.pe_loss(w, target)
    gm = io.pe_gradient(w, target, E, cache, alpha, **kw)
    gt = -0.5 * gm * np.sin(theta)
    assert np.linalg.norm(gt) > 1e-8
    d = -gt / np.linalg.norm(gt)

    def ev(th):
        _, ww, _ = io.imaging_compute(io.theta_to_mask(th), cache, thr, alpha, keep_fields=False)
        return io.pe_loss_with_penalty(ww, target, 2.0, 0.01) if with_penalty else io.pe_loss(ww, target)

    h = 1e-3
    num = (ev(theta + h * d) - ev(theta - h * d)) / (2 * h)
    ana = float((gt * d).sum())
    assert abs(num - ana) <= 1e-3 * max(1.0, abs(num))


@pytest.mark.parametrize("n", [64, 65])
def test_frequency_axis(n):
    """check_grid_dimensions (tests/test_ctm_optimizer.cpp:42-59)."""
    f = oo.normalised_axis(n, 4.0, 1.35, 193.0)
    step = (1.0 / (n * 4.0)) * 193.0 / 1.35
    assert f[n // 2] == 0.0
    assert abs(f[0] + (n // 2) * step) < 1e-12
    assert abs(f[-1] - (n - 1 - n // 2) * step) < 1e-12
    assert np.all(np.abs(np.diff(f) - step) < 1e-12)


def test_compact_socs_equals_dense():
    """tests/test_full_chip_imaging_compare.cpp:83-103 (128^2, 8 nm)."""
    dense = oo.prepare(128, 8.0, 193.0, 1.35, 0.6, 0.9, use_socs=True, compact=False)
    compact = oo.prepare(128, 8.0, 193.0, 1.35, 0.6, 0.9, use_socs=True, compact=True)
    assert np.max(np.abs(np.array(dense.eigenvalues) - np.array(compact.eigenvalues))) < 1e-9
    m = np.random.default_rng(0).random((128, 128))
    a1, w1, _ = io.imaging_compute(m, dense, 0.25, 85.0, keep_fields=False)
    a2, w2, _ = io.imaging_compute(m, compact, 0.25, 85.0, keep_fields=False)
    assert np.max(np.abs(a1 - a2)) < 1e-10
    assert np.max(np.abs(w1 - w2)) < 1e-10


def _x_plane(rows, cols, slope):
    return slope * (np.arange(cols)[None, :] - 0.5 * (cols - 1)) * np.ones((rows, 1))


def test_godunov_planar():
    """test_planar_signed_distance (tests/test_level_set_godunov.cpp:36-65)."""
    rows, cols = 25, 29
    r, c = rows // 2, cols // 2
    pos = np.full((rows, cols), 2.0)
    d, h1, h2 = lo.evolve_normal_weno_godunov(_x_plane(rows, cols, 1.0), pos, 1.0, 1.0)
    assert abs(d[r, c] - 2.0) < 1e-12 and abs(h1[r, c] - 2.0) < 1e-12 and abs(h2[r, c] - 2.0) < 1e-12
    d, _, _ = lo.evolve_normal_weno_godunov(_x_plane(rows, cols, -1.0), pos, 1.0, 1.0)
    assert abs(d[r, c] - 2.0) < 1e-12
    d, _, _ = lo.evolve_normal_weno_godunov(_x_plane(rows, cols, 1.0), -pos, 1.0, 1.0)
    assert abs(d[r, c] + 2.0) < 1e-12
    assert d.shape == (rows, cols)


def test_godunov_extremum():
    """test_godunov_at_one_dimensional_extremum (tests/test_level_set_godunov.cpp:67-96)."""
    rows, cols = 17, 25
    c = cols // 2
    mn = np.abs(np.arange(cols)[None, :] - c) * np.ones((rows, 1))
    one = np.ones((rows, cols))
    cases = [(mn, one, 0.0, 1e-12), (mn, -one, -1.0, 1e-6), (-mn, one, 1.0, 1e-6), (-mn, -one, 0.0, 1e-12)]
    for phi, sp, want, tol in cases:
        d, _, _ = lo.evolve_normal_weno_godunov(phi, sp, 1.0, 1.0)
        assert abs(d[rows // 2, c] - want) < tol


def test_godunov_rejects_mismatch():
    """test_invalid_inputs_are_rejected (tests/test_level_set_godunov.cpp:98-109)."""
    with pytest.raises(ValueError):
        lo.evolve_normal_weno_godunov(np.zeros((5, 7)), np.zeros((5, 6)), 1.0, 1.0)


def circle_phi(size=33, radius=10.0):
    c = 0.5 * (size - 1)
    y, x = np.mgrid[0:size, 0:size].astype(np.float64)
    return radius - np.hypot(x - c, y - c)


def test_circle_symmetry():
    """test_circle_symmetry (tests/test_level_set_godunov.cpp:111-187)."""
    phi = circle_phi()
    d, _, _ = lo.evolve_normal_weno_godunov(phi, np.ones_like(phi), 1.0, 1.0)
    n, m = phi.shape[0], 4
    band = np.abs(phi) <= 3.0
    err = 0.0
    for i in range(m, n - m):
        for j in range(m, n - m):
            if band[i, j]:
                err = max(err, abs(d[i, j] - d[i, n - 1 - j]), abs(d[i, j] - d[n - 1 - i, j]))
    assert err < 1e-12


def test_weno_matches_loop_restatement():
    """The vectorised WENO equals a literal per-element loop of weno5_1d (level_set_utils.cpp:45-113)."""
    rng = np.random.default_rng(5)
    v = np.cumsum(rng.standard_normal(30))
    n = len(v) - 12

    def loop(vv, direction):
        D1 = np.diff(vv)
        out = []
        for i in range(n):
            if direction == "plus":
                a = [D1[i + 5], D1[i + 4], D1[i + 3], D1[i + 2], D1[i + 1]]
            else:
                a = [D1[i + q] for q in range(5)]
            v1, v2, v3, v4, v5 = a
            d1 = v1 / 3 - 7 * v2 / 6 + 11 * v3 / 6
            d2 = -v2 / 6 + 5 * v3 / 6 + v4 / 3
            d3 = v3 / 3 + 5 * v4 / 6 - v5 / 6
            S1 = 13 / 12 * (v1 - 2 * v2 + v3) ** 2 + 0.25 * (v1 - 4 * v2 + 3 * v3) ** 2
            S2 = 13 / 12 * (v2 - 2 * v3 + v4) ** 2 + 0.25 * (v2 - v4) ** 2
            S3 = 13 / 12 * (v3 - 2 * v4 + v5) ** 2 + 0.25 * (3 * v3 - 4 * v4 + v5) ** 2
            eps = 1e-6 * max(x * x for x in a) + 1e-99
            a1, a2, a3 = 0.1 / (S1 + eps) ** 2, 0.6 / (S2 + eps) ** 2, 0.3 / (S3 + eps) ** 2
            out.append((a1 * d1 + a2 * d2 + a3 * d3) / (a1 + a2 + a3))
        return np.array(out)

    for direction in ("plus", "minus"):
        got = lo.weno5_rows(v[None, :], n, 1.0, direction)[0]
        assert np.max(np.abs(got - loop(v, direction))) < 1e-12


def test_golden_fixtures_reproduce():
    """The committed fixtures are what the oracle computes today."""
    import importlib
    wl = importlib.import_module("c-version-lithography_b200.workloads")
    for path in sorted(glob.glob(os.path.join(GOLDEN, "ctm_*.npz"))):
        z = np.load(path)
        name = os.path.basename(path)
        if name.startswith("ctm_real_"):
            n = int(name.split("_")[2].split(".")[0])
            cache = oo.prepare(n, 4.0, 193.0, 1.35, 0.6, 0.9, use_socs=True)
        elif name.startswith("ctm_gauss_"):
            n = int(name.split("_")[2]); socs = "socs" in name
            cache = oo.synthetic_gaussian_cache(n, socs)
            cache.source_ws = np.array([0.3, 0.9])
        else:
            band, r0, c0, w, wss = wl.synthetic_socs_band()
            cache = io.OracleCache(N=128, kernels=list(wl.band_to_dense(band, r0, c0, 128)),
                                   source_ws=np.array([wss]), eigenvalues=tuple(w))
        r = io.ctm_evaluate(z["theta"].astype(np.float64), z["target"].astype(np.float64), cache,
                            float(z["thr"]), float(z["alpha"]))
        tol = 1e-6 if z["aerial"].dtype == np.float32 else 1e-10
        assert np.max(np.abs(r["aerial"] - z["aerial"])) <= tol * np.max(np.abs(z["aerial"])), name
        assert abs(r["loss"] - float(z["loss"])) <= 1e-8 * max(1.0, abs(float(z["loss"]))), name
