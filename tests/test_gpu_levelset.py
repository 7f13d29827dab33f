"""GPU parity of the WENO5-Godunov level-set kernels against the FP64 oracle and the
reference's known answers (tests/test_level_set_godunov.cpp).

FP32 tolerances: known answers 1e-5 absolute (the reference uses 1e-12 / 1e-6
in FP64); oracle comparisons 1e-5 of the field's maximum magnitude.
"""
import importlib
import os

import numpy as np
import pytest

from oracle import levelset_oracle as lo

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def L():
    p = importlib.import_module("c-version-lithography_b200")
    assert torch.cuda.is_available()
    p.load_library()
    return p


def cpu(t):
    return t.detach().cpu().numpy().astype(np.float64)


def rel_max(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-30))


def _x_plane(rows, cols, slope):
    return slope * (np.arange(cols)[None, :] - 0.5 * (cols - 1)) * np.ones((rows, 1))


def test_planar_signed_distance(L):
    rows, cols = 25, 29
    r, c = rows // 2, cols // 2
    pos = np.full((rows, cols), 2.0)
    e = L.LevelSetUtils.evolve_normal_WENO_godunov(_x_plane(rows, cols, 1.0), pos, 1.0, 1.0)
    assert abs(cpu(e.delta)[r, c] - 2.0) < 1e-5
    assert abs(cpu(e.H1_abs)[r, c] - 2.0) < 1e-6 and abs(cpu(e.H2_abs)[r, c] - 2.0) < 1e-6
    e = L.LevelSetUtils.evolve_normal_WENO_godunov(_x_plane(rows, cols, -1.0), pos, 1.0, 1.0)
    assert abs(cpu(e.delta)[r, c] - 2.0) < 1e-5
    e = L.LevelSetUtils.evolve_normal_WENO_godunov(_x_plane(rows, cols, 1.0), -pos, 1.0, 1.0)
    assert abs(cpu(e.delta)[r, c] + 2.0) < 1e-5
    assert tuple(e.delta.shape) == (rows, cols)


def test_godunov_extremum(L):
    rows, cols = 17, 25
    c = cols // 2
    mn = np.abs(np.arange(cols)[None, :] - c) * np.ones((rows, 1))
    one = np.ones((rows, cols))
    for phi, sp, want in [(mn, one, 0.0), (mn, -one, -1.0), (-mn, one, 1.0), (-mn, -one, 0.0)]:
        d = cpu(L.LevelSetUtils.evolve_normal_WENO_godunov(phi, sp, 1.0, 1.0).delta)
        assert abs(d[rows // 2, c] - want) < 1e-5


def test_mismatch_rejected(L):
    with pytest.raises(L.LithoError):
        L.LevelSetUtils.evolve_normal_WENO_godunov(np.zeros((5, 7)), np.zeros((5, 6)), 1.0, 1.0)
    with pytest.raises(L.LithoError):
        L.LevelSetUtils.evolve_normal_WENO_godunov(np.zeros((5, 7)), np.zeros((5, 7)), 1.0, 0.0)


def test_circle_symmetry(L):
    size, radius = 33, 10.0
    cc = 0.5 * (size - 1)
    y, x = np.mgrid[0:size, 0:size].astype(np.float64)
    phi = radius - np.hypot(x - cc, y - cc)
    d = cpu(L.LevelSetUtils.evolve_normal_WENO_godunov(phi, np.ones_like(phi), 1.0, 1.0).delta)
    ref, _, _ = lo.evolve_normal_weno_godunov(phi, np.ones_like(phi), 1.0, 1.0)
    band = np.abs(phi) <= 3.0
    m = 4
    err = 0.0
    for i in range(m, size - m):
        for j in range(m, size - m):
            if band[i, j]:
                err = max(err, abs(d[i, j] - d[i, size - 1 - j]), abs(d[i, j] - d[size - 1 - i, j]))
    assert err < 1e-5
    assert rel_max(d, ref) < 1e-5


def test_fixture_levelset(L):
    z = np.load(os.path.join(GOLDEN, "levelset_40x37.npz"))
    phi, vn = z["phi"], z["vn"]
    dx, dy, cfl, b = float(z["dx"]), float(z["dy"]), float(z["cfl"]), float(z["b"])
    e = L.LevelSetUtils.evolve_normal_WENO_godunov(phi, vn, dy, dx)
    assert rel_max(cpu(e.delta), z["delta"]) < 1e-5
    assert rel_max(cpu(e.H1_abs), z["habs"]) < 1e-6
    assert rel_max(cpu(L.LevelSetUtils.evolve_kappa(phi, dx, dy, b)), z["kappa"]) < 1e-5
    normal, dt = L.LevelSetUtils.evolution_term(phi, vn, dx, dy, cfl, b)
    assert rel_max(cpu(normal), z["normal"]) < 1e-5
    assert abs(dt - float(z["dt"])) < 1e-6 * float(z["dt"])
    nxt, mask, dt2 = L.LevelSetUtils.rk2_update(phi, vn, dx, dy, cfl, b)
    assert rel_max(cpu(nxt), z["phi_next"]) < 1e-5
    assert np.array_equal(cpu(mask), (cpu(nxt) >= 0).astype(np.float64))


@pytest.mark.parametrize("shape", [(3, 3), (7, 5), (257, 300), (1024, 1024)])
def test_random_fields_match_oracle(L, shape):
    rows, cols = shape
    rng = np.random.default_rng(rows * 7 + cols)
    yy, xx = np.mgrid[0:rows, 0:cols].astype(np.float64)
    phi = 20.0 * np.sin(0.05 * xx + 0.3) * np.cos(0.043 * yy) + rng.standard_normal((rows, cols)) * 0.5
    vn = rng.standard_normal((rows, cols))
    dx, dy, cfl, b = 2.0, 1.5, 0.5, 0.01
    ref_n, ref_dt = lo.evolution_term(phi, vn, dx, dy, cfl, b)
    got_n, got_dt = L.LevelSetUtils.evolution_term(phi, vn, dx, dy, cfl, b)
    assert rel_max(cpu(got_n), ref_n) < 2e-5
    assert abs(got_dt - ref_dt) < 1e-6 * ref_dt
    ref_next, _ = lo.lsm_rk2_update(phi, vn, dx, dy, cfl, b)
    got_next, _, _ = L.LevelSetUtils.rk2_update(phi, vn, dx, dy, cfl, b)
    assert rel_max(cpu(got_next), ref_next) < 2e-5


def test_flat_field_is_zero(L):
    """All-zero differences: the reference's eps floor gives exactly 0 (no NaN in FP32)."""
    phi = np.full((16, 16), 3.0)
    d = cpu(L.LevelSetUtils.evolve_normal_WENO_godunov(phi, np.ones_like(phi), 1.0, 1.0).delta)
    assert np.all(d == 0.0)
