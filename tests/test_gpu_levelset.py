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


@pytest.mark.parametrize("shape", [(7, 9), (64, 64), (65, 200), (517, 300), (130, 900), (90, 3100),
                                   (16, 6000), (20, 9000), (12, 17000), (2048, 2048)])
def test_reinit_sdf_matches_opencv(L, shape):
    """reinit_sdf (level_set_utils.cpp:290-319) against cv2.distanceTransform(DIST_L2, 5).

    OpenCV accumulates the chamfer sums in float32 along its raster order; the
    device evaluates the same minimum exactly, so values agree to float
    rounding: 1e-5 relative (plus 1e-6 absolute) per pixel. The row lengths cover
    the three CTA sizes of the transform (128, 256 and 1024 threads), with the
    classification held in registers and, for rows longer than 8192, read directly.
    """
    rows, cols = shape
    rng = np.random.default_rng(rows + cols)
    yy, xx = np.mgrid[0:rows, 0:cols].astype(np.float64)
    phi = np.sin(0.07 * xx + 0.3) * np.cos(0.05 * yy) + 0.3 * rng.standard_normal((rows, cols))
    phi[rows // 3, :] = 0.0  # exact zeros count as outside (phi > 0 is inside)
    ref = lo.reinit_sdf(phi, 2.0, 2.0)
    got, mask = L.LevelSetUtils.reinit_sdf(phi, 2.0, 2.0, with_mask=True)
    got = cpu(got)
    assert np.all(np.abs(got - ref) <= 1e-5 * np.abs(ref) + 1e-6)
    assert np.array_equal(cpu(mask), (got >= 0).astype(np.float64))


def test_reinit_sdf_of_binary_mask(L):
    """The LSM initialisation reinit_sdf(mask - 0.5) (LSM_Optimizer.cpp:62) on a target."""
    wl = importlib.import_module("c-version-lithography_b200.workloads")
    target = wl.manhattan_target(512, 10, seed=4)
    ref = lo.reinit_sdf(target - 0.5, 2.0, 2.0)
    got = cpu(L.LevelSetUtils.reinit_sdf(target - 0.5, 2.0, 2.0))
    assert np.all(np.abs(got - ref) <= 1e-5 * np.abs(ref) + 1e-6)


def test_reinit_sdf_batch(L):
    """reinit_sdf_batch with level 0.5 on binary masks equals reinit_sdf(mask - 0.5) of
    each image (one launch for the batch; the printed mask is sdf >= 0)."""
    torch = pytest.importorskip("torch")
    wl = importlib.import_module("c-version-lithography_b200.workloads")
    masks = np.stack([wl.manhattan_target(300, 6, seed=s) for s in range(3)])
    m = torch.tensor(masks, dtype=torch.float32, device="cuda")
    mask_out = torch.empty_like(m)
    out = L.LevelSetUtils.reinit_sdf_batch(m, 2.0, 2.0, level=0.5, mask_out=mask_out)
    for b in range(3):
        ref = L.LevelSetUtils.reinit_sdf(m[b] - 0.5, 2.0, 2.0)
        assert torch.equal(out[b], ref), b
        assert torch.equal(mask_out[b], (ref >= 0).float()), b
        oc = lo.reinit_sdf(masks[b] - 0.5, 2.0, 2.0)
        assert np.all(np.abs(cpu(out[b]) - oc) <= 1e-5 * np.abs(oc) + 1e-6)
    with pytest.raises(L.LithoError):
        L.LevelSetUtils.reinit_sdf_batch(m, 2.0, 2.0, out=m)


def test_reinit_without_boundary(L):
    """No feature pixel: OpenCV returns FLT_MAX; the sign follows inside/outside."""
    got = cpu(L.LevelSetUtils.reinit_sdf(np.full((8, 8), 2.0), 1.0, 1.0))
    assert np.all(got == np.float32(3.4028235e38))
    got = cpu(L.LevelSetUtils.reinit_sdf(np.full((8, 8), -2.0), 1.0, 1.0))
    assert np.all(got == -np.float32(3.4028235e38))


def test_lsm_optimizer_tracks_oracle(L):
    """LSM_Optimizer::optimize (LSM_Optimizer.cpp:60-149) for 6 iterations on real optics,
    against the FP64 oracle loop: PE history within 1e-3 relative, printed masks
    equal except pixels whose oracle phi is within 1e-3 of zero."""
    from oracle import imaging_oracle as io
    from oracle import optics_oracle as oo
    n, dx = 64, 4.0
    oc = oo.prepare(n, dx, 193.0, 1.35, 0.6, 0.9, use_socs=True)
    target = np.zeros((n, n)); target[23:42, 23:42] = 1.0
    mask0 = target.copy(); mask0[20:45, 26:38] = 1.0
    thr, alpha, cfl, b = 0.25, 85.0, 0.5, 0.01
    # Oracle loop (LSM_Optimizer.cpp:60-128), penalty off.
    phi = lo.reinit_sdf(mask0 - 0.5, dx, dx)
    temp = mask0.copy(); hist = []; phis = []
    for i in range(6):
        _, w, E = io.imaging_compute(temp, oc, thr, alpha)
        hist.append(io.pe_loss_with_penalty(w, target, 1.0, 0.01))
        gm = io.pe_gradient(w, target, E, oc, alpha)
        phi, _ = lo.lsm_rk2_update(phi, gm, dx, dx, cfl, b)
        phis.append(phi.copy())
        temp = (phi >= 0).astype(np.float64)
    cache = L.ImagingCache.from_kernels(np.stack(oc.kernels), oc.source_ws, oc.eigenvalues)
    lsm = L.LSMOptimizer(cache, target, thr, alpha, dx, dx, cfl, b, iterations=6)
    res = lsm.optimize(mask0)
    for a, r in zip(lsm.error_history, hist):
        assert abs(a - r) <= 1e-3 * r, (lsm.error_history, hist)
    assert np.allclose(cpu(res.initial_sdf), lo.reinit_sdf(mask0 - 0.5, dx, dx), rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("shape,scale", [((64, 80), 4), ((37, 29), 3), ((128, 128), 4)])
def test_render_levelset_mask_matches_cv2(shape, scale):
    """render_levelset_mask: Binary bit-exact; Gray against the cv2 INTER_LINEAR upsampling
    the reference calls. cv2's float resize differs from a plain FP32 bilinear product sum
    in the last bit, so a subpixel whose interpolated phi is within rounding of 0 may be
    counted on the other side: coverage may differ by 1/scale^2 at a few pixels."""
    import importlib
    Lm = importlib.import_module("c-version-lithography_b200")
    from oracle import levelset_oracle as lo
    rng = np.random.default_rng(shape[0] + scale)
    yy, xx = np.mgrid[0:shape[0], 0:shape[1]].astype(np.float64)
    phi = (12.0 - np.hypot(yy - shape[0] / 2, xx - shape[1] / 3) + 2.0 * np.sin(xx / 5.0)
           + 0.3 * rng.standard_normal(shape)).astype(np.float32)
    t = torch.from_numpy(phi).cuda()
    b = Lm.render_levelset_mask(t, "Binary").cpu().numpy()
    assert np.array_equal(b, lo.render_levelset_mask(phi, "Binary"))
    g = Lm.render_levelset_mask(t, "Gray", scale).cpu().numpy().astype(np.float64)
    ref = lo.render_levelset_mask(phi, "Gray", scale)
    d = np.abs(g - ref)          # coverage is k / scale^2, stored in float32
    assert d.max() <= 1.0 / scale ** 2 + 1e-6
    assert (d > 1e-6).mean() <= 0.005
    assert g.min() >= 0.0 and g.max() <= 1.0
