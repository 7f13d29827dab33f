"""The L-BFGS vector kernels on the GPU: litho_lbfgs_dots (FP64-accumulated inner
products of one vector with up to 64 stored rows in one pass) against NumPy FP64 to
1e-11 of the sum of the products' magnitudes, litho_lbfgs_combine against NumPy to
FP32 rounding, and the argument errors."""
import importlib

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def L():
    p = importlib.import_module("c-version-lithography_b200")
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    p.load_library()
    return p


@pytest.fixture(scope="module")
def LB():
    return importlib.import_module("c-version-lithography_b200.lbfgs")


@pytest.mark.parametrize("k,n", [(1, 1000), (5, 4097), (20, 300_000), (64, 70_000)])
def test_lbfgs_dots_and_combine(L, LB, k, n):
    ctx = L.default_context()
    rng = np.random.default_rng(k + n)
    rows = rng.standard_normal((k, n)).astype(np.float32)
    v = rng.standard_normal(n).astype(np.float32)
    R = torch.from_numpy(rows).cuda()
    V = torch.from_numpy(v).cuda()
    dev = LB._Device(ctx, n)
    got = dev.dots(R, k, V)
    ref = rows.astype(np.float64) @ v.astype(np.float64)
    assert np.all(np.abs(got - ref) <= 1e-11 * np.abs(rows.astype(np.float64) * v).sum(axis=1))
    coef = rng.standard_normal(k)
    out = dev.combine(R, coef, V, -0.75, torch.empty_like(V))
    want = -0.75 * v.astype(np.float64) + coef @ rows.astype(np.float64)
    assert np.allclose(out.cpu().numpy(), want, rtol=1e-6, atol=1e-6 * np.abs(want).max())


def test_lbfgs_errors(L):
    ctx = L.default_context()
    import ctypes
    V = torch.ones(16, device="cuda")
    buf = np.zeros(65)
    p = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    lib = ctx.lib
    assert lib.litho_lbfgs_dots(ctx.handle, 0, 16, ctypes.c_void_p(V.data_ptr()), 16,
                                ctypes.c_void_p(V.data_ptr()), p) != 0           # k = 0
    assert lib.litho_lbfgs_dots(ctx.handle, 65, 16, ctypes.c_void_p(V.data_ptr()), 16,
                                ctypes.c_void_p(V.data_ptr()), p) != 0           # k > 64
    assert lib.litho_lbfgs_combine(ctx.handle, 1, 16, ctypes.c_void_p(V.data_ptr()), 16, p,
                                   ctypes.c_void_p(V.data_ptr()), 1.0,
                                   ctypes.c_void_p(V.data_ptr())) != 0          # out aliases v
    buf[0] = np.nan
    W = torch.empty_like(V)
    assert lib.litho_lbfgs_combine(ctx.handle, 1, 16, ctypes.c_void_p(V.data_ptr()), 16, p,
                                   ctypes.c_void_p(V.data_ptr()), 1.0,
                                   ctypes.c_void_p(W.data_ptr())) != 0          # NaN coefficient


@pytest.mark.parametrize("nv", [1, 2, 3])
def test_lbfgs_dots3(L, LB, nv):
    """litho_lbfgs_dots3: the inner products of 20 rows with nv vectors in one pass
    equal those of litho_lbfgs_dots per vector (FP64 accumulation, same tolerance)."""
    ctx = L.default_context()
    rng = np.random.default_rng(nv)
    k, n = 20, 123_457
    rows = rng.standard_normal((k, n)).astype(np.float32)
    vs = [rng.standard_normal(n).astype(np.float32) for _ in range(nv)]
    R = torch.from_numpy(rows).cuda()
    Vs = [torch.from_numpy(v).cuda() for v in vs]
    got = LB._Device(ctx, n).dots3(R, k, Vs)
    r64 = rows.astype(np.float64)
    for i, v in enumerate(vs):
        ref = r64 @ v.astype(np.float64)
        assert np.all(np.abs(got[i] - ref) <= 1e-11 * np.abs(r64 * v).sum(axis=1)), i
