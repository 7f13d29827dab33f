"""A compiled C++ consumer of the C ABI (tests/abi_consumer/consumer.cpp).

g++ builds it against include/litho_b200.h and links liblitho_b200.so, as a shim in the
reference code base would; gcc compiles the header as C (tests/abi_consumer/
header_check.c, which binds entry points to function pointers of their declared types).
The library itself includes the header in abi.cu, so a definition whose signature
differed from its declaration would not compile. On the CPU the consumer must build,
link and report the missing GPU with status exit 3; on a GPU its imaging, PE gradient,
CTM objective and RK2 level-set step must equal the package's ctypes calls on the same
inputs bit for bit, a NaN mask must come back as LITHO_ERR_NONFINITE, and the aerial
image must match the FP64 oracle to 1e-5 of its peak.
"""
import importlib
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "abi_consumer")
LIBDIR = os.path.join(ROOT, "c-version-lithography_b200")
CUDA = "/usr/local/cuda"


def build(tmp_path):
    if not shutil.which("g++") or not os.path.exists(os.path.join(LIBDIR, "liblitho_b200.so")):
        pytest.skip("g++ or the built library is missing")
    exe = str(tmp_path / "consumer")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror",
                    f"-I{ROOT}/include", f"-I{CUDA}/include", os.path.join(SRC, "consumer.cpp"),
                    f"-L{LIBDIR}", "-llitho_b200", f"-L{CUDA}/lib64", "-lcudart",
                    f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", f"-I{ROOT}/include", "-c",
                    os.path.join(SRC, "header_check.c"), "-o", str(tmp_path / "hc.o")], check=True)
    return exe


def test_consumer_builds_and_reports_a_missing_gpu(tmp_path):
    exe = build(tmp_path)
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the GPU test runs the consumer")
    r = subprocess.run([exe, str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 3, (r.returncode, r.stdout, r.stderr)


def read_output(path):
    with open(path, "rb") as f:
        N, K, nonfinite = np.frombuffer(f.read(12), dtype=np.int32)
        pe, loss, norm, dt = np.frombuffer(f.read(32), dtype=np.float64)
        ker = np.frombuffer(f.read(16 * K * N * N), dtype=np.complex128).reshape(K, N, N)
        names = ("target", "theta", "mask", "aerial", "wafer", "grad_mask", "grad_theta", "phi",
                 "phi_next")
        mats = {nm: np.frombuffer(f.read(4 * N * N), dtype=np.float32).reshape(N, N)
                for nm in names}
    return int(N), int(nonfinite), (pe, loss, norm, dt), ker, mats


@pytest.mark.gpu
def test_consumer_matches_the_package(tmp_path):
    torch = pytest.importorskip("torch")
    from oracle import imaging_oracle as io
    L = importlib.import_module("c-version-lithography_b200")
    exe = build(tmp_path)
    out = tmp_path / "out.bin"
    r = subprocess.run([exe, str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.stdout, r.stderr)
    N, nonfinite, (pe, loss, norm, dt), ker, m = read_output(out)
    assert nonfinite == 3
    w = np.array([0.7, 0.3])
    ctx = L.Context()
    cache = L.ImagingCache.from_kernels(ker, np.array([0.6, 0.6]), w, ctx=ctx)
    imaging = L.Imaging(cache)
    res = imaging.compute(m["mask"], 0.25, 50.0)
    assert np.array_equal(res.aerial_image.cpu().numpy(), m["aerial"])
    assert np.array_equal(res.wafer_image.cpu().numpy(), m["wafer"])
    grad = L.Gradient(cache, 0.25, 50.0)
    g = grad.pe_gradient(m["wafer"], m["target"], imaging.get_electric_field())
    assert np.array_equal(g.cpu().numpy(), m["grad_mask"]) and grad.last_loss == pe
    opt = L.CTMOptimizer(cache, m["target"], 0.25, 50.0, iterations=1)
    l2, gt, n2 = opt.evaluate(torch.tensor(m["theta"], device="cuda"))
    assert l2 == loss and n2 == norm
    assert np.array_equal(gt.cpu().numpy(), m["grad_theta"])
    nxt, _, dt2 = L.LevelSetUtils.rk2_update(m["phi"], m["grad_mask"], 1.0, 1.0, 0.5, 0.01, ctx=ctx)
    assert dt2 == dt and np.array_equal(nxt.cpu().numpy(), m["phi_next"])
    oc = io.OracleCache(N=N, kernels=list(ker), source_ws=np.array([0.6, 0.6]), eigenvalues=(0.7, 0.3))
    a_ref, _, _ = io.imaging_compute(m["mask"].astype(np.float64), oc, 0.25, 50.0)
    assert np.max(np.abs(m["aerial"] - a_ref)) <= 1e-5 * np.max(a_ref)
    ctx.close()
