"""SOCS kernel generation in the library (litho_socs_prepare / LithoPrepare) against
the FP64 oracle's restatement of LithoPrepare (oracle/optics_oracle.py, numpy SVD).

The SVD fixes each kernel only up to a phase, and a basis within each degenerate
eigenvalue, so the comparison is on observables (as the reference's own
tests/test_full_chip_imaging_compare.cpp:100 does): the eigenvalues sigma_k^2 (1e-9
relative to the largest), the source-weight sum, and the aerial image of a mask
imaged with the library's kernels against the oracle's image with its own kernels,
with K cut between two distinct eigenvalues (FP32 path: 1e-5 of the peak; split-BF16:
1e-4). Cases: the reference tests' optics (64^2 and 65^2 at 4 nm, full and compact
support), a compact 256^2 grid at 8 nm with 24 kernels on the tensor-core path, and
Fringe aberrations (Z4, Z7, Z9).
"""
import importlib

import numpy as np
import pytest

from oracle import imaging_oracle as io
from oracle import optics_oracle as oo

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

OPTICS = dict(wavelength=193.0, na=1.35, sigma_in=0.6, sigma_out=0.9)


@pytest.fixture(scope="module")
def L():
    p = importlib.import_module("c-version-lithography_b200")
    assert torch.cuda.is_available()
    p.load_library()
    return p


def cut_at_gap(ev, kmax):
    """The largest K <= kmax with sigma_K^2 distinct from sigma_{K+1}^2."""
    for k in range(min(kmax, len(ev)), 0, -1):
        if k == len(ev) or abs(ev[k - 1] - ev[k]) > 1e-6 * ev[0]:
            return k
    return 1


@pytest.mark.parametrize("N,px,compact,prec,aberr", [
    (64, 4.0, False, "fp32", None),
    (65, 4.0, False, "fp32", None),
    (64, 4.0, True, "fp32", None),
    (64, 4.0, True, "fp32", {4: 0.05, 7: -0.03, 9: 0.02}),
    (256, 8.0, True, "bf16x3", None),
])
def test_socs_prepare_matches_oracle(L, N, px, compact, prec, aberr):
    ref = oo.prepare(N, px, OPTICS["wavelength"], OPTICS["na"], OPTICS["sigma_in"],
                     OPTICS["sigma_out"], use_socs=True, compact=compact, num_socs=0,
                     aberrations=aberr)
    ev_ref = np.asarray(ref.eigenvalues)
    K = cut_at_gap(ev_ref, 24 if N > 128 else len(ev_ref))
    ctx = L.Context()
    ctx.set_precision(prec)
    prep = L.LithoPrepare(N, px, OPTICS["wavelength"], OPTICS["na"], OPTICS["sigma_in"],
                          OPTICS["sigma_out"], num_socs=K, compact=compact, aberrations=aberr,
                          ctx=ctx)
    info = prep.info
    assert info["K"] == K and info["Ns"] == len(ref.source_ws)
    assert abs(prep.source_ws_sum - float(np.sum(ref.source_ws))) <= 1e-12 * prep.source_ws_sum
    dev = float(np.max(np.abs(prep.eigenvalues - ev_ref[:K]))) / ev_ref[0]
    # aerial image: library kernels through the library vs oracle kernels through the oracle
    rng = np.random.default_rng(N)
    mask = (rng.random((N, N)) > 0.6).astype(np.float64)
    oc = io.OracleCache(N=N, kernels=ref.kernels[:K], source_ws=ref.source_ws,
                        eigenvalues=tuple(ev_ref[:K]))
    a_ref, _, _ = io.imaging_compute(mask, oc, 0.25, 50.0, keep_fields=False)
    a = L.Imaging(prep.cache).compute(mask, 0.25, 50.0).aerial_image.double().cpu().numpy()
    di = float(np.max(np.abs(a - a_ref)) / np.max(a_ref))
    ctx.close()
    print(f"\n{N}^2 {px} nm compact={compact} {prec} aberr={bool(aberr)}: Ns {info['Ns']}, K {K}, "
          f"band {info['Nr']}x{info['Nc']}, max|d sigma^2|/sigma_1^2 {dev:.1e}, "
          f"max|dI|/max I {di:.1e}, energy {info['energy_captured']:.4f}")
    assert dev <= 1e-9
    assert di <= (1e-5 if prec == "fp32" else 1e-4)


def test_socs_prepare_rejects_bad_optics(L):
    with pytest.raises(L.LithoError):
        L.LithoPrepare(64, 4.0, 193.0, 1.35, 0.9, 0.6)          # sigma_in >= sigma_out
    with pytest.raises(L.LithoError):
        L.LithoPrepare(64, -4.0, 193.0, 1.35, 0.6, 0.9)


def test_ctm_evaluation_on_generated_kernels(L):
    """A CTM evaluation on kernels the library generated (no oracle kernels anywhere),
    checked against the oracle evaluating with the same kernels."""
    N = 128
    prep = L.LithoPrepare(N, 8.0, 193.0, 1.35, 0.6, 0.9, num_socs=12, compact=True)
    target = np.zeros((N, N))
    target[40:88, 50:70] = 1.0
    theta = io.initialize_theta(target)
    dense = np.zeros((prep.info["K"], N, N), dtype=np.complex128)
    rows = (prep.info["row0"] + np.arange(prep.info["Nr"])) % N
    cols = (prep.info["col0"] + np.arange(prep.info["Nc"])) % N
    dense[:, rows[:, None], cols[None, :]] = prep.band_kernels
    oc = io.OracleCache(N=N, kernels=list(dense), source_ws=np.array([prep.source_ws_sum]),
                        eigenvalues=tuple(prep.eigenvalues))
    ref = io.ctm_evaluate(theta, target, oc, 0.25, 50.0)
    opt = L.CTMOptimizer(prep.cache, target, 0.25, 50.0, iterations=1)
    loss, g, _ = opt.evaluate(torch.tensor(theta, dtype=torch.float32, device="cuda"))
    gd = g.double().cpu().numpy()
    assert abs(loss - ref["loss"]) <= 1e-5 * ref["loss"]
    assert np.linalg.norm(gd - ref["grad_theta"]) <= 1e-4 * np.linalg.norm(ref["grad_theta"])
