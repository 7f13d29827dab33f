"""Generates the golden fixtures of tests/golden/ from the FP64 oracle.

Run from the repository root:  python tests/golden/make_golden.py
Each case stores its seeded inputs and the oracle's outputs (float64 where
small, float32 for the 128^2 band case). The optical kernels are rebuilt by the tests from the
same deterministic recipes (oracle.optics_oracle / workloads), so the fixtures
stay small; SVD phase freedom does not change any stored quantity.
"""
from __future__ import annotations

import importlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import imaging_oracle as io  # noqa: E402
from oracle import levelset_oracle as lo  # noqa: E402
from oracle import optics_oracle as oo  # noqa: E402

wl = importlib.import_module("c-version-lithography_b200.workloads")
OUT = os.path.dirname(os.path.abspath(__file__))


def ctm_case(name, cache, target, theta, thr, alpha, dtype=np.float64, penalty=None):
    r = io.ctm_evaluate(theta, target, cache, thr, alpha)
    extra = {}
    if penalty is not None:
        _, w, E = io.imaging_compute(io.theta_to_mask(theta), cache, thr, alpha)
        g = io.pe_gradient(w, target, E, cache, alpha, penalty=penalty[0], penalty_threshold=penalty[1])
        extra = dict(grad_mask_penalty=g.astype(dtype),
                     loss_penalty=io.pe_loss_with_penalty(w, target, penalty[0], penalty[1]))
    np.savez_compressed(os.path.join(OUT, name + ".npz"), theta=theta.astype(dtype),
                        target=target.astype(dtype), thr=thr, alpha=alpha,
                        aerial=r["aerial"].astype(dtype), wafer=r["wafer"].astype(dtype),
                        grad_mask=r["grad_mask"].astype(dtype),
                        grad_theta=r["grad_theta"].astype(dtype), loss=r["loss"],
                        grad_norm=r["grad_norm"], **extra)


def main():
    # Real optics of tests/test_ctm_optimizer.cpp:140-160 (64^2 and 65^2, 4 nm, annular 0.6-0.9).
    for n in (64, 65):
        cache = oo.prepare(n, 4.0, 193.0, 1.35, 0.6, 0.9, use_socs=True)
        target = np.zeros((n, n)); target[23:42, 23:42] = 1.0
        ctm_case(f"ctm_real_{n}", cache, target, io.initialize_theta(target), 0.25, 85.0,
                 penalty=(2.0, 0.01))
    # Synthetic smooth kernels of tests/test_micro_gradient_exchange.cpp:27-45 (full band).
    for n, socs in ((12, True), (13, False)):
        cache = oo.synthetic_gaussian_cache(n, socs)
        cache.source_ws = np.array([0.3, 0.9])
        y, x = np.mgrid[0:n, 0:n].astype(np.float64)
        mask = 0.43 + 0.12 * np.sin(0.31 * x + 0.27 * y) + 0.05 * np.cos(0.52 * x - 0.23 * y)
        theta = np.arccos(2.0 * mask - 1.0)
        target = (np.random.default_rng(n).random((n, n)) > 0.5).astype(np.float64)
        ctm_case(f"ctm_gauss_{n}_{'socs' if socs else 'abbe'}", cache, target, theta, 0.18, 8.0)
    # Benchmark-shaped band kernels (35 x 35, K = 24, ratio 0.8) at 128^2.
    band, r0, c0, w, wss = wl.synthetic_socs_band()
    cache = io.OracleCache(N=128, kernels=list(wl.band_to_dense(band, r0, c0, 128)),
                           source_ws=np.array([wss]), eigenvalues=tuple(w))
    target = wl.manhattan_target(128, 4, seed=7)
    ctm_case("ctm_band_128", cache, target, wl.theta_init_reference(target), 0.225, 50.0,
             dtype=np.float32)
    # Level set: random smooth phi and speed on a non-square grid.
    rng = np.random.default_rng(3)
    rows, cols = 40, 37
    yy, xx = np.mgrid[0:rows, 0:cols].astype(np.float64)
    phi = 6.0 - np.hypot(xx - 17.3, yy - 21.1) + 0.3 * np.sin(0.4 * xx) * np.cos(0.3 * yy)
    vn = 0.5 * np.sin(0.21 * xx + 0.13 * yy) + 0.05 * rng.standard_normal((rows, cols))
    dx, dy, cfl, b = 2.0, 2.0, 0.5, 0.01
    delta, h1, _ = lo.evolve_normal_weno_godunov(phi, vn, dy, dx)
    kap = lo.evolve_kappa(phi, dx, dy, b)
    normal, dt = lo.evolution_term(phi, vn, dx, dy, cfl, b)
    phi2, dt2 = lo.lsm_rk2_update(phi, vn, dx, dy, cfl, b)
    np.savez_compressed(os.path.join(OUT, "levelset_40x37.npz"), phi=phi, vn=vn, dx=dx, dy=dy,
                        cfl=cfl, b=b, delta=delta, habs=h1, kappa=kap, normal=normal, dt=dt,
                        phi_next=phi2)
    print("fixtures written to", OUT)


if __name__ == "__main__":
    main()
