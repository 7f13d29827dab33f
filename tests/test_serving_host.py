"""Host logic of the tile server that needs no GPU: the seeded Poisson stream and the
per-solve memory estimate used for HBM-budget admission."""
import importlib

import numpy as np

S = importlib.import_module("c-version-lithography_b200.serving")


def test_poisson_arrivals_seeded_and_proportional():
    make = lambda N, rng: (np.zeros((N, N)), np.zeros((N, N)))
    a = S.poisson_arrivals(400.0, 2000, [256, 512, 1024, 2048], [4, 3, 2, 1], make, 20, seed=5)
    b = S.poisson_arrivals(400.0, 2000, [256, 512, 1024, 2048], [4, 3, 2, 1], make, 20, seed=5)
    assert [x[0] for x in a] == [x[0] for x in b]
    t = np.array([x[0] for x in a])
    assert np.all(np.diff(t) > 0)
    assert abs(t[-1] / len(t) - 1.0 / 400.0) < 0.1 / 400.0        # mean gap 1 / rate
    sizes = np.array([x[1].shape[0] for x in a])
    frac = [np.mean(sizes == n) for n in (256, 512, 1024, 2048)]
    assert np.allclose(frac, [0.4, 0.3, 0.2, 0.1], atol=0.04)
    assert all(x[3] == 20 for x in a)


def test_solve_bytes_scale():
    assert S.TileServer.solve_bytes(2048) == 4 * S.TileServer.solve_bytes(1024)
    # a 120 GB budget holds hundreds of 2048^2 solves
    assert 120e9 / S.TileServer.solve_bytes(2048) > 300
