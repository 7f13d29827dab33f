"""The Gram-form two-loop recursion of the L-BFGS driver equals the two loops over
vectors (Nocedal & Wright Alg. 7.4, as LBFGS++ runs them) on random FP64 data: the
direction -H g agrees to 1e-12 relative, for a full history, a partial one, slots in
ring order after wrap-around, and an empty history (-g)."""
import importlib

import numpy as np
import pytest


@pytest.fixture(scope="module")
def lb():
    return importlib.import_module("c-version-lithography_b200.lbfgs")


def two_loop_vectors(S, Y, g):
    q = g.copy()
    rho = [1.0 / (s @ y) for s, y in zip(S, Y)]
    alphas = []
    for s, y, r in zip(reversed(S), reversed(Y), reversed(rho)):
        a = r * (s @ q)
        alphas.append(a)
        q = q - a * y
    if S:
        q = q * ((S[-1] @ Y[-1]) / (Y[-1] @ Y[-1]))
    for (s, y, r), a in zip(zip(S, Y, rho), reversed(alphas)):
        b = r * (y @ q)
        q = q + (a - b) * s
    return -q


@pytest.mark.parametrize("m,count,first_slot", [(10, 10, 0), (10, 4, 0), (5, 5, 3), (6, 0, 0)])
def test_gram_two_loop_equals_vector_loops(lb, m, count, first_slot):
    rng = np.random.default_rng(m * 100 + count)
    n = 400
    g = rng.standard_normal(n)
    S, Y = [], []
    for _ in range(count):
        s = rng.standard_normal(n)
        y = s + 0.3 * rng.standard_normal(n)       # s . y > 0
        S.append(s); Y.append(y)
    order = [(first_slot + i) % m for i in range(count)]     # oldest first, ring slots
    rows = np.zeros((2 * m, n))
    for slot, s, y in zip(order, S, Y):
        rows[slot], rows[m + slot] = s, y
    SY = rows[:m] @ rows[m:].T
    YY = rows[m:] @ rows[m:].T
    rho = np.array([1.0 / SY[i, i] if SY[i, i] != 0 else 0.0 for i in range(m)])
    gp = rows @ g
    coef, gamma = lb.two_loop_coefficients(order, SY, YY, rho, gp, m)
    d = -gamma * g + coef @ rows
    ref = two_loop_vectors(S, Y, g)
    assert np.linalg.norm(d - ref) <= 1e-12 * np.linalg.norm(ref)
