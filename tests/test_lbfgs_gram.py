"""The Gram-form two-loop recursion of the L-BFGS driver equals the two loops over
vectors (Nocedal & Wright Alg. 7.4, as LBFGS++ runs them) on random FP64 data: the
direction -H g agrees to 1e-12 relative, for a full history, a partial one, slots in
ring order after wrap-around, and an empty history (-g). The driver itself runs on CPU
tensors through an FP64 stand-in for the library's vector kernels: it converges on a
quadratic, and its two failure cases raise LineSearchError where LBFGS++ throws."""
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


class _CpuVectors:
    """The driver's vector operations in FP64 on CPU tensors (the library kernels'
    contract: FP64 inner products, out = cv v + sum_j coef[j] rows[j])."""

    def __init__(self, flip_direction=False):
        self.flip = flip_direction

    def dots(self, rows, k, v):
        return (rows[:k].double() @ v.reshape(-1).double()).numpy()

    def dots3(self, rows, k, vs):
        return np.stack([self.dots(rows, k, v) for v in vs])

    def dot(self, a, b):
        return float(a.reshape(-1).double() @ b.reshape(-1).double())

    def combine(self, rows, coef, v, cv, out):
        import torch
        r = cv * v.double() + torch.from_numpy(np.asarray(coef)) @ rows.double()
        out.copy_((-r if self.flip else r).to(out.dtype))
        return out


def _quadratic(sign_error=False):
    import torch
    scale = torch.linspace(1.0, 4.0, 64, dtype=torch.float32)

    def fg(x):
        g = 2.0 * scale * x
        if sign_error:            # a gradient of the wrong sign: no step lowers f
            g = -g
        return float((scale * x * x).sum()), g, float(g.norm())
    return fg


def test_lbfgs_converges_on_a_quadratic(lb):
    import torch
    x0 = torch.linspace(-1.0, 1.0, 64, dtype=torch.float32)
    x, info = lb.minimize_lbfgs(_quadratic(), x0.clone(), m=5, epsilon=1e-4, max_iterations=50,
                                dev=_CpuVectors())
    assert info["reason"] == "gradient tolerance" and float(x.abs().max()) < 1e-4


def test_lbfgs_line_search_failure_raises_like_lbfgspp(lb):
    """LBFGS++ throws std::runtime_error when its line search runs out of trials; the
    reference lets it propagate. strict=False stops with the reason instead."""
    import torch
    x0 = torch.linspace(-1.0, 1.0, 64, dtype=torch.float32)
    with pytest.raises(lb.LineSearchError, match="maximum number of iterations"):
        lb.minimize_lbfgs(_quadratic(sign_error=True), x0.clone(), dev=_CpuVectors())
    x, info = lb.minimize_lbfgs(_quadratic(sign_error=True), x0.clone(), strict=False,
                                dev=_CpuVectors())
    assert info["reason"] == "line search failed" and torch.equal(x, x0)


def test_lbfgs_ascent_direction_raises_like_lbfgspp(lb):
    """A two-loop direction that does not descend: LBFGS++ throws "the moving direction
    increases the objective function value"; strict=False stops after the first step."""
    import torch
    x0 = torch.linspace(-1.0, 1.0, 64, dtype=torch.float32)
    with pytest.raises(lb.LineSearchError, match="increases the objective"):
        lb.minimize_lbfgs(_quadratic(), x0.clone(), m=5, dev=_CpuVectors(flip_direction=True))
    _, info = lb.minimize_lbfgs(_quadratic(), x0.clone(), m=5, strict=False,
                                dev=_CpuVectors(flip_direction=True))
    assert info["reason"] == "not a descent direction" and info["iterations"] == 1
