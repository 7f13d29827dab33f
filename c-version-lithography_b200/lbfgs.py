"""L-BFGS driver of the CTM theta optimisation.

The reference calls LBFGS++ v0.4.0 (pinned commit c524a407, CMakeLists.txt:100-123)
with m = lbfgs_history_size, epsilon = gradient_tolerance (absolute),
epsilon_rel = 0 and max_iterations = iterations (CTM_Optimizer.cpp:189-227).
LBFGS++ is not available here, so this follows its published algorithm
(Nocedal & Wright, Numerical Optimization, Alg. 7.4 two-loop recursion and
Alg. 3.5/3.6 strong-Wolfe line search, ftol 1e-4, wolfe 0.9, first step
1/||g||, later steps 1): the vectors stay float32 on the device, every inner
product and the recursion scalars are float64.

Stopping rule, as LBFGS++: ||g|| <= epsilon before the first step (zero
iterations, one evaluation) or after any iteration, or ``max_iterations``
iterations done.
"""
from __future__ import annotations

import math


def _dot(a, b) -> float:
    return float((a.double() * b.double()).sum())


def minimize_lbfgs(fg, x, m=10, epsilon=1e-5, max_iterations=100, ftol=1e-4, wolfe=0.9,
                   max_linesearch=20, min_step=1e-20, max_step=1e20):
    """Minimise f from x. ``fg(x) -> (f, g, ||g||)``; returns (x, info)."""
    f, g, gnorm = fg(x)
    info = dict(iterations=0, evaluations=1, f=f, grad_norm=gnorm, reason="gradient tolerance")
    if gnorm <= epsilon:
        return x, info
    S, Y, RHO = [], [], []
    d = -g
    step = 1.0 / math.sqrt(_dot(d, d))
    k = 0
    while True:
        x_old, g_old, f_old = x, g, f
        dg0 = _dot(g, d)
        if dg0 >= 0:
            info["reason"] = "not a descent direction"
            break
        # Strong-Wolfe line search (bracketing + zoom by bisection/interpolation).
        lo, hi = 0.0, math.inf
        f_lo, dg_lo = f_old, dg0
        accepted = False
        for _ in range(max_linesearch):
            xt = x_old + step * d
            ft, gt, gn = fg(xt)
            info["evaluations"] += 1
            dgt = _dot(gt, d)
            if ft > f_old + ftol * step * dg0 or (lo > 0 and ft >= f_lo):
                hi = step
            else:
                if abs(dgt) <= -wolfe * dg0:
                    accepted = True
                    x, f, g, gnorm = xt, ft, gt, gn
                    break
                if dgt * (hi - lo if math.isfinite(hi) else 1.0) >= 0:
                    hi = lo
                lo, f_lo, dg_lo = step, ft, dgt
            if math.isfinite(hi):
                step = 0.5 * (lo + hi)
            else:
                step = min(2.0 * step, max_step)
            if step < min_step:
                break
        if not accepted:
            # Keep the best Armijo point found, as a failed search still moves.
            if lo > 0:
                x = x_old + lo * d
                f, g, gnorm = fg(x)
                info["evaluations"] += 1
            else:
                info["reason"] = "line search failed"
                break
        k += 1
        if gnorm <= epsilon:
            info["reason"] = "gradient tolerance"
            break
        if k >= max_iterations:
            info["reason"] = "maximum iterations"
            break
        s = x - x_old
        y = g - g_old
        sy = _dot(s, y)
        if sy > 1e-10 * _dot(y, y):
            if len(S) == m:
                S.pop(0); Y.pop(0); RHO.pop(0)
            S.append(s); Y.append(y); RHO.append(1.0 / sy)
        # Two-loop recursion (FP64 scalars).
        q = g.clone()
        alphas = []
        for s_i, y_i, r_i in zip(reversed(S), reversed(Y), reversed(RHO)):
            a = r_i * _dot(s_i, q)
            alphas.append(a)
            q = q - a * y_i
        if S:
            q = q * (_dot(S[-1], Y[-1]) / _dot(Y[-1], Y[-1]))
        for (s_i, y_i, r_i), a in zip(zip(S, Y, RHO), reversed(alphas)):
            b = r_i * _dot(y_i, q)
            q = q + (a - b) * s_i
        d = -q
        step = 1.0
    info.update(iterations=k, f=f, grad_norm=gnorm)
    return x, info
