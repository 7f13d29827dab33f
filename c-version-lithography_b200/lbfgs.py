"""L-BFGS driver of the CTM theta optimisation.

The reference calls LBFGS++ v0.4.0 (pinned commit c524a407, CMakeLists.txt:100-123)
with m = lbfgs_history_size, epsilon = gradient_tolerance (absolute),
epsilon_rel = 0 and max_iterations = iterations (CTM_Optimizer.cpp:189-227).
LBFGS++ is not available here, so this follows its published algorithm
(Nocedal & Wright, Numerical Optimization, Alg. 7.4 two-loop recursion and
Alg. 3.5/3.6 strong-Wolfe line search, ftol 1e-4, wolfe 0.9, first step
1/||g||, later steps 1): the vectors stay float32 on the device, every inner
product and the recursion scalars are float64.

The two-loop recursion is evaluated in its Gram form: every inner product it takes
is a combination of s_i . y_j, y_i . y_j, s_i . g and y_i . g, so the library keeps
the history pairs as rows of one device array, returns those inner products in one
pass over the rows (litho_lbfgs_dots, FP64 accumulation), the recursion's scalars
are formed on the host in FP64 exactly as the two loops form them, and one more pass
builds the direction -H g (litho_lbfgs_combine). Per iteration that is one launch
that reads the history once for the new pair's two vectors and the new gradient
together (litho_lbfgs_dots3; those three vectors are read once per group of 8 history
rows) and one for the direction, instead of one pass per inner product.

Stopping rule, as LBFGS++: ||g|| <= epsilon before the first step (zero
iterations, one evaluation) or after any iteration, or ``max_iterations``
iterations done.

Failures, as LBFGS++ (whose std::runtime_error the reference does not catch, so the
run aborts): a search direction that does not descend raises LineSearchError("the
moving direction increases the objective function value"), and a line search that
ends without a strong-Wolfe point raises LineSearchError("the line search routine
reached the maximum number of iterations"). With strict=False the driver instead
moves to the best Armijo point the failed search found (or stops, with the reason in
``info["reason"]``, when it found none), which a long fixed-length benchmark run
uses so that a stall near the optimum does not end it.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np


class LineSearchError(RuntimeError):
    """A failed L-BFGS step (LBFGS++ throws std::runtime_error in these cases)."""


class _Device:
    """The library's L-BFGS vector kernels on float32 CUDA tensors of n elements."""

    def __init__(self, ctx, n: int):
        self.ctx, self.n = ctx, n

    def dots(self, rows, k: int, v) -> np.ndarray:
        """rows[0..k) . v in FP64; rows: a (>= k, n) contiguous float32 tensor."""
        out = np.empty(k, dtype=np.float64)
        self.ctx._check(self.ctx.lib.litho_lbfgs_dots(
            self.ctx.handle, k, self.n, ctypes.c_void_p(rows.data_ptr()), self.n,
            ctypes.c_void_p(v.data_ptr()), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def dots3(self, rows, k: int, vs) -> np.ndarray:
        """rows[0..k) . v for up to three vectors in one pass: an (len(vs), k) array."""
        ptr = [ctypes.c_void_p(v.data_ptr()) for v in vs] + [None] * (3 - len(vs))
        out = np.empty(len(vs) * k, dtype=np.float64)
        self.ctx._check(self.ctx.lib.litho_lbfgs_dots3(
            self.ctx.handle, k, self.n, ctypes.c_void_p(rows.data_ptr()), self.n, *ptr,
            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out.reshape(len(vs), k)

    def dot(self, a, b) -> float:
        return float(self.dots(a, 1, b)[0])

    def combine(self, rows, coef: np.ndarray, v, cv: float, out):
        """out = cv v + sum_j coef[j] rows[j]."""
        c = np.ascontiguousarray(coef, dtype=np.float64)
        self.ctx._check(self.ctx.lib.litho_lbfgs_combine(
            self.ctx.handle, len(c), self.n, ctypes.c_void_p(rows.data_ptr()), self.n,
            c.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.c_void_p(v.data_ptr()),
            float(cv), ctypes.c_void_p(out.data_ptr())))
        return out


def two_loop_coefficients(order, SY, YY, rho, gp, m):
    """The two-loop recursion (Nocedal & Wright Alg. 7.4) in Gram form, FP64.

    order: history slots, oldest first; SY[a, b] = s_a . y_b, YY[a, b] = y_a . y_b,
    rho[a] = 1 / (s_a . y_a); gp = (s_0 . g .. s_{m-1} . g, y_0 . g .. y_{m-1} . g).
    Returns (coef, gamma) with -H g = -gamma g + sum_j coef[j] s_j + coef[m + j] y_j:
    the same alpha_i = rho_i s_i . q (newest first) and beta_i = rho_i y_i . r (oldest
    first) as the loops over vectors, with q and r expanded on the basis {g, s, y}."""
    alpha, beta = {}, {}
    done = []
    for i in reversed(order):                       # q = g - sum_{newer j} alpha_j y_j
        alpha[i] = rho[i] * (gp[i] - sum(alpha[j] * SY[i, j] for j in done))
        done.append(i)
    gamma = SY[order[-1], order[-1]] / YY[order[-1], order[-1]] if order else 1.0
    done = []
    for i in order:                                 # r = gamma q + sum_{older p} (a_p - b_p) s_p
        yr = gamma * (gp[m + i] - sum(alpha[j] * YY[i, j] for j in order))
        yr += sum((alpha[p] - beta[p]) * SY[p, i] for p in done)
        beta[i] = rho[i] * yr
        done.append(i)
    coef = np.zeros(2 * m)
    for j in order:
        coef[j] = -(alpha[j] - beta[j])
        coef[m + j] = gamma * alpha[j]
    return coef, gamma


def minimize_lbfgs(fg, x, m=10, epsilon=1e-5, max_iterations=100, ftol=1e-4, wolfe=0.9,
                   max_linesearch=20, min_step=1e-20, max_step=1e20, ctx=None, strict=True,
                   dev=None):
    """Minimise f from x (a contiguous float32 CUDA tensor). ``fg(x) -> (f, g, ||g||)``;
    returns (x, info). ctx: the library context whose stream the vectors live on.
    strict: raise LineSearchError where LBFGS++ throws (see the module docstring).
    dev: the vector operations (default: the library's kernels on ctx)."""
    if dev is None:
        if ctx is None:
            from . import default_context
            ctx = default_context()
        dev = _Device(ctx, x.numel())
    import torch
    f, g, gnorm = fg(x)
    info = dict(iterations=0, evaluations=1, f=f, grad_norm=gnorm, reason="gradient tolerance")
    if gnorm <= epsilon:
        return x, info
    n = x.numel()
    rows = torch.zeros((2 * m, n), dtype=torch.float32, device=x.device)   # s slots | y slots
    pair = torch.empty((2, n), dtype=torch.float32, device=x.device)        # new s, y
    # Every trial point is formed in the same buffer, so that the evaluations of a
    # line search see the same input (the library replays its captured chain).
    trial = torch.empty_like(x)
    SY = np.zeros((m, m))   # SY[a, b] = s_a . y_b  (slots)
    YY = np.zeros((m, m))   # YY[a, b] = y_a . y_b
    rho = np.zeros(m)
    order: list = []        # slots, oldest first
    d = -g
    step = 1.0 / math.sqrt(dev.dot(d, d))
    k = 0
    while True:
        x_old, g_old, f_old = x, g, f
        dg0 = dev.dot(g, d)
        if dg0 >= 0:
            if strict:
                raise LineSearchError("the moving direction increases the objective function value")
            info["reason"] = "not a descent direction"
            break
        # Strong-Wolfe line search (bracketing + zoom by bisection/interpolation).
        lo, hi = 0.0, math.inf
        f_lo, dg_lo = f_old, dg0
        accepted = False
        for _ in range(max_linesearch):
            torch.add(x_old, d, alpha=step, out=trial)
            ft, gt, gn = fg(trial)
            info["evaluations"] += 1
            dgt = dev.dot(gt, d)
            if ft > f_old + ftol * step * dg0 or (lo > 0 and ft >= f_lo):
                hi = step
            else:
                if abs(dgt) <= -wolfe * dg0:
                    accepted = True
                    x, f, g, gnorm = trial.clone(), ft, gt, gn
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
            if strict:
                raise LineSearchError("the line search routine reached the maximum number of "
                                      "iterations")
            # Keep the best Armijo point found, as a failed search still moves.
            if lo > 0:
                torch.add(x_old, d, alpha=lo, out=trial)
                f, g, gnorm = fg(trial)
                x = trial.clone()
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
        torch.sub(x.view(-1), x_old.view(-1), out=pair[0])
        torch.sub(g.view(-1), g_old.view(-1), out=pair[1])
        sy, yy = dev.dots(pair, 2, pair[1])
        gp = np.zeros(2 * m)
        if sy > 1e-10 * yy:
            if len(order) == m:
                order.pop(0)
            slot = next(i for i in range(m) if i not in order)
            rows[slot].copy_(pair[0])
            rows[m + slot].copy_(pair[1])
            order.append(slot)
            # s . s_b | s . y_b, y . s_b | y . y_b and the new gradient's, in one pass
            ds, dy, gp = dev.dots3(rows, 2 * m, (pair[0], pair[1], g.view(-1)))
            for b in order:
                SY[slot, b] = ds[m + b]
                SY[b, slot] = dy[b]
                YY[slot, b] = YY[b, slot] = dy[m + b]
            rho[slot] = 1.0 / sy
        elif order:
            gp = dev.dots(rows, 2 * m, g.view(-1))
        coef, gamma = two_loop_coefficients(order, SY, YY, rho, gp, m)
        d = dev.combine(rows, coef, g.view(-1), -gamma, torch.empty_like(g)).view_as(g)
        step = 1.0
    info.update(iterations=k, f=f, grad_norm=gnorm)
    return x, info
