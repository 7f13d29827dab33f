"""Continuous-batching server for level-set tile solves.

A tile solve is the LSM_Optimizer loop (source/optimizer/LSM_Optimizer.cpp:60-149) on
one tile: from a binary mask, the signed distance phi; then per iteration the imaging
of the current mask, the tracked loss PE + 1.0 x the background-penalty term at 0.01
(the reference's loss when no penalty is configured, :87-90), the best (lowest loss)
mask, the PE gradient dPE/dM as the normal speed, one RK2 WENO5-Godunov update and,
after iteration i with i % reinit_interval == 0 and i > 0, a chamfer re-initialisation.

:class:`TileServer` keeps every admitted solve's phi, mask, target, best mask, best
loss and loss history resident on the device, in contiguous per-size slot arrays, and
advances all admitted solves of a size together: each :meth:`TileServer.step` runs, per
tile size, ONE batched imaging + gradient pass (``litho_pe_gradient_batch_device``),
the best-state bookkeeping (``litho_lsm_track_batch``) and ONE batched RK2 update
(``litho_lsm_rk2_update_batch_device``, each solve with its own CFL step), plus one
batched re-initialisation per run of due slots. None of these waits for the GPU: the
host only enqueues work on each size class's stream (a size class whose cache lives in
its own Context runs on its own stream, so the classes overlap on the device), keeps
at most ``max_in_flight`` steps of a class queued, and learns that a solve has finished
from a CUDA event. Requests that arrive while others run are admitted at the next step,
as slots and the HBM budget allow; finished solves leave at once and free their slot.
Because every batched pass computes each image exactly as it would alone, a solve's
results do not depend on what it shares the GPU with.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import (ImagingCache, LevelSetUtils, LithoError, _f32, _ptr)


@dataclass
class TileSolve:
    """One request: its inputs, then its results and timings (perf_counter seconds).
    losses, best_loss, best_mask, phi and mask are set when the solve has finished."""
    id: int
    N: int
    iterations: int
    target: object            # (N, N) float32 CUDA tensor
    mask0: object             # (N, N) float32 CUDA tensor, binary
    t_submit: float = 0.0
    t_admit: float = 0.0
    t_done: float = 0.0
    done_iterations: int = 0
    losses: List[float] = field(default_factory=list)
    best_loss: float = math.inf
    best_mask: object = None
    phi: object = None         # final phi
    mask: object = None        # final mask
    _out: object = None        # device results until the completion event is seen
    _event: object = None

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


class _SizeClass:
    """Device slots of one tile size: contiguous [slot][N][N] arrays (so that the admitted
    solves form one batch) and the per-slot best loss, loss history and iteration count."""

    def __init__(self, cache: ImagingCache, slots: int, history_cols: int):
        torch = cache.ctx.torch
        N = cache.N
        self.cache = cache
        self.ctx = cache.ctx
        self.stream = cache.ctx.stream
        self.history_cols = history_cols
        with torch.cuda.stream(self.stream):
            self.phi = torch.empty((slots, N, N), dtype=torch.float32, device="cuda")
            self.phi_next = torch.empty_like(self.phi)
            self.mask = torch.empty_like(self.phi)
            self.target = torch.empty_like(self.phi)
            self.grad = torch.empty_like(self.phi)
            self.best_mask = torch.empty_like(self.phi)
            self.losses = torch.zeros((slots, 2), dtype=torch.float64, device="cuda")
            self.best = torch.full((slots,), math.inf, dtype=torch.float64, device="cuda")
            self.history = torch.zeros((slots, history_cols), dtype=torch.float64, device="cuda")
            self.iters = torch.zeros((slots,), dtype=torch.int32, device="cuda")
        self.solves: List[TileSolve] = []
        self.in_flight: deque = deque()   # events of this class's queued steps

    def compact(self, i: int):
        """Fill slot i with the last active solve (keeps the batch contiguous)."""
        last = len(self.solves) - 1
        if i != last:
            for a in (self.phi, self.mask, self.target, self.best_mask, self.history, self.best,
                      self.iters):
                a[i].copy_(a[last])
            self.solves[i] = self.solves[last]
        self.solves.pop()


class TileServer:
    """Continuous batching of LSM tile solves of mixed sizes on one GPU.

    caches: one ImagingCache per tile size; caches in different Contexts run on
    different streams. max_batch: solves of one size advanced together. hbm_budget:
    bytes of device memory the admitted solves may hold (their resident arrays and
    their share of the batched pass's scratch). max_iterations: the longest solve
    (the length of the per-slot loss history). max_in_flight: steps of one size class
    the host may queue ahead of the GPU."""

    def __init__(self, caches: Dict[int, ImagingCache], threshold: float = 0.225,
                 alpha: float = 50.0, dx: float = 1.0, dy: float = 1.0, cfl: float = 0.5,
                 b: float = 0.01, reinit_interval: int = 20, max_batch: int = 16,
                 hbm_budget: float = 120e9, max_iterations: int = 1000, max_in_flight: int = 2):
        if not caches:
            raise LithoError(1, "TileServer needs at least one ImagingCache")
        self.caches = dict(caches)
        self.threshold, self.alpha = float(threshold), float(alpha)
        self.dx, self.dy, self.cfl, self.b = float(dx), float(dy), float(cfl), float(b)
        self.reinit_interval = int(reinit_interval)
        self.max_batch = int(max_batch)
        self.hbm_budget = float(hbm_budget)
        self.max_iterations = int(max_iterations)
        self.max_in_flight = max(1, int(max_in_flight))
        self.queue: deque = deque()
        self.classes: Dict[int, _SizeClass] = {}
        self.finished: List[TileSolve] = []
        self.pending: List[TileSolve] = []   # retired, completion event not yet seen
        self.held = 0.0
        self._next_id = 0
        self.steps = 0
        self.tile_iterations = 0
        # The working memory of a full batch of every size, allocated now: the steps
        # that follow never allocate device memory.
        for cache in self.caches.values():
            cache.ctx.reserve(cache, self.max_batch)

    @staticmethod
    def solve_bytes(N: int) -> float:
        """Device bytes one admitted N x N solve holds: phi, next phi, mask, target,
        gradient and best-mask slots and about 12 N^2 bytes of its share of the batched
        pass's scratch plus the level-set temporaries."""
        return 4.0 * N * N * 6 + 12.0 * N * N + 4.0 * N * N

    def submit(self, target, mask, iterations: int) -> TileSolve:
        """Queue one solve of `iterations` LSM iterations from the binary `mask`."""
        torch = next(iter(self.caches.values())).ctx.torch
        t = _f32(target, torch)
        if t.dim() != 2 or t.shape[0] != t.shape[1] or t.shape[0] not in self.caches:
            raise LithoError(2, f"no cache for a tile of shape {tuple(t.shape)}")
        if not 1 <= iterations <= self.max_iterations:
            raise LithoError(1, f"a tile solve needs 1 .. {self.max_iterations} iterations")
        N = t.shape[0]
        s = TileSolve(self._next_id, N, int(iterations), t, _f32(mask, torch, (N, N), "mask"),
                      t_submit=time.perf_counter())
        self._next_id += 1
        self.queue.append(s)
        return s

    @property
    def active(self) -> int:
        return sum(len(c.solves) for c in self.classes.values())

    def _class(self, N: int) -> _SizeClass:
        cls = self.classes.get(N)
        if cls is None:
            cls = self.classes[N] = _SizeClass(self.caches[N], self.max_batch, self.max_iterations)
        return cls

    def _admit(self):
        first: Dict[int, int] = {}      # size -> first slot admitted by this call
        while self.queue:
            s = self.queue[0]
            cls = self._class(s.N)
            need = self.solve_bytes(s.N)
            if len(cls.solves) >= self.max_batch or self.held + need > self.hbm_budget:
                break   # first come, first served: a blocked head blocks the queue
            self.queue.popleft()
            i = len(cls.solves)
            first.setdefault(s.N, i)
            cls.solves.append(s)
            self.held += need
            s.t_admit = time.perf_counter()
            with cls.ctx.torch.cuda.stream(cls.stream):
                cls.mask[i].copy_(s.mask0)
                cls.target[i].copy_(s.target)
                cls.best_mask[i].copy_(s.mask0)     # LSM_Optimizer.cpp:77: best = initial mask
                cls.best[i] = math.inf
                cls.iters[i] = 0
        # phi = reinit_sdf(mask - 0.5) (LSM_Optimizer.cpp:62) of every solve admitted
        # here, one launch per size: inside = mask > 0.5 is the same classification.
        for N, i0 in first.items():
            cls = self.classes[N]
            n = len(cls.solves)
            with cls.ctx.torch.cuda.stream(cls.stream):
                LevelSetUtils.reinit_sdf_batch(cls.mask[i0:n], self.dx, self.dy, level=0.5,
                                               out=cls.phi[i0:n], ctx=cls.ctx)

    def _reinit_runs(self, cls: _SizeClass, due: List[int]):
        """reinit_sdf(phi) (LSM_Optimizer.cpp:118-121) and the mask phi >= 0 of the due
        slots, one batched launch per run of consecutive slots."""
        k = 0
        while k < len(due):
            a = due[k]
            while k + 1 < len(due) and due[k + 1] == due[k] + 1:
                k += 1
            z = due[k] + 1
            LevelSetUtils.reinit_sdf_batch(cls.phi[a:z], self.dx, self.dy, level=0.0,
                                           out=cls.phi_next[a:z], mask_out=cls.mask[a:z],
                                           ctx=cls.ctx)
            cls.phi[a:z].copy_(cls.phi_next[a:z])
            k += 1

    def _step_class(self, N: int, cls: _SizeClass) -> List[TileSolve]:
        torch = cls.ctx.torch
        lib, h = cls.ctx.lib, cls.ctx.handle
        n = len(cls.solves)
        # at most max_in_flight steps of this class queued on the device
        while len(cls.in_flight) >= self.max_in_flight:
            cls.in_flight.popleft().synchronize()
        done: List[TileSolve] = []
        with torch.cuda.stream(cls.stream):
            cls.ctx._check(lib.litho_pe_gradient_batch_device(
                h, cls.cache.handle, n, _ptr(cls.mask), _ptr(cls.target), self.threshold,
                self.alpha, 0.01, _ptr(cls.grad), _ptr(cls.losses)))
            cls.ctx._check(lib.litho_lsm_track_batch(
                h, n, N * N, _ptr(cls.losses), 1.0, _ptr(cls.best), _ptr(cls.mask),
                _ptr(cls.best_mask), _ptr(cls.history), cls.history_cols, _ptr(cls.iters)))
            # every solve's RK2 update, each with its own CFL step, in one call
            cls.ctx._check(lib.litho_lsm_rk2_update_batch_device(
                h, n, N, N, _ptr(cls.phi), _ptr(cls.grad), self.dx, self.dy, self.cfl, self.b,
                _ptr(cls.phi_next), _ptr(cls.mask), None))
            cls.phi, cls.phi_next = cls.phi_next, cls.phi
            due = [i for i, s in enumerate(cls.solves)
                   if self.reinit_interval > 0 and s.done_iterations > 0
                   and s.done_iterations % self.reinit_interval == 0]
            if due:
                self._reinit_runs(cls, due)
            for s in cls.solves:
                s.done_iterations += 1
            self.tile_iterations += n
            for i in range(n - 1, -1, -1):
                s = cls.solves[i]
                if s.done_iterations >= s.iterations:
                    s._out = (cls.phi[i].clone(), cls.mask[i].clone(), cls.best_mask[i].clone(),
                              cls.history[i, :s.iterations].clone(), cls.best[i].clone())
                    cls.compact(i)
                    self.held -= self.solve_bytes(N)
                    done.append(s)
            ev = torch.cuda.Event()
            ev.record(cls.stream)
            cls.in_flight.append(ev)
            for s in done:
                s._event = ev
        return done

    def _complete(self, s: TileSolve, now: float):
        s.t_done = now
        s.phi, s.mask, s.best_mask, hist, best = s._out
        s.losses = hist.cpu().tolist()
        s.best_loss = float(best.cpu())
        s._out = s._event = None
        self.finished.append(s)

    def poll(self) -> List[TileSolve]:
        """Solves whose results have been computed since the last poll (non-blocking)."""
        now = time.perf_counter()
        ready = [s._event.query() for s in self.pending]
        out = [s for s, r in zip(self.pending, ready) if r]
        if out:
            self.pending = [s for s, r in zip(self.pending, ready) if not r]
            for s in out:
                self._complete(s, now)
        return out

    def step(self) -> List[TileSolve]:
        """Admit what fits and enqueue one iteration of every admitted solve; returns the
        solves retired by this step (their results are complete once poll() or drain()
        has returned them)."""
        self._admit()
        done: List[TileSolve] = []
        for N, cls in self.classes.items():
            if cls.solves:
                done.extend(self._step_class(N, cls))
        self.steps += 1
        self.pending.extend(done)
        return done

    def check(self):
        """Raise LithoError if any enqueued pass saw a non-finite input or an expired
        wait (waits for the streams)."""
        for cls in self.classes.values():
            cls.ctx._check(cls.ctx.lib.litho_ctx_deferred_status(cls.ctx.handle))

    def drain(self) -> List[TileSolve]:
        """Step until every queued and admitted solve has finished; wait for the results."""
        while self.queue or self.active:
            self.step()
        for cls in self.classes.values():
            while cls.in_flight:
                cls.in_flight.popleft().synchronize()
        now = time.perf_counter()
        for s in self.pending:
            self._complete(s, now)
        self.pending = []
        self.check()
        return self.finished

    def serve(self, arrivals, time_limit: Optional[float] = None) -> Dict[str, float]:
        """Run a stream of requests. arrivals: (t_offset_seconds, target, mask,
        iterations) in order of t_offset; each is submitted once the wall clock has
        passed its offset. Returns throughput and latency statistics (completions
        counted when their results are on the device), the largest queue seen and the
        queue left when the last request arrived."""
        arrivals = sorted(arrivals, key=lambda a: a[0])
        t0 = time.perf_counter()
        k = 0
        solves: List[TileSolve] = []
        queue_max, queue_at_last_arrival = 0, None
        steps0, its0 = self.steps, self.tile_iterations
        while k < len(arrivals) or self.queue or self.active or self.pending:
            now = time.perf_counter() - t0
            while k < len(arrivals) and arrivals[k][0] <= now:
                _, tgt, m, its = arrivals[k]
                solves.append(self.submit(tgt, m, its))
                k += 1
            if k == len(arrivals) and queue_at_last_arrival is None:
                queue_at_last_arrival = len(self.queue)
            queue_max = max(queue_max, len(self.queue))
            if self.queue or self.active:
                self.step()
            elif self.pending:
                self.pending[0]._event.synchronize()
            elif k < len(arrivals):
                time.sleep(min(arrivals[k][0] - now, 0.001))
            self.poll()
            if time_limit is not None and time.perf_counter() - t0 > time_limit:
                break
        self.drain()
        wall = time.perf_counter() - t0
        lat = np.array([s.latency for s in solves if s.t_done > 0.0])
        its = sum(s.done_iterations for s in solves)
        span = arrivals[-1][0] if arrivals else 0.0
        return {"requests": len(solves), "completed": int(lat.size), "seconds": wall,
                "arrival_span_s": span,
                "offered_requests_per_s": len(arrivals) / span if span > 0 else float("nan"),
                "tile_iterations_per_s": its / wall if wall > 0 else 0.0,
                "latency_p50_s": float(np.percentile(lat, 50)) if lat.size else float("nan"),
                "latency_p99_s": float(np.percentile(lat, 99)) if lat.size else float("nan"),
                "queue_max": queue_max,
                "queue_at_last_arrival": queue_at_last_arrival or 0,
                "steps": self.steps - steps0, "tile_iterations": self.tile_iterations - its0}


def poisson_arrivals(rate: float, count: int, sizes, proportions, make_tile, iterations: int,
                     seed: int = 0):
    """A seeded Poisson stream: `count` requests at mean `rate` per second with tile
    sizes drawn from `sizes` in the given proportions; make_tile(N, rng) returns
    (target, mask) as arrays."""
    rng = np.random.default_rng(seed)
    p = np.asarray(proportions, dtype=np.float64)
    p = p / p.sum()
    t = 0.0
    out = []
    for _ in range(count):
        t += rng.exponential(1.0 / rate)
        N = int(rng.choice(sizes, p=p))
        tgt, m = make_tile(N, rng)
        out.append((t, tgt, m, iterations))
    return out
