"""Continuous-batching server for level-set tile solves.

A tile solve is the LSM_Optimizer loop (source/optimizer/LSM_Optimizer.cpp:60-149) on
one tile: from a binary mask, the signed distance phi, then per iteration the
imaging of the current mask, the PE loss, its gradient dPE/dM as the normal speed,
one RK2 WENO5-Godunov update and, every `reinit_interval` iterations, a chamfer
re-initialisation; the best (lowest PE) mask is kept.

:class:`TileServer` keeps every admitted solve's phi, mask and target resident on
the device and advances all of them together: each :meth:`TileServer.step` runs,
per tile size, ONE batched imaging + gradient pass over every admitted solve of that
size (``litho_pe_gradient_batch``), then one batched RK2 level-set update
(``litho_lsm_rk2_update_batch``, each solve with its own CFL step). Requests
that arrive while others run are admitted at the next step, as slots and the HBM
budget allow; finished solves leave at once and free their slot. Because the
batched pass computes every image exactly as it would alone, a solve's results do
not depend on what it shares the GPU with.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import (ImagingCache, LevelSetUtils, LithoError, _f32, pe_gradient_batch)


@dataclass
class TileSolve:
    """One request: its inputs, then its results and timings (perf_counter seconds)."""
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
    phi: object = None         # final phi, set when the solve finishes
    mask: object = None        # final mask

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


class _SizeClass:
    """Device slots of one tile size: contiguous [slot][N][N] arrays so that the
    admitted solves form one batch."""

    def __init__(self, cache: ImagingCache, slots: int):
        torch = cache.ctx.torch
        N = cache.N
        self.cache = cache
        self.phi = torch.empty((slots, N, N), dtype=torch.float32, device="cuda")
        self.phi_next = torch.empty_like(self.phi)
        self.mask = torch.empty_like(self.phi)
        self.target = torch.empty_like(self.phi)
        self.grad = torch.empty_like(self.phi)
        self.solves: List[TileSolve] = []

    def compact(self, i: int):
        """Fill slot i with the last active solve (keeps the batch contiguous)."""
        last = len(self.solves) - 1
        if i != last:
            for a in (self.phi, self.mask, self.target):
                a[i].copy_(a[last])
            self.solves[i] = self.solves[last]
        self.solves.pop()


class TileServer:
    """Continuous batching of LSM tile solves of mixed sizes on one GPU.

    caches: one ImagingCache per tile size (same context). max_batch: solves of one
    size advanced together. hbm_budget: bytes of device memory the admitted solves
    may hold (their resident arrays and their share of the batched pass's scratch)."""

    def __init__(self, caches: Dict[int, ImagingCache], threshold: float = 0.225,
                 alpha: float = 50.0, dx: float = 1.0, dy: float = 1.0, cfl: float = 0.5,
                 b: float = 0.01, reinit_interval: int = 20, max_batch: int = 16,
                 hbm_budget: float = 120e9):
        if not caches:
            raise LithoError(1, "TileServer needs at least one ImagingCache")
        self.caches = dict(caches)
        self.ctx = next(iter(caches.values())).ctx
        self.threshold, self.alpha = float(threshold), float(alpha)
        self.dx, self.dy, self.cfl, self.b = float(dx), float(dy), float(cfl), float(b)
        self.reinit_interval = int(reinit_interval)
        self.max_batch = int(max_batch)
        self.hbm_budget = float(hbm_budget)
        self.queue: deque = deque()
        self.classes: Dict[int, _SizeClass] = {}
        self.finished: List[TileSolve] = []
        self.held = 0.0
        self._next_id = 0
        self.steps = 0
        self.tile_iterations = 0
        # The working memory of a full batch of every size, allocated now: the steps
        # that follow never allocate device memory.
        for cache in self.caches.values():
            self.ctx.reserve(cache, self.max_batch)

    @staticmethod
    def solve_bytes(N: int) -> float:
        """Device bytes one admitted N x N solve holds: phi, mask, target and
        gradient slots, the level-set temporaries and about 12 N^2 bytes of its share
        of the batched pass's scratch."""
        return 4.0 * N * N * 4 + 12.0 * N * N + 3.0 * 4 * N * N

    def submit(self, target, mask, iterations: int) -> TileSolve:
        """Queue one solve of `iterations` LSM iterations from the binary `mask`."""
        torch = self.ctx.torch
        t = _f32(target, torch)
        if t.dim() != 2 or t.shape[0] != t.shape[1] or t.shape[0] not in self.caches:
            raise LithoError(2, f"no cache for a tile of shape {tuple(t.shape)}")
        if iterations < 1:
            raise LithoError(1, "a tile solve needs at least one iteration")
        N = t.shape[0]
        s = TileSolve(self._next_id, N, int(iterations), t, _f32(mask, torch, (N, N), "mask"),
                      t_submit=time.perf_counter())
        self._next_id += 1
        self.queue.append(s)
        return s

    @property
    def active(self) -> int:
        return sum(len(c.solves) for c in self.classes.values())

    def _admit(self):
        first: Dict[int, int] = {}      # size -> first slot admitted by this call
        while self.queue:
            s = self.queue[0]
            cls = self.classes.get(s.N)
            if cls is None:
                cls = self.classes[s.N] = _SizeClass(self.caches[s.N], self.max_batch)
            need = self.solve_bytes(s.N)
            if len(cls.solves) >= self.max_batch or self.held + need > self.hbm_budget:
                break   # first come, first served: a blocked head blocks the queue
            self.queue.popleft()
            i = len(cls.solves)
            first.setdefault(s.N, i)
            cls.solves.append(s)
            self.held += need
            s.t_admit = time.perf_counter()
            cls.mask[i].copy_(s.mask0)
            cls.target[i].copy_(s.target)
            s.best_mask = s.mask0.clone()
        # phi = reinit_sdf(mask - 0.5) (LSM_Optimizer.cpp:62) of every solve admitted
        # here, one launch per size: inside = mask > 0.5 is the same classification.
        for N, i0 in first.items():
            cls = self.classes[N]
            n = len(cls.solves)
            LevelSetUtils.reinit_sdf_batch(cls.mask[i0:n], self.dx, self.dy, level=0.5,
                                           out=cls.phi[i0:n], ctx=self.ctx)

    def step(self) -> List[TileSolve]:
        """Admit what fits, advance every admitted solve by one iteration, retire the
        finished ones; returns the solves finished by this step."""
        self._admit()
        done: List[TileSolve] = []
        for N, cls in self.classes.items():
            n = len(cls.solves)
            if n == 0:
                continue
            losses, _ = pe_gradient_batch(cls.cache, cls.mask[:n], cls.target[:n], self.threshold,
                                          self.alpha, cls.grad[:n])
            for i, s in enumerate(cls.solves):
                pe = losses[i]
                s.losses.append(pe)
                if pe < s.best_loss:
                    s.best_loss = pe
                    s.best_mask = cls.mask[i].clone()
            # every solve's RK2 update, each with its own CFL step, in one call
            LevelSetUtils.rk2_update_batch(cls.phi[:n], cls.grad[:n], self.dx, self.dy, self.cfl,
                                           self.b, cls.phi_next[:n], cls.mask[:n], ctx=self.ctx)
            cls.phi, cls.phi_next = cls.phi_next, cls.phi
            for i, s in enumerate(cls.solves):
                it = s.done_iterations
                if self.reinit_interval > 0 and it % self.reinit_interval == 0 and it > 0:
                    phi, mask = LevelSetUtils.reinit_sdf(cls.phi[i], self.dx, self.dy, ctx=self.ctx,
                                                         with_mask=True)
                    cls.phi[i].copy_(phi)
                    cls.mask[i].copy_(mask)
                s.done_iterations += 1
            self.tile_iterations += n
            for i in range(n - 1, -1, -1):
                s = cls.solves[i]
                if s.done_iterations >= s.iterations:
                    s.phi = cls.phi[i].clone()
                    s.mask = cls.mask[i].clone()
                    cls.compact(i)
                    self.held -= self.solve_bytes(N)
                    done.append(s)
        self.steps += 1
        if done:
            self.ctx.synchronize()
            now = time.perf_counter()
            for s in done:
                s.t_done = now
            self.finished.extend(done)
        return done

    def drain(self) -> List[TileSolve]:
        """Step until every queued and admitted solve has finished."""
        while self.queue or self.active:
            self.step()
        return self.finished

    def serve(self, arrivals, time_limit: Optional[float] = None) -> Dict[str, float]:
        """Run a stream of requests. arrivals: (t_offset_seconds, target, mask,
        iterations) in order of t_offset; each is submitted once the wall clock has
        passed its offset. Returns throughput and latency statistics."""
        arrivals = sorted(arrivals, key=lambda a: a[0])
        t0 = time.perf_counter()
        k = 0
        solves: List[TileSolve] = []
        while k < len(arrivals) or self.queue or self.active:
            now = time.perf_counter() - t0
            while k < len(arrivals) and arrivals[k][0] <= now:
                _, tgt, m, its = arrivals[k]
                solves.append(self.submit(tgt, m, its))
                k += 1
            if self.queue or self.active:
                self.step()
            elif k < len(arrivals):
                time.sleep(min(arrivals[k][0] - now, 0.001))
            if time_limit is not None and time.perf_counter() - t0 > time_limit:
                break
        wall = time.perf_counter() - t0
        lat = np.array([s.latency for s in solves if s.t_done > 0.0])
        its = sum(s.done_iterations for s in solves)
        return {"requests": len(solves), "completed": int(lat.size), "seconds": wall,
                "tile_iterations_per_s": its / wall if wall > 0 else 0.0,
                "latency_p50_s": float(np.percentile(lat, 50)) if lat.size else float("nan"),
                "latency_p99_s": float(np.percentile(lat, 99)) if lat.size else float("nan"),
                "steps": self.steps}


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
