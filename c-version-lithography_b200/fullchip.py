"""Full-chip micro-tile optimisation over the C ABI.

Mirrors the reference's full-chip classes:

* :class:`Partition` - ``Partition`` / ``PartitionMeta`` (include/utils/partition.h,
  source/utils/partition.cpp:21-120): Cores, Halo tiles with periodic wrap,
  Core + Guard update windows, four-neighbour relations.
* :class:`MicroGradientExchange` - ``MicroGradientExchange::compute``
  (source/utils/micro_gradient_exchange.cpp:134-334) for all four loss types (PE,
  PEPenalty, EPE, PE_EPE) with optional Core metrics: per-tile imaging, windowed
  data loss, sparse EPE at caller-selected edge points, raw mask gradients, CEPT
  against the neighbours' Cores and Average / Linear guard fusion.
* :class:`FullChipCTMOptimizer` - ``FullChipCTMOptimizer::optimize``
  (source/optimizer/full_chip_ctm.cpp:25-152): fixed-step theta descent inside
  each tile's Core + Guard window, best state over all evaluations.
* :class:`FullChipLSMOptimizer` - ``FullChipLSMOptimizer::optimize``
  (source/optimizer/full_chip_lsm.cpp:38-254): per-tile SDF from the CTM binary
  mask, windowed RK2 level-set steps, reinitialisation, Binary / Gray rendering.

Local tiles are one float32 CUDA tensor of shape (num_tiles, tile_size,
tile_size), tile id = row * grid_cols + col. Every computation runs in the
library's kernels; there is no CPU path.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import (EXCHANGE_TILE_METRICS, ExchangeEpeC, ExchangeOptionsC, ImagingCache, LithoError,
               _f32, _ptr, default_context)

LOSS_TYPES = {"PE": 0, "PEPenalty": 1, "EPE": 2, "PE_EPE": 3}
LOSS_REGIONS = {"Core": 0, "CoreGuard": 1}
FUSION_MODES = {"Average": 0, "Linear": 1}


@dataclass
class MicroGradientOptions:
    """MicroGradientOptions (include/utils/micro_gradient_exchange.h:19-40). EP
    selection stays with the caller: the EPE types evaluate the edge points given to
    :meth:`MicroGradientExchange.compute`; ``epe_all_eps`` sets all their weights to 1."""
    loss_type: str = "PE"
    loss_region: str = "Core"
    main_region_dilation_pixels: int = 2
    pe_weight: float = 1.0
    epe_weight: float = 1.0
    penalty_weight: float = 2.0
    penalty_threshold: float = 0.01
    epe_all_eps: bool = False
    epe_pixel_size: float = 1.0
    collect_core_metrics: bool = False
    enable_cept: bool = False
    cept_guard_only: bool = False
    cept_weight: float = 1.1
    enable_grad_fusion: bool = False
    fusion_mode: str = "Average"
    fusion_weight_owner: float = 0.5
    fusion_weight_neighbor: float = 0.5

    def to_c(self) -> ExchangeOptionsC:
        for name, table in (("loss_type", LOSS_TYPES), ("loss_region", LOSS_REGIONS),
                            ("fusion_mode", FUSION_MODES)):
            if getattr(self, name) not in table:
                raise LithoError(7, f"MicroGradientOptions.{name}={getattr(self, name)!r} is not "
                                    f"one of {sorted(table)}")
        return ExchangeOptionsC(
            LOSS_TYPES[self.loss_type], LOSS_REGIONS[self.loss_region], self.pe_weight,
            self.penalty_weight, self.penalty_threshold, int(self.enable_cept),
            int(self.cept_guard_only), self.cept_weight, int(self.enable_grad_fusion),
            FUSION_MODES[self.fusion_mode], self.fusion_weight_owner, self.fusion_weight_neighbor)

    def weights(self):
        """micro_loss_weights (micro_gradient_exchange.cpp:95-99): (pe, epe, penalty)."""
        return ((0.0 if self.loss_type == "EPE" else self.pe_weight),
                (self.epe_weight if self.loss_type in ("EPE", "PE_EPE") else 0.0),
                (self.penalty_weight if self.loss_type == "PEPenalty" else 0.0))


@dataclass(frozen=True)
class PartitionRect:
    """PartitionRect: half-open [y0, y1) x [x0, x1)."""
    y0: int
    y1: int
    x0: int
    x1: int

    def rows(self) -> int:
        return self.y1 - self.y0

    def cols(self) -> int:
        return self.x1 - self.x0


@dataclass(frozen=True)
class PartitionTile:
    id: int
    row: int
    col: int
    core_global: PartitionRect
    tile_global: PartitionRect
    core_local: PartitionRect
    update_local: PartitionRect


class Partition:
    """Partition::build (partition.cpp:21-80) on the device: geometry + tile copies.

    By default the Cores are cut at i * extent / count as in the reference; with
    row_cuts / col_cuts (grid_rows + 1 and grid_cols + 1 boundaries from 0 to the
    extent) they take the given, possibly uneven boundaries, every tile keeping the
    one tile size = largest Core side + 2 halo (litho_partition_create_cuts)."""

    def __init__(self, height: int, width: int, grid_rows: int, grid_cols: int, halo: int,
                 guard: int, ctx=None, row_cuts=None, col_cuts=None):
        self.ctx = ctx or default_context()
        lib = self.ctx.lib
        h = ctypes.c_void_p()
        if row_cuts is None and col_cuts is None:
            self.ctx._check(lib.litho_partition_create(self.ctx.handle, height, width, grid_rows,
                                                       grid_cols, halo, guard, ctypes.byref(h)))
        else:
            rc = [int(v) for v in (row_cuts if row_cuts is not None else
                                   [r * height // grid_rows for r in range(grid_rows + 1)])]
            cc = [int(v) for v in (col_cuts if col_cuts is not None else
                                   [c * width // grid_cols for c in range(grid_cols + 1)])]
            if len(rc) != grid_rows + 1 or len(cc) != grid_cols + 1:
                raise LithoError(1, "Partition: grid_rows + 1 row cuts and grid_cols + 1 column "
                                    "cuts are needed")
            self.ctx._check(lib.litho_partition_create_cuts(
                self.ctx.handle, height, width, grid_rows, (ctypes.c_int * len(rc))(*rc),
                grid_cols, (ctypes.c_int * len(cc))(*cc), halo, guard, ctypes.byref(h)))
        self.handle = h
        self.height, self.width = height, width
        self.grid_rows, self.grid_cols = grid_rows, grid_cols
        self.halo, self.guard = halo, guard
        n, ts = ctypes.c_int(), ctypes.c_int()
        lib.litho_partition_info(h, ctypes.byref(n), ctypes.byref(ts))
        self.num_tiles, self.tile_size = n.value, ts.value
        self.tiles: List[PartitionTile] = []
        buf = (ctypes.c_int * 16)()
        for t in range(self.num_tiles):
            self.ctx._check(lib.litho_partition_tile_rects(h, t, buf))
            r = [PartitionRect(*buf[4 * i:4 * i + 4]) for i in range(4)]
            self.tiles.append(PartitionTile(t, t // grid_cols, t % grid_cols, *r))

    def empty_tiles(self):
        torch = self.ctx.torch
        ts = self.tile_size
        return torch.empty((self.num_tiles, ts, ts), dtype=torch.float32, device="cuda")

    def extract_all(self, global_image):
        """Partition::extract_all (partition.cpp:97-103): periodic Halo tiles."""
        g = _f32(global_image, self.ctx.torch, (self.height, self.width), "global image")
        out = self.empty_tiles()
        self.ctx._check(self.ctx.lib.litho_partition_extract(self.ctx.handle, self.handle,
                                                             _ptr(g), _ptr(out)))
        return out

    def assemble_global(self, local_tiles):
        """Partition::assemble_global (partition.cpp:105-113): Cores only."""
        ts = self.tile_size
        loc = _f32(local_tiles, self.ctx.torch, (self.num_tiles, ts, ts), "local tiles")
        out = self.ctx.torch.zeros((self.height, self.width), dtype=self.ctx.torch.float32,
                                   device="cuda")
        self.ctx._check(self.ctx.lib.litho_partition_assemble(self.ctx.handle, self.handle,
                                                              _ptr(loc), _ptr(out)))
        return out

    def close(self):
        if getattr(self, "handle", None):
            self.ctx.lib.litho_partition_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class CoreLossMetrics:
    """CoreLossMetrics (include/utils/micro_gradient_exchange.h:66-75)."""
    pe_loss: float = 0.0
    bg_penalty_raw: float = 0.0
    pe_penalty_loss: float = 0.0
    epe_loss: float = 0.0
    epe_abs_sum_nm: float = 0.0
    ep_count: int = 0
    epe_mean: float = 0.0
    data_loss: float = 0.0


@dataclass
class MicroLocalLoss:
    """The scalars of MicroGradientData (micro_gradient_exchange.h:86-97)."""
    pe_loss: float
    bg_penalty_raw: float
    penalty_loss: float
    data_loss: float
    cept_loss: float
    loss: float
    epe_loss: float = 0.0
    epe_abs_sum_nm: float = 0.0
    epe_count: int = 0
    core: CoreLossMetrics = field(default_factory=CoreLossMetrics)


@dataclass
class MicroGradientExchangeResult:
    """MicroGradientExchangeResult: totals, per-tile losses, gradients (device)."""
    loss: float
    data_loss: float
    cept_loss: float
    locals: List[MicroLocalLoss]
    mask_gradients: object     # (num_tiles, ts, ts) exchanged gradients
    raw_gradients: object      # (num_tiles, ts, ts) before CEPT and fusion


def _edge_points(eps, eps_weights, all_ones: bool):
    """Global EP coordinates (n x 2, y then x) and weight_epe as contiguous float64."""
    if eps is None:
        return np.zeros((0, 2)), np.zeros(0)
    pts = np.ascontiguousarray(np.asarray(eps, dtype=np.float64).reshape(-1, 2))
    if all_ones or eps_weights is None:
        w = np.ones(len(pts))
    else:
        w = np.ascontiguousarray(np.asarray(eps_weights, dtype=np.float64).reshape(-1))
        if len(w) != len(pts):
            raise LithoError(2, "eps and eps_weights must have the same length")
    return pts, w


class MicroGradientExchange:
    """MicroGradientExchange (include/utils/micro_gradient_exchange.h:119-139)."""

    def __init__(self, partition: Partition, cache: ImagingCache, threshold: float = 0.25,
                 alpha: float = 85.0):
        if cache.N != partition.tile_size:
            raise LithoError(2, f"cache N {cache.N} != tile size {partition.tile_size}")
        self.partition = partition
        self.cache = cache
        self.ctx = partition.ctx
        self.threshold, self.alpha = float(threshold), float(alpha)
        self.grad = partition.empty_tiles()
        self.raw = partition.empty_tiles()

    def compute(self, local_masks, global_target, options: Optional[MicroGradientOptions] = None,
                eps=None, eps_weights=None):
        """compute(local_masks, global_target, options) (micro_gradient_exchange.cpp:134-334).

        eps: the selected edge points as global subpixel (y, x) rows (select_micro_epe_points'
        output), eps_weights their weight_epe; used by the EPE types and the Core metrics.
        The returned gradient tensors are reused by the next call."""
        p = self.partition
        torch = self.ctx.torch
        opt = options or MicroGradientOptions()
        copt = opt.to_c()
        pts, w = _edge_points(eps, eps_weights, opt.epe_all_eps)
        cepe = ExchangeEpeC(opt.epe_weight, opt.main_region_dilation_pixels, opt.epe_pixel_size,
                            int(opt.collect_core_metrics),
                            pts.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                            w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(pts))
        ts = p.tile_size
        masks = _f32(local_masks, torch, (p.num_tiles, ts, ts), "local masks")
        tgt = _f32(global_target, torch, (p.height, p.width), "global target")
        M = EXCHANGE_TILE_METRICS
        per = (ctypes.c_double * (M * p.num_tiles))()
        tot = (ctypes.c_double * 3)()
        self.ctx._check(self.ctx.lib.litho_exchange_compute_epe(
            self.ctx.handle, p.handle, self.cache.handle, _ptr(masks), _ptr(tgt),
            self.threshold, self.alpha, ctypes.byref(copt), ctypes.byref(cepe), _ptr(self.raw),
            _ptr(self.grad), per, tot))
        locs = []
        for t in range(p.num_tiles):
            r = per[M * t:M * (t + 1)]
            locs.append(MicroLocalLoss(r[0], r[1], r[2], r[6], r[7], r[8], r[3], r[4], int(r[5]),
                                       CoreLossMetrics(r[9], r[10], r[11], r[12], r[13],
                                                       int(r[14]), r[15], r[16])))
        return MicroGradientExchangeResult(tot[0], tot[1], tot[2], locs, self.grad, self.raw)


@dataclass
class FullChipCTMOptions:
    """FullChipCTMOptions (include/optimizer/full_chip_ctm.h:10-17)."""
    iterations: int = 50
    learning_rate: float = 0.9
    gradient_options: MicroGradientOptions = field(
        default_factory=lambda: MicroGradientOptions(cept_guard_only=True))
    verbose: bool = False
    retain_final_masks: bool = False


@dataclass
class FullChipCTMIteration:
    """FullChipCTMIteration (include/optimizer/full_chip_ctm.h:19-28)."""
    iteration: int
    loss: float
    data_loss: float
    cept_loss: float
    pe_contribution: float
    penalty_contribution: float
    epe_contribution: float
    cept_contribution: float
    pe_loss_raw: float
    bg_penalty_raw: float
    epe_loss_raw: float
    epe_abs_sum_nm: float
    epe_point_count: int


@dataclass
class FullChipCTMResult:
    best_iteration: int
    best_loss: float
    global_mask: object
    local_masks: object
    local_theta: object
    final_local_masks: object
    history: List[FullChipCTMIteration]


class FullChipCTMOptimizer:
    """FullChipCTMOptimizer (include/optimizer/full_chip_ctm.h:38-58)."""

    def __init__(self, partition: Partition, cache: ImagingCache, threshold: float = 0.25,
                 alpha: float = 85.0):
        self.partition = partition
        self.exchange = MicroGradientExchange(partition, cache, threshold, alpha)
        self.ctx = partition.ctx

    @staticmethod
    def initialize_theta(pattern, torch):
        """CTM_Optimizer::_initialize_theta (CTM_Optimizer.cpp:55-64): > 0 -> 0.3 pi, else 0.7 pi."""
        pi = 3.14159265358979323846
        return torch.where(pattern > 0, torch.full_like(pattern, 0.3 * pi),
                           torch.full_like(pattern, 0.7 * pi))

    def optimize(self, global_target, options: Optional[FullChipCTMOptions] = None,
                 initial_pattern=None, eps=None, eps_weights=None) -> FullChipCTMResult:
        """optimize([initial_pattern,] global_target, options) (full_chip_ctm.cpp:25-152).

        eps / eps_weights: the edge points of the EPE loss types (see
        MicroGradientExchange.compute)."""
        opt = options or FullChipCTMOptions()
        if opt.iterations < 0:
            raise LithoError(1, "FullChipCTM iterations must be non-negative")
        if not math.isfinite(opt.learning_rate):
            raise LithoError(3, "FullChipCTM learning_rate must be finite")
        go = MicroGradientOptions(**{**opt.gradient_options.__dict__, "cept_guard_only": True})
        wpe, wepe, _ = go.weights()
        p = self.partition
        torch = self.ctx.torch
        tgt = _f32(global_target, torch, (p.height, p.width), "global target")
        init = tgt if initial_pattern is None else _f32(initial_pattern, torch,
                                                        (p.height, p.width), "initial pattern")
        theta = p.extract_all(self.initialize_theta(init, torch))
        masks = p.empty_tiles()
        lib, h = self.ctx.lib, self.ctx.handle
        self.ctx._check(lib.litho_fullchip_theta_step(h, p.handle, _ptr(theta), None, 0.0,
                                                      _ptr(masks)))
        history: List[FullChipCTMIteration] = []
        best = dict(loss=math.inf, iteration=0, masks=None, theta=None)

        def record(it, ev):
            L = ev.locals
            cept = go.cept_weight * ev.cept_loss if go.enable_cept else 0.0
            history.append(FullChipCTMIteration(
                it, ev.loss, ev.data_loss, ev.cept_loss, sum(wpe * l.pe_loss for l in L),
                sum(l.penalty_loss for l in L), sum(wepe * l.epe_loss for l in L), cept,
                sum(l.pe_loss for l in L), sum(l.bg_penalty_raw for l in L),
                sum(l.epe_loss for l in L), sum(l.epe_abs_sum_nm for l in L),
                sum(l.epe_count for l in L)))
            if ev.loss < best["loss"]:
                best.update(loss=ev.loss, iteration=it, masks=masks.clone(), theta=theta.clone())
            if opt.verbose:
                print(f"CTM {it:>3}/{opt.iterations} data={ev.data_loss:.3f} "
                      f"cept={ev.cept_loss:.3f} total={ev.loss:.3f}")

        ev = self.exchange.compute(masks, tgt, go, eps, eps_weights)
        record(0, ev)
        for it in range(1, opt.iterations + 1):
            self.ctx._check(lib.litho_fullchip_theta_step(h, p.handle, _ptr(theta),
                                                          _ptr(ev.mask_gradients),
                                                          opt.learning_rate, _ptr(masks)))
            ev = self.exchange.compute(masks, tgt, go, eps, eps_weights)
            record(it, ev)
        return FullChipCTMResult(best["iteration"], best["loss"],
                                 p.assemble_global(best["masks"]), best["masks"], best["theta"],
                                 masks.clone() if opt.retain_final_masks else None, history)


@dataclass
class FullChipLSMOptions:
    """FullChipLSMOptions (include/optimizer/full_chip_lsm.h:8-21)."""
    iterations: int = 200
    dx: float = 1.0
    dy: float = 1.0
    cfl: float = 0.7
    curvature_weight: float = 0.01
    reinit_interval: int = 20
    mask_type: str = "Binary"
    render_scale: int = 4
    gradient_options: MicroGradientOptions = field(
        default_factory=lambda: MicroGradientOptions(epe_all_eps=True))
    verbose: bool = False


@dataclass
class FullChipLSMIteration:
    """FullChipLSMIteration (include/optimizer/full_chip_lsm.h:23-36)."""
    iteration: int
    loss: float
    data_loss: float
    cept_loss: float
    min_dt: float
    max_dt: float
    pe_contribution: float
    penalty_contribution: float
    epe_contribution: float
    cept_contribution: float
    core: CoreLossMetrics
    total_pe_loss: float
    total_bg_penalty_raw: float
    total_epe_loss: float
    total_epe_abs_sum_nm: float
    total_ep_count: int
    epe_mean: float


@dataclass
class FullChipLSMResult:
    best_iteration: int
    best_loss: float
    global_mask: object
    global_phi: object
    initial_global_phi: object
    initial_global_mask: object
    local_masks: object
    local_phi: object
    history: List[FullChipLSMIteration]
    best_core_metrics: List[CoreLossMetrics] = field(default_factory=list)


class FullChipLSMOptimizer:
    """FullChipLSMOptimizer (include/optimizer/full_chip_lsm.h:52-69) over the device
    partition: per-tile SDF initialisation, exchange, windowed RK2 level-set steps with
    periodic reinitialisation, rendered masks, best state over all evaluations."""

    def __init__(self, partition: Partition, cache: ImagingCache, threshold: float = 0.25,
                 alpha: float = 85.0):
        self.partition = partition
        self.exchange = MicroGradientExchange(partition, cache, threshold, alpha)
        self.ctx = partition.ctx

    def optimize(self, initial_binary, global_target,
                 options: Optional[FullChipLSMOptions] = None, eps=None,
                 eps_weights=None) -> FullChipLSMResult:
        """optimize(initial_binary, global_target, options) (full_chip_lsm.cpp:38-254).

        eps / eps_weights: the edge points of the EPE loss types and of the Core EPE
        statistics (see MicroGradientExchange.compute)."""
        from . import MASK_TYPES
        opt = options or FullChipLSMOptions()
        if opt.mask_type not in MASK_TYPES:
            raise LithoError(1, f"mask_type must be one of {sorted(MASK_TYPES)}")
        if opt.iterations < 0:
            raise LithoError(1, "FullChipLSM iterations must be non-negative")
        # Core + Guard evaluation, guard-only CEPT, Core metrics (full_chip_lsm.cpp:43-46).
        go = MicroGradientOptions(**{**opt.gradient_options.__dict__, "loss_region": "CoreGuard",
                                     "cept_guard_only": True, "collect_core_metrics": True})
        wpe, wepe, _ = go.weights()
        p = self.partition
        torch = self.ctx.torch
        lib, h = self.ctx.lib, self.ctx.handle
        mt = MASK_TYPES[opt.mask_type]
        init = _f32(initial_binary, torch, (p.height, p.width), "initial binary mask")
        tgt = _f32(global_target, torch, (p.height, p.width), "global target")
        phi, masks = p.empty_tiles(), p.empty_tiles()
        self.ctx._check(lib.litho_fullchip_lsm_init(h, p.handle, _ptr(init), opt.dx, opt.dy, mt,
                                                    opt.render_scale, _ptr(phi), _ptr(masks)))
        initial_global_phi = p.assemble_global(phi)
        initial_global_mask = p.assemble_global(masks)
        history: List[FullChipLSMIteration] = []
        best = dict(loss=math.inf, iteration=0, phi=None, masks=None, core=[])

        def record(it, ev, dmin, dmax):
            # full_chip_lsm.cpp:152-186: weighted contributions, raw totals over the
            # Core + Guard regions, Core sums with the mean over all Core EPs.
            L = ev.locals
            core = CoreLossMetrics(*(sum(getattr(l.core, k) for l in L) for k in (
                "pe_loss", "bg_penalty_raw", "pe_penalty_loss", "epe_loss", "epe_abs_sum_nm",
                "ep_count")), 0.0, sum(l.core.data_loss for l in L))
            core.epe_mean = core.epe_abs_sum_nm / core.ep_count if core.ep_count else 0.0
            cept = go.cept_weight * ev.cept_loss if go.enable_cept else 0.0
            total_abs, total_n = sum(l.epe_abs_sum_nm for l in L), sum(l.epe_count for l in L)
            history.append(FullChipLSMIteration(
                it, ev.loss, ev.data_loss, ev.cept_loss, dmin, dmax,
                sum(wpe * l.pe_loss for l in L), sum(l.penalty_loss for l in L),
                sum(wepe * l.epe_loss for l in L), cept, core, sum(l.pe_loss for l in L),
                sum(l.bg_penalty_raw for l in L), sum(l.epe_loss for l in L), total_abs, total_n,
                total_abs / total_n if total_n else 0.0))
            if ev.loss < best["loss"]:
                best.update(loss=ev.loss, iteration=it, phi=phi.clone(), masks=masks.clone(),
                            core=[l.core for l in L])
            if opt.verbose:
                print(f"LSM {it:>3}/{opt.iterations} data={ev.data_loss:.3f} "
                      f"cept={ev.cept_loss:.3f} total={ev.loss:.3f}")

        ev = self.exchange.compute(masks, tgt, go, eps, eps_weights)
        record(0, ev, 0.0, 0.0)
        nxt = p.empty_tiles()
        dmin, dmax = ctypes.c_double(), ctypes.c_double()
        for it in range(1, opt.iterations + 1):
            reinit = 1 if opt.reinit_interval > 0 and it % opt.reinit_interval == 0 else 0
            self.ctx._check(lib.litho_fullchip_lsm_step(
                h, p.handle, _ptr(phi), _ptr(ev.mask_gradients), opt.dx, opt.dy, opt.cfl,
                opt.curvature_weight, reinit, mt, opt.render_scale, _ptr(nxt), _ptr(masks),
                ctypes.byref(dmin), ctypes.byref(dmax)))
            phi, nxt = nxt, phi
            ev = self.exchange.compute(masks, tgt, go, eps, eps_weights)
            record(it, ev, dmin.value, dmax.value)
        return FullChipLSMResult(best["iteration"], best["loss"], p.assemble_global(best["masks"]),
                                 p.assemble_global(best["phi"]), initial_global_phi,
                                 initial_global_mask, best["masks"], best["phi"], history,
                                 best["core"])
