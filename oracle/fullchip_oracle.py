"""FP64 restatement of the reference full-chip partition, micro-gradient exchange and
full-chip CTM (test infrastructure only, see ``oracle/__init__.py``).

Follows source/utils/partition.cpp:21-120, source/utils/micro_gradient_exchange.cpp:18-334
(PE, PEPenalty, EPE and PE_EPE loss types, Core or Core+Guard loss region, Core
metrics, guard-only or two-sided CEPT, Average or Linear guard-gradient fusion) and
source/optimizer/full_chip_ctm.cpp:25-152. EP selection (ep_select.cpp) is outside
the restated path: the edge points are inputs, as they are for the device exchange.
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional

import numpy as np

from . import imaging_oracle as io


@dataclasses.dataclass(frozen=True)
class Rect:
    """PartitionRect (include/utils/partition.h): half-open [y0, y1) x [x0, x1)."""
    y0: int
    y1: int
    x0: int
    x1: int

    @property
    def rows(self):
        return self.y1 - self.y0

    @property
    def cols(self):
        return self.x1 - self.x0

    def shifted(self, dy, dx):
        return Rect(self.y0 + dy, self.y1 + dy, self.x0 + dx, self.x1 + dx)

    def expanded(self, w):
        return Rect(self.y0 - w, self.y1 + w, self.x0 - w, self.x1 + w)

    @staticmethod
    def intersection(a, b):
        return Rect(max(a.y0, b.y0), min(a.y1, b.y1), max(a.x0, b.x0), min(a.x1, b.x1))


LEFT, RIGHT, TOP, BOTTOM = 0, 1, 2, 3


@dataclasses.dataclass
class Neighbor:
    id: int
    direction: int
    guard_global: Rect
    my_guard_local: Rect
    neighbor_overlap_local: Rect
    overlap_global: Rect
    my_overlap_local: Rect
    neighbor_guard_local: Rect


@dataclasses.dataclass
class Tile:
    id: int
    row: int
    col: int
    halo: int
    guard: int
    core_global: Rect
    tile_global: Rect
    core_local: Rect
    update_local: Rect
    neighbors: List[Neighbor]


@dataclasses.dataclass
class Meta:
    height: int
    width: int
    grid_rows: int
    grid_cols: int
    halo: int
    guard: int
    tile_size: int
    tiles: List[Tile]


def build(height, width, grid_rows, grid_cols, halo, guard, row_cuts=None,
          col_cuts=None) -> Meta:
    """Partition::build (source/utils/partition.cpp:21-80). row_cuts / col_cuts
    (grid_rows + 1 / grid_cols + 1 boundaries from 0 to the extent) replace the
    reference's row * height // grid_rows cuts; the tile size stays the largest Core
    side + 2 halo, rounded up to even (partition.cpp:31-34)."""
    rc = list(row_cuts) if row_cuts is not None else [r * height // grid_rows
                                                      for r in range(grid_rows + 1)]
    cc = list(col_cuts) if col_cuts is not None else [c * width // grid_cols
                                                      for c in range(grid_cols + 1)]
    ts = max(max(b - a for a, b in zip(rc, rc[1:])), max(b - a for a, b in zip(cc, cc[1:])))
    ts += 2 * halo
    ts += ts % 2
    tiles = []
    for row in range(grid_rows):
        for col in range(grid_cols):
            core = Rect(rc[row], rc[row + 1], cc[col], cc[col + 1])
            oy, ox = core.y0 - halo, core.x0 - halo
            tg = Rect(oy, oy + ts, ox, ox + ts)
            cl = core.shifted(-oy, -ox)
            tiles.append(Tile(row * grid_cols + col, row, col, halo, guard, core, tg, cl,
                              cl.expanded(guard), []))
    dirs = [(0, -1, LEFT), (0, 1, RIGHT), (-1, 0, TOP), (1, 0, BOTTOM)]
    for t in tiles:
        for dr, dc, d in dirs:
            r, c = t.row + dr, t.col + dc
            if r < 0 or r >= grid_rows or c < 0 or c >= grid_cols:
                continue
            nb = tiles[r * grid_cols + c]
            gg = Rect.intersection(t.core_global.expanded(guard), nb.core_global)
            og = Rect.intersection(t.core_global, nb.core_global.expanded(guard))
            t.neighbors.append(Neighbor(
                nb.id, d, gg, gg.shifted(-t.tile_global.y0, -t.tile_global.x0),
                gg.shifted(-nb.tile_global.y0, -nb.tile_global.x0), og,
                og.shifted(-t.tile_global.y0, -t.tile_global.x0),
                og.shifted(-nb.tile_global.y0, -nb.tile_global.x0)))
    return Meta(height, width, grid_rows, grid_cols, halo, guard, ts, tiles)


def extract_local_tile(g, tile):
    """Partition::extract_local_tile (partition.cpp:83-95): periodic wrap."""
    H, W = g.shape
    ys = (tile.tile_global.y0 + np.arange(tile.tile_global.rows)) % H
    xs = (tile.tile_global.x0 + np.arange(tile.tile_global.cols)) % W
    return g[np.ix_(ys, xs)].copy()


def assemble_global(locals_, meta):
    """Partition::assemble_global (partition.cpp:105-113): Core only."""
    out = np.zeros((meta.height, meta.width))
    for t in meta.tiles:
        d, s = t.core_global, t.core_local
        out[d.y0:d.y1, d.x0:d.x1] = locals_[t.id][s.y0:s.y1, s.x0:s.x1]
    return out


def _blk(m, r):
    return m[r.y0:r.y1, r.x0:r.x1]


def linear_strength(direction, y, x, rows, cols):
    """micro_gradient_exchange.cpp:56-64."""
    if direction == LEFT:
        return 1.0 if cols == 1 else 1.0 - x / (cols - 1)
    if direction == RIGHT:
        return 1.0 if cols == 1 else x / (cols - 1)
    if direction == TOP:
        return 1.0 if rows == 1 else 1.0 - y / (rows - 1)
    return 1.0 if rows == 1 else y / (rows - 1)


@dataclasses.dataclass
class ExchangeOptions:
    """MicroGradientOptions (include/utils/micro_gradient_exchange.h:19-40)."""
    loss_type: str = "PE"            # "PE", "PEPenalty", "EPE" or "PE_EPE"
    loss_region: str = "Core"        # "Core" or "CoreGuard"
    main_region_dilation_pixels: int = 2
    pe_weight: float = 1.0
    epe_weight: float = 1.0
    penalty_weight: float = 2.0
    penalty_threshold: float = 0.01
    epe_pixel_size: float = 1.0
    collect_core_metrics: bool = False
    enable_cept: bool = False
    cept_guard_only: bool = False
    cept_weight: float = 1.1
    enable_grad_fusion: bool = False
    fusion_mode: str = "Average"     # "Average" or "Linear"
    fusion_weight_owner: float = 0.5
    fusion_weight_neighbor: float = 0.5


def loss_windows(local_target, region, opt):
    """build_micro_loss_windows (micro_gradient_exchange.cpp:65-93): (pe, penalty, epe)."""
    import cv2
    pe = np.zeros_like(local_target)
    pen = np.zeros_like(local_target)
    epe = np.zeros_like(local_target)
    sl = (slice(region.y0, region.y1), slice(region.x0, region.x1))
    pen[sl] = (local_target[sl] < 0.5)
    epe[sl] = 1.0
    pe[sl] = (local_target[sl] > 0.5) if opt.loss_type == "PEPenalty" else 1.0
    if opt.loss_type == "PE_EPE":
        main = (local_target > 0.5).astype(np.uint8)
        if opt.main_region_dilation_pixels > 0:
            main = cv2.dilate(main, np.ones((3, 3), np.uint8),
                              iterations=opt.main_region_dilation_pixels,
                              borderType=cv2.BORDER_CONSTANT, borderValue=0)
        epe[sl] = (main[sl] != 0)
        pe[sl] = 1.0 - epe[sl]
    return pe, pen, epe


def loss_weights(opt):
    """micro_loss_weights (micro_gradient_exchange.cpp:95-99): (pe, epe, penalty)."""
    return (0.0 if opt.loss_type == "EPE" else opt.pe_weight,
            opt.epe_weight if opt.loss_type in ("EPE", "PE_EPE") else 0.0,
            opt.penalty_weight if opt.loss_type == "PEPenalty" else 0.0)


def region_eps_local(eps, weights, tile, region, height, width, periodic_guard, epe_window):
    """region_eps_local (micro_gradient_exchange.cpp:18-50): the EPs (and, across the
    layout edge, their periodic copies) inside the region whose bilinear stencil touches
    the EPE window, in local coordinates, in EP order then copy order."""
    g = region.shifted(tile.tile_global.y0, tile.tile_global.x0)
    periods = 1 if periodic_guard else 0
    out, w = [], []
    for i in range(len(weights)):
        for py in range(-periods, periods + 1):
            for px in range(-periods, periods + 1):
                y = eps[i][0] + py * height
                x = eps[i][1] + px * width
                if g.y0 <= y < g.y1 and g.x0 <= x < g.x1:
                    ly, lx = y - tile.tile_global.y0, x - tile.tile_global.x0
                    st = io.bilinear_stencil(epe_window.shape[0], epe_window.shape[1], ly, lx)
                    if any(epe_window[sy, sx] != 0.0 for (sy, sx, _) in st):
                        out.append((ly, lx))
                        w.append(weights[i])
    return np.array(out, dtype=np.float64).reshape(-1, 2), np.array(w, dtype=np.float64)


def exchange(local_masks, global_target, meta, cache, thr, alpha, opt: ExchangeOptions,
             eps=None, eps_weights=None):
    """MicroGradientExchange::compute (micro_gradient_exchange.cpp:134-334)."""
    wpe, wepe, wpen = loss_weights(opt)
    evaluate_epe = opt.loss_type in ("EPE", "PE_EPE") or opt.collect_core_metrics
    eps = np.zeros((0, 2)) if eps is None else np.asarray(eps, dtype=np.float64)
    eps_weights = np.zeros(0) if eps_weights is None else np.asarray(eps_weights, dtype=np.float64)
    locals_ = []
    for t in meta.tiles:
        m = local_masks[t.id]
        tgt = extract_local_tile(global_target, t)
        aerial, wafer, E = io.imaging_compute(m, cache, thr, alpha)
        region = t.update_local if opt.loss_region == "CoreGuard" else t.core_local
        pe_w, pen_w, epe_w = loss_windows(tgt, region, opt)
        pe_loss = io.pe_loss(_blk(wafer, region), _blk(tgt, region), _blk(pe_w, region))
        bg = io.background_penalty_loss(_blk(wafer, region), _blk(tgt, region),
                                        opt.penalty_threshold, _blk(pen_w, region)) \
            if (opt.loss_type == "PEPenalty" or opt.collect_core_metrics) else 0.0
        if wpen != 0.0:
            raw = io.pe_gradient(wafer, tgt, E, cache, alpha, pe_window=pe_w, pe_weight=wpe,
                                 penalty=wpen, penalty_threshold=opt.penalty_threshold,
                                 penalty_window=pen_w)
        elif wpe != 0.0:
            raw = wpe * io.pe_gradient(wafer, tgt, E, cache, alpha, pe_window=pe_w)
        else:
            raw = np.zeros_like(m)
        epe = dict(weighted_squared_loss=0.0, absolute_sum_nm=0.0, active_count=0)
        if evaluate_epe:
            le, lw = region_eps_local(eps, eps_weights, t, region, meta.height, meta.width,
                                      opt.loss_region == "CoreGuard", epe_w)
            epe = io.evaluate_sparse_epe(aerial, le, lw, thr, opt.epe_pixel_size)
            if wepe != 0.0:
                raw = raw + wepe * io.epe_gradient(aerial, E, cache, le, lw, thr)
        data = wpe * pe_loss + wpen * bg + wepe * epe["weighted_squared_loss"]
        core = dict(pe_loss=0.0, bg_penalty_raw=0.0, pe_penalty_loss=0.0, epe_loss=0.0,
                    epe_abs_sum_nm=0.0, ep_count=0, epe_mean=0.0, data_loss=0.0)
        if opt.collect_core_metrics:
            c = t.core_local
            cw, ct = _blk(wafer, c), _blk(tgt, c)
            core["pe_loss"] = io.pe_loss(cw, ct, _blk(pe_w, c))
            core["bg_penalty_raw"] = io.background_penalty_loss(cw, ct, opt.penalty_threshold,
                                                                _blk(pen_w, c))
            core["pe_penalty_loss"] = opt.pe_weight * io.pe_loss(cw, ct, (ct > 0.5) * 1.0) + \
                opt.penalty_weight * core["bg_penalty_raw"]
            ce, cwt = region_eps_local(eps, eps_weights, t, c, meta.height, meta.width, False,
                                       epe_w)
            cev = io.evaluate_sparse_epe(aerial, ce, cwt, thr, opt.epe_pixel_size)
            core["epe_loss"] = cev["weighted_squared_loss"]
            core["epe_abs_sum_nm"] = cev["absolute_sum_nm"]
            core["ep_count"] = cev["active_count"]
            core["epe_mean"] = core["epe_abs_sum_nm"] / core["ep_count"] if core["ep_count"] else 0.0
            core["data_loss"] = wpe * core["pe_loss"] + wpen * core["bg_penalty_raw"] + \
                wepe * core["epe_loss"]
        locals_.append(dict(pe_loss=pe_loss, bg_penalty_raw=bg, penalty_loss=wpen * bg,
                            epe_loss=epe["weighted_squared_loss"],
                            epe_abs_sum_nm=epe["absolute_sum_nm"], epe_count=epe["active_count"],
                            data_loss=data, loss=data, core=core, raw=raw, grad=raw.copy(),
                            cept_loss=0.0, cept_grad=np.zeros_like(m)))
    for t in meta.tiles:
        L = locals_[t.id]
        for nb in t.neighbors:
            B = locals_[nb.id]
            g_src = nb.neighbor_overlap_local
            recv_guard = _blk(B["raw"], g_src)
            guard = nb.my_guard_local
            if opt.enable_cept:
                diff = _blk(local_masks[t.id], guard) - _blk(local_masks[nb.id], g_src)
                L["cept_loss"] += float(np.sum(diff * diff))
                L["cept_grad"][guard.y0:guard.y1, guard.x0:guard.x1] += 2.0 * diff
                if not opt.cept_guard_only:
                    ov = nb.my_overlap_local
                    d2 = _blk(local_masks[t.id], ov) - _blk(local_masks[nb.id], nb.neighbor_guard_local)
                    L["cept_grad"][ov.y0:ov.y1, ov.x0:ov.x1] += 2.0 * d2
            if opt.enable_grad_fusion:
                for y in range(guard.rows):
                    for x in range(guard.cols):
                        s = 1.0 if opt.fusion_mode == "Average" else \
                            linear_strength(nb.direction, y, x, guard.rows, guard.cols)
                        wn = opt.fusion_weight_neighbor * s
                        if wn == 0.0:
                            continue
                        lv = L["raw"][guard.y0 + y, guard.x0 + x]
                        L["grad"][guard.y0 + y, guard.x0 + x] = \
                            (opt.fusion_weight_owner * lv + wn * recv_guard[y, x]) / \
                            (opt.fusion_weight_owner + wn)
        if opt.enable_cept:
            L["grad"] = L["grad"] + opt.cept_weight * L["cept_grad"]
            L["loss"] = L["loss"] + opt.cept_weight * L["cept_loss"]
    total = sum(l["loss"] for l in locals_)
    data = sum(l["data_loss"] for l in locals_)
    cept = sum(l["cept_loss"] for l in locals_)
    return dict(locals=locals_, loss=total, data_loss=data, cept_loss=cept)


def full_chip_ctm(initial_pattern, global_target, meta, cache, thr, alpha, opt, iterations,
                  learning_rate, eps=None, eps_weights=None):
    """FullChipCTMOptimizer::optimize (source/optimizer/full_chip_ctm.cpp:25-152), CEPT guard-only."""
    opt = dataclasses.replace(opt, cept_guard_only=True)
    theta_g = io.initialize_theta(initial_pattern)
    thetas = [extract_local_tile(theta_g, t) for t in meta.tiles]
    masks = [io.theta_to_mask(th) for th in thetas]
    ev = exchange(masks, global_target, meta, cache, thr, alpha, opt, eps, eps_weights)
    history = [ev["loss"]]
    best = dict(loss=ev["loss"], iteration=0, masks=[m.copy() for m in masks])
    for it in range(1, iterations + 1):
        for t in meta.tiles:
            w = t.update_local
            th = thetas[t.id]
            g = ev["locals"][t.id]["grad"][w.y0:w.y1, w.x0:w.x1]
            gt = -0.5 * g * np.sin(th[w.y0:w.y1, w.x0:w.x1])
            th[w.y0:w.y1, w.x0:w.x1] -= learning_rate * gt
            masks[t.id] = io.theta_to_mask(th)
        ev = exchange(masks, global_target, meta, cache, thr, alpha, opt, eps, eps_weights)
        history.append(ev["loss"])
        if ev["loss"] < best["loss"]:
            best = dict(loss=ev["loss"], iteration=it, masks=[m.copy() for m in masks])
    return dict(history=history, best=best, global_mask=assemble_global(best["masks"], meta),
                thetas=thetas)


def full_chip_lsm(initial_binary, global_target, meta, cache, thr, alpha, opt: ExchangeOptions,
                  iterations, dx=1.0, dy=1.0, cfl=0.7, b=0.01, reinit_interval=20,
                  mask_type="Binary", render_scale=4, eps=None, eps_weights=None):
    """FullChipLSMOptimizer::optimize (source/optimizer/full_chip_lsm.cpp:25-254):
    Core + Guard loss region, guard-only CEPT, Core metrics, per-tile windowed RK2 with
    its own CFL dt, periodic reinitialisation inside the window, masks rendered from the
    full local phi. History rows carry the fields of full_chip_lsm.cpp:152-186."""
    from . import levelset_oracle as lo
    opt = dataclasses.replace(opt, loss_region="CoreGuard", cept_guard_only=True,
                              collect_core_metrics=True)
    wpe, wepe, _ = loss_weights(opt)

    def row(it, ev, dmin, dmax):
        L = ev["locals"]
        core = {k: sum(l["core"][k] for l in L) for k in (
            "pe_loss", "bg_penalty_raw", "pe_penalty_loss", "epe_loss", "epe_abs_sum_nm",
            "ep_count", "data_loss")}
        core["epe_mean"] = core["epe_abs_sum_nm"] / core["ep_count"] if core["ep_count"] else 0.0
        n = sum(l["epe_count"] for l in L)
        a = sum(l["epe_abs_sum_nm"] for l in L)
        return dict(iteration=it, loss=ev["loss"], data_loss=ev["data_loss"],
                    cept_loss=ev["cept_loss"], min_dt=dmin, max_dt=dmax,
                    pe_contribution=sum(wpe * l["pe_loss"] for l in L),
                    penalty_contribution=sum(l["penalty_loss"] for l in L),
                    epe_contribution=sum(wepe * l["epe_loss"] for l in L), core=core,
                    total_pe_loss=sum(l["pe_loss"] for l in L),
                    total_bg_penalty_raw=sum(l["bg_penalty_raw"] for l in L),
                    total_epe_loss=sum(l["epe_loss"] for l in L), total_epe_abs_sum_nm=a,
                    total_ep_count=n, epe_mean=a / n if n else 0.0)

    phis, masks = [], []
    for t in meta.tiles:
        m = extract_local_tile(initial_binary, t)
        phi = lo.reinit_sdf(m - 0.5, dx, dy)
        phis.append(phi)
        masks.append(lo.render_levelset_mask(phi, mask_type, render_scale))
    initial_global_phi = assemble_global(phis, meta)
    ev = exchange(masks, global_target, meta, cache, thr, alpha, opt, eps, eps_weights)
    history = [row(0, ev, 0.0, 0.0)]
    best = dict(loss=ev["loss"], iteration=0, phis=[p.copy() for p in phis],
                masks=[m.copy() for m in masks])
    for it in range(1, iterations + 1):
        nphis, nmasks, steps = [], [], []
        for t in meta.tiles:
            w = t.update_local
            win = np.zeros((meta.tile_size, meta.tile_size))
            win[w.y0:w.y1, w.x0:w.x1] = 1.0
            phi = phis[t.id]
            grad = ev["locals"][t.id]["grad"] * win
            n0, dt = lo.evolution_term(phi, grad, dx, dy, cfl, b)
            steps.append(dt)
            phi1 = phi.copy()
            phi1[w.y0:w.y1, w.x0:w.x1] += dt * n0[w.y0:w.y1, w.x0:w.x1]
            n1, _ = lo.evolution_term(phi1, grad, dx, dy, cfl, b)
            nxt = phi.copy()
            nxt[w.y0:w.y1, w.x0:w.x1] = 0.5 * phi[w.y0:w.y1, w.x0:w.x1] + 0.5 * (
                phi1[w.y0:w.y1, w.x0:w.x1] + dt * n1[w.y0:w.y1, w.x0:w.x1])
            if reinit_interval > 0 and it % reinit_interval == 0:
                signs = (nxt >= 0.0).astype(np.float64) - 0.5
                sdf = lo.reinit_sdf(signs, dx, dy)
                nxt[w.y0:w.y1, w.x0:w.x1] = sdf[w.y0:w.y1, w.x0:w.x1]
            nphis.append(nxt)
            nmasks.append(lo.render_levelset_mask(nxt, mask_type, render_scale))
        phis, masks = nphis, nmasks
        ev = exchange(masks, global_target, meta, cache, thr, alpha, opt, eps, eps_weights)
        history.append(row(it, ev, min(steps), max(steps)))
        if ev["loss"] < best["loss"]:
            best = dict(loss=ev["loss"], iteration=it, phis=[p.copy() for p in phis],
                        masks=[m.copy() for m in masks])
    return dict(history=history, best=best, global_mask=assemble_global(best["masks"], meta),
                global_phi=assemble_global(best["phis"], meta),
                initial_global_phi=initial_global_phi, final_phis=phis)
