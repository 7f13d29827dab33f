"""B200 imaging-and-gradient hot path of wyhcoder/C-version-Lithography.

Host layer over the C ABI of ``liblitho_b200.so`` (declared in
``include/litho_b200.h``). It mirrors the reference's C++ classes so code and
tests read like the reference's:

===========================  =================================================
reference (C++)              here
===========================  =================================================
``ImagingCache``             :class:`ImagingCache` (device band kernels)
``Imaging::compute``         :meth:`Imaging.compute` -> :class:`ImagingResult`
``get_electric_field()``     :meth:`Imaging.get_electric_field` (band field)
``Gradient::pe_gradient*``   :meth:`Gradient.pe_gradient`,
                             :meth:`Gradient.pe_gradient_with_penalty`
``Gradient::_backpropagate`` :meth:`Gradient.backpropagate`
``Loss::pe_loss*``           :class:`Loss`
``LevelSetUtils::*``         :class:`LevelSetUtils`
``CTM_Optimizer``            :class:`CTMOptimizer`
``LSM_Optimizer``            :class:`LSMOptimizer`
``Partition``                :class:`fullchip.Partition`
``MicroGradientExchange``    :class:`fullchip.MicroGradientExchange`
``FullChipCTMOptimizer``     :class:`fullchip.FullChipCTMOptimizer`
===========================  =================================================

Images are float32 CUDA tensors (row = y, col = x). PyTorch provides device
memory and the stream; every computation runs in the library's CUDA kernels.
There is no CPU fallback: without the built library or a GPU the calls raise.
Errors raise :class:`LithoError` (``ValueError`` subclass, as the reference
throws ``std::invalid_argument``).
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblitho_b200.so")

# cudaStreamLegacy: the explicit handle of CUDA's legacy default stream.
CUDA_STREAM_LEGACY = 0x1

# Status codes (include/litho_b200.h).
LITHO_OK = 0
STATUS_NAMES = {0: "ok", 1: "invalid argument", 2: "shape mismatch", 3: "non-finite input",
                4: "out of device memory", 5: "CUDA error", 6: "field not computed",
                7: "unsupported"}

# Every exported symbol and its ctypes signature (restype, argtypes).
_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_PP = ctypes.POINTER(ctypes.c_void_p)
_PD = ctypes.POINTER(ctypes.c_double)
_PI = ctypes.POINTER(ctypes.c_int)


class PeOptions(ctypes.Structure):
    """litho_pe_options (include/litho_b200.h)."""
    _fields_ = [("pe_window", _P), ("penalty_window", _P), ("pe_weight", _D),
                ("penalty", _D), ("penalty_threshold", _D)]


class ExchangeOptionsC(ctypes.Structure):
    """litho_exchange_options (include/litho_b200.h)."""
    _fields_ = [("loss_type", _I), ("loss_region", _I), ("pe_weight", _D),
                ("penalty_weight", _D), ("penalty_threshold", _D), ("enable_cept", _I),
                ("cept_guard_only", _I), ("cept_weight", _D), ("enable_grad_fusion", _I),
                ("fusion_mode", _I), ("fusion_weight_owner", _D),
                ("fusion_weight_neighbor", _D)]


class SocsParamsC(ctypes.Structure):
    """litho_socs_params (include/litho_b200.h)."""
    _fields_ = [("N", ctypes.c_int), ("pixel_nm", ctypes.c_double),
                ("wavelength_nm", ctypes.c_double), ("na", ctypes.c_double),
                ("sigma_in", ctypes.c_double), ("sigma_out", ctypes.c_double),
                ("smoothing", ctypes.c_double), ("upsample", ctypes.c_int),
                ("num_socs", ctypes.c_int), ("compact", ctypes.c_int),
                ("zernike", ctypes.POINTER(ctypes.c_double))]


class SocsInfoC(ctypes.Structure):
    """litho_socs_info (include/litho_b200.h)."""
    _fields_ = [("K", ctypes.c_int), ("Ns", ctypes.c_int), ("Nr", ctypes.c_int),
                ("Nc", ctypes.c_int), ("row0", ctypes.c_int), ("col0", ctypes.c_int),
                ("ws_sum", ctypes.c_double), ("energy_captured", ctypes.c_double)]


class ExchangeEpeC(ctypes.Structure):
    """litho_exchange_epe (include/litho_b200.h)."""
    _fields_ = [("epe_weight", _D), ("main_region_dilation_pixels", _I), ("epe_pixel_size", _D),
                ("collect_core_metrics", _I), ("eps", _PD), ("weights", _PD), ("n_eps", _I)]


EXCHANGE_TILE_METRICS = 17

SIGNATURES = {
    "litho_version": (_I, []),
    "litho_status_string": (ctypes.c_char_p, [_I]),
    "litho_ctx_last_error": (ctypes.c_char_p, [_P]),
    "litho_ctx_create": (_I, [_I, _P, _PP]),
    "litho_ctx_destroy": (_I, [_P]),
    "litho_ctx_synchronize": (_I, [_P]),
    "litho_ctx_set_precision": (_I, [_P, _I]),
    "litho_ctx_launch_count": (ctypes.c_longlong, [_P]),
    "litho_ctx_enable_graphs": (_I, [_P, _I]),
    "litho_ctx_set_tc_schedule": (_I, [_P, _I]),
    "litho_ctx_tuned_schedule": (_I, [_P, _I, _I, _PI, _PI]),
    "litho_ctx_set_exchange_group": (_I, [_P, _I]),
    "litho_ctx_enable_stage_timing": (_I, [_P, _I]),
    "litho_ctx_stage_times": (_I, [_P, _PD, ctypes.POINTER(ctypes.c_longlong)]),
    "litho_cache_create_dense": (_I, [_P, _I, _I, _PD, _PD, _D, _PP]),
    "litho_cache_create_band": (_I, [_P, _I, _I, _I, _I, _I, _I, _PD, _PD, _D, _PP]),
    "litho_socs_prepare": (_I, [_P, _P, _PP, _P, _PD, _PD]),
    "litho_pe_gradient_batch_device": (_I, [_P, _P, _I, _P, _P, _D, _D, _D, _P, _P]),
    "litho_lsm_rk2_update_batch_device": (_I, [_P, _I, _I, _I, _P, _P, _D, _D, _D, _D, _P, _P, _P]),
    "litho_lsm_track_batch": (_I, [_P, _I, ctypes.c_longlong, _P, _D, _P, _P, _P, _P, _I, _P]),
    "litho_ctx_deferred_status": (_I, [_P]),
    "litho_cache_info": (_I, [_P, _PI, _PI, _PI, _PI, _PI, _PI]),
    "litho_cache_destroy": (_I, [_P]),
    "litho_field_create": (_I, [_P, _P, _PP]),
    "litho_field_destroy": (_I, [_P]),
    "litho_field_export": (_I, [_P, _P, _I, _P]),
    "litho_imaging_compute": (_I, [_P, _P, _P, _D, _D, _P, _P, _P]),
    "litho_backpropagate": (_I, [_P, _P, _P, _D, _P]),
    "litho_pe_gradient": (_I, [_P, _P, _P, _P, ctypes.POINTER(PeOptions), _D, _P, _PD]),
    "litho_pe_loss": (_I, [_P, _P, _P, _I, _I, ctypes.POINTER(PeOptions), _PD]),
    "litho_ctm_evaluate": (_I, [_P, _P, _P, _P, _P, _D, _D, _P, _P, _P, _P, _P, _PD, _PD]),
    "litho_ctm_evaluate_host": (_I, [_P, _P, _P, _P, _P, _D, _D, _P, _PD, _PD]),
    "litho_ctm_evaluate_batch": (_I, [_P, _P, _I, _P, _P, _D, _D, _P, _PD, _PD]),
    "litho_pe_gradient_batch": (_I, [_P, _P, _I, _P, _P, _D, _D, _P, _PD]),
    "litho_ctm_evaluate_host_batch": (_I, [_P, _P, _I, _P, _P, _D, _D, _P, _PD, _PD]),
    "litho_lsm_rk2_update_batch": (_I, [_P, _I, _I, _I, _P, _P, _D, _D, _D, _D, _P, _P, _PD]),
    "litho_weno_godunov": (_I, [_P, _I, _I, _P, _P, _D, _D, _P, _P]),
    "litho_kappa": (_I, [_P, _I, _I, _P, _D, _D, _D, _P]),
    "litho_evolution_term": (_I, [_P, _I, _I, _P, _P, _D, _D, _D, _D, _P, _PD]),
    "litho_lsm_rk2_update": (_I, [_P, _I, _I, _P, _P, _D, _D, _D, _D, _P, _P, _PD]),
    "litho_reinit_sdf": (_I, [_P, _I, _I, _P, _D, _D, _P, _P]),
    "litho_reinit_sdf_batch": (_I, [_P, _I, _I, _I, _P, _D, _D, _D, _P, _P]),
    "litho_ctx_autotune": (_I, [_P, _P, _I, _I, _I, _I, _PI, _PI]),
    "litho_ctx_reserve": (_I, [_P, _P, _I]),
    "litho_lbfgs_dots": (_I, [_P, _I, ctypes.c_longlong, _P, ctypes.c_longlong, _P, _PD]),
    "litho_lbfgs_combine": (_I, [_P, _I, ctypes.c_longlong, _P, ctypes.c_longlong, _PD, _P, _D,
                                 _P]),
    "litho_lbfgs_dots3": (_I, [_P, _I, ctypes.c_longlong, _P, ctypes.c_longlong, _P, _P, _P, _PD]),
    "litho_partition_create": (_I, [_P, _I, _I, _I, _I, _I, _I, _PP]),
    "litho_partition_create_cuts": (_I, [_P, _I, _I, _I, _PI, _I, _PI, _I, _I, _PP]),
    "litho_partition_destroy": (_I, [_P]),
    "litho_partition_info": (_I, [_P, _PI, _PI]),
    "litho_partition_tile_rects": (_I, [_P, _I, _PI]),
    "litho_partition_extract": (_I, [_P, _P, _P, _P]),
    "litho_partition_assemble": (_I, [_P, _P, _P, _P]),
    "litho_exchange_compute": (_I, [_P, _P, _P, _P, _P, _D, _D,
                                    ctypes.POINTER(ExchangeOptionsC), _P, _P, _PD, _PD]),
    "litho_exchange_compute_epe": (_I, [_P, _P, _P, _P, _P, _D, _D,
                                        ctypes.POINTER(ExchangeOptionsC),
                                        ctypes.POINTER(ExchangeEpeC), _P, _P, _PD, _PD]),
    "litho_fullchip_theta_step": (_I, [_P, _P, _P, _P, _D, _P]),
    "litho_lsm_rk2_update_noalloc": (_I, [_P, _I, _I, _P, _P, _D, _D, _D, _D, _P, _P, _PD]),
    "litho_render_levelset_mask": (_I, [_P, _I, _I, _P, _I, _I, _P]),
    "litho_evaluate_sparse_epe": (_I, [_P, _I, _I, _P, _I, _PD, _PD, _D, _D, _PD, _PD]),
    "litho_epe_gradient": (_I, [_P, _P, _P, _I, _PD, _PD, _D, _P]),
    "litho_fullchip_lsm_init": (_I, [_P, _P, _P, _D, _D, _I, _I, _P, _P]),
    "litho_fullchip_lsm_step": (_I, [_P, _P, _P, _P, _D, _D, _D, _D, _I, _I, _I, _P, _P, _PD,
                                     _PD]),
}


class LithoError(ValueError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None


def library_path() -> str:
    return LIB_PATH


def load_library(path: Optional[str] = None):
    """Load the C ABI library (no GPU needed to load it)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise LithoError(7, f"{p} is not built; run c-version-lithography_b200/build.py")
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise LithoError(5, "no CUDA device: the B200 library has no CPU path")
    return torch


def _ptr(t) -> Optional[int]:
    return None if t is None else t.data_ptr()


def _f32(t, torch, shape=None, name="array"):
    """Contiguous float32 CUDA tensor view of t (copies host data to the device)."""
    if t is None:
        return None
    if not isinstance(t, torch.Tensor):
        t = torch.as_tensor(np.asarray(t))
    if t.device.type != "cuda":
        t = t.to("cuda")
    t = t.to(torch.float32).contiguous()
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise LithoError(2, f"{name} has shape {tuple(t.shape)}, expected {tuple(shape)}")
    return t


class Context:
    """One CUDA stream plus scratch memory; used by one host thread at a time."""

    def __init__(self, device: int = 0, stream=None):
        torch = _torch()
        self.lib = load_library()
        self.torch = torch
        self.device = device
        torch.cuda.set_device(device)
        if stream is None:
            stream = torch.cuda.current_stream(device)
        self.stream = stream
        # torch's default stream is CUDA's legacy default stream (handle 0), which the
        # library would read as "create a stream of your own": pass the legacy stream's
        # explicit handle instead, so that the library's work and the caller's torch
        # work on that stream stay in one order.
        raw = stream.cuda_stream if stream.cuda_stream else CUDA_STREAM_LEGACY
        h = ctypes.c_void_p()
        self._check(self.lib.litho_ctx_create(device, ctypes.c_void_p(raw), ctypes.byref(h)), None)
        self.handle = h

    def _check(self, status, handle="self"):
        if status != LITHO_OK:
            h = self.handle if handle == "self" else handle
            msg = self.lib.litho_ctx_last_error(h).decode() if h else ""
            raise LithoError(status, msg)

    def synchronize(self):
        self._check(self.lib.litho_ctx_synchronize(self.handle))

    PRECISIONS = {"fp32": 0, "bf16x3": 1}

    def set_precision(self, mode: str):
        """'fp32' (SIMT FP32 DFT passes) or 'bf16x3' (row syntheses on tcgen05 in split-BF16)."""
        self._check(self.lib.litho_ctx_set_precision(self.handle, self.PRECISIONS[mode]))
        self.precision = mode

    @property
    def launch_count(self) -> int:
        return int(self.lib.litho_ctx_launch_count(self.handle))

    STAGES = ("tile_analysis", "tile_reduction", "band_forward", "row_synthesis_resist",
              "adjoint_tile_analysis", "adjoint_tile_reduction", "band_adjoint",
              "adjoint_row_synthesis_theta", "levelset")

    def enable_graphs(self, on: bool = True):
        """CUDA-graph replay of repeated CTM evaluations (on by default)."""
        self._check(self.lib.litho_ctx_enable_graphs(self.handle, 1 if on else 0))

    def set_exchange_group(self, max_tiles: int = 0):
        """Largest number of micro tiles per batched pass of the split-BF16 exchange
        (litho_ctx_set_exchange_group); 0: all tiles within the scratch budget."""
        self._check(self.lib.litho_ctx_set_exchange_group(self.handle, int(max_tiles)))

    TC_SCHEDULES = {"auto": 0, "per_tile": 1, "persistent": 2}

    def set_tc_schedule(self, mode: str):
        """Schedule of the split-BF16 tensor-core passes: 'auto' (the persistent
        pipelines where supported), 'per_tile' (one CTA per 128 x 128 tile) or
        'persistent' (one CTA per SM, warp-specialised, pipelined over the tiles)."""
        self._check(self.lib.litho_ctx_set_tc_schedule(self.handle, self.TC_SCHEDULES[mode]))

    def enable_stage_timing(self, on: bool = True):
        self._check(self.lib.litho_ctx_enable_stage_timing(self.handle, 1 if on else 0))

    def stage_times(self):
        """{stage: (total ms, launches)} since timing was enabled."""
        ms = (ctypes.c_double * 9)()
        cnt = (ctypes.c_longlong * 9)()
        self._check(self.lib.litho_ctx_stage_times(self.handle, ms, cnt))
        return {name: (ms[i], cnt[i]) for i, name in enumerate(self.STAGES)}

    def reserve(self, cache, batch: int):
        """Grow the device scratch to what batched calls on `batch` images of `cache`
        need (litho_ctx_reserve), so that later calls do not allocate."""
        self._check(self.lib.litho_ctx_reserve(self.handle, cache.handle, int(batch)))

    def autotune(self, cache=None, batch: int = 1, shape=None, nimg: int = 0):
        """Time the candidate schedules on this GPU and keep the fastest for the calls
        that follow (litho_ctx_autotune): with `cache`, the small-grid schedule and (split
        BF16, schedule 'auto') the tensor-core schedule for `batch` images of it; with
        `shape` (rows, cols) and nimg > 0, the chamfer CTA size of reinit_sdf for nimg
        such images. Returns the choices."""
        bw, ct = ctypes.c_int(), ctypes.c_int()
        rows, cols = shape if shape is not None else (0, 0)
        self._check(self.lib.litho_ctx_autotune(self.handle, cache.handle if cache else None,
                                                int(batch), int(rows), int(cols), int(nimg),
                                                ctypes.byref(bw), ctypes.byref(ct)))
        out = {"band_chunk_width": bw.value, "chamfer_threads": ct.value}
        if cache is not None:
            tw, ts = ctypes.c_int(), ctypes.c_int()
            self._check(self.lib.litho_ctx_tuned_schedule(self.handle, cache.N, int(batch),
                                                          ctypes.byref(tw), ctypes.byref(ts)))
            out["tc_schedule"] = {0: None, 1: "per_tile", 2: "persistent"}.get(ts.value)
        return out

    def close(self):
        if getattr(self, "handle", None):
            self.lib.litho_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context()
    return _default_ctx


class ImagingCache:
    """Device copy of the optical kernels (ImagingCache, litho_prepare.h:18-47).

    ``kernels`` are K full N x N complex frequency kernels with DC at [0, 0]
    (the reference's ``optical_kernels_frequency``), ``eigenvalues`` the SOCS
    weights (empty for Abbe) and ``source_ws`` the source weights.
    """

    def __init__(self, handle, ctx: Context):
        self.handle = handle
        self.ctx = ctx
        vals = [ctypes.c_int() for _ in range(6)]
        ctx.lib.litho_cache_info(handle, *[ctypes.byref(v) for v in vals])
        self.N, self.K, self.Nr, self.Nc, self.row0, self.col0 = [v.value for v in vals]

    @classmethod
    def from_kernels(cls, kernels, source_ws, eigenvalues=(), ctx: Optional[Context] = None):
        ctx = ctx or default_context()
        ker = np.ascontiguousarray(np.asarray(kernels, dtype=np.complex128))
        if ker.ndim != 3 or ker.shape[1] != ker.shape[2]:
            raise LithoError(2, "kernels must be K x N x N")
        K, N = ker.shape[0], ker.shape[1]
        w = np.asarray(eigenvalues if len(eigenvalues) else source_ws, dtype=np.float64)
        if w.size != K:
            raise LithoError(1, "Imaging: SOCS kernel/value counts do not match" if len(eigenvalues)
                             else "Imaging: Abbe kernel/source counts do not match")
        ws = np.asarray(source_ws, dtype=np.float64)
        if not (np.all(np.isfinite(ws)) and np.all(ws >= 0)):
            raise LithoError(1, "Imaging: source weights must be finite, nonnegative, and have a positive sum")
        flat = ker.view(np.float64).reshape(-1)
        h = ctypes.c_void_p()
        ctx._check(ctx.lib.litho_cache_create_dense(
            ctx.handle, N, K, flat.ctypes.data_as(_PD), np.ascontiguousarray(w).ctypes.data_as(_PD),
            float(ws.sum()), ctypes.byref(h)))
        return cls(h, ctx)

    @classmethod
    def from_band(cls, N, band_kernels, row0, col0, weights, ws_sum, ctx: Optional[Context] = None):
        ctx = ctx or default_context()
        kb = np.ascontiguousarray(np.asarray(band_kernels, dtype=np.complex128))
        K, Nr, Nc = kb.shape
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64))
        h = ctypes.c_void_p()
        ctx._check(ctx.lib.litho_cache_create_band(
            ctx.handle, N, K, Nr, Nc, row0, col0, kb.view(np.float64).reshape(-1).ctypes.data_as(_PD),
            w.ctypes.data_as(_PD), float(ws_sum), ctypes.byref(h)))
        return cls(h, ctx)

    def close(self):
        if getattr(self, "handle", None):
            self.ctx.lib.litho_cache_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class LithoPrepare:
    """LithoPrepare's SOCS set-up (source/litho_model/litho_prepare.cpp:16-385): the
    optics (grid N x N of pixel_nm, wavelength, NA, annular sigma_in..sigma_out, Fringe
    Zernike aberrations {index: waves}) give the source points, the shifted-pupil matrix
    and its num_socs strongest coherent modes, computed in FP64 on the device
    (litho_socs_prepare). ``cache`` is the resulting ImagingCache; ``eigenvalues`` the
    kept sigma_k^2 (largest first), ``source_ws_sum`` the image normaliser, ``info`` the
    sizes and ``band_kernels`` (K x Nr x Nc) the kernels on their band (integer
    frequencies row0.., col0..)."""

    def __init__(self, N: int, pixel_nm: float, wavelength_nm: float, na: float, sigma_in: float,
                 sigma_out: float, num_socs: int = 36, compact: bool = True, aberrations=None,
                 smoothing: float = 0.0, upsample: int = 10, ctx: Optional[Context] = None):
        ctx = ctx or default_context()
        z = None
        if aberrations:
            zc = np.zeros(11)
            for idx, c in dict(aberrations).items():
                if 1 <= int(idx) <= 11:
                    zc[int(idx) - 1] = float(c)
            z = np.ascontiguousarray(zc)
        prm = SocsParamsC(int(N), float(pixel_nm), float(wavelength_nm), float(na),
                          float(sigma_in), float(sigma_out), float(smoothing), int(upsample),
                          int(num_socs), 1 if compact else 0,
                          z.ctypes.data_as(_PD) if z is not None else None)
        info = SocsInfoC()
        h = ctypes.c_void_p()
        ctx._check(ctx.lib.litho_socs_prepare(ctx.handle, ctypes.byref(prm), ctypes.byref(h),
                                              ctypes.byref(info), None, None))
        ctx.lib.litho_cache_destroy(h)
        # second pass with buffers sized from the first (the set-up is deterministic)
        K, M = info.K, info.Nr * info.Nc
        ev = np.zeros(K)
        band = np.zeros(2 * K * M)
        h = ctypes.c_void_p()
        ctx._check(ctx.lib.litho_socs_prepare(ctx.handle, ctypes.byref(prm), ctypes.byref(h),
                                              ctypes.byref(info), ev.ctypes.data_as(_PD),
                                              band.ctypes.data_as(_PD)))
        self.cache = ImagingCache(h, ctx)
        self.eigenvalues = ev
        self.band_kernels = band.view(np.complex128).reshape(K, info.Nr, info.Nc)
        self.source_ws_sum = info.ws_sum
        self.info = {f: getattr(info, f) for f, _ in SocsInfoC._fields_}


class Field:
    """Band-domain electric-field state of one imaging call (get_electric_field())."""

    def __init__(self, cache: ImagingCache):
        self.cache = cache
        self.ctx = cache.ctx
        h = ctypes.c_void_p()
        self.ctx._check(self.ctx.lib.litho_field_create(self.ctx.handle, cache.handle, ctypes.byref(h)))
        self.handle = h

    def export(self, k: int):
        """E_k at full resolution (complex64 N x N), centred like the reference's."""
        torch = self.ctx.torch
        N = self.cache.N
        out = torch.empty((N, N, 2), dtype=torch.float32, device="cuda")
        self.ctx._check(self.ctx.lib.litho_field_export(self.ctx.handle, self.handle, k, _ptr(out)))
        return torch.view_as_complex(out)

    def fields(self) -> List:
        return [self.export(k) for k in range(self.cache.K)]

    def close(self):
        if getattr(self, "handle", None):
            self.ctx.lib.litho_field_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class ImagingResult:
    aerial_image: object
    wafer_image: object


class Imaging:
    """Imaging (include/litho_model/imaging.h:16-53)."""

    def __init__(self, cache: ImagingCache):
        self.cache = cache
        self.ctx = cache.ctx
        self.field = Field(cache)

    def compute(self, mask, threshold: float = 0.25, alpha: float = 50.0) -> ImagingResult:
        """Imaging::compute (source/litho_model/imaging.cpp:60-171)."""
        torch = self.ctx.torch
        N = self.cache.N
        m = _f32(mask, torch, (N, N), "Imaging: mask")
        aerial = torch.empty((N, N), dtype=torch.float32, device="cuda")
        wafer = torch.empty_like(aerial)
        self.ctx._check(self.ctx.lib.litho_imaging_compute(
            self.ctx.handle, self.cache.handle, _ptr(m), float(threshold), float(alpha),
            _ptr(aerial), _ptr(wafer), self.field.handle))
        return ImagingResult(aerial, wafer)

    def get_electric_field(self) -> Field:
        return self.field


class Gradient:
    """Gradient (include/utils/gradient.h:10-89)."""

    def __init__(self, cache: ImagingCache, threshold: float, alpha: float):
        self.cache = cache
        self.ctx = cache.ctx
        self.threshold = threshold
        self.alpha = alpha
        self.last_loss = None

    def backpropagate(self, dLdI, field: Field, output_scale: float):
        """Gradient::_backpropagate (source/utils/gradient.cpp:34-109)."""
        torch = self.ctx.torch
        N = self.cache.N
        g = _f32(dLdI, torch, (N, N), "Gradient: dLdI")
        out = torch.empty((N, N), dtype=torch.float32, device="cuda")
        self.ctx._check(self.ctx.lib.litho_backpropagate(self.ctx.handle, field.handle, _ptr(g),
                                                         float(output_scale), _ptr(out)))
        return out

    def _pe(self, wafer, target, field, pe_window=None, penalty_window=None, pe_weight=1.0,
            penalty=0.0, penalty_threshold=0.01):
        torch = self.ctx.torch
        N = self.cache.N
        w = _f32(wafer, torch, (N, N), "wafer_image")
        t = _f32(target, torch, (N, N), "target_image")
        pw = _f32(pe_window, torch, (N, N), "loss_window")
        qw = _f32(penalty_window, torch, (N, N), "penalty_window")
        opt = PeOptions(_ptr(pw), _ptr(qw), float(pe_weight), float(penalty), float(penalty_threshold))
        out = torch.empty((N, N), dtype=torch.float32, device="cuda")
        loss = ctypes.c_double()
        self.ctx._check(self.ctx.lib.litho_pe_gradient(
            self.ctx.handle, field.handle, _ptr(w), _ptr(t), ctypes.byref(opt), float(self.alpha),
            _ptr(out), ctypes.byref(loss)))
        self.last_loss = loss.value
        return out

    def pe_gradient(self, wafer_image, target_image, electric_field: Field, loss_window=None):
        """Gradient::pe_gradient (gradient.cpp:121-141)."""
        return self._pe(wafer_image, target_image, electric_field, pe_window=loss_window)

    def pe_gradient_with_penalty(self, wafer_image, target_image, electric_field: Field, penalty,
                                 penalty_threshold=0.01, loss_window=None, pe_weight=1.0,
                                 penalty_window=None):
        """Gradient::pe_gradient_with_penalty overloads (gradient.cpp:143-196)."""
        return self._pe(wafer_image, target_image, electric_field, pe_window=loss_window,
                        penalty_window=penalty_window, pe_weight=pe_weight, penalty=penalty,
                        penalty_threshold=penalty_threshold)

    def epe_gradient(self, aerial_image, electric_field: Field, eps, weights, threshold):
        """Gradient::epe_gradient (gradient.cpp:198-227): eps n x 2 (y, x), weights n."""
        torch = self.ctx.torch
        N = self.cache.N
        a = _f32(aerial_image, torch, (N, N), "aerial_image")
        e = np.ascontiguousarray(np.asarray(eps, dtype=np.float64).reshape(-1, 2))
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64).reshape(-1))
        if len(w) != len(e):
            raise LithoError(1, "epe_gradient: eps and weights sizes must match")
        out = torch.empty((N, N), dtype=torch.float32, device="cuda")
        self.ctx._check(self.ctx.lib.litho_epe_gradient(
            self.ctx.handle, electric_field.handle, _ptr(a), len(w), e.ctypes.data_as(_PD),
            w.ctypes.data_as(_PD), float(threshold), _ptr(out)))
        return out


@dataclass
class SparseEpeEvaluation:
    """SparseEpeEvaluation (include/utils/loss.h): per-point signed EPE and totals."""
    signed_epe_pixel: np.ndarray
    weighted_squared_loss: float
    absolute_sum_nm: float
    active_count: int


class Loss:
    """Loss statics (include/utils/loss.h:38-113) evaluated on the device."""

    @staticmethod
    def _run(wafer, target, window=None, penalty=0.0, penalty_threshold=0.01, ctx=None):
        ctx = ctx or default_context()
        torch = ctx.torch
        w = _f32(wafer, torch)
        t = _f32(target, torch, tuple(w.shape), "target")
        win = _f32(window, torch, tuple(w.shape), "loss_window")
        opt = PeOptions(_ptr(win), None, 1.0, float(penalty), float(penalty_threshold))
        out = ctypes.c_double()
        ctx._check(ctx.lib.litho_pe_loss(ctx.handle, _ptr(w), _ptr(t), w.shape[0], w.shape[1],
                                         ctypes.byref(opt), ctypes.byref(out)))
        return out.value

    @staticmethod
    def pe_loss(wafer, target, loss_window=None, ctx=None) -> float:
        return Loss._run(wafer, target, loss_window, ctx=ctx)

    @staticmethod
    def pe_loss_with_penalty(wafer, target, penalty, penalty_threshold, loss_window=None,
                             ctx=None) -> float:
        return Loss._run(wafer, target, loss_window, penalty, penalty_threshold, ctx=ctx)

    @staticmethod
    def evaluate_sparse_epe(aerial_image, eps, weights, threshold, pixel_size_nm,
                            ctx=None) -> SparseEpeEvaluation:
        """Loss::evaluate_sparse_epe (loss.cpp:125-163): eps n x 2 (y, x), weights n."""
        ctx = ctx or default_context()
        a = _f32(aerial_image, ctx.torch)
        e = np.ascontiguousarray(np.asarray(eps, dtype=np.float64).reshape(-1, 2))
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64).reshape(-1))
        if len(w) != len(e):
            raise LithoError(1, "evaluate_sparse_epe: eps and weights sizes must match")
        se = np.empty(len(w), dtype=np.float64)
        tot = (ctypes.c_double * 3)()
        ctx._check(ctx.lib.litho_evaluate_sparse_epe(
            ctx.handle, a.shape[0], a.shape[1], _ptr(a), len(w), e.ctypes.data_as(_PD),
            w.ctypes.data_as(_PD), float(threshold), float(pixel_size_nm),
            se.ctypes.data_as(_PD), tot))
        return SparseEpeEvaluation(se, tot[0], tot[1], int(round(tot[2])))


@dataclass
class EvolveParams:
    delta: object
    H1_abs: object
    H2_abs: object


class LevelSetUtils:
    """LevelSetUtils statics (include/utils/level_set_utils.h:14-33) on the device."""

    @staticmethod
    def evolve_normal_WENO_godunov(phi, Vn, dy, dx, ctx=None) -> EvolveParams:
        ctx = ctx or default_context()
        torch = ctx.torch
        p = _f32(phi, torch)
        v = _f32(Vn, torch)
        if p.shape != v.shape:
            raise LithoError(1, "evolve_normal_WENO_godunov: phi and Vn sizes must match")
        if p.dim() != 2:
            raise LithoError(2, "phi must be 2-D")
        rows, cols = p.shape
        delta = torch.empty_like(p)
        h = torch.empty_like(p)
        ctx._check(ctx.lib.litho_weno_godunov(ctx.handle, rows, cols, _ptr(p), _ptr(v), float(dy),
                                              float(dx), _ptr(delta), _ptr(h)))
        return EvolveParams(delta, h, h.clone())

    @staticmethod
    def evolve_kappa(phi, dx, dy, b, ctx=None):
        ctx = ctx or default_context()
        torch = ctx.torch
        p = _f32(phi, torch)
        out = torch.empty_like(p)
        ctx._check(ctx.lib.litho_kappa(ctx.handle, p.shape[0], p.shape[1], _ptr(p), float(dx),
                                       float(dy), float(b), _ptr(out)))
        return out

    @staticmethod
    def evolution_term(phi, Vn, dx, dy, cfl, b, ctx=None):
        """LSM_Optimizer::_caculate_evolution_term -> (normal, dt)."""
        ctx = ctx or default_context()
        torch = ctx.torch
        p = _f32(phi, torch)
        v = _f32(Vn, torch, tuple(p.shape), "Vn")
        out = torch.empty_like(p)
        dt = ctypes.c_double()
        ctx._check(ctx.lib.litho_evolution_term(ctx.handle, p.shape[0], p.shape[1], _ptr(p), _ptr(v),
                                                float(dx), float(dy), float(cfl), float(b),
                                                _ptr(out), ctypes.byref(dt)))
        return out, dt.value

    @staticmethod
    def get_dt_normal_kappa(cfl, dx, dy, H1_abs, H2_abs, b) -> float:
        """LevelSetUtils::get_dt_normal_kappa (level_set_utils.cpp:280-288), host scalar."""
        h1 = float(H1_abs.max()) if hasattr(H1_abs, "max") else float(H1_abs)
        h2 = float(H2_abs.max()) if hasattr(H2_abs, "max") else float(H2_abs)
        den = h1 / dx + h2 / dy + b * (1.0 / (dx * dx) + 1.0 / (dy * dy)) * 2
        return 1e-3 if den < 1e-9 else cfl / den

    @staticmethod
    def reinit_sdf(phi, dx, dy, ctx=None, with_mask=False):
        """LevelSetUtils::reinit_sdf (level_set_utils.cpp:290-319) on the device."""
        ctx = ctx or default_context()
        torch = ctx.torch
        p = _f32(phi, torch)
        out = torch.empty_like(p)
        mask = torch.empty_like(p) if with_mask else None
        ctx._check(ctx.lib.litho_reinit_sdf(ctx.handle, p.shape[0], p.shape[1], _ptr(p), float(dx),
                                            float(dy), _ptr(out), _ptr(mask)))
        return (out, mask) if with_mask else out

    @staticmethod
    def reinit_sdf_batch(phi, dx, dy, level=0.0, out=None, mask_out=None, ctx=None):
        """reinit_sdf of a batch (batch, rows, cols) in one launch, inside = phi > level
        (level 0.5 on binary masks: the LSM initialisation reinit_sdf(mask - 0.5)).
        Writes `out` (allocated when None) and `mask_out` (optional); returns out."""
        ctx = ctx or default_context()
        torch = ctx.torch
        p = _f32(phi, torch)
        if p.dim() != 3:
            raise LithoError(2, "phi must be (batch, rows, cols)")
        if out is None:
            out = torch.empty_like(p)
        for t in (out, mask_out):
            if t is not None and (t.shape != p.shape or t.dtype != torch.float32
                                  or not t.is_contiguous() or not t.is_cuda):
                raise LithoError(2, "outputs must be contiguous float32 CUDA tensors shaped like phi")
        ctx._check(ctx.lib.litho_reinit_sdf_batch(ctx.handle, p.shape[0], p.shape[1], p.shape[2],
                                                  _ptr(p), float(level), float(dx), float(dy),
                                                  _ptr(out), _ptr(mask_out)))
        return out

    @staticmethod
    def rk2_update_batch(phi, Vn, dx, dy, cfl, b, phi_out, mask_out=None, ctx=None):
        """rk2_update for a batch (batch, rows, cols) of images with one host round trip;
        writes phi_out (and mask_out) and returns the per-image dt."""
        ctx = ctx or default_context()
        torch = ctx.torch
        p = _f32(phi, torch)
        if p.dim() != 3:
            raise LithoError(2, "phi must be (batch, rows, cols)")
        v = _f32(Vn, torch, tuple(p.shape), "Vn")
        for t in (phi_out, mask_out):
            if t is not None and (t.shape != p.shape or t.dtype != torch.float32
                                  or not t.is_contiguous()):
                raise LithoError(2, "outputs must be contiguous float32 shaped like phi")
        B = p.shape[0]
        dts = (ctypes.c_double * B)()
        ctx._check(ctx.lib.litho_lsm_rk2_update_batch(
            ctx.handle, B, p.shape[1], p.shape[2], _ptr(p), _ptr(v), float(dx), float(dy),
            float(cfl), float(b), _ptr(phi_out), _ptr(mask_out), dts))
        return list(dts)

    @staticmethod
    def rk2_update(phi, Vn, dx, dy, cfl, b, ctx=None):
        """One RK2 update (LSM_Optimizer.cpp:109-115) -> (phi_next, mask, dt)."""
        ctx = ctx or default_context()
        torch = ctx.torch
        p = _f32(phi, torch)
        v = _f32(Vn, torch, tuple(p.shape), "Vn")
        out = torch.empty_like(p)
        mask = torch.empty_like(p)
        dt = ctypes.c_double()
        ctx._check(ctx.lib.litho_lsm_rk2_update(ctx.handle, p.shape[0], p.shape[1], _ptr(p), _ptr(v),
                                                float(dx), float(dy), float(cfl), float(b),
                                                _ptr(out), _ptr(mask), ctypes.byref(dt)))
        return out, mask, dt.value


def ctm_evaluate_batch(cache: "ImagingCache", thetas, targets, threshold: float, alpha: float,
                       grads=None):
    """The CTM objective of CTM_Optimizer::_evaluate_theta_objective
    (CTM_Optimizer.cpp:175-187) for a batch of images in one pass of the kernel chain.

    thetas, targets: (batch, N, N) float32 CUDA tensors. Returns (losses, grads, norms):
    per-image PE and ||dPE/dtheta||_2 (lists of floats) and dPE/dtheta (batch, N, N),
    written into `grads` when given. Each image's results equal its own single-image
    evaluation."""
    ctx = cache.ctx
    torch = ctx.torch
    N = cache.N
    th = _f32(thetas, torch)
    if th.dim() != 3 or th.shape[1:] != (N, N):
        raise LithoError(2, f"thetas must be (batch, {N}, {N})")
    B = th.shape[0]
    tg = _f32(targets, torch, (B, N, N), "targets")
    out = grads if grads is not None else torch.empty_like(th)
    if out.shape != th.shape or out.dtype != torch.float32 or not out.is_contiguous():
        raise LithoError(2, "grads must be a contiguous float32 tensor shaped like thetas")
    losses = (ctypes.c_double * B)()
    norms = (ctypes.c_double * B)()
    ctx._check(ctx.lib.litho_ctm_evaluate_batch(ctx.handle, cache.handle, B, _ptr(th), _ptr(tg),
                                                float(threshold), float(alpha), _ptr(out),
                                                losses, norms))
    return list(losses), out, list(norms)


def pe_gradient_batch(cache: "ImagingCache", masks, targets, threshold: float, alpha: float,
                      grads=None):
    """Imaging, PE loss and dPE/dM (Gradient::pe_gradient, gradient.cpp:121-133) for a
    batch of masks in one pass of the kernel chain.

    masks, targets: (batch, N, N) float32 CUDA tensors. Returns (losses, grads): the
    PE of every image and dPE/dM (batch, N, N), written into `grads` when given."""
    ctx = cache.ctx
    torch = ctx.torch
    N = cache.N
    m = _f32(masks, torch)
    if m.dim() != 3 or m.shape[1:] != (N, N):
        raise LithoError(2, f"masks must be (batch, {N}, {N})")
    B = m.shape[0]
    tg = _f32(targets, torch, (B, N, N), "targets")
    out = grads if grads is not None else torch.empty_like(m)
    if out.shape != m.shape or out.dtype != torch.float32 or not out.is_contiguous():
        raise LithoError(2, "grads must be a contiguous float32 tensor shaped like masks")
    losses = (ctypes.c_double * B)()
    ctx._check(ctx.lib.litho_pe_gradient_batch(ctx.handle, cache.handle, B, _ptr(m), _ptr(tg),
                                               float(threshold), float(alpha), _ptr(out), losses))
    return list(losses), out


class CTMOptimizer:
    """CTM_Optimizer (source/optimizer/CTM_Optimizer.cpp) over the fused evaluation."""

    def __init__(self, cache: ImagingCache, target, threshold, alpha, iterations, learning_rate=0.9,
                 optimizer_method="lbfgs", lbfgs_history_size=10, gradient_tolerance=0.0,
                 lbfgs_strict=True):
        if optimizer_method not in ("gradient_descent", "lbfgs"):
            raise LithoError(1, "CTM optimizer must be gradient_descent or lbfgs")
        if iterations <= 0:
            raise LithoError(1, "CTM max_iteration must be positive")
        if not (math.isfinite(learning_rate) and learning_rate > 0):
            raise LithoError(1, "CTM learning_rate must be finite and positive")
        if lbfgs_history_size <= 0:
            raise LithoError(1, "CTM lbfgs_history_size must be positive")
        if not (math.isfinite(gradient_tolerance) and gradient_tolerance >= 0):
            raise LithoError(1, "CTM gradient_tolerance must be finite and non-negative")
        self.cache = cache
        self.ctx = cache.ctx
        torch = self.ctx.torch
        N = cache.N
        self.target = _f32(target, torch, (N, N), "target")
        self.threshold, self.alpha = float(threshold), float(alpha)
        self.iterations = iterations
        self.learning_rate = learning_rate
        self.method = optimizer_method
        self.m = lbfgs_history_size
        self.tol = gradient_tolerance
        # strict: a failed L-BFGS line search raises lbfgs.LineSearchError, as LBFGS++
        # throws; False moves to the best Armijo point instead
        self.lbfgs_strict = bool(lbfgs_strict)
        self.field = Field(cache)
        self.error_history: List[float] = []
        self.grad_theta = torch.empty((N, N), dtype=torch.float32, device="cuda")
        self.mask = torch.empty_like(self.grad_theta)

    def initialize_theta(self):
        """CTM_Optimizer::_initialize_theta (CTM_Optimizer.cpp:55-64)."""
        torch = self.ctx.torch
        pi = 3.14159265358979323846
        return torch.where(self.target > 0, torch.full_like(self.target, 0.3 * pi),
                           torch.full_like(self.target, 0.7 * pi))

    def evaluate(self, theta, want_mask=False):
        """CTM_Optimizer::_evaluate_theta_objective (CTM_Optimizer.cpp:175-187)."""
        loss = ctypes.c_double()
        norm = ctypes.c_double()
        self.ctx._check(self.ctx.lib.litho_ctm_evaluate(
            self.ctx.handle, self.cache.handle, self.field.handle, _ptr(theta), _ptr(self.target),
            self.threshold, self.alpha, _ptr(self.mask) if want_mask else None, None, None, None,
            _ptr(self.grad_theta), ctypes.byref(loss), ctypes.byref(norm)))
        return loss.value, self.grad_theta, norm.value

    def optimize(self):
        return self._lbfgs() if self.method == "lbfgs" else self._gd()

    def _gd(self):
        """_optimize_gradient_descent (CTM_Optimizer.cpp:109-173)."""
        torch = self.ctx.torch
        self.error_history = []
        theta = self.initialize_theta()
        best_mask = 0.5 * (1.0 + torch.cos(theta))
        min_pe = float("inf")
        for _ in range(self.iterations):
            pe, gt, norm = self.evaluate(theta, want_mask=True)
            self.error_history.append(pe)
            if pe < min_pe:
                min_pe = pe
                best_mask = self.mask.clone()
            if norm <= self.tol:
                break
            # in place: the evaluation's buffers stay fixed, so repeats replay its CUDA graph
            theta.sub_(self.learning_rate * gt)
        self.theta = theta
        return best_mask

    def _lbfgs(self):
        """optimize_lbfgs (CTM_Optimizer.cpp:189-227): L-BFGS with FP64 two-loop scalars."""
        from .lbfgs import minimize_lbfgs
        torch = self.ctx.torch
        self.error_history = []
        theta = self.initialize_theta()

        def fg(x):
            pe, gt, norm = self.evaluate(x)
            self.error_history.append(pe)
            return pe, gt.clone(), norm

        theta, self.lbfgs_info = minimize_lbfgs(fg, theta, m=self.m, epsilon=self.tol,
                                                max_iterations=self.iterations, ctx=self.ctx,
                                                strict=self.lbfgs_strict)
        self.theta = theta
        return 0.5 * (1.0 + torch.cos(theta))


MASK_TYPES = {"Binary": 0, "Gray": 1}


def render_levelset_mask(phi, mask_type: str = "Gray", scale: int = 4, ctx=None):
    """render_levelset_mask (levelset_mask_renderer.cpp:7-33): Binary (phi >= 0) or
    Gray (subpixel coverage of the scale-times bilinear upsampling of phi)."""
    ctx = ctx or default_context()
    if mask_type not in MASK_TYPES:
        raise LithoError(1, f"mask_type must be one of {sorted(MASK_TYPES)}")
    phi = _f32(phi, ctx.torch)
    out = ctx.torch.empty_like(phi)
    ctx._check(ctx.lib.litho_render_levelset_mask(ctx.handle, phi.shape[0], phi.shape[1],
                                                  _ptr(phi), MASK_TYPES[mask_type], scale,
                                                  _ptr(out)))
    return out


@dataclass
class LevelSetResult:
    """Level_set_result of LSM_Optimizer::optimize: (best_sdf, best_mask, initial_sdf)."""
    best_sdf: object
    best_mask: object
    initial_sdf: object


class LSMOptimizer:
    """LSM_Optimizer (source/optimizer/LSM_Optimizer.cpp:60-149) over the device kernels.

    Per iteration: imaging of the current binary mask, PE (+ penalty) loss, the
    PE gradient as the normal speed, one RK2 WENO5-Godunov update with the
    first stage's dt, a chamfer re-initialisation every 20 iterations and the
    printed mask phi >= 0. Best-state bookkeeping follows the reference,
    including that best_sdf records the previous iteration's phi.
    """

    def __init__(self, cache: ImagingCache, target, threshold, alpha, dx, dy, cfl=0.5, b=0.01,
                 iterations=200, penalty=0.0, penalty_threshold=0.01):
        self.cache = cache
        self.ctx = cache.ctx
        torch = self.ctx.torch
        N = cache.N
        self.target = _f32(target, torch, (N, N), "target")
        self.threshold, self.alpha = float(threshold), float(alpha)
        self.dx, self.dy, self.cfl, self.b = float(dx), float(dy), float(cfl), float(b)
        self.iterations = int(iterations)
        self.penalty, self.penalty_threshold = float(penalty), float(penalty_threshold)
        self.imaging = Imaging(cache)
        self.gradient = Gradient(cache, threshold, alpha)
        self.error_history: List[float] = []

    def optimize(self, mask) -> LevelSetResult:
        torch = self.ctx.torch
        N = self.cache.N
        m0 = _f32(mask, torch, (N, N), "mask")
        phi_n = LevelSetUtils.reinit_sdf(m0 - 0.5, self.dx, self.dy, ctx=self.ctx)
        initial_sdf = phi_n.clone()
        phi_M = torch.zeros_like(phi_n)
        best_sdf = torch.zeros_like(phi_n)
        best_mask = m0.clone()
        temp = m0.clone()
        min_error = float("inf")
        self.error_history = []
        for i in range(self.iterations):
            r = self.imaging.compute(temp, self.threshold, self.alpha)
            if self.penalty > 0.0:
                pe = Loss.pe_loss_with_penalty(r.wafer_image, self.target, self.penalty,
                                               self.penalty_threshold, ctx=self.ctx)
            else:
                pe = Loss.pe_loss_with_penalty(r.wafer_image, self.target, 1.0, 0.01, ctx=self.ctx)
            if pe < min_error:
                min_error = pe
                best_mask = temp.clone()
                best_sdf = phi_M.clone()
            self.error_history.append(pe)
            field = self.imaging.get_electric_field()
            if self.penalty > 0.0:
                gm = self.gradient.pe_gradient_with_penalty(r.wafer_image, self.target, field,
                                                            self.penalty, self.penalty_threshold)
            else:
                gm = self.gradient.pe_gradient(r.wafer_image, self.target, field)
            phi_next, mask_next, _ = LevelSetUtils.rk2_update(phi_n, gm, self.dx, self.dy, self.cfl,
                                                              self.b, ctx=self.ctx)
            phi_M = phi_next
            if i % 20 == 0 and i > 0:
                phi_M, mask_next = LevelSetUtils.reinit_sdf(phi_M, self.dx, self.dy, ctx=self.ctx,
                                                            with_mask=True)
            phi_n = phi_M
            temp = mask_next
        return LevelSetResult(best_sdf, best_mask, initial_sdf)
