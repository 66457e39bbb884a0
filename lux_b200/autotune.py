"""Autotuner bindings (lux_autotune_trace / lux_autotune_render): time candidate
tunables on the caller's workload and keep the fastest in the context."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

from . import _check, _ptr, load_library


class _TuneResult(ctypes.Structure):
    _fields_ = [("trace_variant", ctypes.c_int32), ("budget", ctypes.c_int32),
                ("render_batch", ctypes.c_int64), ("best_ms", ctypes.c_float),
                ("default_ms", ctypes.c_float), ("candidates", ctypes.c_int32),
                ("refill_blocks", ctypes.c_int32)]


@dataclass
class TuneResult:
    trace_variant: int
    budget: int
    render_batch: int
    best_ms: float
    default_ms: float
    candidates: int
    refill_blocks: int = 0


def _result(r: _TuneResult) -> TuneResult:
    return TuneResult(r.trace_variant, r.budget, r.render_batch, r.best_ms, r.default_ms,
                      r.candidates, r.refill_blocks)


def autotune_trace(ctx, bvh, rays) -> TuneResult:
    """rays: a CUDA tensor of n x 8 floats (the lux_trace_closest layout)."""
    r = _TuneResult()
    n = rays.numel() // 8
    _check(load_library().lux_autotune_trace(ctx.handle, bvh.handle, _ptr(rays), n,
                                             ctypes.byref(r)))
    return _result(r)


def autotune_render(ctx, scene, probe) -> TuneResult:
    """probe: a scene.RenderRequest the size of the renders to come."""
    r = _TuneResult()
    _check(load_library().lux_autotune_render(ctx.handle, scene.handle, ctypes.byref(probe),
                                              ctypes.byref(r)))
    return _result(r)
