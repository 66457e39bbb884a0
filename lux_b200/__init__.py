"""LUX-B200: B200-native LBVH and wavefront path tracing behind a C ABI.

This module is a thin ctypes binding of liblux_gpu.so (include/lux_gpu.h).  Array
arguments may be numpy arrays (host memory; the library stages them) or CUDA tensors
(anything exposing ``data_ptr()``; device memory, stream ordered).  There is no CPU
implementation behind it: if the shared library is missing or no GPU is present the
calls fail with LuxError.

Python names mirror the reference's C++ API (paths relative to the reference's src/):
    build_gpu_lbvh                bvh/gpu_bvh.cuh:51
    refit_gpu_lbvh                bvh/gpu_bvh.cuh:52
    download_bvh_for_validation   bvh/gpu_bvh.cuh:53
    intersect_gpu_bvh_stackless   bvh/gpu_bvh.cuh:60-62
    query_aabb_overlaps_self      bvh/bvh_overlap.cuh:21
    query_aabb_overlaps_cross     bvh/bvh_overlap.cuh:22-23
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "liblux_gpu.so")
# Validation build: the same sources with float sinf/cosf/powf/acosf/atan2f evaluated in
# double and rounded (LUX_ROUNDED_DOUBLE_MATH); only the rounding-isolation test uses it.
DMATH_LIBRARY_PATH = os.path.join(_HERE, "liblux_gpu_dmath.so")

LUX_OK = 0
LUX_ERR_INVALID_ARGUMENT = 1
LUX_ERR_CUDA = 2
LUX_ERR_OUT_OF_MEMORY = 3
LUX_ERR_MISMATCH = 4
LUX_ERR_DEVICE_CHECK = 5
LUX_ERR_QUEUE_OVERFLOW = 6
LUX_ERR_BUDGET = 7

PRIM_TRIANGLES = 0
PRIM_AABBS = 1

OPT_TRACE_VARIANT = 1   # 0 auto, 1 one thread per ray, 2/4 persistent (binary/4-wide), 3 4-wide
OPT_TRACE_BUDGET = 2    # traversal steps per refill round (ray queries)
OPT_PATH_BUDGET = 4     # traversal steps per refill round (path tracer)
OPT_SCRATCH_BYTES = 5   # read only: the context's reusable device scratch
OPT_STAGING_BYTES = 6   # read only: the context's reusable device staging
OPT_REFILL_BLOCKS = 7   # blocks per SM of the refilling path-tracer kernels (0: max)
OPT_RENDER_BATCH = 3    # paths in flight per wavefront batch

# Every symbol include/lux_gpu.h declares, with its ctypes signature.
_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
SIGNATURES = {
    "lux_abi_version": (ctypes.c_int, []),
    "lux_last_error": (ctypes.c_char_p, []),
    "lux_ctx_create": (ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_int, _P]),
    "lux_ctx_destroy": (ctypes.c_int, [_P]),
    "lux_ctx_set_stream": (ctypes.c_int, [_P, _P]),
    "lux_ctx_synchronize": (ctypes.c_int, [_P]),
    "lux_ctx_launch_count": (ctypes.c_int, [_P, ctypes.POINTER(_I64)]),
    "lux_ctx_set_option": (ctypes.c_int, [_P, _I32, _I64]),
    "lux_ctx_get_option": (ctypes.c_int, [_P, _I32, ctypes.POINTER(_I64)]),
    "lux_lbvh_build": (ctypes.c_int, [_P, _P, _I32, _I32, _I32, ctypes.POINTER(_P)]),
    "lux_lbvh_refit": (ctypes.c_int, [_P, _P, _P, _I32]),
    "lux_lbvh_rebuild": (ctypes.c_int, [_P, _P, _P, _I32]),
    "lux_trace_closest_stats": (ctypes.c_int, [_P, _P, _P, _I32, _P]),
    "lux_bvh_destroy": (ctypes.c_int, [_P]),
    "lux_bvh_attach_triangles": (ctypes.c_int, [_P, _P, _P, _I32]),
    "lux_bvh_info": (ctypes.c_int, [_P, _P, _P, _P, _P, _P]),
    "lux_bvh_download": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    "lux_autotune_trace": (ctypes.c_int, [_P, _P, _P, _I32, _P]),
    "lux_autotune_render": (ctypes.c_int, [_P, _P, _P, _P]),
    "lux_film_encode": (ctypes.c_int, [_P, _P, _I32, _I32, _I32, _I32, _P]),
    "lux_bvh_validate_structure": (ctypes.c_int, [_P, _P, _P, _P, _I32]),
    "lux_bvh_validate_primitives": (ctypes.c_int, [_P, _P, _P, _I32, _P, _P, _I32]),
    "lux_lbvh_morton_sort_static": (ctypes.c_int, [_P, _P, _I32, _I32, _I32, _P, _P]),
    "lux_trace_closest": (ctypes.c_int, [_P, _P, _P, _I32, _P, _P]),
    "lux_trace_any": (ctypes.c_int, [_P, _P, _P, _I32, _P]),
    "lux_camera_perspective": (ctypes.c_int, [_P, _P, ctypes.c_float, ctypes.c_float,
                                              ctypes.c_float, ctypes.c_float, _P]),
    "lux_scene_create": (ctypes.c_int, [_P, _P, ctypes.POINTER(_P)]),
    "lux_scene_destroy": (ctypes.c_int, [_P]),
    "lux_scene_info": (ctypes.c_int, [_P, _P, _P, _P]),
    "lux_scene_update_mesh": (ctypes.c_int, [_P, _P, _I32, _P]),
    "lux_scene_select_lights": (ctypes.c_int, [_P, _P, _I32, _P, _P, _I32, _P, _P, _P]),
    "lux_render_aovs": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    "lux_render_path_log": (ctypes.c_int, [_P, _P, _P, _P, _P, _I64, ctypes.POINTER(_I64)]),
    "lux_obj_load": (ctypes.c_int, [ctypes.c_char_p, _P, _P]),
    "lux_obj_mesh_free": (None, [_P]),
    "lux_render": (ctypes.c_int, [_P, _P, _P, _P]),
    "lux_render_samples": (ctypes.c_int, [_P, _P, _P, _P]),
    "lux_render_ray_counts": (ctypes.c_int, [_P, _P]),
    "lux_render_traversal_stats": (ctypes.c_int, [_P, _P, _P, _P, _P]),
    "lux_server_create": (ctypes.c_int, [ctypes.c_int, _P, _I32, _P, ctypes.POINTER(_P)]),
    "lux_server_submit": (ctypes.c_int, [_P, _I32, _P, _P, ctypes.POINTER(_I64)]),
    "lux_server_poll": (ctypes.c_int, [_P, _I64, ctypes.POINTER(_I32)]),
    "lux_server_wait": (ctypes.c_int, [_P, _I64, _I64, ctypes.POINTER(_I32)]),
    "lux_server_wait_all": (ctypes.c_int, [_P, _I64]),
    "lux_server_cancel": (ctypes.c_int, [_P, _I64]),
    "lux_server_update_mesh": (ctypes.c_int, [_P, _I32, _I32, _P]),
    "lux_server_request_times": (ctypes.c_int, [_P, _I64, _P]),
    "lux_server_stats": (ctypes.c_int, [_P, _P]),
    "lux_server_destroy": (ctypes.c_int, [_P]),
    "lux_overlap_self": (ctypes.c_int, [_P, _P, _P, _I64, _P]),
    "lux_overlap_cross": (ctypes.c_int, [_P, _P, _P, _P, _I64, _P]),
}


class LuxError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"lux status {status}: {message}")
        self.status = status


_lib = None


def load_library(path: str = LIBRARY_PATH) -> ctypes.CDLL:
    """Loads liblux_gpu.so and binds every declared entry point (no GPU needed)."""
    global _lib
    if _lib is not None and path == LIBRARY_PATH:
        return _lib
    if not os.path.exists(path):
        raise LuxError(LUX_ERR_CUDA, f"{path} is missing: run `python -m lux_b200.build`")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path == LIBRARY_PATH:
        _lib = lib
    return lib


def _check(status: int) -> None:
    if status != LUX_OK:
        msg = _lib.lux_last_error().decode(errors="replace") if _lib else ""
        raise LuxError(status, msg)


def _ptr(a):
    """Raw address of a numpy array (host) or a tensor-like object (device)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    raise TypeError(f"unsupported array type {type(a)!r}")


def _count(a, per: int) -> int:
    if isinstance(a, np.ndarray):
        return a.size // per
    return a.numel() // per


class Context:
    """A lux_ctx: one CUDA device and one stream (``stream`` is a cudaStream_t int)."""

    def __init__(self, device: int = 0, stream: int | None = None, library: str | None = None):
        """library: another build of the same ABI to bind (the validation build
        liblux_gpu_dmath.so); default the product library."""
        lib = load_library(library or LIBRARY_PATH)
        handle = _P()
        _check(lib.lux_ctx_create(ctypes.byref(handle), device, stream))
        self._h = handle
        self._lib = lib

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream: int | None) -> None:
        _check(self._lib.lux_ctx_set_stream(self._h, stream))

    def synchronize(self) -> None:
        _check(self._lib.lux_ctx_synchronize(self._h))

    def set_option(self, option: int, value: int) -> None:
        _check(self._lib.lux_ctx_set_option(self._h, option, value))

    def get_option(self, option: int) -> int:
        v = _I64()
        _check(self._lib.lux_ctx_get_option(self._h, option, ctypes.byref(v)))
        return v.value

    def launch_count(self) -> int:
        v = _I64()
        _check(self._lib.lux_ctx_launch_count(self._h, ctypes.byref(v)))
        return v.value

    def close(self) -> None:
        if self._h:
            self._lib.lux_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -------------------------------------------------------------- LBVH
    def build_lbvh(self, prims, kind: int = PRIM_TRIANGLES, morton_bits: int = 30) -> "Bvh":
        per = 9 if kind == PRIM_TRIANGLES else 6
        n = _count(prims, per)
        handle = _P()
        _check(self._lib.lux_lbvh_build(self._h, _ptr(prims), n, kind, morton_bits,
                                        ctypes.byref(handle)))
        return Bvh(self, handle, n, kind, morton_bits)


class Bvh:
    """A lux_bvh handle (device memory owned by the handle)."""

    def __init__(self, ctx: Context, handle, n: int, kind: int, morton_bits: int):
        self.ctx = ctx
        self._h = handle
        self.n = n
        self.kind = kind
        self.morton_bits = morton_bits

    @property
    def handle(self):
        return self._h

    def refit(self, prims) -> None:
        per = 9 if self.kind == PRIM_TRIANGLES else 6
        _check(self.ctx._lib.lux_lbvh_refit(self.ctx._h, self._h, _ptr(prims),
                                            _count(prims, per)))

    def attach_triangles(self, tris) -> None:
        """Makes a box BVH answer triangle ray queries (triangles in input order)."""
        _check(self.ctx._lib.lux_bvh_attach_triangles(self.ctx._h, self._h, _ptr(tris),
                                                      _count(tris, 9)))

    def rebuild(self, prims) -> None:
        per = 9 if self.kind == PRIM_TRIANGLES else 6
        n = _count(prims, per)
        _check(self.ctx._lib.lux_lbvh_rebuild(self.ctx._h, self._h, _ptr(prims), n))
        self.n = n

    def trace_stats(self, rays) -> tuple[int, int]:
        """(box tests, triangle tests) that trace_closest performs on these rays."""
        totals = np.zeros(2, np.int64)
        _check(self.ctx._lib.lux_trace_closest_stats(self.ctx._h, self._h, _ptr(rays),
                                                     _count(rays, 8), totals.ctypes.data))
        return int(totals[0]), int(totals[1])

    def root_bounds(self) -> np.ndarray:
        out = np.zeros(6, np.float32)
        _check(self.ctx._lib.lux_bvh_info(self.ctx._h, self._h, None, None, None,
                                          out.ctypes.data))
        return out

    def download(self) -> "HostTree":
        n = self.n
        count = max(2 * n - 1, 0)
        codes = np.zeros(n, np.uint64)
        ids = np.zeros(n, np.int32)
        left = np.zeros(count, np.int32)
        right = np.zeros(count, np.int32)
        bounds = np.zeros((count, 6), np.float32)
        if n > 0:
            _check(self.ctx._lib.lux_bvh_download(self.ctx._h, self._h, codes.ctypes.data,
                                                  ids.ctypes.data, left.ctypes.data,
                                                  right.ctypes.data, bounds.ctypes.data))
        return HostTree(codes, ids, left, right, bounds)

    def validate(self, prims=None) -> tuple[bool, str]:
        """validate_gpu_bvh_structure / validate_gpu_bvh_matches_primitives: (ok, message)."""
        valid = ctypes.c_int32()
        msg = ctypes.create_string_buffer(256)
        if prims is None:
            _check(self.ctx._lib.lux_bvh_validate_structure(self.ctx._h, self._h,
                                                            ctypes.byref(valid), msg, 256))
        else:
            per = 9 if self.kind == PRIM_TRIANGLES else 6
            _check(self.ctx._lib.lux_bvh_validate_primitives(
                self.ctx._h, self._h, _ptr(prims), _count(prims, per), ctypes.byref(valid),
                msg, 256))
        return bool(valid.value), msg.value.decode()

    def trace_closest(self, rays, hit_id=None, hit_t=None):
        nrays = _count(rays, 8)
        if hit_id is None:
            hit_id = np.empty(nrays, np.int32)
            hit_t = np.empty(nrays, np.float32)
        _check(self.ctx._lib.lux_trace_closest(self.ctx._h, self._h, _ptr(rays), nrays,
                                               _ptr(hit_id), _ptr(hit_t)))
        return hit_id, hit_t

    def trace_any(self, rays, hit_id=None):
        nrays = _count(rays, 8)
        if hit_id is None:
            hit_id = np.empty(nrays, np.int32)
        _check(self.ctx._lib.lux_trace_any(self.ctx._h, self._h, _ptr(rays), nrays,
                                           _ptr(hit_id)))
        return hit_id

    def overlap_self(self, max_pairs: int = 1 << 20, pairs=None):
        return _overlap(self.ctx, self, None, max_pairs, pairs)

    def overlap_cross(self, right: "Bvh", max_pairs: int = 1 << 20, pairs=None):
        return _overlap(self.ctx, self, right, max_pairs, pairs)

    def close(self) -> None:
        if self._h:
            self.ctx._lib.lux_bvh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class HostTree:
    """The reference's host tree layout (bvh/cpu_bvh.h:15-32)."""
    sorted_codes: np.ndarray
    sorted_ids: np.ndarray
    node_left: np.ndarray
    node_right: np.ndarray
    node_bounds: np.ndarray


@dataclass
class OverlapQueryResult:
    """bvh/bvh_overlap.cuh:15-19."""
    pairs: np.ndarray
    found_count: int
    truncated: bool


def _overlap(ctx, left, right, max_pairs, pairs):
    if pairs is None:
        pairs = np.zeros((max(max_pairs, 0), 2), np.int32)
    found = _I64()
    if right is None:
        _check(ctx._lib.lux_overlap_self(ctx._h, left._h, _ptr(pairs), max_pairs,
                                          ctypes.addressof(found)))
    else:
        _check(ctx._lib.lux_overlap_cross(ctx._h, left._h, right._h, _ptr(pairs), max_pairs,
                                           ctypes.addressof(found)))
    count = min(found.value, max_pairs)
    return OverlapQueryResult(pairs[:count], found.value, found.value > max_pairs)


# ------------------------------------------------------------------ reference-named API

def build_gpu_lbvh(ctx: Context, prims, kind: int = PRIM_TRIANGLES, morton_bits: int = 30):
    return ctx.build_lbvh(prims, kind, morton_bits)


def refit_gpu_lbvh(bvh: Bvh, prims) -> bool:
    """Returns False on a primitive-count mismatch, as the reference does."""
    try:
        bvh.refit(prims)
    except LuxError as e:
        if e.status == LUX_ERR_MISMATCH:
            return False
        raise
    return True


def download_bvh_for_validation(bvh: Bvh) -> HostTree:
    return bvh.download()


def intersect_gpu_bvh_stackless(bvh: Bvh, rays):
    return bvh.trace_closest(rays)


def query_aabb_overlaps_self(bvh: Bvh, max_pairs: int = 1 << 20):
    return bvh.overlap_self(max_pairs)


def query_aabb_overlaps_cross(left: Bvh, right: Bvh, max_pairs: int = 1 << 20):
    return left.overlap_cross(right, max_pairs)
