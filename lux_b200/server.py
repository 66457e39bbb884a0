"""Batched / served rendering (lux_server_*): resident scenes, one persistent path pool,
continuous batching of requests, memory-budget admission, refits between iterations."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _check, _ptr, load_library
from .scene import RenderRequest, Scene

QUEUED, RUNNING, DONE, CANCELLED, FAILED = range(5)


class ServerOptions(ctypes.Structure):
    _fields_ = [("pool_paths", ctypes.c_int64), ("memory_budget_bytes", ctypes.c_int64),
                ("max_requests", ctypes.c_int32), ("path_budget", ctypes.c_int32)]


class Server:
    def __init__(self, scenes: list[Scene], device: int = 0, pool_paths: int = 0,
                 memory_budget_bytes: int = 0, max_requests: int = 0, path_budget: int = 0):
        lib = load_library()
        self._lib = lib
        self.scenes = list(scenes)  # keep the scenes alive
        arr = (ctypes.c_void_p * len(scenes))(*[s.handle.value for s in scenes])
        opts = ServerOptions(pool_paths, memory_budget_bytes, max_requests, path_budget)
        h = ctypes.c_void_p()
        _check(lib.lux_server_create(device, arr, len(scenes), ctypes.byref(opts), ctypes.byref(h)))
        self._h = h
        self._films = {}

    def submit(self, scene: int, req: RenderRequest, film=None):
        """Queues a request; returns (request id, film array written on completion)."""
        if film is None:
            film = np.zeros((req.height, req.width, 3), np.float32)
        rid = ctypes.c_int64()
        _check(self._lib.lux_server_submit(self._h, scene, ctypes.byref(req), _ptr(film),
                                           ctypes.byref(rid)))
        self._films[rid.value] = film
        return rid.value, film

    def poll(self, rid: int) -> int:
        st = ctypes.c_int32()
        _check(self._lib.lux_server_poll(self._h, rid, ctypes.byref(st)))
        return st.value

    def wait(self, rid: int, timeout_s: float = -1) -> int:
        st = ctypes.c_int32()
        us = -1 if timeout_s < 0 else int(timeout_s * 1e6)
        _check(self._lib.lux_server_wait(self._h, rid, us, ctypes.byref(st)))
        return st.value

    def wait_all(self, timeout_s: float = -1) -> None:
        _check(self._lib.lux_server_wait_all(self._h, -1 if timeout_s < 0 else int(timeout_s * 1e6)))

    def cancel(self, rid: int) -> None:
        _check(self._lib.lux_server_cancel(self._h, rid))

    def update_mesh(self, scene: int, mesh: int, vertices: np.ndarray) -> None:
        v = np.ascontiguousarray(vertices, np.float32)
        _check(self._lib.lux_server_update_mesh(self._h, scene, mesh, v.ctypes.data))

    def times(self, rid: int) -> tuple[int, int, int]:
        """(submitted, admitted, completed) steady-clock nanoseconds."""
        t = np.zeros(3, np.int64)
        _check(self._lib.lux_server_request_times(self._h, rid, t.ctypes.data))
        return int(t[0]), int(t[1]), int(t[2])

    def stats(self) -> dict:
        s = np.zeros(9, np.int64)
        _check(self._lib.lux_server_stats(self._h, s.ctypes.data))
        keys = ["iterations", "rays", "shadow_rays", "completed", "admitted", "refits",
                "bytes_in_use", "longest_pass_ns", "longest_wait_ns"]
        return dict(zip(keys, (int(v) for v in s)))

    def close(self) -> None:
        if self._h:
            self._lib.lux_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
