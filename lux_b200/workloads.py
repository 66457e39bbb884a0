"""Seeded synthetic workloads (counter-based, reproducible byte for byte).

LBVH microbench (seed 7):
  * 1,048,576 triangles: centroid c ~ U[0,1]^3; each vertex c + u * l with u uniform on
    the unit sphere and l ~ LogNormal(ln 2e-3, 0.5);
  * 4,194,304 rays: origin ~ U[0,1]^3, direction uniform on the sphere, t in [0, inf);
  * refit input: every vertex coordinate jittered by N(0, 1e-4);
  * 1,048,576 query boxes: centre ~ U[0,1]^3, half extent 1e-3.

Every stream is SplitMix64 over (seed, stream id, counter), so any prefix of a stream
is the same whatever the total size; samples are computed in float64 and rounded to
float32 once.
"""
from __future__ import annotations

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_STREAM = np.uint64(0xD1B54A32D192ED03)

STREAM_CENTROID = 1
STREAM_VERTEX_DIR = 2
STREAM_VERTEX_LEN = 3
STREAM_RAY_ORIGIN = 4
STREAM_RAY_DIR = 5
STREAM_JITTER = 6
STREAM_QUERY = 7


def splitmix_uniform(seed: int, stream: int, count: int, offset: int = 0) -> np.ndarray:
    """count doubles in [0, 1) from SplitMix64 keyed by (seed, stream, index)."""
    with np.errstate(over="ignore"):
        idx = np.arange(offset, offset + count, dtype=np.uint64)
        z = (np.uint64(seed) * _GOLDEN + np.uint64(stream) * _STREAM
             + (idx + np.uint64(1)) * _GOLDEN)
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _unit_sphere(u0: np.ndarray, u1: np.ndarray) -> np.ndarray:
    z = 1.0 - 2.0 * u0
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = 2.0 * np.pi * u1
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=-1)


def _normal(u0: np.ndarray, u1: np.ndarray) -> np.ndarray:
    # Box-Muller; u0 in (0, 1].
    return np.sqrt(-2.0 * np.log(1.0 - u0)) * np.cos(2.0 * np.pi * u1)


def soup_triangles(n: int, seed: int = 7, median_len: float = 2e-3,
                   sigma: float = 0.5) -> np.ndarray:
    """n x 9 float32 triangle soup in the unit cube."""
    c = splitmix_uniform(seed, STREAM_CENTROID, 3 * n).reshape(n, 3)
    ud = splitmix_uniform(seed, STREAM_VERTEX_DIR, 6 * n).reshape(n, 3, 2)
    ul = splitmix_uniform(seed, STREAM_VERTEX_LEN, 6 * n).reshape(n, 3, 2)
    dirs = _unit_sphere(ud[..., 0], ud[..., 1])                      # n x 3 x 3
    lens = np.exp(np.log(median_len) + sigma * _normal(ul[..., 0], ul[..., 1]))  # n x 3
    verts = c[:, None, :] + dirs * lens[..., None]
    return verts.reshape(n, 9).astype(np.float32)


def uniform_rays(count: int, seed: int = 7) -> np.ndarray:
    """count x 8 float32 rays: origin.xyz, t_min=0, direction.xyz, t_max=inf."""
    o = splitmix_uniform(seed, STREAM_RAY_ORIGIN, 3 * count).reshape(count, 3)
    u = splitmix_uniform(seed, STREAM_RAY_DIR, 2 * count).reshape(count, 2)
    d = _unit_sphere(u[:, 0], u[:, 1])
    out = np.empty((count, 8), np.float32)
    out[:, 0:3] = o
    out[:, 3] = 0.0
    out[:, 4:7] = d
    out[:, 7] = np.inf
    return out


def jitter_triangles(tris: np.ndarray, seed: int = 7, sigma: float = 1e-4) -> np.ndarray:
    """Every coordinate plus N(0, sigma) (refit input)."""
    m = tris.size
    u = splitmix_uniform(seed, STREAM_JITTER, 2 * m).reshape(m, 2)
    noise = sigma * _normal(u[:, 0], u[:, 1])
    return (tris.astype(np.float64).reshape(-1) + noise).reshape(tris.shape).astype(np.float32)


def query_boxes(count: int, seed: int = 7, half_extent: float = 1e-3) -> np.ndarray:
    """count x 6 float32 boxes (min.xyz, max.xyz)."""
    c = splitmix_uniform(seed, STREAM_QUERY, 3 * count).reshape(count, 3)
    out = np.empty((count, 6), np.float32)
    out[:, 0:3] = c - half_extent
    out[:, 3:6] = c + half_extent
    return out


def lbvh_microbench(n_tris: int = 1 << 20, n_rays: int = 1 << 22, n_queries: int = 1 << 20,
                    seed: int = 7) -> dict:
    tris = soup_triangles(n_tris, seed)
    return {
        "triangles": tris,
        "rays": uniform_rays(n_rays, seed),
        "refit_triangles": jitter_triangles(tris, seed),
        "queries": query_boxes(n_queries, seed),
    }
