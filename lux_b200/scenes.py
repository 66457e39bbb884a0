"""Seeded synthetic scenes of the heavy, batched and served workloads.

* heavy_render_scene(): the Cornell box enclosing an icosphere subdivided 7 times
  (327,680 triangles) radially displaced by seeded 3-octave value noise (amplitude 5% of
  the radius), GGX roughness 0.3, plus a dielectric icosphere (IOR 1.5, 5,120
  triangles).  The sphere centres/radii are this build's choice (the workload fixes only
  the tessellation and materials): displaced sphere at (-0.4, 1.25, 0.6), r = 0.35, above
  the short box; glass sphere at (0, 0.25, 1.65), r = 0.25, on the floor in front.
* soup_scene(): the LBVH microbench generator's triangles (Lambert) in the unit cube,
  lit by a ceiling quad and a dim uniform environment.
* sphere_grid_scene(): 16 x 16 instances of one 20,480-triangle icosphere over a floor,
  with per-instance material overrides cycling Lambert / GGX / glass / tinted filter.

All geometry is float32, generated deterministically from the seed.
"""
from __future__ import annotations

import numpy as np

from . import scene as S
from . import workloads as W


# ------------------------------------------------------------------ icosphere

def icosphere(subdivisions: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: (vertices V x 3 float64, indices T x 3 uint32), 20 * 4^s faces."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
             (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = np.array(verts, np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array(faces, np.int64)
    for _ in range(subdivisions):
        # Midpoint of every edge, shared between the two faces that use it.
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        key = np.minimum(e[:, 0], e[:, 1]) * len(v) + np.maximum(e[:, 0], e[:, 1])
        uniq, inv = np.unique(key, return_inverse=True)
        a, b = uniq // len(v), uniq % len(v)
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = (inv + len(v)).reshape(3, -1).T      # midpoint vertex of edges 01, 12, 20
        v = np.concatenate([v, mid])
        f0, f1, f2 = f[:, 0], f[:, 1], f[:, 2]
        m01, m12, m20 = m[:, 0], m[:, 1], m[:, 2]
        f = np.concatenate([np.stack([f0, m01, m20], 1), np.stack([f1, m12, m01], 1),
                            np.stack([f2, m20, m12], 1), np.stack([m01, m12, m20], 1)])
    return v, f.astype(np.uint32)


def _hash3(ix, iy, iz, seed):
    with np.errstate(over="ignore"):
        h = (ix.astype(np.uint64) * np.uint64(0x8DA6B343) ^ iy.astype(np.uint64) * np.uint64(0xD8163841)
             ^ iz.astype(np.uint64) * np.uint64(0xCB1AB31F) ^ np.uint64(seed) * np.uint64(0x9E3779B9))
        h = (h ^ (h >> np.uint64(13))) * np.uint64(0xBF58476D1CE4E5B9)
        h ^= h >> np.uint64(31)
    return (h >> np.uint64(11)).astype(np.float64) * (2.0 / 9007199254740992.0) - 1.0


def value_noise(p: np.ndarray, seed: int) -> np.ndarray:
    """Trilinear value noise in [-1, 1] with smoothstep weights, hashed lattice values."""
    q = np.floor(p)
    f = p - q
    w = f * f * (3 - 2 * f)
    i = q.astype(np.int64) + (1 << 20)
    out = np.zeros(len(p))
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                h = _hash3(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz, seed)
                wt = ((w[:, 0] if dx else 1 - w[:, 0]) * (w[:, 1] if dy else 1 - w[:, 1])
                      * (w[:, 2] if dz else 1 - w[:, 2]))
                out += wt * h
    return out


def displaced_sphere(subdivisions: int, center, radius, amplitude=0.05, seed=3,
                     octaves=3, base_frequency=2.0):
    """Icosphere displaced radially by r * amplitude * fbm(direction)."""
    v, f = icosphere(subdivisions)
    n = np.zeros(len(v))
    norm = 0.0
    for o in range(octaves):
        n += 0.5 ** o * value_noise(v * base_frequency * 2 ** o, seed + o)
        norm += 0.5 ** o
    r = radius * (1.0 + amplitude * n / norm)
    verts = (v * r[:, None] + np.asarray(center, np.float64)).astype(np.float32)
    return verts, f


def sphere(subdivisions: int, center, radius):
    v, f = icosphere(subdivisions)
    return (v * radius + np.asarray(center, np.float64)).astype(np.float32), f


# ------------------------------------------------------------------ scenes

def heavy_render_scene(width: int = 1024, height: int = 1024, seed: int = 3) -> S.SceneBuilder:
    b = S.make_cornell_scene(width, height)
    f = np.float32
    rough = b.add_material(S.ggx((f(0.8), f(0.55), f(0.35)), f(0.3), f(0.0)))
    glass = b.add_material(S.dielectric((1, 1, 1), f(1.5)))
    v, idx = displaced_sphere(7, (-0.4, 1.25, 0.6), 0.35, 0.05, seed)
    b.add_mesh(S.Mesh(v, idx, np.full(len(idx), rough, np.int32)))
    b.add_instance(len(b.meshes) - 1)
    v, idx = sphere(4, (0.0, 0.25, 1.65), 0.25)
    b.add_mesh(S.Mesh(v, idx, np.full(len(idx), glass, np.int32)))
    b.add_instance(len(b.meshes) - 1)
    return b


def soup_scene(width: int, height: int, n_tris: int = 1 << 21, seed: int = 7) -> S.SceneBuilder:
    b = S.SceneBuilder()
    f = np.float32
    white = b.add_material(S.lambert((f(0.7), f(0.7), f(0.7))))
    light = b.add_material(S.emissive((8.0, 8.0, 7.0)))
    tris = W.soup_triangles(n_tris, seed)
    n = len(tris)
    b.add_mesh(S.Mesh(tris.reshape(-1, 3).copy(), np.arange(3 * n, dtype=np.uint32).reshape(n, 3),
                      np.full(n, white, np.int32)))
    b.add_instance(0)
    b.add_quad((-0.5, 1.6, -0.5), (-0.5, 1.6, 1.5), (1.5, 1.6, 1.5), (1.5, 1.6, -0.5), light)
    b.add_uniform_infinite_light((0.1, 0.1, 0.12))
    b.set_pinhole_camera((0.5, 0.5, 2.6), (0.5, 0.5, 0.5), 40.0, float(f(width) / f(height)))
    return b


def sphere_grid_scene(width: int, height: int, grid: int = 16) -> S.SceneBuilder:
    b = S.SceneBuilder()
    f = np.float32
    floor = b.add_material(S.lambert((f(0.6), f(0.6), f(0.6))))
    light = b.add_material(S.emissive((10.0, 10.0, 9.0)))
    mats = [b.add_material(S.lambert((f(0.8), f(0.3), f(0.2)))),
            b.add_material(S.ggx((f(0.9), f(0.8), f(0.5)), f(0.25), f(1.0))),
            b.add_material(S.dielectric((1, 1, 1), f(1.5))),
            b.add_material(S.tinted_filter((f(0.3), f(0.7), f(1.0))))]
    half = grid / 2.0
    b.add_quad((-half, 0, half), (half, 0, half), (half, 0, -half), (-half, 0, -half), floor)
    b.add_quad((-2, 6, -2), (2, 6, -2), (2, 6, 2), (-2, 6, 2), light)
    b.add_uniform_infinite_light((0.15, 0.15, 0.2))
    v, idx = sphere(5, (0.0, 0.0, 0.0), 0.4)
    mesh = b.add_mesh(S.Mesh(v, idx, np.full(len(idx), mats[0], np.int32)))
    for i in range(grid):
        for j in range(grid):
            m = np.array([[1, 0, 0, i - half + 0.5], [0, 1, 0, 0.45], [0, 0, 1, j - half + 0.5]],
                         np.float32)
            b.add_instance(mesh, m, mats[(i + j) % 4])
    b.set_pinhole_camera((0.0, 9.0, 13.0), (0.0, 0.0, 0.0), 45.0, float(f(width) / f(height)))
    return b


def resident_scenes(width: int = 512, height: int = 512) -> list[S.SceneBuilder]:
    """The four scenes of the batched and served workloads (camera aspect 1)."""
    return [S.make_cornell_scene(width, height), heavy_render_scene(width, height),
            soup_scene(width, height), sphere_grid_scene(width, height)]


def batched_requests(count: int = 64, seed: int = 11, scenes: int = 4) -> list[dict]:
    """Requests of the batched workload: resolution log-uniform in 128^2..1024^2, spp
    log-uniform in 16..256, depth uniform in 4..12, scene uniform over the resident ones."""
    u = W.splitmix_uniform(seed, 21, 5 * count).reshape(count, 5)
    out = []
    for k in range(count):
        side = int(round(np.exp(np.log(128) + u[k, 0] * (np.log(1024) - np.log(128)))))
        spp = int(round(np.exp(np.log(16) + u[k, 1] * (np.log(256) - np.log(16)))))
        depth = 4 + min(8, int(u[k, 2] * 9))
        scene = min(scenes - 1, int(u[k, 3] * scenes))
        out.append({"width": side, "height": side, "spp": spp, "max_depth": depth,
                    "scene": scene, "seed": int(seed * 1000 + k)})
    return out
