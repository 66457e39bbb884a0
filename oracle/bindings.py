"""ctypes bindings of the oracle libraries -- test infrastructure only.

* Oracle: the plain-C restatement (oracle/lux_oracle.c -> oracle/liblux_oracle.so).
* Ref: the reference's own host code (oracle/_ref/libluxref.so, built from the reference
  sources by oracle/build.py; present wherever it was built).
* PT64: the FP64 high-spp path-tracing oracle (oracle/pt64.c -> oracle/liblux_pt64.so).
* RefGpu / RefPt: the reference's own GPU LBVH and GPU wavefront path tracer, compiled
  for sm_100a (oracle/_ref/libluxrefgpu.so, oracle/_ref/libluxrefpt.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liblux_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libluxref.so")
REF_GPU_LIB = os.path.join(HERE, "_ref", "libluxrefgpu.so")
REF_PT_LIB = os.path.join(HERE, "_ref", "libluxrefpt.so")
REF_DMATH_LIB = os.path.join(HERE, "_ref", "libluxref_dmath.so")
PT64_LIB = os.path.join(HERE, "liblux_pt64.so")

_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64


def _addr(a):
    return None if a is None else a.ctypes.data


class Oracle:
    def __init__(self, path: str = ORACLE_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `python oracle/build.py`")
        lib = ctypes.CDLL(path)
        lib.orc_triangle_bounds.argtypes = [_P, _I, _P]
        lib.orc_root_bounds.argtypes = [_P, _I, _P]
        lib.orc_morton30.argtypes = [_P, _I, _P, _P]
        lib.orc_morton63.argtypes = [_P, _I, _P, _P]
        lib.orc_stable_order.argtypes = [_P, _I, _P]
        lib.orc_lbvh_build.argtypes = [_P, _I, _I, _P, _P, _P, _P, _P, _P]
        lib.orc_lbvh_build.restype = _I
        lib.orc_trace.argtypes = [_P, _P, _P, _P, _I, _P, _I, _I, _I, _P, _P, _P]
        lib.orc_overlap.argtypes = [_P, _P, _P, _I, _P, _I, _I, _P, _I64]
        lib.orc_overlap.restype = _I64
        self.lib = lib

    def triangle_bounds(self, tris: np.ndarray) -> np.ndarray:
        tris = np.ascontiguousarray(tris, np.float32)
        n = tris.size // 9
        out = np.empty((n, 6), np.float32)
        self.lib.orc_triangle_bounds(tris.ctypes.data, n, out.ctypes.data)
        return out

    def build(self, bounds: np.ndarray, morton_bits: int = 30) -> dict:
        bounds = np.ascontiguousarray(bounds, np.float32)
        n = bounds.size // 6
        count = max(2 * n - 1, 0)
        out = {
            "sorted_codes": np.zeros(n, np.uint64),
            "sorted_ids": np.zeros(n, np.int32),
            "child": np.zeros(max(2 * (n - 1), 1), np.uint32),
            "node_left": np.zeros(count, np.int32),
            "node_right": np.zeros(count, np.int32),
            "node_bounds": np.zeros((count, 6), np.float32),
        }
        if n:
            self.lib.orc_lbvh_build(bounds.ctypes.data, n, morton_bits,
                                    out["sorted_codes"].ctypes.data,
                                    out["sorted_ids"].ctypes.data, out["child"].ctypes.data,
                                    out["node_left"].ctypes.data,
                                    out["node_right"].ctypes.data,
                                    out["node_bounds"].ctypes.data)
        out["n"] = n
        return out

    def trace(self, tris: np.ndarray, tree: dict, rays: np.ndarray, any_hit: bool = False,
              ignored: int = -1, stats: bool = False):
        tris = np.ascontiguousarray(tris, np.float32)
        rays = np.ascontiguousarray(rays, np.float32)
        nrays = rays.size // 8
        hit_id = np.empty(nrays, np.int32)
        hit_t = np.empty(nrays, np.float32)
        st = np.zeros((nrays, 2), np.int64) if stats else None
        self.lib.orc_trace(tris.ctypes.data, tree["node_bounds"].ctypes.data,
                           tree["child"].ctypes.data, tree["sorted_ids"].ctypes.data,
                           tree["n"], rays.ctypes.data, nrays, int(any_hit), ignored,
                           hit_id.ctypes.data, hit_t.ctypes.data, _addr(st))
        return (hit_id, hit_t, st) if stats else (hit_id, hit_t)

    def overlap(self, tree: dict, queries: np.ndarray, self_pairs: bool,
                max_pairs: int = 1 << 24):
        queries = np.ascontiguousarray(queries, np.float32)
        nq = queries.size // 6
        pairs = np.zeros((max_pairs, 2), np.int32)
        found = self.lib.orc_overlap(tree["node_bounds"].ctypes.data, tree["child"].ctypes.data,
                                     tree["sorted_ids"].ctypes.data, tree["n"],
                                     queries.ctypes.data, nq, int(self_pairs),
                                     pairs.ctypes.data, max_pairs)
        return pairs[:min(found, max_pairs)], found


class Ref:
    """The reference's own host code."""

    def __init__(self, path: str = REF_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing (built only where the reference exists)")
        lib = ctypes.CDLL(path)
        lib.ref_lbvh_build.argtypes = [_P, _I, _I, _P, _P, _P, _P, _P]
        lib.ref_lbvh_build.restype = _I
        lib.ref_build_and_trace.argtypes = [_P, _I, _P, _I, _I, _I, _P, _P]
        lib.ref_cornell_scene.argtypes = [_I, _I, _P, _P, _P, _P]
        lib.ref_cornell_scene.restype = _I
        lib.ref_cornell_render.argtypes = [_I, _I, _I, _I, ctypes.c_uint64, _I, _I, _I,
                                           _P, _P, _P]
        lib.ref_render_scene.argtypes = [_P, _I, _P, _P, _I, _P, _I, _P, _I, _I, _I, _I,
                                         ctypes.c_uint64, _I, _I, _I, _I, _P, _P, _I, _I,
                                         _P, _P]
        lib.ref_select_lights.argtypes = [_P, _I, _P, _P, _I, _P, _I, _P, _I, _P, _P, _I,
                                          _P, _P, _P]
        lib.ref_render_aovs.argtypes = [_P, _I, _P, _P, _I, _P, _I, _P, _I, _I, _I, _I,
                                        ctypes.c_uint64, _I, _P, _P, _P, _P]
        lib.ref_path_log.argtypes = [_P, _I, _P, _P, _I, _P, _I, _P, _I, _I, _I, _I,
                                     ctypes.c_uint64, _I, _P, ctypes.c_longlong]
        lib.ref_path_log.restype = ctypes.c_longlong
        lib.ref_obj_load.argtypes = [ctypes.c_char_p, _I, _I, _I, _I, ctypes.c_float, _I, _I,
                                     ctypes.c_float, _P, _P, _I, _I, _P]
        lib.ref_obj_load.restype = _P
        lib.ref_obj_copy.argtypes = [_P, _P, _P, _P, _P, _P, _P, _P]
        lib.ref_obj_free.argtypes = [_P]
        lib.ref_asset_scene.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_float, _P,
                                        _P, _P, _P]
        lib.ref_asset_render.argtypes = [ctypes.c_char_p, ctypes.c_char_p, _I, _I, _I, _I,
                                         ctypes.c_uint64, _I, _I, _I, _I, _P]
        lib.ref_tree_create.argtypes = [_P, _I, _I]
        lib.ref_tree_create.restype = _P
        lib.ref_tree_destroy.argtypes = [_P]
        lib.ref_tree_trace.argtypes = [_P, _P, _I, _I, _P, _P]
        lib.ref_desc_scene_create.argtypes = [_P]
        lib.ref_desc_scene_create.restype = _P
        lib.ref_desc_scene_destroy.argtypes = [_P]
        lib.ref_desc_render.argtypes = [_P, _P, _I, _I, _I, _I, _I, _P, _P]
        lib.ref_desc_render.restype = _I
        self.lib = lib

    def desc_scene(self, builder):
        """The reference's PreparedScene (host two-level BVH) of a lux_b200 SceneBuilder,
        built from the same lux_scene_desc that lux_scene_create receives."""
        from lux_b200 import scene as S

        desc, keep = S.scene_desc(builder)
        handle = self.lib.ref_desc_scene_create(ctypes.addressof(desc))
        del keep
        return handle

    def desc_scene_destroy(self, handle) -> None:
        self.lib.ref_desc_scene_destroy(handle)

    def desc_render(self, handle, req, rows=None, cols=None, threads=1, samples=False):
        """trace_path over the pixels rows [y0, y1) x cols [x0, x1) of the request's frame
        (lux_b200.scene.request; default the whole frame): the rectangle's film sums
        (rows x cols x 3) and, with samples=True, every sample's radiance
        (rows * cols x spp x 3, row-major)."""
        y0, y1 = rows if rows is not None else (0, req.height)
        x0, x1 = cols if cols is not None else (0, req.width)
        film = np.zeros((y1 - y0, x1 - x0, 3), np.float32)
        out = np.zeros(((y1 - y0) * (x1 - x0), req.spp, 3), np.float32) if samples else None
        self.lib.ref_desc_render(handle, ctypes.addressof(req), x0, y0, x1, y1, threads,
                                 _addr(out), film.ctypes.data)
        return (film, out) if samples else film

    def render_scene(self, tris, material_ids, materials, lights, camera, width, height, spp,
                     max_depth, seed, light_sampler=1, rows=None, threads=1, env_image=None,
                     material_ext=None, uvs=None):
        """Per-sample radiance [pixel][spp][3] of a single-mesh scene (see ref_harness.cpp).

        materials: N x 11 (type, albedo3, emission3, roughness, metallic, eta, two_sided);
        lights: L x 7 (kind, vec3, value3); camera: origin3, look_at3, vfov, aspect;
        material_ext: N x 5 (emission source, image, scale3); uvs: T x 6 corner texcoords;
        env_image: scene image 0 (also the image light's, if there is one).
        """
        tris = np.ascontiguousarray(tris, np.float32)
        mids = np.ascontiguousarray(material_ids, np.int32)
        mats = np.ascontiguousarray(materials, np.float32)
        lights = np.ascontiguousarray(lights, np.float32).reshape(-1, 7)
        cam = np.ascontiguousarray(camera, np.float32)
        y0, y1 = rows if rows is not None else (0, height)
        out = np.zeros(((y1 - y0) * width, spp, 3), np.float32)
        env = None if env_image is None else np.ascontiguousarray(env_image, np.float32)
        ext = None if material_ext is None else np.ascontiguousarray(material_ext, np.float32)
        tuv = None if uvs is None else np.ascontiguousarray(uvs, np.float32)
        self.lib.ref_render_scene(tris.ctypes.data, len(tris), mids.ctypes.data, mats.ctypes.data,
                                  len(mats), lights.ctypes.data if len(lights) else None,
                                  len(lights), cam.ctypes.data, width, height, spp, max_depth,
                                  seed, light_sampler, y0, y1, threads, out.ctypes.data,
                                  None if env is None else env.ctypes.data,
                                  0 if env is None else env.shape[1],
                                  0 if env is None else env.shape[0],
                                  None if ext is None else ext.ctypes.data,
                                  None if tuv is None else tuv.ctypes.data)
        return out

    def select_lights(self, tris, material_ids, materials, lights, camera, light_sampler,
                      positions, select_u):
        """sample_light + light_pmf of a single-mesh scene (as render_scene builds it) at
        each position: (light index or -1, the selection's pmf, light_pmf)."""
        tris = np.ascontiguousarray(tris, np.float32)
        mids = np.ascontiguousarray(material_ids, np.int32)
        mats = np.ascontiguousarray(materials, np.float32)
        lights = np.ascontiguousarray(lights, np.float32).reshape(-1, 7)
        cam = np.ascontiguousarray(camera, np.float32)
        pos = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        u = np.ascontiguousarray(select_u, np.float32).reshape(-1)
        n = len(u)
        index = np.zeros(n, np.int32)
        pmf = np.zeros(n, np.float32)
        eval_pmf = np.zeros(n, np.float32)
        self.lib.ref_select_lights(tris.ctypes.data, len(tris), mids.ctypes.data, mats.ctypes.data,
                                   len(mats), lights.ctypes.data if len(lights) else None,
                                   len(lights), cam.ctypes.data, light_sampler, pos.ctypes.data,
                                   u.ctypes.data, n, index.ctypes.data, pmf.ctypes.data,
                                   eval_pmf.ctypes.data)
        return index, pmf, eval_pmf

    def render_aovs(self, tris, material_ids, materials, lights, camera, width, height, spp,
                    max_depth, seed, light_sampler=1):
        """The reference CPU tracer's film and debug images (shadow, ng, ns), each
        height x width x 3 per-pixel sums, on a single-mesh scene."""
        tris = np.ascontiguousarray(tris, np.float32)
        mids = np.ascontiguousarray(material_ids, np.int32)
        mats = np.ascontiguousarray(materials, np.float32)
        lights = np.ascontiguousarray(lights, np.float32).reshape(-1, 7)
        cam = np.ascontiguousarray(camera, np.float32)
        out = [np.zeros((height, width, 3), np.float32) for _ in range(4)]
        self.lib.ref_render_aovs(tris.ctypes.data, len(tris), mids.ctypes.data, mats.ctypes.data,
                                 len(mats), lights.ctypes.data if len(lights) else None,
                                 len(lights), cam.ctypes.data, width, height, spp, max_depth,
                                 seed, light_sampler, *(o.ctypes.data for o in out))
        return tuple(out)

    def path_log(self, tris, material_ids, materials, lights, camera, width, height, spp,
                 max_depth, seed, light_sampler=1, dtype=None):
        """The path log records of a render on a single-mesh scene, in (sample, pixel,
        vertex) order, as a structured array of dtype (the lux_path_log_record layout)."""
        tris = np.ascontiguousarray(tris, np.float32)
        mids = np.ascontiguousarray(material_ids, np.int32)
        mats = np.ascontiguousarray(materials, np.float32)
        lights = np.ascontiguousarray(lights, np.float32).reshape(-1, 7)
        cam = np.ascontiguousarray(camera, np.float32)
        capacity = width * height * spp * (max_depth + 1)
        out = np.zeros(capacity, dtype)
        n = self.lib.ref_path_log(tris.ctypes.data, len(tris), mids.ctypes.data,
                                  mats.ctypes.data, len(mats),
                                  lights.ctypes.data if len(lights) else None, len(lights),
                                  cam.ctypes.data, width, height, spp, max_depth, seed,
                                  light_sampler, out.ctypes.data, capacity)
        assert n <= capacity
        return out[:n]

    def obj_load(self, path, normal_mode=0, reverse=False, flip_v=False, scale_mode=0,
                 target_extent=1.0, center_xz=False, ground_to_y=False, target_y=0.0,
                 bindings=None, default_material=-1):
        """The reference's load_obj_into_scene_with_result: the mesh it adds (object space)
        and its instance transform, or None when loading fails or adds nothing."""
        bindings = bindings or {}
        names = (ctypes.c_char_p * max(len(bindings), 1))(*[k.encode() for k in bindings])
        ids = np.array(list(bindings.values()) or [0], np.int32)
        counts = np.zeros(5, np.int32)
        h = self.lib.ref_obj_load(path.encode(), normal_mode, int(reverse), int(flip_v),
                                  scale_mode, target_extent, int(center_xz), int(ground_to_y),
                                  target_y, names, ids.ctypes.data, len(bindings),
                                  default_material, counts.ctypes.data)
        if not h:
            return None
        nv, nt = int(counts[0]), int(counts[1])
        out = {"vertices": np.zeros((nv, 3), np.float32), "normals": np.zeros((nv, 3), np.float32),
               "uvs": np.zeros((nv, 2), np.float32), "indices": np.zeros((nt, 3), np.uint32),
               "material_ids": np.zeros(nt, np.int32), "object_to_world": np.zeros((3, 4), np.float32),
               "bounds": np.zeros(6, np.float32)}
        self.lib.ref_obj_copy(h, *(out[k].ctypes.data for k in (
            "vertices", "normals", "uvs", "indices", "material_ids", "object_to_world", "bounds")))
        self.lib.ref_obj_free(h)
        out["skipped"] = tuple(int(c) for c in counts[2:5])
        return out

    def asset_scene(self, name, root, aspect):
        """World triangles, material ids and materials (11 floats) of the runner's asset
        scene, or None when it cannot be made."""
        counts = np.zeros(2, np.int32)
        if self.lib.ref_asset_scene(name.encode(), root.encode(), aspect, counts.ctypes.data,
                                    None, None, None) != 0:
            return None
        tris = np.zeros((counts[0], 9), np.float32)
        mids = np.zeros(counts[0], np.int32)
        mats = np.zeros((counts[1], 11), np.float32)
        self.lib.ref_asset_scene(name.encode(), root.encode(), aspect, counts.ctypes.data,
                                 tris.ctypes.data, mids.ctypes.data, mats.ctypes.data)
        return tris, mids, mats

    def asset_render(self, name, root, width, height, spp, max_depth, seed, light_sampler=1,
                     rows=None, threads=1):
        """Per-sample radiance [pixel][spp][3] of an asset scene's rows."""
        y0, y1 = rows if rows is not None else (0, height)
        out = np.zeros(((y1 - y0) * width, spp, 3), np.float32)
        st = self.lib.ref_asset_render(name.encode(), root.encode(), width, height, spp,
                                       max_depth, seed, light_sampler, y0, y1, threads,
                                       out.ctypes.data)
        assert st == 0, f"reference could not make scene {name}"
        return out

    def write_image(self, film_sum: np.ndarray, spp: int, path: str, kind: int = 0) -> bytes:
        """The reference's write_ppm (0), write_debug_ppm_linear (1) or write_pfm (2) on a
        film of sums (height, width, 3); returns the file's bytes."""
        h, w = film_sum.shape[:2]
        f = np.ascontiguousarray(film_sum, np.float32)
        self.lib.ref_write_image.argtypes = [_P, _I, _I, _I, ctypes.c_char_p, _I]
        self.lib.ref_write_image(f.ctypes.data, w, h, spp, path.encode(), kind)
        with open(path, "rb") as fh:
            return fh.read()

    def tree_create(self, prims: np.ndarray, kind: int = 0):
        """Builds and keeps a host tree (build_cpu_lbvh_tree); returns an opaque handle."""
        prims = np.ascontiguousarray(prims, np.float32)
        n = prims.size // (9 if kind == 0 else 6)
        return self.lib.ref_tree_create(prims.ctypes.data, n, kind)

    def tree_destroy(self, handle) -> None:
        self.lib.ref_tree_destroy(handle)

    def tree_trace(self, handle, rays: np.ndarray, threads: int = 1):
        """Closest hit through intersect_cpu_bvh_tree on a kept tree."""
        rays = np.ascontiguousarray(rays, np.float32)
        nrays = rays.size // 8
        hit_id = np.empty(nrays, np.int32)
        hit_t = np.empty(nrays, np.float32)
        self.lib.ref_tree_trace(handle, rays.ctypes.data, nrays, threads, hit_id.ctypes.data,
                                hit_t.ctypes.data)
        return hit_id, hit_t

    @staticmethod
    def available(path: str = REF_LIB) -> bool:
        return os.path.exists(path)

    def lbvh_build(self, prims: np.ndarray, kind: int = 0) -> dict:
        prims = np.ascontiguousarray(prims, np.float32)
        n = prims.size // (9 if kind == 0 else 6)
        count = max(2 * n - 1, 0)
        out = {
            "sorted_codes": np.zeros(n, np.uint32),
            "sorted_ids": np.zeros(n, np.int32),
            "node_left": np.zeros(count, np.int32),
            "node_right": np.zeros(count, np.int32),
            "node_bounds": np.zeros((count, 6), np.float32),
        }
        if n:
            self.lib.ref_lbvh_build(prims.ctypes.data, n, kind, out["sorted_codes"].ctypes.data,
                                    out["sorted_ids"].ctypes.data, out["node_left"].ctypes.data,
                                    out["node_right"].ctypes.data,
                                    out["node_bounds"].ctypes.data)
        return out

    def build_and_trace(self, tris: np.ndarray, rays: np.ndarray, gpu_order: bool = True,
                        threads: int = 1):
        tris = np.ascontiguousarray(tris, np.float32)
        rays = np.ascontiguousarray(rays, np.float32)
        nrays = rays.size // 8
        hit_id = np.empty(nrays, np.int32)
        hit_t = np.empty(nrays, np.float32)
        self.lib.ref_build_and_trace(tris.ctypes.data, tris.size // 9, rays.ctypes.data, nrays,
                                     0 if gpu_order else 1, threads, hit_id.ctypes.data,
                                     hit_t.ctypes.data)
        return hit_id, hit_t

    def cornell_scene(self, width: int = 256, height: int = 256) -> dict:
        tris = np.zeros((64, 9), np.float32)
        mids = np.zeros(64, np.int32)
        mats = np.zeros((16, 7), np.float32)
        cam = np.zeros(12, np.float32)
        n = self.lib.ref_cornell_scene(width, height, tris.ctypes.data, mids.ctypes.data,
                                       mats.ctypes.data, cam.ctypes.data)
        nm = int(mids[:n].max()) + 1
        return {"triangles": tris[:n], "material_ids": mids[:n], "materials": mats[:nm],
                "camera": cam.reshape(4, 3)}

    def cornell_render(self, width: int, height: int, spp: int, max_depth: int, seed: int,
                       rows=None, threads: int = 1, samples: bool = False):
        y0, y1 = rows if rows is not None else (0, height)
        total = np.zeros((height * width, 3), np.float32)
        total2 = np.zeros((height * width, 3), np.float32)
        smp = np.zeros(((y1 - y0) * width, spp, 3), np.float32) if samples else None
        self.lib.ref_cornell_render(width, height, spp, max_depth, seed, y0, y1, threads,
                                    total.ctypes.data, total2.ctypes.data, _addr(smp))
        return (total, total2, smp) if samples else (total, total2)


class PT64:
    """FP64 high-spp path-tracing oracle (oracle/pt64.c)."""

    def __init__(self, path: str = PT64_LIB):
        lib = ctypes.CDLL(path)
        lib.pt64_render.argtypes = [_P, _I, _P, _P, _I, _P, _I, _P, _I, _I, _I, _I,
                                    ctypes.c_uint64, _I, _I, _I, _I, _I, _P, _P]
        lib.pt64_render.restype = _I
        self.lib = lib

    def render(self, tris, material_ids, materials, lights, camera_frame, width, height, spp,
               max_depth, seed=1, rect=None, threads=1):
        """Per-pixel mean radiance and per-sample variance (double) over rect
        (x0, y0, x1, y1), shape (rows, cols, 3) each.  camera_frame: origin, lower_left,
        horizontal, vertical (12 floats)."""
        x0, y0, x1, y1 = rect if rect is not None else (0, 0, width, height)
        tris = np.ascontiguousarray(tris, np.float32)
        mids = np.ascontiguousarray(material_ids, np.int32)
        mats = np.ascontiguousarray(materials, np.float32)
        lights = np.ascontiguousarray(lights, np.float32).reshape(-1, 7)
        cam = np.ascontiguousarray(camera_frame, np.float32)
        mean = np.zeros((y1 - y0, x1 - x0, 3), np.float64)
        var = np.zeros_like(mean)
        self.lib.pt64_render(tris.ctypes.data, len(tris), mids.ctypes.data, mats.ctypes.data,
                             len(mats), lights.ctypes.data if len(lights) else None, len(lights),
                             cam.ctypes.data, width, height, spp, max_depth, seed, x0, y0, x1, y1,
                             threads, mean.ctypes.data, var.ctypes.data)
        return mean, var

    @staticmethod
    def available() -> bool:
        return os.path.exists(PT64_LIB)


class RefGpu:
    """The reference's own GPU LBVH (build_gpu_lbvh, intersect_gpu_bvh_stackless,
    refit_gpu_lbvh, query_aabb_overlaps_cross) compiled for sm_100a."""

    def __init__(self, path: str = REF_GPU_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing (built only where the reference exists)")
        lib = ctypes.CDLL(path)
        lib.refgpu_last_error.restype = ctypes.c_char_p
        lib.refgpu_trace.argtypes = [_P, _I, _P, _I, _P, _P]
        lib.refgpu_trace.restype = _I
        lib.refgpu_microbench.argtypes = [_P, _I, _P, _I, _P, _P, _I, _I, _I, _P, _P]
        lib.refgpu_microbench.restype = _I
        self.lib = lib

    @staticmethod
    def available(path: str = REF_GPU_LIB) -> bool:
        return os.path.exists(path)

    def _check(self, status):
        if status != 0:
            raise RuntimeError("reference GPU code: " + self.lib.refgpu_last_error().decode())

    def trace(self, tris, rays):
        """Closest hits (ids, t) of rays (8 floats each) against triangles (9 floats each)."""
        tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        hid = np.empty(len(rays), np.int32)
        ht = np.empty(len(rays), np.float32)
        self._check(self.lib.refgpu_trace(tris.ctypes.data, len(tris), rays.ctypes.data,
                                          len(rays), hid.ctypes.data, ht.ctypes.data))
        return hid, ht

    def microbench(self, tris, rays, refit_tris, queries, max_pairs=1 << 21, reps=3):
        """Median ms of each phase of the LBVH microbench step (refgpu_microbench) and the
        overlap count."""
        tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        refit = np.ascontiguousarray(refit_tris, np.float32).reshape(-1, 9)
        queries = np.ascontiguousarray(queries, np.float32).reshape(-1, 6)
        times = np.zeros(6, np.float64)
        found = np.zeros(1, np.int64)
        self._check(self.lib.refgpu_microbench(tris.ctypes.data, len(tris), rays.ctypes.data,
                                               len(rays), refit.ctypes.data, queries.ctypes.data,
                                               len(queries), max_pairs, reps, times.ctypes.data,
                                               found.ctypes.data))
        names = ("build", "trace_api", "trace_kernel", "refit", "query_build", "overlap")
        return dict(zip(names, times.tolist())), int(found[0])


class RefPt:
    """The reference's own GPU wavefront path tracer (PreparedScene::prepare_gpu +
    WavefrontPathTracer::render) compiled for sm_100a, on scenes given as lux_b200
    SceneBuilders (the same lux_scene_desc lux_scene_create receives)."""

    def __init__(self, path: str = REF_PT_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing (built only where the reference exists)")
        lib = ctypes.CDLL(path)
        lib.refpt_scene_create.argtypes = [_P, ctypes.c_char_p, _I]
        lib.refpt_scene_create.restype = _P
        lib.refpt_scene_destroy.argtypes = [_P]
        lib.refpt_render.argtypes = [_P, _P, _I, _P, _P, ctypes.c_char_p, _I]
        lib.refpt_render.restype = _I
        lib.refpt_render_path_log.argtypes = [_P, _P, _I, _P, _P, _I64, _P, ctypes.c_char_p, _I]
        lib.refpt_render_path_log.restype = _I
        self.lib = lib

    @staticmethod
    def available(path: str = REF_PT_LIB) -> bool:
        return os.path.exists(path)

    def scene(self, builder):
        from lux_b200 import scene as S

        desc, keep = S.scene_desc(builder)
        err = ctypes.create_string_buffer(512)
        handle = self.lib.refpt_scene_create(ctypes.addressof(desc), err, 512)
        del keep
        if not handle:
            raise RuntimeError("reference GPU scene: " + err.value.decode())
        return handle

    def destroy(self, handle) -> None:
        self.lib.refpt_scene_destroy(handle)

    def render(self, handle, req, batch_size=0):
        """(film sum height x width x 3, CUDA-event ms, host ms) of one render."""
        film = np.zeros((req.height, req.width, 3), np.float32)
        ms = np.zeros(2, np.float64)
        err = ctypes.create_string_buffer(512)
        status = self.lib.refpt_render(handle, ctypes.addressof(req), batch_size,
                                       film.ctypes.data, ms.ctypes.data, err, 512)
        if status != 0:
            raise RuntimeError("reference GPU render: " + err.value.decode())
        return film, float(ms[0]), float(ms[1])

    def path_log(self, handle, req, capacity=None, batch_size=0):
        """(film sum, records) with the path log on; records as
        lux_b200.scene.PATH_LOG_RECORD sorted by (sample_index, pixel_index, vertex)."""
        from lux_b200 import scene as S

        if capacity is None:
            capacity = req.width * req.height * req.spp * (req.max_depth + 1)
        film = np.zeros((req.height, req.width, 3), np.float32)
        records = np.zeros(max(int(capacity), 1), S.PATH_LOG_RECORD)
        count = np.zeros(1, np.int64)
        err = ctypes.create_string_buffer(512)
        status = self.lib.refpt_render_path_log(handle, ctypes.addressof(req), batch_size,
                                                film.ctypes.data, records.ctypes.data,
                                                int(capacity), count.ctypes.data, err, 512)
        if status < 0:
            raise RuntimeError("reference GPU path log: " + err.value.decode())
        if status > 0:
            raise RuntimeError(f"reference GPU path log: {int(count[0])} records exceed "
                               f"the capacity {capacity}")
        return film, records[:int(count[0])]


REF_SHIM_LIB = os.path.join(HERE, "_ref", "libluxshim.so")


class RefShim:
    """The drop-in shims (lux_b200/integration/) called through the reference's own types
    (oracle/ref_shim_harness.cpp; oracle/_ref/libluxshim.so, linked to liblux_gpu.so)."""

    def __init__(self, path: str = REF_SHIM_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing (built only where the reference exists)")
        lib = ctypes.CDLL(path)
        _S = ctypes.c_char_p
        lib.shim_build.argtypes = [_P, _P, _I, _S, _I]
        lib.shim_build.restype = _P
        lib.shim_destroy.argtypes = [_P]
        lib.shim_refit.argtypes = [_P, _P, _P, _I, _S, _I]
        lib.shim_refit.restype = _I
        lib.shim_download.argtypes = [_P, _P, _P, _P, _P, _P, _P, _P, _P, _S, _I]
        lib.shim_download.restype = _I
        lib.shim_validate.argtypes = [_P, _P, _P, _I, _P, _P, _S, _I]
        lib.shim_validate.restype = _I
        lib.shim_intersect.argtypes = [_P, _P, _I, _P, _I, _P, _P, _S, _I]
        lib.shim_intersect.restype = _I
        lib.shim_overlap.argtypes = [_P, _P, _I, _P, _P, _S, _I]
        lib.shim_overlap.restype = ctypes.c_longlong
        lib.shim_render.argtypes = [_P, _P, _P, _P, _P, _P, _I, _S, _I]
        lib.shim_render.restype = ctypes.c_longlong
        self.lib = lib
        self.err = ctypes.create_string_buffer(1024)

    @staticmethod
    def available(path: str = REF_SHIM_LIB) -> bool:
        return os.path.exists(path)

    def _fail(self, what):
        raise RuntimeError(f"{what}: {self.err.value.decode()}")

    def build(self, boxes, ids):
        """build_gpu_lbvh over boxes (n x 6) with primitive ids; an opaque GpuBvh*."""
        boxes = np.ascontiguousarray(boxes, np.float32).reshape(-1, 6)
        ids = np.ascontiguousarray(ids, np.int32)
        h = self.lib.shim_build(boxes.ctypes.data, ids.ctypes.data, len(ids), self.err, 1024)
        if not h and len(ids):
            self._fail("build_gpu_lbvh")
        return h

    def destroy(self, h):
        self.lib.shim_destroy(h)

    def refit(self, h, boxes, ids) -> bool:
        boxes = np.ascontiguousarray(boxes, np.float32).reshape(-1, 6)
        ids = np.ascontiguousarray(ids, np.int32)
        st = self.lib.shim_refit(h, boxes.ctypes.data, ids.ctypes.data, len(ids), self.err, 1024)
        if st < 0:
            self._fail("refit_gpu_lbvh")
        return bool(st)

    def download(self, h, n):
        """download_bvh_for_validation as arrays, plus GpuBvh::root_bounds."""
        m = max(2 * n - 1, 1)
        out = {k: np.zeros(m, np.int32) for k in ("left", "right", "first", "count")}
        bounds = np.zeros((m, 6), np.float32)
        pids = np.zeros(max(n, 1), np.int32)
        root = np.zeros(1, np.int32)
        rb = np.zeros(6, np.float32)
        k = self.lib.shim_download(h, root.ctypes.data, out["left"].ctypes.data,
                                   out["right"].ctypes.data, out["first"].ctypes.data,
                                   out["count"].ctypes.data, bounds.ctypes.data, pids.ctypes.data,
                                   rb.ctypes.data, self.err, 1024)
        if k < 0:
            self._fail("download_bvh_for_validation")
        out = {key: v[:k] for key, v in out.items()}
        out.update(bounds=bounds[:k], primitive_ids=pids[:n], root=int(root[0]), root_bounds=rb)
        return out

    def validate(self, h, boxes, ids):
        """(validate_gpu_bvh_structure, validate_gpu_bvh_matches_primitives, message)."""
        boxes = np.ascontiguousarray(boxes, np.float32).reshape(-1, 6)
        ids = np.ascontiguousarray(ids, np.int32)
        s, m = ctypes.c_int(), ctypes.c_int()
        msg = ctypes.create_string_buffer(512)
        if self.lib.shim_validate(h, boxes.ctypes.data, ids.ctypes.data, len(ids),
                                  ctypes.byref(s), ctypes.byref(m), msg, 512) < 0:
            raise RuntimeError("validators: " + msg.value.decode())
        return bool(s.value), bool(m.value), msg.value.decode()

    def intersect(self, h, tris_by_id, rays):
        tris = np.ascontiguousarray(tris_by_id, np.float32).reshape(-1, 9)
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        hid = np.zeros(len(rays), np.int32)
        ht = np.zeros(len(rays), np.float32)
        if self.lib.shim_intersect(h, tris.ctypes.data, len(tris), rays.ctypes.data, len(rays),
                                   hid.ctypes.data, ht.ctypes.data, self.err, 1024) < 0:
            self._fail("intersect_gpu_bvh_stackless")
        return hid, ht

    def overlap(self, left, right, max_pairs):
        """(pairs k x 2, found_count, truncated) of query_aabb_overlaps_self (right None)
        or query_aabb_overlaps_cross."""
        pairs = np.zeros((max(max_pairs, 1), 2), np.int32)
        trunc = ctypes.c_int()
        found = self.lib.shim_overlap(left, right, max_pairs, pairs.ctypes.data,
                                      ctypes.byref(trunc), self.err, 1024)
        if found < 0:
            self._fail("query_aabb_overlaps")
        return pairs[:min(found, max_pairs)], int(found), bool(trunc.value)

    def render(self, builder, req, aovs=False, path_log=False):
        """make_integrator(WavefrontPathTracer)->render on the reference's Scene (the
        reference's Cornell box when builder is None): (film, shadow, ng, ns, log count)."""
        from lux_b200 import scene as S

        keep = None
        desc_ptr = None
        if builder is not None:
            desc, keep = S.scene_desc(builder)
            desc_ptr = ctypes.addressof(desc)
        shape = (req.height, req.width, 3)
        film = np.zeros(shape, np.float32)
        extra = [np.zeros(shape, np.float32) if aovs else None for _ in range(3)]
        n = self.lib.shim_render(desc_ptr, ctypes.addressof(req), film.ctypes.data,
                                 *(_addr(a) for a in extra), int(path_log), self.err, 1024)
        del keep
        if n < 0:
            self._fail("WavefrontPathTracer::render")
        return film, extra[0], extra[1], extra[2], int(n)
