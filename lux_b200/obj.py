"""OBJ meshes through lux_obj_load (host code; no GPU needed), and the reference's asset
scenes built on them (scene/stanford_bunny.h, scene/lux_cover.h, scene/stanford_dragon.h
with the runner's cameras, app/render_runner.cpp:148-170)."""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _check, load_library
from . import scene as S

NORMALS_SOURCE, NORMALS_SMOOTH, NORMALS_FACE = 0, 1, 2
SCALE_NONE, SCALE_MAX_EXTENT, SCALE_X_EXTENT = 0, 1, 2


class ObjOptions(ctypes.Structure):
    _fields_ = [("normal_mode", ctypes.c_int32), ("reverse_orientation", ctypes.c_int32),
                ("flip_texcoord_v", ctypes.c_int32), ("scale_mode", ctypes.c_int32),
                ("target_extent", ctypes.c_float), ("center_xz", ctypes.c_int32),
                ("ground_to_y", ctypes.c_int32), ("target_y", ctypes.c_float),
                ("binding_names", ctypes.POINTER(ctypes.c_char_p)),
                ("binding_ids", ctypes.POINTER(ctypes.c_int32)),
                ("binding_count", ctypes.c_int32), ("default_material", ctypes.c_int32)]


class ObjMesh(ctypes.Structure):
    _fields_ = [("vertex_count", ctypes.c_int32), ("triangle_count", ctypes.c_int32),
                ("vertices", ctypes.POINTER(ctypes.c_float)),
                ("normals", ctypes.POINTER(ctypes.c_float)),
                ("uvs", ctypes.POINTER(ctypes.c_float)),
                ("indices", ctypes.POINTER(ctypes.c_uint32)),
                ("material_ids", ctypes.POINTER(ctypes.c_int32)),
                ("object_to_world", ctypes.c_float * 12), ("bounds", ctypes.c_float * 6),
                ("skipped_invalid", ctypes.c_int32), ("skipped_nonfinite", ctypes.c_int32),
                ("skipped_degenerate", ctypes.c_int32)]


def load_obj(path, normal_mode=NORMALS_SOURCE, reverse=False, flip_v=False,
             scale_mode=SCALE_NONE, target_extent=1.0, center_xz=False, ground_to_y=False,
             target_y=0.0, bindings=None, default_material=-1):
    """The mesh lux_obj_load makes of path (object space) and its placement, or None
    when no face survives."""
    lib = load_library()
    bindings = bindings or {}
    names = (ctypes.c_char_p * max(len(bindings), 1))(*[k.encode() for k in bindings])
    ids = (ctypes.c_int32 * max(len(bindings), 1))(*bindings.values())
    opt = ObjOptions(normal_mode, int(reverse), int(flip_v), scale_mode, target_extent,
                     int(center_xz), int(ground_to_y), target_y, names, ids, len(bindings),
                     default_material)
    out = ctypes.POINTER(ObjMesh)()
    _check(lib.lux_obj_load(os.fsencode(path), ctypes.byref(opt), ctypes.byref(out)))
    if not out:
        return None
    m = out.contents
    nv, nt = m.vertex_count, m.triangle_count
    res = {"vertices": np.ctypeslib.as_array(m.vertices, (nv, 3)).copy(),
           "normals": np.ctypeslib.as_array(m.normals, (nv, 3)).copy(),
           "uvs": np.ctypeslib.as_array(m.uvs, (nv, 2)).copy(),
           "indices": np.ctypeslib.as_array(m.indices, (nt, 3)).copy(),
           "material_ids": np.ctypeslib.as_array(m.material_ids, (nt,)).copy(),
           "object_to_world": np.array(m.object_to_world, np.float32).reshape(3, 4),
           "bounds": np.array(m.bounds, np.float32),
           "skipped": (m.skipped_invalid, m.skipped_nonfinite, m.skipped_degenerate)}
    lib.lux_obj_mesh_free(out)
    return res


def _add_loaded(b: S.SceneBuilder, mesh: dict) -> int:
    normals = mesh["normals"] if np.any(mesh["normals"] != 0) else None
    mid = b.add_mesh(S.Mesh(mesh["vertices"], mesh["indices"], mesh["material_ids"], normals,
                            mesh["uvs"]))
    b.add_instance(mid, mesh["object_to_world"])
    return mid


def bunny_scene(asset_root, width, height) -> S.SceneBuilder:
    """make_stanford_bunny_scene: floor, ceiling light and the bunny grounded at y = 0 with
    its default material turned thin Lambert."""
    f = np.float32
    b = S.SceneBuilder()
    floor = b.add_material(S.lambert((f(0.5), f(0.5), f(0.5))))
    light = b.add_material(S.emissive((15.0, 14.0, 12.0)))
    b.add_quad((-1, 0, 1), (1, 0, 1), (1, 0, -1), (-1, 0, -1), floor)
    b.add_quad((-0.3, 0.5, -0.3), (0.3, 0.5, -0.3), (0.3, 0.5, 0.3), (-0.3, 0.5, 0.3), light)
    default = len(b.materials)
    mesh = load_obj(os.path.join(asset_root, "models", "stanford-bunny.obj"), ground_to_y=True,
                    default_material=default)
    if mesh is None:
        raise RuntimeError("Stanford Bunny OBJ loaded no triangles")
    b.add_material(S.material(S.THIN_LAMBERT, (f(0.8), f(0.8), f(0.8))))
    _add_loaded(b, mesh)
    b.set_pinhole_camera((0.0, 0.3, 0.5), (-0.02, 0.11, 0.0), 40.0, float(f(width) / f(height)))
    return b


def lux_cover_scene(asset_root, width, height) -> S.SceneBuilder:
    """make_lux_cover_scene: floor and back wall, a two-sided key light and the LUX logo
    (usemtl L_lambert / U_glass / X_metal bound to Lambert, glass and metal), scaled to
    1.85 across x, centred and grounded, with smooth normals where the file has none."""
    f = np.float32
    b = S.SceneBuilder()
    floor = b.add_material(S.lambert((f(0.42), f(0.43), f(0.42))))
    key = b.add_material(S.emissive((22.0, 21.0, 19.0), two_sided=True))
    l_mat = b.add_material(S.lambert((f(0.78), f(0.76), f(0.70))))
    u_mat = b.add_material(S.dielectric((f(0.90), f(0.97), f(1.00)), f(1.5)))
    x_mat = b.add_material(S.ggx((f(0.82), f(0.78), f(0.68)), f(0.22), f(1.0)))
    b.add_quad((-2.1, 0, 0.18), (2.1, 0, 0.18), (2.1, 0, -2.2), (-2.1, 0, -2.2), floor)
    b.add_quad((-2.1, 0, 0.18), (-2.1, 1.8, 0.18), (2.1, 1.8, 0.18), (2.1, 0, 0.18), floor)
    b.add_quad((-1.25, 1.85, -0.55), (1.25, 1.85, -0.55), (1.25, 1.85, 0.80),
               (-1.25, 1.85, 0.80), key)
    mesh = load_obj(os.path.join(asset_root, "models", "LUX.obj"), normal_mode=NORMALS_SMOOTH,
                    scale_mode=SCALE_X_EXTENT, target_extent=1.85, center_xz=True,
                    ground_to_y=True,
                    bindings={"L_lambert": l_mat, "U_glass": u_mat, "X_metal": x_mat})
    if mesh is None:
        raise RuntimeError("LUX cover OBJ loaded no triangles")
    _add_loaded(b, mesh)
    b.set_pinhole_camera((0.0, 0.52, -3.0), (0.0, 0.36, 0.0), 32.0, float(f(width) / f(height)))
    return b
