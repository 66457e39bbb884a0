"""Scenes and rendering through the C ABI (lux_scene_create / lux_render).

SceneBuilder mirrors the reference's scene authoring calls (scene/scene_edit.h:
add_triangle, add_quad; scene/scene_build.h: add_point_light, add_distant_light,
add_uniform_infinite_light; instances of meshes with transforms), and
make_cornell_scene() restates the reference's built-in Cornell box
(scene/cornell_box.h:31-56) with the camera of app/render_runner.cpp:85-90.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _check, _ptr, load_library

LAMBERT, THIN_LAMBERT, GGX, DIELECTRIC, INTERFACE, TRANSPARENT = range(6)
LIGHT_POINT, LIGHT_DISTANT, LIGHT_UNIFORM_INFINITE, LIGHT_IMAGE_INFINITE = 1, 2, 3, 4
SAMPLER_UNIFORM, SAMPLER_POWER, SAMPLER_TREE = 0, 1, 2   # LightSamplerKind (Uniform, Power, Bvh)

_F3 = ctypes.c_float * 3
_F12 = ctypes.c_float * 12


class Material(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("albedo", _F3), ("emission", _F3),
                ("emission_two_sided", ctypes.c_int32), ("roughness", ctypes.c_float),
                ("metallic", ctypes.c_float), ("eta", ctypes.c_float),
                ("emission_source", ctypes.c_int32), ("emission_image", ctypes.c_int32),
                ("emission_scale", _F3)]


class MeshDesc(ctypes.Structure):
    _fields_ = [("vertices", ctypes.c_void_p), ("normals", ctypes.c_void_p),
                ("uvs", ctypes.c_void_p), ("vertex_count", ctypes.c_int32),
                ("indices", ctypes.c_void_p), ("material_ids", ctypes.c_void_p),
                ("triangle_count", ctypes.c_int32)]


class InstanceDesc(ctypes.Structure):
    _fields_ = [("mesh", ctypes.c_int32), ("material_override", ctypes.c_int32),
                ("object_to_world", _F12), ("world_to_object", _F12)]


class LightDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("vec", _F3), ("value", _F3), ("image", ctypes.c_int32)]


class EnvImageDesc(ctypes.Structure):
    _fields_ = [("pixels", ctypes.c_void_p), ("width", ctypes.c_int32),
                ("height", ctypes.c_int32)]


class CameraDesc(ctypes.Structure):
    _fields_ = [("origin", _F3), ("lower_left", _F3), ("horizontal", _F3), ("vertical", _F3),
                ("lens_u", _F3), ("lens_v", _F3), ("lens_radius", ctypes.c_float)]


class SceneDesc(ctypes.Structure):
    _fields_ = [("materials", ctypes.c_void_p), ("material_count", ctypes.c_int32),
                ("meshes", ctypes.c_void_p), ("mesh_count", ctypes.c_int32),
                ("instances", ctypes.c_void_p), ("instance_count", ctypes.c_int32),
                ("lights", ctypes.c_void_p), ("light_count", ctypes.c_int32),
                ("camera", CameraDesc), ("images", ctypes.c_void_p),
                ("image_count", ctypes.c_int32)]


class RenderRequest(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32), ("spp", ctypes.c_int32),
                ("max_depth", ctypes.c_int32), ("seed", ctypes.c_uint64),
                ("frame_index", ctypes.c_int32), ("sample_offset", ctypes.c_int32),
                ("light_sampler", ctypes.c_int32)]


def material(kind: int, albedo=(0.8, 0.8, 0.8), emission=(0, 0, 0), roughness=0.5,
             metallic=0.0, eta=1.5, two_sided=False) -> Material:
    """Material constructors of material/material.h:43-103."""
    return Material(kind, _F3(*albedo), _F3(*emission), int(two_sided), roughness, metallic, eta)


def lambert(albedo):
    return material(LAMBERT, albedo)


def emissive(emission, albedo=(0, 0, 0), two_sided=False):
    return material(LAMBERT, albedo, emission, two_sided=two_sided)


def ggx(albedo, roughness, metallic=0.0):
    return material(GGX, albedo, roughness=roughness, metallic=metallic)


def dielectric(albedo=(1, 1, 1), eta=1.5):
    return material(DIELECTRIC, albedo, roughness=0.0, metallic=0.0, eta=eta)


def image_emissive(image, scale=(1, 1, 1), albedo=(0, 0, 0), two_sided=False):
    """Material::image_emissive: emission read from scene image `image` at the surface's
    texture coordinates (nearest texel), times scale."""
    m = material(LAMBERT, albedo, (0, 0, 0), two_sided=two_sided)
    m.emission_source = 1
    m.emission_image = image
    m.emission_scale = _F3(*scale)
    return m


def tinted_filter(transmittance=(1, 1, 1)):
    return material(TRANSPARENT, transmittance)


def interface():
    return material(INTERFACE, (1, 1, 1))


IDENTITY = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0]], np.float32)


@dataclass
class Mesh:
    vertices: np.ndarray            # V x 3 float32
    indices: np.ndarray             # T x 3 uint32
    material_ids: np.ndarray        # T int32
    normals: np.ndarray | None = None
    uvs: np.ndarray | None = None


@dataclass
class SceneBuilder:
    materials: list = field(default_factory=list)
    meshes: list = field(default_factory=list)
    instances: list = field(default_factory=list)   # (mesh, 3x4 matrix, override)
    lights: list = field(default_factory=list)
    images: list = field(default_factory=list)      # (height, width, 3) float32 images
    camera: CameraDesc | None = None
    _default_mesh: int = -1
    _tris: list = field(default_factory=list)
    _mids: list = field(default_factory=list)

    def add_material(self, m: Material) -> int:
        self.materials.append(m)
        return len(self.materials) - 1

    def add_triangle(self, v0, v1, v2, material_id: int) -> None:
        """scene/scene_edit.h:98-124: three new vertices in the default mesh."""
        if self._default_mesh < 0:
            self._default_mesh = len(self.meshes)
            self.meshes.append(None)
            self.instances.append((self._default_mesh, IDENTITY, -1))
        self._tris.append((v0, v1, v2))
        self._mids.append(material_id)

    def add_quad(self, p0, p1, p2, p3, material_id: int) -> None:
        """scene/scene_edit.h:261-265."""
        self.add_triangle(p0, p1, p2, material_id)
        self.add_triangle(p0, p2, p3, material_id)

    def add_mesh(self, mesh: Mesh) -> int:
        self.meshes.append(mesh)
        return len(self.meshes) - 1

    def add_instance(self, mesh: int, object_to_world=IDENTITY, material_override: int = -1):
        self.instances.append((mesh, np.asarray(object_to_world, np.float32)[:3], material_override))
        return len(self.instances) - 1

    def add_point_light(self, position, intensity):
        self.lights.append(LightDesc(LIGHT_POINT, _F3(*position), _F3(*intensity)))

    def add_distant_light(self, direction_to_light, radiance):
        self.lights.append(LightDesc(LIGHT_DISTANT, _F3(*direction_to_light), _F3(*radiance)))

    def add_uniform_infinite_light(self, radiance):
        self.lights.append(LightDesc(LIGHT_UNIFORM_INFINITE, _F3(0, 0, 0), _F3(*radiance)))

    def add_image(self, pixels) -> int:
        """A scene image (height, width, 3) for image emission; returns its index."""
        self.images.append(np.ascontiguousarray(pixels, np.float32))
        return len(self.images) - 1

    def world_uvs(self) -> np.ndarray:
        """Corner texture coordinates of each scene triangle (6 floats), in
        world_triangles order; zero for meshes without them."""
        out = []
        for mesh_id, _, _ in self.instances:
            mesh = self.default_mesh() if mesh_id == self._default_mesh else self.meshes[mesh_id]
            if mesh.uvs is None:
                out.append(np.zeros((len(mesh.indices), 6), np.float32))
            else:
                uv = np.asarray(mesh.uvs, np.float32)
                out.append(uv[np.asarray(mesh.indices).reshape(-1)].reshape(-1, 6))
        return np.concatenate(out) if out else np.zeros((0, 6), np.float32)

    def add_image_infinite_light(self, pixels, scale=(1.0, 1.0, 1.0)):
        """add_image_infinite_light (scene/scene_build.h:67-89): pixels is an
        (height, width, 3) latitude-longitude image, row 0 at the +y pole."""
        img = np.ascontiguousarray(pixels, np.float32)
        self.images.append(img)
        self.lights.append(LightDesc(LIGHT_IMAGE_INFINITE, _F3(0, 0, 0), _F3(*scale),
                                     len(self.images) - 1))

    def set_pinhole_camera(self, origin, look_at, vfov_degrees, aspect):
        """make_pinhole_camera (camera/pinhole_camera.h:13-17): lens 0, focal distance 1."""
        self.set_perspective_camera(origin, look_at, vfov_degrees, aspect, 0.0, 1.0)

    def set_perspective_camera(self, origin, look_at, vfov_degrees, aspect, lens_radius,
                               focal_distance):
        lib = load_library()
        cam = CameraDesc()
        o = (ctypes.c_float * 3)(*origin)
        a = (ctypes.c_float * 3)(*look_at)
        _check(lib.lux_camera_perspective(o, a, vfov_degrees, aspect, lens_radius,
                                          focal_distance, ctypes.byref(cam)))
        self.camera = cam

    def default_mesh(self) -> Mesh:
        tris = np.asarray(self._tris, np.float32).reshape(-1, 3, 3)
        n = len(tris)
        return Mesh(tris.reshape(-1, 3).copy(), np.arange(3 * n, dtype=np.uint32).reshape(n, 3),
                    np.asarray(self._mids, np.int32))

    def world_triangles(self) -> np.ndarray:
        """Scene triangles in scene order (instances, then local order), world space."""
        out = []
        for mesh_id, m, _ in self.instances:
            mesh = self.default_mesh() if mesh_id == self._default_mesh else self.meshes[mesh_id]
            v = mesh.vertices[mesh.indices.reshape(-1)].astype(np.float32)
            w = v @ m[:, :3].T + m[:, 3]
            out.append(w.reshape(-1, 9).astype(np.float32))
        return np.concatenate(out) if out else np.zeros((0, 9), np.float32)

    def world_material_ids(self) -> np.ndarray:
        """Material id of each scene triangle, in world_triangles order."""
        out = []
        for mesh_id, _, override in self.instances:
            mesh = self.default_mesh() if mesh_id == self._default_mesh else self.meshes[mesh_id]
            ids = np.asarray(mesh.material_ids, np.int32)
            out.append(np.full(len(ids), override, np.int32) if override >= 0 else ids)
        return np.concatenate(out) if out else np.zeros(0, np.int32)


def scene_desc(builder: SceneBuilder):
    """The lux_scene_desc of a SceneBuilder and the arrays it points into (keep them
    alive while the descriptor is in use)."""
    keep = []
    mats = (Material * max(len(builder.materials), 1))(*builder.materials)
    meshes = []
    for i, mesh in enumerate(builder.meshes):
        if i == builder._default_mesh:
            mesh = builder.default_mesh()
        v = np.ascontiguousarray(mesh.vertices, np.float32)
        idx = np.ascontiguousarray(mesh.indices, np.uint32)
        mid = np.ascontiguousarray(mesh.material_ids, np.int32)
        nrm = None if mesh.normals is None else np.ascontiguousarray(mesh.normals, np.float32)
        uv = None if mesh.uvs is None else np.ascontiguousarray(mesh.uvs, np.float32)
        keep += [v, idx, mid, nrm, uv]
        meshes.append(MeshDesc(v.ctypes.data, None if nrm is None else nrm.ctypes.data,
                               None if uv is None else uv.ctypes.data, len(v),
                               idx.ctypes.data, mid.ctypes.data, len(mid)))
    mesh_arr = (MeshDesc * max(len(meshes), 1))(*meshes)
    insts = []
    for mesh_id, m, override in builder.instances:
        insts.append(InstanceDesc(mesh_id, override, _F12(*np.asarray(m, np.float32).reshape(-1)),
                                  _F12(*([0.0] * 12))))
    inst_arr = (InstanceDesc * max(len(insts), 1))(*insts)
    light_arr = (LightDesc * max(len(builder.lights), 1))(*builder.lights)
    images = [np.ascontiguousarray(im, np.float32) for im in builder.images]
    keep += images
    img_arr = (EnvImageDesc * max(len(images), 1))(
        *[EnvImageDesc(im.ctypes.data, im.shape[1], im.shape[0]) for im in images])
    keep += [mats, mesh_arr, inst_arr, light_arr, img_arr]
    desc = SceneDesc(ctypes.addressof(mats), len(builder.materials),
                     ctypes.addressof(mesh_arr), len(meshes),
                     ctypes.addressof(inst_arr), len(insts),
                     ctypes.addressof(light_arr), len(builder.lights),
                     builder.camera if builder.camera is not None else CameraDesc(),
                     ctypes.addressof(img_arr), len(images))
    return desc, keep


class Scene:
    """A lux_scene handle resident on the context's device."""

    def __init__(self, ctx, builder: SceneBuilder):
        self.ctx = ctx
        lib = ctx._lib
        desc, keep = scene_desc(builder)
        handle = ctypes.c_void_p()
        _check(lib.lux_scene_create(ctx.handle, ctypes.byref(desc), ctypes.byref(handle)))
        self._h = handle
        self._lib = lib
        del keep

    @property
    def handle(self):
        return self._h

    def info(self):
        t, a, l = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        _check(self._lib.lux_scene_info(self._h, ctypes.byref(t), ctypes.byref(a), ctypes.byref(l)))
        return {"triangles": t.value, "area_lights": a.value, "lights": l.value}

    def select_lights(self, positions: np.ndarray, select_u: np.ndarray,
                      light_sampler=SAMPLER_TREE):
        """sample_scene_light + light_pmf at each position: (light index or -1, the
        selection's pmf, light_pmf of that light)."""
        pos = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        u = np.ascontiguousarray(select_u, np.float32).reshape(-1)
        n = len(u)
        assert len(pos) == n
        index = np.zeros(n, np.int32)
        pmf = np.zeros(n, np.float32)
        eval_pmf = np.zeros(n, np.float32)
        _check(self._lib.lux_scene_select_lights(self.ctx.handle, self._h, light_sampler,
                                                 pos.ctypes.data, u.ctypes.data, n,
                                                 index.ctypes.data, pmf.ctypes.data,
                                                 eval_pmf.ctypes.data))
        return index, pmf, eval_pmf

    def update_mesh(self, mesh: int, vertices: np.ndarray) -> None:
        v = np.ascontiguousarray(vertices, np.float32)
        _check(self._lib.lux_scene_update_mesh(self.ctx.handle, self._h, mesh, v.ctypes.data))

    def close(self):
        if self._h:
            self._lib.lux_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def request(width, height, spp, max_depth, seed=0, frame_index=0, sample_offset=0,
            light_sampler=SAMPLER_POWER) -> RenderRequest:
    return RenderRequest(width, height, spp, max_depth, seed, frame_index, sample_offset,
                         light_sampler)


def render(ctx, scene: Scene, req: RenderRequest, out=None):
    """Film SUM over spp, height x width x 3 (Film::pixels)."""
    if out is None:
        out = np.zeros((req.height, req.width, 3), np.float32)
    _check(ctx._lib.lux_render(ctx.handle, scene.handle, ctypes.byref(req), _ptr(out)))
    return out


def render_aovs(ctx, scene: Scene, req: RenderRequest, shadow=True, ng=True, ns=True):
    """Film sum and the wanted debug images (per-pixel sums over spp, height x width x 3;
    None where not wanted), as lux_render_aovs makes them."""
    film = np.zeros((req.height, req.width, 3), np.float32)
    out = [np.zeros_like(film) if want else None for want in (shadow, ng, ns)]
    _check(ctx._lib.lux_render_aovs(ctx.handle, scene.handle, ctypes.byref(req), _ptr(film),
                                    *(None if a is None else _ptr(a) for a in out)))
    return film, out[0], out[1], out[2]


# lux_path_log_record (PathLogRecord, integrator/pathstate.cuh:41-65).
PATH_LOG_RECORD = np.dtype([
    ("pixel_index", "<i4"), ("sample_index", "<i4"), ("depth", "<i4"), ("triangle_id", "<i4"),
    ("instance_id", "<i4"), ("mesh_id", "<i4"), ("local_primitive_id", "<i4"),
    ("primitive_kind", "<i4"), ("material_id", "<i4"), ("vertex", "<i4"),
    ("position", "<f4", 3), ("ng", "<f4", 3), ("ns", "<f4", 3), ("wo", "<f4", 3),
    ("wi", "<f4", 3), ("throughput_before", "<f4", 3), ("throughput_after", "<f4", 3),
    ("bsdf_pdf", "<f4"), ("guide_pdf", "<f4"), ("light_pdf", "<f4"),
    ("bsdf_pdf_measure", "u1"), ("guide_pdf_measure", "u1"), ("light_pdf_measure", "u1"),
    ("sample_source", "u1"), ("bsdf_flags", "<u4"), ("termination_flags", "<u4"),
    ("event_flags", "<u4")])
assert PATH_LOG_RECORD.itemsize == 152

# PathLogEventFlags / PathLogTerminationFlags (integrator/pathstate.cuh:19-39).
EVENT_SURFACE_HIT, EVENT_EMISSION, EVENT_LIGHT_SAMPLED, EVENT_LIGHT_VALID = 1, 2, 4, 8
EVENT_BSDF_SAMPLED, EVENT_TERMINATED, EVENT_SPAWNED_RAY, EVENT_DELTA = 16, 32, 64, 128
EVENT_PASSTHROUGH = 256
END_NON_SCATTERING, END_MAX_DEPTH, END_INVALID_BSDF = 1, 2, 4
END_RUSSIAN_ROULETTE, END_ZERO_THROUGHPUT = 8, 16


def render_path_log(ctx, scene: Scene, req: RenderRequest, capacity=None):
    """Film sum and the path log of one render (lux_render_path_log): a structured array
    of PATH_LOG_RECORD sorted by (sample_index, pixel_index, vertex).  capacity defaults
    to the bound width * height * spp * (max_depth + 1), at 152 bytes a record on the
    host and in the context's device staging: pass a smaller one for large renders
    (an exhausted capacity raises LuxError with status 6)."""
    if capacity is None:
        capacity = req.width * req.height * req.spp * (req.max_depth + 1)
    film = np.zeros((req.height, req.width, 3), np.float32)
    records = np.zeros(max(int(capacity), 1), PATH_LOG_RECORD)
    count = ctypes.c_int64(0)
    _check(ctx._lib.lux_render_path_log(ctx.handle, scene.handle, ctypes.byref(req), _ptr(film),
                                        records.ctypes.data, int(capacity), ctypes.byref(count)))
    return film, records[:count.value]


def render_samples(ctx, scene: Scene, req: RenderRequest):
    out = np.zeros((req.height * req.width, req.spp, 3), np.float32)
    _check(ctx._lib.lux_render_samples(ctx.handle, scene.handle, ctypes.byref(req), _ptr(out)))
    return out


def ray_counts(ctx) -> tuple[int, int]:
    c = np.zeros(2, np.int64)
    _check(ctx._lib.lux_render_ray_counts(ctx.handle, c.ctypes.data))
    return int(c[0]), int(c[1])


def traversal_stats(ctx, scene: Scene, req: RenderRequest) -> dict:
    """The render's traversal work in the reference's visit order
    (lux_render_traversal_stats): rays, shadow segments, box tests, triangle tests and
    instance visits, with the film the counted render made."""
    film = np.zeros((req.height, req.width, 3), np.float32)
    c = np.zeros(5, np.int64)
    _check(ctx._lib.lux_render_traversal_stats(ctx.handle, scene.handle, ctypes.byref(req),
                                               _ptr(film), c.ctypes.data))
    return {"rays": int(c[0]), "shadow_segments": int(c[1]), "box_tests": int(c[2]),
            "tri_tests": int(c[3]), "instance_visits": int(c[4]), "film": film}


def _add_box(b: SceneBuilder, lo, hi, mat):
    """cornell_box_detail::add_box (scene/cornell_box.h:11-27)."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    p000, p001, p010, p011 = (x0, y0, z0), (x0, y0, z1), (x0, y1, z0), (x0, y1, z1)
    p100, p101, p110, p111 = (x1, y0, z0), (x1, y0, z1), (x1, y1, z0), (x1, y1, z1)
    b.add_quad(p000, p100, p110, p010, mat)
    b.add_quad(p101, p001, p011, p111, mat)
    b.add_quad(p001, p000, p010, p011, mat)
    b.add_quad(p100, p101, p111, p110, mat)
    b.add_quad(p010, p110, p111, p011, mat)
    b.add_quad(p001, p101, p100, p000, mat)


def make_cornell_box() -> SceneBuilder:
    """scene/cornell_box.h:31-56."""
    b = SceneBuilder()
    f = np.float32
    white = b.add_material(lambert((f(0.78), f(0.78), f(0.74))))
    red = b.add_material(lambert((f(0.65), f(0.05), f(0.05))))
    green = b.add_material(lambert((f(0.12), f(0.45), f(0.15))))
    light = b.add_material(emissive((15.0, 14.0, 12.0)))
    b.add_quad((-1, 0, 2), (1, 0, 2), (1, 0, 0), (-1, 0, 0), white)
    b.add_quad((-1, 2, 0), (1, 2, 0), (1, 2, 2), (-1, 2, 2), white)
    b.add_quad((-1, 0, 0), (1, 0, 0), (1, 2, 0), (-1, 2, 0), white)
    b.add_quad((-1, 0, 2), (-1, 0, 0), (-1, 2, 0), (-1, 2, 2), red)
    b.add_quad((1, 0, 0), (1, 0, 2), (1, 2, 2), (1, 2, 0), green)
    _add_box(b, (-0.65, 0, 0.35), (-0.15, 0.8, 0.9), white)
    _add_box(b, (0.25, 0, 0.75), (0.75, 1.2, 1.35), white)
    b.add_quad((-0.35, 1.99, 0.75), (0.35, 1.99, 0.75), (0.35, 1.99, 1.35), (-0.35, 1.99, 1.35),
               light)
    return b


def make_cornell_scene(width: int, height: int) -> SceneBuilder:
    """app/render_runner.cpp:85-90: pinhole at (0,1,3.35) looking at (0,1,0.9), fov 40."""
    b = make_cornell_box()
    aspect = float(np.float32(width) / np.float32(height))
    b.set_pinhole_camera((0, 1, 3.35), (0, 1, 0.9), 40.0, aspect)
    return b
