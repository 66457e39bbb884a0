"""Debug images (`-debug-aov shadow,ng,ns`, lux_render_aovs) against the reference CPU
tracer's own (render_cpu_path_tracer with RenderOutputs, run from oracle/_ref).

The GPU images follow the reference's wavefront tracer.  Its CPU tracer computes the same
images from the same random numbers, with two differences: for an invalid light sample
the wavefront tracer adds orange and the CPU tracer nothing, and the CPU tracer's search
for the first scattering surface behind a pass-through surface seen by the camera keeps
the previous hit's distance as the bound of the next search (cpu_path_tracer.cpp:339-366
reuses `hit`, which intersect_scene_two_level_bvh, scene/scene_intersection.h:150-151,
takes as t_max), so it mostly finds nothing there, where the wavefront tracer continues
the path.  The scene here has only two-sided emitters, point, distant and sky lights (no
invalid light sample), and its camera sees no pass-through surface directly, while
shadow rays cross the filter; there the two agree.  Images are per-pixel sums over
samples.  The GPU sums with atomics, so values agree to float rounding; a pixel may also
differ where a last-bit difference flipped a first-bounce decision (at most 1 %).
"""
import os

import numpy as np
import pytest

from lux_b200 import scene as S
from oracle.bindings import Ref

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not Ref.available(), reason="reference harness not built")]

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def aov_scene(w=48, h=48):
    """A room with every material kind, two-sided emitters and point, distant and sky
    lights; the pass-through surfaces (tinted filter, interface) sit above the camera's
    view, the filter between the floor and the main lamp."""
    f = np.float32
    b = S.SceneBuilder()
    white = b.add_material(S.lambert((f(0.75), f(0.75), f(0.72))))
    glossy = b.add_material(S.ggx((f(0.8), f(0.6), f(0.3)), f(0.3), f(0.0)))
    thin = b.add_material(S.material(S.THIN_LAMBERT, (f(0.6), f(0.8), f(0.6))))
    glass = b.add_material(S.dielectric((1, 1, 1), f(1.5)))
    tint = b.add_material(S.tinted_filter((f(0.25), f(0.65), f(1.0))))
    iface = b.add_material(S.interface())
    lamp = b.add_material(S.emissive((9.0, 8.0, 7.0), two_sided=True))
    lamp2 = b.add_material(S.emissive((2.0, 2.5, 4.0), two_sided=True))
    b.add_quad((-1, 0, 2), (1, 0, 2), (1, 0, -1), (-1, 0, -1), white)
    b.add_quad((-1, 0, -1), (1, 0, -1), (1, 2, -1), (-1, 2, -1), white)
    b.add_quad((-1, 0, 2), (-1, 0, -1), (-1, 2, -1), (-1, 2, 2), glossy)
    b.add_quad((-0.8, 0.1, 0.2), (-0.2, 0.1, 0.2), (-0.2, 0.8, 0.2), (-0.8, 0.8, 0.2), thin)
    b.add_quad((0.2, 0.05, 0.6), (0.7, 0.05, 0.6), (0.7, 0.7, 0.3), (0.2, 0.7, 0.3), glass)
    b.add_quad((-0.9, 1.2, 1.0), (0.9, 1.2, 1.0), (0.9, 1.2, 0.4), (-0.9, 1.2, 0.4), tint)
    b.add_quad((-0.5, 1.3, 1.3), (0.5, 1.3, 1.3), (0.5, 1.9, 1.3), (-0.5, 1.9, 1.3), iface)
    b.add_quad((-0.3, 1.7, 0.3), (0.3, 1.7, 0.3), (0.3, 1.7, 0.9), (-0.3, 1.7, 0.9), lamp)
    b.add_quad((0.5, 1.5, -0.95), (0.9, 1.5, -0.95), (0.9, 1.9, -0.95), (0.5, 1.9, -0.95), lamp2)
    b.add_point_light((0.0, 1.4, 1.5), (1.5, 1.5, 1.5))
    b.add_distant_light((-0.3, 1.0, 0.4), (0.3, 0.3, 0.3))
    b.add_uniform_infinite_light((0.05, 0.05, 0.08))
    cam = ((0.0, 0.6, 3.0), (0.0, 0.3, 0.0), 38.0, float(f(w) / f(h)))
    b.set_pinhole_camera(*cam)
    return b, cam


def _ref_arrays(b):
    tris = b.world_triangles()
    mats = np.array([[m.type, *m.albedo, *m.emission, m.roughness, m.metallic, m.eta,
                      m.emission_two_sided] for m in b.materials], np.float32)
    lights = np.array([[l.kind, *l.vec, *l.value] for l in b.lights], np.float32).reshape(-1, 7)
    return tris, b.world_material_ids(), mats, lights


def _close_pixels(got, want, rtol=1e-4):
    ok = np.all(np.abs(got - want) <= rtol * (1.0 + np.abs(want)), axis=-1)
    return ok.mean()


@pytest.mark.parametrize("sampler", [S.SAMPLER_POWER, S.SAMPLER_TREE])
def test_debug_images_match_reference_cpu_tracer(ctx, sampler):
    w = h = 48
    spp, depth, seed = 16, 5, 4
    b, cam = aov_scene(w, h)
    sc = S.Scene(ctx, b)
    req = S.request(w, h, spp, depth, seed, light_sampler=sampler)
    film, shadow, ng, ns = S.render_aovs(ctx, sc, req)
    # The beauty film is lux_render's.
    assert np.array_equal(film, S.render(ctx, sc, req))
    tris, mids, mats, lights = _ref_arrays(b)
    camera = np.array([*cam[0], *cam[1], cam[2], cam[3]], np.float32)
    _, want_shadow, want_ng, want_ns = Ref().render_aovs(tris, mids, mats, lights, camera, w, h,
                                                         spp, depth, seed, sampler)
    assert _close_pixels(ng, want_ng, 1e-5) == 1.0
    assert _close_pixels(ns, want_ns, 1e-5) == 1.0
    assert _close_pixels(shadow, want_shadow) >= 0.99
    # Most pixels see the room; the shadow image holds several classes.
    assert (ng.sum(axis=-1) > 0).mean() > 0.9 and shadow.sum() > 0
    assert len(np.unique(np.round(shadow.reshape(-1, 3) / spp, 3), axis=0)) > 8


def test_debug_images_are_optional_and_scale_with_spp(ctx):
    b, _ = aov_scene(16, 16)
    sc = S.Scene(ctx, b)
    film, shadow, ng, ns = S.render_aovs(ctx, sc, S.request(16, 16, 4, 3, 1), shadow=False,
                                         ns=False)
    assert shadow is None and ns is None
    # ng sums one encoded normal per sample: each channel in [0, spp].
    assert ng.min() >= 0 and ng.max() <= 4.0 + 1e-5
