"""Wavefront path tracer vs the reference CPU tracer (B200).

The GPU tracer draws the same random numbers in the same order and restates the same
arithmetic, so most samples agree to ~1e-6; the few that differ are paths where CUDA's
sinf/cosf/powf rounded a last bit differently and a later discrete decision flipped.
Criteria: (1) per-sample agreement within 1e-4 relative for >= 99% of samples; (2) the
north_star's per-pixel mean within 3 sigma at equal spp (fraction of pixels with |z| > 3
at most 1%); (3) film sums equal the sum of the per-sample values in sample order.
"""
import os

import numpy as np
import pytest

import lux_b200
from lux_b200 import scene as S
from oracle.bindings import Ref

pytestmark = pytest.mark.gpu

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
THREADS = os.cpu_count() or 1


def _agreement(gpu, ref, rtol=1e-4):
    close = np.all(np.abs(gpu - ref) <= rtol * (1.0 + np.abs(ref)), axis=-1)
    return close.mean()


def _z_fraction(gpu, ref):
    """Fraction of pixel-channels whose mean differs by more than 3 sigma."""
    n = gpu.shape[1]
    mg, mr = gpu.mean(axis=1), ref.mean(axis=1)
    vg, vr = gpu.var(axis=1, ddof=1), ref.var(axis=1, ddof=1)
    se = np.sqrt((vg + vr) / n)
    diff = np.abs(mg - mr)
    # Zero variance on both sides: the means must then be equal.
    outside = np.where(se > 0, diff > 3 * se, diff > 0)
    return outside.mean()


def _ref_arrays(b: S.SceneBuilder):
    tris = b.world_triangles()
    mids = b.world_material_ids()
    mats = np.array([[m.type, *m.albedo, *m.emission, m.roughness, m.metallic, m.eta,
                      m.emission_two_sided] for m in b.materials], np.float32)
    lights = np.array([[l.kind, *l.vec, *l.value] for l in b.lights], np.float32).reshape(-1, 7)
    return tris, mids, mats, lights


def test_cornell_matches_reference_fixture(ctx):
    g = np.load(os.path.join(ROOT, "tests", "golden", "cornell_reference.npz"))
    w, h, spp, depth, seed = (int(g[k]) for k in ("width", "height", "spp", "max_depth", "seed"))
    b = S.make_cornell_scene(w, h)
    assert np.array_equal(b.world_triangles(), g["triangles"])
    sc = S.Scene(ctx, b)
    req = S.request(w, h, spp, depth, seed)
    samples = S.render_samples(ctx, sc, req)
    assert _agreement(samples, g["samples"]) >= 0.99
    assert _z_fraction(samples, g["samples"]) <= 0.01
    film = S.render(ctx, sc, req).reshape(-1, 3)
    want = np.zeros_like(film)
    for s in range(spp):
        want = (want + samples[:, s]).astype(np.float32)
    assert np.array_equal(film, want)
    rel = np.abs(film - g["film_sum"]) / (1 + np.abs(g["film_sum"]))
    assert np.quantile(rel, 0.99) < 1e-4


@pytest.mark.skipif(not Ref.available(), reason="reference harness not built")
def test_cornell_config1_shape_matches_reference_live(ctx):
    """Config-1 settings (power sampler, depth 4, seed 1) at 96x96, 16 spp."""
    w = h = 96
    spp, depth, seed = 16, 4, 1
    sc = S.Scene(ctx, S.make_cornell_scene(w, h))
    gpu = S.render_samples(ctx, sc, S.request(w, h, spp, depth, seed))
    ref = Ref()
    _, _, want = ref.cornell_render(w, h, spp, depth, seed, threads=THREADS, samples=True)
    assert _agreement(gpu, want) >= 0.99
    assert _z_fraction(gpu, want) <= 0.01
    counts = S.ray_counts(ctx)
    assert counts[0] >= w * h * spp and counts[1] > 0


def material_zoo(width=48, height=48, glass_y0=0.0):
    """Every BSDF and light kind the wavefront path supports, in one closed room.  The
    glass box stands on the floor: its bottom face lies in the floor's plane (glass_y0
    lifts it)."""
    b = S.SceneBuilder()
    f = np.float32
    white = b.add_material(S.lambert((f(0.75), f(0.75), f(0.72))))
    blue = b.add_material(S.lambert((f(0.2), f(0.3), f(0.7))))
    glossy = b.add_material(S.ggx((f(0.8), f(0.6), f(0.3)), f(0.3), f(0.0)))
    metal = b.add_material(S.ggx((f(0.9), f(0.9), f(0.9)), f(0.15), f(1.0)))
    thin = b.add_material(S.material(S.THIN_LAMBERT, (f(0.6), f(0.8), f(0.6))))
    glass = b.add_material(S.dielectric((1, 1, 1), f(1.5)))
    tint = b.add_material(S.tinted_filter((f(0.25), f(0.65), f(1.0))))
    iface = b.add_material(S.interface())
    light = b.add_material(S.emissive((12.0, 11.0, 9.0)))
    light2 = b.add_material(S.emissive((3.0, 3.0, 5.0), two_sided=True))
    b.add_quad((-1, 0, 2), (1, 0, 2), (1, 0, -1), (-1, 0, -1), white)        # floor
    b.add_quad((-1, 2, -1), (1, 2, -1), (1, 2, 2), (-1, 2, 2), white)        # ceiling
    b.add_quad((-1, 0, -1), (1, 0, -1), (1, 2, -1), (-1, 2, -1), blue)       # back
    b.add_quad((-1, 0, 2), (-1, 0, -1), (-1, 2, -1), (-1, 2, 2), glossy)     # left (GGX)
    b.add_quad((1, 0, -1), (1, 0, 2), (1, 2, 2), (1, 2, -1), metal)          # right (metal)
    b.add_quad((-0.8, 0.1, 0.2), (-0.2, 0.1, 0.2), (-0.2, 0.8, 0.2), (-0.8, 0.8, 0.2), thin)
    # glass box
    x0, y0, z0, x1, y1, z1 = 0.2, glass_y0, 0.3, 0.7, 0.6, 0.8
    p = [(x0, y0, z0), (x0, y0, z1), (x0, y1, z0), (x0, y1, z1),
         (x1, y0, z0), (x1, y0, z1), (x1, y1, z0), (x1, y1, z1)]
    for q in [(0, 4, 6, 2), (5, 1, 3, 7), (1, 0, 2, 3), (4, 5, 7, 6), (2, 6, 7, 3), (1, 5, 4, 0)]:
        b.add_quad(p[q[0]], p[q[1]], p[q[2]], p[q[3]], glass)
    b.add_quad((-0.9, 1.2, 1.0), (0.9, 1.2, 1.0), (0.9, 1.2, 0.4), (-0.9, 1.2, 0.4), tint)
    b.add_quad((-0.5, 0.9, 1.3), (0.5, 0.9, 1.3), (0.5, 1.6, 1.3), (-0.5, 1.6, 1.3), iface)
    b.add_quad((-0.3, 1.99, 0.3), (0.3, 1.99, 0.3), (0.3, 1.99, 0.9), (-0.3, 1.99, 0.9), light)
    b.add_quad((0.5, 1.5, -0.95), (0.9, 1.5, -0.95), (0.9, 1.9, -0.95), (0.5, 1.9, -0.95), light2)
    b.add_point_light((0.0, 1.7, 1.5), (2.0, 2.0, 2.0))
    b.add_distant_light((-0.3, 1.0, 0.4), (0.3, 0.3, 0.3))
    b.add_uniform_infinite_light((0.05, 0.05, 0.08))
    cam = ((0.0, 1.0, 3.2), (0.0, 0.9, 0.5), 45.0, float(f(width) / f(height)))
    b.set_pinhole_camera(*cam)
    return b, cam


@pytest.mark.skipif(not Ref.available(), reason="reference harness not built")
@pytest.mark.parametrize("sampler,depth", [(S.SAMPLER_POWER, 6), (S.SAMPLER_UNIFORM, 3),
                                           (S.SAMPLER_TREE, 5)])
def test_material_zoo_matches_reference_live(ctx, sampler, depth):
    w = h = 48
    spp, seed = 32, 5
    b, cam = material_zoo(w, h)
    sc = S.Scene(ctx, b)
    gpu = S.render_samples(ctx, sc, S.request(w, h, spp, depth, seed, light_sampler=sampler))
    tris, mids, mats, lights = _ref_arrays(b)
    camera = np.array([*cam[0], *cam[1], cam[2], cam[3]], np.float32)
    ref = Ref().render_scene(tris, mids, mats, lights, camera, w, h, spp, depth, seed,
                             light_sampler=sampler, threads=THREADS)
    assert np.isfinite(gpu).all()
    assert _agreement(gpu, ref) >= 0.97
    assert _z_fraction(gpu, ref) <= 0.01
    # The scene exercises every path: lights, passthrough and glass contribute.
    assert gpu.mean() > 0


def test_render_is_deterministic_and_batches_agree(ctx):
    """Repeated renders, and renders split into many batches (which run on several lanes
    at once, their film accumulation kept in batch order), give the same film."""
    w = h = 40
    sc = S.Scene(ctx, S.make_cornell_scene(w, h))
    req = S.request(w, h, 12, 4, 3)
    a = S.render(ctx, sc, req)
    b = S.render(ctx, sc, req)
    assert np.array_equal(a, b)
    old = ctx.get_option(3)
    try:
        ctx.set_option(3, 1000)   # force many small batches (pixel ranges x 1 sample)
        c = S.render(ctx, sc, req)
        ctx.set_option(3, 5 * w * h)  # sample ranges of 5
        d = S.render(ctx, sc, req)
    finally:
        ctx.set_option(3, old)
    assert np.array_equal(a, c)
    assert np.array_equal(a, d)


@pytest.mark.parametrize("extra", [1, 2, 3, 4])
def test_small_tlas_walks_render_as_the_binary_walk(ctx, extra):
    """Scenes of two to five instances: the refilling walks enter a TLAS of at most four
    instances leaf by leaf, the one-path-per-thread kernels walk its binary nodes.  The
    instance boxes overlap, and two instances sit at the same place under different
    materials, so their hits tie at equal t and the left-first order decides which one
    is seen.  Both kernel families render the same film."""
    from lux_b200 import scenes as SC
    w = h = 48
    f = np.float32
    b = S.make_cornell_scene(w, h)
    v, idx = SC.displaced_sphere(2, (0.0, 0.0, 0.0), 0.3, 0.03, 4)
    red = b.add_material(S.lambert((f(0.8), f(0.1), f(0.1))))
    green = b.add_material(S.ggx((f(0.1), f(0.8), f(0.1)), f(0.3), f(0.0)))
    mesh = b.add_mesh(S.Mesh(v, idx, np.full(len(idx), red, np.int32)))
    places = [(-0.3, 0.5, 0.9, -1), (-0.3, 0.5, 0.9, green), (0.1, 0.45, 1.0, -1),
              (0.3, 0.9, 0.8, green)]
    for x, y, z, override in places[:extra]:
        m = np.array([[1, 0, 0, x], [0, 1, 0, y], [0, 0, 1, z]], np.float32)
        b.add_instance(mesh, m, override)
    sc = S.Scene(ctx, b)
    req = S.request(w, h, 8, 5, 11)
    old = ctx.get_option(lux_b200.OPT_TRACE_VARIANT)
    try:
        ctx.set_option(lux_b200.OPT_TRACE_VARIANT, 1)
        want = S.render(ctx, sc, req)
        ctx.set_option(lux_b200.OPT_TRACE_VARIANT, 0)
        got = S.render(ctx, sc, req)
    finally:
        ctx.set_option(lux_b200.OPT_TRACE_VARIANT, old)
    assert want.mean() > 0
    assert np.array_equal(got, want)


def test_sample_offset_and_frame_index_continue_the_sequence(ctx):
    """RenderSettings::sample_offset (integrator/render_context.h:52): two halves of the
    samples rendered separately equal the full render's samples."""
    w = h = 24
    sc = S.Scene(ctx, S.make_cornell_scene(w, h))
    full = S.render_samples(ctx, sc, S.request(w, h, 8, 4, 9))
    first = S.render_samples(ctx, sc, S.request(w, h, 4, 4, 9))
    second = S.render_samples(ctx, sc, S.request(w, h, 4, 4, 9, sample_offset=4))
    assert np.array_equal(full[:, :4], first)
    assert np.array_equal(full[:, 4:], second)
    other = S.render_samples(ctx, sc, S.request(w, h, 8, 4, 9, frame_index=1))
    assert not np.array_equal(full, other)


def test_invalid_requests_fail_cleanly(ctx):
    sc = S.Scene(ctx, S.make_cornell_scene(8, 8))
    for bad in [S.request(0, 8, 1, 4), S.request(8, 8, 0, 4), S.request(8, 8, 1, -1),
                S.request(8, 8, 1, 4, light_sampler=3)]:
        with pytest.raises(lux_b200.LuxError) as e:
            S.render(ctx, sc, bad)
        assert e.value.status == lux_b200.LUX_ERR_INVALID_ARGUMENT


def test_empty_scene_renders_black(ctx):
    b = S.SceneBuilder()
    b.add_material(S.lambert((0.5, 0.5, 0.5)))
    b.set_pinhole_camera((0, 0, 3), (0, 0, 0), 40.0, 1.0)
    sc = S.Scene(ctx, b)
    film = S.render(ctx, sc, S.request(8, 8, 2, 3))
    assert np.all(film == 0)


def test_device_mesh_update_matches_a_fresh_scene(ctx):
    """lux_scene_update_mesh on a mesh with two transformed instances renders like a
    scene created from the moved vertices (world triangles and instance boxes are
    computed with the host restatement's arithmetic)."""
    from lux_b200 import scenes as SC

    def build(vertices=None):
        b = S.make_cornell_scene(32, 32)
        v, idx = SC.displaced_sphere(4, (0.0, 0.0, 0.0), 0.3, 0.04, 5)
        if vertices is not None:
            v = vertices
        rough = b.add_material(S.ggx((0.8, 0.5, 0.3), 0.35, 0.0))
        mesh = b.add_mesh(S.Mesh(v, idx, np.full(len(idx), rough, np.int32)))
        c, s_ = np.float32(np.cos(0.7)), np.float32(np.sin(0.7))
        b.add_instance(mesh, np.array([[c, 0, s_, 0.5], [0, 1.3, 0, 0.6], [-s_, 0, c, 0.9]],
                                      np.float32))
        b.add_instance(mesh, np.array([[0.8, 0, 0, -0.4], [0, 0.8, 0, 1.2], [0, 0, 0.8, 0.4]],
                                      np.float32))
        return b, mesh, v

    b, mesh, v = build()
    sc = S.Scene(ctx, b)
    moved = v.copy()
    moved[:, 1] += np.float32(0.03) * np.sin(5.0 * moved[:, 2]).astype(np.float32)
    sc.update_mesh(mesh, moved)
    req = S.request(32, 32, 4, 5, 3)
    got = S.render_samples(ctx, sc, req)
    fresh = S.render_samples(ctx, S.Scene(ctx, build(moved)[0]), req)
    same = np.all(got == fresh, axis=-1)
    assert same.mean() > 0.999, same.mean()


def _fp64_check(film_mean, fixture, spp):
    """Relative RMSE of the render against the FP64 oracle, with the oracle's own noise
    (its per-sample variance / its spp) taken out of the mean squared error, and the
    ratio of measured to noise-predicted MSE (1 for an unbiased renderer)."""
    ref = fixture["mean"].astype(np.float64)
    var = fixture["var"].astype(np.float64)
    mse = np.mean((film_mean - ref) ** 2)
    oracle_noise = np.mean(var / int(fixture["spp"]))
    predicted = np.mean(var / spp) + oracle_noise
    rel_rmse = np.sqrt(max(mse - oracle_noise, 0.0)) / np.sqrt(np.mean(ref ** 2))
    return rel_rmse, mse / predicted


def test_cornell_config_is_unbiased_against_fp64_oracle(ctx):
    """Cornell 256^2, 64 spp, depth 4, seed 1 against the 2048-spp FP64 oracle: the error
    is Monte Carlo noise only (MSE ratio ~1) and the relative RMSE is stated."""
    g = np.load(os.path.join(ROOT, "tests", "golden", "cornell_fp64.npz"))
    sc = S.Scene(ctx, S.make_cornell_scene(256, 256))
    film = S.render(ctx, sc, S.request(256, 256, 64, 4, 1)).astype(np.float64) / 64
    rel_rmse, ratio = _fp64_check(film, g, 64)
    assert 0.9 < ratio < 1.1, ratio
    assert rel_rmse < 0.2, rel_rmse
    # At 8192 spp the relative RMSE is under 1% (noise shrinks as 1/sqrt(spp)).
    film = S.render(ctx, sc, S.request(256, 256, 8192, 4, 1)).astype(np.float64) / 8192
    rel_rmse, ratio = _fp64_check(film, g, 8192)
    assert rel_rmse < 0.01 and 0.8 < ratio < 1.2, (rel_rmse, ratio)


def test_heavy_config_crop_is_unbiased_against_fp64_oracle(ctx):
    """Heavy render (1024^2, depth 8, GGX + glass) at 64 spp against the FP64 oracle's
    4096-spp centre crop."""
    from lux_b200 import scenes as SC
    g = np.load(os.path.join(ROOT, "tests", "golden", "heavy_fp64.npz"))
    x0, y0, x1, y1 = (int(v) for v in g["rect"])
    sc = S.Scene(ctx, SC.heavy_render_scene(1024, 1024))
    film = S.render(ctx, sc, S.request(1024, 1024, 64, 8, 1)).astype(np.float64) / 64
    rel_rmse, ratio = _fp64_check(film[y0:y1, x0:x1], g, 64)
    assert 0.8 < ratio < 1.25, ratio
    assert rel_rmse < 0.3, rel_rmse


def test_autotune_render_keeps_the_image(ctx):
    from lux_b200 import autotune
    from lux_b200 import scenes as SC
    sc = S.Scene(ctx, SC.heavy_render_scene(96, 96))
    req = S.request(96, 96, 8, 6, 2)
    want = S.render(ctx, sc, req)
    saved = [ctx.get_option(o) for o in (1, 3, 4, 7)]
    try:
        res = autotune.autotune_render(ctx, sc, req)
        assert res.candidates >= 6 and res.best_ms <= res.default_ms
        assert ctx.get_option(lux_b200.OPT_PATH_BUDGET) == res.budget
        assert ctx.get_option(lux_b200.OPT_REFILL_BLOCKS) == res.refill_blocks
        assert res.refill_blocks in (0, 1, 2)
        assert np.array_equal(S.render(ctx, sc, req), want)
        # Every launch shape of the refilling kernels renders the same image.
        ctx.set_option(lux_b200.OPT_TRACE_VARIANT, 0)
        for blocks in (1, 2, 3, 0):
            ctx.set_option(lux_b200.OPT_REFILL_BLOCKS, blocks)
            assert np.array_equal(S.render(ctx, sc, req), want)
    finally:
        for o, v in zip((1, 3, 4, 7), saved):
            ctx.set_option(o, v)


def _env_scene(w, h, image, scale=(0.35, 0.35, 0.35)):
    """The reference's image-env probe scene (app/render_runner.cpp:98-136)."""
    b = S.SceneBuilder()
    receiver = b.add_material(S.lambert((np.float32(0.75),) * 3))
    glossy = b.add_material(S.ggx((np.float32(0.8), np.float32(0.6), np.float32(0.3)),
                                  np.float32(0.25), np.float32(0.0)))
    b.add_quad((-1.2, 0, 1.2), (1.2, 0, 1.2), (1.2, 0, -1.2), (-1.2, 0, -1.2), receiver)
    b.add_quad((-0.4, 0.05, 0.3), (0.4, 0.05, 0.3), (0.4, 0.7, 0.0), (-0.4, 0.7, 0.0), glossy)
    b.add_image_infinite_light(image, scale)
    cam = ((0.0, 0.8, 2.8), (0.0, 0.0, 0.0), 35.0, float(np.float32(w) / np.float32(h)))
    b.set_pinhole_camera(*cam)
    return b, cam


@pytest.mark.skipif(not Ref.available(), reason="reference harness not built")
@pytest.mark.parametrize("which", ["cli_2x2", "random_32x16"])
def test_image_environment_light_matches_reference(ctx, which):
    """Image infinite light (sampling by texel weights, lookup on misses, MIS) against
    the reference CPU tracer's add_image_infinite_light."""
    w = h = 40
    spp, depth, seed = 64, 4, 3
    if which == "cli_2x2":
        image = np.array([[[1.4, 1.0, 0.7], [0.2, 0.3, 0.8]],
                          [[0.1, 0.2, 0.5], [0.8, 1.1, 1.5]]], np.float32)
    else:
        image = np.random.default_rng(8).gamma(0.6, 1.5, (16, 32, 3)).astype(np.float32)
    b, cam = _env_scene(w, h, image)
    sc = S.Scene(ctx, b)
    gpu = S.render_samples(ctx, sc, S.request(w, h, spp, depth, seed))
    tris, mids, mats, lights = _ref_arrays(b)
    camera = np.array([*cam[0], *cam[1], cam[2], cam[3]], np.float32)
    ref = Ref().render_scene(tris, mids, mats, lights, camera, w, h, spp, depth, seed,
                             threads=THREADS, env_image=image)
    assert np.isfinite(gpu).all() and gpu.mean() > 0
    assert _agreement(gpu, ref) >= 0.95
    assert _z_fraction(gpu, ref) <= 0.01


def many_lights(width=48, height=48, count=96, seed=21):
    """A floor lit by many small emissive triangles of different powers at different
    heights, a point light among them, a distant light and a dim sky: the case the light
    tree is for."""
    rng = np.random.default_rng(seed)
    b = S.SceneBuilder()
    f = np.float32
    floor = b.add_material(S.lambert((f(0.7), f(0.7), f(0.7))))
    glossy = b.add_material(S.ggx((f(0.8), f(0.7), f(0.5)), f(0.35), f(0.0)))
    b.add_quad((-3, 0, 3), (3, 0, 3), (3, 0, -3), (-3, 0, -3), floor)
    b.add_quad((-1.0, 0.0, -0.5), (1.0, 0.0, -0.5), (1.0, 1.2, -0.8), (-1.0, 1.2, -0.8), glossy)
    for i in range(count):
        e = rng.gamma(1.0, 4.0, 3).astype(f) + f(0.1)
        m = b.add_material(S.emissive(tuple(e), two_sided=bool(i % 3 == 0)))
        c = np.array([rng.uniform(-2.8, 2.8), rng.uniform(0.05, 1.5), rng.uniform(-2.8, 2.8)])
        size = rng.uniform(0.03, 0.12)
        d = rng.normal(size=(2, 3))
        v0 = c
        v1 = c + size * d[0] / np.linalg.norm(d[0])
        v2 = c + size * d[1] / np.linalg.norm(d[1])
        b.add_triangle(tuple(v0), tuple(v1), tuple(v2), m)
    b.add_point_light((0.4, 0.6, 0.9), (0.8, 0.7, 0.6))
    b.add_distant_light((0.2, 1.0, 0.3), (0.15, 0.15, 0.12))
    b.add_uniform_infinite_light((0.02, 0.02, 0.03))
    cam = ((0.0, 2.6, 3.4), (0.0, 0.0, 0.0), 50.0, float(np.float32(width) / np.float32(height)))
    b.set_pinhole_camera(*cam)
    return b, cam


@pytest.mark.skipif(not Ref.available(), reason="reference harness not built")
@pytest.mark.parametrize("scene", ["many_lights", "material_zoo"])
def test_light_selection_matches_reference(ctx, scene):
    """sample_scene_light + light_pmf for the uniform, power and tree samplers at random
    shading positions: the same light, the same pmf bits."""
    b, cam = many_lights() if scene == "many_lights" else material_zoo()
    sc = S.Scene(ctx, b)
    tris, mids, mats, lights = _ref_arrays(b)
    camera = np.array([*cam[0], *cam[1], cam[2], cam[3]], np.float32)
    rng = np.random.default_rng(4)
    n = 20000
    pos = rng.uniform([-3.5, -0.5, -3.5], [3.5, 2.5, 3.5], (n, 3)).astype(np.float32)
    u = rng.random(n, dtype=np.float32)
    u[:4] = [0.0, np.float32(0.99999994), 1.0, np.float32(0.5)]
    ref = Ref()
    for sampler in (S.SAMPLER_UNIFORM, S.SAMPLER_POWER, S.SAMPLER_TREE):
        got = sc.select_lights(pos, u, sampler)
        want = ref.select_lights(tris, mids, mats, lights, camera, sampler, pos, u)
        assert np.array_equal(got[0], want[0]), sampler
        assert np.array_equal(got[1], want[1]), sampler
        assert np.array_equal(got[2], want[2]), sampler
        assert (got[0] >= 0).all()
    # The tree picks by position: the pmfs differ from the power table's.
    tree = sc.select_lights(pos, u, S.SAMPLER_TREE)
    power = sc.select_lights(pos, u, S.SAMPLER_POWER)
    assert not np.array_equal(tree[1], power[1])


@pytest.mark.skipif(not Ref.available(), reason="reference harness not built")
def test_light_tree_render_matches_reference(ctx):
    """-light-sampler bvh: per-sample agreement and per-pixel means against the reference
    CPU tracer with the same sampler, and a lower median pixel variance than power
    selection here (the reference's own tracer gives 0.0077 against 0.0103)."""
    w = h = 48
    spp, depth, seed = 32, 4, 9
    b, cam = many_lights(w, h)
    sc = S.Scene(ctx, b)
    gpu = S.render_samples(ctx, sc, S.request(w, h, spp, depth, seed,
                                              light_sampler=S.SAMPLER_TREE))
    tris, mids, mats, lights = _ref_arrays(b)
    camera = np.array([*cam[0], *cam[1], cam[2], cam[3]], np.float32)
    ref = Ref().render_scene(tris, mids, mats, lights, camera, w, h, spp, depth, seed,
                             light_sampler=S.SAMPLER_TREE, threads=THREADS)
    assert np.isfinite(gpu).all() and gpu.mean() > 0
    assert _agreement(gpu, ref) >= 0.97
    assert _z_fraction(gpu, ref) <= 0.01
    power = S.render_samples(ctx, sc, S.request(w, h, spp, depth, seed))
    assert np.median(gpu.var(axis=1)) < 0.85 * np.median(power.var(axis=1))


def emissive_mesh_scene(vertices=None, w=32, h=32):
    """Cornell box plus a mesh of separate emissive triangles (two instances; the first
    triangle starts with no area, so no light) and a point light."""
    rng = np.random.default_rng(17)
    b = S.make_cornell_scene(w, h)
    if vertices is None:
        c = rng.uniform([-0.6, 0.2, -0.6], [0.6, 1.0, 0.6], (12, 1, 3))
        vertices = (c + rng.normal(scale=0.08, size=(12, 3, 3))).reshape(-1, 3).astype(np.float32)
        vertices[1] = vertices[2] = vertices[0]          # degenerate: no light
    n = len(vertices) // 3
    mats = [b.add_material(S.emissive((float(2 + i % 4), 3.0, float(1 + i % 3)),
                                      two_sided=bool(i % 2))) for i in range(n)]
    mesh = b.add_mesh(S.Mesh(vertices, np.arange(3 * n, dtype=np.uint32).reshape(n, 3),
                             np.asarray(mats, np.int32)))
    b.add_instance(mesh, np.array([[1, 0, 0, 0.0], [0, 1, 0, 0.5], [0, 0, 1, 0.2]], np.float32))
    c_, s_ = np.float32(np.cos(0.5)), np.float32(np.sin(0.5))
    b.add_instance(mesh, np.array([[c_, 0, s_, 0.1], [0, 0.9, 0, 0.4], [-s_, 0, c_, -0.3]],
                                  np.float32))
    b.add_point_light((0.2, 1.6, 0.5), (0.6, 0.6, 0.5))
    return b, mesh, vertices


@pytest.mark.parametrize("change", ["move", "grow", "shrink"])
def test_emissive_mesh_update_rederives_light_tables(ctx, change):
    """Moving an emissive mesh re-derives areas, powers, the alias table and the light
    tree: selections, pmfs and renders equal a scene created from the moved vertices,
    also when the light count grows past or falls below the tables' first size."""
    b, mesh, v = emissive_mesh_scene()
    sc = S.Scene(ctx, b)
    moved = v.copy()
    moved[:, 1] += np.float32(0.05) * np.sin(4.0 * moved[:, 0]).astype(np.float32)
    if change == "grow":                  # the degenerate triangle gains area
        moved[1] += np.float32(0.1)
        moved[2] += np.float32([0.0, 0.0, 0.1])
    elif change == "shrink":              # two triangles lose theirs
        moved[4] = moved[5] = moved[3]
        moved[7] = moved[6]
    sc.update_mesh(mesh, moved)
    fresh_b = emissive_mesh_scene(moved)[0]
    fresh = S.Scene(ctx, fresh_b)
    assert sc.info() == fresh.info()
    before = S.Scene(ctx, b).info()["area_lights"]
    after = sc.info()["area_lights"]
    assert {"move": after == before, "grow": after == before + 2,
            "shrink": after == before - 4}[change]
    rng = np.random.default_rng(3)
    pos = rng.uniform([-1, 0, -1], [1, 2, 1], (4096, 3)).astype(np.float32)
    u = rng.random(4096, dtype=np.float32)
    for sampler in (S.SAMPLER_POWER, S.SAMPLER_TREE):
        got = sc.select_lights(pos, u, sampler)
        want = fresh.select_lights(pos, u, sampler)
        for g, w in zip(got, want):
            assert np.array_equal(g, w)
    req = S.request(32, 32, 4, 5, 3, light_sampler=S.SAMPLER_TREE)
    got = S.render_samples(ctx, sc, req)
    want = S.render_samples(ctx, fresh, req)
    assert np.all(got == want, axis=-1).mean() > 0.999


@pytest.mark.skipif(not Ref.available(), reason="reference harness not built")
def test_device_prepared_instances_and_overrides_match_reference(ctx):
    """Scene preparation on the device: an instanced mesh with normals and texcoords, one
    instance overridden to an emissive material and one to glass; the light tables (area
    lights from the override, in scene-triangle order) select like the reference scene
    built from the same world triangles: the same lights and pmf bits."""
    from lux_b200 import scenes as SC
    w = h = 32
    b = S.make_cornell_scene(w, h)
    v, idx = SC.displaced_sphere(2, (0.0, 0.0, 0.0), 0.2, 0.03, 9)
    nrm = (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)
    uv = np.random.default_rng(2).random((len(v), 2)).astype(np.float32)
    rough = b.add_material(S.ggx((0.7, 0.6, 0.5), 0.3, 0.0))
    glow = b.add_material(S.emissive((2.0, 1.5, 1.0)))
    glass = b.add_material(S.dielectric((1, 1, 1), 1.5))
    mesh = b.add_mesh(S.Mesh(v, idx, np.full(len(idx), rough, np.int32), nrm, uv))
    for k, override in enumerate([-1, glow, glass]):
        m = np.array([[1, 0, 0, -0.5 + 0.5 * k], [0, 1, 0, 0.4], [0, 0, 1, 0.9]], np.float32)
        b.add_instance(mesh, m, override)
    sc = S.Scene(ctx, b)
    tris, mids, mats, lights = _ref_arrays(b)
    info = sc.info()
    assert info["triangles"] == len(tris) and info["area_lights"] == 2 + len(idx)
    rng = np.random.default_rng(5)
    pos = rng.uniform([-1, 0, 0], [1, 2, 2], (4096, 3)).astype(np.float32)
    u = rng.random(4096, dtype=np.float32)
    cam = ((0.0, 1.0, 3.35), (0.0, 1.0, 0.9), 40.0, 1.0)
    camera = np.array([*cam[0], *cam[1], cam[2], cam[3]], np.float32)
    ref = Ref()
    for sampler in (S.SAMPLER_POWER, S.SAMPLER_TREE):
        got = sc.select_lights(pos, u, sampler)
        want = ref.select_lights(tris, mids, mats, lights, camera, sampler, pos, u)
        for g, x in zip(got, want):
            assert np.array_equal(g, x)


def image_emission_scene(w=40, h=40, with_env=False):
    """A floor under two image-emissive panels (texture coordinates past [0, 1], so the
    lookup wraps; one panel two-sided with its own scale), a constant lamp, and
    optionally an image light on the same image."""
    f = np.float32
    rng = np.random.default_rng(13)
    image = rng.gamma(0.8, 2.0, (6, 8, 3)).astype(f)
    b = S.SceneBuilder()
    img = b.add_image(image)
    floor = b.add_material(S.lambert((f(0.7), f(0.7), f(0.7))))
    glossy = b.add_material(S.ggx((f(0.8), f(0.7), f(0.5)), f(0.3), f(0.0)))
    panel = b.add_material(S.image_emissive(img, (f(1.5), f(1.2), f(1.0))))
    panel2 = b.add_material(S.image_emissive(img, (f(0.4), f(0.6), f(0.9)), two_sided=True))
    lamp = b.add_material(S.emissive((2.0, 2.0, 2.0)))
    b.add_quad((-1.5, 0, 1.5), (1.5, 0, 1.5), (1.5, 0, -1.5), (-1.5, 0, -1.5), floor)
    b.add_quad((-0.2, 0.1, -0.6), (0.6, 0.1, -0.6), (0.6, 0.7, -0.9), (-0.2, 0.7, -0.9), glossy)
    b.add_quad((-0.7, 1.6, -0.2), (0.7, 1.6, -0.2), (0.7, 1.6, 0.6), (-0.7, 1.6, 0.6), lamp)
    v = np.array([[-1.0, 1.2, -0.8], [0.2, 1.2, -0.8], [0.2, 1.2, 0.4], [-1.0, 1.2, 0.4],
                  [0.5, 0.2, 0.8], [1.1, 0.2, 0.8], [1.1, 0.9, 0.8], [0.5, 0.9, 0.8]], f)
    uv = np.array([[-0.3, 0.2], [1.7, 0.1], [1.6, 2.4], [-0.2, 2.3],
                   [0.1, 0.1], [0.9, 0.1], [0.9, 0.9], [0.1, 0.9]], f)
    idx = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7]], np.uint32)
    mesh = b.add_mesh(S.Mesh(v, idx, np.array([panel, panel, panel2, panel2], np.int32), None, uv))
    b.add_instance(mesh)
    if with_env:
        b.lights.append(S.LightDesc(S.LIGHT_IMAGE_INFINITE, S._F3(0, 0, 0), S._F3(0.05, 0.05, 0.05),
                                    img))
    cam = ((0.0, 0.9, 3.0), (0.0, 0.5, 0.0), 45.0, float(f(w) / f(h)))
    b.set_pinhole_camera(*cam)
    return b, cam, image


@pytest.mark.skipif(not Ref.available(), reason="reference harness not built")
@pytest.mark.parametrize("sampler,with_env", [(S.SAMPLER_POWER, False), (S.SAMPLER_TREE, True),
                                              (S.SAMPLER_UNIFORM, True)])
def test_image_emission_matches_reference(ctx, sampler, with_env):
    """Material::image_emissive: emission read at the hit's texture coordinates (seen
    directly, by NEE at the sampled point and in MIS), light power from the image's mean
    luminance, against the reference CPU tracer; the env light shares the image."""
    w = h = 40
    spp, depth, seed = 32, 4, 6
    b, cam, image = image_emission_scene(w, h, with_env)
    sc = S.Scene(ctx, b)
    assert sc.info()["area_lights"] == 2 + 4
    gpu = S.render_samples(ctx, sc, S.request(w, h, spp, depth, seed, light_sampler=sampler))
    tris, mids, mats, lights = _ref_arrays(b)
    ext = np.array([[m.emission_source, m.emission_image, *m.emission_scale]
                    for m in b.materials], np.float32)
    camera = np.array([*cam[0], *cam[1], cam[2], cam[3]], np.float32)
    ref = Ref().render_scene(tris, mids, mats, lights, camera, w, h, spp, depth, seed,
                             light_sampler=sampler, threads=THREADS, env_image=image,
                             material_ext=ext, uvs=b.world_uvs())
    assert np.isfinite(gpu).all() and gpu.mean() > 0
    assert _agreement(gpu, ref) >= 0.97
    assert _z_fraction(gpu, ref) <= 0.01
