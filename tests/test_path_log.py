"""Path log (lux_render_path_log; RenderOutputs::set_path_log with the wavefront tracer's
records, integrator/pathstate.cuh:19-96, integrator/wavefront_kernels.cu:84-138, 356-558).

The oracle is ref_path_log in the reference harness: the wavefront tracer's record rules
over trace_path's walk, run on the reference's own CPU scene query, light sampler,
direct-light estimate and BSDF sampling.  The CPU tests pin it against the reference
CPU tracer's own debug images (its vertex-0 records are the camera hits the ng / ns
images sum) and check the log's internal rules; the GPU tests compare lux_b200's records
with it, path by path.
"""
import numpy as np
import pytest

from lux_b200 import scene as S
from oracle.bindings import Ref

needs_ref = pytest.mark.skipif(not Ref.available(), reason="reference harness not built")


def log_scene(w=24, h=24):
    """Every material kind, pass-through surfaces in the camera's view (a tinted filter
    and an interface), a one-sided and a two-sided emitter, and point, distant and sky
    lights."""
    f = np.float32
    b = S.SceneBuilder()
    white = b.add_material(S.lambert((f(0.75), f(0.75), f(0.72))))
    glossy = b.add_material(S.ggx((f(0.8), f(0.6), f(0.3)), f(0.3), f(0.0)))
    thin = b.add_material(S.material(S.THIN_LAMBERT, (f(0.6), f(0.8), f(0.6))))
    glass = b.add_material(S.dielectric((1, 1, 1), f(1.5)))
    tint = b.add_material(S.tinted_filter((f(0.25), f(0.65), f(1.0))))
    iface = b.add_material(S.interface())
    lamp = b.add_material(S.emissive((9.0, 8.0, 7.0), two_sided=True))
    lamp2 = b.add_material(S.emissive((2.0, 2.5, 4.0)))
    b.add_quad((-1, 0, 2), (1, 0, 2), (1, 0, -1), (-1, 0, -1), white)
    b.add_quad((-1, 0, -1), (1, 0, -1), (1, 2, -1), (-1, 2, -1), white)
    b.add_quad((-1, 0, 2), (-1, 0, -1), (-1, 2, -1), (-1, 2, 2), glossy)
    b.add_quad((-0.8, 0.1, 0.2), (-0.2, 0.1, 0.2), (-0.2, 0.8, 0.2), (-0.8, 0.8, 0.2), thin)
    b.add_quad((0.2, 0.05, 0.6), (0.7, 0.05, 0.6), (0.7, 0.7, 0.3), (0.2, 0.7, 0.3), glass)
    b.add_quad((-0.1, 0.2, 1.2), (0.5, 0.2, 1.2), (0.5, 0.6, 1.2), (-0.1, 0.6, 1.2), tint)
    b.add_quad((-0.7, 0.5, 1.4), (-0.3, 0.5, 1.4), (-0.3, 0.9, 1.4), (-0.7, 0.9, 1.4), iface)
    b.add_quad((-0.3, 1.7, 0.3), (0.3, 1.7, 0.3), (0.3, 1.7, 0.9), (-0.3, 1.7, 0.9), lamp)
    b.add_quad((0.5, 1.5, -0.95), (0.9, 1.5, -0.95), (0.9, 1.9, -0.95), (0.5, 1.9, -0.95), lamp2)
    b.add_point_light((0.0, 1.4, 1.5), (1.5, 1.5, 1.5))
    b.add_distant_light((-0.3, 1.0, 0.4), (0.3, 0.3, 0.3))
    b.add_uniform_infinite_light((0.05, 0.05, 0.08))
    cam = ((0.0, 0.6, 3.0), (0.0, 0.3, 0.0), 38.0, float(f(w) / f(h)))
    b.set_pinhole_camera(*cam)
    return b, cam


def _ref_log(b, cam, w, h, spp, depth, seed, sampler):
    tris = b.world_triangles()
    mats = np.array([[m.type, *m.albedo, *m.emission, m.roughness, m.metallic, m.eta,
                      m.emission_two_sided] for m in b.materials], np.float32)
    lights = np.array([[l.kind, *l.vec, *l.value] for l in b.lights], np.float32).reshape(-1, 7)
    camera = np.array([*cam[0], *cam[1], cam[2], cam[3]], np.float32)
    args = (tris, b.world_material_ids(), mats, lights, camera, w, h, spp, depth, seed, sampler)
    return Ref().path_log(*args, dtype=S.PATH_LOG_RECORD), args


def _paths(log):
    """Row ranges of each path, keyed by (sample, pixel)."""
    key = log["sample_index"].astype(np.int64) << 32 | log["pixel_index"]
    starts = np.flatnonzero(np.r_[True, key[1:] != key[:-1]])
    ends = np.r_[starts[1:], len(log)]
    return {int(key[s]): (s, e) for s, e in zip(starts, ends)}


def _encode(n):
    return (n / np.linalg.norm(n, axis=-1, keepdims=True) + 1.0) * 0.5


# --------------------------------------------------------------------- oracle (CPU)

@needs_ref
def test_oracle_camera_vertices_sum_to_reference_debug_images():
    """Vertex 0 of each path is the camera ray's hit: summed per pixel, its encoded
    normals are the reference CPU tracer's own ng / ns debug images."""
    w = h = 16
    spp, depth, seed = 4, 5, 3
    b, cam = log_scene(w, h)
    log, args = _ref_log(b, cam, w, h, spp, depth, seed, S.SAMPLER_POWER)
    _, _, want_ng, want_ns = Ref().render_aovs(*args[:-1], S.SAMPLER_POWER)
    first = log[log["vertex"] == 0]
    for field, want in (("ng", want_ng), ("ns", want_ns)):
        got = np.zeros((w * h, 3), np.float64)
        np.add.at(got, first["pixel_index"], _encode(first[field].astype(np.float64)))
        np.testing.assert_allclose(got.reshape(h, w, 3), want, rtol=1e-5, atol=1e-5)


@needs_ref
def test_oracle_log_rules():
    """The record rules of evaluate_hit_kernel hold along every logged path."""
    b, cam = log_scene(16, 16)
    depth = 6
    log, _ = _ref_log(b, cam, 16, 16, 4, depth, 5, S.SAMPLER_TREE)
    assert len(log) > 0
    ev, term = log["event_flags"], log["termination_flags"]
    assert np.all(ev & S.EVENT_SURFACE_HIT)
    # Terminated exactly when a termination reason is set; a spawned ray otherwise.
    assert np.array_equal((ev & S.EVENT_TERMINATED) != 0, term != 0)
    assert np.array_equal((ev & S.EVENT_SPAWNED_RAY) != 0, term == 0)
    passthrough = (ev & S.EVENT_PASSTHROUGH) != 0
    assert passthrough.any() and (~passthrough).any()
    assert np.all(log["bsdf_pdf"][passthrough] == 1.0)
    assert np.all(log["bsdf_pdf_measure"][passthrough] == 3)
    assert set(np.unique(term)) >= {0, S.END_MAX_DEPTH, S.END_NON_SCATTERING}
    assert np.all(log["depth"] <= depth)
    kinds = set()
    for s, e in _paths(log).values():
        p = log[s:e]
        assert np.array_equal(p["vertex"], np.arange(e - s))          # one vertex per step
        assert np.all(p["termination_flags"][:-1] == 0)                # only the last ends
        d = p["depth"]
        pt = (p["event_flags"] & S.EVENT_PASSTHROUGH) != 0
        # Depth grows by one after a scattering vertex, not after a pass-through one.
        assert np.array_equal(d[1:] - d[:-1], (~pt[:-1]).astype(np.int32))
        # The throughput chain: each vertex starts where the previous one left it.
        assert np.array_equal(p["throughput_before"][1:], p["throughput_after"][:-1])
        # The next vertex is seen along the sampled direction.
        np.testing.assert_allclose(p["wo"][1:], -p["wi"][:-1], atol=1e-6)
        kinds.update(int(x) for x in p["material_id"])
    assert len(kinds) >= 7


@needs_ref
def test_oracle_log_capacity():
    """ref_path_log reports every record and writes no more than its capacity."""
    b, cam = log_scene(8, 8)
    full, args = _ref_log(b, cam, 8, 8, 2, 4, 1, S.SAMPLER_POWER)
    tris, mids, mats, lights, camera = args[:5]
    out = np.zeros(8 + 4, S.PATH_LOG_RECORD)
    out["pixel_index"] = -7
    lib = Ref().lib
    n = lib.ref_path_log(tris.ctypes.data, len(tris), mids.ctypes.data, mats.ctypes.data,
                         len(mats), lights.ctypes.data, len(lights), camera.ctypes.data, 8, 8,
                         2, 4, 1, S.SAMPLER_POWER, out.ctypes.data, 8)
    assert n == len(full) > 8
    assert np.array_equal(out[:8], full[:8]) and np.all(out["pixel_index"][8:] == -7)


# --------------------------------------------------------------------- GPU parity

def _compare(got, want, min_match=0.99):
    """Path-by-path comparison; a path matches when its records agree in every integer
    field and to 1e-4 in every float field."""
    gp, wp = _paths(got), _paths(want)
    assert abs(len(gp) - len(wp)) <= max(2, 0.01 * len(wp))
    ints = [n for n in S.PATH_LOG_RECORD.names if S.PATH_LOG_RECORD[n].base.kind in "iu"]
    floats = [n for n in S.PATH_LOG_RECORD.names if S.PATH_LOG_RECORD[n].base.kind == "f"]
    assert len(ints) == 17 and len(floats) == 10
    matched = 0
    for key, (ws, we) in wp.items():
        if key not in gp:
            continue
        gs, ge = gp[key]
        if ge - gs != we - ws:
            continue
        g, w = got[gs:ge], want[ws:we]
        if all(np.array_equal(g[n], w[n]) for n in ints) and all(
                np.allclose(g[n], w[n], rtol=1e-4, atol=1e-5) for n in floats):
            matched += 1
    assert matched >= min_match * len(wp), (matched, len(wp))
    return matched


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("sampler", [S.SAMPLER_POWER, S.SAMPLER_TREE])
def test_path_log_matches_reference(ctx, sampler):
    w = h = 24
    spp, depth, seed = 8, 6, 7
    b, cam = log_scene(w, h)
    sc = S.Scene(ctx, b)
    req = S.request(w, h, spp, depth, seed, light_sampler=sampler)
    film, got = S.render_path_log(ctx, sc, req)
    # The film is lux_render's, and the log is sorted by (sample, pixel, vertex).
    assert np.array_equal(film, S.render(ctx, sc, req))
    order = np.lexsort((got["vertex"], got["pixel_index"], got["sample_index"]))
    assert np.array_equal(order, np.arange(len(got)))
    want, _ = _ref_log(b, cam, w, h, spp, depth, seed, sampler)
    _compare(got, want)
    assert (got["event_flags"] & S.EVENT_PASSTHROUGH).any()
    assert (got["event_flags"] & S.EVENT_LIGHT_VALID).any()


@pytest.mark.gpu
def test_path_log_overflow_and_sample_offset(ctx):
    import lux_b200
    b, _ = log_scene(8, 8)
    sc = S.Scene(ctx, b)
    req = S.request(8, 8, 2, 4, 1)
    _, full = S.render_path_log(ctx, sc, req)
    assert len(full) > 8
    with pytest.raises(lux_b200.LuxError) as e:
        S.render_path_log(ctx, sc, req, capacity=8)
    assert e.value.status == 6                      # LUX_ERR_QUEUE_OVERFLOW
    _, exact = S.render_path_log(ctx, sc, req, capacity=len(full))
    assert np.array_equal(exact, full)
    # sample_offset shifts the logged sample index with the samples themselves.
    _, shifted = S.render_path_log(ctx, sc, S.request(8, 8, 1, 4, 1, sample_offset=1))
    assert np.array_equal(shifted, full[full["sample_index"] == 1])
    # Depth 0: every path ends at its first vertex.
    _, flat = S.render_path_log(ctx, sc, S.request(8, 8, 2, 0, 1))
    assert np.all(flat["vertex"] == 0) and np.all(flat["termination_flags"] != 0)
