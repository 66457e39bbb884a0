"""The drop-in shims (lux_b200/integration/: the reference's own GPU LBVH, overlap and
wavefront-integrator interfaces over liblux_gpu.so), compiled against the reference's
headers (oracle/build.py, build_ref_shim) and called through the reference's own types
(oracle/ref_shim_harness.cpp).

Without a GPU: the shims compile and link against the reference and the library (the
build), and the harness loads.  On the B200: build_gpu_lbvh / refit_gpu_lbvh /
download_bvh_for_validation / the validators / intersect_gpu_bvh_stackless /
query_aabb_overlaps_self and _cross with primitive ids that are not the input order, and
make_integrator(WavefrontPathTracer)->render, against the reference's host builder, the
oracle and this library's own C ABI."""
import numpy as np
import pytest

import lux_b200
from lux_b200 import scene as S
from lux_b200 import scenes as SC
from lux_b200 import workloads as W
from oracle.bindings import Oracle, Ref, RefShim

needs_shim = pytest.mark.skipif(not RefShim.available(), reason="shim harness not built")


@needs_shim
def test_shims_link_and_the_harness_loads():
    lib = RefShim().lib
    for name in ("shim_build", "shim_refit", "shim_download", "shim_validate",
                 "shim_intersect", "shim_overlap", "shim_render"):
        assert hasattr(lib, name)


def _case(n, seed):
    """Triangles and their boxes, with primitive ids a permutation of 0..n-1 shifted by
    1000 (the reference reports BvhBuildPrimitive::primitive_id, not input positions);
    triangles_by_id is indexed by primitive id, as intersect_gpu_bvh_stackless reads it."""
    tris = W.soup_triangles(n, seed)
    boxes = Oracle().triangle_bounds(tris)
    ids = (np.random.default_rng(seed).permutation(n) + 1000).astype(np.int32)
    by_id = np.zeros((n + 1000, 9), np.float32)
    by_id[ids] = tris
    return tris, boxes, ids, by_id


@pytest.mark.gpu
@needs_shim
def test_lbvh_shim_matches_the_reference_builder_and_oracle(ctx):
    n = 20_000
    tris, boxes, ids, by_id = _case(n, 21)
    shim = RefShim()
    h = shim.build(boxes, ids)
    try:
        # Topology, boxes and order of the reference's own host builder, ids mapped.
        want = Ref().lbvh_build(boxes, kind=1)
        got = shim.download(h, n)
        assert got["root"] == 0
        assert np.array_equal(got["primitive_ids"], ids[want["sorted_ids"]])
        assert np.array_equal(got["left"], want["node_left"])
        assert np.array_equal(got["right"], want["node_right"])
        assert np.array_equal(got["bounds"], want["node_bounds"])
        assert np.array_equal(got["count"][n - 1:], np.ones(n, np.int32))
        assert np.array_equal(got["root_bounds"], want["node_bounds"][0])
        # Validators: valid as built; a moved box and a repeated id are reported.
        assert shim.validate(h, boxes, ids) == (True, True, "")
        moved = boxes.copy()
        moved[7, 3] += np.float32(0.01)
        ok_s, ok_m, msg = shim.validate(h, moved, ids)
        assert ok_s and not ok_m and msg == "BVH primitive bounds do not match scene primitive"
        dup = ids.copy()
        dup[1] = dup[0]
        assert shim.validate(h, boxes, dup)[2] == "Scene primitive ids are not unique"
        # Closest hits: the oracle's (the reference's stackless order), ids mapped.
        rays = W.uniform_rays(50_000, seed=22).reshape(-1, 8)
        ora = Oracle()
        tree = ora.build(boxes)
        want_id, want_t = ora.trace(tris, tree, rays)
        for _ in range(2):   # the second query reuses the attached triangles
            hid, ht = shim.intersect(h, by_id, rays)
            assert np.array_equal(hid, np.where(want_id >= 0, ids[np.maximum(want_id, 0)], -1))
            assert np.array_equal(ht, want_t)
        # Self overlap: the oracle's pair set in primitive ids, a < b; truncation.
        pairs, found, trunc = shim.overlap(h, None, 1 << 20)
        opairs, ofound = ora.overlap(tree, boxes, self_pairs=True)
        assert found == ofound and not trunc
        mapped = np.sort(ids[opairs], axis=1)
        assert np.all(pairs[:, 0] < pairs[:, 1])
        assert set(map(tuple, pairs.tolist())) == set(map(tuple, mapped.tolist()))
        small, found_small, trunc_small = shim.overlap(h, None, 10)
        assert trunc_small and found_small == found and len(small) == 10
        # Cross overlap against query boxes with their own ids.
        q = W.query_boxes(5_000, 23, half_extent=2e-3)
        qids = (np.arange(len(q)) * 3 + 7).astype(np.int32)
        hq = shim.build(q, qids)
        try:
            cpairs, cfound, _ = shim.overlap(h, hq, 1 << 20)
            wpairs, wfound = ora.overlap(tree, q, self_pairs=False)
            assert cfound == wfound
            wmapped = np.stack([ids[wpairs[:, 0]], qids[wpairs[:, 1]]], axis=1)
            assert set(map(tuple, cpairs.tolist())) == set(map(tuple, wmapped.tolist()))
        finally:
            shim.destroy(hq)
        # Refit: new boxes, same ids -> the reference builder's boxes over the old order;
        # different ids or counts -> false.
        jitter = W.soup_triangles(n, 21) + np.float32(1e-3)
        jboxes = Oracle().triangle_bounds(jitter)
        assert shim.refit(h, jboxes, ids)
        bvh = ctx.build_lbvh(boxes, kind=lux_b200.PRIM_AABBS)
        bvh.refit(jboxes)
        assert np.array_equal(shim.download(h, n)["bounds"], bvh.download().node_bounds)
        assert not shim.refit(h, jboxes, ids[::-1].copy())
        assert not shim.refit(h, jboxes[:-1], ids[:-1])
    finally:
        shim.destroy(h)


@pytest.mark.gpu
@needs_shim
def test_empty_and_single_primitive_shims(ctx):
    shim = RefShim()
    empty = shim.build(np.zeros((0, 6), np.float32), np.zeros(0, np.int32))
    try:
        assert shim.validate(empty, np.zeros((0, 6), np.float32), np.zeros(0, np.int32))[1]
        assert shim.overlap(empty, None, 16)[1] == 0
    finally:
        shim.destroy(empty)
    box = np.array([[0, 0, 0, 1, 1, 1]], np.float32)
    one = shim.build(box, np.array([42], np.int32))
    try:
        got = shim.download(one, 1)
        assert got["primitive_ids"].tolist() == [42] and got["count"].tolist() == [1]
        assert shim.validate(one, box, np.array([42], np.int32))[:2] == (True, True)
    finally:
        shim.destroy(one)


@pytest.mark.gpu
@needs_shim
@pytest.mark.parametrize("which", ["cornell", "sphere_grid"])
def test_integrator_shim_renders_what_the_library_renders(ctx, which):
    """make_integrator(WavefrontPathTracer)->render of the reference's own Scene through the
    shim: the film, debug images and path-log length of lux_render / lux_render_aovs /
    lux_render_path_log on the same scene."""
    w = h = 48
    req = S.request(w, h, 4, 5, 3)
    if which == "cornell":
        builder, desc_builder = S.make_cornell_scene(w, h), None   # the reference's Cornell box
    else:
        builder = desc_builder = SC.sphere_grid_scene(w, h)
    film, shadow, ng, ns, _ = RefShim().render(desc_builder, req, aovs=True)
    _, _, _, _, log_count = RefShim().render(desc_builder, req, path_log=True)
    sc = S.Scene(ctx, builder)
    want = S.render(ctx, sc, req)
    assert np.array_equal(film, want)
    wf, ws, wg, wn = S.render_aovs(ctx, sc, req)
    assert np.array_equal(film, wf)
    # The debug images are per-pixel atomic sums: equal up to the order of the additions.
    for got, exp in ((shadow, ws), (ng, wg), (ns, wn)):
        np.testing.assert_allclose(got, exp, rtol=1e-5, atol=1e-6)
    _, records = S.render_path_log(ctx, sc, req)
    assert log_count == len(records) > 0
