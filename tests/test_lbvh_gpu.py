"""LBVH CUDA path vs the oracle, through the C ABI (B200)."""
import numpy as np
import pytest

import lux_b200
from lux_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _bounds(oracle, case):
    prims = case["prims"]
    return oracle.triangle_bounds(prims) if int(case["kind"]) == 0 else prims


def _assert_tree_equal(got, want, codes_too=True):
    assert np.array_equal(got.sorted_ids, want["sorted_ids"])
    assert np.array_equal(got.node_left, want["node_left"])
    assert np.array_equal(got.node_right, want["node_right"])
    assert np.array_equal(got.node_bounds, want["node_bounds"])
    if codes_too and len(got.sorted_ids) > 1:
        assert np.array_equal(got.sorted_codes, want["sorted_codes"].astype(np.uint64))


def test_build_matches_reference_fixtures(ctx, golden_lbvh):
    for name, case in golden_lbvh.items():
        kind = int(case["kind"])
        bvh = ctx.build_lbvh(case["prims"], kind=kind)
        _assert_tree_equal(bvh.download(), case)


def test_trace_matches_reference_fixtures(ctx, golden_lbvh):
    for name, case in golden_lbvh.items():
        if int(case["kind"]) != 0:
            continue
        bvh = ctx.build_lbvh(case["prims"])
        hid, ht = bvh.trace_closest(case["rays"])
        assert np.array_equal(hid, case["hit_id_gpu_order"]), name
        assert np.array_equal(ht, case["hit_t_gpu_order"]), name
        aid = bvh.trace_any(case["rays"])
        assert np.array_equal(aid >= 0, hid >= 0), name


# Sizes at the climb's 256-leaf blocks and the sort's 8192-key tiles, at the 4096-key
# tiles of the allocation-free sort, and well above them.
@pytest.mark.parametrize("n,seed", [(1, 1), (2, 2), (5, 3), (256, 8), (257, 9), (4095, 4),
                                    (4096, 5), (4097, 6), (8191, 10), (8192, 11), (8193, 12),
                                    (16385, 13), (100_000, 7)])
@pytest.mark.parametrize("bits", [30, 63])
def test_build_matches_oracle(ctx, oracle, n, seed, bits):
    tris = W.soup_triangles(n, seed=seed)
    want = oracle.build(oracle.triangle_bounds(tris), morton_bits=bits)
    got = ctx.build_lbvh(tris, morton_bits=bits).download()
    _assert_tree_equal(got, want)


def test_duplicate_codes_keep_input_order(ctx, oracle):
    base = W.soup_triangles(64, seed=9)
    tris = np.concatenate([np.tile(base[:1], (3000, 1)), base, np.tile(base[5:6], (2000, 1))])
    for bits in (30, 63):
        want = oracle.build(oracle.triangle_bounds(tris), morton_bits=bits)
        _assert_tree_equal(ctx.build_lbvh(tris, morton_bits=bits).download(), want)


def test_trace_matches_oracle_with_ties(ctx, oracle):
    # A grid of coplanar unit quads (two triangles each): rays through shared edges and
    # vertices hit several triangles at the same t.
    g = 24
    tris = []
    for i in range(g):
        for j in range(g):
            p0 = (i / g, j / g, 0.5); p1 = ((i + 1) / g, j / g, 0.5)
            p2 = ((i + 1) / g, (j + 1) / g, 0.5); p3 = (i / g, (j + 1) / g, 0.5)
            tris.append(p0 + p1 + p2)
            tris.append(p0 + p2 + p3)
    tris = np.array(tris, np.float32)
    xs = (np.arange(4 * g) / (4 * g)).astype(np.float32)
    xx, yy = np.meshgrid(xs, xs)
    rays = np.zeros((xx.size, 8), np.float32)
    rays[:, 0] = xx.ravel(); rays[:, 1] = yy.ravel(); rays[:, 2] = 1.0
    rays[:, 6] = -1.0; rays[:, 7] = np.inf
    tree = oracle.build(oracle.triangle_bounds(tris))
    want_id, want_t = oracle.trace(tris, tree, rays)
    bvh = ctx.build_lbvh(tris)
    got_id, got_t = bvh.trace_closest(rays)
    assert (want_id >= 0).mean() > 0.9
    assert np.array_equal(got_id, want_id)
    assert np.array_equal(got_t, want_t)


def test_trace_matches_oracle_random(ctx, oracle):
    tris = W.soup_triangles(200_000, seed=11)
    rays = W.uniform_rays(60_000, seed=12)
    tree = oracle.build(oracle.triangle_bounds(tris))
    want_id, want_t = oracle.trace(tris, tree, rays)
    bvh = ctx.build_lbvh(tris)
    got_id, got_t = bvh.trace_closest(rays)
    assert (want_id >= 0).sum() > 1000
    assert np.array_equal(got_id, want_id)
    assert np.array_equal(got_t, want_t)
    any_id = bvh.trace_any(rays)
    assert np.array_equal(any_id >= 0, want_id >= 0)


@pytest.mark.parametrize("variant,budget", [(1, 32), (2, 1), (2, 7), (2, 32), (2, 256), (3, 32), (4, 1), (4, 16), (4, 64)])
def test_trace_variants_identical(ctx, oracle, variant, budget):
    """Tunables change speed only: every traversal variant returns the oracle's hits."""
    tris = W.soup_triangles(100_000, seed=21)
    rays = W.uniform_rays(30_000, seed=22)
    rays[:5, 4:7] = [[1, 0, 0], [0, 1e-13, 1], [0, 0, -1], [0, 1, 0], [1e-14, 0, 1]]
    rays[:5, 4:7] /= np.linalg.norm(rays[:5, 4:7], axis=1, keepdims=True)
    tree = oracle.build(oracle.triangle_bounds(tris))
    want_id, want_t = oracle.trace(tris, tree, rays)
    bvh = ctx.build_lbvh(tris)
    try:
        ctx.set_option(lux_b200.OPT_TRACE_VARIANT, variant)
        ctx.set_option(lux_b200.OPT_TRACE_BUDGET, budget)
        got_id, got_t = bvh.trace_closest(rays)
        any_id = bvh.trace_any(rays)
    finally:
        ctx.set_option(lux_b200.OPT_TRACE_VARIANT, 0)
        ctx.set_option(lux_b200.OPT_TRACE_BUDGET, 16)
    assert np.array_equal(got_id, want_id)
    assert np.array_equal(got_t, want_t)
    assert np.array_equal(any_id >= 0, want_id >= 0)


def test_refit_matches_rebuild_bounds(ctx, oracle):
    tris = W.soup_triangles(50_000, seed=13)
    moved = W.jitter_triangles(tris, seed=14)
    bvh = ctx.build_lbvh(tris)
    before = bvh.download()
    assert lux_b200.refit_gpu_lbvh(bvh, moved)
    after = bvh.download()
    # Topology and order are kept; every box is recomputed from the moved geometry.
    assert np.array_equal(after.sorted_ids, before.sorted_ids)
    assert np.array_equal(after.node_left, before.node_left)
    n = len(tris)
    leaf_boxes = oracle.triangle_bounds(moved)[after.sorted_ids]
    assert np.array_equal(after.node_bounds[n - 1:], leaf_boxes)
    ni = n - 1
    left, right, nb = after.node_left, after.node_right, after.node_bounds
    union = np.concatenate([np.minimum(nb[left[:ni], :3], nb[right[:ni], :3]),
                            np.maximum(nb[left[:ni], 3:], nb[right[:ni], 3:])], axis=1)
    assert np.array_equal(nb[:ni], union)
    assert np.array_equal(bvh.root_bounds(),
                          np.concatenate([leaf_boxes[:, :3].min(0), leaf_boxes[:, 3:].max(0)]))
    # Traversal over the refit tree equals the oracle over the same refit tree.
    rays = W.uniform_rays(20_000, seed=15)
    tree = oracle.build(oracle.triangle_bounds(tris))
    tree["node_bounds"] = after.node_bounds
    want_id, want_t = oracle.trace(moved, tree, rays)
    got_id, got_t = bvh.trace_closest(rays)
    assert np.array_equal(got_id, want_id) and np.array_equal(got_t, want_t)
    # A count mismatch is refused, as refit_gpu_lbvh returns false.
    assert not lux_b200.refit_gpu_lbvh(bvh, moved[:-1])


def test_overlap_self_and_cross_match_oracle(ctx, oracle):
    boxes = W.query_boxes(30_000, seed=16, half_extent=0.004)
    tree = oracle.build(boxes)
    want_pairs, want_found = oracle.overlap(tree, boxes, self_pairs=True)
    bvh = ctx.build_lbvh(boxes, kind=lux_b200.PRIM_AABBS)
    res = bvh.overlap_self(max_pairs=want_found + 10)
    assert res.found_count == want_found and not res.truncated
    assert set(map(tuple, res.pairs.tolist())) == set(map(tuple, want_pairs.tolist()))
    assert np.all(res.pairs[:, 0] < res.pairs[:, 1])

    queries = W.query_boxes(20_000, seed=17, half_extent=0.003)
    qbvh = ctx.build_lbvh(queries, kind=lux_b200.PRIM_AABBS)
    want_pairs, want_found = oracle.overlap(tree, queries, self_pairs=False)
    res = bvh.overlap_cross(qbvh, max_pairs=want_found + 10)
    assert res.found_count == want_found
    assert set(map(tuple, res.pairs.tolist())) == set(map(tuple, want_pairs.tolist()))

    # Truncation: found counts every pair, at most max_pairs are written.
    res = bvh.overlap_cross(qbvh, max_pairs=100)
    assert res.truncated and res.found_count == want_found and len(res.pairs) == 100
    assert set(map(tuple, res.pairs.tolist())) <= set(map(tuple, want_pairs.tolist()))


def test_box_bvh_with_attached_triangles(ctx, oracle):
    """The reference builds from BvhBuildPrimitive boxes and passes triangles at query
    time (bvh/gpu_bvh.cu:893-915): a box BVH + attached triangles answers exactly as the
    triangle BVH does."""
    tris = W.soup_triangles(40_000, seed=31)
    rays = W.uniform_rays(20_000, seed=32)
    boxes = oracle.triangle_bounds(tris)
    box_bvh = ctx.build_lbvh(boxes, kind=lux_b200.PRIM_AABBS)
    with pytest.raises(lux_b200.LuxError):
        box_bvh.trace_closest(rays)
    box_bvh.attach_triangles(tris)
    got_id, got_t = box_bvh.trace_closest(rays)
    want_id, want_t = ctx.build_lbvh(tris).trace_closest(rays)
    assert np.array_equal(got_id, want_id) and np.array_equal(got_t, want_t)
    assert (got_id >= 0).sum() > 100
    with pytest.raises(lux_b200.LuxError) as e:
        box_bvh.attach_triangles(tris[:-1])
    assert e.value.status == lux_b200.LUX_ERR_MISMATCH


def test_empty_and_single(ctx):
    empty = ctx.build_lbvh(np.zeros((0, 9), np.float32))
    rays = W.uniform_rays(10)
    hid, ht = empty.trace_closest(rays)
    assert np.all(hid == -1) and np.all(np.isinf(ht))
    res = empty.overlap_self()
    assert res.found_count == 0
    one = ctx.build_lbvh(np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0]], np.float32))
    r = np.array([[0.2, 0.2, 1, 0, 0, 0, -1, np.inf]], np.float32)
    hid, ht = one.trace_closest(r)
    assert hid[0] == 0 and ht[0] == np.float32(1.0)


def test_device_pointers_stream_ordered(ctx, oracle):
    torch = pytest.importorskip("torch")
    tris = W.soup_triangles(30_000, seed=18)
    rays = W.uniform_rays(10_000, seed=19)
    dt = torch.from_numpy(tris).cuda()
    dr = torch.from_numpy(rays).cuda()
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    try:
        bvh = ctx.build_lbvh(dt)
        hid = torch.empty(len(rays), dtype=torch.int32, device="cuda")
        ht = torch.empty(len(rays), dtype=torch.float32, device="cuda")
        bvh.trace_closest(dr, hid, ht)
        torch.cuda.synchronize()
        want_id, want_t = oracle.trace(tris, oracle.build(oracle.triangle_bounds(tris)), rays)
        assert np.array_equal(hid.cpu().numpy(), want_id)
        assert np.array_equal(ht.cpu().numpy(), want_t)
    finally:
        ctx.set_stream(None)


def test_chunked_host_ray_queries_equal_one_launch(ctx, oracle):
    """Host rays of a query of 1M rays or more are copied in chunks, each traced as it
    lands: results equal the one-launch query over device rays, for host (pinned or
    pageable) and device outputs, without hit distances, and for any-hit."""
    torch = pytest.importorskip("torch")
    tris = W.soup_triangles(200_000, seed=21)
    n = (1 << 20) + 12_345                      # a ragged last chunk
    rays = W.uniform_rays(n, seed=22)
    bvh = ctx.build_lbvh(tris)
    dr = torch.from_numpy(rays).cuda()
    want_id = torch.empty(n, dtype=torch.int32, device="cuda")
    want_t = torch.empty(n, dtype=torch.float32, device="cuda")
    bvh.trace_closest(dr, want_id, want_t)
    want_any = torch.empty(n, dtype=torch.int32, device="cuda")
    bvh.trace_any(dr, want_any)
    torch.cuda.synchronize()
    want_id, want_t, want_any = (x.cpu().numpy() for x in (want_id, want_t, want_any))
    # The one-launch query itself, on a sample, against the oracle.
    sample = rays[:4096]
    o_id, o_t = oracle.trace(tris, oracle.build(oracle.triangle_bounds(tris)), sample)
    assert np.array_equal(want_id[:4096], o_id) and np.array_equal(want_t[:4096], o_t)
    for rounds in range(2):
        hid, ht = bvh.trace_closest(rays)                        # pageable host buffers
        assert np.array_equal(hid, want_id) and np.array_equal(ht, want_t)
    pinned_rays = torch.from_numpy(rays).pin_memory()
    p_id = torch.empty(n, dtype=torch.int32).pin_memory()
    p_t = torch.empty(n, dtype=torch.float32).pin_memory()
    bvh.trace_closest(pinned_rays, p_id, p_t)
    assert np.array_equal(p_id.numpy(), want_id) and np.array_equal(p_t.numpy(), want_t)
    only_id = np.empty(n, np.int32)
    lux_b200._check(ctx._lib.lux_trace_closest(ctx._h, bvh._h, rays.ctypes.data, n,
                                               only_id.ctypes.data, None))
    assert np.array_equal(only_id, want_id)
    d_id = torch.empty(n, dtype=torch.int32, device="cuda")
    d_t = torch.empty(n, dtype=torch.float32, device="cuda")
    bvh.trace_closest(rays, d_id, d_t)                           # host rays, device hits
    torch.cuda.synchronize()
    assert np.array_equal(d_id.cpu().numpy(), want_id)
    assert np.array_equal(d_t.cpu().numpy(), want_t)
    assert np.array_equal(bvh.trace_any(rays), want_any)
    assert (want_id >= 0).any() and (want_id < 0).any()


def test_full_size_microbench_properties(ctx):
    """1,048,576 triangles / 4,194,304 rays: size-independent checks at full size."""
    data = W.lbvh_microbench(n_rays=1 << 22)
    tris, rays = data["triangles"], data["rays"]
    bvh = ctx.build_lbvh(tris)
    t = bvh.download()
    n = len(tris)
    assert np.all(np.diff(t.sorted_codes.astype(np.int64)) >= 0)
    assert np.array_equal(np.sort(t.sorted_ids), np.arange(n))
    same = t.sorted_codes[1:] == t.sorted_codes[:-1]
    assert np.all(t.sorted_ids[1:][same] > t.sorted_ids[:-1][same])
    # every node reached exactly once from the root
    child = np.concatenate([t.node_left[: n - 1], t.node_right[: n - 1]])
    assert np.array_equal(np.sort(child), np.arange(1, 2 * n - 1))
    hid, ht = bvh.trace_closest(rays)
    hit = hid >= 0
    assert 0.2 < hit.mean() < 0.99
    # Every reported hit is a real intersection at the reported t (float64 recheck).
    idx = np.nonzero(hit)[0][:: max(1, hit.sum() // 20000)]
    v = tris[hid[idx]].reshape(-1, 3, 3).astype(np.float64)
    o = rays[idx, 0:3].astype(np.float64); d = rays[idx, 4:7].astype(np.float64)
    p = o + d * ht[idx, None].astype(np.float64)
    nrm = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0])
    dist = np.abs(np.einsum("ij,ij->i", p - v[:, 0], nrm)) / np.linalg.norm(nrm, axis=1)
    assert np.percentile(dist, 99) < 1e-5
    aid = bvh.trace_any(rays)
    assert np.array_equal(aid >= 0, hit)


@pytest.mark.parametrize("n,bits", [(1, 30), (2, 63), (1000, 30), (20000, 63)])
def test_validators_accept_built_trees(ctx, n, bits):
    tris = W.soup_triangles(n, 13)
    bvh = ctx.build_lbvh(tris, lux_b200.PRIM_TRIANGLES, bits)
    assert bvh.validate() == (True, "")
    assert bvh.validate(tris) == (True, "")
    boxes = W.query_boxes(n, 14)
    bb = ctx.build_lbvh(boxes, lux_b200.PRIM_AABBS, bits)
    assert bb.validate(boxes) == (True, "")


def test_validators_report_the_reference_messages(ctx):
    tris = W.soup_triangles(4096, 15)
    bvh = ctx.build_lbvh(tris, lux_b200.PRIM_TRIANGLES, 30)
    moved = tris.copy()
    moved[17, :3] += np.float32(0.25)
    assert bvh.validate(moved) == (False, "BVH primitive bounds do not match scene primitive")
    assert bvh.validate(tris[:4095]) == (
        False, "BVH primitive count does not match scene primitive count")
    bvh.refit(moved)
    assert bvh.validate(moved) == (True, "")
    empty = ctx.build_lbvh(np.zeros((0, 9), np.float32), lux_b200.PRIM_TRIANGLES, 30)
    assert empty.validate() == (False, "BVH is not valid")
    assert empty.validate(np.zeros((0, 9), np.float32)) == (True, "")
    assert bvh.validate(np.zeros((0, 9), np.float32)) == (
        False, "BVH contains primitives for an empty scene")


def _with_variant(ctx, variant, fn):
    try:
        ctx.set_option(lux_b200.OPT_TRACE_VARIANT, variant)
        return fn()
    finally:
        ctx.set_option(lux_b200.OPT_TRACE_VARIANT, 0)


@pytest.mark.parametrize("bits", [30, 63])
def test_wide_walk_matches_binary_walk_through_refits_and_ties(ctx, oracle, bits):
    """The 4-wide walk returns the binary walk's closest and first-found hits, including
    equal-t ties between duplicated triangles, and follows refits and rebuilds."""
    tris = W.soup_triangles(60_000, seed=31)
    tris = np.concatenate([tris, tris[:5000]])          # exact duplicates: t ties
    rays = W.uniform_rays(40_000, seed=32)
    bvh = ctx.build_lbvh(tris, lux_b200.PRIM_TRIANGLES, bits)
    for step in range(3):
        ref_c = _with_variant(ctx, 1, lambda: bvh.trace_closest(rays))
        ref_a = _with_variant(ctx, 1, lambda: bvh.trace_any(rays))
        for variant in (3, 4):
            got_c = _with_variant(ctx, variant, lambda: bvh.trace_closest(rays))
            got_a = _with_variant(ctx, variant, lambda: bvh.trace_any(rays))
            assert np.array_equal(got_c[0], ref_c[0]) and np.array_equal(got_c[1], ref_c[1])
            assert np.array_equal(got_a, ref_a)
        if step == 0:
            tris = W.jitter_triangles(tris, seed=33)
            bvh.refit(tris)
        else:
            tris = W.soup_triangles(70_000, seed=34)
            bvh.rebuild(tris)
    tree = oracle.build(oracle.triangle_bounds(tris))
    want_id, want_t = oracle.trace(tris, tree, rays)
    assert np.array_equal(got_c[0], want_id) and np.array_equal(got_c[1], want_t)


@pytest.mark.parametrize("case", ["planar", "huge", "tiny", "far_offset"])
def test_wide_walk_exact_on_degenerate_extents(ctx, oracle, case):
    """Quantised wide nodes steer only: on flat, huge, tiny and far-offset geometry the
    wide walks return the binary walk's (and the oracle's) hits exactly."""
    tris = W.soup_triangles(20_000, seed=41).reshape(-1, 3, 3)
    rays = W.uniform_rays(20_000, seed=42)
    if case == "planar":
        tris[:, :, 2] = np.float32(0.5)                  # zero extent in z
    elif case == "huge":
        tris = tris * np.float32(1e20)
        rays[:, :3] *= np.float32(1e20)
    elif case == "tiny":
        tris = tris * np.float32(1e-20)
        rays[:, :3] *= np.float32(1e-20)
    else:
        tris = tris + np.float32(3e4)                    # ulp(3e4) ~ 2e-3: coarse grids
        rays[:, :3] += np.float32(3e4)
    tris = np.ascontiguousarray(tris.reshape(-1, 9), np.float32)
    bvh = ctx.build_lbvh(tris)
    want = _with_variant(ctx, 1, lambda: bvh.trace_closest(rays))
    tree = oracle.build(oracle.triangle_bounds(tris))
    oid, ot = oracle.trace(tris, tree, rays)
    assert np.array_equal(want[0], oid) and np.array_equal(want[1], ot)
    for variant in (3, 4):
        got = _with_variant(ctx, variant, lambda: bvh.trace_closest(rays))
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
        got_a = _with_variant(ctx, variant, lambda: bvh.trace_any(rays))
        assert np.array_equal(got_a, _with_variant(ctx, 1, lambda: bvh.trace_any(rays)))


def test_autotune_trace_keeps_results_and_picks_a_candidate(ctx):
    import torch
    from lux_b200 import autotune
    tris = W.soup_triangles(200_000, seed=51)
    rays = W.uniform_rays(100_000, seed=52)
    bvh = ctx.build_lbvh(tris)
    before = bvh.trace_closest(rays)
    variant0 = ctx.get_option(lux_b200.OPT_TRACE_VARIANT)
    budget0 = ctx.get_option(lux_b200.OPT_TRACE_BUDGET)
    try:
        res = autotune.autotune_trace(ctx, bvh, torch.from_numpy(rays).cuda())
        assert res.candidates >= 5 and res.best_ms <= res.default_ms
        assert ctx.get_option(lux_b200.OPT_TRACE_VARIANT) == res.trace_variant
        after = bvh.trace_closest(rays)
        assert np.array_equal(after[0], before[0]) and np.array_equal(after[1], before[1])
    finally:
        ctx.set_option(lux_b200.OPT_TRACE_VARIANT, variant0)
        ctx.set_option(lux_b200.OPT_TRACE_BUDGET, budget0)
