"""The oracle restatement pinned against the reference (CPU only).

Pins: the committed fixtures (tests/golden/lbvh_reference.npz, written by the reference's
own host code through tests/golden/make_golden.py) and, where the reference is present,
the reference live (oracle/_ref).
"""
import numpy as np
import pytest

from lux_b200 import workloads as W
from oracle.bindings import Ref

FIELDS = ["sorted_ids", "node_left", "node_right", "node_bounds"]


def _bounds(oracle, case):
    prims = case["prims"]
    return oracle.triangle_bounds(prims) if int(case["kind"]) == 0 else prims


def test_oracle_matches_golden_lbvh(oracle, golden_lbvh):
    for name, case in golden_lbvh.items():
        tree = oracle.build(_bounds(oracle, case))
        for f in FIELDS:
            assert np.array_equal(tree[f], case[f]), (name, f)
        if len(case["sorted_ids"]) > 1:
            assert np.array_equal(tree["sorted_codes"].astype(np.uint32), case["sorted_codes"]), name


def test_oracle_trace_matches_golden_gpu_order(oracle, golden_lbvh):
    for name, case in golden_lbvh.items():
        if int(case["kind"]) != 0:
            continue
        tree = oracle.build(_bounds(oracle, case))
        hid, ht = oracle.trace(case["prims"], tree, case["rays"])
        assert np.array_equal(hid, case["hit_id_gpu_order"]), name
        assert np.array_equal(ht, case["hit_t_gpu_order"]), name
        assert (hid >= 0).sum() > 0 or len(case["sorted_ids"]) < 4, name


def test_cpu_order_differs_only_by_ties(oracle, golden_lbvh):
    """bvh/bvh_validation.h:63-85: an equal-t different-triangle result is a tie."""
    for name, case in golden_lbvh.items():
        if int(case["kind"]) != 0:
            continue
        g_id, g_t = case["hit_id_gpu_order"], case["hit_t_gpu_order"]
        c_id, c_t = case["hit_id_cpu_order"], case["hit_t_cpu_order"]
        assert np.array_equal(g_id >= 0, c_id >= 0), name
        hit = g_id >= 0
        assert np.array_equal(g_t[hit], c_t[hit]), name


def test_any_hit_agrees_with_closest(oracle, golden_lbvh):
    for name, case in golden_lbvh.items():
        if int(case["kind"]) != 0:
            continue
        tree = oracle.build(_bounds(oracle, case))
        a_id, _ = oracle.trace(case["prims"], tree, case["rays"], any_hit=True)
        assert np.array_equal(a_id >= 0, case["hit_id_gpu_order"] >= 0), name


def _brute_overlap(boxes_a, boxes_b, self_pairs):
    lo_a, hi_a = boxes_a[:, None, 0:3], boxes_a[:, None, 3:6]
    lo_b, hi_b = boxes_b[None, :, 0:3], boxes_b[None, :, 3:6]
    ov = ~((lo_b > hi_a) | (hi_b < lo_a)).any(axis=2)     # ov[a, b]
    a, b = np.nonzero(ov)
    if self_pairs:
        keep = b > a
        return {(int(x), int(y)) for x, y in zip(a[keep], b[keep])}
    return {(int(x), int(y)) for x, y in zip(a, b)}


def test_oracle_overlap_matches_brute_force(oracle):
    boxes = W.query_boxes(600, seed=41, half_extent=0.03)
    tree = oracle.build(boxes)
    pairs, found = oracle.overlap(tree, boxes, self_pairs=True)
    assert found == len(pairs)
    assert {tuple(p) for p in pairs.tolist()} == _brute_overlap(boxes, boxes, True)
    queries = W.query_boxes(300, seed=42, half_extent=0.02)
    pairs, found = oracle.overlap(tree, queries, self_pairs=False)
    # cross pairs are (tree primitive, query primitive)
    assert {tuple(p) for p in pairs.tolist()} == _brute_overlap(boxes, queries, False)


def test_oracle_63bit_tree_is_consistent(oracle):
    """63-bit codes have no reference; check the Karras invariants directly."""
    tris = W.soup_triangles(5000, seed=51)
    b = oracle.triangle_bounds(tris)
    t = oracle.build(b, morton_bits=63)
    codes = t["sorted_codes"]
    assert np.all(codes[1:] >= codes[:-1])
    n = len(codes)
    seen = np.zeros(2 * n - 1, np.int32)
    stack = [0]
    while stack:
        i = stack.pop()
        seen[i] += 1
        if t["node_left"][i] >= 0:
            stack += [t["node_left"][i], t["node_right"][i]]
    assert np.all(seen == 1)
    # Leaves keep input order among equal codes (stability).
    ids = t["sorted_ids"]
    same = codes[1:] == codes[:-1]
    assert np.all(ids[1:][same] > ids[:-1][same])
    # 30-bit and 63-bit trees agree on every hit (different shapes, same closest hit).
    rays = W.uniform_rays(4000, seed=52)
    t30 = oracle.build(b)
    h30, tt30 = oracle.trace(tris, t30, rays)
    h63, tt63 = oracle.trace(tris, t, rays)
    assert np.array_equal(tt30, tt63)


@pytest.mark.skipif(not Ref.available(), reason="reference not built here")
@pytest.mark.parametrize("n,seed", [(5, 1), (64, 2), (999, 3), (20000, 4)])
def test_oracle_matches_reference_live(oracle, n, seed):
    ref = Ref()
    tris = W.soup_triangles(n, seed=seed)
    r = ref.lbvh_build(tris)
    o = oracle.build(oracle.triangle_bounds(tris))
    for f in FIELDS:
        assert np.array_equal(o[f], r[f]), f
    assert np.array_equal(o["sorted_codes"].astype(np.uint32), r["sorted_codes"])
    rays = W.uniform_rays(3000, seed=seed + 100)
    rid, rt = ref.build_and_trace(tris, rays, gpu_order=True)
    oid, ot = oracle.trace(tris, o, rays)
    assert np.array_equal(oid, rid)
    assert np.array_equal(ot, rt)


@pytest.mark.skipif(not Ref.available(), reason="reference harness not built")
def test_fp64_oracle_agrees_with_reference_cpu_tracer():
    """The FP64 oracle and the reference's own CPU tracer estimate the same image: per-
    pixel z-scores are standard normal and the MSE is what their noise predicts."""
    from lux_b200 import scene as S
    from oracle import build as oracle_build
    from oracle.bindings import PT64
    oracle_build.build_pt64()
    w = h = 24
    spp = 256
    b = S.make_cornell_scene(w, h)
    tris = b.world_triangles()
    mids = b.world_material_ids()
    mats = np.array([[m.type, *m.albedo, *m.emission, m.roughness, m.metallic, m.eta,
                      m.emission_two_sided] for m in b.materials], np.float32)
    c = b.camera
    frame = np.array([*c.origin, *c.lower_left, *c.horizontal, *c.vertical], np.float32)
    mo, vo = PT64().render(tris, mids, mats, np.zeros((0, 7), np.float32), frame, w, h, spp, 4,
                           seed=9, threads=4)
    tot, tot2 = Ref().cornell_render(w, h, spp, 4, 1, threads=4)
    mr = (tot.astype(np.float64) / spp).reshape(h, w, 3)
    vr = ((tot2.astype(np.float64) / spp).reshape(h, w, 3) - mr ** 2) * spp / (spp - 1)
    z = (mo - mr) / np.sqrt(vo / spp + vr / spp + 1e-30)
    assert abs(z.mean()) < 0.15 and 0.85 < z.std() < 1.15
    ratio = np.mean((mo - mr) ** 2) / np.mean(vo / spp + vr / spp)
    assert 0.8 < ratio < 1.2
