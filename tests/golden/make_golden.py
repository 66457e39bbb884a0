"""Regenerates tests/golden/*.npz from the reference's own host code.

Runs the reference (oracle/_ref/libluxref.so, compiled from the reference sources by
oracle/build.py) on small seeded inputs and stores inputs and outputs.  The fixtures pin
the oracle restatement on machines where the reference itself is absent.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

from lux_b200 import workloads as W  # noqa: E402
from oracle import build as oracle_build  # noqa: E402
from oracle.bindings import Ref  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def lbvh_cases():
    """(name, kind, prims) triples covering sizes and edge cases the reference handles."""
    cases = []
    for n, seed in [(1, 11), (2, 12), (3, 13), (17, 14), (257, 15), (1024, 16)]:
        cases.append((f"soup{n}", 0, W.soup_triangles(n, seed=seed)))
    # All centroids equal: every Morton code ties, order falls back to input index.
    cases.append(("duplicates", 0, np.tile(W.soup_triangles(1, seed=21), (40, 1))))
    # Flat scene (z = 0.5 everywhere): zero extent on one axis (normalized_offset -> 0.5).
    flat = W.soup_triangles(200, seed=22).reshape(200, 3, 3)
    flat[:, :, 2] = 0.5
    cases.append(("flat", 0, flat.reshape(200, 9)))
    # Degenerate triangles (collinear / single point) mixed with regular ones.
    deg = W.soup_triangles(100, seed=23).reshape(100, 3, 3)
    deg[::3, 1] = deg[::3, 0]
    deg[::3, 2] = deg[::3, 0]
    deg[1::5, 2] = 0.5 * (deg[1::5, 0] + deg[1::5, 1])
    cases.append(("degenerate", 0, deg.reshape(100, 9)))
    # Boxes instead of triangles.
    cases.append(("boxes", 1, W.query_boxes(500, seed=24, half_extent=0.02)))
    return cases


def main():
    oracle_build.build_ref()
    ref = Ref()
    lbvh = {}
    for name, kind, prims in lbvh_cases():
        r = ref.lbvh_build(prims, kind)
        lbvh[f"{name}/kind"] = np.array(kind)
        lbvh[f"{name}/prims"] = prims
        for key, val in r.items():
            lbvh[f"{name}/{key}"] = val
        if kind == 0:
            rays = W.uniform_rays(512, seed=31)
            # Aim half the rays at triangle centroids so that hits are plentiful.
            c = prims.reshape(-1, 3, 3).mean(axis=1)
            m = len(rays) // 2
            tgt = c[np.arange(m) % len(c)]
            d = tgt - rays[:m, 0:3]
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            rays[:m, 4:7] = d
            gid, gt = ref.build_and_trace(prims, rays, gpu_order=True)
            cid, ct = ref.build_and_trace(prims, rays, gpu_order=False)
            lbvh[f"{name}/rays"] = rays
            lbvh[f"{name}/hit_id_gpu_order"] = gid
            lbvh[f"{name}/hit_t_gpu_order"] = gt
            lbvh[f"{name}/hit_id_cpu_order"] = cid
            lbvh[f"{name}/hit_t_cpu_order"] = ct
    np.savez_compressed(os.path.join(OUT, "lbvh_reference.npz"), **lbvh)

    scene = ref.cornell_scene(32, 32)
    total, total2, samples = ref.cornell_render(32, 32, 8, 4, 1, threads=os.cpu_count() or 1,
                                                samples=True)
    np.savez_compressed(os.path.join(OUT, "cornell_reference.npz"),
                        width=32, height=32, spp=8, max_depth=4, seed=1,
                        triangles=scene["triangles"], material_ids=scene["material_ids"],
                        materials=scene["materials"], camera=scene["camera"],
                        film_sum=total, film_sumsq=total2, samples=samples)
    print("wrote", os.listdir(OUT))


if __name__ == "__main__":
    main()
