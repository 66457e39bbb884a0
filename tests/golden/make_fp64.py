"""FP64 high-spp oracle images for the render configurations (test fixtures).

Renders, with the double-precision oracle (oracle/pt64.c), the per-pixel mean radiance
and per-sample variance of
  * the Cornell box at 256x256, max depth 4 (the Cornell render configuration), all
    pixels, 2048 samples per pixel;
  * the heavy render scene at 1024x1024, max depth 8, the 64x64 crop at the image centre
    (pixels 480..543 in x and y), 4096 samples per pixel.
The tests and the bench compare GPU renders of the same configurations with these:
relative RMSE, and the ratio of the measured mean squared error to the one Monte Carlo
noise alone predicts (1 for an unbiased renderer).

    python tests/golden/make_fp64.py [threads]
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

from lux_b200 import scene as S  # noqa: E402
from lux_b200 import scenes as SC  # noqa: E402
from oracle import build as oracle_build  # noqa: E402
from oracle.bindings import PT64  # noqa: E402

HEAVY_RECT = (480, 480, 544, 544)


def scene_arrays(b):
    tris = b.world_triangles()
    mids = b.world_material_ids()
    mats = np.array([[m.type, *m.albedo, *m.emission, m.roughness, m.metallic, m.eta,
                      m.emission_two_sided] for m in b.materials], np.float32)
    lights = np.array([[l.kind, *l.vec, *l.value] for l in b.lights], np.float32).reshape(-1, 7)
    c = b.camera
    frame = np.array([*c.origin, *c.lower_left, *c.horizontal, *c.vertical], np.float32)
    return tris, mids, mats, lights, frame


def render(b, w, h, spp, depth, rect, threads):
    tris, mids, mats, lights, frame = scene_arrays(b)
    t0 = time.time()
    mean, var = PT64().render(tris, mids, mats, lights, frame, w, h, spp, depth, seed=20261203,
                              rect=rect, threads=threads)
    print(f"  {w}x{h} rect {rect} {spp} spp depth {depth}: {time.time() - t0:.1f} s")
    return mean, var


def main():
    threads = int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 1)
    oracle_build.build_pt64()
    out = os.path.dirname(os.path.abspath(__file__))
    mean, var = render(S.make_cornell_scene(256, 256), 256, 256, 2048, 4, None, threads)
    np.savez_compressed(os.path.join(out, "cornell_fp64.npz"), mean=mean.astype(np.float32),
                        var=var.astype(np.float32), spp=2048, width=256, height=256,
                        max_depth=4)
    mean, var = render(SC.heavy_render_scene(1024, 1024), 1024, 1024, 4096, 8, HEAVY_RECT,
                       threads)
    np.savez_compressed(os.path.join(out, "heavy_fp64.npz"), mean=mean.astype(np.float32),
                        var=var.astype(np.float32), spp=4096, width=1024, height=1024,
                        max_depth=8, rect=np.array(HEAVY_RECT))


if __name__ == "__main__":
    main()
