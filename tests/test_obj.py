"""OBJ meshes (lux_obj_load) against the reference's own loader (load_obj_into_scene,
run from oracle/_ref), and the asset scenes built on them (bunny, lux-cover, dragon)
through the Python API and lux-render against the reference CPU tracer.

Loader parity is bit-exact: the same triangles in the same order, the same per-corner
vertices in first-use order, normals, texcoords, material ids, mesh box and placement
matrix.  The OBJ files are generated here (seeded), so the tests run where the reference
sources are absent; the reference's own assets are compared too where they exist.
"""
import math
import os
import subprocess

import numpy as np
import pytest

import lux_b200
from lux_b200 import obj as O
from lux_b200 import scene as S
from oracle.bindings import Ref
from oracle.build import REF_ROOT

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
CLI = os.path.join(ROOT, "lux_b200", "lux-render")
REF_ASSETS = os.path.join(REF_ROOT, "assets")
THREADS = os.cpu_count() or 1
KEYS = ("vertices", "normals", "uvs", "indices", "material_ids", "object_to_world", "bounds")

needs_ref = pytest.mark.skipif(not Ref.available(), reason="reference harness not built")


def blob_obj(seed=3, subdiv=12, quads=True, normals="some", texcoords=True, materials=None,
             extras=True, crlf=False):
    """A seeded, bumpy latitude-longitude sphere as OBJ text: quads (both diagonals win
    somewhere) and triangle caps; per-corner normals on some faces, zero-length and
    missing ones elsewhere; texcoords; usemtl groups; negative indices; comments; and,
    with extras, faces the loader must skip (degenerate, non-finite, out of range)."""
    rng = np.random.default_rng(seed)
    rows, cols = subdiv, 2 * subdiv
    lines = ["# generated blob", "o blob"]
    verts = []
    for i in range(rows + 1):
        th = math.pi * i / rows
        for j in range(cols):
            ph = 2 * math.pi * j / cols
            r = 0.3 * (1 + 0.15 * rng.standard_normal())
            verts.append((r * math.sin(th) * math.cos(ph) + 0.05, r * math.cos(th) + 0.31,
                          r * math.sin(th) * math.sin(ph) - 0.02))
    for v in verts:
        lines.append("v %.6f %.6f %.6f" % v)
    for k, v in enumerate(verts):
        n = np.array(v) - np.array([0.05, 0.31, -0.02])
        if k % 17 == 0:
            n = n * 0.0                                     # zero-length normal
        lines.append("vn %.5f %.5f %.5f" % tuple(n))
    for k in range(len(verts)):
        lines.append("vt %.4f %.4f" % (rng.random(), rng.random()))
    mats = materials or [None]

    def vid(i, j):
        return i * cols + (j % cols) + 1

    face = 0
    for i in range(rows):
        m = mats[(i * len(mats)) // rows]
        if m is not None and (i == 0 or mats[((i - 1) * len(mats)) // rows] != m):
            lines.append("usemtl " + m)
        for j in range(cols):
            a, b, c, d = vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)

            def corner(x, rel=False):
                idx = x - len(verts) - 1 if rel else x
                parts = [str(idx)]
                use_t = texcoords and (face % 5 != 1)
                use_n = normals == "all" or (normals == "some" and face % 3 != 0)
                if use_t and use_n:
                    parts = [str(idx), str(idx), str(idx)]
                elif use_n:
                    parts = [str(idx), "", str(idx)]
                elif use_t:
                    parts = [str(idx), str(idx)]
                return "/".join(parts)

            rel = face % 7 == 3
            if quads and (i + j) % 2 == 0:
                lines.append("f " + " ".join(corner(x, rel) for x in (a, b, c, d)))
            else:
                lines.append("f " + " ".join(corner(x, rel) for x in (a, b, c)))
                lines.append("f " + " ".join(corner(x, rel) for x in (a, c, d)))
            face += 1
    if extras:
        lines.append("f 1 1 2")                                  # degenerate
        lines.append("v inf 0 0")
        lines.append("v NaN 0.5 0")                              # reads as 0
        n = len(verts) + 1
        lines.append("f %d 2 3" % n)                             # non-finite position
        lines.append("f %d 2 3" % (n + 1))
        lines.append("f 2 3 %d" % (n + 40))                      # out of range
        lines.append("f 4 5 6 # trailing comment")
    text = "\n".join(lines) + "\n"
    return text.replace("\n", "\r\n") if crlf else text


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def _same(a, b):
    assert a is not None and b is not None
    for k in KEYS:
        assert a[k].shape == b[k].shape, k
        assert np.array_equal(a[k], b[k]), k
    assert a["skipped"] == b["skipped"]


CASES = {
    "source_normals": (dict(), dict(default_material=0)),
    "smooth_normals": (dict(), dict(normal_mode=O.NORMALS_SMOOTH, default_material=2)),
    "face_normals_reversed": (dict(), dict(normal_mode=O.NORMALS_FACE, reverse=True,
                                           default_material=1)),
    "smooth_reversed_flipped_scaled": (dict(normals="all"), dict(
        normal_mode=O.NORMALS_SMOOTH, reverse=True, flip_v=True, scale_mode=O.SCALE_MAX_EXTENT,
        target_extent=0.5, center_xz=True, ground_to_y=True, target_y=0.25, default_material=0)),
    "x_extent_bindings": (dict(materials=["red", "glass", "red", "metal"]), dict(
        normal_mode=O.NORMALS_SMOOTH, scale_mode=O.SCALE_X_EXTENT, target_extent=1.85,
        center_xz=True, ground_to_y=True, bindings={"red": 3, "glass": 7, "metal": 11})),
    "bindings_with_default": (dict(materials=[None, "glass"]), dict(
        bindings={"glass": 5}, default_material=9)),
    "triangles_only_no_attributes": (dict(quads=False, normals="none", texcoords=False),
                                     dict(ground_to_y=True, default_material=0)),
    "crlf": (dict(crlf=True), dict(default_material=0)),
}


@needs_ref
@pytest.mark.parametrize("case", sorted(CASES))
def test_loader_matches_reference_loader(tmp_path, case):
    gen, opts = CASES[case]
    path = _write(tmp_path, "blob.obj", blob_obj(**gen))
    got = O.load_obj(path, **opts)
    want = Ref().obj_load(path, **opts)
    _same(got, want)
    assert got["skipped"][:2] == (1, 1) and got["skipped"][2] >= 1
    assert got["indices"].shape[0] > 400


@needs_ref
@pytest.mark.skipif(not os.path.isdir(REF_ASSETS), reason="reference assets absent")
@pytest.mark.parametrize("name,opts", [
    ("stanford-bunny.obj", dict(ground_to_y=True, default_material=2)),
    ("LUX.obj", dict(normal_mode=O.NORMALS_SMOOTH, scale_mode=O.SCALE_X_EXTENT,
                     target_extent=1.85, center_xz=True, ground_to_y=True,
                     bindings={"L_lambert": 2, "U_glass": 3, "X_metal": 4}))])
def test_loader_matches_reference_on_its_assets(name, opts):
    path = os.path.join(REF_ASSETS, "models", name)
    _same(O.load_obj(path, **opts), Ref().obj_load(path, **opts))


def test_loader_errors_like_the_reference(tmp_path):
    with pytest.raises(lux_b200.LuxError) as e:
        O.load_obj(str(tmp_path / "missing.obj"))
    assert "Cannot open OBJ file" in str(e.value)
    p = _write(tmp_path, "a.obj", blob_obj(materials=["red", "blue"], extras=False))
    with pytest.raises(lux_b200.LuxError) as e:
        O.load_obj(p, bindings={"red": 1})                    # blue is unbound
    assert "has no material binding" in str(e.value)
    p = _write(tmp_path, "b.obj", blob_obj(materials=[None, "red"], extras=False))
    with pytest.raises(lux_b200.LuxError) as e:
        O.load_obj(p, bindings={"red": 1})                    # untagged faces, no default
    assert "no usemtl tag" in str(e.value)
    p = _write(tmp_path, "c.obj", "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 0 1 2\n")
    with pytest.raises(lux_b200.LuxError):
        O.load_obj(p)
    p = _write(tmp_path, "d.obj", "v 0 0 0\nv 1 0 0\nv 2 0 0\nf 1 2 3\n")
    assert O.load_obj(p) is None                              # only a degenerate face


def test_cli_reports_missing_assets_like_the_reference(tmp_path):
    if not os.path.exists(CLI):
        from lux_b200 import build
        build.build()
    r = subprocess.run([CLI, "-scene", "dragon"], capture_output=True, text=True,
                       cwd=str(tmp_path), timeout=120)
    assert r.returncode == 1
    assert "Scene setup failed: Failed to load dragon OBJ: " in r.stderr
    assert "dragon.obj" in r.stderr


def _asset_dir(tmp_path):
    """assets/models with a generated stanford-bunny.obj (plain triangles, no normals,
    as the real file) and LUX.obj (quads, normals, three usemtl groups)."""
    models = tmp_path / "assets" / "models"
    models.mkdir(parents=True)
    bunny = blob_obj(seed=5, subdiv=14, quads=False, normals="none", texcoords=False,
                     extras=False).replace("0.31", "0.11")
    (models / "stanford-bunny.obj").write_text(bunny)
    (models / "LUX.obj").write_text(blob_obj(seed=6, subdiv=10, normals="some",
                                             materials=["L_lambert", "U_glass", "X_metal"],
                                             extras=False))
    return str(tmp_path / "assets")


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("name", ["bunny", "lux-cover"])
def test_asset_scene_matches_reference(ctx, tmp_path, name):
    """The asset scene built through lux_obj_load: the same world triangles as the
    reference scene, and per-sample agreement with its CPU tracer."""
    w = h = 40
    spp, depth, seed = 16, 5, 2
    root = _asset_dir(tmp_path)
    make = O.bunny_scene if name == "bunny" else O.lux_cover_scene
    b = make(root, w, h)
    want_tris, want_mids, want_mats = Ref().asset_scene(name, root, float(np.float32(w) / h))
    assert np.array_equal(b.world_triangles().reshape(-1, 9), want_tris)
    assert np.array_equal(b.world_material_ids(), want_mids)
    mats = np.array([[m.type, *m.albedo, *m.emission, m.roughness, m.metallic, m.eta,
                      m.emission_two_sided] for m in b.materials], np.float32)
    assert np.array_equal(mats, want_mats)
    sc = S.Scene(ctx, b)
    gpu = S.render_samples(ctx, sc, S.request(w, h, spp, depth, seed))
    ref = Ref().asset_render(name, root, w, h, spp, depth, seed, threads=THREADS)
    from test_pathtracer_gpu import _agreement, _z_fraction
    assert np.isfinite(gpu).all() and gpu.mean() > 0
    assert _agreement(gpu, ref) >= 0.97
    assert _z_fraction(gpu, ref) <= 0.01


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("name", ["bunny", "lux-cover"])
def test_cli_asset_scene_matches_reference(tmp_path, name):
    """`lux-render -gpu -scene bunny|lux-cover` from a directory holding assets/: its
    film against the reference CPU tracer's (seed 0, as the reference CLI) per pixel."""
    if not os.path.exists(CLI):
        from lux_b200 import build
        build.build()
    w = h = 32
    spp = 64
    root = _asset_dir(tmp_path)
    out = tmp_path / "o.pfm"
    r = subprocess.run([CLI, "-gpu", "-scene", name, "-size", str(w), str(h), "-spp", str(spp),
                        "-depth", "4", "-output", str(out)], capture_output=True, text=True,
                       cwd=str(tmp_path), timeout=300)
    assert r.returncode == 0, r.stderr
    assert "2 instances, 2 meshes" in r.stdout
    with open(out, "rb") as f:
        assert f.readline() == b"PF\n"
        f.readline()
        f.readline()
        mean = np.frombuffer(f.read(), np.float32).reshape(h, w, 3)[::-1].reshape(-1, 3)
    ref = Ref().asset_render(name, root, w, h, spp, 4, 0, threads=THREADS)
    mr = ref.mean(axis=1)
    se = np.sqrt(2 * ref.var(axis=1, ddof=1) / spp) + 1e-7
    assert np.mean(np.abs(mean - mr) > 4 * se) < 0.01
    assert abs(mean.mean() - mr.mean()) < 0.02 * mr.mean()
