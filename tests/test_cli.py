"""lux-render, the reference's render command line over liblux_gpu.so, and the film
encoders it writes images with (lux_film_encode)."""
import os
import subprocess

import numpy as np
import pytest

import lux_b200
from oracle.bindings import Ref

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
CLI = os.path.join(ROOT, "lux_b200", "lux-render")


@pytest.fixture(scope="module")
def cli():
    if not os.path.exists(CLI):
        from lux_b200 import build
        build.build()
    return CLI


def _run(cli, *args, cwd=None):
    return subprocess.run([cli, *args], capture_output=True, text=True, cwd=cwd, timeout=300)


def test_cli_reports_usage_and_rejects_like_the_reference(cli):
    assert _run(cli, "-help").returncode == 0
    r = _run(cli, "-scene", "teapot")
    assert r.returncode == 1 and "Unknown scene 'teapot'. Available scenes: cornell" in r.stderr
    r = _run(cli, "-scene", "bunny")
    assert r.returncode == 1 and "Scene setup failed" in r.stderr
    assert _run(cli, "-spp", "0").returncode == 1          # parse_positive_int
    assert _run(cli, "-depth", "-1").returncode == 1
    assert _run(cli, "-size", "8").returncode == 1          # missing operand
    assert _run(cli, "-light-sampler", "tree").returncode == 1  # parse_light_sampler_kind
    assert _run(cli, "-debug-aov", "ng,foo").returncode == 1      # parse_debug_aov_list
    assert _run(cli, "-debug-mode", "path").returncode == 1       # a probe needs its pixel
    assert _run(cli, "-debug-probe", "1", "2", "-debug-aov", "ng").returncode == 1
    assert _run(cli, "a.ppm", "b.ppm").returncode == 1           # one positional, alone
    for args in (["-debug-probe", "1", "2"], ["-debug-mesh", "winding"],
                 ["-debug-aov", "orientation,ng"]):
        r = _run(cli, *args)
        assert r.returncode == 1 and "not supported" in r.stderr


def _read_pfm(path):
    with open(path, "rb") as f:
        assert f.readline() == b"PF\n"
        w, h = (int(v) for v in f.readline().split())
        assert float(f.readline()) == -1.0
        data = np.frombuffer(f.read(), np.float32).reshape(h, w, 3)
    return data[::-1]  # PFM rows are bottom first


@pytest.mark.gpu
def test_cli_cornell_matches_reference_cpu_tracer(cli, tmp_path):
    """`lux-render -gpu` on the Cornell box (seed 0, as the reference CLI) against the
    reference's own CPU tracer at the same settings: per-pixel means within noise."""
    w = h = 48
    spp = 64
    out = tmp_path / "c.pfm"
    r = _run(cli, "-gpu", "-size", str(w), str(h), "-spp", str(spp), "-depth", "4",
             "-output", str(out), "-time")
    assert r.returncode == 0, r.stderr
    assert "Wrote" in r.stdout and "Timing breakdown" in r.stdout
    mean = _read_pfm(out).astype(np.float64)
    tot, tot2 = Ref().cornell_render(w, h, spp, 4, 0, threads=8)
    mr = (tot.astype(np.float64) / spp).reshape(h, w, 3)
    var = ((tot2.astype(np.float64) / spp).reshape(h, w, 3) - mr ** 2) * spp / (spp - 1)
    z = (mean - mr) / np.sqrt(2 * var / spp + 1e-12)
    assert np.mean(np.abs(z) > 4) < 0.005
    assert abs(mean.mean() - mr.mean()) < 0.01 * mr.mean()
    # Default output path: out/<scene>/<scene>.ppm, a binary P6 image.
    r = _run(cli, "-gpu", "-size", "16", "16", "-spp", "2", cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    data = (tmp_path / "out" / "cornell" / "cornell.ppm").read_bytes()
    assert data.startswith(b"P6\n16 16\n255\n") and len(data) == 13 + 16 * 16 * 3


@pytest.mark.gpu
@pytest.mark.parametrize("scene", ["direct-light", "point-light", "distant-light", "uniform-env",
                                   "image-env", "transparent-filter"])
@pytest.mark.parametrize("sampler", ["power", "bvh"])
def test_cli_renders_every_code_defined_scene(cli, tmp_path, scene, sampler):
    out = tmp_path / f"{scene}.pfm"
    r = _run(cli, "-gpu", "-scene", scene, "-size", "24", "24", "-spp", "8", "-output", str(out),
             "-light-sampler", sampler)
    assert r.returncode == 0, r.stderr
    img = _read_pfm(out)
    assert np.isfinite(img).all() and img.mean() > 0


@pytest.mark.gpu
def test_film_encoders_match_the_reference_writers(ctx, tmp_path):
    """lux_film_encode's PPM bytes, linear-debug bytes and PFM floats against the
    reference's write_ppm / write_debug_ppm_linear / write_pfm on the same film."""
    rng = np.random.default_rng(5)
    h, w, spp = 37, 53, 16
    film = (rng.gamma(0.7, 3.0, (h, w, 3)) * spp).astype(np.float32)
    film[0, 0] = [0.0, -1.0, np.float32(1e9)]
    lib = lux_b200.load_library()
    ref = Ref()
    ppm = np.zeros(h * w * 3, np.uint8)
    assert lib.lux_film_encode(ctx.handle, film.ctypes.data, w, h, spp, 0,
                               ppm.ctypes.data) == lux_b200.LUX_OK
    want = np.frombuffer(ref.write_image(film, spp, str(tmp_path / "a.ppm"), 0)[-h * w * 3:],
                         np.uint8)
    diff = np.abs(ppm.astype(int) - want.astype(int))
    assert diff.max() <= 1 and np.mean(diff > 0) < 1e-3   # powf last-bit rounding only
    lin = np.zeros(h * w * 3, np.uint8)
    assert lib.lux_film_encode(ctx.handle, film.ctypes.data, w, h, spp, 1,
                               lin.ctypes.data) == lux_b200.LUX_OK
    want = np.frombuffer(ref.write_image(film, spp, str(tmp_path / "b.ppm"), 1)[-h * w * 3:],
                         np.uint8)
    assert np.array_equal(lin, want)
    pfm = np.zeros(h * w * 3, np.float32)
    assert lib.lux_film_encode(ctx.handle, film.ctypes.data, w, h, spp, 2,
                               pfm.ctypes.data) == lux_b200.LUX_OK
    want = np.frombuffer(ref.write_image(film, spp, str(tmp_path / "c.pfm"), 2)[-h * w * 12:],
                         np.float32)
    assert np.array_equal(pfm, want)
    assert lib.lux_film_encode(ctx.handle, film.ctypes.data, w, h, spp, 7,
                               pfm.ctypes.data) == lux_b200.LUX_ERR_INVALID_ARGUMENT


@pytest.mark.gpu
def test_cli_writes_debug_images(cli, ctx, tmp_path):
    """`-debug-aov shadow,ng,ns` writes <prefix>_shadow / _ng / _ns next to the image (PFM
    for a .pfm prefix, linear PPM otherwise), as the reference's runner names them; the
    ng image is the per-sample mean lux_render_aovs gives for the same settings."""
    from lux_b200 import scene as S
    out = tmp_path / "c.pfm"
    r = _run(cli, "-gpu", "-size", "24", "24", "-spp", "4", "-debug-aov", "shadow,ng,ns",
             "-output", str(out))
    assert r.returncode == 0, r.stderr
    for name in ("shadow", "ng", "ns"):
        assert (tmp_path / f"c_{name}.pfm").exists() and f"c_{name}.pfm" in r.stdout
    ng = _read_pfm(tmp_path / "c_ng.pfm")
    sc = S.Scene(ctx, S.make_cornell_scene(24, 24))
    _, _, want, _ = S.render_aovs(ctx, sc, S.request(24, 24, 4, 4, 0), shadow=False, ns=False)
    assert np.allclose(ng, want / 4, rtol=1e-5, atol=1e-6)
    prefix = tmp_path / "dbg" / "x.ppm"
    r = _run(cli, "-gpu", "-size", "16", "16", "-spp", "2", "-debug-aov", "ng",
             "-debug-output", str(prefix), "-output", str(tmp_path / "b.ppm"))
    assert r.returncode == 0, r.stderr
    data = (tmp_path / "dbg" / "x_ng.ppm").read_bytes()
    assert data.startswith(b"P6\n16 16\n255\n") and len(data) == 13 + 16 * 16 * 3
