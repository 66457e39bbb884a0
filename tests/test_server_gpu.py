"""Batched / served rendering: equivalence with lux_render, mix-independence, admission
by memory budget, cancellation and refits (B200)."""
import time

import numpy as np
import pytest

import lux_b200
from lux_b200 import scene as S
from lux_b200 import server as SV

pytestmark = pytest.mark.gpu


def _zoo():
    from test_pathtracer_gpu import material_zoo
    return material_zoo(64, 64)[0]


@pytest.fixture(scope="module")
def scenes(ctx):
    cornell = S.Scene(ctx, S.make_cornell_scene(64, 64))
    zoo = S.Scene(ctx, _zoo())
    return [cornell, zoo]


def _close(a, b, rtol=2e-5):
    return np.all(np.abs(a - b) <= rtol * (1.0 + np.abs(b)))


REQUESTS = [(0, S.request(64, 64, 16, 4, 1)), (1, S.request(64, 64, 8, 6, 2)),
            (0, S.request(64, 64, 5, 9, 3, light_sampler=S.SAMPLER_UNIFORM)),
            (1, S.request(64, 64, 12, 3, 4, frame_index=2)),
            (0, S.request(64, 64, 3, 0, 5)), (1, S.request(64, 64, 7, 5, 6, sample_offset=11))]


def test_batched_requests_match_single_renders(ctx, scenes):
    want = [S.render(ctx, scenes[s], r) for s, r in REQUESTS]
    with SV.Server(scenes, pool_paths=1 << 16) as srv:
        ids = [srv.submit(s, r) for s, r in REQUESTS]
        srv.wait_all(timeout_s=120)
        for (rid, film), w in zip(ids, want):
            assert srv.poll(rid) == SV.DONE
            assert _close(film, w)
        st = srv.stats()
        assert st["completed"] == len(REQUESTS) and st["rays"] > 0 and st["shadow_rays"] > 0


def test_request_is_identical_alone_and_in_the_mix(scenes):
    s, r = REQUESTS[1]
    with SV.Server(scenes, pool_paths=1 << 15) as srv:
        rid, alone = srv.submit(s, r)
        srv.wait_all(timeout_s=120)
    with SV.Server(scenes, pool_paths=1 << 15) as srv:
        out = [srv.submit(ss, rr) for ss, rr in REQUESTS]
        srv.wait_all(timeout_s=120)
    mixed = out[1][1]
    assert np.array_equal(alone, mixed)


def test_budget_admission_queues_and_rejects(scenes):
    film_bytes = 64 * 64 * 3 * 12   # fixed-point film + host staging
    pool = 1 << 14
    pool_bytes = pool * (16 * 12 + 4 * 7 + 4 * 5 + 16 * 7 + 4 + 4)   # two pools
    budget = pool_bytes + 2 * film_bytes + 100       # two requests at a time
    with SV.Server(scenes, pool_paths=pool, memory_budget_bytes=budget) as srv:
        ids = [srv.submit(s, r)[0] for s, r in REQUESTS]
        states = [srv.poll(i) for i in ids]
        assert states.count(SV.RUNNING) <= 2
        srv.wait_all(timeout_s=120)
        assert all(srv.poll(i) == SV.DONE for i in ids)
        assert srv.stats()["bytes_in_use"] <= budget
        # A film that can never fit is refused at submission.
        with pytest.raises(lux_b200.LuxError) as e:
            srv.submit(0, S.request(256, 256, 1, 1))
        assert e.value.status == lux_b200.LUX_ERR_BUDGET


def test_cancel_queued_and_running(ctx, scenes):
    with SV.Server(scenes, pool_paths=1 << 14, max_requests=1) as srv:
        big, _ = srv.submit(1, S.request(64, 64, 512, 8, 7))
        queued, _ = srv.submit(0, S.request(64, 64, 4, 4, 8))
        keep, film = srv.submit(0, S.request(64, 64, 4, 4, 9))
        srv.cancel(queued)
        assert srv.poll(queued) == SV.CANCELLED
        time.sleep(0.05)
        srv.cancel(big)
        assert srv.wait(big, timeout_s=60) == SV.CANCELLED
        assert srv.wait(keep, timeout_s=60) == SV.DONE
        assert _close(film, S.render(ctx, scenes[0], S.request(64, 64, 4, 4, 9)))


def test_refit_between_frames(ctx):
    from lux_b200 import scenes as SC
    b = SC.heavy_render_scene(32, 32)
    sc = S.Scene(ctx, b)
    mesh = 1                       # the displaced icosphere
    base = b.meshes[mesh].vertices.copy()
    with SV.Server([sc], pool_paths=1 << 15) as srv:
        r0, f0 = srv.submit(0, S.request(32, 32, 4, 5, 1))
        srv.wait(r0, timeout_s=60)
        moved = base.copy()
        moved[:, 1] += 0.05 * np.sin(3.0 * moved[:, 0])
        srv.update_mesh(0, mesh, moved)
        r1, f1 = srv.submit(0, S.request(32, 32, 4, 5, 1))
        srv.wait(r1, timeout_s=60)
        assert srv.stats()["refits"] == 1
    assert not np.array_equal(f0, f1)
    # The refit scene renders like a scene built from the moved vertices.
    b2 = SC.heavy_render_scene(32, 32)
    b2.meshes[mesh].vertices = moved
    fresh = S.render(ctx, S.Scene(ctx, b2), S.request(32, 32, 4, 5, 1))
    rel = np.abs(f1 - fresh) / (1 + np.abs(fresh))
    assert np.mean(rel < 1e-4) > 0.99


def test_emissive_refit_updates_the_served_light_tables(ctx):
    """A served scene whose emissive mesh moves (and gains a light) renders like a scene
    created from the moved vertices: the staged scene view follows the new tables."""
    from test_pathtracer_gpu import emissive_mesh_scene
    b, mesh, v = emissive_mesh_scene()
    sc = S.Scene(ctx, b)
    moved = v.copy()
    moved[:, 1] += np.float32(0.04)
    moved[1] += np.float32(0.1)
    moved[2] += np.float32([0.0, 0.0, 0.1])
    req = S.request(32, 32, 8, 5, 2, light_sampler=S.SAMPLER_TREE)
    with SV.Server([sc], pool_paths=1 << 15) as srv:
        r0, _ = srv.submit(0, req)
        srv.wait(r0, timeout_s=60)
        srv.update_mesh(0, mesh, moved)
        r1, film = srv.submit(0, req)
        srv.wait(r1, timeout_s=60)
        assert srv.stats()["refits"] == 1
    fresh = S.render(ctx, S.Scene(ctx, emissive_mesh_scene(moved)[0]), req)
    assert _close(film, fresh)


def test_refits_faster_than_iterations_do_not_starve_requests(ctx):
    from lux_b200 import scenes as SC
    b = SC.heavy_render_scene(32, 32)
    sc = S.Scene(ctx, b)
    base = b.meshes[1].vertices.copy()
    with SV.Server([sc], pool_paths=1 << 15) as srv:
        ids = [srv.submit(0, S.request(32, 32, 16, 6, k))[0] for k in range(4)]
        pushed = 0
        for k in range(200):
            moved = base.copy()
            moved[:, 1] += 0.01 * np.sin(3.0 * moved[:, 0] + 0.1 * k)
            srv.update_mesh(0, 1, moved)
            pushed += 1
        srv.wait_all(timeout_s=120)
        assert all(srv.poll(i) == SV.DONE for i in ids)
        refits = srv.stats()["refits"]
        assert 1 <= refits <= pushed


def test_mixed_batch_over_the_four_resident_scenes_matches_single_renders(ctx):
    """A mix over the four resident scenes of the batched and served workloads (Cornell,
    the displaced icosphere with glass, the 2,097,152-triangle soup and the 256-instance
    grid), of uneven size, spp and depth: every request's film equals its lux_render
    film, and a request's film is the same alone as in the mix."""
    from lux_b200 import scenes as SC
    builders = SC.resident_scenes(96, 96)
    scenes = [S.Scene(ctx, b) for b in builders]
    mix = [(0, S.request(96, 96, 8, 4, 1)), (1, S.request(80, 80, 6, 8, 2)),
           (2, S.request(64, 64, 4, 6, 3)), (3, S.request(96, 96, 5, 12, 4)),
           (3, S.request(48, 48, 9, 5, 5, light_sampler=S.SAMPLER_TREE)),
           (2, S.request(72, 72, 3, 10, 6)), (1, S.request(40, 40, 16, 4, 7)),
           (0, S.request(56, 56, 2, 9, 8, sample_offset=5))]
    want = [S.render(ctx, scenes[s], r) for s, r in mix]
    with SV.Server(scenes, pool_paths=1 << 16) as srv:
        out = [srv.submit(s, r) for s, r in mix]
        srv.wait_all(timeout_s=300)
        assert all(srv.poll(rid) == SV.DONE for rid, _ in out)
    for (_, film), w in zip(out, want):
        assert _close(film, w)
    with SV.Server(scenes, pool_paths=1 << 16) as srv:
        rid, alone = srv.submit(*mix[3])
        srv.wait_all(timeout_s=300)
    assert np.array_equal(alone, out[3][1])
