"""One render split across ranks (lux_b200.distributed): sample shares and the film sum,
world size 2 over gloo on CPU with a stand-in renderer (per-sample values keyed like the
path tracer's, by pixel and sample), and on one GPU against lux_render."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _fake_render(req, film):
    """Sum over the request's samples of a value that depends only on (pixel, sample)."""
    import torch
    h, w = req.height, req.width
    pix = torch.arange(h * w, dtype=torch.float64).reshape(h, w, 1)
    acc = torch.zeros((h, w, 3), dtype=torch.float64)
    for s in range(req.sample_offset, req.sample_offset + req.spp):
        acc += torch.sin(pix * 0.37 + s * 1.3) ** 2 + torch.tensor([0.1, 0.2, 0.3])
    film.copy_(acc.to(film.dtype))


def _worker(rank, world, port, spp, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from lux_b200 import distributed as D
    from lux_b200 import scene as S
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        req = S.request(6, 5, spp, 3, 7, sample_offset=2)
        film = torch.zeros((5, 6, 3), dtype=torch.float32)
        sub = D.render_sharded(_fake_render, req, film)
        out.put((rank, sub.sample_offset, sub.spp, film.numpy().copy()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("spp", [7, 1])
def test_render_sharded_world_size_2_equals_one_render(spp):
    import socket

    import torch
    import torch.multiprocessing as mp
    from lux_b200 import distributed as D
    from lux_b200 import scene as S
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, spp, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    # The shares tile the request's samples.
    assert [(r[1], r[2]) for r in results] == [(2 + a, n) for a, n in
                                               (D.sample_range(spp, 0, 2), D.sample_range(spp, 1, 2))]
    assert sum(r[2] for r in results) == spp
    whole = torch.zeros((5, 6, 3), dtype=torch.float32)
    _fake_render(S.request(6, 5, spp, 3, 7, sample_offset=2), whole)
    np.testing.assert_allclose(results[0][3], whole.numpy(), rtol=1e-6)   # dst rank 0


def test_sample_ranges_tile_for_any_world():
    from lux_b200 import distributed as D
    for spp in (1, 3, 64, 257):
        for world in (1, 2, 3, 8, 300):
            shares = [D.sample_range(spp, r, world) for r in range(world)]
            assert shares[0][0] == 0 and sum(c for _, c in shares) == spp
            assert all(a + c == b for (a, c), (b, _) in zip(shares, shares[1:]))


@pytest.mark.gpu
def test_render_sharded_without_a_group_is_lux_render(ctx):
    import torch
    from lux_b200 import distributed as D
    from lux_b200 import scene as S
    sc = S.Scene(ctx, S.make_cornell_scene(24, 24))
    req = S.request(24, 24, 8, 4, 1)
    film = torch.zeros((24, 24, 3), dtype=torch.float32, device="cuda")
    D.render_sharded(lambda r, f: S.render(ctx, sc, r, f), req, film)
    torch.cuda.synchronize()
    assert np.array_equal(film.cpu().numpy(), S.render(ctx, sc, req))
    # Two shares rendered one after the other add up to the whole film.
    parts = []
    for rank in range(2):
        sub = D.shard_request(req, rank, 2)
        parts.append(S.render(ctx, sc, sub))
    np.testing.assert_allclose(parts[0] + parts[1], S.render(ctx, sc, req), rtol=1e-5, atol=1e-6)
