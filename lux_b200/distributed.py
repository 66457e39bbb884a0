"""One render split across GPUs, one process per GPU.

A path's random numbers are keyed by (seed, pixel, sample) (sampler/sampler.h:165-176)
and the film is a sum over samples (film/film.h:19-21), so samples are independent work
units: rank r of N renders the request's sample range [spp * r / N, spp * (r + 1) / N)
(its sample_offset shifted by the range start), and the ranks' films are added with one
reduce (NCCL over NVLink between GPUs; gloo in the CPU tests).  That film sum is the only
exchange.  The result equals a single-GPU render of the whole request up to the order of
the float additions.
"""
from __future__ import annotations


def sample_range(spp: int, rank: int, world: int) -> tuple[int, int]:
    """(first sample, count) of rank's share of spp samples; the shares tile [0, spp)."""
    start = spp * rank // world
    return start, spp * (rank + 1) // world - start


def shard_request(req, rank: int, world: int):
    """The part of render request req (a lux_render_request) that rank renders."""
    start, count = sample_range(req.spp, rank, world)
    sub = type(req).from_buffer_copy(req)
    sub.spp = count
    sub.sample_offset = req.sample_offset + start
    return sub


def render_sharded(render, req, film, group=None, dst: int | None = 0):
    """Renders this rank's share of req into film (a tensor of width*height*3 sums) with
    render(sub_request, film), then sums the ranks' films: into dst's film (reduce), or
    into every rank's film when dst is None (all-reduce).  Without an initialised process
    group this is a plain render of req.  Returns this rank's sub-request."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        render(req, film)
        return req
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    sub = shard_request(req, rank, world)
    if sub.spp > 0:
        render(sub, film)
    else:
        film.zero_()
    if dst is None:
        dist.all_reduce(film, op=dist.ReduceOp.SUM, group=group)
    else:
        dist.reduce(film, dst, op=dist.ReduceOp.SUM, group=group)
    return sub
