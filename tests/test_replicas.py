"""Views across ranks, on the CPU: two gloo ranks spawned as processes.

Rendering shards by view with no exchange, so the multi-rank logic to check
is the host side: every view goes to exactly one rank, the job's time is the
slowest rank's, and the one real exchange of training over views -- the sum
of the ranks' parameter gradients -- is right whether or not autograd left
the gradients in the bucket the backward writes them to."""
from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from lucabrtrender_b200.replicas import GRAD_FLOATS_PER_SPLAT, GradientBucket, max_over_ranks, views_for_rank

WORLD = 2
SPLATS = 37   # not a multiple of 4: every part's offset still lines up as the kernels need


def test_views_are_split_into_contiguous_blocks_covering_each_once():
    for count in (0, 1, 5, 20, 64, 65):
        for world in (1, 2, 3, 8):
            got = [list(views_for_rank(count, r, world)) for r in range(world)]
            assert sum(got, []) == list(range(count))
            assert max(map(len, got)) - min(map(len, got)) <= 1
    with pytest.raises(ValueError):
        views_for_rank(4, 2, 2)


def test_the_bucket_lays_the_sh_gradient_first_and_every_part_end_to_end():
    b = GradientBucket(SPLATS, torch.device("cpu"))
    assert b.flat.numel() == SPLATS * GRAD_FLOATS_PER_SPLAT
    assert b.layout["sh"][0] == 0   # the 16-byte stores of the SH gradient start at the buffer's start
    spans = sorted(b.layout.values())
    assert spans[0][0] == 0 and all(a + n == c for (a, n), (c, _) in zip(spans, spans[1:]))
    assert [tuple(v.shape) for v in b.ordered()] == [(SPLATS, 3), (SPLATS, 3), (SPLATS, 4), (SPLATS,),
                                                     (SPLATS, 16, 3)]


def _params(rank: int) -> list[torch.Tensor]:
    shapes = [(SPLATS, 3), (SPLATS, 3), (SPLATS, 4), (SPLATS,), (SPLATS, 16, 3)]
    out = []
    for k, shape in enumerate(shapes):
        p = torch.zeros(shape, requires_grad=True)
        g = torch.arange(p.numel(), dtype=torch.float32).reshape(shape) * (k + 1) + 1000.0 * rank
        out.append((p, g))
    return out


def _rank(rank: int, port: int, out_dir: str) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=timedelta(seconds=60))
    try:
        result = {}
        # Gradients inside the bucket (what rasterize(..., grad_bucket=) leaves).
        bucket = GradientBucket(SPLATS, torch.device("cpu"))
        params = _params(rank)
        for (p, g), v in zip(params, bucket.ordered()):
            v.copy_(g)
            p.grad = v
        assert bucket.holds([p.grad for p, _ in params])
        bucket.all_reduce([p for p, _ in params])
        result["inside"] = [p.grad.clone() for p, _ in params]
        # Gradients autograd kept elsewhere: copied in, summed, copied back.
        params = _params(rank)
        for p, g in params:
            p.grad = g.clone()
        other = GradientBucket(SPLATS, torch.device("cpu"))
        assert not other.holds([p.grad for p, _ in params])
        other.all_reduce([p for p, _ in params], average=True)
        result["outside_average"] = [p.grad.clone() for p, _ in params]
        result["max"] = max_over_ranks(1.5 + rank)
        views = [None] * WORLD
        dist.all_gather_object(views, list(views_for_rank(20, rank, WORLD)))
        result["views"] = views
        torch.save(result, os.path.join(out_dir, f"rank{rank}.pt"))
    finally:
        dist.destroy_process_group()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_sum_their_gradients_and_agree_on_time_and_views(tmp_path):
    mp.spawn(_rank, args=(_free_port(), str(tmp_path)), nprocs=WORLD, join=True)
    results = [torch.load(tmp_path / f"rank{r}.pt") for r in range(WORLD)]
    want = [sum(g for _, g in (_params(r)[k] for r in range(WORLD))) for k in range(5)]
    for res in results:
        for got, w in zip(res["inside"], want):
            assert torch.equal(got, w)
        for got, w in zip(res["outside_average"], want):
            assert torch.equal(got, w / WORLD)
        assert res["max"] == 1.5 + (WORLD - 1)
        assert sum(res["views"], []) == list(range(20))
