"""Views across GPUs: one process per GPU, each holding the whole scene.

Rendering shards by view and needs no exchange: each rank renders its own
share of a view list (an orbit's frames, a batch's cameras). Training over
views has one real exchange per step: the ranks' parameter gradients are
summed before the optimizer step. Here that is one all-reduce over a single
flat bucket the backward writes every gradient into, so there is no gather
or scatter copy around it. torch.distributed is the plumbing: NCCL between
GPUs (over NVLink/NVSwitch), gloo on the CPU (the tests).

No reference counterpart: the reference renders on one device.
"""
from __future__ import annotations

from typing import Sequence

import torch
import torch.distributed as dist

# Floats of gradient per splat: means 3, log-scales 3, quaternions 4, opacity
# logit 1, SH 48.
GRAD_FLOATS_PER_SPLAT = 3 + 3 + 4 + 1 + 48


def views_for_rank(count: int, rank: int, world: int) -> range:
    """The views rank `rank` of `world` renders: a contiguous block, the first
    `count % world` ranks taking one more. Every view goes to exactly one rank."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    base, extra = divmod(count, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def max_over_ranks(value: float, device: torch.device | None = None) -> float:
    """The largest `value` over the ranks (the job's time is its slowest rank's)."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class GradientBucket:
    """One flat fp32 buffer holding every parameter gradient of a splat cloud.
    Passed to ``rasterize(..., grad_bucket=...)``, the backward writes the
    gradients straight into it; ``all_reduce`` then sums them over the ranks
    in place (one collective per step). The SH gradient comes first: the
    backward writes it with 16-byte stores, and the buffer's start is aligned."""

    ORDER = ("means", "log_scales", "quats", "opacity_logits", "sh")

    def __init__(self, count: int, device: torch.device):
        self.count = count
        self.flat = torch.empty(count * GRAD_FLOATS_PER_SPLAT, dtype=torch.float32, device=device)
        self.layout = {}   # name -> (first float, floats)
        at = 0
        for name, per in (("sh", 48), ("means", 3), ("log_scales", 3), ("quats", 4), ("opacity_logits", 1)):
            self.layout[name] = (at, per * count)
            at += per * count
        shapes = {"means": (count, 3), "log_scales": (count, 3), "quats": (count, 4), "opacity_logits": (count,),
                  "sh": (count, 16, 3)}
        self.views = {k: self.slice(k).view(shapes[k]) for k in self.ORDER}

    def slice(self, name: str) -> torch.Tensor:
        """A fresh flat view of one gradient's part of the buffer."""
        at, size = self.layout[name]
        return self.flat[at:at + size]

    def ordered(self) -> list[torch.Tensor]:
        return [self.views[k] for k in self.ORDER]

    def holds(self, grads: Sequence[torch.Tensor | None]) -> bool:
        """Whether these gradients are the bucket's own views (autograd kept them)."""
        return all(g is not None and g.data_ptr() == v.data_ptr() for g, v in zip(grads, self.ordered()))

    def all_reduce(self, params: Sequence[torch.Tensor], average: bool = False) -> None:
        """Sum (or average) the ranks' gradients of `params` (means,
        log-scales, quaternions, opacity logits, SH). Gradients autograd did
        not leave in the bucket are copied in first and the result copied
        back, so the sum is right either way. Each backward into the bucket
        rewrites it."""
        grads = [p.grad for p in params]
        inside = self.holds(grads)
        if not inside:
            for g, v in zip(grads, self.ordered()):
                v.copy_(g.reshape(v.shape) if g is not None else torch.zeros_like(v))
        if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
            dist.all_reduce(self.flat, op=dist.ReduceOp.SUM)
            if average:
                self.flat.div_(dist.get_world_size())
        if not inside:
            for p, v in zip(params, self.ordered()):
                if p.grad is None:
                    p.grad = v.clone().reshape(p.shape)
                else:
                    p.grad.copy_(v.reshape(p.grad.shape))
