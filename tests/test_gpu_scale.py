"""The sort-heavy configuration (6M splats, 3840x2160, means N(0, 2),
log-scales N(-3.5, 0.7)) on the GPU, through properties that hold at any
size: the pair words are in (tile, depth key, slot) order, every tile's range
holds exactly its pairs, the ranges partition the pairs, the touched counts
sum to the pair count, frames are deterministic, and the batched path draws
the same image. (The CPU oracle checks the same invariants bit for bit on the
smaller scenes; at this size it would take minutes a frame.)"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import lucabrtrender_b200 as L

pytestmark = pytest.mark.gpu


def test_the_sort_heavy_frame_keeps_every_invariant(rasterizer):
    raw = L.synthetic_records(6_000_000, 7, mean_sigma=2.0, log_scale_mean=-3.5, log_scale_sigma=0.7)
    cloud = L.to_device(L.pack_splats(raw, 15, 3))
    settings = L.RenderSettings(width=3840, height=2160)
    cam = L.square_pixel_camera((0.0, 0.0, 4.0), (0.0, 0.0, 0.0), 3840, 2160)
    a = L.RenderTargets()
    stats = rasterizer.render(cam, [L.SplatInstance(cloud)], settings, a)
    dbg = rasterizer.debug_arrays()
    words = dbg["pairs"].cpu().numpy().view(np.uint64)
    sb, db = dbg["slot_bits"], dbg["depth_bits"]
    assert stats.pairs == words.size > 50_000_000
    assert int(dbg["touched"].cpu().numpy().astype(np.int64).sum()) == words.size
    slots = words & np.uint64((1 << sb) - 1)
    tiles = (words >> np.uint64(db + sb)).astype(np.int64)
    # (tile, 24-bit depth key, slot) ascending
    depth = dbg["depth_keys"].cpu().numpy().view(np.uint32)[slots.astype(np.int64)].astype(np.uint64)
    key = (tiles.astype(np.uint64) << np.uint64(24)) | depth
    assert np.all(key[1:] >= key[:-1])
    ties = key[1:] == key[:-1]
    assert np.all(slots[1:][ties] > slots[:-1][ties])
    ranges = dbg["ranges"].cpu().numpy().astype(np.int64)
    lengths = ranges[:, 1] - ranges[:, 0]
    assert lengths.sum() == words.size and np.all(lengths >= 0)
    counts = np.bincount(tiles, minlength=ranges.shape[0])
    assert np.array_equal(counts, lengths)
    nz = np.nonzero(lengths)[0]
    assert np.array_equal(tiles[ranges[nz, 0]], nz) and np.array_equal(tiles[ranges[nz, 1] - 1], nz)
    b = L.RenderTargets()
    rasterizer.render(cam, [L.SplatInstance(cloud)], settings, b)
    assert torch.equal(a.colour, b.colour) and torch.equal(a.depth, b.depth)
    batched, _ = rasterizer.render_batch([(cam, 3840, 2160)], [L.SplatInstance(cloud)], settings)
    assert torch.equal(batched[0].colour, a.colour) and torch.equal(batched[0].depth, a.depth)
