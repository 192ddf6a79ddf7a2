"""The opt-in Mip-Splatting 3D filter on the GPU (lrt_rast_filter3d and a
cloud's filter3d array), against the oracle's restatement of the same
method. Parity here is with that restatement only: the reference has no 3D
filter, so nothing of the reference's pins it."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import lucabrtrender_b200 as L

import bench_workload as W
import helpers as H
import oracle as ora

pytestmark = pytest.mark.gpu


def _views(count, seed, sizes=((320, 240), (640, 480), (256, 256))):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        w, h = sizes[k % len(sizes)]
        cam = L.square_pixel_camera(tuple(d * rng.uniform(2.5, 6.0)), (0.0, 0.0, 0.0), w, h, 60.0, 0.01)
        out.append((L.projection_for(cam, w, h), w, h))
    return out


def test_filter_variance_equals_the_oracle_bit_for_bit(rasterizer):
    packed = L.pack_splats(L.synthetic_records(200_000, 3), 15, 3)
    cloud = L.to_device(packed)
    views = _views(24, 1)
    got = rasterizer.filter3d(cloud, views, 0.2).cpu().numpy()
    want = ora.filter3d(H.host_cloud(packed), [(p.struct(), w, h) for p, w, h in views], 0.2)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert np.all(got > 0)


def test_a_filtered_frame_equals_the_oracle_and_an_unfiltered_one_is_unchanged(rasterizer):
    packed = L.pack_splats(L.synthetic_records(100_000, 4), 15, 3)
    cloud = L.to_device(packed)
    views = _views(16, 2)
    var = rasterizer.filter3d(cloud, views, 0.2)
    scene = H.synthetic_scene(100_000, 512, 512, seed=4)
    plain_targets = L.RenderTargets()
    rasterizer.render(scene.camera, [L.SplatInstance(cloud)], scene.settings, plain_targets)
    filtered = L.GpuSplats(cloud.positions, cloud.shape, cloud.sh, cloud.rest_per_colour, var)
    targets = L.RenderTargets()
    stats = rasterizer.render(scene.camera, [L.SplatInstance(filtered)], scene.settings, targets)
    dbg = rasterizer.debug_arrays()
    host = H.host_cloud(packed)
    host.filter3d = var.cpu().numpy()
    ref = ora.render(scene.projection().struct(), [(host, np.eye(4), None)], scene.settings.struct(), 0)
    assert stats.pairs == ref["pairs"]
    assert np.array_equal(dbg["proj"].cpu().numpy().view(np.uint32), ref["proj"].view(np.uint32))
    tiles, _, slots = H.pair_words_to_tile_slot(dbg["pairs"].cpu().numpy().view(np.uint64), dbg["slot_bits"], dbg["depth_bits"])
    assert np.array_equal(tiles, ref["pair_tiles"]) and np.array_equal(slots, ref["pair_slots"])
    assert np.abs(targets.colour.cpu().numpy() - ref["colour"]).max() <= 1e-5
    # the filter changed the frame; the same cloud without it renders as before
    assert not torch.equal(targets.colour, plain_targets.colour)
    again = L.RenderTargets()
    rasterizer.render(scene.camera, [L.SplatInstance(cloud)], scene.settings, again)
    assert torch.equal(again.colour, plain_targets.colour)


def test_a_batch_with_the_filter_equals_single_filtered_renders(rasterizer):
    packed = L.pack_splats(L.synthetic_records(50_000, 5), 15, 3)
    cloud = L.to_device(packed)
    views = _views(6, 3)
    filtered = L.GpuSplats(cloud.positions, cloud.shape, cloud.sh, cloud.rest_per_colour,
                           rasterizer.filter3d(cloud, views, 0.2))
    inst = [L.SplatInstance(filtered)]
    batched = [L.RenderTargets(w, h) for _, w, h in views]
    for _ in range(3):   # tune, capture, replay
        rasterizer.render_batch(views, inst, L.RenderSettings(), batched)
    for (p, w, h), b in zip(views, batched):
        t = L.RenderTargets()
        rasterizer.render(p, inst, L.RenderSettings(width=w, height=h), t)
        assert torch.equal(t.colour, b.colour) and torch.equal(t.depth, b.depth)
