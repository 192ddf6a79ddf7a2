"""Frames returned as soon as they are enqueued (lrt_rast_render_async, read
back by lrt_rast_settle): every image equals the waiting render of the same
view bit for bit, frames on other streams are ordered after them, and an
enqueued frame that runs out of pair buffer is reported by settle, after which
the frame drawn again is exact."""
from __future__ import annotations

import math

import pytest
import torch

import lucabrtrender_b200 as L
from lucabrtrender_b200 import _abi

import helpers as H

pytestmark = pytest.mark.gpu


def orbit(k: int, w: int, h: int, radius: float = 4.0):
    th = 2.0 * math.pi * k / 12
    return L.square_pixel_camera((radius * math.sin(th), 0.3, radius * math.cos(th)), (0.0, 0.0, 0.0), w, h)


def test_enqueued_frames_equal_waiting_frames():
    scene = H.synthetic_scene(60_000, 64, 64, seed=31)
    instances = [L.SplatInstance(L.to_device(scene.clouds[0][0]))]
    settings = L.RenderSettings(width=320, height=240)
    raster = L.TileRasterizer.create(0)
    try:
        want = []
        for k in range(8):
            t = L.RenderTargets()
            raster.render(orbit(k, 320, 240), instances, settings, t)
            want.append((t.colour.clone(), t.depth.clone()))
        got = [L.RenderTargets(320, 240) for _ in range(8)]
        for k in range(8):
            raster.render_async(orbit(k, 320, 240), instances, settings, got[k])
        stats = raster.settle()
        assert stats.splats == 60_000 and stats.pairs > 0
        for (colour, depth), t in zip(want, got):
            assert torch.equal(t.colour, colour)
            assert torch.equal(t.depth, depth)
    finally:
        raster.close()


def test_a_frame_on_another_stream_waits_for_the_enqueued_ones():
    scene = H.synthetic_scene(60_000, 64, 64, seed=32)
    instances = [L.SplatInstance(L.to_device(scene.clouds[0][0]))]
    settings = L.RenderSettings(width=320, height=240)
    raster = L.TileRasterizer.create(0)
    try:
        want = L.RenderTargets()
        raster.render(orbit(5, 320, 240), instances, settings, want)
        want = (want.colour.clone(), want.depth.clone())
        first = L.RenderTargets(320, 240)
        raster.render(orbit(0, 320, 240), instances, settings, first)   # sizes the shape
        side = torch.cuda.Stream()
        for k in range(4):
            raster.render_async(orbit(k, 320, 240), instances, settings, first)
        other = L.RenderTargets(320, 240)
        raster.render(orbit(5, 320, 240), instances, settings, other, side)
        torch.cuda.synchronize()
        raster.settle()
        assert torch.equal(other.colour, want[0]) and torch.equal(other.depth, want[1])
    finally:
        raster.close()


def test_an_enqueued_frame_that_overflows_is_reported_and_redrawn_exactly():
    # 20k splats: the first frame's pair buffer holds 80k pairs; the far view
    # emits about 45k (so frames of this shape are enqueued), the near one 107k.
    scene = H.synthetic_scene(20_000, 64, 64, seed=33, log_scale_mean=-3.0)
    instances = [L.SplatInstance(L.to_device(scene.clouds[0][0]))]
    settings = L.RenderSettings(width=256, height=256)
    far, near = orbit(0, 256, 256, radius=9.0), orbit(0, 256, 256, radius=1.6)
    raster = L.TileRasterizer.create(0)
    reference = L.TileRasterizer.create(0)
    try:
        t = L.RenderTargets(256, 256)
        first = raster.render(far, instances, settings, t)   # sizes the pair buffer
        raster.render_async(far, instances, settings, t)
        assert raster.settle().pairs == first.pairs
        raster.render_async(near, instances, settings, t)
        with pytest.raises(L.LrtError) as info:
            raster.settle()
        assert info.value.code == _abi.OVERFLOW
        raster.render(near, instances, settings, t)
        want = L.RenderTargets(256, 256)
        reference.render(near, instances, settings, want)
        assert torch.equal(t.colour, want.colour) and torch.equal(t.depth, want.depth)
    finally:
        raster.close()
        reference.close()


def test_a_shape_whose_pairs_crowd_the_buffer_grows_it_and_stays_exact():
    # 20k splats: the first frame's pair buffer holds 80k pairs. A view that
    # emits between 64k and 80k fits it, but leaves less than a quarter free,
    # so the next enqueued frame of that view grows the buffer (and waits);
    # every image stays equal to a fresh handle's.
    scene = H.synthetic_scene(20_000, 64, 64, seed=33, log_scale_mean=-3.0)
    instances = [L.SplatInstance(L.to_device(scene.clouds[0][0]))]
    settings = L.RenderSettings(width=256, height=256)
    probe = L.TileRasterizer.create(0)
    try:
        view = None
        t = L.RenderTargets(256, 256)
        for k in range(60):
            radius = 9.0 * (1.6 / 9.0) ** (k / 59)
            pairs = probe.render(orbit(0, 256, 256, radius=radius), instances, settings, t).pairs
            if 64_000 < pairs <= 80_000:
                view = orbit(0, 256, 256, radius=radius)
                break
    finally:
        probe.close()
    assert view is not None, "no view of this scene emits between 64k and 80k pairs"
    raster = L.TileRasterizer.create(0)
    reference = L.TileRasterizer.create(0)
    try:
        want = L.RenderTargets(256, 256)
        reference.render(view, instances, settings, want)
        first = L.RenderTargets(256, 256)
        raster.render(view, instances, settings, first)   # sizes the shape: 80k pairs of buffer
        got = [L.RenderTargets(256, 256) for _ in range(4)]
        for g in got:
            raster.render_async(view, instances, settings, g)
        raster.settle()
        for g in [first] + got:
            assert torch.equal(g.colour, want.colour) and torch.equal(g.depth, want.depth)
    finally:
        raster.close()
        reference.close()


def test_a_frame_side_above_the_limit_is_unsupported():
    # The projection packs tile rectangles into 16-bit fields: a frame side
    # holds at most 2^15 tiles of 16 pixels.
    scene = H.synthetic_scene(1000, 64, 64, seed=34)
    instances = [L.SplatInstance(L.to_device(scene.clouds[0][0]))]
    raster = L.TileRasterizer.create(0)
    try:
        wide = (1 << 19) + 1
        settings = L.RenderSettings(width=wide, height=1)
        with pytest.raises(L.LrtError) as info:
            raster.render(orbit(0, wide, 1), instances, settings, L.RenderTargets(wide, 1))
        assert info.value.code == _abi.UNSUPPORTED
        # The handle still renders a frame of an ordinary size.
        t = L.RenderTargets(64, 64)
        assert raster.render(orbit(0, 64, 64), instances, L.RenderSettings(width=64, height=64), t).splats == 1000
    finally:
        raster.close()


def test_many_enqueued_frames_back_to_back_stay_exact():
    # Frames enqueued back to back run their kernels chained (each waits for
    # the one before it as its first step); 48 of them over two views, each
    # image copied out on another stream as the next frame renders, must
    # equal the waiting renders bit for bit.
    scene = H.synthetic_scene(80_000, 64, 64, seed=35)
    instances = [L.SplatInstance(L.to_device(scene.clouds[0][0]))]
    settings = L.RenderSettings(width=400, height=300)
    views = [orbit(1, 400, 300), orbit(5, 400, 300)]
    raster = L.TileRasterizer.create(0)
    try:
        want = []
        for v in views:
            t = L.RenderTargets(400, 300)
            raster.render(v, instances, settings, t)
            want.append((t.colour.clone(), t.depth.clone()))
        targets = [L.RenderTargets(400, 300) for _ in range(2)]
        copies = [[torch.empty_like(want[0][0]), torch.empty_like(want[0][1])] for _ in range(48)]
        stream = torch.cuda.current_stream()
        side = torch.cuda.Stream()
        for k in range(48):
            t = targets[k % 2]
            raster.render_async(views[k % 2], instances, settings, t, stream)
            done = torch.cuda.Event()
            done.record(stream)
            side.wait_event(done)
            with torch.cuda.stream(side):
                copies[k][0].copy_(t.colour)
                copies[k][1].copy_(t.depth)
            stream.wait_stream(side)   # the next frame into these targets waits for the copy
        raster.settle()
        torch.cuda.synchronize()
        for k in range(48):
            assert torch.equal(copies[k][0], want[k % 2][0]) and torch.equal(copies[k][1], want[k % 2][1]), k
    finally:
        raster.close()
