"""Points as discs and the under layer on the GPU (lrt_rast_render_composite):
bit for bit against the oracle's restatement of points_project.slang and
splatBlendComposite -- records, keys, pairs, ranges and images -- and against
the brute force with the reference's thresholds
(tests/render/test_points.cpp:75-99, 153-200)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import lucabrtrender_b200 as L
from lucabrtrender_b200 import _abi

import helpers as H
import oracle as ora

pytestmark = pytest.mark.gpu


def proj_of(eye, w, h):
    return L.projection_for(L.Camera.looking_at(eye, (0.0, 0.0, 0.0)), w, h)


def gpu_points(raw, kind=2):
    packed = L.pack_points(raw, kind)
    return packed, L.points_to_device(packed)


def host_points(packed):
    return ora.HostPoints(packed.positions, packed.colours)


def check_frame(rasterizer, out, ref, targets):
    dbg = rasterizer.debug_arrays()
    assert np.array_equal(dbg["proj"].cpu().numpy().view(np.uint32), ref["proj"].view(np.uint32))
    assert np.array_equal(dbg["touched"].cpu().numpy().view(np.uint32), ref["touched"])
    assert np.array_equal(dbg["depth_keys"].cpu().numpy().view(np.uint32), ref["depth_keys"])
    assert np.array_equal(dbg["ranges"].cpu().numpy().view(np.uint32), ref["ranges"])
    tiles, slots = H.pair_words_to_tile_slot(dbg["pairs"].cpu().numpy().view(np.uint64), dbg["slot_bits"], dbg["depth_bits"])[::2]
    assert np.array_equal(tiles, ref["pair_tiles"]) and np.array_equal(slots, ref["pair_slots"])
    assert np.array_equal(targets.colour.cpu().numpy().view(np.uint32), ref["colour"].view(np.uint32))
    assert np.array_equal(targets.depth.cpu().numpy().view(np.uint32), ref["depth"].view(np.uint32))
    assert out.visible == ref["visible"] and out.pairs == ref["pairs"]


@pytest.mark.parametrize("mode,size", [(0, 0.06), (1, 5.0)], ids=["world", "pixels"])
def test_discs_equal_the_oracle_and_match_the_brute_force(rasterizer, mode, size):
    packed, dev = gpu_points(ora.random_points(4000, 3))
    settings = H.settings(230, 170, linearise=False)
    pr = proj_of((1.0, 2.0, 6.0), 230, 170)
    style = L.PointStyle(size_mode=mode, size=size)
    targets = L.RenderTargets()
    out = rasterizer.render(pr, [], settings, targets, points=[L.PointInstance(dev, np.eye(4), style)])
    hp = [(host_points(packed), np.eye(4), H.point_style(mode, size))]
    ref = ora.render(pr.struct(), [], settings.struct(), points=hp)
    check_frame(rasterizer, out, ref, targets)
    truth, _, over = ora.reference_render(pr.struct(), [], settings.struct(), points=hp)
    assert over == 0
    assert ora.compare_images(targets.colour.cpu().numpy(), truth).p99 <= 2


def test_splats_and_discs_in_one_sort_equal_the_oracle(rasterizer):
    scene = H.synthetic_scene(30_000, 200, 150, seed=41, log_scale_mean=-3.5)
    packed, dev = gpu_points(ora.random_points(6000, 4))
    pr = scene.projection()
    m = H.translation((0.2, -0.1, 0.3)) @ H.rotation_y(20)
    style = L.PointStyle(size_mode=0, size=0.04)
    targets = L.RenderTargets()
    out = rasterizer.render(pr, [L.SplatInstance(L.to_device(scene.clouds[0][0]))], scene.settings, targets,
                            points=[L.PointInstance(dev, m, style)])
    ref = ora.render(pr.struct(), scene.oracle_instances(), scene.settings.struct(),
                     points=[(host_points(packed), m, H.point_style(0, 0.04))])
    check_frame(rasterizer, out, ref, targets)


def test_constant_colour_discs(rasterizer):
    packed, dev = gpu_points(ora.random_points(3000, 8))
    settings = H.settings(160, 120, background=(0.1, 0.2, 0.3, 1.0))
    pr = proj_of((0.0, 1.0, 6.0), 160, 120)
    style = L.PointStyle(size_mode=1, size=3.0, constant_colour=True, colour=(0.9, 0.1, 0.4))
    targets = L.RenderTargets()
    out = rasterizer.render(pr, [], settings, targets, points=[L.PointInstance(dev, np.eye(4), style)])
    ref = ora.render(pr.struct(), [], settings.struct(),
                     points=[(host_points(packed), np.eye(4), H.point_style(1, 3.0, True, (0.9, 0.1, 0.4)))])
    check_frame(rasterizer, out, ref, targets)


@pytest.mark.parametrize("depth_mode", [0, 1])
def test_splats_over_an_under_layer_equal_the_oracle_and_one_mixed_sort(rasterizer, depth_mode):
    packed, dev = gpu_points(ora.random_points(8000, 5))
    fog = L.pack_splats(H.fog_records(), 3, 3)
    settings = H.settings(256, 180, depth=depth_mode)
    pr = proj_of((0.5, 0.5, 7.0), 256, 180)
    style = L.PointStyle(size_mode=0, size=0.05)
    layer = L.RenderTargets()
    rasterizer.render(pr, [], settings, layer, points=[L.PointInstance(dev, np.eye(4), style)])
    layer_host = (layer.colour.cpu().numpy(), layer.depth.cpu().numpy())
    composited = L.RenderTargets()
    fog_dev = [L.SplatInstance(L.to_device(fog))]
    out = rasterizer.render(pr, fog_dev, settings, composited, under=layer)
    ref = ora.render(pr.struct(), [(H.host_cloud(fog), np.eye(4), None)], settings.struct(), under=layer_host)
    check_frame(rasterizer, out, ref, composited)
    mixed = L.RenderTargets()
    rasterizer.render(pr, fog_dev, settings, mixed, points=[L.PointInstance(dev, np.eye(4), style)])
    assert ora.compare_images(composited.colour.cpu().numpy(), mixed.colour.cpu().numpy()).p99 <= 2


def test_an_under_layer_of_the_wrong_size_is_refused(rasterizer):
    layer = L.RenderTargets(32, 32)
    with pytest.raises(L.LrtError) as info:
        rasterizer.render(proj_of((0, 0, 4), 64, 64), [], H.settings(64, 64), L.RenderTargets(), under=layer)
    assert info.value.code == _abi.INVALID_ARGUMENT
