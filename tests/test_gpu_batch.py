"""Many views in one call (lrt_rast_render_batch): every view's image equals
the single-view render of that view bit for bit -- the first batch of a shape
(autotuned, eager), the second (captured into a CUDA graph) and later ones
(replayed with new cameras) -- and equals the oracle on a small case."""
from __future__ import annotations

import math

import numpy as np
import pytest
import torch

import lucabrtrender_b200 as L

import helpers as H

pytestmark = pytest.mark.gpu

SIZES = [(256, 256), (640, 480), (320, 180), (96, 160)]


def cameras(count: int, seed: int):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        radius = rng.uniform(3.0, 6.0)
        w, h = SIZES[rng.integers(len(SIZES))]
        out.append((L.square_pixel_camera(tuple(d * radius), (0.0, 0.0, 0.0), int(w), int(h)), int(w), int(h)))
    return out


def singles(rasterizer, views, instances, settings):
    out = []
    for cam, w, h in views:
        t = L.RenderTargets()
        st = L.RenderSettings(**{**settings.__dict__, "width": w, "height": h})
        rasterizer.render(cam, instances, st, t)
        out.append((t.colour.clone(), t.depth.clone()))
    return out


def test_batch_equals_single_view_renders_across_tuning_capture_and_replay(rasterizer):
    scene = H.synthetic_scene(50_000, 64, 64, seed=21)
    packed = scene.clouds[0][0]
    instances = [L.SplatInstance(L.to_device(packed))]
    settings = L.RenderSettings()
    replayed = []
    for rep, seed in enumerate((1, 2, 3, 4)):
        views = cameras(12, seed) if rep < 1 else [(c, w, h) for (c, w, h) in cameras(12, 1)]
        if rep >= 1:   # same shape, new cameras: move every eye a little
            views = [(L.square_pixel_camera(tuple(np.asarray(c.camera_to_world)[:3, 3] * (1.0 + 0.05 * rep)),
                                            (0.0, 0.0, 0.0), w, h), w, h) for (c, w, h) in views]
        targets, stats = rasterizer.render_batch(views, instances, settings)
        want = singles(rasterizer, views, instances, settings)
        for (colour, depth), t in zip(want, targets):
            assert torch.equal(t.colour, colour)
            assert torch.equal(t.depth, depth)
        assert stats.views == 12 and stats.pairs > 0
        replayed.append(stats.graph_replayed)
    assert replayed[0] == 0 and replayed[-1] == 1


def test_batch_matches_the_oracle_on_a_small_case(rasterizer):
    scene = H.reference_render_scenes()[0]
    instances = scene.gpu_instances()
    views = [(H.camera((1.5, 1.0, 6.0), focal=30.0), 250, 190), (H.camera((0.0, 3.0, 5.0), focal=40.0), 128, 96)]
    targets, _ = rasterizer.render_batch(views, instances, scene.settings)
    for (cam, w, h), t in zip(views, targets):
        ref = H.Scene("v", scene.clouds, cam, H.settings(w, h)).oracle_render(want_pairs=False)
        assert np.abs(t.colour.cpu().numpy() - ref["colour"]).max() <= 1e-5


def test_batch_with_two_instances_and_an_edit(rasterizer):
    cloud = H.random_cloud_packed(3000, 29)
    edit = L.SplatEdit(active=True, mode=L.EditMode.GRADE, size=(1.0, 1.0, 1.0), tint=(1.0, 0.5, 0.2))
    instances = [L.SplatInstance(L.to_device(cloud)),
                 L.SplatInstance(L.to_device(cloud), H.translation((0.5, 0.0, -1.5)) @ H.rotation_y(40.0), edit)]
    settings = L.RenderSettings(antialias=False, background=(0.1, 0.2, 0.3, 1.0))
    views = cameras(6, 9)
    targets, _ = rasterizer.render_batch(views, instances, settings)
    want = singles(rasterizer, views, instances, settings)
    for (colour, depth), t in zip(want, targets):
        assert torch.equal(t.colour, colour) and torch.equal(t.depth, depth)


@pytest.mark.parametrize("views", [1, 3])
def test_a_batch_of_one_or_an_odd_number_of_views(rasterizer, views):
    """Any number of (view, instance) parameter blocks: their per-view
    records after them stay aligned for the pointers they hold."""
    scene = H.synthetic_scene(20_000, 64, 64, seed=23)
    instances = [L.SplatInstance(L.to_device(scene.clouds[0][0]))]
    settings = L.RenderSettings()
    vs = cameras(views, 9)
    for _ in range(3):   # tuning, capture, replay
        targets, _ = rasterizer.render_batch(vs, instances, settings)
    for (colour, depth), t in zip(singles(rasterizer, vs, instances, settings), targets):
        assert torch.equal(t.colour, colour) and torch.equal(t.depth, depth)
