"""The stand-in for the reference's GPU path (baseline/standin: the
reference's stage sequence and launch shapes in CUDA, used only as the
comparison figure of bench.py) draws the same image as the product, bit for
bit: the two differ in schedule, not in arithmetic."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest
import torch

import lucabrtrender_b200 as L

import helpers as H

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "baseline" / "standin"))
import standin as S  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,w,h", [(100_000, 512, 512), (30_000, 640, 480)])
def test_the_stand_in_draws_the_product_image(rasterizer, n, w, h):
    scene = H.synthetic_scene(n, w, h, seed=n)
    packed = scene.clouds[0][0]
    cloud = L.to_device(packed)
    ours = L.RenderTargets()
    stats = rasterizer.render(scene.camera, [L.SplatInstance(cloud)], scene.settings, ours)
    theirs = L.RenderTargets(w, h)
    s = S.Standin(0)
    try:
        stages = s.render(scene.projection().struct(), cloud.struct(), scene.settings.struct(), theirs.struct())
    finally:
        s.close()
    assert stats.pairs > 0 and all(v >= 0.0 for v in stages.values())
    assert torch.equal(ours.colour, theirs.colour)
    assert torch.equal(ours.depth, theirs.depth)
