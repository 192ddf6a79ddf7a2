"""Parity metrics on the device (compareImages, compareHdr, countDifferent):
the same histograms and numbers as the CPU restatement, on image pairs that
differ by small noise, by large edits and not at all, and used the way the
reference uses them -- the GPU render against the brute force, read back as
three numbers instead of two images."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import lucabrtrender_b200 as L

import helpers as H
import oracle as ora

pytestmark = pytest.mark.gpu


def image_pair(seed: int, w: int = 333, h: int = 217):
    rng = np.random.default_rng(seed)
    a = rng.uniform(0, 1.4, (h, w, 4)).astype(np.float32)
    b = a.copy()
    b[..., :3] += rng.normal(0, 0.004, (h, w, 3)).astype(np.float32)
    b[40:60, 10:200] = rng.uniform(0, 1, (20, 190, 4))
    b[100, 100] = a[100, 100]
    return a, b


@pytest.mark.parametrize("seed", [1, 2])
def test_compare_images_equals_the_restatement(rasterizer, seed):
    a, b = image_pair(seed)
    diff, hist = rasterizer.compare_images(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda())
    want = ora.compare_images(a, b)
    assert np.array_equal(hist, want.histogram)
    assert (diff.pixels, diff.p99, diff.max, diff.over2) == (want.pixels, want.p99, want.max, want.over2)
    same, _ = rasterizer.compare_images(torch.from_numpy(a).cuda(), torch.from_numpy(a).cuda())
    assert same.max == 0 and same.over2 == 0 and same.pixels == a.shape[0] * a.shape[1]


def test_compare_hdr_equals_the_restatement(rasterizer):
    a, b = image_pair(3)
    got = rasterizer.compare_hdr(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda())
    hist, err = ora.compare_hdr(a, b)
    pixels = a.shape[0] * a.shape[1]
    assert got.pixels == pixels
    assert got.rel_mse == pytest.approx(float(np.float32(err)) / pixels, rel=0, abs=0)
    nz = np.nonzero(hist)[0]
    assert got.max_relative == pytest.approx(2.0 ** (nz[-1] / 8.0 - 16.0))
    running = np.cumsum(hist)
    p99 = int(np.argmax(running >= pixels - pixels // 100))
    assert got.p99_relative == pytest.approx(2.0 ** (p99 / 8.0 - 16.0))


def test_count_different(rasterizer):
    rng = np.random.default_rng(4)
    a = rng.integers(0, 2**32, 1_000_003, dtype=np.uint64).astype(np.uint32)
    b = a.copy()
    flip = rng.choice(a.size, 12345, replace=False)
    b[flip] ^= 1
    n = rasterizer.count_different(torch.from_numpy(a.view(np.int32)).cuda(), torch.from_numpy(b.view(np.int32)).cuda())
    assert n == 12345 == ora.count_different(a, b)


def test_the_render_against_the_brute_force_read_back_as_numbers(rasterizer):
    scene = H.reference_render_scenes()[0]
    targets = L.RenderTargets()
    instances = [L.SplatInstance(L.to_device(p), m) for p, m, _ in scene.clouds]
    rasterizer.render(scene.projection(), instances, scene.settings, targets)
    truth, _, over = scene.oracle_reference()
    diff, _ = rasterizer.compare_images(targets.colour, torch.from_numpy(truth).cuda())
    want = ora.compare_images(targets.colour.cpu().numpy(), truth)
    assert over == 0 and (diff.p99, diff.max) == (want.p99, want.max)
    assert diff.p99 <= 2 and diff.max <= 16
