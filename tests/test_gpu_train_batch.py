"""The batched training step (lrt_rast_train_batch) against single-view steps.

For every view the batch must draw the single-view training forward's image
and depth bit for bit and take the same L1 loss; its gradients must be the
single-view gradients summed in view order in float32 (the order the batch
accumulates them), equal up to the sign of zero. Runs with views of mixed
sizes, with chunkings fixed by the test hook (several chunks, and chunk
boundaries inside the views' list), and over repeated steps with new cameras,
which replay the captured step.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import lucabrtrender_b200 as L
from lucabrtrender_b200 import _abi

import train_fixtures as TF

pytestmark = pytest.mark.gpu

NAMES = ("means", "log_scales", "quats", "logits", "sh")
GRAD_KEYS = {"means": "means", "log_scales": "log_scales", "quats": "quats", "logits": "opacity_logits", "sh": "sh"}


@pytest.fixture(scope="module")
def raster():
    r = L.TileRasterizer.create(0)
    yield r
    r.close()


def views_for(count: int, seed: int):
    rng = np.random.default_rng(seed)
    sizes = [(200, 150), (96, 96), (320, 180), (64, 64), (200, 200), (128, 72)]
    out = []
    for k in range(count):
        w, h = sizes[k % len(sizes)]
        d = rng.normal(size=3)
        eye = tuple(float(v) for v in d / np.linalg.norm(d) * rng.uniform(3.0, 6.0))
        cam = L.square_pixel_camera(eye, (0.0, 0.0, 0.0), w, h, 60.0, 0.01)
        target = torch.from_numpy(rng.uniform(0, 1, (h, w, 3)).astype(np.float32)).cuda()
        out.append((cam, target))
    return out


def params_of(n: int, seed: int):
    return {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in TF.make_params(n, seed).items()}


def single_view_steps(raster, p, views):
    """Each view through rasterize + l1_loss + backward, the gradients summed in view order."""
    images, losses, acc = [], [], None
    for cam, target in views:
        t = {k: v.clone().requires_grad_(True) for k, v in p.items()}
        h, w = target.shape[:2]
        colour, depth = L.rasterize(t["means"], t["log_scales"], t["quats"], t["logits"], t["sh"], cam,
                                    L.RenderSettings(width=w, height=h), raster)
        loss = L.l1_loss(colour, target, raster)
        loss.backward()
        images.append((colour.detach().cpu().numpy(), depth.cpu().numpy()))
        losses.append(float(loss.detach()))
        g = {k: t[k].grad.detach().cpu().numpy() for k in NAMES}
        acc = g if acc is None else {k: (acc[k] + g[k]).astype(np.float32) for k in NAMES}
    return images, losses, acc


@pytest.mark.parametrize("count,n,seed", [(5, 20000, 31), (19, 8000, 32)], ids=["one-chunk", "two-chunks"])
def test_the_batch_equals_single_view_steps(raster, count, n, seed):
    p = params_of(n, seed)
    views = views_for(count, seed)
    colours, depths, losses, grads, stats = L.train_batch(p["means"], p["log_scales"], p["quats"], p["logits"], p["sh"],
                                                          views, L.RenderSettings(), raster)
    assert stats.views == count
    assert stats.chunks == (count + stats.views_per_chunk - 1) // stats.views_per_chunk
    images, want_losses, want = single_view_steps(raster, p, views)
    for k, ((colour, depth), c, d) in enumerate(zip(images, colours, depths)):
        assert np.array_equal(c.cpu().numpy().view(np.uint32), colour.view(np.uint32)), k
        assert np.array_equal(d.cpu().numpy().view(np.uint32), depth.view(np.uint32)), k
    assert losses.cpu().numpy().tolist() == pytest.approx(want_losses, rel=0, abs=0)
    for name in NAMES:
        got = grads[GRAD_KEYS[name]].cpu().numpy()
        assert not np.isnan(got).any(), name
        assert np.array_equal(got, want[name]), name   # equal values (+0 and -0 alike)


def test_a_bucket_and_an_fp16_working_copy_give_the_same_batch(raster):
    from lucabrtrender_b200.replicas import GradientBucket
    n = 12001
    p = params_of(n, 33)
    views = views_for(4, 33)
    _, _, la, ga, _ = L.train_batch(p["means"], p["log_scales"], p["quats"], p["logits"], p["sh"], views,
                                    L.RenderSettings(), raster)
    bucket = GradientBucket(n, torch.device("cuda"))
    sh16 = p["sh"].reshape(n, 48).half().contiguous()
    _, _, lb, gb, _ = L.train_batch(p["means"], p["log_scales"], p["quats"], p["logits"], p["sh"], views,
                                    L.RenderSettings(), raster, sh_storage=sh16, grad_bucket=bucket)
    assert torch.equal(la, lb)
    for k in ga:
        assert gb[k].data_ptr() == bucket.views[k].data_ptr()
        assert torch.equal(ga[k].view(torch.int32), gb[k].view(torch.int32)), k


def _check_equal(raster, p, views, out):
    colours, depths, losses, grads, _ = out
    images, want_losses, want = single_view_steps(raster, p, views)
    for k, ((colour, depth), c, d) in enumerate(zip(images, colours, depths)):
        assert np.array_equal(c.cpu().numpy().view(np.uint32), colour.view(np.uint32)), k
        assert np.array_equal(d.cpu().numpy().view(np.uint32), depth.view(np.uint32)), k
    assert losses.cpu().numpy().tolist() == pytest.approx(want_losses, rel=0, abs=0)
    for name in NAMES:
        assert np.array_equal(grads[GRAD_KEYS[name]].cpu().numpy(), want[name]), name


@pytest.mark.parametrize("chunk,blocks", [(4, 2), (7, 8), (16, 4)])
def test_fixed_chunkings_equal_single_view_steps(chunk, blocks):
    r = L.TileRasterizer.create(0)
    lib = _abi.load()
    try:
        assert lib.lrt_rast_debug_train_chunking(r._handle, chunk, blocks) == _abi.OK
        p = params_of(9000, 40 + chunk)
        views = views_for(19, 40 + chunk)
        out = L.train_batch(p["means"], p["log_scales"], p["quats"], p["logits"], p["sh"], views,
                            L.RenderSettings(), r)
        stats = out[4]
        assert stats.views_per_chunk == chunk and stats.blend_blocks_per_sm == blocks
        assert stats.chunks == (19 + chunk - 1) // chunk
        _check_equal(r, p, views, out)
    finally:
        r.close()


def test_repeated_steps_replay_the_captured_step_with_new_cameras():
    r = L.TileRasterizer.create(0)
    try:
        p = params_of(15000, 50)
        outs = []
        for step in range(4):   # tune, capture, replay, replay
            views = views_for(6, 60 + step)
            # the same view sizes every step: one shape
            out = L.train_batch(p["means"], p["log_scales"], p["quats"], p["logits"], p["sh"], views,
                                L.RenderSettings(), r)
            outs.append((views, out))
        replays = [o[4].graph_replayed for _, o in outs]
        assert replays[0] == 0 and replays[-1] == 1, replays
        for views, out in outs[2:]:
            _check_equal(r, p, views, out)
    finally:
        r.close()
