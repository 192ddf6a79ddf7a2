"""Parity at the sizes the benchmark measures, through the C-ABI:

- the headline workload (1M splats, 1920x1080, frames 0 and 3 of the
  20-frame orbit at radius 4): every projection record, rect, touched count
  and depth key, every sorted pair and every tile range equal to the
  oracle's bit for bit; colour and depth within 1e-5 max-abs and 1e-6 at the
  99th percentile;
- the sort-heavy workload (6M splats, means N(0,2), log-scales N(-3.5,0.7),
  3840x2160, about 256M pairs): every record, key, pair and range bit for
  bit, and the images of 64 seeded tiles (the oracle blends only those);
- the differentiable workload (the same 1M splats as raw parameters, frame
  0 at 1920x1080): gradients of an L1 loss over the 64x64 crop at the
  frame's centre against the FP64 per-pixel oracle and FP64 central
  differences (h = 1e-4) on 256 parameters, within 1e-4 relative.

The inputs are built by the oracle's copy of the benchmark workload
(oracle/bench_workload.py, held equal to the package's by
tests/test_bench_workload.py)."""
from __future__ import annotations

import math

import numpy as np
import pytest
import torch

import lucabrtrender_b200 as L

import bench_workload as W
import grad_oracle as G
import helpers as H
import oracle as ora

pytestmark = pytest.mark.gpu

IMAGE_MAX = 1e-5
IMAGE_P99 = 1e-6
REL = 1e-4


def _compare_frame(dbg, stats, ref, colour, depth, tiles_checked=None, settings=None):
    assert stats.splats == ref["slots"]
    assert stats.visible == ref["visible"]
    assert stats.pairs == ref["pairs"]
    assert np.array_equal(dbg["proj"].cpu().numpy().view(np.uint32), ref["proj"].view(np.uint32)), "records differ"
    assert np.array_equal(dbg["rects"].cpu().numpy().view(np.uint32), ref["rects"])
    assert np.array_equal(dbg["touched"].cpu().numpy().view(np.uint32), ref["touched"])
    assert np.array_equal(dbg["depth_keys"].cpu().numpy().view(np.uint32), ref["depth_keys"])
    words = dbg["pairs"].cpu().numpy().view(np.uint64)
    tiles, keys, slots = H.pair_words_to_tile_slot(words, dbg["slot_bits"], dbg["depth_bits"])
    del words
    assert np.array_equal(tiles, ref["pair_tiles"]), "tile order differs"
    del tiles
    assert np.array_equal(slots, ref["pair_slots"]), "splat order differs"
    if keys is not None:
        assert np.array_equal(keys, ref["depth_keys"][ref["pair_slots"]])
    del keys, slots
    assert np.array_equal(dbg["ranges"].cpu().numpy().view(np.uint32), ref["ranges"])
    c = colour.cpu().numpy()
    d = depth.cpu().numpy()
    if tiles_checked is not None:
        tx = (settings.width + 15) // 16
        sel = np.zeros(c.shape[:2], bool)
        for t in tiles_checked:
            y, x = divmod(int(t), tx)
            sel[y * 16:(y + 1) * 16, x * 16:(x + 1) * 16] = True
        c, d = c[sel], d[sel]
        rc, rd = ref["colour"][sel], ref["depth"][sel]
    else:
        rc, rd = ref["colour"], ref["depth"]
    dc = np.abs(c - rc)
    dd = np.abs(d - rd)
    assert dc.max() <= IMAGE_MAX and dd.max() <= IMAGE_MAX, (dc.max(), dd.max())
    assert np.quantile(dc, 0.99) <= IMAGE_P99 and np.quantile(dd, 0.99) <= IMAGE_P99


@pytest.fixture(scope="module")
def headline_cloud():
    packed = L.pack_splats(L.synthetic_records(1_000_000, 1), 15, 3)
    return packed, W.packed_cloud(1_000_000, 1)


@pytest.mark.parametrize("frame", [0, 3])
def test_headline_orbit_frames_equal_the_oracle(rasterizer, headline_cloud, frame):
    packed, host = headline_cloud
    th = 2.0 * math.pi * frame / 20
    cam = L.square_pixel_camera((4.0 * math.sin(th), 0.0, 4.0 * math.cos(th)), (0.0, 0.0, 0.0), 1920, 1080, 60.0,
                                0.01)
    settings = L.RenderSettings(width=1920, height=1080)
    targets = L.RenderTargets()
    stats = rasterizer.render(cam, [L.SplatInstance(L.to_device(packed))], settings, targets)
    dbg = rasterizer.debug_arrays()
    ref = ora.render(W.orbit_projection(frame, 20, 4.0, 1920, 1080), [(host, np.eye(4), None)],
                     W.settings(1920, 1080), 0, want_pairs=True)
    assert stats.pairs > 4_000_000
    _compare_frame(dbg, stats, ref, targets.colour, targets.depth)


def test_sort_heavy_frame_equals_the_oracle(rasterizer):
    dist = dict(mean_sigma=2.0, log_scale_mean=-3.5, log_scale_sigma=0.7)
    raw = L.synthetic_records(6_000_000, 7, **dist)
    packed = L.pack_splats(raw, 15, 3)
    del raw
    cam = L.square_pixel_camera((0.0, 0.0, 4.0), (0.0, 0.0, 0.0), 3840, 2160, 60.0, 0.01)
    settings = L.RenderSettings(width=3840, height=2160)
    targets = L.RenderTargets()
    stats = rasterizer.render(cam, [L.SplatInstance(L.to_device(packed))], settings, targets)
    dbg = rasterizer.debug_arrays()
    assert dbg["tile_bits"] == 15
    host = W.packed_cloud(6_000_000, 7, **dist)
    st = W.settings(3840, 2160)
    rng = np.random.default_rng(5)
    sample = rng.choice(240 * 135, 64, replace=False)
    ref = ora.render(W.square_pixel_projection((0.0, 0.0, 4.0), (0.0, 0.0, 0.0), 3840, 2160), [(host, np.eye(4), None)],
                     st, 0, want_pairs=True, blend_tiles=ora.tile_mask(st, sample))
    assert stats.pairs > 100_000_000
    _compare_frame(dbg, stats, ref, targets.colour, targets.depth, tiles_checked=sample, settings=settings)


def _raw_params(count: int, seed: int) -> dict:
    raw = W.synthetic_records(count, seed)
    n = raw.shape[0]
    sh = np.zeros((n, 16, 3), np.float32)
    sh[:, 0, :] = raw[:, 11:14]
    for c in range(3):
        sh[:, 1:, c] = raw[:, 14 + 15 * c:14 + 15 * (c + 1)]
    sh = sh.astype(np.float16).astype(np.float32)
    return dict(means=np.ascontiguousarray(raw[:, 0:3]), log_scales=np.ascontiguousarray(raw[:, 4:7]),
                quats=np.ascontiguousarray(raw[:, 7:11]), logits=np.ascontiguousarray(raw[:, 3]), sh=sh)


def test_headline_frame_gradients_on_the_centre_crop_match_the_fp64_oracles(rasterizer):
    p = _raw_params(1_000_000, 1)
    crop = (928, 508, 64, 64)
    x0, y0, w, h = crop
    target = np.random.default_rng(3).uniform(0, 1, (h, w, 3))
    pr = W.orbit_projection(0, 20, 4.0, 1920, 1080)
    st = W.settings(1920, 1080)
    cloud = ora.RawCloud(p["means"], p["log_scales"], p["quats"], p["logits"],
                         np.ascontiguousarray(p["sh"].astype(np.float16)))
    out = ora.train_render(pr, cloud, st, crop, crop_only=True)
    prob = G.CropProblem(G.camera_from(pr, st), crop, out["list_offsets"], out["list_slots"], target)
    assert len(prob.used) > 500 and prob.k > 50      # a deep crop: the frame's densest region
    want, loss64 = G.gradients(prob, p)

    cam = L.square_pixel_camera((0.0, 0.0, 4.0), (0.0, 0.0, 0.0), 1920, 1080, 60.0, 0.01)
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda().requires_grad_(True) for k, v in p.items()}
    colour, _ = L.rasterize(t["means"], t["log_scales"], t["quats"], t["logits"], t["sh"], cam,
                            L.RenderSettings(width=1920, height=1080), rasterizer)
    # the training forward's crop is the oracle's
    ref_crop = out["colour"][y0:y0 + h, x0:x0 + w]
    assert np.abs(colour.detach()[y0:y0 + h, x0:x0 + w].cpu().numpy() - ref_crop).max() <= IMAGE_MAX
    tgt = torch.from_numpy(target).cuda()
    loss = torch.abs(colour[y0:y0 + h, x0:x0 + w, :3] - tgt).sum() / (3.0 * w * h)
    loss.backward()
    got = {k: v.grad.detach().cpu().numpy() for k, v in t.items()}
    assert abs(float(loss.detach()) - loss64) <= 1e-5 * max(1.0, abs(loss64))
    used = prob.used
    for name in ("means", "log_scales", "quats", "logits", "sh"):
        g = got[name].reshape(got[name].shape[0], -1)[used].astype(np.float64)
        wv = want[name].reshape(len(used), -1)
        err = np.linalg.norm(g - wv) / max(np.linalg.norm(wv), 1e-30)
        assert err <= REL, (name, err)
    unused = np.setdiff1d(np.arange(p["means"].shape[0]), used)
    assert np.all(got["means"][unused] == 0) and np.all(got["logits"][unused] == 0)

    rng = np.random.default_rng(11)
    names = ["means", "log_scales", "quats", "logits", "sh"]
    picks = []
    for _ in range(256):
        name = names[rng.integers(len(names))]
        row = int(rng.integers(len(used)))
        width = int(np.prod(p[name].shape[1:])) if p[name].ndim > 1 else 1
        picks.append((name, row, int(rng.integers(width))))
    fd = G.finite_difference(prob, p, picks, h=1e-4)
    gpu = np.array([got[n].reshape(got[n].shape[0], -1)[used[r], c] for n, r, c in picks], np.float64)
    scale = np.abs(fd).max()
    err = np.abs(gpu - fd)
    assert np.all(err <= REL * np.abs(fd) + REL * scale), (err / scale).max()
