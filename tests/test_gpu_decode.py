"""Cloud decode on the device (lrt_rast_decode_splats / _points): validate,
compact and pack in one kernel, bit for bit equal to the restated decode for
every encoding, across many blocks (the compaction's look-back), and a cloud
decoded on the device renders the same frame as one packed on the host."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import lucabrtrender_b200 as L

import decode_fixtures as D
import helpers as H
import oracle as ora

pytestmark = pytest.mark.gpu


def as_host(g: L.GpuSplats):
    return (g.positions.cpu().numpy(), g.shape.cpu().numpy().view(np.uint32), g.sh.cpu().numpy().view(np.uint32))


@pytest.mark.parametrize("kind", D.ENCODINGS)
@pytest.mark.parametrize("count,keep", [(5000, 15), (70001, 8)])
def test_device_decode_equals_the_restatement(rasterizer, kind, count, keep):
    raw = D.records(kind, count, 11)
    e = D.encoding(kind)
    got = rasterizer.decode_splats(torch.from_numpy(raw).cuda(), e, keep)
    want = ora.decode_splats(raw, e, keep)
    pos, shape, sh = as_host(got)
    assert got.count == want.count < count
    assert np.array_equal(pos.view(np.uint32), want.positions.view(np.uint32))
    assert np.array_equal(shape, want.shape) and np.array_equal(sh, want.sh)


def test_device_point_decode_equals_the_packer(rasterizer):
    raw = ora.random_points(300_000, 2)
    raw[::997, 0] = np.inf
    for kind, detail in ((2, 1.0), (1, 1.0), (0, 0.4)):
        r = raw.copy()
        if kind == 1:
            r[:, 3:] *= 255.0
        got = rasterizer.decode_points(torch.from_numpy(r).cuda(), kind, detail)
        want = ora.pack_points(r, kind, detail)
        assert got.count == want.count
        assert np.array_equal(got.positions.cpu().numpy(), want.positions)
        assert np.array_equal(got.colours.cpu().numpy().view(np.uint32), want.colours)


def test_a_device_decoded_cloud_renders_as_the_host_packed_one(rasterizer):
    raw = L.synthetic_records(1_000_000, 21)
    raw[::1000, 3] = -40.0   # faint: dropped
    dev = rasterizer.decode_splats(torch.from_numpy(raw).cuda(), L.ply_encoding(15), 15)
    host = L.to_device(L.pack_splats(raw, 15, 3))
    assert dev.count == host.count
    settings = L.RenderSettings(width=640, height=360)
    cam = L.square_pixel_camera((0.0, 0.5, 4.0), (0.0, 0.0, 0.0), 640, 360)
    a, b = L.RenderTargets(), L.RenderTargets()
    rasterizer.render(cam, [L.SplatInstance(dev)], settings, a)
    rasterizer.render(cam, [L.SplatInstance(host)], settings, b)
    assert torch.equal(a.colour, b.colour) and torch.equal(a.depth, b.depth)
