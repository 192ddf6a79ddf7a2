"""The reference's own splat fixtures on the GPU: decoded on the device into
the same bytes as the host packing, and the reference's framing of them
(tests/render/test_sog.cpp:41-66) drawn bit for bit as the oracle draws it,
with and without harmonics."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import lucabrtrender_b200 as L

import fixture_clouds as FC
import helpers as H

from test_gpu_parity import check_parity

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["tiny", "sh3"])
def test_fixture_decodes_on_the_device_as_on_the_host(rasterizer, name):
    raw, per_colour = FC.raw_records(name)
    packed = L.pack_splats(raw, per_colour, 3)
    cloud = rasterizer.decode_splats(torch.from_numpy(raw).cuda(), L.ply_encoding(per_colour), min(per_colour, 15))
    assert cloud.count == 64
    assert np.array_equal(cloud.positions.cpu().numpy().view(np.uint32), packed.positions.view(np.uint32))
    assert np.array_equal(cloud.shape.cpu().numpy().view(np.uint32), packed.shape)
    assert np.array_equal(cloud.sh.cpu().numpy().view(np.uint32), packed.sh)


@pytest.mark.parametrize("name,degree", [("tiny", 0), ("sh3", 0), ("sh3", 3)])
def test_fixture_frame_equals_the_oracle(rasterizer, name, degree):
    raw, per_colour = FC.raw_records(name)
    packed = L.pack_splats(raw, per_colour, 3)
    scene = H.Scene(name, [(packed, np.eye(4), None)], FC.sog_test_camera(packed.positions),
                    H.settings(240, 180, max_sh_degree=degree))
    check_parity(rasterizer, scene)
