"""The restated cloud decode for every encoding (splat_encoding.slang), on the
CPU: with the 3DGS PLY encoding it equals the packer the rasteriser tests use
(the reference's decode known answers are pinned on that packer in
test_oracle_pin.py), and the other modes decode as the reference's formulas
say on hand-made records."""
from __future__ import annotations

import math

import numpy as np
import pytest

import lucabrtrender_b200 as L

import decode_fixtures as D
import oracle as ora


def halves(w):
    w = np.asarray(w, np.uint32)
    return (np.stack([w & 0xFFFF, w >> 16], -1).astype(np.uint16).view(np.float16).astype(np.float32))


@pytest.mark.parametrize("rest,keep", [(15, 15), (15, 3), (3, 3), (0, 0)])
def test_the_ply_encoding_decodes_as_the_packer_packs(rest, keep):
    raw = D.records("ply", 5000, 3, rest)
    a = ora.decode_splats(raw, L.ply_encoding(rest), keep)
    b = ora.pack(raw, rest, keep)
    assert a.count == b.count < 5000
    assert np.array_equal(a.positions.view(np.uint32), b.positions.view(np.uint32))
    assert np.array_equal(a.shape, b.shape) and np.array_equal(a.sh, b.sh)


def test_modes_decode_by_the_reference_formulas():
    e = D.encoding("linear", 0)
    raw = np.zeros((1, 14), np.float32)
    raw[0, :3] = [1, 2, 3]
    raw[0, 3] = 0.5                      # linear opacity
    raw[0, 4:7] = [0.1, 0.2, 0.4]        # linear scales -> log
    raw[0, 7:11] = [1, 0, 0, 0]
    raw[0, 11:14] = [0.25, 0.5, 0.75]    # linear colour
    c = ora.decode_splats(raw, e, 0)
    assert c.positions[0, 3] == np.float32(0.5)
    ls = halves(c.shape[0, 1:3]).reshape(-1)
    assert np.allclose(ls[:3], np.log([0.1, 0.2, 0.4]), atol=2e-3)
    assert np.allclose(ls[3], 0.25, atol=1e-3) and np.allclose(halves(c.shape[0, 3]), [0.5, 0.75], atol=1e-3)

    e = D.encoding("bytes", 3)
    raw = np.zeros((1, 23), np.float32)
    raw[0, 3] = 255                      # byte opacity -> 1
    raw[0, 4:7] = -3
    raw[0, 7:11] = [255, 128, 128, 128]  # w x y z bytes -> (1, 0, 0, 0) up to the byte step
    raw[0, 11:14] = [0, 51, 255]         # byte colour
    raw[0, 14:] = 192                    # byte rest -> 0.5
    c = ora.decode_splats(raw, e, 3)
    assert c.positions[0, 3] == 1.0
    assert np.allclose(halves(c.shape[0, 2])[1], 0.0) and np.allclose(halves(c.shape[0, 3]), [0.2, 1.0], atol=1e-3)
    assert np.all(halves(c.sh[0]).reshape(-1)[:9] == 0.5)

    # SPZ: fixed point, byte log scale, first-three rotation, flipped axes
    e = D.encoding("spz_first_three", 3)
    raw = np.zeros((1, 23), np.float32)
    raw[0, :3] = [4096, 8192, -4096]
    raw[0, 3] = 255
    raw[0, 4:7] = 16 * 6                 # log scale 6 - 10 = -4
    raw[0, 7:11] = [0, 127.5, 127.5, 127.5]
    raw[0, 14:] = 192
    c = ora.decode_splats(raw, e, 3)
    assert np.array_equal(c.positions[0], np.float32([1.0, -2.0, 1.0, 1.0]))
    assert np.all(halves(c.shape[0, 1]) == -4.0)
    signs = np.array([-1, -1, 1], np.float32)   # degree-1 bases under the y, z flip
    assert np.array_equal(halves(c.sh[0]).reshape(-1)[:9], np.repeat(signs * 0.5, 3))


def test_the_linear_light_colour_mode_goes_to_the_srgb_curve():
    e = D.encoding("light", 0)
    raw = np.zeros((3, 14), np.float32)
    raw[:, 3] = 5.0
    raw[:, 7] = 1
    raw[:, 11] = [0.001, 0.5, 1.5]
    c = ora.decode_splats(raw, e, 0)
    got = halves(c.shape[:, 2])[:, 1]
    want = [0.001 * 12.92, 1.055 * 0.5 ** (1 / 2.4) - 0.055, 1.055 * 1.5 ** (1 / 2.4) - 0.055]
    assert np.allclose(got, want, atol=2e-3)
