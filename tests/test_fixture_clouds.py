"""The reference's own splat fixtures through the oracle (CPU): the package's
host packing equals the oracle's packing byte for byte, and the restated
rasteriser draws the reference's framing of them within the reference's
ground-truth thresholds (p99 <= 2, max <= 16 8-bit codes) of the restated
brute force, with and without harmonics."""
from __future__ import annotations

import numpy as np
import pytest

import lucabrtrender_b200 as L

import fixture_clouds as FC
import helpers as H
import oracle as ora


@pytest.mark.parametrize("name", ["tiny", "sh3"])
def test_fixture_packs_alike_in_the_package_and_the_oracle(name):
    raw, per_colour = FC.raw_records(name)
    keep = 15 if per_colour >= 15 else per_colour
    ours = L.pack_splats(raw, per_colour, 3)
    theirs = ora.pack(raw, per_colour, keep)
    assert ours.positions.shape[0] == theirs.count == 64
    assert np.array_equal(ours.positions.view(np.uint32), theirs.positions.view(np.uint32))
    assert np.array_equal(ours.shape, theirs.shape)
    assert np.array_equal(ours.sh, theirs.sh)


@pytest.mark.parametrize("name,degree", [("tiny", 0), ("sh3", 0), ("sh3", 3)])
def test_fixture_frame_is_within_the_reference_thresholds_of_the_brute_force(name, degree):
    raw, per_colour = FC.raw_records(name)
    packed = L.pack_splats(raw, per_colour, 3)
    scene = H.Scene(name, [(packed, np.eye(4), None)], FC.sog_test_camera(packed.positions),
                    H.settings(240, 180, max_sh_degree=degree))
    ref = scene.oracle_render()
    truth, _, overflow = scene.oracle_reference()
    assert overflow == 0
    assert ref["pairs"] > 0
    diff = ora.compare_images(ref["colour"], truth)
    assert diff.p99 <= 2 and diff.max <= 16, (diff.p99, diff.max)
