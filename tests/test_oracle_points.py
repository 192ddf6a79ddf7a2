"""The restated disc route and composite blend, on the CPU: points packed as
the reference's loader packs them, drawn as opaque discs sorted with the
splats, checked against the restated brute force with the reference's own
thresholds (tests/render/test_points.cpp:75-99), and splats composited over a
layer of discs against the same splats and discs in one sort (:153-200, with
the layer drawn by the disc route: the reference's raster route needs a
rasterisation pipeline)."""
from __future__ import annotations

import math

import numpy as np
import pytest

import lucabrtrender_b200 as L

import helpers as H
import oracle as ora


def proj_of(eye, w, h, target=(0, 0, 0)):
    return L.projection_for(L.Camera.looking_at(eye, target), w, h).struct()


def test_the_library_packs_points_as_the_oracle_does():
    raw = ora.random_points(5000, 9)
    raw[17, 1] = np.inf
    raw[:, 3:] *= 255.0
    for kind, detail in ((0, 1.0), (1, 1.0), (2, 1.0), (2, 0.5)):
        a = L.pack_points(raw, kind, detail)
        b = ora.pack_points(raw, kind, detail)
        assert np.array_equal(a.positions, b.positions) and np.array_equal(a.colours, b.colours), (kind, detail)


def test_pack_points_decodes_like_the_loader():
    raw = np.array([[0, 1, 2, 255, 128, 0], [np.nan, 0, 0, 1, 1, 1], [3, 4, 5, 0.25, 0.5, 1.0]], np.float32)
    for kind in (0, 1, 2):
        p = ora.pack_points(raw, kind)
        assert p.count == 2                                   # the NaN point is dropped, order kept
        assert np.array_equal(p.positions, np.array([[0, 1, 2, 1], [3, 4, 5, 1]], np.float32))
        half = lambda w: np.array([w & 0xFFFF], np.uint16).view(np.float16)[0]  # noqa: E731
        got = np.array([[half(c[0]), half(c[0] >> 16), half(c[1]), half(c[1] >> 16)] for c in p.colours], np.float32)
        if kind == 0:
            want = np.ones((2, 4), np.float32)
        elif kind == 2:
            want = np.array([[255, 128, 0, 1], [0.25, 0.5, 1.0, 1]], np.float32).astype(np.float16).astype(np.float32)
        else:
            lin = ora.math_eval(2, np.array([1.0, 128 / 255, 0.0, 0.25 / 255, 0.5 / 255, 1.0 / 255], np.float32))
            want = np.array([[*lin[:3], 1], [*lin[3:], 1]], np.float32).astype(np.float16).astype(np.float32)
        assert np.array_equal(got, want), kind
    # thinning by the index hash: deterministic, and about `detail` of the points
    many = ora.random_points(20000, 1)
    a, b = ora.pack_points(many, 2, 0.3), ora.pack_points(many, 2, 0.3)
    assert np.array_equal(a.positions, b.positions)
    assert 0.28 < a.count / 20000 < 0.32


@pytest.mark.parametrize("mode,size", [(0, 0.06), (1, 5.0)], ids=["world", "pixels"])
def test_discs_match_the_brute_force(mode, size):
    pts = ora.pack_points(ora.random_points(4000, 3), 2)
    st = H.settings(230, 170, linearise=False).struct()
    pr = proj_of((1.0, 2.0, 6.0), 230, 170)
    points = [(pts, np.eye(4), H.point_style(mode, size))]
    ours = ora.render(pr, [], st, points=points, want_pairs=False)
    truth, _, over = ora.reference_render(pr, [], st, points=points)
    assert over == 0
    diff = ora.compare_images(ours["colour"], truth)
    assert diff.p99 <= 2, (diff.p99, diff.max)
    assert ours["visible"] > 2000
    # every visible disc is opaque: alpha one, colour.w one, cut at one radius
    vis = ours["touched"] > 0
    rec = ours["proj"][vis]
    assert np.all(rec[:, 7] == 1.0) and np.all(rec[:, 11] == 1.0) and np.all(rec[:, 3] == 1.0)


def test_a_disc_is_a_hard_opaque_edge():
    pts = ora.pack_points(np.array([[0, 0, 0, 0.2, 0.4, 0.8]], np.float32), 2)
    st = H.settings(64, 64, linearise=False, background=(0.0, 0.0, 0.0, 0.0)).struct()
    pr = proj_of((0.0, 0.0, 4.0), 64, 64)
    out = ora.render(pr, [], st, points=[(pts, np.eye(4), H.point_style(1, 10.0))], want_pairs=False)
    c = out["colour"]
    centre = c[32, 32]
    assert np.allclose(centre, [0.2, 0.4, 0.8, 1.0], atol=1e-3)   # f16 of the colour, alpha one
    assert out["depth"][32, 32] == pytest.approx(4.0, rel=1e-5)
    assert np.all(c[0, 0] == 0) and np.all(c[32, 50] == 0)          # outside the 5-pixel radius: nothing


def test_splats_over_a_disc_layer_match_one_mixed_sort():
    pts = ora.pack_points(ora.random_points(8000, 5), 2)
    fog = ora.pack(H.fog_records(), 3, 3)
    st = H.settings(256, 180).struct()
    pr = proj_of((0.5, 0.5, 7.0), 256, 180)
    points = [(pts, np.eye(4), H.point_style(0, 0.05))]
    layer = ora.render(pr, [], st, points=points, want_pairs=False)
    composited = ora.render(pr, [(fog, np.eye(4), None)], st, under=(layer["colour"], layer["depth"]),
                            want_pairs=False)
    mixed = ora.render(pr, [(fog, np.eye(4), None)], st, points=points, want_pairs=False)
    diff = ora.compare_images(composited["colour"], mixed["colour"])
    assert diff.p99 <= 2, (diff.p99, diff.max)
    # the fog does change the picture
    assert ora.compare_images(composited["colour"], layer["colour"]).max > 16


def test_a_splat_in_front_of_the_layer_blends_over_it_and_one_behind_is_hidden():
    st = H.settings(64, 64, linearise=False).struct()
    pr = proj_of((0.0, 0.0, 5.0), 64, 64)
    under_colour = np.zeros((64, 64, 4), np.float32)
    under_colour[...] = [0.1, 0.7, 0.2, 1.0]
    under_depth = np.full((64, 64), 5.0, np.float32)      # the layer at view depth 5
    front = ora.pack(np.stack([H.cloud_record(0, 0, 1.0, 0.9, 0.3, 0.3, 0.3, (1, 0, 0, 0), (1.0, 0.0, 0.0))]), 3, 3)
    behind = ora.pack(np.stack([H.cloud_record(0, 0, -1.0, 0.9, 0.3, 0.3, 0.3, (1, 0, 0, 0), (1.0, 0.0, 0.0))]), 3, 3)
    a = ora.render(pr, [(front, np.eye(4), None)], st, under=(under_colour, under_depth), want_pairs=False)
    b = ora.render(pr, [(behind, np.eye(4), None)], st, under=(under_colour, under_depth), want_pairs=False)
    # in front (view z 4 < 5): red over green at the centre; behind (z 6): only the layer
    assert a["colour"][32, 32, 0] > 0.5 and a["colour"][32, 32, 1] < 0.7
    assert np.allclose(b["colour"][32, 32], [0.1, 0.7, 0.2, 1.0])
    assert b["depth"][32, 32] == pytest.approx(5.0)
