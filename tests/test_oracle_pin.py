"""Pinning the oracle (CPU, no GPU): the reference's own known answers, golden
camera vectors from the reference's C++ camera code, and the invariants the
reference's tests assert, all checked against the CPU restatement."""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

import lucabrtrender_b200 as L
from lucabrtrender_b200 import _abi

import helpers as H
import oracle as ora

GOLDEN = Path(__file__).resolve().parent / "golden"


def _golden_cases():
    return json.loads((GOLDEN / "camera_ref.json").read_text())


def _hexs(xs):
    return [float.fromhex(x) for x in xs]


@pytest.mark.parametrize("case", _golden_cases(), ids=lambda c: c["name"])
def test_camera_matches_reference_camera_code(case):
    """projectionFor/lookingAt restated (product C++ and oracle) equal what the
    reference's own Camera.cpp computed, to the last bit."""
    cam = H.camera(case["eye"], case["target"], focal=case["focal"], orthographic=bool(case["orthographic"]),
                   window_translate=case["window_translate"], window_scale=case["window_scale"],
                   roll=case["window_roll"], near=case["near_z"])
    p = L.projection_for(cam, case["width"], case["height"])
    want_m = _hexs(case["world_to_view"])
    want_f = _hexs(case["focal_centre_near_far"])
    want_e = _hexs(case["eye_world"])
    assert list(np.asarray(p.world_to_view).reshape(16)) == want_m
    assert [p.focal_x, p.focal_y, p.centre_x, p.centre_y, p.near_z, p.far_z] == want_f
    assert list(p.eye_world) == want_e

    oc = ora.looking_at(case["eye"], case["target"], case["up"])
    oc.lens.focal = case["focal"]
    oc.lens.orthographic = case["orthographic"]
    oc.lens.window_translate[:] = case["window_translate"]
    oc.lens.window_scale[:] = case["window_scale"]
    oc.lens.window_roll = case["window_roll"]
    oc.lens.near_z = case["near_z"]
    op = ora.projection_for(oc, case["width"], case["height"])
    assert list(op.world_to_view) == want_m
    assert [op.focal_x, op.focal_y, op.centre_x, op.centre_y, op.near_z, op.far_z] == want_f


def test_camera_live_reference_if_built():
    """When the reference's camera code is built here (oracle/_ref), compare live too."""
    if not ora.REF_LIB.exists():
        pytest.skip("oracle/_ref not built")
    import ctypes as C
    lib = C.CDLL(str(ora.REF_LIB))
    d3 = C.c_double * 3
    lib.ref_camera_projection.argtypes = [d3, d3, d3, C.c_int] + [C.c_double] * 7 + [C.c_uint32, C.c_uint32,
                                                                                       C.c_void_p, C.c_void_p,
                                                                                       C.c_void_p]
    rng = np.random.default_rng(5)
    for _ in range(50):
        eye = rng.normal(size=3) * 5
        target = rng.normal(size=3)
        focal = float(rng.uniform(10, 80))
        roll = float(rng.uniform(-90, 90))
        m, f6, e3 = (C.c_double * 16)(), (C.c_double * 6)(), (C.c_double * 3)()
        lib.ref_camera_projection(d3(*eye), d3(*target), d3(0, 1, 0), 0, focal, 0.1, -0.2, 1.1, 0.9, roll, 0.05,
                                  333, 211, m, f6, e3)
        cam = H.camera(eye, target, focal=focal, window_translate=(0.1, -0.2), window_scale=(1.1, 0.9), roll=roll,
                       near=0.05)
        p = L.projection_for(cam, 333, 211)
        assert list(np.asarray(p.world_to_view).reshape(16)) == list(m)
        assert [p.focal_x, p.focal_y, p.centre_x, p.centre_y, p.near_z, p.far_z] == list(f6)


# --------------------------------------------------------------- math ------
def _ulp_err(got: np.ndarray, want: np.ndarray) -> np.ndarray:
    got = got.astype(np.float64)
    ulp = np.spacing(np.abs(want).astype(np.float32)).astype(np.float64)
    return np.abs(got - want) / ulp


def test_oracle_exp_log_accuracy():
    """The project's own exp/log are within 2 ulp of the true value."""
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.uniform(-87, 88, 200000), rng.uniform(-4.5, 0, 200000),
                        np.linspace(-103, -87, 5000)]).astype(np.float32)
    y = ora.math_eval(0, x)
    want = np.exp(x.astype(np.float64))
    normal = want > 1.2e-38
    assert _ulp_err(y[normal], want[normal]).max() <= 2.0
    assert np.all(np.abs(y[~normal] - want[~normal]) <= 1.5e-45)
    xl = np.concatenate([rng.uniform(1e-30, 1e30, 100000), rng.uniform(0.5, 2.0, 200000),
                         rng.uniform(1.0001, 255, 200000), np.float32([1e-42, 3e-40, 1.0, 2.0])]).astype(np.float32)
    yl = ora.math_eval(1, xl)
    wl = np.log(xl.astype(np.float64))
    err = np.abs(yl.astype(np.float64) - wl) / np.spacing(np.maximum(np.abs(wl), 1e-30).astype(np.float32))
    assert err.max() <= 2.0
    assert ora.math_eval(0, np.float32([np.nan, np.inf, -np.inf, 100.0]))[1:].tolist() == [np.inf, 0.0, np.inf]
    assert np.isnan(ora.math_eval(1, np.float32([-1.0]))[0])


def test_oracle_half_rounding_is_ieee_nearest_even():
    """fn 4 (the packing's float-to-half) rounds as IEEE binary16 nearest-even
    (numpy's float16 conversion); NaN becomes the quiet NaN 0x7E00."""
    x = H.half_sweep()
    got = ora.math_eval(4, x).view(np.uint32)
    with np.errstate(over="ignore"):
        want = x.astype(np.float16).view(np.uint16).astype(np.uint32)
    assert np.array_equal(got, want)
    assert ora.math_eval(4, np.float32([np.nan])).view(np.uint32).tolist() == [0x7E00]
    pair = ora.math_eval(5, x).view(np.uint32)
    with np.errstate(over="ignore"):
        high = (np.float32(-0.5) * x).astype(np.float16).view(np.uint16).astype(np.uint32)
    assert np.array_equal(pair, want | (high << np.uint32(16)))


# ------------------------------------------------------------- packing -----
def _decode_splat(p: L.PackedSplats, i: int):
    """What shaders/lrt/test/splat_inspect.slang reads back: position, opacity,
    linear scales, quaternion (x, y, z, w), base colour, rest coefficients."""
    f16 = lambda h: np.frombuffer(np.uint16(h).tobytes(), np.float16)[0].astype(np.float32)  # noqa: E731
    s = p.shape[i]
    scale = [math.exp(f16(s[1] & 0xFFFF)), math.exp(f16(s[1] >> 16)), math.exp(f16(s[2] & 0xFFFF))]
    base = [f16(s[2] >> 16), f16(s[3] & 0xFFFF), f16(s[3] >> 16)]
    w = int(s[0])
    largest = w & 3
    small = [((w >> 22) & 1023), ((w >> 12) & 1023), ((w >> 2) & 1023)]
    small = [(v / 1023.0 * 2 - 1) * 0.70710678 for v in small]
    rest = math.sqrt(max(0.0, 1 - sum(v * v for v in small)))
    q, it = [], iter(small)
    for k in range(4):
        q.append(rest if k == largest else next(it))
    halves = []
    for word in p.sh[i]:
        halves += [f16(word & 0xFFFF), f16(word >> 16)]
    return list(p.positions[i]), scale, q, base, halves


def test_decode_matches_reference_known_values():
    """tests/scene/test_loading.cpp:91-165: a 3DGS record decodes opacity,
    scale, rotation, colour and harmonics; faint and NaN records are dropped,
    order kept."""
    fpr = 14 + 9

    def rec(x, y, z, opacity, scales, rot_wxyz, dc, rest):
        r = np.zeros(fpr, np.float32)
        r[:14] = [x, y, z, opacity, *scales, *rot_wxyz, *dc]
        r[14:] = rest
        return r

    rest = [0.1 * (k + 1) for k in range(9)]   # r .1 .2 .3, g .4 .5 .6, b .7 .8 .9
    first = rec(1, 2, 3, 0.0, [0.0, 0.6931472, -0.6931472], [2, 0, 0, 0], [0, 0, 0], rest)
    faint = first.copy()
    faint[3] = -10.0
    broken = first.copy()
    broken[0] = np.nan
    last = rec(-4, 5, -6, 1.0986123, [0.0, 0.6931472, -0.6931472], [0, 0, 0, -3], [1.0 / 0.28209479, 0, 0], rest)
    raw = np.stack([first, faint, broken, last])
    for packer in ("product", "oracle"):
        if packer == "product":
            p = L.pack_splats(raw, 3, 3)
        else:
            hc = ora.pack(raw, 3, 3)
            p = L.PackedSplats(hc.positions, hc.shape, hc.sh, hc.rest_per_colour)
        assert p.count == 2
        assert p.rest_per_colour == 3
        pos, scale, q, base, halves = _decode_splat(p, 0)
        assert pos[:3] == [1.0, 2.0, 3.0]
        assert abs(pos[3] - 0.5) <= 1e-6
        assert scale == pytest.approx([1.0, 2.0, 0.5], rel=2e-3)
        assert abs(q[3] - 1.0) <= 1e-3
        assert abs(base[0] - 0.5) <= 1e-3
        assert halves[:4] == pytest.approx([0.1, 0.4, 0.7, 0.2], abs=1e-3)
        pos, scale, q, base, halves = _decode_splat(p, 1)
        assert pos[0] == -4.0
        assert abs(pos[3] - 0.75) <= 1e-5
        assert abs(abs(q[2]) - 1.0) <= 1e-3
        assert abs(base[0] - 1.5) <= 1e-3
    flat = L.pack_splats(raw, 3, 0)
    assert flat.rest_per_colour == 0 and flat.sh_words == 1


def test_product_packer_equals_oracle_packer():
    """lrt_pack_splats and the oracle's restatement give the same bytes."""
    raws = [(L.synthetic_records(20000, 3), 15, 3), (L.synthetic_records(5000, 4, degree=2), 8, 2),
            (ora.random_cloud(3000, 7), 3, 3), (L.synthetic_records(3000, 5, degree=3), 15, 1)]
    edge = L.synthetic_records(64, 9)
    edge[0, 0] = np.nan
    edge[1, 3] = -20.0          # faint
    edge[2, 4] = 70.0           # |log scale| >= 60
    edge[3, 7:11] = 0.0         # zero quaternion -> identity
    edge[4, 4:7] = 1e6          # clamped by halfSafe? no: dropped (>= 60)
    edge[5, 14:] = 1e6          # rest past f16 range -> halfSafe clamp
    raws.append((edge, 15, 3))
    for raw, fpc, deg in raws:
        a = L.pack_splats(raw, fpc, deg)
        keep = min(fpc, {0: 0, 1: 3, 2: 8, 3: 15}[deg])
        b = ora.pack(raw, fpc, keep)
        assert a.count == b.count
        assert np.array_equal(a.positions.view(np.uint32), b.positions.view(np.uint32))
        assert np.array_equal(a.shape, b.shape)
        assert np.array_equal(a.sh, b.sh)


# ------------------------------------------------ the reference's renders ----
@pytest.mark.parametrize("scene", H.reference_render_scenes(), ids=lambda s: s.name)
def test_oracle_raster_matches_brute_force(scene):
    """test_splat_render.cpp:70-121 on the restatement: the tile rasteriser
    against the per-pixel ground truth, p99 <= 2 and max <= 16 codes, no
    overflowing pixel."""
    ours = scene.oracle_render(want_pairs=False)
    truth, _, overflow = scene.oracle_reference()
    assert overflow == 0
    diff = ora.compare_images(ours["colour"], truth)
    assert diff.p99 <= 2
    assert diff.max <= 16
    assert ours["pairs"] > 0


@pytest.mark.parametrize("scene", H.edit_scenes(), ids=lambda s: s.name)
def test_oracle_edit_matches_brute_force(scene):
    """test_splat_render.cpp:231-283: SplatEdit vs the ground truth, and the
    edit visibly changes the picture."""
    ours = scene.oracle_render(want_pairs=False)
    truth, _, overflow = scene.oracle_reference()
    assert overflow == 0
    assert ora.compare_images(ours["colour"], truth).p99 <= 2
    plain = H.Scene("plain", [(c, m, None) for c, m, _ in scene.clouds], scene.camera, scene.settings)
    changed = ora.compare_images(ours["colour"], plain.oracle_render(want_pairs=False)["colour"])
    assert changed.over2 > changed.pixels // 20


def single_splat_scene() -> H.Scene:
    raw = H.cloud_record(1.0, 0.5, -10.0, 0.9, 0.02, 0.02, 0.02, (1, 0, 0, 0), (1, 1, 1))[None]
    cam = L.Camera()                      # at the origin, looking down -Z
    cam.lens.focal = cam.lens.haperture   # fx = width
    return H.Scene("single", [(L.pack_splats(raw, 3, 3), np.eye(4), None)], cam, H.settings(320, 240))


def test_oracle_single_splat_lands_on_the_arithmetic_pixel():
    """test_splat_render.cpp:123-150: x = 160 + 320 * 1/10 = 192, y = 120 + 320 * 0.5/10 = 136."""
    out = single_splat_scene().oracle_render(want_pairs=False)
    a = out["colour"][..., 3]
    y, x = np.unravel_index(np.argmax(a), a.shape)
    assert abs(int(x) - 192) <= 1 and abs(int(y) - 136) <= 1


def occlusion_clouds():
    raws = np.stack([
        H.cloud_record(0.0, 0.0, -1.0, 0.99, 0.5, 0.5, 0.05, (1, 0, 0, 0), (1, 0, 0)),   # red, z = -1
        H.cloud_record(0.0, 0.0, 1.0, 0.99, 0.5, 0.5, 0.05, (1, 0, 0, 0), (0, 0, 1)),    # blue, z = +1
        H.cloud_record(-3.0, 0.0, 0.0, 0.99, 0.3, 0.3, 0.3, (1, 0, 0, 0), (0, 1, 0)),    # green, -x
    ])
    return L.pack_splats(raws, 3, 3)


def test_oracle_nearer_splat_wins_and_left_stays_left():
    """test_splat_render.cpp:152-200."""
    cloud = occlusion_clouds()
    st = H.settings(200, 100, linearise=False)
    for eye, front, back, green_left in (((0, 0, 10), 2, 0, True), ((0, 0, -10), 0, 2, False)):
        sc = H.Scene("occ", [(cloud, np.eye(4), None)], H.camera(eye), st)
        p = sc.oracle_render(want_pairs=False)["colour"]
        centre = p[50, 100]
        assert centre[front] > 0.9 and centre[back] < 0.1
        bx = int(np.argmax(p[50, :, 1]))
        assert (bx < 100) == green_left


def test_oracle_antialias_pays_back_energy():
    """test_splat_render.cpp:202-229: with < 0.6 * without."""
    raw = H.cloud_record(0.0, 0.0, -50.0, 0.9, 0.002, 0.002, 0.002, (1, 0, 0, 0), (1, 1, 1))[None]
    cloud = L.pack_splats(raw, 3, 3)
    energies = []
    for aa in (True, False):
        sc = H.Scene("aa", [(cloud, np.eye(4), None)], L.Camera(), H.settings(64, 64, antialias=aa))
        energies.append(float(sc.oracle_render(want_pairs=False)["colour"][..., 3].astype(np.float64).sum()))
    with_aa, without = energies
    assert without > 0.0 and with_aa < 0.6 * without


def test_oracle_edit_is_per_instance_in_object_space():
    """test_splat_render.cpp:285-324."""
    raw = H.cloud_record(0.0, 0.0, 0.0, 0.95, 0.3, 0.3, 0.3, (1, 0, 0, 0), (1, 1, 1))[None]
    cloud = L.pack_splats(raw, 3, 3)
    keep_nothing = L.SplatEdit(active=True, mode=L.EditMode.KEEP, centre=(5.0, 0.0, 0.0))
    green_only = L.SplatEdit(active=True, mode=L.EditMode.GRADE, size=(1.0, 1.0, 1.0), tint=(0.0, 1.0, 0.0))
    sc = H.Scene("edit2", [(cloud, H.translation((-1, 0, 0)), keep_nothing),
                           (cloud, H.translation((1, 0, 0)), green_only)],
                 H.camera((0, 0, 5)), H.settings(65, 65))
    p = sc.oracle_render(want_pairs=False)["colour"]
    left, right = p[32, 32 - 26], p[32, 32 + 26]
    assert left[3] < 0.01
    assert right[3] > 0.5 and right[0] < 0.01 and right[2] < 0.01 and right[1] > 0.3


def test_oracle_pair_order_is_tile_then_depth_key_then_slot():
    """frame.slang:17-20: the depth sort then the stable tile sort leave each
    tile's pairs in (24-bit depth key, slot) order -- the order one sort of
    (tile | key) over pairs emitted in slot order gives."""
    for scene in H.reference_render_scenes()[:2] + [H.synthetic_scene(20000, 160, 96)]:
        out = scene.oracle_render()
        tiles, slots = out["pair_tiles"], out["pair_slots"]
        keys = out["depth_keys"][slots]
        order = np.lexsort((slots, keys, tiles))
        assert np.array_equal(order, np.arange(tiles.size))
        assert tiles.size == out["pairs"] == int(out["touched"].sum())
        # ranges are exactly the runs of equal tiles
        r = out["ranges"]
        for t in np.unique(tiles):
            idx = np.nonzero(tiles == t)[0]
            assert r[t, 0] == idx[0] and r[t, 1] == idx[-1] + 1


def test_oracle_culled_slots_and_empty_frame():
    """splat_project.slang:39-49: a culled slot has key 0x00FFFFFF, rect (1,1,0,0)."""
    raw = H.cloud_record(0.0, 0.0, 50.0, 0.9, 0.1, 0.1, 0.1, (1, 0, 0, 0), (1, 1, 1))[None]   # behind the camera
    sc = H.Scene("behind", [(L.pack_splats(raw, 3, 3), np.eye(4), None)], L.Camera(), H.settings(40, 30))
    out = sc.oracle_render()
    assert out["pairs"] == 0 and out["visible"] == 0
    assert out["depth_keys"][0] == 0x00FFFFFF
    assert out["rects"][0].tolist() == [1, 1, 0, 0]
    assert np.all(out["colour"] == 0)
