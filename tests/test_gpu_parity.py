"""Parity of the sm_100a path (through the C-ABI) with the oracle: projection
records, tile rectangles, touched counts and depth keys bit for bit; the
sorted pair list and the tile ranges bit for bit; colour and depth within
1e-5 max-abs (they come out identical); and the reference's own render tests
(brute-force thresholds, analytic cases) run on the GPU path."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import lucabrtrender_b200 as L
from lucabrtrender_b200 import _abi

import helpers as H
import oracle as ora

pytestmark = pytest.mark.gpu

IMAGE_TOL = 1e-5   # max-abs on colour and depth (BASELINE tolerance for FP32 images)


def gpu_frame(rasterizer, scene: H.Scene, time_stages=False):
    targets = L.RenderTargets()
    st = scene.settings
    st.time_stages = time_stages
    stats = rasterizer.render(scene.camera, scene.gpu_instances(), st, targets)
    dbg = rasterizer.debug_arrays()
    return targets, stats, dbg


def check_parity(rasterizer, scene: H.Scene, oracle_out=None):
    targets, stats, dbg = gpu_frame(rasterizer, scene)
    ref = oracle_out if oracle_out is not None else scene.oracle_render()
    assert stats.splats == ref["slots"]
    assert stats.visible == ref["visible"]
    assert stats.pairs == ref["pairs"]
    # (a) projection, bit for bit
    proj = dbg["proj"].cpu().numpy()
    assert np.array_equal(proj.view(np.uint32), ref["proj"].view(np.uint32)), "ProjRecord bits differ"
    assert np.array_equal(dbg["rects"].cpu().numpy().view(np.uint32), ref["rects"])
    assert np.array_equal(dbg["touched"].cpu().numpy().view(np.uint32), ref["touched"])
    assert np.array_equal(dbg["depth_keys"].cpu().numpy().view(np.uint32), ref["depth_keys"])
    # (b, c) sorted pairs: tile and slot per position, bit for bit
    words = dbg["pairs"].cpu().numpy().view(np.uint64)
    tiles, keys, slots = H.pair_words_to_tile_slot(words, dbg["slot_bits"], dbg["depth_bits"])
    if "pair_tiles" in ref:
        assert np.array_equal(tiles, ref["pair_tiles"]), "tile order differs"
        assert np.array_equal(slots, ref["pair_slots"]), "splat order differs"
        if keys is not None:
            assert np.array_equal(keys, ref["depth_keys"][ref["pair_slots"]])
    # (d) ranges
    assert np.array_equal(dbg["ranges"].cpu().numpy().view(np.uint32), ref["ranges"])
    # (e) images
    colour = targets.colour.cpu().numpy()
    depth = targets.depth.cpu().numpy()
    assert np.abs(colour - ref["colour"]).max() <= IMAGE_TOL
    assert np.abs(depth - ref["depth"]).max() <= IMAGE_TOL
    return targets, stats, dbg, ref


def test_device_math_bits_equal_the_oracle():
    rng = np.random.default_rng(11)
    sweeps = {
        0: np.concatenate([rng.uniform(-110, 90, 300000), rng.uniform(-4.5, 0, 300000),
                           np.float32([0.0, -0.0, np.inf, -np.inf, 88.7, -103.5])]),
        1: np.concatenate([rng.uniform(1e-38, 1e30, 200000), rng.uniform(1.0001, 255, 300000),
                           np.float32([1e-42, 1.0, 0.0, np.inf])]),
        2: np.concatenate([rng.uniform(-0.5, 3.0, 400000), np.float32([0.04045, 0.0, 1.0])]),
        3: rng.uniform(0.0, 1.0, 300000),
        4: np.concatenate([H.half_sweep(), np.float32([np.nan, -np.nan])]),
        5: H.half_sweep(),   # no NaN: the sign of -x/2 for a NaN x differs between CPUs and GPUs
        # the blend's exp without range checks, over its whole domain
        6: np.concatenate([rng.uniform(-87, 88, 300000), rng.uniform(-4.5, 0, 300000),
                           np.float32([0.0, -0.0, -87.0, 88.0, -4.5])]),
    }
    for fn, x in sweeps.items():
        x = x.astype(np.float32)
        want = ora.math_eval(fn, x)
        got = L.math_eval(fn, torch.from_numpy(x).cuda()).cpu().numpy()
        bad = np.flatnonzero(got.view(np.uint32) != want.view(np.uint32))
        assert bad.size == 0, (fn, bad.size, [(float(x[k]), hex(int(got.view(np.uint32)[k])),
                                              hex(int(want.view(np.uint32)[k]))) for k in bad[:4]])


@pytest.mark.parametrize("scene", H.reference_render_scenes(), ids=lambda s: s.name)
def test_reference_scenes_bit_exact(rasterizer, scene):
    """The reference's five render-test set-ups (3000 splats, 250x190)."""
    check_parity(rasterizer, scene)


@pytest.mark.parametrize("scene", H.edit_scenes(), ids=lambda s: s.name)
def test_edit_scenes_bit_exact(rasterizer, scene):
    check_parity(rasterizer, scene)


@pytest.mark.parametrize("scene", H.reference_render_scenes() + H.edit_scenes(), ids=lambda s: s.name)
def test_gpu_matches_brute_force_ground_truth(rasterizer, scene):
    """test_splat_render.cpp:42-121 on the GPU path: against the per-pixel
    ground truth, p99 <= 2 and max <= 16 8-bit codes, no overflow."""
    targets, _, _ = gpu_frame(rasterizer, scene)
    truth, _, overflow = scene.oracle_reference()
    assert overflow == 0
    diff = ora.compare_images(targets.colour.cpu().numpy(), truth)
    assert diff.p99 <= 2
    assert diff.max <= 16


def test_small_synthetic_config_bit_exact(rasterizer):
    """The CPU-runnable configuration: 100k seeded Gaussians, 512x512, 60 degree
    vertical field of view, 4 units out, SH degree 3."""
    check_parity(rasterizer, H.synthetic_scene(100_000, 512, 512, seed=1))


@pytest.mark.parametrize("w,h,n", [(1, 1, 500), (17, 33, 4000), (640, 480, 30000), (96, 1000, 20000)])
def test_odd_sizes_bit_exact(rasterizer, w, h, n):
    check_parity(rasterizer, H.synthetic_scene(n, w, h, seed=w + h))


def test_settings_variants_bit_exact(rasterizer):
    base = H.synthetic_scene(20000, 200, 150, seed=3)
    for kw in (dict(linearise=False), dict(background=(0.2, 0.3, 0.4, 1.0)), dict(depth=1, threshold=0.3),
               dict(max_sh_degree=0), dict(max_sh_degree=1), dict(max_sh_degree=2), dict(antialias=False)):
        scene = H.Scene(base.name, base.clouds, base.camera, H.settings(200, 150, **kw))
        check_parity(rasterizer, scene)


def test_degree_zero_and_two_clouds_bit_exact(rasterizer):
    for degree, fpc in ((0, 15), (2, 8)):
        raw = L.synthetic_records(8000, 21, degree=3 if fpc == 15 else 2)
        packed = L.pack_splats(raw, fpc, degree)
        cam = L.square_pixel_camera((0, 0, 4), (0, 0, 0), 128, 96)
        check_parity(rasterizer, H.Scene("deg", [(packed, np.eye(4), None)], cam, H.settings(128, 96)))


def test_empty_and_culled_frames(rasterizer):
    st = H.settings(48, 32, background=(0.1, 0.2, 0.3, 0.4))
    targets = L.RenderTargets()
    stats = rasterizer.render(L.Camera(), [], st, targets)
    assert stats.splats == 0 and stats.pairs == 0
    assert torch.allclose(targets.colour, torch.tensor([0.1, 0.2, 0.3, 0.4], device="cuda").expand(32, 48, 4))
    raw = H.cloud_record(0.0, 0.0, 50.0, 0.9, 0.1, 0.1, 0.1, (1, 0, 0, 0), (1, 1, 1))[None]   # behind the camera
    scene = H.Scene("behind", [(L.pack_splats(raw, 3, 3), np.eye(4), None)], L.Camera(), st)
    _, stats, dbg, _ = check_parity(rasterizer, scene)
    assert stats.visible == 0 and stats.pairs == 0
    assert dbg["depth_keys"].cpu().numpy().view(np.uint32)[0] == 0x00FFFFFF


def test_argument_errors(rasterizer):
    targets = L.RenderTargets(10, 10)
    with pytest.raises(_abi.LrtError) as e:
        rasterizer.render(L.Camera(), [], H.settings(0, 10), targets)
    assert e.value.code == _abi.INVALID_ARGUMENT
    bad = L.RenderTargets(10, 10)
    st = H.settings(12, 10)
    # A target of the wrong size is reallocated by the Python mirror (as the reference's
    # reserveTargets does); the raw ABI refuses it.
    pr = L.projection_for(L.Camera(), 12, 10).struct()
    s = st.struct()
    tg = bad.struct()
    stats = _abi.FrameStatsStruct()
    import ctypes as C
    arr = (_abi.SplatInstanceStruct * 1)()
    code = _abi.load().lrt_rast_render(rasterizer._handle, C.byref(pr), arr, 0, C.byref(s), C.byref(tg),
                                       C.byref(stats), None)
    assert code == _abi.INVALID_ARGUMENT


def test_single_splat_lands_on_the_arithmetic_pixel(rasterizer):
    from test_oracle_pin import single_splat_scene
    targets, _, _ = gpu_frame(rasterizer, single_splat_scene())
    a = targets.colour[..., 3].cpu().numpy()
    y, x = np.unravel_index(np.argmax(a), a.shape)
    assert abs(int(x) - 192) <= 1 and abs(int(y) - 136) <= 1


def test_nearer_splat_wins_and_left_stays_left(rasterizer):
    from test_oracle_pin import occlusion_clouds
    cloud = occlusion_clouds()
    st = H.settings(200, 100, linearise=False)
    for eye, front, back, green_left in (((0, 0, 10), 2, 0, True), ((0, 0, -10), 0, 2, False)):
        targets, _, _ = gpu_frame(rasterizer, H.Scene("occ", [(cloud, np.eye(4), None)], H.camera(eye), st))
        p = targets.colour.cpu().numpy()
        assert p[50, 100, front] > 0.9 and p[50, 100, back] < 0.1
        assert (int(np.argmax(p[50, :, 1])) < 100) == green_left


def test_antialias_pays_back_energy(rasterizer):
    raw = H.cloud_record(0.0, 0.0, -50.0, 0.9, 0.002, 0.002, 0.002, (1, 0, 0, 0), (1, 1, 1))[None]
    cloud = L.pack_splats(raw, 3, 3)
    e = []
    for aa in (True, False):
        targets, _, _ = gpu_frame(rasterizer, H.Scene("aa", [(cloud, np.eye(4), None)], L.Camera(),
                                                      H.settings(64, 64, antialias=aa)))
        e.append(float(targets.colour[..., 3].double().sum()))
    assert e[1] > 0 and e[0] < 0.6 * e[1]


def test_stage_times_and_buffer_growth(rasterizer):
    small = H.synthetic_scene(2000, 64, 64, seed=5)
    big = H.synthetic_scene(60000, 320, 240, seed=6)
    for scene in (small, big, small):
        targets, stats, _ = gpu_frame(rasterizer, scene, time_stages=True)
        assert stats.project_ms > 0 and stats.blend_ms > 0 and stats.total_ms > 0
    check_parity(rasterizer, small)
    check_parity(rasterizer, big)


# ------------------------------------------------------- sort and scan -----
def pcg(v: np.ndarray) -> np.ndarray:
    """shaders/lrt/test/sort_generate.slang:72-76 in uint32 arithmetic."""
    v = v.astype(np.uint64)
    state = (v * 747796405 + 2891336453) & 0xFFFFFFFF
    word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & 0xFFFFFFFF
    return ((word >> 22) ^ word).astype(np.uint32)


def sort_generate(count: int, mode: int, key_bits: int):
    """sort_generate.slang:78-97 with the seed of test_algo.cpp:60-67."""
    seed = np.uint32(0x9E3779B9 ^ count ^ (mode << 8))
    i = np.arange(count, dtype=np.uint32)
    if mode == 0:
        lo = pcg(i ^ seed)
        hi = pcg((lo.astype(np.uint64) + int(seed)) & 0xFFFFFFFF)
    elif mode == 1:
        lo = np.full(count, 0x5A5A5A5A, np.uint32)
        hi = np.full(count, 0xA5A5, np.uint32)
    elif mode == 2:
        lo, hi = i.copy(), np.zeros(count, np.uint32)
    elif mode == 3:
        lo, hi = (count - 1 - i).astype(np.uint32), np.full(count, 7, np.uint32)
    else:
        lo = pcg(i ^ seed) % np.uint32(13)
        hi = pcg((i.astype(np.uint64) + int(seed)) & 0xFFFFFFFF) % np.uint32(3)
    mask_lo = 0xFFFFFFFF if key_bits >= 32 else (1 << key_bits) - 1
    mask_hi = (1 << (key_bits - 32)) - 1 if key_bits > 32 else 0
    lo &= np.uint32(mask_lo)
    hi &= np.uint32(mask_hi)
    return lo, hi, i


@pytest.mark.parametrize("count,key_bits", [(1, 32), (2, 32), (4097, 13), (65537, 32), (300007, 24),
                                            (250001, 64), (100000, 40)])
@pytest.mark.parametrize("mode", range(5))
def test_radix_sort_orders_stably_and_loses_nothing(rasterizer, count, key_bits, mode):
    """test_algo.cpp:347-379: every pattern, ordered, stable on ties, a permutation."""
    lo, hi, vals = sort_generate(count, mode, key_bits)
    if key_bits > 32:
        keys = (hi.astype(np.uint64) << np.uint64(32)) | lo.astype(np.uint64)
        kt = torch.from_numpy(keys.view(np.int64)).cuda()
    else:
        keys = lo
        kt = torch.from_numpy(keys.view(np.int32)).cuda()
    vt = torch.from_numpy(vals.view(np.int32)).cuda()
    rasterizer.radix_sort(kt, vt, key_bits)
    order = np.argsort(keys, kind="stable")
    got_k = kt.cpu().numpy().view(keys.dtype)
    got_v = vt.cpu().numpy().view(np.uint32)
    assert np.array_equal(got_k, keys[order])
    assert np.array_equal(got_v, vals[order])


def test_radix_sort_without_values_and_partial_bits(rasterizer):
    rng = np.random.default_rng(2)
    keys = rng.integers(0, 2**63, 1_000_003, dtype=np.uint64)
    kt = torch.from_numpy(keys.view(np.int64)).cuda()
    rasterizer.radix_sort(kt, None, 20)    # only the low 20 bits are ordered: 3 passes of 8 bits
    got = kt.cpu().numpy().view(np.uint64)
    want = keys[np.argsort(keys & np.uint64((1 << 24) - 1), kind="stable")]
    assert np.array_equal(got, want)


@pytest.mark.parametrize("count", [1, 7, 4095, 4096, 4097, 100003, 1 << 22])
def test_prefix_sum_every_size(rasterizer, count):
    """test_algo.cpp:72-109 with counts_generate.slang's values."""
    h = pcg(np.arange(count, dtype=np.uint32) ^ np.uint32(1234))
    counts = np.where((h & 7) == 0, 0, h % 37).astype(np.uint32)
    inp = torch.from_numpy(counts.view(np.int32)).cuda()
    out = torch.empty_like(inp)
    total = torch.zeros(1, dtype=torch.int32, device="cuda")
    rasterizer.prefix_sum(inp, out, total)
    want = np.concatenate([[0], np.cumsum(counts.astype(np.uint64))[:-1]]).astype(np.uint32)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), want)
    assert int(total.cpu().numpy().view(np.uint32)[0]) == int(counts.astype(np.uint64).sum())
