"""Levels of detail on the device, through the C-ABI, against the oracle.

The build (store, codes, each level's cells and merged Gaussians, the finest
level's starts) and every cut (the drawn cloud and its counts) must equal the
CPU restatement bit for bit. The reference's own LOD tests
(tests/lod/test_lod.cpp:82-189) then run on the device renderer and the
device compareImages with the reference's bounds; at a million splats the
size-independent properties hold (sorted codes, threshold 0 = the store, a
huge threshold = the coarsest level, every splat drawn exactly once)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import lucabrtrender_b200 as L

import helpers as H
import oracle as ora

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def raster():
    r = L.TileRasterizer.create(0)
    yield r
    r.close()


def u32(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy().view(np.uint32)


def proj_of(eye, w, h, target=(0, 0, 0), orthographic=False):
    return L.projection_for(H.camera(eye, target, orthographic=orthographic), w, h)


def assert_build_matches(lod: L.LodCloud, o: ora.OracleLod):
    info, oi = lod.info, o.info
    for f in ("count", "rest_per_colour", "sh_words", "levels", "coarsest", "finest", "merged"):
        assert getattr(info, f) == getattr(oi, f), f
    assert list(info.bounds_lo) == list(oi.bounds_lo) and list(info.bounds_hi) == list(oi.bounds_hi)
    assert np.float32(info.extent) == np.float32(oi.extent)
    assert list(info.level_groups[:info.levels]) == o.level_groups
    store, ostore = lod.splats, o.store
    assert np.array_equal(u32(lod.codes), o.codes)
    assert np.array_equal(store.positions.cpu().numpy(), ostore.positions)
    assert np.array_equal(u32(store.shape), ostore.shape)
    assert np.array_equal(u32(store.sh), ostore.sh)
    assert np.array_equal(u32(lod.starts), o.starts)
    merged = o.merged
    cells = o.cells
    at = 0
    for k, level in enumerate(lod.levels):
        g = level.gaussians.count
        assert level.level == oi.coarsest + k
        assert np.array_equal(u32(level.cells), cells[at:at + g])
        assert np.array_equal(level.gaussians.positions.cpu().numpy(), merged.positions[at:at + g]), k
        assert np.array_equal(u32(level.gaussians.shape), merged.shape[at:at + g]), k
        assert np.array_equal(u32(level.gaussians.sh), merged.sh[at:at + g]), k
        at += g


def cut_arrays(inst: L.SplatInstance):
    s = inst.splats
    return s.positions.cpu().numpy(), u32(s.shape), u32(s.sh)


CLOUDS = [
    ("random5000", lambda: ora.random_cloud(5000, 41), 3, 3, {}),
    ("dense60000", lambda: ora.random_cloud(60000, 43, 0.003, 0.05), 3, 3, {}),
    ("degree0", lambda: ora.random_cloud(20000, 5), 3, 0, {}),
    ("coarsest3", lambda: ora.random_cloud(20000, 6), 3, 3, dict(coarsest_level=3)),
    ("fraction1", lambda: H.single_splat_cells_records(), 3, 3, dict(max_group_fraction=1.0)),
    ("bounds", lambda: ora.random_cloud(8000, 7), 3, 3, dict(bounds=(-3, -2, -3, 3, 2, 3))),
]


@pytest.mark.parametrize("name,make,file_rest,degree,kw", CLOUDS, ids=[c[0] for c in CLOUDS])
def test_the_build_equals_the_oracle(raster, name, make, file_rest, degree, kw):
    packed = H.packed_from_raw(make(), file_rest, degree)
    builder = L.LodBuilder.create(raster)
    settings = L.LodBuildSettings(max_group_fraction=kw.get("max_group_fraction", 0.5),
                                  coarsest_level=kw.get("coarsest_level", 1))
    lod = builder.build(L.to_device(packed), settings, bounds=kw.get("bounds"))
    o = ora.lod_build(H.host_cloud(packed), bounds=kw.get("bounds"), max_group_fraction=settings.max_group_fraction,
                      coarsest_level=settings.coarsest_level)
    assert_build_matches(lod, o)


def test_a_degree_three_cloud_builds_like_the_oracle(raster):
    rng = np.random.default_rng(3)
    records = ora.random_cloud(30000, 9)
    # Degree 3 records: the degree-1 fixture with 36 more rest coefficients.
    full = np.zeros((records.shape[0], 14 + 45), np.float32)
    full[:, :14] = records[:, :14]
    full[:, 14:] = rng.uniform(-0.3, 0.3, (records.shape[0], 45)).astype(np.float32)
    packed = H.packed_from_raw(full, 15, 3)
    assert packed.rest_per_colour == 15
    lod = L.LodBuilder.create(raster).build(L.to_device(packed))
    assert_build_matches(lod, ora.lod_build(H.host_cloud(packed)))


CUTS = [((1.5, 1.0, 6.0), False), ((0.3, 0.2, 0.4), False), ((6.0, 4.0, 30.0), False), ((1.5, 1.0, 6.0), True)]


@pytest.mark.parametrize("threshold", [0.0, 0.5, 1.0, 2.0, 4.0, 1e6])
@pytest.mark.parametrize("eye,orthographic", CUTS)
def test_the_cut_equals_the_oracle(raster, threshold, eye, orthographic):
    packed = H.packed_from_raw(ora.random_cloud(20000, 41), 3, 3)
    lod = L.LodBuilder.create(raster).build(L.to_device(packed))
    o = ora.lod_build(H.host_cloud(packed))
    pr = proj_of(eye, 200, 150, orthographic=orthographic)
    for m in (np.eye(4), H.translation((0.5, -0.25, 1.0)) @ H.scaling((1.5, 1.5, 1.5))):
        stats = []
        out = L.CutSelector.create(raster).select(pr, [L.LodInstance(lod, m)], threshold, stats)
        ocut, osplats, omerged = o.cut(pr.struct(), m, threshold)
        assert (stats[0].splats, stats[0].merged, stats[0].available) == (osplats, omerged, packed.count)
        assert len(out) == (1 if osplats + omerged else 0)
        if out:
            pos, shape, sh = cut_arrays(out[0])
            assert np.array_equal(pos, ocut.positions) and np.array_equal(shape, ocut.shape)
            assert np.array_equal(sh, ocut.sh)
            assert np.array_equal(out[0].object_to_world, m)


def test_several_instances_each_get_their_own_cut(raster):
    a = H.packed_from_raw(ora.random_cloud(12000, 1), 3, 3)
    b = H.packed_from_raw(ora.random_cloud(7000, 2), 3, 0)
    builder = L.LodBuilder.create(raster)
    la, lb = builder.build(L.to_device(a)), builder.build(L.to_device(b))
    oa, ob = ora.lod_build(H.host_cloud(a)), ora.lod_build(H.host_cloud(b))
    pr = proj_of((2.0, 1.0, 9.0), 240, 180)
    ma, mb = np.eye(4), H.translation((3.0, 0.0, 0.0)) @ H.rotation_y(30)
    instances = [L.LodInstance(la, ma), L.LodInstance(None), L.LodInstance(lb, mb, threshold=3.0),
                 L.LodInstance(la, mb, threshold=0.0)]
    stats = []
    out = L.CutSelector.create(raster).select(pr, instances, 1.5, stats)
    expect = [oa.cut(pr.struct(), ma, 1.5), None, ob.cut(pr.struct(), mb, 3.0), oa.cut(pr.struct(), mb, 0.0)]
    assert len(stats) == 4 and (stats[1].splats, stats[1].merged, stats[1].available) == (0, 0, 0)
    got = iter(out)
    for s, e in zip(stats, expect):
        if e is None:
            continue
        cut, splats, merged = e
        assert (s.splats, s.merged) == (splats, merged)
        pos, shape, sh = cut_arrays(next(got))
        assert np.array_equal(pos, cut.positions) and np.array_equal(shape, cut.shape) and np.array_equal(sh, cut.sh)


def _gpu_compare(raster, pr, settings, full: L.GpuSplats, instances):
    ta, tb = L.RenderTargets(), L.RenderTargets()
    raster.render(pr, [L.SplatInstance(full)], settings, ta)
    raster.render(pr, instances, settings, tb)
    return raster.compare_images(ta.colour, tb.colour)[0]


def test_threshold_zero_draws_the_cloud_as_it_is_on_the_device(raster):
    """tests/lod/test_lod.cpp:82-106 on the device."""
    packed = H.packed_from_raw(ora.random_cloud(5000, 41), 3, 3)
    cloud = L.to_device(packed)
    lod = L.LodBuilder.create(raster).build(cloud)
    assert lod.levels
    pr = proj_of((1.5, 1.0, 6.0), 200, 150)
    stats = []
    out = L.CutSelector.create(raster).select(pr, [L.LodInstance(lod)], 0.0, stats)
    assert (stats[0].splats, stats[0].merged) == (cloud.count, 0)
    d = _gpu_compare(raster, pr, H.settings(200, 150), cloud, out)
    assert d.p99 <= 1 and d.over2 * 100 <= d.pixels


def test_a_cell_holding_one_splat_merges_into_that_splat_on_the_device(raster):
    """tests/lod/test_lod.cpp:108-152 on the device."""
    packed = H.packed_from_raw(H.single_splat_cells_records(), 3, 3)
    cloud = L.to_device(packed)
    lod = L.LodBuilder.create(raster).build(cloud, L.LodBuildSettings(max_group_fraction=1.0, coarsest_level=1))
    assert lod.levels[0].gaussians.count == 6
    pr = proj_of((3.0, 2.0, 12.0), 200, 150)
    stats = []
    out = L.CutSelector.create(raster).select(pr, [L.LodInstance(lod)], 1e6, stats)
    assert (stats[0].splats, stats[0].merged) == (0, 6)
    d = _gpu_compare(raster, pr, H.settings(200, 150), cloud, out)
    assert d.p99 <= 1 and d.over2 * 100 <= d.pixels


def test_far_away_a_dense_cloud_draws_a_fraction_on_the_device(raster):
    """tests/lod/test_lod.cpp:154-189 on the device, with its bounds."""
    packed = H.packed_from_raw(ora.random_cloud(60000, 43, 0.003, 0.05), 3, 3)
    cloud = L.to_device(packed)
    lod = L.LodBuilder.create(raster).build(cloud)
    pr = proj_of((6.0, 4.0, 30.0), 240, 180)
    selector = L.CutSelector.create(raster)
    for threshold in (1.0, 2.0, 4.0):
        stats = []
        out = selector.select(pr, [L.LodInstance(lod)], threshold, stats)
        d = _gpu_compare(raster, pr, H.settings(240, 180), cloud, out)
        drawn = stats[0].splats + stats[0].merged
        assert stats[0].available == cloud.count
        if threshold == 1.0:
            assert d.p99 <= 1, d
        elif threshold == 2.0:
            assert drawn < cloud.count * 3 // 4 and d.p99 <= 12, (drawn, d)
        else:
            assert drawn < cloud.count // 4 and d.p99 <= 36, (drawn, d)


def test_a_million_splats_keep_the_cut_invariants(raster):
    """At full size: the build equals the oracle, codes are sorted, threshold 0
    draws the store, a huge threshold the coarsest level, and in between each
    splat is drawn once (drawn count = the restated rule's count)."""
    scene = H.synthetic_scene(1_000_000, 1920, 1080, seed=11)
    packed = scene.clouds[0][0]
    cloud = L.to_device(packed)
    lod = L.LodBuilder.create(raster).build(cloud)
    o = ora.lod_build(H.host_cloud(packed))
    assert_build_matches(lod, o)
    codes = u32(lod.codes).astype(np.int64)
    assert np.all(np.diff(codes) >= 0)
    # From about 30 units the finest cells span 9 to 12 pixels across the
    # cloud's depth: thresholds 10, 11 and 20 mix splats and several levels.
    pr = L.projection_for(H.camera((6.0, 4.0, 30.0)), 1920, 1080)
    selector = L.CutSelector.create(raster)
    for threshold in (0.0, 10.0, 11.0, 20.0, 40.0, 1e6):
        stats = []
        out = selector.select(pr, [L.LodInstance(lod)], threshold, stats)
        ocut, osplats, omerged = o.cut(pr.struct(), np.eye(4), threshold)
        assert (stats[0].splats, stats[0].merged) == (osplats, omerged), threshold
        pos, shape, sh = cut_arrays(out[0])
        assert np.array_equal(pos, ocut.positions) and np.array_equal(shape, ocut.shape), threshold
        assert np.array_equal(sh, ocut.sh), threshold
        if threshold == 0.0:
            assert osplats == packed.count and np.array_equal(pos, lod.splats.positions.cpu().numpy())
        if threshold == 1e6:
            assert (osplats, omerged) == (0, o.level_groups[0])


def test_bad_clouds_are_refused(raster):
    builder = L.LodBuilder.create(raster)
    empty = L.to_device(H.packed_from_raw(ora.random_cloud(10, 1)[:0], 3, 3))
    with pytest.raises(L.LrtError) as e:
        builder.build(empty)
    assert e.value.code == 3
