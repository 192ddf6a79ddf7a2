"""The restated levels of detail, on the CPU.

Pinned two ways: (1) against an independent numpy restatement of what the
build must produce -- Morton codes from the positions (morton.slang), the
stable order, each stored level's groups as the distinct top-3r-bit prefixes
of the codes, the finest level by the reference's fraction rule (Lod.cpp:
200-211) -- and of the cut's rule (lod_cut.slang), which must draw every
place exactly once; (2) by the reference's own LOD tests
(tests/lod/test_lod.cpp:82-189), restated over the oracle's renderer and
compareImages with the reference's bounds."""
from __future__ import annotations

import numpy as np
import pytest

import lucabrtrender_b200 as L

import helpers as H
import oracle as ora


def proj_of(eye, w, h, target=(0, 0, 0)):
    return L.projection_for(L.Camera.looking_at(eye, target), w, h).struct()


def cloud_of(count, seed, *size):
    return H.host_cloud(H.packed_from_raw(ora.random_cloud(count, seed, *size), 3, 3))


@pytest.fixture(scope="module")
def cloud5000():
    return cloud_of(5000, 41)


def test_the_build_sorts_by_morton_code_and_groups_by_prefix(cloud5000):
    c = cloud5000
    lod = ora.lod_build(c)
    info = lod.info
    lo = c.positions[:, :3].min(axis=0)
    hi = c.positions[:, :3].max(axis=0)
    assert np.array_equal(np.array(info.bounds_lo[:], np.float32), lo)
    assert np.array_equal(np.array(info.bounds_hi[:], np.float32), hi)
    extent = np.float32(max(np.float32(max((hi - lo).max(), 0)), np.float32(1e-6))) * np.float32(1.0001)
    assert np.float32(info.extent) == extent
    codes = H.morton_codes(c.positions, lo, extent)
    order = np.argsort(codes, kind="stable")
    assert np.array_equal(lod.codes, codes[order])
    store = lod.store
    assert np.array_equal(store.positions, c.positions[order])
    assert np.array_equal(store.shape, c.shape[order])
    assert np.array_equal(store.sh, c.sh[order])
    # Levels: consecutive, coarsest 1, finest by the fraction rule.
    sorted_codes = codes[order]
    counts = {r: len(np.unique(sorted_codes >> np.uint32(3 * (10 - r)))) for r in range(1, 11)}
    assert info.coarsest == 1
    finest = info.finest
    assert info.levels == finest - info.coarsest + 1
    for r in range(2, finest + 1):
        assert counts[r] <= 0.5 * c.count
    if finest < 10:
        assert counts[finest + 1] > 0.5 * c.count
    assert lod.level_groups == [counts[r] for r in range(1, finest + 1)]
    assert info.merged == sum(lod.level_groups)
    cells = lod.cells
    at = 0
    for r, g in zip(range(1, finest + 1), lod.level_groups):
        prefix = sorted_codes >> np.uint32(3 * (10 - r))
        first = np.concatenate([[True], prefix[1:] != prefix[:-1]])
        assert np.array_equal(cells[at:at + g], prefix[first])
        if r == finest:
            assert np.array_equal(lod.starts, np.nonzero(first)[0].astype(np.uint32))
        at += g


def test_threshold_zero_draws_the_store_and_nothing_merged(cloud5000):
    lod = ora.lod_build(cloud5000)
    cut, splats, merged = lod.cut(proj_of((1.5, 1.0, 6.0), 200, 150), threshold=0.0)
    assert (splats, merged) == (cloud5000.count, 0)
    store = lod.store
    for a, b in ((cut.positions, store.positions), (cut.shape, store.shape), (cut.sh, store.sh)):
        assert np.array_equal(a, b)


def test_a_threshold_every_cell_meets_draws_the_coarsest_level(cloud5000):
    lod = ora.lod_build(cloud5000)
    cut, splats, merged = lod.cut(proj_of((1.5, 1.0, 6.0), 200, 150), threshold=1e6)
    g0 = lod.level_groups[0]
    assert (splats, merged) == (0, g0)
    m = lod.merged
    assert np.array_equal(cut.positions, m.positions[:g0]) and np.array_equal(cut.shape, m.shape[:g0])


@pytest.mark.parametrize("threshold", [0.5, 1.0, 2.0, 4.0, 16.0])
@pytest.mark.parametrize("eye,orthographic", [((1.5, 1.0, 6.0), False), ((0.3, 0.2, 0.4), False),
                                              ((6.0, 4.0, 30.0), False), ((1.5, 1.0, 6.0), True)])
def test_every_place_is_drawn_exactly_once(cloud5000, threshold, eye, orthographic):
    """lod_cut.slang's rule restated in numpy float32: the drawn groups and
    splats match the oracle's counts, and together they hold every splat once."""
    lod = ora.lod_build(cloud5000)
    info = lod.info
    cam = H.camera(eye, orthographic=orthographic)
    pr = L.projection_for(cam, 200, 150).struct()
    lo = np.array(info.bounds_lo[:], np.float32)
    ppu = np.float32(pr.focal_x)
    codes = lod.codes
    cells = lod.cells
    eye_f = np.array(pr.eye_world[:], np.float64).astype(np.float32)
    small = {}
    covered = 0
    merged = 0
    at = 0
    for k, g in enumerate(lod.level_groups):
        r = info.coarsest + k
        c = cells[at:at + g]
        here = (threshold > 0) & (H.projected_edge(c, r, lo, info.extent, eye_f, ppu, orthographic) <= threshold)
        above = np.zeros(g, bool) if k == 0 else small[r - 1][np.searchsorted(small_cells[r - 1], c >> np.uint32(3))]
        drawn = here & ~above
        prefix = codes >> np.uint32(3 * (10 - r))
        sizes = np.diff(np.concatenate([np.nonzero(np.concatenate([[True], prefix[1:] != prefix[:-1]]))[0],
                                        [len(codes)]]))
        covered += int(sizes[drawn].sum())
        merged += int(drawn.sum())
        small[r] = here
        small_cells = {**(small_cells if k else {}), r: c}
        at += g
    finest = info.finest
    splat_small = small[finest][np.searchsorted(small_cells[finest], codes >> np.uint32(3 * (10 - finest)))]
    covered += int((~splat_small).sum())
    _, n_splats, n_merged = lod.cut(pr, threshold=threshold)
    assert (n_splats, n_merged) == (int((~splat_small).sum()), merged)
    assert covered == cloud5000.count


def _compare(pr, settings, a_cloud, b_cloud, a_m=None, b_m=None):
    m = np.eye(4)
    a = ora.render(pr, [(a_cloud, m if a_m is None else a_m, None)], settings.struct(), want_pairs=False)
    b = ora.render(pr, [(b_cloud, m if b_m is None else b_m, None)], settings.struct(), want_pairs=False)
    return ora.compare_images(a["colour"], b["colour"])


def test_a_cut_with_threshold_zero_draws_the_cloud_as_it_is(cloud5000):
    """tests/lod/test_lod.cpp:82-106: not bit-identical (Morton order changes
    which of two tying depth keys goes first), p99 <= 1 and at most 1% of
    pixels over 2 code values."""
    lod = ora.lod_build(cloud5000)
    pr = proj_of((1.5, 1.0, 6.0), 200, 150)
    cut, splats, merged = lod.cut(pr, threshold=0.0)
    assert (splats, merged) == (cloud5000.count, 0)
    d = _compare(pr, H.settings(200, 150), cloud5000, cut)
    assert d.p99 <= 1 and d.over2 * 100 <= d.pixels


def test_a_cell_holding_one_splat_merges_into_that_splat():
    """tests/lod/test_lod.cpp:108-152: six splats, one to a level-1 cell; kept
    from level 1 though nothing merges; a threshold every cell meets draws the
    six merged Gaussians, each its splat again (covariance to the f16 log
    scales and the 10-bit quaternion), and the render agrees."""
    raw = H.single_splat_cells_records()
    cloud = H.host_cloud(H.packed_from_raw(raw, 3, 3))
    assert cloud.count == 6
    lod = ora.lod_build(cloud, coarsest_level=1, max_group_fraction=1.0)
    assert lod.level_groups[0] == 6
    pr = proj_of((3.0, 2.0, 12.0), 200, 150)
    cut, splats, merged = lod.cut(pr, threshold=1e6)
    assert (splats, merged) == (0, 6)
    store = lod.store

    def covariance(cl):
        """Sigma = R S^2 R^T from the packed words (packing.slang:52-69)."""
        out = []
        for i in range(cl.count):
            w = int(cl.shape[i, 0])
            small = [((w >> s) & 1023) / 1023.0 * 2.0 - 1.0 for s in (22, 12, 2)]
            small = [v * 0.70710678 for v in small]
            rest = np.sqrt(max(0.0, 1.0 - sum(v * v for v in small)))
            q, it = [], iter(small)
            for k in range(4):
                q.append(rest if k == (w & 3) else next(it))
            x, y, z, qw = q
            r = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - qw * z), 2 * (x * z + qw * y)],
                          [2 * (x * y + qw * z), 1 - 2 * (x * x + z * z), 2 * (y * z - qw * x)],
                          [2 * (x * z - qw * y), 2 * (y * z + qw * x), 1 - 2 * (x * x + y * y)]])
            halves = cl.shape[i, 1:3].astype(np.uint32).view(np.uint16).view(np.float16).astype(np.float64)
            sc = np.exp(halves[:3])
            out.append(r @ np.diag(sc * sc) @ r.T)
        return np.stack(out)

    a, b = covariance(store), covariance(cut)
    for i in range(6):
        assert np.abs(a[i] - b[i]).max() <= 3e-3 * np.abs(a[i]).max(), (i, a[i], b[i])
    # The base colours and rest coefficients survive to f16 rounding.
    hs = store.shape[:, 2:4].astype(np.uint32).view(np.uint16).view(np.float16).astype(np.float64)[:, 1:]
    hc = cut.shape[:, 2:4].astype(np.uint32).view(np.uint16).view(np.float16).astype(np.float64)[:, 1:]
    assert np.allclose(hs, hc, rtol=2e-3, atol=1e-3)
    rs = store.sh.astype(np.uint32).view(np.uint16).view(np.float16).astype(np.float64)[:, :9]
    rc = cut.sh.astype(np.uint32).view(np.uint16).view(np.float16).astype(np.float64)[:, :9]
    assert np.allclose(rs, rc, rtol=2e-3, atol=1e-3)
    # Same centres (to rounding), opacities and colours.
    assert np.allclose(cut.positions[:, :3], store.positions[:, :3], rtol=1e-6, atol=1e-6)
    assert np.allclose(cut.positions[:, 3], store.positions[:, 3], rtol=2e-3)
    d = _compare(pr, H.settings(200, 150), cloud, cut)
    assert d.p99 <= 1 and d.over2 * 100 <= d.pixels


def test_far_away_a_dense_cloud_draws_a_fraction_of_its_splats_and_looks_the_same():
    """tests/lod/test_lod.cpp:154-189 with its bounds: p99 <= 1 at 1 px; at
    2 px under 3/4 of the splats drawn and p99 <= 12; at 4 px under 1/4 and
    p99 <= 36."""
    cloud = cloud_of(60000, 43, 0.003, 0.05)
    lod = ora.lod_build(cloud)
    pr = proj_of((6.0, 4.0, 30.0), 240, 180)
    for threshold in (1.0, 2.0, 4.0):
        cut, splats, merged = lod.cut(pr, threshold=threshold)
        d = _compare(pr, H.settings(240, 180), cloud, cut)
        drawn = splats + merged
        if threshold == 1.0:
            assert d.p99 <= 1, d
        elif threshold == 2.0:
            assert drawn < cloud.count * 3 // 4 and d.p99 <= 12, (drawn, d)
        else:
            assert drawn < cloud.count // 4 and d.p99 <= 36, (drawn, d)


def test_bounds_given_by_the_caller_replace_the_positions_own(cloud5000):
    lod = ora.lod_build(cloud5000, bounds=(-4, -4, -4, 4, 4, 4))
    assert list(lod.info.bounds_lo) == [-4, -4, -4] and np.float32(lod.info.extent) == np.float32(8) * np.float32(1.0001)
    codes = H.morton_codes(cloud5000.positions, (-4, -4, -4), np.float32(8) * np.float32(1.0001))
    assert np.array_equal(lod.codes, np.sort(codes, kind="stable"))


def test_coarsest_level_and_fraction_settings(cloud5000):
    lod = ora.lod_build(cloud5000, coarsest_level=3, max_group_fraction=0.5)
    assert lod.info.coarsest == 3 and lod.level_groups[0] == 384
    lod = ora.lod_build(cloud5000, coarsest_level=1, max_group_fraction=0.005)
    # Level 2's 48 groups already pass 0.5% of the splats: only the coarsest is kept.
    assert lod.info.finest == 1 and lod.level_groups == [8]
