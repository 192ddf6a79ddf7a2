"""The Mip-Splatting 3D filter (Yu et al., CVPR 2024, section 4.1) in the
oracle, against a float64 numpy statement of the same method: per splat the
highest sampling rate focal / z over the cameras that see it (in front of
the near plane, projected inside the image widened by 15% a side), variance
coefficient / rate^2, unseen splats at the lowest seen rate. Also: the
filtered splat keeps its rotation, its scales become sqrt(s^2 + v) and its
opacity sqrt(prod s^2 / prod(s^2 + v)) of the original, which the oracle's
rendered records show."""
from __future__ import annotations

import math

import numpy as np

import bench_workload as W
import oracle as ora


def _views(count=12, seed=3, w=320, h=240):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        r = rng.uniform(2.5, 6.0)
        out.append((W.square_pixel_projection(tuple(d * r), (0.0, 0.0, 0.0), w, h), w, h))
    return out


def _numpy_filter(positions, views, coefficient):
    p = positions[:, :3].astype(np.float64)
    best = np.zeros(len(p))
    for pr, w, h in views:
        m = np.asarray(pr.world_to_view[:], np.float64).reshape(4, 4)
        t = p @ m[:3, :3].T + m[:3, 3]
        z = t[:, 2]
        ok = z > pr.near_z
        zz = np.where(ok, z, 1.0)
        sx = pr.focal_x * t[:, 0] / zz + pr.centre_x
        sy = pr.focal_y * t[:, 1] / zz + pr.centre_y
        ok &= (sx >= -0.15 * w) & (sx <= 1.15 * w) & (sy >= -0.15 * h) & (sy <= 1.15 * h)
        rate = np.where(ok, pr.focal_x / zz, 0.0)
        best = np.maximum(best, rate)
    seen = best > 0
    if seen.any():
        best[~seen] = best[seen].min()
        return coefficient / best ** 2
    return np.zeros(len(p))


def test_filter_variance_matches_the_method():
    cloud = W.packed_cloud(20_000, 2)
    views = _views()
    got = ora.filter3d(cloud, views, 0.2)
    want = _numpy_filter(cloud.positions, views, 0.2)
    # the float32 restatement against float64: a few ulps, except splats at
    # the very edge of a camera's band, where the two may decide differently
    close = np.abs(got - want) <= 1e-5 * want
    assert close.mean() > 0.999, close.mean()
    assert np.all(got > 0)


def test_no_camera_sees_anything_gives_no_filter():
    cloud = W.packed_cloud(1000, 4)
    behind = [(W.square_pixel_projection((0.0, 0.0, -50.0), (0.0, 0.0, -100.0), 64, 64), 64, 64)]
    assert np.all(ora.filter3d(cloud, behind, 0.2) == 0.0)


def test_filtered_records_widen_and_pay_the_energy_back():
    cloud = W.packed_cloud(3000, 5)
    views = _views(8, 6, 256, 256)
    pr, w, h = views[0]
    st = W.settings(w, h)
    plain = ora.render(pr, [(cloud, np.eye(4), None)], st, 0, want_pairs=False)
    var = ora.filter3d(cloud, views, 0.2)
    filtered_cloud = ora.HostCloud(cloud.positions, cloud.shape, cloud.sh, cloud.rest_per_colour, var * 50.0)
    filt = ora.render(pr, [(filtered_cloud, np.eye(4), None)], st, 0, want_pairs=False)
    both = (plain["touched"] > 0) & (filt["touched"] > 0)
    assert both.sum() > 100
    # wider footprints (the conic shrinks: its determinant drops) and lower peak opacity
    det = lambda r: r[:, 4] * r[:, 6] - r[:, 5] ** 2  # noqa: E731
    assert np.all(det(filt["proj"][both]) < det(plain["proj"][both]))
    assert np.all(filt["proj"][both, 7] < plain["proj"][both, 7])
