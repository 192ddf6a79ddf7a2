"""The benchmark's CPU legs build their inputs with the oracle alone
(oracle/bench_workload.py), so that the reference arm never loads the
package's library. These checks hold those inputs equal, bit for bit, to the
ones the GPU arm builds through the package: the seeded records, the packed
cloud of the headline workload, and the orbit's twenty projections."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

import lucabrtrender_b200 as L

import bench_workload as W
import oracle as ora


def _bytes(struct) -> bytes:
    return C.string_at(C.addressof(struct), C.sizeof(struct))


def test_records_are_the_packages_records():
    for count, seed, dist in ((20_000, 1, {}), (5_000, 3, dict(mean_sigma=2.0, log_scale_mean=-3.5,
                                                               log_scale_sigma=0.7))):
        assert np.array_equal(W.synthetic_records(count, seed, **dist), L.synthetic_records(count, seed, **dist))


def test_the_headline_cloud_packs_to_the_same_bytes():
    ours = W.packed_cloud(1_000_000, 1)
    theirs = L.pack_splats(L.synthetic_records(1_000_000, 1), 15, 3)
    assert ours.rest_per_colour == theirs.rest_per_colour == 15
    assert np.array_equal(ours.positions.view(np.uint32), theirs.positions.view(np.uint32))
    assert np.array_equal(ours.shape, theirs.shape)
    assert np.array_equal(ours.sh, theirs.sh)


def test_orbit_projections_are_the_packages_projections():
    for k in range(20):
        th = 2.0 * math.pi * k / 20
        cam = L.square_pixel_camera((4.0 * math.sin(th), 0.0, 4.0 * math.cos(th)), (0.0, 0.0, 0.0), 1920, 1080,
                                    60.0, 0.01)
        theirs = L.projection_for(cam, 1920, 1080).struct()
        ours = W.orbit_projection(k, 20, 4.0, 1920, 1080)
        assert _bytes(ours) == _bytes(theirs), k


def test_default_settings_are_the_packages_defaults():
    assert _bytes(W.settings(1920, 1080)) == _bytes(L.RenderSettings(width=1920, height=1080).struct())


def test_the_oracle_imports_nothing_from_the_package():
    import sys
    import subprocess
    code = ("import sys; sys.path[:0] = ['oracle']; import bench_workload as W, oracle as ora; "
            "W.orbit_projection(0, 20, 4.0, 64, 64); W.packed_cloud(100, 1); "
            "assert not [m for m in sys.modules if m.startswith('lucabrtrender_b200')], sys.modules.keys(); "
            "import os; maps = open('/proc/self/maps').read(); assert 'liblrt_raster' not in maps")
    from pathlib import Path
    subprocess.run([sys.executable, "-c", code], check=True, cwd=Path(__file__).resolve().parents[1])
