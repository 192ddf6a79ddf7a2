"""Raw splat records in several encodings (io::SplatEncoding modes), seeded,
with invalid records mixed in: the inputs of the decode parity tests."""
from __future__ import annotations

import numpy as np

import lucabrtrender_b200 as L
from lucabrtrender_b200 import _abi

ENCODINGS = ["ply", "linear", "bytes", "spz_first_three", "spz_smallest_three", "light"]


def encoding(kind: str, rest: int = 15) -> _abi.SplatEncoding:
    e = L.ply_encoding(rest)
    if kind == "linear":
        e.opacity_mode, e.scale_mode, e.colour_mode = 1, 1, 1
    elif kind == "bytes":
        e.opacity_mode, e.colour_mode, e.rotation_mode, e.rest_mode = 2, 2, 1, 1
    elif kind == "spz_first_three":
        # SPZ-like: fixed-point positions, byte log scales, byte DC, first-three
        # rotation, rgb-per-basis byte harmonics, right-up-back axes.
        e.position_scale = 1.0 / 4096.0
        e.opacity_mode, e.scale_mode, e.colour_mode, e.rotation_mode, e.rest_mode = 2, 2, 3, 2, 1
        e.rest_colour_outer = 0
        e.flip_yz = 1
    elif kind == "spz_smallest_three":
        e.position_scale = 1.0 / 4096.0
        e.opacity_mode, e.scale_mode, e.colour_mode, e.rotation_mode, e.rest_mode = 2, 2, 3, 3, 1
        e.rest_colour_outer = 0
        e.flip_yz = 1
    elif kind == "light":
        e.colour_mode = 4
    return e


def records(kind: str, count: int, seed: int, rest: int = 15) -> np.ndarray:
    rng = np.random.default_rng(seed)
    fpr = 14 + 3 * rest
    r = rng.standard_normal((count, fpr)).astype(np.float32)
    byte = lambda shape: rng.integers(0, 256, shape).astype(np.float32)  # noqa: E731
    if kind == "linear":
        r[:, 3] = rng.uniform(0.0, 1.0, count)
        r[:, 4:7] = rng.uniform(0.001, 0.3, (count, 3))
        r[:, 11:14] = rng.uniform(0.0, 1.2, (count, 3))
    elif kind == "bytes":
        r[:, 3] = byte(count)
        r[:, 4:7] = rng.normal(-4.0, 1.0, (count, 3))
        r[:, 7:11] = byte((count, 4))
        r[:, 11:14] = byte((count, 3))
        r[:, 14:] = byte((count, fpr - 14))
    elif kind.startswith("spz"):
        r[:, 0:3] = rng.integers(-40000, 40000, (count, 3)).astype(np.float32)
        r[:, 3] = byte(count)
        r[:, 4:7] = byte((count, 3))
        r[:, 11:14] = byte((count, 3))
        r[:, 14:] = byte((count, fpr - 14))
        if kind == "spz_first_three":
            r[:, 7:11] = byte((count, 4))
        else:
            comp = rng.integers(0, 2**32, count, dtype=np.uint64)
            r[:, 8] = (comp & 0xFFFF).astype(np.float32)
            r[:, 9] = (comp >> 16).astype(np.float32)
    elif kind == "light":
        r[:, 11:14] = rng.uniform(-0.1, 1.5, (count, 3))
    # invalid records: non-finite position, huge scale, faint opacity
    bad = rng.choice(count, size=max(1, count // 50), replace=False)
    r[bad[0::3], 1] = np.nan
    r[bad[1::3], 5] = 1e9 if kind in ("linear",) else 200.0
    r[bad[2::3], 3] = -30.0 if kind in ("ply", "light") else 0.0
    return r
