"""The reference's own splat fixtures (tests/data/splats/tiny.ply, 64 splats
of degree 0, and sh3.ply, 64 splats of degree 3, in the lucabRTrender tree),
as raw records stored in tests/golden/splat_fixtures.json by
tests/golden/make_splat_fixtures.py, and the frame the reference's SOG test
draws of them (tests/render/test_sog.cpp:41-66): 240x180, the camera at the
cloud's bounds centre + (0.3, 0.2, 1.6) x its largest extent, looking at the
centre, 30 mm lens."""
from __future__ import annotations

import base64
import json
from pathlib import Path

import numpy as np

import lucabrtrender_b200 as L

GOLDEN = Path(__file__).resolve().parent / "golden" / "splat_fixtures.json"


def raw_records(name: str) -> tuple[np.ndarray, int]:
    d = json.loads(GOLDEN.read_text())[name]
    recs = np.frombuffer(base64.b64decode(d["records_f32_base64"]), np.float32)
    return recs.reshape(d["count"], d["floats_per_record"]).copy(), d["rest_per_colour"]


def sog_test_camera(positions: np.ndarray) -> L.Camera:
    lo = positions[:, :3].min(axis=0).astype(np.float64)
    hi = positions[:, :3].max(axis=0).astype(np.float64)
    centre = (lo + hi) * 0.5
    extent = float(max(hi - lo))
    cam = L.Camera.looking_at(tuple(centre + np.array([0.3, 0.2, 1.6]) * extent), tuple(centre))
    cam.lens.focal = 30.0
    return cam
