"""Shared set-up of the training-path tests: seeded differentiable parameters,
a camera, and the oracle's view of the same frame."""
from __future__ import annotations

import numpy as np

import lucabrtrender_b200 as L

import oracle as ora


def make_params(n: int, seed: int, spread: float = 0.8, log_scale_mean: float = -3.2, log_scale_sigma: float = 0.4):
    """fp32 parameters; the SH values are fp16-representable (what the kernels read)."""
    rng = np.random.default_rng(seed)
    means = (rng.standard_normal((n, 3)) * spread).astype(np.float32)
    log_scales = (rng.standard_normal((n, 3)) * log_scale_sigma + log_scale_mean).astype(np.float32)
    quats = rng.standard_normal((n, 4)).astype(np.float32)
    logits = rng.standard_normal(n).astype(np.float32)
    sh = np.zeros((n, 16, 3), np.float32)
    sh[:, 0, :] = rng.standard_normal((n, 3)) * 0.5
    sh[:, 1:, :] = rng.standard_normal((n, 15, 3)) * 0.05
    sh = sh.astype(np.float16).astype(np.float32)
    return dict(means=means, log_scales=log_scales, quats=quats, logits=logits, sh=sh)


def raw_cloud(p) -> ora.RawCloud:
    return ora.RawCloud(np.ascontiguousarray(p["means"]), np.ascontiguousarray(p["log_scales"]),
                        np.ascontiguousarray(p["quats"]), np.ascontiguousarray(p["logits"]),
                        np.ascontiguousarray(p["sh"].astype(np.float16)))


def raw_records(p) -> np.ndarray:
    """The same splats as 3DGS records, for the packed (quantised) path."""
    n = p["means"].shape[0]
    r = np.zeros((n, 14 + 45), np.float32)
    r[:, 0:3] = p["means"]
    r[:, 3] = p["logits"]
    r[:, 4:7] = p["log_scales"]
    r[:, 7:11] = p["quats"]                 # w x y z
    r[:, 11:14] = p["sh"][:, 0, :]          # DC
    for colour in range(3):
        r[:, 14 + colour * 15:14 + (colour + 1) * 15] = p["sh"][:, 1:, colour]
    return r


def frame(width=128, height=128, eye=(0.0, 0.0, 4.0)):
    cam = L.square_pixel_camera(eye, (0.0, 0.0, 0.0), width, height, 60.0, 0.01)
    settings = L.RenderSettings(width=width, height=height)
    return cam, settings
