"""The FP64 gradient oracle checked against itself on the CPU: its autograd
gradients equal central finite differences (h = 1e-4) of its own FP64 loss,
with the frame's discrete choices (from the fp32 oracle) held fixed."""
from __future__ import annotations

import numpy as np
import pytest

import lucabrtrender_b200 as L

import grad_oracle as G
import oracle as ora
import train_fixtures as TF


def test_fp64_autograd_equals_finite_differences():
    p = TF.make_params(3000, 5)
    cam, settings = TF.frame(96, 96)
    pr = L.projection_for(cam, 96, 96).struct()
    st = settings.struct()
    crop = (16, 16, 64, 64)
    out = ora.train_render(pr, TF.raw_cloud(p), st, crop)
    assert len(out["list_slots"]) > 1000
    rng = np.random.default_rng(1)
    target = rng.uniform(0, 1, (64, 64, 3))
    prob = G.CropProblem(G.camera_from(pr, st), crop, out["list_offsets"], out["list_slots"], target)
    grads, _ = G.gradients(prob, p)
    names = ["means", "log_scales", "quats", "logits", "sh"]
    picks = []
    for _ in range(64):
        name = names[rng.integers(len(names))]
        row = int(rng.integers(len(prob.used)))
        comp = int(rng.integers(int(np.prod(np.asarray(p[name]).shape[1:])) if np.asarray(p[name]).ndim > 1 else 1))
        picks.append((name, row, comp))
    fd = G.finite_difference(prob, p, picks)
    ad = np.array([grads[n].reshape(len(prob.used), -1)[r, c] for n, r, c in picks])
    scale = max(np.abs(ad).max(), 1e-12)
    # Central differences at h = 1e-4 carry an O(h^2) truncation error: a few
    # 1e-6 of the largest gradient here (it falls to ~1e-8 at h = 1e-5).
    assert np.all(np.abs(fd - ad) <= 2e-5 * np.abs(ad) + 2e-5 * scale), np.abs(fd - ad).max() / scale
