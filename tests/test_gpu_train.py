"""The differentiable path on the GPU through the C-ABI (lrt_rast_train_forward
/ lrt_rast_train_backward, wrapped in a torch.autograd.Function):

- its forward equals the oracle's restatement of the training
  parameterisation bit for bit (records, keys, ranges, image);
- its forward matches the plain forward of the same splats packed (the
  packed layout quantises rotation to 10 bits and log-scales to f16) within
  the reference's image tolerances;
- its gradients equal the FP64 brute-force per-pixel oracle over a 64x64
  crop (float64 autograd with the frame's discrete choices held fixed) and
  FP64 central finite differences (h = 1e-4) on 256 random parameters,
  within 1e-4 relative.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import lucabrtrender_b200 as L

import grad_oracle as G
import oracle as ora
import train_fixtures as TF

pytestmark = pytest.mark.gpu

REL = 1e-4   # gradient tolerance, relative to the FP64 oracle


def to_cuda(p, requires_grad=False):
    out = {}
    for k, v in p.items():
        t = torch.from_numpy(np.ascontiguousarray(v)).cuda()
        t.requires_grad_(requires_grad)
        out[k] = t
    return out


def gpu_forward(rasterizer, p, cam, settings, requires_grad=False, sort_values=False):
    t = to_cuda(p, requires_grad)
    colour, depth = L.rasterize(t["means"], t["log_scales"], t["quats"], t["logits"], t["sh"], cam, settings,
                                rasterizer, sort_values=sort_values)
    return t, colour, depth


@pytest.mark.parametrize("sort_values", [False, True], ids=["emit-low-field", "emit-sort-value"])
@pytest.mark.parametrize("n,size,seed", [(3000, 96, 5), (20000, 200, 6)])
def test_train_forward_bit_exact(rasterizer, n, size, seed, sort_values):
    p = TF.make_params(n, seed)
    cam, settings = TF.frame(size, size)
    _, colour, depth = gpu_forward(rasterizer, p, cam, settings, sort_values=sort_values)
    dbg = rasterizer.debug_arrays()
    pr = L.projection_for(cam, size, size).struct()
    ref = ora.train_render(pr, TF.raw_cloud(p), settings.struct())
    assert np.array_equal(dbg["proj"].cpu().numpy().view(np.uint32), ref["proj"].view(np.uint32))
    assert np.array_equal(dbg["depth_keys"].cpu().numpy().view(np.uint32), ref["depth_keys"])
    assert np.array_equal(dbg["ranges"].cpu().numpy().view(np.uint32), ref["ranges"])
    assert np.abs(colour.detach().cpu().numpy() - ref["colour"]).max() <= 1e-5
    assert np.abs(depth.cpu().numpy() - ref["depth"]).max() <= 1e-5


def test_train_forward_matches_the_packed_forward(rasterizer):
    p = TF.make_params(20000, 7)
    cam, settings = TF.frame(160, 160)
    _, colour, _ = gpu_forward(rasterizer, p, cam, settings)
    packed = L.pack_splats(TF.raw_records(p), 15, 3)
    targets = L.RenderTargets()
    rasterizer.render(cam, [L.SplatInstance(L.to_device(packed))], settings, targets)
    diff = ora.compare_images(colour.detach().cpu().numpy(), targets.colour.cpu().numpy())
    assert diff.p99 <= 2 and diff.max <= 16, (diff.p99, diff.max)


def _crop_problem(p, cam, settings, crop, target):
    pr = L.projection_for(cam, settings.width, settings.height).struct()
    st = settings.struct()
    out = ora.train_render(pr, TF.raw_cloud(p), st, crop)
    return G.CropProblem(G.camera_from(pr, st), crop, out["list_offsets"], out["list_slots"], target), out


def _gpu_crop_gradients(rasterizer, p, cam, settings, crop, target, sort_values=False):
    t, colour, _ = gpu_forward(rasterizer, p, cam, settings, requires_grad=True, sort_values=sort_values)
    x0, y0, w, h = crop
    tgt = torch.from_numpy(target).cuda()
    loss = torch.abs(colour[y0:y0 + h, x0:x0 + w, :3] - tgt).sum() / (3.0 * w * h)
    loss.backward()
    return {k: v.grad.detach().cpu().numpy() for k, v in t.items()}, float(loss.detach())


@pytest.mark.parametrize("sort_values", [False, True], ids=["emit-low-field", "emit-sort-value"])
def test_gradients_match_the_fp64_per_pixel_oracle_on_a_crop(rasterizer, sort_values):
    p = TF.make_params(6000, 8)
    cam, settings = TF.frame(128, 128)
    crop = (32, 32, 64, 64)
    target = np.random.default_rng(3).uniform(0, 1, (64, 64, 3))
    prob, _ = _crop_problem(p, cam, settings, crop, target)
    want, loss64 = G.gradients(prob, p)
    got, loss32 = _gpu_crop_gradients(rasterizer, p, cam, settings, crop, target, sort_values)
    assert abs(loss32 - loss64) <= 1e-5 * max(1.0, abs(loss64))
    used = prob.used
    report = {}
    for name in ("means", "log_scales", "quats", "logits", "sh"):
        g = got[name].reshape(got[name].shape[0], -1)[used].astype(np.float64)
        w = want[name].reshape(len(used), -1)
        err = np.linalg.norm(g - w) / max(np.linalg.norm(w), 1e-30)
        report[name] = err
        assert err <= REL, (name, err)
    # splats no crop pixel sees get exactly zero
    unused = np.setdiff1d(np.arange(p["means"].shape[0]), used)
    assert np.all(got["means"][unused] == 0) and np.all(got["logits"][unused] == 0)


def test_gradients_match_fp64_finite_differences(rasterizer):
    p = TF.make_params(6000, 9)
    cam, settings = TF.frame(128, 128)
    crop = (32, 32, 64, 64)
    target = np.random.default_rng(4).uniform(0, 1, (64, 64, 3))
    prob, _ = _crop_problem(p, cam, settings, crop, target)
    got, _ = _gpu_crop_gradients(rasterizer, p, cam, settings, crop, target)
    rng = np.random.default_rng(11)
    names = ["means", "log_scales", "quats", "logits", "sh"]
    picks = []
    for _ in range(256):
        name = names[rng.integers(len(names))]
        row = int(rng.integers(len(prob.used)))
        width = int(np.prod(np.asarray(p[name]).shape[1:])) if np.asarray(p[name]).ndim > 1 else 1
        picks.append((name, row, int(rng.integers(width))))
    fd = G.finite_difference(prob, p, picks, h=1e-4)
    gpu = np.array([got[n].reshape(got[n].shape[0], -1)[prob.used[r], c] for n, r, c in picks], np.float64)
    scale = np.abs(fd).max()
    err = np.abs(gpu - fd)
    # per parameter: within REL of its own value or of the largest sampled gradient
    assert np.all(err <= REL * np.abs(fd) + REL * scale), (err / scale).max()


def test_an_enqueued_frame_that_overflows_is_reported_and_the_redraw_is_exact():
    """Training frames after the first of a shape are only enqueued. One that
    emits more pairs than the buffer holds is reported as OVERFLOW when its
    counts are read (here by the debug view), with the buffers grown, and the
    same frame drawn again equals the oracle bit for bit."""
    from lucabrtrender_b200 import _abi
    raster = L.TileRasterizer.create(0)
    try:
        p = TF.make_params(3000, 12, log_scale_mean=-2.0)
        far, settings = TF.frame(96, 96, eye=(0.0, 0.0, 8.0))     # ~7.1k pairs: sizes the buffers (12k)
        near, _ = TF.frame(96, 96, eye=(0.0, 0.0, 1.2))           # ~21k pairs
        gpu_forward(raster, p, far, settings)
        gpu_forward(raster, p, far, settings)
        raster.debug_arrays()
        gpu_forward(raster, p, near, settings)
        with pytest.raises(L.LrtError) as info:
            raster.debug_arrays()
        assert info.value.code == _abi.OVERFLOW
        _, colour, _ = gpu_forward(raster, p, near, settings)
        dbg = raster.debug_arrays()
        pr = L.projection_for(near, 96, 96).struct()
        ref = ora.train_render(pr, TF.raw_cloud(p), settings.struct())
        assert np.array_equal(dbg["ranges"].cpu().numpy().view(np.uint32), ref["ranges"])
        assert np.abs(colour.detach().cpu().numpy() - ref["colour"]).max() <= 1e-5
    finally:
        raster.close()


def test_both_emit_index_layouts_give_the_same_gradients_bit_for_bit(rasterizer):
    """The emit index as the pair word's low field or as a sort value: the same
    pair order, the same partial slots, so the same sums in the same order."""
    p = TF.make_params(20000, 13)
    cam, settings = TF.frame(200, 200)
    crop = (0, 0, 200, 200)
    target = np.random.default_rng(5).uniform(0, 1, (200, 200, 3))
    a, la = _gpu_crop_gradients(rasterizer, p, cam, settings, crop, target, sort_values=False)
    b, lb = _gpu_crop_gradients(rasterizer, p, cam, settings, crop, target, sort_values=True)
    assert la == lb
    for name in a:
        assert np.array_equal(a[name].view(np.uint32), b[name].view(np.uint32)), name


def test_the_l1_loss_equals_torch_and_its_gradient_is_the_same(rasterizer):
    gen = torch.Generator(device="cuda").manual_seed(3)
    colour = torch.rand((181, 243, 4), generator=gen, device="cuda", requires_grad=True)
    target = torch.rand((181, 243, 3), generator=gen, device="cuda")
    loss = L.l1_loss(colour, target, rasterizer)
    (2.5 * loss).backward()
    ours = colour.grad.clone()
    colour.grad = None
    want = torch.abs(colour[..., :3] - target).mean()
    (2.5 * want).backward()
    assert abs(float(loss.detach()) - float(want.detach().double())) <= 2e-6 * float(want.detach())
    assert torch.equal(ours, colour.grad)


def test_gradients_written_into_a_bucket_are_the_same_and_stay_there(rasterizer):
    """rasterize(..., grad_bucket=): the backward writes every gradient into one
    flat buffer (ready for a single all-reduce over ranks); the gradients equal
    the unbucketed ones bit for bit and autograd keeps them in the bucket."""
    from lucabrtrender_b200.replicas import GradientBucket
    p = TF.make_params(20001, 17)   # an odd count: the SH gradient still starts aligned
    cam, settings = TF.frame(200, 200)
    target = torch.from_numpy(np.random.default_rng(17).uniform(0, 1, (200, 200, 3)).astype(np.float32)).cuda()
    names = ("means", "log_scales", "quats", "logits", "sh")
    out = []
    for bucket in (None, GradientBucket(20001, torch.device("cuda"))):
        for _ in range(2):   # a second step rewrites the same bucket
            t = to_cuda(p, requires_grad=True)
            colour, _ = L.rasterize(t["means"], t["log_scales"], t["quats"], t["logits"], t["sh"], cam, settings,
                                    rasterizer, grad_bucket=bucket)
            L.l1_loss(colour, target, rasterizer).backward()
            if bucket is not None:
                assert bucket.holds([t[k].grad for k in names])
                bucket.all_reduce([t[k] for k in names])   # one rank: nothing to sum
        out.append({k: t[k].grad.detach().cpu().numpy().copy() for k in names})
    for k in names:
        assert np.array_equal(out[0][k].view(np.uint32), out[1][k].view(np.uint32)), k


def test_an_fp16_working_copy_of_the_coefficients_gives_the_same_step(rasterizer):
    """rasterize(..., sh_storage=): the kernels read the caller's fp16 copy of
    the coefficients instead of converting `sh` each call; image, loss and
    gradients (the SH one still with respect to the fp32 `sh`) are the same
    bit for bit. A copy of the wrong type is refused."""
    p = TF.make_params(20000, 23)
    p["sh"] = np.random.default_rng(23).normal(0.0, 0.5, p["sh"].shape).astype(np.float32)   # needs rounding
    cam, settings = TF.frame(200, 200)
    target = torch.from_numpy(np.random.default_rng(23).uniform(0, 1, (200, 200, 3)).astype(np.float32)).cuda()
    names = ("means", "log_scales", "quats", "logits", "sh")
    out = []
    for working in (False, True):
        t = to_cuda(p, requires_grad=True)
        sh16 = t["sh"].detach().reshape(-1, 48).half().contiguous() if working else None
        colour, _ = L.rasterize(t["means"], t["log_scales"], t["quats"], t["logits"], t["sh"], cam, settings,
                                rasterizer, sh_storage=sh16)
        loss = L.l1_loss(colour, target, rasterizer)
        loss.backward()
        assert t["sh"].grad.dtype == torch.float32
        out.append((colour.detach().cpu().numpy(), float(loss.detach()),
                    {k: t[k].grad.detach().cpu().numpy() for k in names}))
    (ca, la, ga), (cb, lb, gb) = out
    assert np.array_equal(ca.view(np.uint32), cb.view(np.uint32)) and la == lb
    for k in names:
        assert np.array_equal(ga[k].view(np.uint32), gb[k].view(np.uint32)), k
    t = to_cuda(p, requires_grad=True)
    with pytest.raises(ValueError):
        L.rasterize(t["means"], t["log_scales"], t["quats"], t["logits"], t["sh"], cam, settings, rasterizer,
                    sh_storage=t["sh"].detach())
