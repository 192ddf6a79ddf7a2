"""The differentiable rasteriser: a torch.autograd.Function over the C-ABI's
training entry points (``lrt_rast_train_forward`` / ``lrt_rast_train_backward``).

Parameters (one cloud, world space): means [N,3], log_scales [N,3],
quats [N,4] as (w, x, y, z) (normalised in the forward), opacity_logits [N],
sh [N,16,3] (DC first). The SH coefficients are kept in fp32 by the caller
and read by the kernels as fp16; their gradient is fp32. The colour image
[H,W,4] is differentiable; depth is not.

``sort_values=True`` makes the pair sort carry each pair's emit index as a
value (``LRT_TRAIN_SORT_VALUES``) instead of in the pair word's low field;
images and gradients are the same either way.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _abi
from .camera import Camera, Projection, projection_for
from .raster import FrameStats, RenderSettings, TileRasterizer, _stream_ptr


class _Rasterize(torch.autograd.Function):
    @staticmethod
    def forward(ctx, means, log_scales, quats, opacity_logits, sh, raster: TileRasterizer, projection: Projection,
                settings: RenderSettings, sort_values: bool, grad_bucket, sh_storage):
        dev = means.device
        n = means.shape[0]
        means = means.contiguous().float()
        log_scales = log_scales.contiguous().float()
        quats = quats.contiguous().float()
        opacity_logits = opacity_logits.contiguous().float()
        if sh_storage is not None:
            # The caller's fp16 working copy of `sh` (kept in step with it by
            # the optimizer): read as it is, no conversion this step.
            if (sh_storage.dtype != torch.float16 or sh_storage.numel() != n * 48 or
                    not sh_storage.is_contiguous() or sh_storage.data_ptr() % 16 != 0 or
                    sh_storage.device != sh.device):
                raise ValueError("sh_storage must be a contiguous, 16-byte aligned fp16 tensor of N x 48 "
                                 "coefficients on the parameters' device")
            shk = sh_storage.detach().reshape(n, 48)
        else:
            shk = sh.detach().reshape(n, 48).to(torch.float16).contiguous()
        colour = torch.empty((settings.height, settings.width, 4), dtype=torch.float32, device=dev)
        depth = torch.empty((settings.height, settings.width), dtype=torch.float32, device=dev)
        p = _abi.TrainParams()
        p.count = n
        p.flags = _abi.TRAIN_SORT_VALUES if sort_values else 0
        p.means, p.log_scales, p.quats = means.data_ptr(), log_scales.data_ptr(), quats.data_ptr()
        p.opacity_logits, p.sh = opacity_logits.data_ptr(), shk.data_ptr()
        t = _abi.TargetsStruct()
        t.width, t.height, t.colour, t.depth = settings.width, settings.height, colour.data_ptr(), depth.data_ptr()
        pr = projection.struct()
        st = settings.struct()
        stats = _abi.FrameStatsStruct()
        raster._check(_abi.load().lrt_rast_train_forward(raster._handle, C.byref(pr), C.byref(p), C.byref(st),
                                                         C.byref(t), C.byref(stats), _stream_ptr(None)))
        ctx.raster = raster
        ctx.grad_bucket = grad_bucket
        ctx.shapes = [t.shape for t in (means, log_scales, quats, opacity_logits, sh)]
        raster.last_train_stats = FrameStats.from_struct(stats)
        # The handle keeps pointers to these until the backward.
        ctx.save_for_backward(means, log_scales, quats, opacity_logits, shk)
        ctx.mark_non_differentiable(depth)
        ctx.set_materialize_grads(False)   # no zero image for the depth's gradient
        return colour, depth

    @staticmethod
    def backward(ctx, grad_colour, grad_depth):
        means, log_scales, quats, opacity_logits, _ = ctx.saved_tensors
        if grad_colour is None:
            return None, None, None, None, None, None, None, None, None, None, None
        n = means.shape[0]
        bucket = ctx.grad_bucket
        if bucket is not None and bucket.count == n:
            # Fresh views of the bucket (no other reference), so autograd keeps
            # them as the parameters' .grad rather than copying.
            g = [bucket.slice(name).view(shape) for name, shape in zip(bucket.ORDER, ctx.shapes)]
        else:
            g = [torch.empty_like(means), torch.empty_like(log_scales), torch.empty_like(quats),
                 torch.empty_like(opacity_logits), torch.empty((n, 16, 3), dtype=torch.float32, device=means.device)]
        grads = _abi.TrainGrads()
        grads.means, grads.log_scales, grads.quats = g[0].data_ptr(), g[1].data_ptr(), g[2].data_ptr()
        grads.opacity_logits, grads.sh = g[3].data_ptr(), g[4].data_ptr()
        gc = grad_colour.contiguous().float()
        raster = ctx.raster
        raster._check(_abi.load().lrt_rast_train_backward(raster._handle, gc.data_ptr(), C.byref(grads),
                                                          _stream_ptr(None)))
        return g[0], g[1], g[2], g[3], g[4], None, None, None, None, None, None


class _L1Loss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, colour, target, raster: TileRasterizer):
        colour = colour.contiguous().float()
        target = target.contiguous().float()
        if colour.shape[:-1] != target.shape[:-1] or colour.shape[-1] != 4 or target.shape[-1] != 3:
            raise ValueError("colour must be [..., 4] and target [..., 3] over the same pixels")
        pixels = colour.numel() // 4
        loss = torch.empty((), dtype=torch.float32, device=colour.device)
        raster._check(_abi.load().lrt_rast_l1_loss(raster._handle, colour.data_ptr(), target.data_ptr(), pixels,
                                                   loss.data_ptr(), _stream_ptr(None)))
        ctx.save_for_backward(colour, target)
        return loss

    @staticmethod
    def backward(ctx, grad_loss):
        colour, target = ctx.saved_tensors
        grad_loss = grad_loss.contiguous().float()
        grad = torch.empty_like(colour)
        code = _abi.load().lrt_l1_loss_grad(colour.data_ptr(), target.data_ptr(), colour.numel() // 4,
                                            grad_loss.data_ptr(), grad.data_ptr(), _stream_ptr(None))
        _abi.check(code, "l1_loss backward")
        return grad, None, None


def l1_loss(colour: torch.Tensor, target: torch.Tensor, raster: TileRasterizer) -> torch.Tensor:
    """mean |colour.rgb - target| (colour [..., 4] from rasterize, target
    [..., 3]), one kernel each way, summed in a fixed order."""
    return _L1Loss.apply(colour, target, raster)


def rasterize(means, log_scales, quats, opacity_logits, sh, view: Camera | Projection, settings: RenderSettings,
              raster: TileRasterizer, sort_values: bool = False, grad_bucket=None, sh_storage=None):
    """Render the differentiable cloud; returns (colour [H,W,4], depth [H,W]).
    The kernels read the SH coefficients as fp16 (the gradient with respect to
    `sh` is fp32): by default `sh` is converted every call; `sh_storage`, an
    fp16 copy of `sh` the caller keeps in step with it (a mixed-precision
    optimizer writes both), is read as it is instead.
    `grad_bucket` (a replicas.GradientBucket for this cloud): the backward
    writes every gradient into it, ready for one all-reduce over ranks."""
    projection = view if isinstance(view, Projection) else projection_for(view, settings.width, settings.height)
    return _Rasterize.apply(means, log_scales, quats, opacity_logits, sh, raster, projection, settings, sort_values,
                            grad_bucket, sh_storage)


def backward_times(raster: TileRasterizer) -> tuple[float, float]:
    a, b = C.c_double(), C.c_double()
    raster._check(_abi.load().lrt_rast_backward_times(raster._handle, C.byref(a), C.byref(b)))
    return a.value, b.value


def train_batch(means, log_scales, quats, opacity_logits, sh, views, settings: RenderSettings, raster: TileRasterizer,
                sh_storage=None, grad_bucket=None, stream=None):
    """One training step over many views in one call (lrt_rast_train_batch):
    each view rendered as `rasterize` renders it, its L1 loss against its
    target taken as `l1_loss` takes it, and the gradients of the sum of the
    views' losses accumulated view by view, in the given order.

    views: a sequence of (Camera | Projection, target [H, W, 3] float32 on the
    device); each view's size is its target's. The settings' size is ignored.
    sh_storage: as for `rasterize` (the fp16 copy the kernels read; made here
    when not given). grad_bucket: a replicas.GradientBucket to write the
    gradients into (else new tensors).

    Returns (colours [list of [H, W, 4]], depths [list of [H, W]], losses [V]
    tensor, grads: dict of means, log_scales, quats, opacity_logits, sh, each
    shaped like its parameter) and the batch's stats (BatchStats).
    """
    dev = means.device
    n = means.shape[0]
    means = means.detach().contiguous().float()
    log_scales = log_scales.detach().contiguous().float()
    quats = quats.detach().contiguous().float()
    opacity_logits = opacity_logits.detach().contiguous().float()
    if sh_storage is None:
        sh_storage = sh.detach().reshape(n, 48).to(torch.float16).contiguous()
    elif sh_storage.dtype != torch.float16 or sh_storage.numel() != n * 48 or not sh_storage.is_contiguous():
        raise ValueError("sh_storage must be a contiguous fp16 tensor of N x 48 coefficients")
    p = _abi.TrainParams()
    p.count = n
    p.means, p.log_scales, p.quats = means.data_ptr(), log_scales.data_ptr(), quats.data_ptr()
    p.opacity_logits, p.sh = opacity_logits.data_ptr(), sh_storage.data_ptr()
    colours, depths, targets = [], [], []
    losses = torch.zeros(len(views), dtype=torch.float32, device=dev)
    arr = (_abi.TrainViewStruct * max(1, len(views)))()
    for k, (view, target) in enumerate(views):
        h, w = int(target.shape[0]), int(target.shape[1])
        if target.shape[-1] != 3:
            raise ValueError("a view's target must be [H, W, 3]")
        target = target.contiguous().float()
        targets.append(target)
        pr = view if isinstance(view, Projection) else projection_for(view, w, h)
        colour = torch.empty((h, w, 4), dtype=torch.float32, device=dev)
        depth = torch.empty((h, w), dtype=torch.float32, device=dev)
        colours.append(colour)
        depths.append(depth)
        arr[k].projection = pr.struct()
        arr[k].width, arr[k].height = w, h
        arr[k].colour, arr[k].depth, arr[k].target = colour.data_ptr(), depth.data_ptr(), target.data_ptr()
        arr[k].loss = losses.data_ptr() + 4 * k
    shapes = {"means": means.shape, "log_scales": log_scales.shape, "quats": quats.shape,
              "opacity_logits": opacity_logits.shape, "sh": sh.shape}
    if grad_bucket is not None and grad_bucket.count == n:
        grads = {k: grad_bucket.slice(k).view(shapes[k]) for k in grad_bucket.ORDER}
    else:
        grads = {k: torch.empty(shapes[k], dtype=torch.float32, device=dev) for k in shapes}
    g = _abi.TrainGrads()
    g.means, g.log_scales, g.quats = grads["means"].data_ptr(), grads["log_scales"].data_ptr(), grads["quats"].data_ptr()
    g.opacity_logits, g.sh = grads["opacity_logits"].data_ptr(), grads["sh"].data_ptr()
    st = settings.struct()
    stats = _abi.BatchStats()
    raster._check(_abi.load().lrt_rast_train_batch(raster._handle, C.byref(p), arr, len(views), C.byref(st),
                                                   C.byref(g), C.byref(stats), _stream_ptr(stream)))
    return colours, depths, losses, grads, stats
