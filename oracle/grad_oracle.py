"""ORACLE -- test infrastructure, not product code.

FP64 gradient oracle for the training path. It is a brute-force per-pixel
evaluation of the rasteriser's forward in float64 (torch autograd on the CPU)
over a crop of the image. The discrete choices of the frame are held fixed:
which splats reach each pixel, in which order, and where the pixel stops.
They come from the fp32 oracle (`oracle.train_render`), which makes them
exactly as the kernels do. Over those choices the image is a smooth function
of the parameters, except at the clamps (alpha <= 0.99, colour >= 0, the
Jacobian's frustum clamp, the 2D filter's max(det, 0)). This module gives
its FP64 gradient by autograd and by central finite differences.

Forward restated from shaders/lrt/splat/splat_project.slang:72-169 and
splat_blend.slang:50-107, in the training parameterisation: scale =
exp(log-scale), opacity = sigmoid(logit), quaternion (w, x, y, z) normalised,
base colour 0.5 + SH0 * DC, SH read at the fp16 values the kernels read.
Loss: L1 of the linearised rgb against a target over the crop,
mean over pixels and channels.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

SH0 = 0.28209479177387814
C1 = 0.4886025119029199
C2 = [1.0925484305920792, -1.0925484305920792, 0.31539156525252005, -1.0925484305920792, 0.5462742152960396]
C3 = [-0.5900435899266435, 2.890611442640554, -0.4570457994644658, 0.3731763325901154, -0.4570457994644658,
      1.445305721320277, -0.5900435899266435]


@dataclass
class Camera64:
    """The per-frame constants, as the kernels hold them (fp32 values)."""
    W: torch.Tensor      # [3, 4] object -> view
    eye: torch.Tensor    # [3]
    fx: float
    fy: float
    cx: float
    cy: float
    width: int
    height: int
    ortho: bool
    antialias: bool
    sh_limit: int
    linearise: bool
    bg: torch.Tensor     # [4]


def camera_from(projection, settings) -> Camera64:
    m = np.asarray(projection.world_to_view[:], np.float64).reshape(4, 4)
    f32 = lambda v: float(np.float32(v))  # noqa: E731
    W = torch.tensor(m[:3, :4].astype(np.float32).astype(np.float64))
    eye = torch.tensor(np.asarray(projection.eye_world[:], np.float64).astype(np.float32).astype(np.float64))
    return Camera64(W, eye, f32(projection.focal_x), f32(projection.focal_y), f32(projection.centre_x),
                    f32(projection.centre_y), settings.width, settings.height, bool(projection.orthographic),
                    bool(settings.antialias), int(settings.max_sh_degree), bool(settings.linearise),
                    torch.tensor(np.asarray(settings.background[:], np.float32).astype(np.float64)))


def sh_rest(dirs: torch.Tensor, coeffs: torch.Tensor, degree: int) -> torch.Tensor:
    """sh.slang:25-51: the view-dependent part; coeffs [M, 15, 3]."""
    x, y, z = dirs[:, 0:1], dirs[:, 1:2], dirs[:, 2:3]
    out = torch.zeros(dirs.shape[0], 3, dtype=dirs.dtype)
    if degree == 0:
        return out
    b = [-C1 * y, C1 * z, -C1 * x]
    if degree >= 2:
        xx, yy, zz = x * x, y * y, z * z
        b += [C2[0] * x * y, C2[1] * y * z, C2[2] * (2 * zz - xx - yy), C2[3] * x * z, C2[4] * (xx - yy)]
    if degree >= 3:
        b += [C3[0] * y * (3 * xx - yy), C3[1] * x * y * z, C3[2] * y * (4 * zz - xx - yy),
              C3[3] * z * (2 * zz - 3 * xx - 3 * yy), C3[4] * x * (4 * zz - xx - yy), C3[5] * z * (xx - yy),
              C3[6] * x * (xx - 3 * yy)]
    for k, bk in enumerate(b):
        out = out + bk * coeffs[:, k, :]
    return out


def project(cam: Camera64, means, log_scales, quats, logits, sh):
    """Per splat: centre [M,2], conic [M,3], alpha0 [M], colour [M,3] (float64)."""
    t = means @ cam.W[:, :3].T + cam.W[:, 3]
    q = quats / torch.linalg.norm(quats, dim=1, keepdim=True)
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    R = torch.stack([
        torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
        torch.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
        torch.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1)], 1)
    M = R * torch.exp(log_scales)[:, None, :]
    zeros = torch.zeros_like(t[:, 0])
    if cam.ortho:
        centre = torch.stack([cam.fx * t[:, 0] + cam.cx, cam.fy * t[:, 1] + cam.cy], -1)
        jx = torch.stack([zeros + cam.fx, zeros, zeros], -1)
        jy = torch.stack([zeros, zeros + cam.fy, zeros], -1)
    else:
        iz = 1.0 / t[:, 2]
        centre = torch.stack([cam.fx * t[:, 0] * iz + cam.cx, cam.fy * t[:, 1] * iz + cam.cy], -1)
        lox = (-0.15 * cam.width - cam.cx) / cam.fx
        hix = (1.15 * cam.width - cam.cx) / cam.fx
        loy = (-0.15 * cam.height - cam.cy) / cam.fy
        hiy = (1.15 * cam.height - cam.cy) / cam.fy
        tx = torch.clamp(t[:, 0] * iz, lox, hix) * t[:, 2]
        ty = torch.clamp(t[:, 1] * iz, loy, hiy) * t[:, 2]
        jx = torch.stack([cam.fx * iz, zeros, -cam.fx * tx * iz * iz], -1)
        jy = torch.stack([zeros, cam.fy * iz, -cam.fy * ty * iz * iz], -1)
    Wl = cam.W[:, :3]
    T2x = jx @ Wl
    T2y = jy @ Wl
    ax = torch.einsum("mi,mij->mj", T2x, M)
    ay = torch.einsum("mi,mij->mj", T2y, M)
    a0 = (ax * ax).sum(-1)
    b = (ax * ay).sum(-1)
    c0 = (ay * ay).sum(-1)
    det_before = a0 * c0 - b * b
    a = a0 + 0.3
    c = c0 + 0.3
    det = a * c - b * b
    opacity = torch.sigmoid(logits)
    alpha0 = opacity * torch.sqrt(torch.clamp(det_before, min=0.0) / det) if cam.antialias else opacity
    conic = torch.stack([c / det, -b / det, a / det], -1)
    d = means - cam.eye
    dirs = d / torch.linalg.norm(d, dim=1, keepdim=True)
    base = 0.5 + SH0 * sh[:, 0, :]
    colour = torch.clamp(base + sh_rest(dirs, sh[:, 1:, :], min(3, cam.sh_limit)), min=0.0)
    return centre, conic, alpha0, colour


def srgb_to_linear(c: torch.Tensor) -> torch.Tensor:
    c = torch.clamp(c, min=0.0)
    return torch.where(c <= 0.04045, c / 12.92, ((c + 0.055) / 1.055) ** 2.4)


class CropProblem:
    """The loss over a crop with the frame's contributor lists held fixed."""

    def __init__(self, cam: Camera64, crop, list_offsets: np.ndarray, list_slots: np.ndarray,
                 target: np.ndarray):
        self.cam = cam
        x0, y0, w, h = crop
        self.crop = crop
        counts = np.diff(list_offsets.astype(np.int64))
        self.k = int(max(1, counts.max(initial=1)))
        npix = w * h
        idx = np.zeros((npix, self.k), np.int64)
        mask = np.zeros((npix, self.k), bool)
        for p in range(npix):
            s = list_slots[list_offsets[p]:list_offsets[p + 1]]
            idx[p, :len(s)] = s
            mask[p, :len(s)] = True
        self.used = np.unique(list_slots) if len(list_slots) else np.zeros(0, np.int64)
        remap = {int(s): i for i, s in enumerate(self.used)}
        self.idx = torch.tensor(np.vectorize(lambda v: remap.get(int(v), 0))(idx) if len(self.used) else idx)
        self.mask = torch.tensor(mask)
        ys, xs = np.mgrid[y0:y0 + h, x0:x0 + w]
        self.px = torch.tensor(xs.reshape(-1) + 0.5, dtype=torch.float64)
        self.py = torch.tensor(ys.reshape(-1) + 0.5, dtype=torch.float64)
        self.target = torch.tensor(target.reshape(npix, 3), dtype=torch.float64)

    def loss(self, means, log_scales, quats, logits, sh) -> torch.Tensor:
        """Parameters of the used splats only ([M, ...], float64)."""
        centre, conic, alpha0, colour = project(self.cam, means, log_scales, quats, logits, sh)
        i = self.idx
        dx = self.px[:, None] - centre[i, 0]
        dy = self.py[:, None] - centre[i, 1]
        power = conic[i, 0] * dx * dx + 2.0 * conic[i, 1] * dx * dy + conic[i, 2] * dy * dy
        alpha = torch.clamp(alpha0[i] * torch.exp(-0.5 * power), max=0.99)
        alpha = torch.where(self.mask, alpha, torch.zeros_like(alpha))
        one_minus = 1.0 - alpha
        T_before = torch.cumprod(torch.cat([torch.ones_like(alpha[:, :1]), one_minus[:, :-1]], 1), 1)
        weight = T_before * alpha
        rgb = (weight[:, :, None] * colour[i]).sum(1)
        T = torch.prod(one_minus, 1)
        cov = 1.0 - T
        lin = torch.where((cov > 1e-6)[:, None] if self.cam.linearise else torch.zeros_like(cov, dtype=bool)[:, None],
                          srgb_to_linear(rgb / cov.clamp(min=1e-30)[:, None]) * cov[:, None], rgb)
        out = lin + T[:, None] * self.cam.bg[:3]
        return torch.abs(out - self.target).sum() / (3.0 * out.shape[0])


def gradients(problem: CropProblem, params: dict) -> dict:
    """FP64 autograd gradients w.r.t. the used splats' parameters."""
    used = problem.used
    leaves = {k: torch.tensor(np.asarray(v)[used], dtype=torch.float64, requires_grad=True) for k, v in params.items()}
    L = problem.loss(leaves["means"], leaves["log_scales"], leaves["quats"], leaves["logits"], leaves["sh"])
    L.backward()
    return {k: v.grad.numpy() for k, v in leaves.items()}, float(L.detach())


def finite_difference(problem: CropProblem, params: dict, picks, h: float = 1e-4) -> np.ndarray:
    """Central differences of the FP64 loss for (name, used-index, component) picks."""
    base = {k: torch.tensor(np.asarray(v)[problem.used], dtype=torch.float64) for k, v in params.items()}
    out = []
    with torch.no_grad():
        for name, row, comp in picks:
            vals = []
            for sgn in (1.0, -1.0):
                p = {k: v.clone() for k, v in base.items()}
                flat = p[name].view(p[name].shape[0], -1)
                flat[row, comp] += sgn * h
                vals.append(float(problem.loss(p["means"], p["log_scales"], p["quats"], p["logits"], p["sh"])))
            out.append((vals[0] - vals[1]) / (2 * h))
    return np.array(out)
