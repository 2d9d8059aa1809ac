"""torch.autograd.Function around the library's forward render and adjoint
(test harness only; the library itself exposes only the C-ABI).

`DepthShade.apply(theta, setup)` renders the depth of every pixel for the
parameter vector theta (float64, the differentiated parameters of
adjoint_check.PARAMS[kind], in that order), with its Lambert term from FP64
distance estimates at the six normal samples, and, in backward,
returns dL/dtheta from mbr_adjoint: the implicit-function derivative of the
hit depth and the derivative of the Lambert term through the six normal
samples, with the formula iteration recomputed in the backward pass.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from mandelbulber2_b200 import abi
from mandelbulber2_b200.render import camera_rotation

from .adjoint_check import PARAMS, copy, put


def view_dirs(cam):
    """Unit view direction of every pixel (CalculateViewVector, three-point,
    then the camera rotation), as the kernels compute it."""
    m, _ = camera_rotation(cam)
    M = np.array(m).reshape(3, 3)
    W, Hh = cam.width, cam.height
    x = np.arange(W, dtype=np.float64)
    y = np.arange(Hh, dtype=np.float64)
    fov = 2.0 * math.tan(cam.fov_deg / 360.0 * math.pi)
    ix = ((1.0 / W) * x[None, :] + -0.5) * (W / Hh)
    iy = (-1.0 / Hh) * y[:, None] + 0.5
    v = np.stack([np.broadcast_to(ix * fov, (Hh, W)), np.ones((Hh, W)), np.broadcast_to(iy * fov, (Hh, W))], -1)
    v = v.reshape(-1, 3)
    v = v / np.linalg.norm(v, axis=1, keepdims=True)
    w = v @ M.T
    return w / np.linalg.norm(w, axis=1, keepdims=True)


def lambert_fp64(r, sc, cam, p, t, hit, light):
    """FP64 Lambert term max(N.L, 0) of the hit pixels, N from FP64 distance
    estimates at the six central-difference samples of CalculateNormals
    (delta = threshold * smoothness), and the root test |dist - thr| <= 1e-6
    thr at the depth."""
    s = np.zeros_like(t)
    root = np.zeros_like(hit)
    idx = np.nonzero(hit)[0]
    if len(idx) == 0:
        return s, root
    r.set_scene(sc)
    cpos = np.array(cam.camera[:])
    pts = cpos[None, :] + view_dirs(cam)[idx] * t[idx, None]
    fov = 2.0 * math.tan(cam.fov_deg / 360.0 * math.pi)
    thr = np.linalg.norm(pts - cpos[None, :], axis=1) * (1.0 / cam.height) * fov / p.detail_level
    d0, _ = r.distance(torch.from_numpy(pts), 0.0, False, abi.ENGINE_PLAIN_FP64)
    root[idx] = np.abs(d0.cpu().numpy() - thr) <= 1e-6 * thr
    delta = thr * p.smoothness
    vals = []
    for a in range(3):
        e = np.zeros(3)
        e[a] = 1.0
        for q in (pts + delta[:, None] * e, pts - delta[:, None] * e):
            dv, _ = r.distance(torch.from_numpy(np.ascontiguousarray(q)), 0.0, True, abi.ENGINE_PLAIN_FP64)
            vals.append(dv.cpu().numpy())
    g = np.stack([vals[0] - vals[1], vals[2] - vals[3], vals[4] - vals[5]], 1)
    n = g / np.linalg.norm(g, axis=1, keepdims=True)
    s[idx] = np.maximum(n @ np.asarray(light), 0.0)
    return s, root


def fp64_depth_shade(r, sc, cam, p, light):
    """FP64 depth (plain FP64 engine, root refinement), hit, FP64 Lambert
    term and the root test of every pixel."""
    r.set_scene(sc)
    fr = r.render(cam, p, abi.ENGINE_PLAIN_FP64, outputs=("depth", "hit"))
    t = fr["depth"].cpu().numpy()
    hit = fr["hit"].cpu().numpy().astype(bool)
    s, root = lambert_fp64(r, sc, cam, p, t, hit, light)
    return t, hit, s, root


@dataclass
class RenderSetup:
    renderer: object      # mandelbulber2_b200.render.Renderer
    kind: str             # "mandelbulb" or "mandelbox"
    scene: abi.Scene
    camera: abi.Camera
    params: abi.RenderParams
    forward_engine: int = abi.ENGINE_PLAIN_MIXED   # FP32 march, FP64 root refinement
    adjoint_engine: int = abi.ENGINE_PLAIN_MIXED   # FP32 recomputation of the iteration


def scene_at(setup: RenderSetup, theta: torch.Tensor):
    sc, cam = copy(setup.scene, setup.camera)
    for k, v in zip(PARAMS[setup.kind], theta.detach().cpu().tolist()):
        put(sc, cam, k, float(v))
    return sc, cam


class DepthShade(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta: torch.Tensor, setup: RenderSetup):
        sc, cam = scene_at(setup, theta)
        r = setup.renderer
        r.set_scene(sc)
        fr = r.render(cam, setup.params, setup.forward_engine, outputs=("depth", "hit"))
        depth, hit = fr["depth"], fr["hit"]
        ctx.setup = setup
        ctx.scene_cam = (sc, cam)
        ctx.save_for_backward(depth, hit)
        p = setup.params
        light = np.asarray(p.light_direction[:]) / np.linalg.norm(p.light_direction[:])
        s, _ = lambert_fp64(r, sc, cam, p, depth.cpu().numpy(), hit.cpu().numpy().astype(bool), light)
        shade = torch.from_numpy(s).to(depth.device)
        ctx.mark_non_differentiable(hit)
        return depth.clone(), shade, hit

    @staticmethod
    def backward(ctx, g_depth, g_shade, g_hit):
        depth, hit = ctx.saved_tensors
        setup = ctx.setup
        sc, cam = ctx.scene_cam
        r = setup.renderer
        r.set_scene(sc)
        hitb = hit.to(torch.bool)
        gd = torch.where(hitb, g_depth, torch.zeros_like(g_depth)).to(torch.float32).contiguous()
        gs = torch.where(hitb, g_shade, torch.zeros_like(g_shade)).to(torch.float32).contiguous()
        grad = r.adjoint(cam, setup.params, depth.contiguous(), hit.contiguous(), gd, gs, setup.adjoint_engine)
        out = torch.tensor([float(grad[k]) for k in PARAMS[setup.kind]], dtype=torch.float64)
        return out, None


def masked_l2(theta: torch.Tensor, setup: RenderSetup, mask: torch.Tensor, t_star: torch.Tensor,
              s_star: torch.Tensor) -> torch.Tensor:
    """The C4 loss over a fixed pixel mask: sum (t - t*)^2 + (s - s*)^2."""
    t, s, _ = DepthShade.apply(theta, setup)
    m = mask.to(t.device)
    return (torch.where(m, (t - t_star) ** 2 + (s - s_star) ** 2, torch.zeros_like(t))).sum()
