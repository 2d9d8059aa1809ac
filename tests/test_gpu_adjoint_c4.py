"""The adjoint at the differentiation configuration: 256 x 256 Mandelbulb and
Mandelbox depth-plus-Lambert renders, each of the six parameters (power,
Mandelbox scale, min radius squared, camera x, y, z, yaw), over seeded
parameter draws (MBR_C4_DRAWS, default 64 per formula).

For every draw theta the target is the render at theta perturbed by 1 %,
and the loss is L = sum_M (t - t*)^2 + (s - s*)^2 over a fixed pixel mask M.
The forward render is the FP32 march with FP64 root refinement
(MBR_ENGINE_PLAIN_MIXED); the adjoint recomputes the formula iteration in
FP32 (MBR_ENGINE_PLAIN_MIXED) from the stored depth.  The reference is FP64
central differences (h = 1e-5) of the same loss: FP64 depth from the plain
FP64 engine with root refinement and FP64 Lambert terms from FP64 distance
estimates at the six normal samples.  Bar: the FP32 adjoint within 1e-3 of
the differences, relative to the largest gradient of the draw.  The mask
keeps the pixels where every render of the draw hits, the depth is a root of
dist - threshold, both terms are smooth in every parameter (second
differences at the rounding level) and the surface faces the light; a draw
must keep at least 256 such pixels.

Against the oracle's forward-mode dual numbers (the reference iteration in
FP64 dual arithmetic) the FP64 adjoint agrees to 1e-6 on the first draws.
The torch.autograd.Function wrapper (tests/autograd_render.py) passes a
gradcheck of the masked loss against central differences, with backward
reentrant to the bit (the adjoint sums its per-block partials in block
order).
"""
import os

import numpy as np
import pytest
import torch

from mandelbulber2_b200 import abi, configs

from .adjoint_check import PARAMS, copy, get, put
from .autograd_render import fp64_depth_shade

pytestmark = pytest.mark.gpu
N_DRAWS = int(os.environ.get("MBR_C4_DRAWS", "64"))
H = 1e-5
SIZE = 256


def draw(kind, k, rng):
    sc, cam, p = configs.adjoint_256(kind, SIZE, SIZE)
    p.shading_enable = 1
    for j in PARAMS[kind]:
        v = get(sc, cam, j)
        if j in (abi.GRAD_CAMERA_X, abi.GRAD_CAMERA_Y, abi.GRAD_CAMERA_Z):
            put(sc, cam, j, v + rng.uniform(-0.1, 0.1))
        elif j == abi.GRAD_YAW:
            put(sc, cam, j, v + rng.uniform(-0.05, 0.05))
        else:
            put(sc, cam, j, v * (1.0 + rng.uniform(-0.03, 0.03)))
    return sc, cam, p


def perturb(sc, cam, kind, rel=0.01):
    s2, c2 = copy(sc, cam)
    for j in PARAMS[kind]:
        v = get(s2, c2, j)
        put(s2, c2, j, v * (1.0 + rel) if v != 0.0 else rel)
    return s2, c2


def check_draw(renderer, kind, sc, cam, p, light):
    ts, tc = perturb(sc, cam, kind)
    tt, thit, tsh, _ = fp64_depth_shade(renderer, ts, tc, p, light)
    t0, hit0, s0, root0 = fp64_depth_shade(renderer, sc, cam, p, light)
    mask = hit0 & thit & root0 & (s0 > 1e-3) & (tsh > 0.0)
    plus, minus = {}, {}
    for j in PARAMS[kind]:
        v = get(sc, cam, j)
        for sign, store in ((1.0, plus), (-1.0, minus)):
            s2, c2 = copy(sc, cam)
            put(s2, c2, j, v + sign * H)
            store[j] = fp64_depth_shade(renderer, s2, c2, p, light)
            mask &= store[j][1] & (store[j][2] > 0.0)
        d2t = np.abs(plus[j][0] - 2.0 * t0 + minus[j][0])
        d2s = np.abs(plus[j][2] - 2.0 * s0 + minus[j][2])
        mask &= (d2t <= 1e-9 * np.maximum(t0, 1.0)) & (d2s <= 1e-7)

    def loss(t, s):
        return float(np.sum(np.where(mask, (t - tt) ** 2 + (s - tsh) ** 2, 0.0)))

    fd = np.array([(loss(plus[j][0], plus[j][2]) - loss(minus[j][0], minus[j][2])) / (2 * H) for j in PARAMS[kind]])
    # FP32 forward (FP64 root refinement) -> FP32 adjoint
    renderer.set_scene(sc)
    fr = renderer.render(cam, p, abi.ENGINE_PLAIN_MIXED, outputs=("depth", "hit"))
    dev = renderer.device
    wt = torch.from_numpy(np.where(mask, 2.0 * (t0 - tt), 0.0).astype(np.float32)).to(dev)
    ws = torch.from_numpy(np.where(mask, 2.0 * (s0 - tsh), 0.0).astype(np.float32)).to(dev)
    g32 = renderer.adjoint(cam, p, fr["depth"], fr["hit"], wt, ws, abi.ENGINE_PLAIN_MIXED).cpu().numpy()
    g64 = renderer.adjoint(cam, p, fr["depth"], fr["hit"], wt, ws, abi.ENGINE_PLAIN_FP64).cpu().numpy()
    return mask, fd, np.array([g32[j] for j in PARAMS[kind]]), np.array([g64[j] for j in PARAMS[kind]]), \
        (t0, hit0, wt, ws)


@pytest.mark.parametrize("kind", ["mandelbulb", "mandelbox"])
def test_adjoint_c4_draws(renderer, oracle, kind):
    rng = np.random.default_rng(4 if kind == "mandelbulb" else 5)
    worst32, worst64, n_pix = 0.0, 0.0, []
    for k in range(N_DRAWS):
        sc, cam, p = draw(kind, k, rng)
        light = np.asarray(p.light_direction[:]) / np.linalg.norm(p.light_direction[:])
        mask, fd, g32, g64, extra = check_draw(renderer, kind, sc, cam, p, light)
        n_pix.append(int(mask.sum()))
        assert mask.sum() >= 256, (kind, k, int(mask.sum()))
        scale = np.max(np.abs(fd))
        e32 = np.max(np.abs(g32 - fd)) / scale
        e64 = np.max(np.abs(g64 - fd)) / scale
        worst32, worst64 = max(worst32, e32), max(worst64, e64)
        if k == 0:  # the dual-number reference of the oracle on the first draw
            t0, hit0, wt, ws = extra
            dt, ds, _ = oracle.pixel_gradients(sc, cam, p, t0, hit0.astype(np.uint8))
            gref = (wt.cpu().numpy().astype(np.float64)[:, None] * dt).sum(0) + \
                   (ws.cpu().numpy().astype(np.float64)[:, None] * ds).sum(0)
            gref = np.array([gref[j] for j in PARAMS[kind]])
            print(kind, "dual", gref, "adjoint64", g64)
            assert np.max(np.abs(g64 - gref)) <= 1e-6 * np.max(np.abs(gref)), (g64, gref)
        print(kind, k, "pixels", int(mask.sum()), "fd", fd, "rel err fp32", e32, "fp64", e64)
        assert e32 <= 1e-3, (kind, k, fd, g32)
        assert e64 <= 1e-3, (kind, k, fd, g64)
    print(kind, N_DRAWS, "draws: worst relative error fp32", worst32, "fp64", worst64, "mask pixels min/median",
          min(n_pix), int(np.median(n_pix)))


def test_autograd_function_gradcheck(renderer):
    """torch.autograd.gradcheck of the masked C4 loss through the
    DepthShade function (FP64 forward, FP64 adjoint) against central
    differences of the same function."""
    from .autograd_render import RenderSetup, masked_l2

    sc, cam, p = configs.adjoint_256("mandelbox", 64, 64)
    p.shading_enable = 1
    setup = RenderSetup(renderer, "mandelbox", sc, cam, p, abi.ENGINE_PLAIN_FP64, abi.ENGINE_PLAIN_FP64)
    theta0 = torch.tensor([get(sc, cam, j) for j in PARAMS["mandelbox"]], dtype=torch.float64)
    light = np.asarray(p.light_direction[:]) / np.linalg.norm(p.light_direction[:])
    ts, tc = perturb(sc, cam, "mandelbox")
    tt, thit, tsh, _ = fp64_depth_shade(renderer, ts, tc, p, light)
    # the mask: smooth pixels of the FP64 check at theta0
    mask, fd, _, _, _ = check_draw(renderer, "mandelbox", sc, cam, p, light)
    assert mask.sum() > 100
    t_star = torch.from_numpy(tt).to(renderer.device)
    s_star = torch.from_numpy(tsh).to(renderer.device)
    m = torch.from_numpy(mask).to(renderer.device)

    def f(theta):
        return masked_l2(theta, setup, m, t_star, s_star)

    theta = theta0.clone().requires_grad_(True)
    loss = f(theta)
    loss.backward()
    assert torch.isfinite(theta.grad).all() and loss.item() > 0.0
    # gradcheck compares the backward (the adjoint) with central differences
    # of the forward (FP64 depth and FP64 Lambert terms), component by
    # component within rtol 1e-3 plus an atol of 1e-4 of the largest gradient
    # (the C4 bar is relative to the largest gradient; the smallest
    # components, 1e-4 of it, carry the differences' own noise)
    atol = 1e-4 * float(np.max(np.abs(fd)))
    assert torch.autograd.gradcheck(f, (theta0.clone().requires_grad_(True),), eps=1e-5, atol=atol, rtol=1e-3,
                                    raise_exception=True)
